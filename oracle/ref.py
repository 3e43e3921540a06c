"""ctypes binding of the reference's own stage-2 build (oracle/_ref/, made by
oracle/build_ref.sh from the reference sources) -- TEST INFRASTRUCTURE.

Used to generate golden vectors (tests/golden/make_golden.py) and to time the
reference GPU build next to the product (bench.py).  Needs a CUDA device.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_h = None
_cabi = None


def available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_harness.so"))


def harness():
    global _h
    if _h is None:
        L = ctypes.CDLL(os.path.join(REF_DIR, "libref_harness.so"))
        L.ref_round_canonical.restype = ctypes.c_int
        L.ref_round_canonical.argtypes = [_f32p, _i32p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_float, ctypes.c_float, ctypes.c_int, _f32p, _i32p, _i32p, _i32p,
                                          _i32p, ctypes.c_int, _u32p, ctypes.c_int, _i32p, ctypes.c_int, _u8p, _i32p]
        L.ref_forward_raw.restype = ctypes.c_int
        L.ref_forward_raw.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int]
        L.ref_state.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int)]
        L.ref_self_intersect.restype = ctypes.c_int
        L.ref_self_intersect.argtypes = [_f32p, _i32p, ctypes.c_int, ctypes.c_int, _u8p]
        L.ref_copy_state.restype = ctypes.c_int
        L.ref_copy_state.argtypes = [ctypes.c_void_p] * 5
        L.ref_pow2.restype = ctypes.c_int
        L.ref_pow2.argtypes = [_f32p, _f32p, ctypes.c_int]
        _h = L
    return _h


def cabi():
    global _cabi
    if _cabi is None:
        L = ctypes.CDLL(os.path.join(REF_DIR, "libpamo_ref_cabi.so"))
        L.pamo_simplify.restype = None
        L.pamo_simplify.argtypes = [_f32p, _i32p, _f32p, _i32p, _i32p, ctypes.c_float]
        _cabi = L
    return _cabi


def round_canonical(P, T, undo, scale, threshold, is_stuck):
    """One reference round with canonical adjacency order (see ref_harness.cu)."""
    P = np.ascontiguousarray(P, np.float32)
    T = np.ascontiguousarray(T, np.int32)
    U = np.ascontiguousarray(undo, np.int32)
    n, m = len(P), len(T)
    op = np.empty((n, 3), np.float32)
    ot = np.empty((m, 3), np.int32)
    oo = np.empty(n, np.int32)
    om = np.empty(n, np.int32)
    ucap = 16 * (n + 1)
    ou = np.empty(ucap, np.int32)
    ecap = 3 * m + 1
    oc = np.empty(ecap, np.uint32)
    ocl = np.empty(ecap, np.int32)
    oi = np.empty(max(m, 1), np.uint8)
    st = np.zeros(6, np.int32)
    rc = harness().ref_round_canonical(P, T, U.ctypes.data if len(U) else None, len(U), n, m, float(scale),
                                       float(threshold), int(bool(is_stuck)), op, ot, oo, om, ou, ucap, oc, ecap, ocl,
                                       ecap, oi, st)
    if rc != 0:
        raise RuntimeError(f"reference round failed: cuda error {rc}")
    n_edges, n_main, n_total, passes, nvu, undo0 = [int(x) for x in st]
    return dict(pts=op, tris=ot, occ=oo, map=om, undo=ou[:nvu].copy(), cost=oc[:n_edges].copy(),
                collapsed=ocl[:n_total].copy(), isect0=oi[:m].copy(), n_edges=n_edges, n_main=n_main,
                n_total=n_total, undo_passes=passes, undo0=undo0)


def self_intersect_flags(P, T):
    P = np.ascontiguousarray(P, np.float32)
    T = np.ascontiguousarray(T, np.int32)
    out = np.zeros(max(len(T), 1), np.uint8)
    rc = harness().ref_self_intersect(P, T, len(P), len(T), out)
    if rc != 0:
        raise RuntimeError(f"reference self_intersect failed: {rc}")
    return out[: len(T)]


def pow2(x):
    x = np.ascontiguousarray(x, np.float32)
    y = np.empty_like(x)
    rc = harness().ref_pow2(x, y, len(x))
    if rc != 0:
        raise RuntimeError(f"ref_pow2 failed: {rc}")
    return y


def pamo_run_stage2_torch(points, triangles, ratio, tolerance=4, threshold=1e-3, iters=1000000,
                          min_verts=10000000000, stats=None):
    """PaMO.run's stage-2 loop (simp_cuda/pamo/__init__.py:122-189, stage 1 and 3
    off) with the reference's unmodified CUSimp_Free::forward and the same torch
    compaction; the per-round tensors are cloned as pybind.cpp:74-100 does.
    Returns host numpy (verts, faces) like PaMO.run."""
    import torch

    L = harness()
    target = max(int(ratio * len(triangles)), min_verts)
    tris = points[triangles].cpu().numpy()
    tris_mean = tris.mean(axis=1).mean(axis=0)
    verts = points - torch.from_numpy(tris_mean).to(points.device)
    faces = triangles
    verts_undo = torch.empty(0, dtype=torch.int32, device="cuda")
    n_verts_undo = 0
    count = 0
    is_stuck = 0
    scale = max(max(verts[:, 0].max() - verts[:, 0].min(), verts[:, 1].max() - verts[:, 1].min()),
                verts[:, 2].max() - verts[:, 2].min())
    init = True
    rounds = 0
    ptrs = (ctypes.c_void_p * 5)()
    cnt = (ctypes.c_int * 3)()
    for _ in range(iters):
        num_prev = faces.shape[0]
        verts = verts.contiguous()
        faces = faces.contiguous()
        rc = L.ref_forward_raw(verts.data_ptr(), faces.data_ptr(), verts_undo.data_ptr() if n_verts_undo else None,
                               n_verts_undo, verts.shape[0], faces.shape[0], float(scale), float(threshold),
                               int(is_stuck), int(init))
        if rc != 0:
            raise RuntimeError(f"reference forward failed: {rc}")
        rounds += 1
        L.ref_state(ptrs, cnt)
        n_pts, n_tris, nvu = cnt[0], cnt[1], cnt[2]

        v_out = torch.empty((n_pts, 3), dtype=torch.float32, device="cuda")
        f_out = torch.empty((n_tris, 3), dtype=torch.int32, device="cuda")
        occ = torch.empty((n_pts, 1), dtype=torch.int32, device="cuda")
        vmap = torch.empty((n_pts, 1), dtype=torch.int32, device="cuda")
        undo = torch.empty((nvu,), dtype=torch.int32, device="cuda")
        rc = L.ref_copy_state(v_out.data_ptr(), f_out.data_ptr(), occ.data_ptr(), vmap.data_ptr(),
                              undo.data_ptr() if nvu else None)
        if rc != 0:
            raise RuntimeError(f"reference state copy failed: {rc}")
        init = False
        verts_undo = undo
        n_verts_undo = undo.shape[0]
        verts = v_out[occ.view(-1).bool()]
        faces = f_out[f_out[:, 0] >= 0]
        faces[:, 0] = vmap[faces[:, 0].long()].view(-1)
        faces[:, 1] = vmap[faces[:, 1].long()].view(-1)
        faces[:, 2] = vmap[faces[:, 2].long()].view(-1)
        num_cur = faces.shape[0]
        if num_cur <= target or num_cur <= 10:
            break
        if num_cur == num_prev:
            count += 1
        else:
            count = 0
            is_stuck = 0
        if count >= 2:
            is_stuck = 1
        if count == tolerance:
            break
    if stats is not None:
        stats["rounds"] = rounds
    v = verts.cpu().numpy() + tris_mean
    f = faces.cpu().numpy()
    return v, f
