"""ctypes binding of the CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs import this module.  It is the checker the CUDA path is compared against,
never part of the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        L.s2o_create.restype = ctypes.c_void_p
        L.s2o_destroy.argtypes = [ctypes.c_void_p]
        L.s2o_forward.restype = ctypes.c_int
        L.s2o_forward.argtypes = [ctypes.c_void_p, _f32p, _i32p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, _f32p, _i32p, _i32p,
                                  _i32p, ctypes.POINTER(ctypes.c_int)]
        for name in ("s2o_undo_list", "s2o_edges", "s2o_collapsed", "s2o_first_near", "s2o_near"):
            getattr(L, name).restype = ctypes.POINTER(ctypes.c_int)
            getattr(L, name).argtypes = [ctypes.c_void_p]
        L.s2o_isect0.restype = ctypes.POINTER(ctypes.c_uint8)
        L.s2o_isect0.argtypes = [ctypes.c_void_p]
        L.s2o_edge_cost.restype = ctypes.POINTER(ctypes.c_uint32)
        L.s2o_edge_cost.argtypes = [ctypes.c_void_p]
        L.s2o_Q.restype = ctypes.POINTER(ctypes.c_float)
        L.s2o_Q.argtypes = [ctypes.c_void_p]
        L.s2o_n_edges.argtypes = [ctypes.c_void_p]
        L.s2o_stats.argtypes = [ctypes.c_void_p, _i32p]
        L.s2o_shuffle_faces.argtypes = [_i32p, ctypes.c_int]
        L.s2o_tris_mean.argtypes = [_f32p, _i32p, ctypes.c_int, _f32p]
        L.s2o_run.restype = ctypes.c_int
        L.s2o_run.argtypes = [ctypes.c_void_p, _f32p, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                              ctypes.c_float, ctypes.c_int, _f32p, _i32p, _i32p]
        L.s2o_pair_flag.restype = ctypes.c_int
        L.s2o_pair_flag.argtypes = [_f32p, _i32p, _f32p, _i32p, ctypes.c_float]
        L.s2o_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def shuffle_faces(F: np.ndarray) -> np.ndarray:
    """The reference's round-0 face permutation (thrust::shuffle, default engine)."""
    out = np.ascontiguousarray(F, dtype=np.int32).copy()
    lib().s2o_shuffle_faces(out, len(out))
    return out


def tris_mean(V: np.ndarray, F: np.ndarray) -> np.ndarray:
    out = np.zeros(3, np.float32)
    lib().s2o_tris_mean(np.ascontiguousarray(V, np.float32), np.ascontiguousarray(F, np.int32), len(F), out)
    return out


def pair_flag(cur9, cur_idx, qry9, qry_idx, eps=1e-3) -> bool:
    return bool(lib().s2o_pair_flag(np.ascontiguousarray(cur9, np.float32).ravel(),
                                    np.ascontiguousarray(cur_idx, np.int32), np.ascontiguousarray(qry9, np.float32).ravel(),
                                    np.ascontiguousarray(qry_idx, np.int32), eps))


class Stage2Oracle:
    """One simplifier context; mirrors the reference's CUDSP_Free object
    (simp_cuda/src/pybind.cpp:16-103), including the state kept between rounds."""

    def __init__(self):
        self._c = lib().s2o_create()

    def __del__(self):
        try:
            lib().s2o_destroy(self._c)
        except Exception:
            pass

    def forward(self, points, triangles, verts_undo, n_verts_undo, scale, threshold, is_stuck):
        """One round.  ``triangles`` must already carry the init shuffle."""
        P = np.ascontiguousarray(points, np.float32)
        T = np.ascontiguousarray(triangles, np.int32)
        n, m = len(P), len(T)
        U = np.ascontiguousarray(verts_undo, np.int32)
        op = np.empty((n, 3), np.float32)
        ot = np.empty((m, 3), np.int32)
        oo = np.empty(n, np.int32)
        om = np.empty(n, np.int32)
        nu = ctypes.c_int(0)
        rc = lib().s2o_forward(self._c, P, T, U.ctypes.data if len(U) else None, int(n_verts_undo), n, m,
                               float(scale), float(threshold), int(bool(is_stuck)), op, ot, oo, om, ctypes.byref(nu))
        if rc != 0:
            raise RuntimeError(f"oracle forward failed: {rc}")
        undo = np.ctypeslib.as_array(lib().s2o_undo_list(self._c), shape=(max(nu.value, 1),))[: nu.value].copy()
        return op, ot, oo.reshape(-1, 1), om.reshape(-1, 1), undo

    # introspection of the last round
    def stats(self):
        s = np.zeros(14, np.int32)
        lib().s2o_stats(self._c, s)
        keys = ["n_edges", "n_main", "n_total", "n_considered", "n_undo_passes", "n_vertices_undo"]
        d = {k: int(s[i]) for i, k in enumerate(keys)}
        d["undo_counts"] = [int(x) for x in s[6:14]]
        return d

    def edges(self):
        e = lib().s2o_n_edges(self._c)
        return np.ctypeslib.as_array(lib().s2o_edges(self._c), shape=(max(2 * e, 1),))[: 2 * e].reshape(-1, 2).copy()

    def edge_cost(self):
        e = lib().s2o_n_edges(self._c)
        return np.ctypeslib.as_array(lib().s2o_edge_cost(self._c), shape=(max(e, 1),))[:e].copy()

    def collapsed(self):
        s = self.stats()
        n = s["n_total"]
        return np.ctypeslib.as_array(lib().s2o_collapsed(self._c), shape=(max(n, 1),))[:n].copy()

    def isect0(self, n_tris):
        """Per-face flags of the last round's first self-intersection pass."""
        return np.ctypeslib.as_array(lib().s2o_isect0(self._c), shape=(max(n_tris, 1),))[:n_tris].copy()

    def quadrics(self, n_pts):
        return np.ctypeslib.as_array(lib().s2o_Q(self._c), shape=(n_pts * 10,)).reshape(n_pts, 10).copy()

    def run(self, points_centred, triangles_shuffled, target_faces, tolerance=4, threshold=1e-3, iters=1000000):
        P = np.ascontiguousarray(points_centred, np.float32)
        T = np.ascontiguousarray(triangles_shuffled, np.int32)
        op = np.empty_like(P)
        ot = np.empty_like(T)
        n = np.zeros(2, np.int32)
        rounds = lib().s2o_run(self._c, P, T, len(P), len(T), int(target_faces), int(tolerance), float(threshold),
                               int(iters), op, ot, n)
        return op[: n[0]].copy(), ot[: n[1]].copy(), rounds


def pamo_run_stage2(V, F, ratio, tolerance=4, threshold=1e-3, iters=1000000, min_verts=10000000000):
    """CPU restatement of PaMO.run's stage-2 part (pamo/__init__.py:122-189) with
    stage 1 off: centre by tris_mean, shuffle, rounds, compaction, "+ tris_mean"."""
    V = np.ascontiguousarray(V, np.float32)
    F = np.ascontiguousarray(F, np.int32)
    target = max(int(ratio * len(F)), min_verts)
    m = tris_mean(V, F)
    Vc = (V - m).astype(np.float32)
    Fs = shuffle_faces(F)
    o = Stage2Oracle()
    v, f, rounds = o.run(Vc, Fs, target, tolerance, threshold, iters)
    return (v + m).astype(np.float32), f, rounds
