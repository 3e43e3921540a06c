"""pamo_b200: the PaMO mesh-optimization hot path on NVIDIA B200 (sm_100a).

Drop-in surface (simp_cuda/pamo/__init__.py):

    PaMO(input_mesh, use_stage1=True, use_stage3=True).run(
        points, triangles, ratio, tolerance=4, threshold=1e-3, iter=1000000,
        min_verts=10000000000) -> (verts: np.ndarray [n,3], faces: np.ndarray [m,3])

and the per-round extension class ``CUDSP_Free`` (simp_cuda/src/pybind.cpp).
All compute runs in libpamo_b200.so (hand-written CUDA for sm_100a) through its
C ABI; torch only provides device memory and the current stream.
"""
from __future__ import annotations

import copy
import time

import numpy as np

from . import _lib
from ._lib import Context, PamoError, check
from . import metrics  # noqa: F401  (acceptance checks: check_mesh, hausdorff)

__all__ = ["PaMO", "CUDSP_Free", "Context", "PamoError", "stage2_run", "self_intersect", "remesh", "metrics"]
__version__ = "0.1.0"


def _torch():
    import torch

    return torch


def _stream_ptr(device):
    torch = _torch()
    return ctypes_void(torch.cuda.current_stream(device).cuda_stream)


def ctypes_void(x):
    import ctypes

    return ctypes.c_void_p(int(x) if x else 0)


def _mesh_arrays(mesh):
    """(V float64 [n,3], F int64 [m,3]) from a trimesh-like object or a (V, F) pair."""
    if isinstance(mesh, (tuple, list)) and len(mesh) == 2:
        V, F = mesh
    else:
        V, F = mesh.vertices, mesh.faces
    return np.asarray(V, dtype=np.float64), np.asarray(F, dtype=np.int64)


class CUDSP_Free:
    """One stage-2 simplifier; mirrors the reference's pybind class
    (simp_cuda/src/pybind.cpp:16-103): ``forward`` runs one collapse round and
    returns cloned ``(verts[n,3] f32, tris[m,3] i32, verts_occ[n,1] i32,
    verts_map[n,1] i32, verts_undo[k] i32)`` CUDA tensors."""

    def __init__(self, device: int = 0):
        self.ctx = Context(device)

    def forward(self, points, triangles, verts_undo, n_verts_undo, scale, threshold, is_stuck, init):
        torch = _torch()
        for name, t in (("points", points), ("triangles", triangles), ("verts_undo", verts_undo)):
            if not t.is_cuda:
                raise AssertionError(f"{name} must be a CUDA tensor")
            if not t.is_contiguous():
                raise AssertionError(f"{name} must be contiguous")
        if points.dtype != torch.float32:
            raise RuntimeError("points type must match the pamo class")
        if triangles.dtype != torch.int32:
            raise RuntimeError("triangles type must match the pamo class")
        n, m = int(points.shape[0]), int(triangles.shape[0])
        dev = points.device
        ov = torch.empty((n, 3), dtype=torch.float32, device=dev)
        ot = torch.empty((m, 3), dtype=torch.int32, device=dev)
        oo = torch.empty((n, 1), dtype=torch.int32, device=dev)
        om = torch.empty((n, 1), dtype=torch.int32, device=dev)
        import ctypes

        nu = ctypes.c_int(0)
        stream = _stream_ptr(dev)
        check("pamo_free_forward", _lib.lib().pamo_free_forward(
            self.ctx.handle, points.data_ptr(), triangles.data_ptr(),
            verts_undo.data_ptr() if int(n_verts_undo) > 0 else None, int(n_verts_undo), n, m, float(scale),
            float(threshold), int(bool(is_stuck)), int(bool(init)), stream, ov.data_ptr(), ot.data_ptr(),
            oo.data_ptr(), om.data_ptr(), ctypes.byref(nu)))
        undo = torch.empty((nu.value,), dtype=torch.int32, device=dev)
        check("pamo_free_copy_undo", _lib.lib().pamo_free_copy_undo(
            self.ctx.handle, undo.data_ptr() if nu.value else None, nu.value, stream))
        return ov, ot, oo, om, undo


def stage2_run(ctx: Context, points, triangles, target_faces: int, tolerance=4, threshold=1e-3, iters=1000000,
               offset=None):
    """Device-resident stage-2 loop of PaMO.run.  Returns (verts, faces) CUDA
    tensors (verts already shifted back by the centring offset) and the number of
    rounds.  With `offset` (3 floats) the points are already centred -- stage
    1's output -- and `offset` is added back instead of centring here."""
    import ctypes

    torch = _torch()
    points = points.contiguous()
    triangles = triangles.contiguous()
    dev = points.device
    stream = _stream_ptr(dev)
    on, om, rounds = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    args = (int(min(int(target_faces), 2**62)), int(tolerance), float(threshold), int(min(iters, 2**31 - 1)), stream,
            ctypes.byref(on), ctypes.byref(om), ctypes.byref(rounds))
    if offset is None:
        check("pamo_stage2_run", _lib.lib().pamo_stage2_run(
            ctx.handle, points.data_ptr(), triangles.data_ptr(), int(points.shape[0]), int(triangles.shape[0]), *args))
    else:
        off = (ctypes.c_float * 3)(*[float(x) for x in offset])
        check("pamo_stage2_run_centred", _lib.lib().pamo_stage2_run_centred(
            ctx.handle, points.data_ptr(), triangles.data_ptr(), int(points.shape[0]), int(triangles.shape[0]), off,
            *args))
    v = torch.empty((on.value, 3), dtype=torch.float32, device=dev)
    f = torch.empty((om.value, 3), dtype=torch.int32, device=dev)
    check("pamo_stage2_fetch", _lib.lib().pamo_stage2_fetch(ctx.handle, v.data_ptr(), f.data_ptr(), 0, stream))
    return v, f, rounds.value


def remesh(ctx: Context, points, triangles, resolution=256):
    """Stage 1 of PaMO.run on the device (pamo_remesh): returns (verts, faces)
    CUDA tensors in the frame centred on the input's tris_mean, and tris_mean
    (numpy float32 [3]), as the reference's preprocess_mesh + remesh give them
    (simp_cuda/pamo/__init__.py:60-142)."""
    import ctypes

    torch = _torch()
    points = points.contiguous()
    triangles = triangles.contiguous()
    dev = points.device
    stream = _stream_ptr(dev)
    nv, nt = ctypes.c_int(), ctypes.c_int()
    check("pamo_remesh", _lib.lib().pamo_remesh(ctx.handle, points.data_ptr(), triangles.data_ptr(),
                                                int(points.shape[0]), int(triangles.shape[0]), int(resolution), stream,
                                                ctypes.byref(nv), ctypes.byref(nt)))
    v = torch.empty((nv.value, 3), dtype=torch.float32, device=dev)
    f = torch.empty((nt.value, 3), dtype=torch.int32, device=dev)
    off = (ctypes.c_float * 3)()
    check("pamo_remesh_fetch", _lib.lib().pamo_remesh_fetch(ctx.handle, v.data_ptr(), f.data_ptr(), off, stream))
    return v, f, np.array(off[:], np.float32)


def stage1_resolution(target_faces):
    """PaMO.run's grid resolution for stage 1 (pamo/__init__.py:134-137)."""
    R = 256
    if target_faces <= 1000:
        R = 128
    if target_faces <= 50:
        R = 64
    return R


def self_intersect(ctx: Context, points, triangles):
    """Per-face flags (uint8 CUDA tensor) of the faces in intersecting pairs, with
    the reference's pair predicate; also returns the number of candidate pairs."""
    import ctypes

    torch = _torch()
    points = points.contiguous()
    triangles = triangles.contiguous()
    out = torch.zeros(int(triangles.shape[0]), dtype=torch.uint8, device=points.device)
    npairs = ctypes.c_longlong(0)
    check("pamo_self_intersect", _lib.lib().pamo_self_intersect(
        ctx.handle, points.data_ptr(), triangles.data_ptr(), int(points.shape[0]), int(triangles.shape[0]),
        out.data_ptr(), ctypes.byref(npairs), _stream_ptr(points.device)))
    return out, npairs.value


class PaMO:
    """Drop-in for the reference's ``PaMO`` (simp_cuda/pamo/__init__.py:18-205).

    ``input_mesh`` is any object with ``vertices``/``faces`` (e.g. a trimesh) or a
    ``(V, F)`` pair; it is kept as the ground truth for stage 3.  ``quality=True``
    switches stage 2 to its quality mode (see pamo_set_quality); the default is
    the reference's algorithm.
    """

    def __init__(self, input_mesh, use_stage1=True, use_stage3=True, device: int = 0, verbose: bool = True,
                 quality: bool = False):
        self.use_stage1 = use_stage1
        self.use_stage3 = use_stage3
        self.verbose = verbose
        if verbose:
            print("Stage1 : ", self.use_stage1)
            print("Stage3 : ", self.use_stage3)
        V, F = _mesh_arrays(input_mesh)
        self.bbox = np.stack([V.min(0), V.max(0)]) if len(V) else np.zeros((2, 3))
        self.gt_mesh = (copy.deepcopy(V), copy.deepcopy(F))
        # a float32 input is kept as such too, so stage 3 can normalise it on the device
        V_in = input_mesh[0] if isinstance(input_mesh, (tuple, list)) else getattr(input_mesh, "vertices", None)
        self._gt_f32 = np.array(V_in, dtype=np.float32) if getattr(V_in, "dtype", None) == np.float32 else None
        self._gt_f32_pinned = None
        self.ctx = Context(device)
        # quality mode (no reference counterpart): FP64 quadrics, the quadric's
        # minimiser as collapse position, exact-predicate undo (pamo_set_quality)
        self.quality = bool(quality)
        if self.quality:
            check("pamo_set_quality", _lib.lib().pamo_set_quality(self.ctx.handle, 1))
        self.device = device
        self.target_faces = None
        self.last_rounds = 0
        self.timings = {}
        if use_stage3:
            from .safe_project import Stage3Config, Stage3System

            self.config = Stage3Config()
            self.system = Stage3System(self.config, device=device)

    def run(self, points, triangles, ratio, tolerance=4, threshold=1e-3, iter=1000000, min_verts=10000000000):
        torch = _torch()
        self.target_faces = max(int(ratio * len(triangles)), min_verts)
        if self.verbose:
            print("Target faces : {}".format(self.target_faces))
        offset = None
        if self.use_stage1:
            t0 = time.time()
            points, triangles, offset = remesh(self.ctx, points, triangles, stage1_resolution(self.target_faces))
            self.timings["stage1"] = time.time() - t0
            self.stage1_faces = int(triangles.shape[0])
            if self.verbose:
                print(f"Time for Remeshing: {self.timings['stage1']} sec")
        t0 = time.time()
        v, f, rounds = stage2_run(self.ctx, points, triangles, self.target_faces, tolerance, threshold, iter,
                                  offset=offset)
        self.last_rounds = rounds
        verts = v.cpu().numpy()
        faces = f.cpu().numpy()
        self.timings["stage2"] = time.time() - t0
        if self.verbose:
            print(f"Time for Simplification: {self.timings['stage2']} sec")
        if self.use_stage3:
            from .safe_project import has_duplicate_vertices, merge_vertices, process

            t0 = time.time()
            # the reference wraps the stage-2 result in trimesh.Trimesh(process=True),
            # which merges coincident vertices (pamo/__init__.py:193-203); the
            # device check finds whether there is anything to merge
            if has_duplicate_vertices(v):
                v2, f2 = merge_vertices(verts.astype(np.float64), faces)
            else:
                v2, f2 = verts.astype(np.float64), faces
            gt_v = self.gt_mesh[0]
            if self._gt_f32 is not None:
                if self._gt_f32_pinned is None:  # page-locked host copies of the ground truth
                    self._gt_f32_pinned = torch.from_numpy(self._gt_f32).pin_memory()
                    self._gt_f_pinned = torch.from_numpy(self.gt_mesh[1].astype(np.int32)).pin_memory()
                gt_v = self._gt_f32_pinned
            gt_f = self._gt_f_pinned if self._gt_f32 is not None else self.gt_mesh[1]
            # the ground truth is this object's own copy, the same on every run
            verts, faces = process(gt_v, gt_f, v2, f2, 5, system=self.system, config=self.config, gt_static=True)
            self.timings["stage3"] = time.time() - t0
        return verts, faces
