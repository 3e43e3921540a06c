"""ctypes binding of the C++ stage-3 restatement (s3_cpu.cpp in liboracle.so)
-- TEST AND BASELINE INFRASTRUCTURE.

Only tests/ and bench.py's CPU legs (cpu_baseline, --impl reference) use it.
`process` has the meaning of pamo_safe_project.process
(simp_cuda/safe_project/src/pamo_safe_project/processing.py:23-108): normalise
by the ground truth, run `n_iters` steps of the default configuration in
float32 on the host cores, undo the normalisation.  It follows s3_oracle.py
(the FP64 numpy restatement) step for step.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import oracle as _O
from . import s3_oracle as S3

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_bound = False


def _lib():
    global _bound
    L = _O.lib()
    if not _bound:
        L.s3c_process.restype = ctypes.c_longlong
        L.s3c_process.argtypes = [_f32p, ctypes.c_int, _i32p, ctypes.c_int, _f32p, ctypes.c_int, _i32p, ctypes.c_int,
                                  _i32p, ctypes.c_int, _i32p, ctypes.c_int, _f32p, ctypes.c_int, _f32p]
        L.s3c_num_threads.restype = ctypes.c_int
        _bound = True
    return L


def num_threads():
    return _lib().s3c_num_threads()


def process(gt_V, gt_F, V, F, n_iters=5, stats=None):
    """(vertices, faces) after `n_iters` stage-3 steps; `stats` (a dict) gets
    the contact-block count of the last detection."""
    scale, t = S3.normalization(np.asarray(gt_V, np.float64))
    gV = np.ascontiguousarray(np.asarray(gt_V, np.float64) * scale + t, np.float32)
    sV64 = np.asarray(V, np.float64) * scale + t
    sV = np.ascontiguousarray(sV64, np.float32)
    F = np.ascontiguousarray(F, np.int32)
    ang = S3.internal_angles(sV64, F)
    if np.min(ang) * 180 / np.pi <= S3.Stage3Config().min_angle_thres:  # degenerate: left as it is
        return np.asarray(V, np.float32).copy(), F
    E = np.ascontiguousarray(S3.edges_unique(F), np.int32)
    H = np.ascontiguousarray(S3.hinges(F), np.int32)
    vor = np.ascontiguousarray(S3.voronoi_areas(sV64, F), np.float32)
    out = np.empty_like(sV)
    nb = _lib().s3c_process(gV, len(gV), np.ascontiguousarray(gt_F, np.int32), len(gt_F), sV, len(sV), F, len(F), E,
                            len(E), H, len(H), vor, int(n_iters), out)
    if stats is not None:
        stats["blocks"] = int(nb)
    return ((out.astype(np.float64) - t) / scale).astype(np.float32), F
