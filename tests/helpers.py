"""Shared test helpers: round drivers for the oracle and the CUDA path."""
from __future__ import annotations

import numpy as np


def prepare(V, F):
    """PaMO.run's centring / scale and the round-0 permutation (oracle side)."""
    from oracle import oracle as O

    tm = O.tris_mean(V, F)
    P = (V - tm).astype(np.float32)
    sx = P[:, 0].max() - P[:, 0].min()
    sy = P[:, 1].max() - P[:, 1].min()
    sz = P[:, 2].max() - P[:, 2].min()
    scale = np.float32(max(max(sx, sy), sz))
    return P, F.astype(np.int32), scale, tm


def compact(pts, tris, occ, vmap):
    occ = np.asarray(occ).reshape(-1).astype(bool)
    vmap = np.asarray(vmap).reshape(-1)
    P = pts[occ]
    keep = tris[:, 0] >= 0
    T = vmap[tris[keep]].astype(np.int32)
    return np.ascontiguousarray(P, np.float32), np.ascontiguousarray(T, np.int32)


def next_state(cur, prev, count, stuck, tolerance=4):
    """PaMO.run's progress bookkeeping (pamo/__init__.py:176-185)."""
    if cur == prev:
        count += 1
    else:
        count = 0
        stuck = 0
    if count >= 2:
        stuck = 1
    return count, stuck, count == tolerance


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a
