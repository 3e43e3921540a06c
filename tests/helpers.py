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


def crafted_mesh():
    """Small meshes with touching, coplanar and shared-element configurations."""
    V = np.array([
        [0, 0, 0], [1, 0, 0], [0, 1, 0],          # 0-2 base triangle in z = 0
        [0.25, 0.25, 0], [1.25, 0.25, 0], [0.25, 1.25, 0],  # 3-5 coplanar overlapping
        [0.5, 0.5, -1], [0.5, 0.5, 1], [2, 2, 0.5],  # 6-8 piercing triangle
        [1, 1, 0], [2, 0, 0],                     # 9-10 share edge 1-2 coplanar, opposite side / folded
        [0.2, 0.2, 0], [0, 0, 1],                 # 11-12 folded onto edge (0,1) side
        [1, 0, 1], [3, 3, 3],                     # 13-14
        [0.5, 0, 0], [0.5, -1, 0],                # 15-16 touching at an edge point
    ], np.float32)
    F = np.array([
        [0, 1, 2],      # 0
        [3, 4, 5],      # 1 coplanar overlap with 0
        [6, 7, 8],      # 2 pierces 0
        [1, 9, 2],      # 3 shares edge (1,2) with 0, coplanar, opposite side: fine
        [0, 1, 11],     # 4 shares edge (0,1), coplanar, same side: folded
        [0, 12, 13],    # 5 shares vertex 0, leaves the plane: fine
        [2, 12, 14],    # 6 shares vertex 2
        [15, 16, 10],   # 7 touches edge (0,1) of face 0 at a point
    ], np.int32)
    return V, F
