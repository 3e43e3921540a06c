"""CPU oracle of the mesh acceptance checker (test infrastructure only).

The library's checker (pamo_b200/csrc/checker.cu, pamo_check_mesh) decides with
exact-sign orientation predicates whether a triangle mesh is intersection-free,
manifold and watertight.  This module answers the same questions by a different
route, in exact rational arithmetic (fractions.Fraction on the float32
coordinates), for meshes small enough to compare every pair of faces:

  * candidate pairs: every pair of faces whose closed bounding boxes overlap
    (all pairs, in numpy);
  * per pair, the set the two closed triangles share is computed exactly --
    a segment on the planes' common line for non-coplanar faces, a convex
    polygon from Sutherland-Hodgman clipping for coplanar ones -- and the pair
    intersects when that set is not contained in what the faces share by index
    (a vertex, an edge, or the whole face for a repeated face);
  * a float filter with a wide margin (1e-8 relative) skips the exact work for
    pairs that are clearly separated by a plane.

The role model is the reference's exact CGAL checker
(simp_cuda/safe_project/scripts/cgal_intersect/main.cpp:19-111,
PMP::self_intersections), whose pair semantics this restates: faces sharing
a vertex or an edge intersect only beyond what they share.

Manifold checks follow their definitions: every undirected edge in exactly two
faces, once in each direction (watertight, consistently oriented), and the
faces around every vertex forming one closed fan.
"""
from __future__ import annotations

from fractions import Fraction as Fr

import numpy as np


def _vec(p):
    return tuple(Fr(float(x)) for x in p)


def _sub(a, b):
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def _add(a, b):
    return (a[0] + b[0], a[1] + b[1], a[2] + b[2])


def _mul(a, s):
    return (a[0] * s, a[1] * s, a[2] * s)


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def _is_zero(v):
    return v[0] == 0 and v[1] == 0 and v[2] == 0


def _on_segment(p, a, b):
    """p on the closed segment ab (a != b)."""
    d = _sub(b, a)
    if not _is_zero(_cross(d, _sub(p, a))):
        return False
    t = _dot(_sub(p, a), d)
    return 0 <= t <= _dot(d, d)


def _in_shared(p, shared_pts):
    if len(shared_pts) == 1:
        return p == shared_pts[0]
    return _on_segment(p, shared_pts[0], shared_pts[1])


def _plane_section(T, n, o):
    """Points where the closed triangle T meets the plane n . (x - o) = 0: its
    vertices on the plane and its edges' crossing points."""
    d = [_dot(n, _sub(t, o)) for t in T]
    pts = [T[i] for i in range(3) if d[i] == 0]
    for i in range(3):
        j = (i + 1) % 3
        if (d[i] < 0 < d[j]) or (d[j] < 0 < d[i]):
            pts.append(_add(T[i], _mul(_sub(T[j], T[i]), d[i] / (d[i] - d[j]))))
    return pts


def _clip(poly, B, nB):
    """Sutherland-Hodgman: the part of the convex polygon `poly` (in B's plane)
    inside the closed triangle B."""
    for i in range(3):
        a, b = B[i], B[(i + 1) % 3]
        e = _sub(b, a)
        val = [(_dot(_cross(e, _sub(x, a)), nB)) for x in poly]
        out = []
        m = len(poly)
        for k in range(m):
            x, y = poly[k], poly[(k + 1) % m]
            sx, sy = val[k], val[(k + 1) % m]
            if sx >= 0:
                out.append(x)
            if (sx < 0 < sy) or (sy < 0 < sx):
                out.append(_add(x, _mul(_sub(y, x), sx / (sx - sy))))
        poly = out
        if not poly:
            return []
    return poly


def shared_set(A, B):
    """Vertices of the set the closed non-degenerate triangles A and B share
    (empty list: disjoint).  A convex set is contained in a convex set iff its
    vertices are."""
    nA = _cross(_sub(A[1], A[0]), _sub(A[2], A[0]))
    nB = _cross(_sub(B[1], B[0]), _sub(B[2], B[0]))
    D = _cross(nA, nB)
    if _is_zero(D):
        if _dot(nA, _sub(B[0], A[0])) != 0:
            return []  # parallel planes
        return _clip(list(A), B, nB)
    sa = _plane_section(A, nB, B[0])
    sb = _plane_section(B, nA, A[0])
    if not sa or not sb:
        return []
    ta = sorted(sa, key=lambda p: _dot(D, p))
    tb = sorted(sb, key=lambda p: _dot(D, p))
    lo = ta[0] if _dot(D, ta[0]) >= _dot(D, tb[0]) else tb[0]
    hi = ta[-1] if _dot(D, ta[-1]) <= _dot(D, tb[-1]) else tb[-1]
    if _dot(D, lo) > _dot(D, hi):
        return []
    return [lo, hi]


def degenerate(V, f):
    a, b, c = (_vec(V[i]) for i in f)
    return len(set(int(i) for i in f)) < 3 or _is_zero(_cross(_sub(b, a), _sub(c, a)))


def faces_intersect(V, fa, fb):
    """Faces (index triples) of one mesh intersect beyond the vertices they
    share; both must be non-degenerate."""
    shared_idx = sorted(set(int(i) for i in fa) & set(int(i) for i in fb))
    if len(shared_idx) >= 3:
        return True
    A = [_vec(V[i]) for i in fa]
    B = [_vec(V[i]) for i in fb]
    I = shared_set(A, B)
    if not I:
        return False
    if not shared_idx:
        return True
    S = [_vec(V[i]) for i in shared_idx]
    return any(not _in_shared(p, S) for p in I)


def _candidate_pairs(V, F, chunk=2048):
    """All pairs f < g whose closed bounding boxes overlap."""
    P = V[F]
    lo, hi = P.min(1), P.max(1)
    out = []
    m = len(F)
    for s in range(0, m, chunk):
        e = min(m, s + chunk)
        ok = np.all((lo[s:e, None, :] <= hi[None, :, :]) & (lo[None, :, :] <= hi[s:e, None, :]), axis=2)
        f, g = np.nonzero(ok)
        f = f + s
        keep = f < g
        out.append(np.stack([f[keep], g[keep]], 1))
    return np.concatenate(out) if out else np.zeros((0, 2), np.int64)


def _clearly_apart(V, F, pairs):
    """Float filter: True where the two faces are certainly disjoint beyond
    their shared vertices (every unshared vertex of one face strictly on one
    side of the other's plane, by a margin far above double rounding)."""
    if not len(pairs):
        return np.zeros(0, bool)
    Vd = V.astype(np.float64)

    def side(f, g):
        a = Vd[F[f]]
        n = np.cross(a[:, 1] - a[:, 0], a[:, 2] - a[:, 0])
        b = Vd[F[g]]
        d = np.einsum("pj,pkj->pk", n, b - a[:, None, 0])
        scale = np.linalg.norm(n, axis=1)[:, None] * np.linalg.norm(b - a[:, None, 0], axis=2)
        shared = (F[g][:, :, None] == F[f][:, None, :]).any(2)
        tol = 1e-8 * scale + 1e-300
        pos = (d > tol) | shared
        neg = (d < -tol) | shared
        # all unshared vertices strictly on one side, and at least one unshared vertex
        return (pos.all(1) | neg.all(1)) & ~shared.all(1)

    f, g = pairs[:, 0], pairs[:, 1]
    return side(f, g) | side(g, f)


def check_mesh(V, F):
    """Exact check of a small mesh.  Returns a dict with per-face intersection
    flags and the counts the library's checker reports."""
    V = np.asarray(V, np.float32)
    F = np.asarray(F, np.int64)
    live = ~np.all(F == -1, axis=1)
    deg = np.array([live[i] and degenerate(V, F[i]) for i in range(len(F))], bool)
    ok_face = live & ~deg
    flags = np.zeros(len(F), np.uint8)
    n_pairs = 0
    idx = np.nonzero(ok_face)[0]
    cand = _candidate_pairs(V, F[idx]) if len(idx) else np.zeros((0, 2), np.int64)
    cand = idx[cand] if len(cand) else cand
    apart = _clearly_apart(V, F, cand)
    for f, g in cand[~apart]:
        if faces_intersect(V, F[f], F[g]):
            flags[f] = flags[g] = 1
            n_pairs += 1
    # edges: directed half-edges of live faces
    L = F[live]
    a = np.concatenate([L[:, 0], L[:, 1], L[:, 2]])
    b = np.concatenate([L[:, 1], L[:, 2], L[:, 0]])
    from collections import Counter

    directed = Counter(zip(a.tolist(), b.tolist()))
    boundary = nonmanifold = 0
    for (u, w), c in directed.items():
        back = directed.get((w, u), 0)
        if c > 1 or back > 1:
            nonmanifold += c
        elif back == 0:
            boundary += c
    # vertex fans: faces around v linked by their shared edges through v form one cycle
    around = {}
    for t in L.tolist():
        for k in range(3):
            v, x, y = t[k], t[(k + 1) % 3], t[(k + 2) % 3]
            around.setdefault(v, []).append((x, y))
    bad_vertex = 0
    for v, fan in around.items():
        nxt = {}
        dup = False
        for x, y in fan:
            if x in nxt:
                dup = True
            nxt[x] = y
        if dup:
            bad_vertex += 1
            continue
        start = fan[0][0]
        cur, steps = start, 0
        while steps <= len(fan):
            if cur not in nxt:
                break
            cur = nxt[cur]
            steps += 1
            if cur == start:
                break
        if not (cur == start and steps == len(fan)):
            bad_vertex += 1
    used = np.zeros(len(V), bool)
    used[L.reshape(-1)] = True
    return {"flags": flags, "pairs": n_pairs, "degenerate": int(deg.sum()), "boundary_half_edges": boundary,
            "nonmanifold_half_edges": nonmanifold, "nonmanifold_vertices": bad_vertex,
            "unreferenced_vertices": int((~used).sum()), "candidates": int(len(cand))}


def point_mesh_distances(P, V, F, chunk=1024):
    """Distance of each point to the closest point of the triangle mesh (V, F),
    in float64, brute force over all faces."""
    from oracle import s3_oracle as S

    Q = S.closest_points_on_mesh(np.asarray(P, np.float64), np.asarray(V, np.float64), np.asarray(F, np.int64))
    return np.linalg.norm(Q - np.asarray(P, np.float64), axis=1)


def face_samples(V, F, k):
    """Barycentric grid samples (i/k, j/k), i + j <= k, of every face, in float64
    with the arithmetic the library's sampler uses: a + s (b - a) + t (c - a)."""
    V = np.asarray(V, np.float64)
    F = np.asarray(F, np.int64)
    ij = np.array([(i, j) for i in range(k + 1) for j in range(k + 1 - i)], np.float64) / k
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    return (a[:, None] + ij[None, :, 0:1] * (b - a)[:, None] + ij[None, :, 1:2] * (c - a)[:, None]).reshape(-1, 3)


def one_sided_hausdorff(VA, FA, VB, FB, k):
    """max over A's samples of the distance to mesh B (the library's estimate)."""
    P = face_samples(VA, FA, k)
    return float(point_mesh_distances(P, VB, FB).max())
