"""The library's exact predicates (pamo_b200/csrc/exact.cuh), built for the host
from the same header, against rational arithmetic: orientation signs on random
and on (nearly) degenerate float32 inputs, and the pair decisions of the mesh
checker against the rational oracle (oracle/check_oracle.py)."""
import ctypes
import os
import subprocess
from fractions import Fraction as Fr

import numpy as np
import pytest
from helpers import crafted_mesh

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("exact") / "libexact_harness.so")
    src = os.path.join(ROOT, "tests", "native", "exact_harness.cpp")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", src, "-o", out], check=True)
    lib = ctypes.CDLL(out)
    for name in ("h_orient3d", "h_orient2d", "h_faces_intersect"):
        getattr(lib, name).restype = None
    return lib


def _sign(x):
    return (x > 0) - (x < 0)


def _orient3d_frac(a, b, c, d):
    r = [[Fr(float(p[k])) - Fr(float(d[k])) for k in range(3)] for p in (a, b, c)]
    det = (r[0][0] * (r[1][1] * r[2][2] - r[1][2] * r[2][1]) - r[0][1] * (r[1][0] * r[2][2] - r[1][2] * r[2][0]) +
           r[0][2] * (r[1][0] * r[2][1] - r[1][1] * r[2][0]))
    return _sign(det)


def _orient2d_frac(a, b, c):
    ax, ay, bx, by, cx, cy = (Fr(float(x)) for x in (*a, *b, *c))
    return _sign((ax - cx) * (by - cy) - (ay - cy) * (bx - cx))


def _near_coplanar(rng, n):
    """Quadruples whose fourth point is a float32 rounding of a point in the
    plane of the first three: mostly undecidable by a plain double evaluation."""
    a, b, c = (rng.standard_normal((n, 3)) * 10.0 ** rng.integers(-3, 4, (n, 1)) for _ in range(3))
    s, t = rng.random((n, 1)), rng.random((n, 1))
    d = a + s * (b - a) + t * (c - a)
    q = np.stack([a, b, c, d], 1).astype(np.float32)
    # exact cases: integer points on a plane, and repeated / collinear points
    k = n // 4
    g = rng.integers(-1000, 1000, (k, 3, 2)).astype(np.float64)
    base = rng.integers(-5, 5, (k, 3)).astype(np.float64)
    u, v = np.array([1.0, 2.0, 3.0]), np.array([-2.0, 0.5, 1.0])
    pts = base[:, None, :] + g[:, :, 0:1] * u + g[:, :, 1:2] * v
    w = rng.integers(-1000, 1000, (k, 2)).astype(np.float64)
    q[:k, :3] = pts
    q[:k, 3] = base + w[:, 0:1] * u + w[:, 1:2] * v
    q[k:2 * k, 3] = q[k:2 * k, 0]
    q[2 * k:3 * k, 2] = 0.5 * (q[2 * k:3 * k, 0] + q[2 * k:3 * k, 1])
    return q


def test_orient3d_signs_exact(harness):
    rng = np.random.default_rng(0)
    q = np.concatenate([rng.standard_normal((2000, 4, 3)).astype(np.float32), _near_coplanar(rng, 4000)])
    q = np.ascontiguousarray(q, np.float32)
    out = np.zeros(len(q), np.int32)
    harness.h_orient3d(q.ctypes.data_as(ctypes.c_void_p), ctypes.c_longlong(len(q)), out.ctypes.data_as(ctypes.c_void_p))
    want = np.array([_orient3d_frac(*x) for x in q])
    assert np.array_equal(out, want), np.nonzero(out != want)[0][:10]
    assert (want == 0).sum() > 500  # degenerate cases are exercised
    # a plain double evaluation gets a share of the near-coplanar ones wrong
    qd = q.astype(np.float64)
    r = qd[:, :3] - qd[:, 3:4]
    naive = np.sign(np.linalg.det(r)).astype(int)
    assert (naive != want).sum() > 50


def test_orient2d_signs_exact(harness):
    rng = np.random.default_rng(1)
    a, b = rng.standard_normal((3000, 2)), rng.standard_normal((3000, 2))
    t = rng.random((3000, 1))
    c = a + t * (b - a)  # nearly collinear after rounding
    x = np.concatenate([np.stack([a, b, c], 1), rng.standard_normal((1000, 3, 2))]).astype(np.float32)
    x[:300, 2] = x[:300, 0]
    x = np.ascontiguousarray(x.reshape(-1, 6))
    out = np.zeros(len(x), np.int32)
    harness.h_orient2d(x.ctypes.data_as(ctypes.c_void_p), ctypes.c_longlong(len(x)), out.ctypes.data_as(ctypes.c_void_p))
    want = np.array([_orient2d_frac(r[0:2], r[2:4], r[4:6]) for r in x])
    assert np.array_equal(out, want)


def _meshes():
    from pamo_b200 import meshgen as mg

    g = np.load(os.path.join(ROOT, "tests", "golden", "isect.npz"))
    out = [crafted_mesh()]
    out += [(g[f"{k}_V"].astype(np.float32), g[f"{k}_F"].astype(np.int32)) for k in ("crumpled", "folded_grids", "soup")]
    V, F = mg.displaced_icosphere(2, 3)
    out.append((V.astype(np.float32), F.astype(np.int32)))
    return out


def test_pair_decisions_match_rational_oracle(harness):
    from oracle import check_oracle as C

    for V, F in _meshes():
        V = np.ascontiguousarray(V, np.float32)
        F = np.ascontiguousarray(F, np.int32)
        cand = C._candidate_pairs(V, F.astype(np.int64))
        if len(cand) > 6000:
            cand = cand[np.random.default_rng(0).choice(len(cand), 6000, replace=False)]
        pairs = np.ascontiguousarray(cand, np.int32)
        out = np.zeros(len(pairs), np.int32)
        harness.h_faces_intersect(V.ctypes.data_as(ctypes.c_void_p), F.ctypes.data_as(ctypes.c_void_p),
                                  pairs.ctypes.data_as(ctypes.c_void_p), ctypes.c_longlong(len(pairs)),
                                  out.ctypes.data_as(ctypes.c_void_p))
        for (f, g), got in zip(pairs, out):
            if C.degenerate(V, F[f]) or C.degenerate(V, F[g]):
                assert got == -1
                continue
            want = C.faces_intersect(V, F[f], F[g])
            assert got == int(want), (f, g, F[f], F[g], got, want)


def test_crafted_mesh_decisions(harness):
    """The crafted cases decide as their construction says."""
    from oracle import check_oracle as C

    V, F = crafted_mesh()
    res = C.check_mesh(V, F)
    # face 0 meets 1 (coplanar overlap), 2 (pierced), 4 (folded), 7 (touch); 3 and 5 only share
    want = {(0, 1), (0, 2), (0, 4), (0, 7)}
    got = set()
    for f in range(len(F)):
        for g in range(f + 1, len(F)):
            if C.faces_intersect(V, F[f], F[g]):
                got.add((f, g))
    assert want <= got
    assert (0, 3) not in got and (0, 5) not in got and (0, 6) not in got
    assert res["flags"][0] == 1 and res["pairs"] == len(got)
