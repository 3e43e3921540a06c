"""Seeded synthetic meshes for the simplification workloads.

The reference evaluates on scanned/CAD datasets (DTC, Thingi10K) that are not
available here; these generators stand in for them with the shapes, sizes and
value distributions the workloads name:

* ``displaced_icosphere(level, seed)`` -- recursive midpoint icosphere whose
  vertices are scaled radially by ``1 + 0.1 * sum_lm c_lm Y_lm`` (real
  spherical harmonics up to degree 8, ``c_lm ~ N(0,1)/(l+1)^2``).  Level 5 gives
  10,242 vertices / 20,480 faces.
* ``noisy_torus(nu, nv, seed)`` -- ``nu x nv`` torus grid (R=1, r=0.35),
  displaced along the normal by ``0.02 * value_noise`` (4 octaves, base
  frequency 8).  1024 x 1024 gives 1,048,576 vertices / 2,097,152 faces.
* ``geodesic_sphere(freq)`` / ``displaced_geodesic(faces, seed)`` -- class-I
  geodesic spheres of any frequency (``20 * freq^2`` faces) for the mixed-size
  batches.
* ``thin_shell_pair(faces, gap, seed)`` -- two concentric displaced spheres
  separated by ``gap`` (contact stress for the safe projection).

All outputs are ``(float32 [V,3], int32 [F,3])`` closed, consistently
(outward) oriented 2-manifolds.
"""
from __future__ import annotations

import math

import numpy as np

__all__ = [
    "icosahedron",
    "icosphere",
    "displaced_icosphere",
    "noisy_torus",
    "geodesic_sphere",
    "displaced_geodesic",
    "thin_shell_pair",
    "sh_radial_field",
    "value_noise3",
    "mixed_batch",
]


def icosahedron():
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array(
        [
            [-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
            [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
            [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1],
        ],
        dtype=np.float64,
    )
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array(
        [
            [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
            [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
            [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
            [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1],
        ],
        dtype=np.int64,
    )
    return v, f


def icosphere(level: int):
    """Recursive midpoint subdivision, each new vertex projected to the unit sphere."""
    v, f = icosahedron()
    verts = [tuple(x) for x in v]
    verts = list(v)
    for _ in range(level):
        cache = {}
        new_f = np.empty((len(f) * 4, 3), dtype=np.int64)

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            idx = cache.get(key)
            if idx is None:
                p = (verts[a] + verts[b]) * 0.5
                p = p / np.linalg.norm(p)
                idx = len(verts)
                verts.append(p)
                cache[key] = idx
            return idx

        for n, (a, b, c) in enumerate(f):
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            new_f[4 * n + 0] = (a, ab, ca)
            new_f[4 * n + 1] = (b, bc, ab)
            new_f[4 * n + 2] = (c, ca, bc)
            new_f[4 * n + 3] = (ab, bc, ca)
        f = new_f
    return np.asarray(verts, dtype=np.float64), f


def _legendre_all(lmax: int, x: np.ndarray):
    """Associated Legendre P_l^m(x) for 0<=m<=l<=lmax (no Condon-Shortley phase)."""
    P = {}
    s = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    P[(0, 0)] = np.ones_like(x)
    for m in range(1, lmax + 1):
        P[(m, m)] = P[(m - 1, m - 1)] * (2 * m - 1) * s
    for m in range(0, lmax):
        P[(m + 1, m)] = x * (2 * m + 1) * P[(m, m)]
    for m in range(0, lmax + 1):
        for l in range(m + 2, lmax + 1):
            P[(l, m)] = ((2 * l - 1) * x * P[(l - 1, m)] - (l + m - 1) * P[(l - 2, m)]) / (l - m)
    return P


def sh_radial_field(dirs: np.ndarray, lmax: int = 8, seed: int = 0) -> np.ndarray:
    """sum_lm c_lm Y_lm(dir) with real orthonormal SH and c_lm ~ N(0,1)/(l+1)^2."""
    rng = np.random.default_rng(seed)
    d = dirs / np.linalg.norm(dirs, axis=1, keepdims=True)
    ct = np.clip(d[:, 2], -1.0, 1.0)
    phi = np.arctan2(d[:, 1], d[:, 0])
    P = _legendre_all(lmax, ct)
    out = np.zeros(len(d), dtype=np.float64)
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            c = rng.standard_normal() / (l + 1) ** 2
            am = abs(m)
            norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
            if m == 0:
                y = norm * P[(l, 0)]
            elif m > 0:
                y = math.sqrt(2.0) * norm * P[(l, am)] * np.cos(am * phi)
            else:
                y = math.sqrt(2.0) * norm * P[(l, am)] * np.sin(am * phi)
            out += c * y
    return out


def displaced_icosphere(level: int = 5, seed: int = 0, amplitude: float = 0.1):
    v, f = icosphere(level)
    r = 1.0 + amplitude * sh_radial_field(v, 8, seed)
    v = v * r[:, None]
    return v.astype(np.float32), f.astype(np.int32)


def value_noise3(p: np.ndarray, seed: int = 0, octaves: int = 4, base_freq: float = 8.0) -> np.ndarray:
    """Seeded lattice value noise in [-1,1], smoothstep-trilinear, summed over octaves
    (frequency doubles, amplitude halves) and normalised by the amplitude sum."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(256).astype(np.int64)
    perm = np.concatenate([perm, perm])
    vals = rng.uniform(-1.0, 1.0, 256)

    def lattice(ix, iy, iz):
        h = perm[(perm[(perm[ix & 255] + iy) & 255] + iz) & 255]
        return vals[h]

    total = np.zeros(len(p), dtype=np.float64)
    amp, freq, asum = 1.0, base_freq, 0.0
    for _ in range(octaves):
        q = p * freq
        i0 = np.floor(q).astype(np.int64)
        t = q - i0
        t = t * t * (3.0 - 2.0 * t)
        acc = np.zeros(len(p), dtype=np.float64)
        for dx in (0, 1):
            wx = t[:, 0] if dx else 1.0 - t[:, 0]
            for dy in (0, 1):
                wy = t[:, 1] if dy else 1.0 - t[:, 1]
                for dz in (0, 1):
                    wz = t[:, 2] if dz else 1.0 - t[:, 2]
                    acc += wx * wy * wz * lattice(i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz)
        total += amp * acc
        asum += amp
        amp *= 0.5
        freq *= 2.0
    return total / asum


def noisy_torus(nu: int = 1024, nv: int = 1024, seed: int = 0, R: float = 1.0, r: float = 0.35,
                amplitude: float = 0.02):
    i = np.arange(nu, dtype=np.float64)
    j = np.arange(nv, dtype=np.float64)
    u = 2.0 * np.pi * i / nu
    w = 2.0 * np.pi * j / nv
    U, W = np.meshgrid(u, w, indexing="ij")
    cu, su, cw, sw = np.cos(U), np.sin(U), np.cos(W), np.sin(W)
    pos = np.stack([(R + r * cw) * cu, (R + r * cw) * su, r * sw], axis=-1).reshape(-1, 3)
    nrm = np.stack([cw * cu, cw * su, sw], axis=-1).reshape(-1, 3)
    disp = amplitude * value_noise3(pos, seed=seed)
    pos = pos + nrm * disp[:, None]
    ii, jj = np.meshgrid(np.arange(nu), np.arange(nv), indexing="ij")
    a = ii * nv + jj
    b = ((ii + 1) % nu) * nv + jj
    c = ((ii + 1) % nu) * nv + (jj + 1) % nv
    d = ii * nv + (jj + 1) % nv
    f = np.stack([np.stack([a, b, c], -1), np.stack([a, c, d], -1)], axis=2).reshape(-1, 3)
    # orient outward: normal of the first face must agree with the radial normal
    v0, v1, v2 = pos[f[0, 0]], pos[f[0, 1]], pos[f[0, 2]]
    if np.dot(np.cross(v1 - v0, v2 - v0), nrm[f[0, 0]]) < 0:
        f = f[:, [0, 2, 1]]
    return pos.astype(np.float32), f.astype(np.int32)


def geodesic_sphere(freq: int):
    """Class-I geodesic sphere: each icosahedron face split into freq^2 triangles,
    points pushed out to the unit sphere.  Vertices: the 12 corners, then the
    freq-1 points of each of the 30 edges (walking from its lower corner), then
    each face's interior points row by row; a point shared by faces is computed
    once, from its edge."""
    f_ = max(1, int(freq))
    cv, cf = icosahedron()
    cv = np.asarray(cv, np.float64)
    cf = np.asarray(cf, np.int64)
    ne = f_ - 1
    edges = sorted({(min(a, b), max(a, b)) for t in cf for a, b in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0]))})
    eid = {e: k for k, e in enumerate(edges)}
    e_lo = cv[[e[0] for e in edges]]
    e_hi = cv[[e[1] for e in edges]]
    st = (np.arange(1, f_) / f_)[None, :, None]
    ep = (e_lo[:, None, :] + (e_hi - e_lo)[:, None, :] * st).reshape(-1, 3)
    # interior grid points (i, j) with i, j, k = freq - i - j all >= 1, row-major
    I, J = np.meshgrid(np.arange(f_ + 1), np.arange(f_ + 1), indexing="ij")
    K = f_ - I - J
    inner = (I >= 1) & (J >= 1) & (K >= 1)
    ii, jj, kk = I[inner], J[inner], K[inner]
    n_in = len(ii)
    A, B, C = cv[cf[:, 0]], cv[cf[:, 1]], cv[cf[:, 2]]
    ip = (A[:, None, :] * (kk / f_)[None, :, None] + B[:, None, :] * (ii / f_)[None, :, None] +
          C[:, None, :] * (jj / f_)[None, :, None]).reshape(-1, 3)
    pos = np.concatenate([cv, ep, ip], axis=0)
    pos = pos / np.sqrt((pos * pos).sum(axis=1))[:, None]
    base_e, base_i = 12, 12 + 30 * ne

    def edge_ids(x, y, t):  # t-th point (1..freq-1) walking from corner x to corner y
        if x < y:
            return base_e + eid[(x, y)] * ne + (t - 1)
        return base_e + eid[(y, x)] * ne + (f_ - t - 1)

    inner_pos = np.full((f_ + 1, f_ + 1), -1, np.int64)
    inner_pos[inner] = np.arange(n_in)
    faces = []
    valid = K >= 0
    for fi, (a, b, c) in enumerate(cf):
        idx = np.full((f_ + 1, f_ + 1), -1, np.int64)
        idx[inner] = base_i + fi * n_in + inner_pos[inner]
        idx[0, 0], idx[f_, 0], idx[0, f_] = a, b, c
        t = np.arange(1, f_)
        if ne:
            idx[t, 0] = edge_ids(a, b, t)          # j = 0: from a towards b
            idx[0, t] = edge_ids(a, c, t)          # i = 0: from a towards c
            idx[f_ - t, t] = edge_ids(b, c, t)     # k = 0: from b towards c
        i0, j0 = np.nonzero(valid & (I < f_) & (J < f_ - I))
        faces.append(np.stack([idx[i0, j0], idx[i0 + 1, j0], idx[i0, j0 + 1]], 1))
        i1, j1 = np.nonzero(valid & (I + J + 2 <= f_))
        faces.append(np.stack([idx[i1 + 1, j1], idx[i1 + 1, j1 + 1], idx[i1, j1 + 1]], 1))
    F = np.concatenate(faces, axis=0)
    return pos, F


def displaced_geodesic(n_faces: int, seed: int = 0, amplitude: float = 0.1, radius: float = 1.0):
    freq = max(1, int(round(math.sqrt(n_faces / 20.0))))
    v, f = geodesic_sphere(freq)
    r = radius * (1.0 + amplitude * sh_radial_field(v, 8, seed))
    return (v * r[:, None]).astype(np.float32), f.astype(np.int32)


def thin_shell_pair(n_faces: int = 500_000, gap: float = 2e-3, seed: int = 0, amplitude: float = 0.05):
    """Two concentric displaced spheres (n_faces/2 faces each), the outer one offset
    radially by ``gap``; both outward oriented."""
    freq = max(1, int(round(math.sqrt(n_faces / 2 / 20.0))))
    v, f = geodesic_sphere(freq)
    r = 1.0 + amplitude * sh_radial_field(v, 8, seed)
    inner = v * r[:, None]
    outer = v * (r + gap)[:, None]
    V = np.concatenate([inner, outer], axis=0)
    F = np.concatenate([f, f + len(v)], axis=0)
    return V.astype(np.float32), F.astype(np.int32)


def mixed_batch(n_meshes: int = 256, fmin: int = 5_000, fmax: int = 500_000, seed: int = 0,
                ratios=(0.001, 0.01, 0.05)):
    """Mixed-size request list: (name, V, F, ratio) with face counts log-uniform in
    [fmin, fmax], mixing displaced spheres, noisy tori and thin-shell pairs."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_meshes):
        nf = int(math.exp(rng.uniform(math.log(fmin), math.log(fmax))))
        fam = int(rng.integers(0, 3))
        ratio = float(ratios[int(rng.integers(0, len(ratios)))])
        s = int(rng.integers(0, 2**31 - 1))
        if fam == 0:
            V, F = displaced_geodesic(nf, seed=s)
            name = "sphere"
        elif fam == 1:
            n = max(8, int(round(math.sqrt(nf / 2.0))))
            V, F = noisy_torus(n, n, seed=s)
            name = "torus"
        else:
            gap = float(rng.uniform(1e-3, 1e-2))
            V, F = thin_shell_pair(nf, gap=gap, seed=s)
            name = "shell"
        out.append((name, V, F, ratio))
    return out
