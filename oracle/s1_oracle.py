"""CPU restatement of stage 1 of PaMO.run (remeshing) -- TEST INFRASTRUCTURE.

The reference (simp_cuda/pamo/__init__.py:60-120,130-142) normalises the input
triangles into the unit cube (preprocess_mesh), computes a narrow-band signed
distance field on an R^3 grid with torchcumesh2sdf.get_sdf(tris, R, band),
shifts it by -0.9/R, extracts a quad mesh with pdmc.DMC (dual marching cubes)
and splits every quad into the two triangles that keep the larger smallest
angle.  Neither torchcumesh2sdf nor pdmc is in the reference tree or installed
here, so their steps are restated from their published descriptions and parity
with them is unpinned; this module defines the semantics the CUDA stage 1
(pamo_b200/csrc/stage1.cu) must reproduce bit for bit:

  * preprocess: exactly the reference's float32 numpy arithmetic
    (pamo/__init__.py:60-72);
  * grid samples at ((i + 0.5) / R, (j + 0.5) / R, (k + 0.5) / R);
  * unsigned distance (float64) from each sample to the nearest triangle when
    it is below `band`, else `band`;
  * sign by flood fill: samples farther than half a voxel from every triangle
    are free; free samples 6-connected to the grid's boundary are outside (+),
    every other sample is inside (-); then d - 0.9 / R (float64);
  * dual marching cubes with one vertex per surface patch of a cell: a sample
    is inside when its value is negative; on each cube face the crossed edges
    pair up (two crossings pair; on a face with four crossings each outside
    corner is cut off by pairing its two edges, a rule that depends only on the
    face and so agrees between the two cells sharing it), the pairings split a
    cell's crossed edges into cycles, each cycle is a patch with one vertex at
    the mean of its edges' crossing points, and every crossed grid edge gives a
    quad through the patch vertices of its four cells, wound so the normal
    points outside;
  * quad split: per quad the configuration (0,1,3),(1,2,3) or (0,1,2),(0,2,3)
    whose largest corner cosine is smaller, the first kind listed first, as the
    reference orders them (pamo/__init__.py:95-118); cosines in float64;
  * vertices mapped back to the centred frame by the inverse of the
    normalisation, in float64, then rounded to float32.

Orders: vertices by cell (x fastest) and patch within the cell; quads by axis
(x, y, z edges) then by the edge's lower sample (x fastest).
"""
from __future__ import annotations

import numpy as np

# cube corners c = x + 2 y + 4 z; edges 0-3 along x, 4-7 along y, 8-11 along z
EDGE_CORNERS = [(0, 1), (2, 3), (4, 5), (6, 7), (0, 2), (1, 3), (4, 6), (5, 7), (0, 4), (1, 5), (2, 6), (3, 7)]
# faces as corner cycles, and the edge between consecutive corners
FACE_CORNERS = [(0, 2, 6, 4), (1, 3, 7, 5), (0, 1, 5, 4), (2, 3, 7, 6), (0, 1, 3, 2), (4, 5, 7, 6)]


def _edge_of(a, b):
    for i, (p, q) in enumerate(EDGE_CORNERS):
        if {p, q} == {a, b}:
            return i
    raise ValueError


def patch_table():
    """For each of the 256 sign cases (bit c set: corner c inside): the patch
    of each of the 12 edges (-1: not crossed) and the number of patches."""
    table = np.full((256, 12), -1, np.int32)
    counts = np.zeros(256, np.int32)
    for case in range(256):
        inside = [(case >> c) & 1 for c in range(8)]
        crossed = [inside[a] != inside[b] for a, b in EDGE_CORNERS]
        link = {e: [] for e in range(12) if crossed[e]}
        for cyc in FACE_CORNERS:
            es = [_edge_of(cyc[k], cyc[(k + 1) % 4]) for k in range(4)]
            cr = [e for e in es if crossed[e]]
            if len(cr) == 2:
                link[cr[0]].append(cr[1])
                link[cr[1]].append(cr[0])
            elif len(cr) == 4:
                # cut off each outside corner: pair its two edges on this face
                for k in range(4):
                    if not inside[cyc[k]]:
                        e1, e2 = es[(k + 3) % 4], es[k]  # edges before and after corner k
                        link[e1].append(e2)
                        link[e2].append(e1)
        pid = -np.ones(12, np.int32)
        n = 0
        for e in range(12):
            if crossed[e] and pid[e] < 0:
                stack = [e]
                pid[e] = n
                while stack:
                    x = stack.pop()
                    for y in link[x]:
                        if pid[y] < 0:
                            pid[y] = n
                            stack.append(y)
                n += 1
        table[case] = pid
        counts[case] = n
    return table, counts


def preprocess(points, triangles, band, margin):
    """pamo/__init__.py:60-72 in numpy float32: (tris [m,3,3], tris_min [3],
    tris_max scalar, tris_mean [3])."""
    tris = np.asarray(points, np.float32)[np.asarray(triangles, np.int64)]
    tris_mean = tris.mean(axis=1).mean(axis=0)
    tris = tris - tris_mean
    tris_min = tris.min(0).min(0)
    tris = tris - tris_min
    tris_max = tris.max()
    tris = (tris / tris_max + np.float32(band)) / np.float32(margin)
    return tris.astype(np.float32), tris_min, tris_max, tris_mean


def _point_tri_d2(p, a, b, c):
    """Squared distance from points p to triangles (a, b, c), float64, the
    closest point by Voronoi regions (Ericson 2005, 5.1.5); dot products as
    x0 y0 + x1 y1 + x2 y2."""
    def dot(u, v):
        return u[..., 0] * v[..., 0] + u[..., 1] * v[..., 1] + u[..., 2] * v[..., 2]

    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = dot(ab, ap), dot(ac, ap)
    bp = p - b
    d3, d4 = dot(ab, bp), dot(ac, bp)
    cp = p - c
    d5, d6 = dot(ab, cp), dot(ac, cp)
    vc = d1 * d4 - d3 * d2
    vb = d5 * d2 - d1 * d6
    va = d3 * d6 - d5 * d4
    q = np.empty_like(p)
    done = np.zeros(p.shape[:-1], bool)

    def put(mask, val):
        m = mask & ~done
        q[m] = val[m]
        done[...] = done | m

    with np.errstate(divide="ignore", invalid="ignore"):
        put((d1 <= 0) & (d2 <= 0), np.broadcast_to(a, p.shape))
        put((d3 >= 0) & (d4 <= d3), np.broadcast_to(b, p.shape))
        v = d1 / (d1 - d3)
        put((vc <= 0) & (d1 >= 0) & (d3 <= 0), a + v[..., None] * ab)
        put((d6 >= 0) & (d5 <= d6), np.broadcast_to(c, p.shape))
        w = d2 / (d2 - d6)
        put((vb <= 0) & (d2 >= 0) & (d6 <= 0), a + w[..., None] * ac)
        w = (d4 - d3) / ((d4 - d3) + (d5 - d6))
        put((va <= 0) & ((d4 - d3) >= 0) & ((d5 - d6) >= 0), b + w[..., None] * (c - b))
        den = 1.0 / (va + vb + vc)
        v, w = vb * den, vc * den
        put(np.ones(p.shape[:-1], bool), a + v[..., None] * ab + w[..., None] * ac)
    dd = p - q
    return dot(dd, dd)


def unsigned_distance(tris, R, band):
    """Per sample min(band, distance to the nearest triangle), float64 [R,R,R]
    indexed [z, y, x].  Each triangle visits the samples of its box grown by
    `band` (those are the only ones it can bring below `band`)."""
    tris = np.asarray(tris, np.float64)
    d2 = np.full((R, R, R), band * band, np.float64)
    lo = np.floor((tris.min(1) - band) * R - 0.5).astype(np.int64)
    hi = np.ceil((tris.max(1) + band) * R - 0.5).astype(np.int64)
    lo = np.clip(lo, 0, R - 1)
    hi = np.clip(hi, 0, R - 1)
    for t in range(len(tris)):
        (x0, y0, z0), (x1, y1, z1) = lo[t], hi[t]
        zs, ys, xs = np.meshgrid(np.arange(z0, z1 + 1), np.arange(y0, y1 + 1), np.arange(x0, x1 + 1), indexing="ij")
        P = np.stack([(xs + 0.5) / R, (ys + 0.5) / R, (zs + 0.5) / R], -1)
        a, b, c = tris[t]
        dd = _point_tri_d2(P, a, b, c)
        sub = d2[z0:z1 + 1, y0:y1 + 1, x0:x1 + 1]
        np.minimum(sub, dd, out=sub)
    return np.sqrt(d2)


def signed_distance(tris, R, band):
    """The field stage 1 contours: flood-filled sign, minus 0.9 / R."""
    from scipy import ndimage

    ud = unsigned_distance(tris, R, band)
    free = ud > 0.5 / R
    lab, _ = ndimage.label(free, structure=ndimage.generate_binary_structure(3, 1))
    border = np.unique(np.concatenate([lab[0].ravel(), lab[-1].ravel(), lab[:, 0].ravel(), lab[:, -1].ravel(),
                                       lab[:, :, 0].ravel(), lab[:, :, -1].ravel()]))
    outside = np.isin(lab, border[border > 0])
    return np.where(outside, ud, -ud) - 0.9 / R


def dual_mc(d):
    """Quads and vertices (sample-index coordinates, float64) of the level set
    d = 0 of d [R,R,R] (indexed [z, y, x]), inside where d < 0."""
    R = d.shape[0]
    table, counts = patch_table()
    inside = d < 0
    C = R - 1
    # case of each cell [cz, cy, cx]
    case = np.zeros((C, C, C), np.int32)
    for c in range(8):
        ox, oy, oz = c & 1, (c >> 1) & 1, (c >> 2) & 1
        case |= inside[oz:oz + C, oy:oy + C, ox:ox + C].astype(np.int32) << c
    npatch = counts[case]
    first = np.concatenate([[0], np.cumsum(npatch.ravel())]).astype(np.int64)
    nv = int(first[-1])
    V = np.zeros((nv, 3), np.float64)
    # vertices: mean of the crossing points of each patch's edges, in edge order
    cz, cy, cx = np.nonzero(npatch)
    for z, y, x in zip(cz.tolist(), cy.tolist(), cx.tolist()):
        cs = case[z, y, x]
        base = first[(z * C + y) * C + x]
        acc = {}
        for e in range(12):
            p = table[cs, e]
            if p < 0:
                continue
            a, b = EDGE_CORNERS[e]
            pa = np.array([x + (a & 1), y + ((a >> 1) & 1), z + ((a >> 2) & 1)], np.float64)
            pb = np.array([x + (b & 1), y + ((b >> 1) & 1), z + ((b >> 2) & 1)], np.float64)
            da = d[int(pa[2]), int(pa[1]), int(pa[0])]
            db = d[int(pb[2]), int(pb[1]), int(pb[0])]
            t = da / (da - db)
            q = pa + t * (pb - pa)
            s, k = acc.get(p, (np.zeros(3), 0))
            acc[p] = (s + q, k + 1)
        for p, (s, k) in acc.items():
            V[base + p] = s / k
    # quads: crossed grid edges, axis by axis, lower sample in x-fastest order
    quads = []
    # (the edge's axis, the other two axes in cyclic order)
    axes = [(0, 1, 2), (1, 2, 0), (2, 0, 1)]
    edge_index = np.zeros((3, 8), np.int64)  # cube edge from (axis, lower corner)
    for e, (a, b) in enumerate(EDGE_CORNERS):
        ax = {1: 0, 2: 1, 4: 2}[b - a]
        edge_index[ax, a] = e
    for ax, bax, cax in axes:
        sl_lo = [slice(None)] * 3
        sl_hi = [slice(None)] * 3
        # arrays are [z, y, x]: axis k of (x, y, z) is array dimension 2 - k
        sl_lo[2 - ax] = slice(0, R - 1)
        sl_hi[2 - ax] = slice(1, R)
        cross = np.zeros((R, R, R), bool)
        cross[tuple(sl_lo)] = inside[tuple(sl_lo)] != inside[tuple(sl_hi)]
        # all four cells must exist: the other coordinates in [1, R - 2]
        for k in (bax, cax):
            sl = [slice(None)] * 3
            sl[2 - k] = 0
            cross[tuple(sl)] = False
            sl[2 - k] = R - 1
            cross[tuple(sl)] = False
        z, y, x = np.nonzero(cross)  # row-major: x fastest
        P = np.stack([x, y, z], 1)
        vs = []
        for ob, oc in ((0, 0), (-1, 0), (-1, -1), (0, -1)):
            cc = P.copy()
            cc[:, bax] += ob
            cc[:, cax] += oc
            lo_corner = (P[:, 0] - cc[:, 0]) + 2 * (P[:, 1] - cc[:, 1]) + 4 * (P[:, 2] - cc[:, 2])
            e = edge_index[ax, lo_corner]
            cs = case[cc[:, 2], cc[:, 1], cc[:, 0]]
            vs.append(first[(cc[:, 2] * C + cc[:, 1]) * C + cc[:, 0]] + table[cs, e])
        vs = np.stack(vs, 1)
        lower_inside = inside[z, y, x]
        vs = np.where(lower_inside[:, None], vs, vs[:, ::-1])
        quads.append(vs)
    quads = np.concatenate(quads) if quads else np.zeros((0, 4), np.int64)
    return V, np.array(quads, np.int64).reshape(-1, 4)


def split_quads(v, q):
    """pamo/__init__.py:95-118: per quad the split with the smaller largest
    corner cosine (float64 here); config-1 quads first."""
    v = np.asarray(v, np.float64)

    def maxcos(i0, i1, i2):
        a, b, c = v[i0], v[i1], v[i2]

        def cosang(p, r, s):
            u, w = r - p, s - p
            nu = np.sqrt(u[:, 0] * u[:, 0] + u[:, 1] * u[:, 1] + u[:, 2] * u[:, 2])
            nw = np.sqrt(w[:, 0] * w[:, 0] + w[:, 1] * w[:, 1] + w[:, 2] * w[:, 2])
            u = u / np.maximum(nu, 1e-12)[:, None]
            w = w / np.maximum(nw, 1e-12)[:, None]
            return u[:, 0] * w[:, 0] + u[:, 1] * w[:, 1] + u[:, 2] * w[:, 2]

        return np.maximum(np.maximum(cosang(a, b, c), cosang(b, c, a)), cosang(c, a, b))

    a1 = np.maximum(maxcos(q[:, 0], q[:, 1], q[:, 3]), maxcos(q[:, 1], q[:, 2], q[:, 3]))
    a2 = np.maximum(maxcos(q[:, 0], q[:, 1], q[:, 2]), maxcos(q[:, 0], q[:, 2], q[:, 3]))
    c1 = a1 < a2
    f1 = q[c1][:, [0, 1, 3, 1, 2, 3]].reshape(-1, 3)
    f2 = q[~c1][:, [0, 1, 2, 0, 2, 3]].reshape(-1, 3)
    return np.concatenate([f1, f2]).astype(np.int32)


def remesh(points, triangles, R=256):
    """Stage 1: (vertices float32 in the centred frame, faces int32, tris_mean)."""
    band = 3.0 / R
    margin = band * 2 + 1
    tris, tmin, tmax, tmean = preprocess(points, triangles, band, margin)
    d = signed_distance(tris, R, band)
    V, Q = dual_mc(d)
    x = (V + 0.5) / R
    v = ((x * margin - band) * np.float64(tmax) + tmin.astype(np.float64)).astype(np.float32)
    f = split_quads(v.astype(np.float64), Q)
    return v, f, tmean
