"""FP64 oracle of the stage-3 safe projection -- TEST INFRASTRUCTURE.

Only tests/ and bench.py's error report import this module; the product
(pamo_b200/safe_project.py + csrc/stage3.cu) never calls it.

A vectorised numpy restatement, in float64, of the reference's default
configuration (simp_cuda/safe_project/src/pamo_safe_project):
  * normalisation by the ground truth      processing.py:15-20,57-59
  * per step: closest point on the GT       geometry_kernels.py:82-94 (via energy.py:200-211)
  * 10 Newton iterations, each:             system.py:411-470
      contact detection (PT + EE, radius)   contact_detection.py:120-216
      energy / gradient / diagonal          energy.py, kernels/energy_kernels/*
      40 Jacobi-PCG iterations              cg_solver.py:46-158, solver_kernels.py:4-58
      step clamp                            solver_kernels.py:80-94
      additive CCD                          ccd_kernels.py:8-110
      10-halving line search                system.py:393-409, solver_kernels.py:61-77
The distance-type classification follows distance_kernels.py:76-228 and
:326-442.  Distance gradients are the gradients of the same distance
functions, written with the closest-point weights (envelope form); the
hinge Hessian follows Tamstorf & Grinspun, "Discrete bending forces and their
Jacobians" (2013), the formulation the reference implements
(hinge_energy.py:91-254).

Parity with the reference is unpinned: its Warp fork (wp.Bvh, wp.Mesh,
wp.spd_project_blocks) is not available.  The SPD projection is interpreted as
an eigenvalue clamp of the 9x9 matrix of the first three hinge vertices with
`spd_max_iters` cyclic Jacobi sweeps, the fourth vertex's rows refilled by
translation invariance (utils_kernels.py:20-39).
"""
from __future__ import annotations

import numpy as np

# distance types (defs.py)
PT, PP01, PP02, PE012, PP03, PE031, PE023 = range(7)
EE_PP02, EE_PP03, EE_PP12, EE_PP13, EE_PE023, EE_PE123, EE_PE201, EE_PE301, EE_EE = range(9)
BLOCK_PT, BLOCK_EE = 3, 4


class Stage3Config:
    """Defaults of config.py:6-73 that the default energy set uses."""

    def __init__(self):
        self.n_newton_iters = 10
        self.n_cg_iters = 40
        self.n_line_search_iters = 10
        self.d_hat = 1e-3
        self.coll_stiffness = 1e2
        self.contact_detection_radius = 1e-2
        self.ee_classify_thres = 1e-3
        self.ccd_slackness = 0.7
        self.ccd_thickness = 1e-6
        self.ccd_max_iters = 100
        self.spd_max_iters = 3
        self.elas_young_modulus = 1e-1
        self.elas_poisson_ratio = 0.0
        self.hinge_stiffness = 1e-2
        self.mesh2gt_dist_stiffness = 1e3
        self.min_angle_thres = 0.0
        self.max_blocks = 1 << 25


# ----------------------------------------------------------------- geometry
def normalization(gt_V):
    center = gt_V.mean(axis=0)
    extents = gt_V.max(axis=0) - gt_V.min(axis=0)
    scale = 1.0 / extents.max()
    return scale, -center * scale


def edges_unique(F):
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
    e = np.sort(e, axis=1)
    return np.unique(e, axis=0)



def _scatter_add(out, idx, vals):
    """out[idx[k]] += vals[k] for every k (np.add.at, through bincount per column)."""
    idx = np.asarray(idx).ravel()
    vals = np.asarray(vals, dtype=out.dtype)
    n = out.shape[0]
    if out.ndim == 1:
        out += np.bincount(idx, weights=vals.ravel(), minlength=n)[:n]
    else:
        v2 = vals.reshape(len(idx), -1)
        o2 = out.reshape(n, -1)
        for c in range(o2.shape[1]):
            o2[:, c] += np.bincount(idx, weights=v2[:, c], minlength=n)[:n]

def voronoi_areas(V, F):
    """Mixed Voronoi vertex areas (Meyer, Desbrun, Schroeder, Barr 2003): for a
    non-obtuse triangle each corner gets (|e_ij|^2 cot + |e_ik|^2 cot)/8; for an
    obtuse triangle the obtuse corner gets A/2 and the others A/4."""
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    ea, eb, ec = c - b, a - c, b - a  # opposite to a, b, c
    la2, lb2, lc2 = (ea * ea).sum(1), (eb * eb).sum(1), (ec * ec).sum(1)
    area = 0.5 * np.linalg.norm(np.cross(ec, -eb), axis=1)
    cos_a = -(eb * ec).sum(1) / np.sqrt(lb2 * lc2)
    cos_b = -(ec * ea).sum(1) / np.sqrt(lc2 * la2)
    cos_c = -(ea * eb).sum(1) / np.sqrt(la2 * lb2)
    with np.errstate(divide="ignore", invalid="ignore"):
        cot = lambda cs: cs / np.sqrt(np.maximum(1 - cs * cs, 0))
        cot_a, cot_b, cot_c = cot(cos_a), cot(cos_b), cot(cos_c)
    out = np.zeros(len(V))
    obtuse = (cos_a < 0) | (cos_b < 0) | (cos_c < 0)
    vor = np.stack([(lb2 * cot_b + lc2 * cot_c) / 8, (lc2 * cot_c + la2 * cot_a) / 8,
                    (la2 * cot_a + lb2 * cot_b) / 8], 1)
    mix = np.stack([np.where(cos_a < 0, area / 2, area / 4), np.where(cos_b < 0, area / 2, area / 4),
                    np.where(cos_c < 0, area / 2, area / 4)], 1)
    w = np.where(obtuse[:, None], mix, vor)
    for k in range(3):
        _scatter_add(out, F[:, k], w[:, k])
    return out


def internal_angles(V, F):
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]

    def ang(p, q, r):
        u, v = q - p, r - p
        cs = (u * v).sum(1) / (np.linalg.norm(u, axis=1) * np.linalg.norm(v, axis=1))
        return np.arccos(np.clip(cs, -1, 1))

    return np.stack([ang(a, b, c), ang(b, c, a), ang(c, a, b)], 1)


def hinges(F):
    """(i0, i1, i2, i3) per interior edge: face t0 holds the directed edge i1->i2
    with i1 < i2, face t1 holds i2->i1; i0 / i3 are their third vertices
    (hinge_energy.py:21-57)."""
    F = np.asarray(F)
    rows = []
    for k in range(3):
        rows.append(np.stack([F[:, k], F[:, (k + 1) % 3], F[:, (k + 2) % 3]], 1))
    D = np.concatenate(rows)  # (src, dst, opposite)
    fwd = D[D[:, 0] < D[:, 1]]
    bwd = D[D[:, 0] > D[:, 1]]
    kf = fwd[:, 0].astype(np.int64) * (F.max() + 1) + fwd[:, 1]
    kb = bwd[:, 1].astype(np.int64) * (F.max() + 1) + bwd[:, 0]
    ob = np.argsort(kb)
    pos = np.searchsorted(kb[ob], kf)
    ok = (pos < len(kb)) & (kb[ob][np.minimum(pos, len(kb) - 1)] == kf)
    fwd = fwd[ok]
    opp = bwd[ob][pos[ok]][:, 2]
    H = np.stack([fwd[:, 2], fwd[:, 0], fwd[:, 1], opp], 1)
    order = np.lexsort((H[:, 2], H[:, 1]))
    return H[order]


def hinge_angle(x0, x1, x2, x3):
    e12 = x2 - x1
    e12 = e12 / np.linalg.norm(e12, axis=-1, keepdims=True)
    n1 = np.cross(e12, x0 - x1)
    n1 /= np.linalg.norm(n1, axis=-1, keepdims=True)
    n2 = np.cross(x3 - x1, e12)
    n2 /= np.linalg.norm(n2, axis=-1, keepdims=True)
    c = (n1 * n2).sum(-1)
    s = (np.cross(n1, n2) * e12).sum(-1)
    return np.arctan2(s, c)


# --------------------------------------------------- closest points (stage 3 target)
def point_triangle_closest(p, a, b, c):
    """Closest point on triangles (a,b,c) to points p (Ericson, Real-Time
    Collision Detection, 5.1.5), all arrays [n,3]."""
    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = (ab * ap).sum(1), (ac * ap).sum(1)
    bp = p - b
    d3, d4 = (ab * bp).sum(1), (ac * bp).sum(1)
    cp = p - c
    d5, d6 = (ab * cp).sum(1), (ac * cp).sum(1)
    vc = d1 * d4 - d3 * d2
    vb = d5 * d2 - d1 * d6
    va = d3 * d6 - d5 * d4
    out = np.empty_like(p)
    done = np.zeros(len(p), bool)

    def put(mask, val):
        nonlocal done
        m = mask & ~done
        out[m] = val[m] if val.ndim == 2 else val
        done |= m

    put((d1 <= 0) & (d2 <= 0), a)
    put((d3 >= 0) & (d4 <= d3), b)
    with np.errstate(divide="ignore", invalid="ignore"):
        v = d1 / (d1 - d3)
        put((vc <= 0) & (d1 >= 0) & (d3 <= 0), a + v[:, None] * ab)
        put((d6 >= 0) & (d5 <= d6), c)
        w = d2 / (d2 - d6)
        put((vb <= 0) & (d2 >= 0) & (d6 <= 0), a + w[:, None] * ac)
        w = (d4 - d3) / ((d4 - d3) + (d5 - d6))
        put((va <= 0) & ((d4 - d3) >= 0) & ((d5 - d6) >= 0), b + w[:, None] * (c - b))
        denom = 1.0 / (va + vb + vc)
        v = vb * denom
        w = vc * denom
    put(np.ones(len(p), bool), a + v[:, None] * ab + w[:, None] * ac)
    return out


def closest_points_on_mesh(P, V, F, chunk=2048):
    """Exact closest point on the triangle mesh (V,F) for every point of P."""
    from scipy.spatial import cKDTree

    cen = V[F].mean(1)
    rad = np.max(np.linalg.norm(V[F] - cen[:, None], axis=2), axis=1)
    tree = cKDTree(cen)
    rmax = rad.max()
    out = np.empty_like(P)
    d_near, _ = tree.query(P)
    for s in range(0, len(P), chunk):
        Pc = P[s:s + chunk]
        cands = tree.query_ball_point(Pc, d_near[s:s + chunk] + rmax)
        for k, (p, cand) in enumerate(zip(Pc, cands)):
            cand = np.asarray(cand)
            tri = V[F[cand]]
            q = point_triangle_closest(np.repeat(p[None], len(cand), 0), tri[:, 0], tri[:, 1], tri[:, 2])
            d = np.linalg.norm(q - p, axis=1)
            out[s + k] = q[np.argmin(d)]
    return out


# -------------------------------------------------------- pair distances
def _dot(a, b):
    return (a * b).sum(-1)


def _norm(a):
    return np.linalg.norm(a, axis=-1)


def pp_distance(x0, x1):
    return _norm(x1 - x0)


def pe_distance(x0, x1, x2):
    return _norm(np.cross(x1 - x0, x2 - x0)) / _norm(x1 - x2)


def pt_distance(x0, x1, x2, x3):
    n = np.cross(x2 - x1, x3 - x1)
    n = n / _norm(n)[..., None]
    return np.abs(_dot(x0 - x1, n))


def ee_distance(x0, x1, x2, x3):
    n = np.cross(x1 - x0, x3 - x2)
    n = n / _norm(n)[..., None]
    return np.abs(_dot(x0 - x2, n))


def pt_classify(x0, x1, x2, x3):
    """distance_kernels.py:76-228, vectorised."""
    n_ = len(x0)
    out = np.full(n_, -1, np.int64)
    x10, x12, x13 = x0 - x1, x2 - x1, x3 - x1
    cr = np.cross(x12, x13)
    area_sq = _dot(cr, cr)
    degen = (area_sq <= 1e-6 * (_dot(x12, x12) * _dot(x13, x13))) | (area_sq <= 1e-16)
    d1, d2, d3 = _norm(x10), _norm(x0 - x2), _norm(x0 - x3)
    dg = np.where(d1 < d2, np.where(d1 < d3, PP01, PP03), np.where(d2 < d3, PP02, PP03))
    out[degen] = dg[degen]
    with np.errstate(divide="ignore", invalid="ignore"):
        n = cr / np.sqrt(area_sq)[:, None]
    proj = x0 - _dot(n, x10)[:, None] * n
    x10p, x20p, x30p = proj - x1, proj - x2, proj - x3
    a00, a01, a11 = _dot(x12, x12), _dot(x12, x13), _dot(x13, x13)
    b0, b1 = _dot(x10p, x12), _dot(x10p, x13)
    det = a00 * a11 - a01 * a01
    beta = b0 * a11 - b1 * a01
    gamma = a00 * b1 - b0 * a01
    alpha = det - beta - gamma
    neg = (alpha < 0).astype(int) + (beta < 0) + (gamma < 0)
    live = ~degen
    m0 = live & (neg == 0)
    out[m0] = PT
    m1 = live & (neg == 1)
    # one negative coordinate: the edge region opposite to it
    x23, x20 = x3 - x2, x0 - x2
    dr = _dot(x23, x20)
    t_a = np.where(dr < 0, PP02, np.where(dr > _dot(x23, x23), PP03, PE023))
    x31, x30 = x1 - x3, x0 - x3
    dr = _dot(x31, x30)
    t_b = np.where(dr < 0, PP03, np.where(dr > _dot(x31, x31), PP01, PE031))
    dr = _dot(x12, x10p)
    t_c = np.where(dr < 0, PP01, np.where(dr > _dot(x12, x12), PP02, PE012))
    t1 = np.where(alpha < 0, t_a, np.where(beta < 0, t_b, t_c))
    out[m1] = t1[m1]
    m2 = live & (neg >= 2)
    # two negative coordinates: vertex region of the non-negative one
    dot12, dot13 = _dot(x12, x10p), _dot(x13, x10p)
    va = np.where((dot12 > 0) & (dot13 <= 0), np.where(_dot(x12, x20p) > 0, PP02, PE012),
                  np.where((dot13 > 0) & (dot12 <= 0), np.where(_dot(x13, x30p) > 0, PP03, PE031), PP01))
    x21 = x1 - x2
    dot23, dot21 = _dot(x23, x20p), _dot(x21, x20p)
    vb = np.where((dot23 > 0) & (dot21 <= 0), np.where(_dot(x23, x30p) > 0, PP03, PE023),
                  np.where((dot21 > 0) & (dot23 <= 0), np.where(_dot(x21, x10p) > 0, PP01, PE012), PP02))
    x32 = x2 - x3
    dot31, dot32 = _dot(x31, x30p), _dot(x32, x30p)
    vc = np.where((dot31 > 0) & (dot32 <= 0), np.where(_dot(x31, x10p) > 0, PP01, PE031),
                  np.where((dot32 > 0) & (dot31 <= 0), np.where(_dot(x32, x20p) > 0, PP02, PE023), PP03))
    t2 = np.where(alpha >= 0, va, np.where(beta >= 0, vb, vc))
    out[m2] = t2[m2]
    return out


def ee_classify(x0, x1, x2, x3, sin_thres):
    """distance_kernels.py:326-442, vectorised."""
    e0, e1 = x0 - x1, x2 - x3
    e0_sq, e1_sq = _dot(e0, e0), _dot(e1, e1)
    a00, a01, a10, a11 = e0_sq, -_dot(e0, e1), _dot(e0, e1), -e1_sq
    b0, b1 = _dot(x3 - x1, e0), _dot(x3 - x1, e1)
    mu0 = -(b0 * a11 - b1 * a01)
    mu1 = -(a00 * b1 - a10 * b0)
    det = -(a00 * a11 - a01 * a10)
    with np.errstate(divide="ignore", invalid="ignore"):
        s = _norm(np.cross(e0 / _norm(e0)[:, None], e1 / _norm(e1)[:, None]))
    inside = (mu0 >= 0) & (mu0 <= det) & (mu1 >= 0) & (mu1 <= det) & (s >= sin_thres) & (e0_sq > 1e-15) & (
        e1_sq > 1e-15)
    best = np.full(len(x0), 1e9)
    typ = np.full(len(x0), -1, np.int64)

    def consider(d, t):
        nonlocal best, typ
        m = d < best
        best = np.where(m, d, best)
        typ = np.where(m, t, typ)

    def endpoint(p, a, b, t_pp_a, t_pp_b, t_pe, ev, ev_sq, ref):
        tt = _dot(p - ref, ev)
        d_a = pp_distance(p, a)
        d_b = pp_distance(p, b)
        with np.errstate(divide="ignore", invalid="ignore"):
            d_e = pe_distance(p, a, b)
        d = np.where(tt >= ev_sq, d_a, np.where(tt <= 0, d_b, d_e))
        t = np.where(tt >= ev_sq, t_pp_a, np.where(tt <= 0, t_pp_b, t_pe))
        return d, t

    consider(*endpoint(x0, x2, x3, EE_PP02, EE_PP03, EE_PE023, e1, e1_sq, x3))
    consider(*endpoint(x1, x2, x3, EE_PP12, EE_PP13, EE_PE123, e1, e1_sq, x3))
    consider(*endpoint(x2, x0, x1, EE_PP02, EE_PP12, EE_PE201, e0, e0_sq, x1))
    consider(*endpoint(x3, x0, x1, EE_PP03, EE_PP13, EE_PE301, e0, e0_sq, x1))
    return np.where(inside, EE_EE, typ)


# For each type: the participating local vertices and the distance kind.
PT_TYPES = {PT: ("pt", (0, 1, 2, 3)), PP01: ("pp", (0, 1)), PP02: ("pp", (0, 2)), PE012: ("pe", (0, 1, 2)),
            PP03: ("pp", (0, 3)), PE031: ("pe", (0, 3, 1)), PE023: ("pe", (0, 2, 3))}
EE_TYPES = {EE_PP02: ("pp", (0, 2)), EE_PP03: ("pp", (0, 3)), EE_PP12: ("pp", (1, 2)), EE_PP13: ("pp", (1, 3)),
            EE_PE023: ("pe", (0, 2, 3)), EE_PE123: ("pe", (1, 2, 3)), EE_PE201: ("pe", (2, 0, 1)),
            EE_PE301: ("pe", (3, 0, 1)), EE_EE: ("ee", (0, 1, 2, 3))}


def pair_distance_grad(X, block_kind, sub_type, want_grad=True):
    """Distance and d(distance)/dx (4 x 3 per block) for classified blocks.
    X: [n,4,3] positions, block_kind: BLOCK_PT/BLOCK_EE, sub_type per block."""
    n = len(X)
    d = np.full(n, 1e9)
    G = np.zeros((n, 4, 3))
    table = {BLOCK_PT: PT_TYPES, BLOCK_EE: EE_TYPES}
    for bk in (BLOCK_PT, BLOCK_EE):
        for t, (kind, idx) in table[bk].items():
            m = (block_kind == bk) & (sub_type == t)
            if not m.any():
                continue
            P = [X[m, i] for i in idx]
            if kind == "pp":
                diff = P[0] - P[1]
                dd = _norm(diff)
                u = diff / dd[:, None]
                d[m] = dd
                g = np.zeros((m.sum(), 4, 3))
                g[:, idx[0]] = u
                g[:, idx[1]] = -u
            elif kind == "pe":
                x0, x1, x2 = P
                e = x2 - x1
                t_ = _dot(x0 - x1, e) / _dot(e, e)
                c = x1 + t_[:, None] * e
                diff = x0 - c
                dd = pe_distance(x0, x1, x2)
                u = diff / _norm(diff)[:, None]
                d[m] = dd
                g = np.zeros((m.sum(), 4, 3))
                g[:, idx[0]] = u
                g[:, idx[1]] = -(1 - t_)[:, None] * u
                g[:, idx[2]] = -t_[:, None] * u
            elif kind == "pt":
                x0, x1, x2, x3 = P
                nrm = np.cross(x2 - x1, x3 - x1)
                nrm /= _norm(nrm)[:, None]
                sd = _dot(x0 - x1, nrm)
                dd = np.abs(sd)
                u = np.sign(sd)[:, None] * nrm
                proj = x0 - sd[:, None] * nrm
                a00, a01, a11 = _dot(x2 - x1, x2 - x1), _dot(x2 - x1, x3 - x1), _dot(x3 - x1, x3 - x1)
                b0, b1 = _dot(proj - x1, x2 - x1), _dot(proj - x1, x3 - x1)
                det = a00 * a11 - a01 * a01
                be = (b0 * a11 - b1 * a01) / det
                ga = (a00 * b1 - b0 * a01) / det
                al = 1 - be - ga
                d[m] = dd
                g = np.zeros((m.sum(), 4, 3))
                g[:, 0] = u
                g[:, 1] = -al[:, None] * u
                g[:, 2] = -be[:, None] * u
                g[:, 3] = -ga[:, None] * u
            else:  # ee
                x0, x1, x2, x3 = P
                nrm = np.cross(x1 - x0, x3 - x2)
                nrm /= _norm(nrm)[:, None]
                sd = _dot(x0 - x2, nrm)
                dd = np.abs(sd)
                u = np.sign(sd)[:, None] * nrm
                # closest-point parameters of the two lines
                e0, e1, w0 = x1 - x0, x3 - x2, x0 - x2
                a, b, c = _dot(e0, e0), _dot(e0, e1), _dot(e1, e1)
                dq, eq = _dot(e0, w0), _dot(e1, w0)
                den = a * c - b * b
                s_ = (b * eq - c * dq) / den
                t_ = (a * eq - b * dq) / den
                d[m] = dd
                g = np.zeros((m.sum(), 4, 3))
                g[:, 0] = (1 - s_)[:, None] * u
                g[:, 1] = s_[:, None] * u
                g[:, 2] = -(1 - t_)[:, None] * u
                g[:, 3] = -t_[:, None] * u
            G[m] = g
    return d, G


# ------------------------------------------------------------------ system
class Stage3Oracle:
    """Holds one registered mesh and runs steps (system.py Stage3System)."""

    def __init__(self, config: Stage3Config | None = None, dtype=np.float64):
        self.c = config or Stage3Config()
        self.dt = dtype

    def register(self, V_gt, F_gt, V, F):
        c = self.c
        self.F = np.asarray(F, np.int64)
        self.q = np.asarray(V, self.dt).copy()
        self.q_rest = self.q.copy()
        self.V_gt = np.asarray(V_gt, np.float64)
        self.F_gt = np.asarray(F_gt, np.int64)
        self.E = edges_unique(self.F)
        self.H = hinges(self.F)
        ang = internal_angles(np.asarray(V, np.float64), self.F)
        self.do_nothing = np.min(ang) * 180 / np.pi <= c.min_angle_thres
        self.w = voronoi_areas(np.asarray(V, np.float64), self.F).astype(self.dt)
        X = self.q_rest
        x01 = X[self.F[:, 1]] - X[self.F[:, 0]]
        x02 = X[self.F[:, 2]] - X[self.F[:, 0]]
        self.area = 0.5 * _norm(np.cross(x01, x02))
        Dm = self._local(x01, x02)
        self.inv_Dm = np.linalg.inv(Dm)
        h = self.H
        self.rest_angle = hinge_angle(X[h[:, 0]], X[h[:, 1]], X[h[:, 2]], X[h[:, 3]])
        self.rest_elen = _norm(X[h[:, 1]] - X[h[:, 2]])
        self.mu = c.elas_young_modulus / (2 * (1 + c.elas_poisson_ratio))
        self.la = c.elas_young_modulus * c.elas_poisson_ratio / (
            (1 + c.elas_poisson_ratio) * (1 - 2 * c.elas_poisson_ratio))
        self.radius = c.contact_detection_radius
        self.blocks = np.zeros((0, 4), np.int64)
        self.kinds = np.zeros(0, np.int64)
        # per Newton iteration: energy at the iterate, energy after the line
        # search, CCD step, last halving tried, contact blocks, blocks within d_hat
        self.trace = []
        self.nact = 0

    @staticmethod
    def _frame(x01, x02):
        b1 = x01 / _norm(x01)[:, None]
        b2 = x02 - _dot(x02, b1)[:, None] * b1
        b2 /= _norm(b2)[:, None]
        return b1, b2

    def _local(self, x01, x02, frame=None):
        b1, b2 = frame if frame is not None else self._frame(x01, x02)
        D = np.empty((len(x01), 2, 2))
        D[:, 0, 0], D[:, 0, 1] = _dot(b1, x01), _dot(b1, x02)
        D[:, 1, 0], D[:, 1, 1] = _dot(b2, x01), _dot(b2, x02)
        return D

    # ---------------------------------------------------------------- target
    def update_target(self):
        self.target = closest_points_on_mesh(np.asarray(self.q, np.float64), self.V_gt, self.F_gt).astype(self.dt)

    # ------------------------------------------------------------- contacts
    def detect(self):
        c = self.c
        from scipy.spatial import cKDTree

        q = self.q
        thr = 2.0 * self.radius + c.d_hat
        F, E = self.F, self.E
        # point-triangle: candidate pairs with overlapping boxes, then distance
        lo, hi = q[F].min(1), q[F].max(1)
        cen = 0.5 * (lo + hi)
        half = 0.5 * (hi - lo)
        tree = cKDTree(cen)
        rmax = np.max(_norm(half)) + thr * np.sqrt(3)
        cand = tree.query_ball_point(q, rmax)
        pv = np.repeat(np.arange(len(q)), [len(x) for x in cand])
        pt = np.concatenate([np.asarray(x, np.int64) for x in cand]) if len(pv) else np.zeros(0, np.int64)
        ok = np.all((q[pv] >= lo[pt] - thr) & (q[pv] <= hi[pt] + thr), axis=1)
        ok &= ~np.any(F[pt] == pv[:, None], axis=1)
        pv, pt = pv[ok], pt[ok]
        X = np.stack([q[pv], q[F[pt, 0]], q[F[pt, 1]], q[F[pt, 2]]], 1)
        ty = pt_classify(X[:, 0], X[:, 1], X[:, 2], X[:, 3])
        d, _ = pair_distance_grad(X, np.full(len(X), BLOCK_PT), ty, want_grad=False)
        keep = d <= thr
        b_pt = np.stack([pv[keep], F[pt[keep], 0], F[pt[keep], 1], F[pt[keep], 2]], 1)
        # edge-edge
        elo, ehi = np.minimum(q[E[:, 0]], q[E[:, 1]]), np.maximum(q[E[:, 0]], q[E[:, 1]])
        ecen = 0.5 * (elo + ehi)
        etree = cKDTree(ecen)
        er = np.max(_norm(0.5 * (ehi - elo)))
        pairs = etree.query_pairs(2 * er + thr * np.sqrt(3) + 1e-12, output_type="ndarray")
        if len(pairs):
            a, b = pairs[:, 0], pairs[:, 1]
            a, b = np.minimum(a, b), np.maximum(a, b)
            ok = np.all((ehi[a] + thr >= elo[b] - 0) & (ehi[b] >= elo[a] - thr), axis=1)
            ok = np.all((elo[a] - thr <= ehi[b]) & (elo[b] <= ehi[a] + thr), axis=1)
            sh = (E[a, 0] == E[b, 0]) | (E[a, 0] == E[b, 1]) | (E[a, 1] == E[b, 0]) | (E[a, 1] == E[b, 1])
            ok &= ~sh
            a, b = a[ok], b[ok]
            X = np.stack([q[E[a, 0]], q[E[a, 1]], q[E[b, 0]], q[E[b, 1]]], 1)
            ty = ee_classify(X[:, 0], X[:, 1], X[:, 2], X[:, 3], c.ee_classify_thres)
            d, _ = pair_distance_grad(X, np.full(len(X), BLOCK_EE), ty, want_grad=False)
            keep = d <= thr
            b_ee = np.stack([E[a[keep], 0], E[a[keep], 1], E[b[keep], 0], E[b[keep], 1]], 1)
        else:
            b_ee = np.zeros((0, 4), np.int64)
        self.blocks = np.concatenate([b_pt, b_ee]).astype(np.int64)
        self.kinds = np.concatenate([np.full(len(b_pt), BLOCK_PT), np.full(len(b_ee), BLOCK_EE)])
        if len(self.blocks) > c.max_blocks:
            self.radius /= 2.0
            return self.detect()
        return len(self.blocks)

    def _classify_blocks(self, q):
        X = q[self.blocks]
        ty = np.where(self.kinds == BLOCK_PT, pt_classify(X[:, 0], X[:, 1], X[:, 2], X[:, 3]),
                      ee_classify(X[:, 0], X[:, 1], X[:, 2], X[:, 3], self.c.ee_classify_thres))
        return X, ty

    # ---------------------------------------------------------------- energy
    @staticmethod
    def barrier(d, dh):
        return np.where(d < dh, -(d - dh) ** 2 * np.log(d / dh), 0.0)

    @staticmethod
    def barrier_d1(d, dh):
        t = d - dh
        return np.where(d < dh, -2 * t * np.log(d / dh) - t * t / d, 0.0)

    @staticmethod
    def barrier_d2(d, dh):
        return np.where(d < dh, -2 * np.log(d / dh) - 2 * (d - dh) / d - 1 + dh * dh / (d * d), 0.0)

    def energy(self, q):
        c = self.c
        e_dist = 0.5 * np.sum(_norm(q - self.target) ** 2 * self.w * c.mesh2gt_dist_stiffness)
        e_el = self._elastic_energy(q)
        h = self.H
        th = hinge_angle(q[h[:, 0]], q[h[:, 1]], q[h[:, 2]], q[h[:, 3]])
        e_h = np.sum(0.5 * c.hinge_stiffness * (th - self.rest_angle) ** 2 * self.rest_elen)
        e_c = 0.0
        if len(self.blocks):
            X, ty = self._classify_blocks(q)
            d, _ = pair_distance_grad(X, self.kinds, ty)
            with np.errstate(divide="ignore", invalid="ignore"):
                e_c = np.sum(np.where(d < c.d_hat, self.barrier(d, c.d_hat), 0.0)) * c.coll_stiffness
        return e_dist + e_el + e_h + e_c

    def _elastic_F(self, q):
        F = self.F
        x01 = q[F[:, 1]] - q[F[:, 0]]
        x02 = q[F[:, 2]] - q[F[:, 0]]
        fr = self._frame(x01, x02)
        Ds = self._local(x01, x02, fr)
        return Ds @ self.inv_Dm, fr, Ds

    def _elastic_energy(self, q):
        Fm, _, _ = self._elastic_F(q)
        E = 0.5 * (np.transpose(Fm, (0, 2, 1)) @ Fm - np.eye(2))
        trE = np.trace(E, axis1=1, axis2=2)
        psi = self.mu * np.sum(E * E, axis=(1, 2)) + 0.5 * self.la * trE * trE
        return np.sum(self.area * psi)

    def diff(self, q):
        """(grad with coefficient -1, hess diagonal); also caches the Hessian parts."""
        c = self.c
        n = len(q)
        g = np.zeros((n, 3))
        dg = np.zeros((n, 3))
        wk = self.w * c.mesh2gt_dist_stiffness
        g += -(q - self.target) * wk[:, None]
        dg += wk[:, None]
        # elastic (no diagonal contribution, energy.py:423-446)
        Fm, (b1, b2), _ = self._elastic_F(q)
        E = 0.5 * (np.transpose(Fm, (0, 2, 1)) @ Fm - np.eye(2))
        trE = np.trace(E, axis1=1, axis2=2)
        P = Fm @ (2 * self.mu * E + self.la * trE[:, None, None] * np.eye(2))
        Hm = -1.0 * self.area[:, None, None] * P @ np.transpose(self.inv_Dm, (0, 2, 1))
        f1 = Hm[:, 0, 0, None] * b1 + Hm[:, 1, 0, None] * b2
        f2 = Hm[:, 0, 1, None] * b1 + Hm[:, 1, 1, None] * b2
        f0 = -f1 - f2
        for k, f in ((0, f0), (1, f1), (2, f2)):
            _scatter_add(g, self.F[:, k], f)
        # hinge
        Hb, gh = self._hinge_blocks(q)
        for k in range(4):
            _scatter_add(g, self.H[:, k], -gh[:, k])
            _scatter_add(dg, self.H[:, k], np.stack([Hb[:, k, k, i, i] for i in range(3)], 1))
        self.hinge_blocks = spd_project(Hb, c.spd_max_iters)
        # collision (Gauss-Newton)
        self.coll = None
        self.nact = 0
        if len(self.blocks):
            X, ty = self._classify_blocks(q)
            d, G = pair_distance_grad(X, self.kinds, ty)
            act = d < c.d_hat
            self.nact = int(act.sum())
            with np.errstate(divide="ignore", invalid="ignore"):
                b1c = self.barrier_d1(d, c.d_hat) * c.coll_stiffness
                b2c = self.barrier_d2(d, c.d_hat) * c.coll_stiffness
            b1c = np.where(act, b1c, 0.0)
            b2c = np.where(act, b2c, 0.0)
            for k in range(4):
                _scatter_add(g, self.blocks[:, k], -G[:, k] * b1c[:, None])
                _scatter_add(dg, self.blocks[:, k], b2c[:, None] * G[:, k] ** 2)
            self.coll = (G, b2c)
        return g, dg

    def _hinge_blocks(self, q):
        """Energy gradient dE/dx (per hinge, 4 x 3) and Hessian (4 x 4 x 3 x 3)
        of 0.5 k (theta - theta0)^2 l0 (Tamstorf & Grinspun 2013)."""
        c = self.c
        h = self.H
        x0, x1, x2, x3 = q[h[:, 0]], q[h[:, 1]], q[h[:, 2]], q[h[:, 3]]
        e0, e1, e2 = x2 - x1, x0 - x2, x0 - x1
        e1_, e2_ = x3 - x2, x3 - x1
        l0 = _norm(e0)
        u0, u1, u2 = e0 / l0[:, None], e1 / _norm(e1)[:, None], e2 / _norm(e2)[:, None]
        u1_, u2_ = e1_ / _norm(e1_)[:, None], e2_ / _norm(e2_)[:, None]
        ca1, ca2 = _dot(u2, u0), -_dot(u1, u0)
        ca1_, ca2_ = _dot(u2_, u0), -_dot(u1_, u0)
        h0 = _norm(np.cross(e1, e2)) / l0
        h1 = _norm(np.cross(e0, e2)) / _norm(e1)
        h2 = _norm(np.cross(e0, e1)) / _norm(e2)
        h0_ = _norm(np.cross(e1_, e2_)) / l0
        h1_ = _norm(np.cross(e0, e2_)) / _norm(e1_)
        h2_ = _norm(np.cross(e0, e1_)) / _norm(e2_)
        n = np.cross(e0, e2)
        n /= _norm(n)[:, None]
        n_ = np.cross(e2_, e0)
        n_ /= _norm(n_)[:, None]
        th = np.arctan2(_dot(np.cross(n, n_), e0) / l0, _dot(n, n_))
        dE = c.hinge_stiffness * (th - self.rest_angle) * self.rest_elen
        d2E = c.hinge_stiffness * self.rest_elen
        g0 = -n / h0[:, None]
        g3 = -n_ / h0_[:, None]
        g1 = n * (ca2 / h1)[:, None] + n_ * (ca2_ / h1_)[:, None]
        g2 = n * (ca1 / h2)[:, None] + n_ * (ca1_ / h2_)[:, None]
        gt = np.stack([g0, g1, g2, g3], 1)
        grad = dE[:, None, None] * gt

        def unit(v):
            return v / _norm(v)[:, None]

        m0, m1, m2 = unit(np.cross(e0, n)), unit(np.cross(e1, n)), unit(np.cross(n, e2))
        m0_, m1_, m2_ = unit(np.cross(n_, e0)), unit(np.cross(n_, e1_)), unit(np.cross(e2_, n_))
        out = lambda a, b: a[:, :, None] * b[:, None, :]
        M0, M1, M2 = out(n, m0), out(n, m1), out(n, m2)
        M0_, M1_, M2_ = out(n_, m0_), out(n_, m1_), out(n_, m2_)
        T = lambda A: np.transpose(A, (0, 2, 1))
        sym = lambda A: A + T(A)
        s_ = lambda v: v[:, None, None]
        N0, N0_ = M0 / s_(l0 * l0), M0_ / s_(l0 * l0)
        P10, P11, P12 = s_(ca1 / (h1 * h0)) * T(M0), s_(ca1 / (h1 * h1)) * T(M1), s_(ca1 / (h1 * h2)) * T(M2)
        P20, P21, P22 = s_(ca2 / (h2 * h0)) * T(M0), s_(ca2 / (h2 * h1)) * T(M1), s_(ca2 / (h2 * h2)) * T(M2)
        P10_, P11_, P12_ = (s_(ca1_ / (h1_ * h0_)) * T(M0_), s_(ca1_ / (h1_ * h1_)) * T(M1_),
                            s_(ca1_ / (h1_ * h2_)) * T(M2_))
        P20_, P21_, P22_ = (s_(ca2_ / (h2_ * h0_)) * T(M0_), s_(ca2_ / (h2_ * h1_)) * T(M1_),
                            s_(ca2_ / (h2_ * h2_)) * T(M2_))
        Q0, Q1, Q2 = M0 / s_(h0 * h0), M1 / s_(h0 * h1), M2 / s_(h0 * h2)
        Q0_, Q1_, Q2_ = M0_ / s_(h0_ * h0_), M1_ / s_(h0_ * h1_), M2_ / s_(h0_ * h2_)
        B = np.zeros((len(h), 4, 4, 3, 3))
        a, k2 = s_(dE), s_(d2E)
        B[:, 0, 0] = -sym(Q0) * a + k2 * out(g0, g0)
        B[:, 3, 3] = -sym(Q0_) * a + k2 * out(g3, g3)
        B[:, 1, 1] = (sym(P11) - N0 + sym(P11_) - N0_) * a + k2 * out(g1, g1)
        B[:, 2, 2] = (sym(P22) - N0 + sym(P22_) - N0_) * a + k2 * out(g2, g2)
        B[:, 1, 0] = (P10 - Q1) * a + k2 * out(g1, g0)
        B[:, 2, 0] = (P20 - Q2) * a + k2 * out(g2, g0)
        B[:, 1, 3] = (P10_ - Q1_) * a + k2 * out(g1, g3)
        B[:, 2, 3] = (P20_ - Q2_) * a + k2 * out(g2, g3)
        B[:, 1, 2] = (P12 + T(P21) + N0 + P12_ + T(P21_) + N0_) * a + k2 * out(g1, g2)
        B[:, 0, 3] = k2 * out(g0, g3)
        B[:, 0, 1], B[:, 0, 2] = T(B[:, 1, 0]), T(B[:, 2, 0])
        B[:, 3, 1], B[:, 3, 2] = T(B[:, 1, 3]), T(B[:, 2, 3])
        B[:, 2, 1], B[:, 3, 0] = T(B[:, 1, 2]), T(B[:, 0, 3])
        return B, grad

    def hess_dx(self, q, dx):
        c = self.c
        out = dx * (self.w * c.mesh2gt_dist_stiffness)[:, None]
        # elastic: product with the frame held fixed (elastic_energy.py:152-220)
        F = self.F
        Fm, (b1, b2), _ = self._elastic_F(q)
        dx01 = dx[F[:, 1]] - dx[F[:, 0]]
        dx02 = dx[F[:, 2]] - dx[F[:, 0]]
        dDs = self._local(dx01, dx02, (b1, b2))
        dF = dDs @ self.inv_Dm
        E = 0.5 * (np.transpose(Fm, (0, 2, 1)) @ Fm - np.eye(2))
        trE = np.trace(E, axis1=1, axis2=2)
        dE = 0.5 * (np.transpose(dF, (0, 2, 1)) @ Fm + np.transpose(Fm, (0, 2, 1)) @ dF)
        trdE = np.trace(dE, axis1=1, axis2=2)
        I = np.eye(2)
        dP = dF @ (2 * self.mu * E + self.la * trE[:, None, None] * I) + Fm @ (
            2 * self.mu * dE + self.la * trdE[:, None, None] * I)
        dH = self.area[:, None, None] * dP @ np.transpose(self.inv_Dm, (0, 2, 1))
        df1 = dH[:, 0, 0, None] * b1 + dH[:, 1, 0, None] * b2
        df2 = dH[:, 0, 1, None] * b1 + dH[:, 1, 1, None] * b2
        df0 = -df1 - df2
        for k, f in ((0, df0), (1, df1), (2, df2)):
            _scatter_add(out, F[:, k], f)
        # hinge blocks
        Hb = self.hinge_blocks
        dxh = dx[self.H]  # [nh,4,3]
        contrib = np.einsum("hijab,hjb->hia", Hb, dxh)
        for k in range(4):
            _scatter_add(out, self.H[:, k], contrib[:, k])
        # collision Gauss-Newton
        if self.coll is not None:
            G, b2c = self.coll
            s = np.einsum("hjb,hjb->h", G, dx[self.blocks])
            for k in range(4):
                _scatter_add(out, self.blocks[:, k], G[:, k] * (b2c * s)[:, None])
        return out

    # ---------------------------------------------------------------- solver
    def cg(self, g, dg):
        c = self.c
        p = np.zeros_like(g)
        r = g.copy()
        z = r / (dg + 1e-6)
        v = z.copy()
        zr = np.sum(z * r)
        for _ in range(c.n_cg_iters):
            Av = self.hess_dx(self.q, v)
            vAv = np.sum(v * Av)
            zr_last = zr
            if vAv > 1e-16:
                alpha = zr_last / vAv
                p = p + alpha * v
                r = r - alpha * Av
            with np.errstate(divide="ignore", invalid="ignore"):
                z = r / dg
            zr = np.sum(z * r)
            v = z + (zr / zr_last) * v
        return p

    def clamp(self, p, q_prev, q_det):
        r = self.c.contact_detection_radius
        dq = q_prev + p - q_det
        ln = _norm(dq)
        big = ln > r
        p = p.copy()
        p[big] = dq[big] / ln[big, None] * r + q_det[big] - q_prev[big]
        return p

    def accd(self, p):
        """Additive CCD step bound over all blocks (ccd_kernels.py:8-110), every
        block advanced together (each block's loop is the reference's; blocks
        leave the set as their own loops end)."""
        c = self.c
        nb = len(self.blocks)
        if not nb:
            return 1.0
        idx = np.asarray(self.blocks)
        kinds = np.asarray(self.kinds)
        x = self.q[idx].copy()
        v = p[idx].copy()
        v = v - v.mean(1, keepdims=True)
        nv = np.sqrt((v * v).sum(2))
        is_pt = kinds == BLOCK_PT
        lv = np.where(is_pt, nv[:, 0] + nv[:, 1:].max(1), nv[:, :2].max(1) + nv[:, 2:].max(1))

        def dist(X, K):
            ty = np.empty(len(X), np.int64)
            m = K == BLOCK_PT
            if m.any():
                ty[m] = pt_classify(X[m, 0], X[m, 1], X[m, 2], X[m, 3])
            if (~m).any():
                ty[~m] = ee_classify(X[~m, 0], X[~m, 1], X[~m, 2], X[~m, 3], c.ee_classify_thres)
            d, _ = pair_distance_grad(X, K, ty)
            return d

        def dminus(d):
            return np.maximum((d * d - c.ccd_thickness ** 2) / (d + c.ccd_thickness), 0.0)

        act = lv >= 1e-12
        step = 1.0
        d = np.zeros(nb)
        d[act] = dist(x[act], kinds[act])
        dmt = dminus(d)
        gap = (1 - c.ccd_slackness) * dmt
        t = np.zeros(nb)
        tl = np.where(act, c.ccd_slackness * dmt / np.where(act, lv, 1.0), 0.0)
        i = 0
        while act.any():
            a = np.nonzero(act)[0]
            x[a] = x[a] + tl[a, None, None] * v[a]
            d[a] = dist(x[a], kinds[a])
            dmt[a] = dminus(d[a])
            done = ((i > 0) & (dmt[a] <= gap[a])) | (i >= c.ccd_max_iters)
            if done.any():
                step = min(step, float(t[a[done]].min()))
                act[a[done]] = False
            a = a[~done]
            t[a] = t[a] + tl[a]
            over = t[a] > 1.0
            act[a[over]] = False
            a = a[~over]
            tl[a] = 0.8 * dmt[a] / lv[a]
            i += 1
        return step

    def newton(self):
        c = self.c
        q_prev = self.q.copy()
        self.detect()
        q_det = self.q.copy()
        e0 = self.energy(self.q)
        g, dg = self.diff(self.q)
        p = self.cg(g, dg)
        p = self.clamp(p, q_prev, q_det)
        step = self.accd(p)
        e = e0
        last = -1
        for nh in range(c.n_line_search_iters):
            if nh > 0 and e < e0:
                break
            self.q = q_prev + step * (0.5 ** nh) * p
            e = self.energy(self.q)
            last = nh
        self.trace.append((e0, e, step, last, len(self.blocks), self.nact))
        return e

    def step(self):
        if self.do_nothing:
            return
        self.update_target()
        for _ in range(self.c.n_newton_iters):
            self.newton()


def spd_project(B, sweeps):
    """Clamp the negative eigenvalues of the 9 x 9 matrix of hinge vertices 0-2
    (cyclic Jacobi, `sweeps` sweeps) and refill vertex 3's rows and columns from
    translation invariance."""
    n = len(B)
    A = B[:, :3, :3].transpose(0, 1, 3, 2, 4).reshape(n, 9, 9).copy()
    A = 0.5 * (A + np.transpose(A, (0, 2, 1)))
    Vm = np.tile(np.eye(9), (n, 1, 1))
    for _ in range(sweeps):
        for p_ in range(8):
            for q_ in range(p_ + 1, 9):
                apq = A[:, p_, q_]
                app, aqq = A[:, p_, p_], A[:, q_, q_]
                nz = np.abs(apq) > 1e-30
                theta = np.where(nz, (aqq - app) / (2 * np.where(nz, apq, 1)), 0)
                t = np.where(nz, np.sign(theta + (theta == 0)) / (np.abs(theta) + np.sqrt(theta * theta + 1)), 0)
                cs = 1 / np.sqrt(t * t + 1)
                sn = t * cs
                Jm = np.tile(np.eye(9), (n, 1, 1))
                Jm[:, p_, p_], Jm[:, q_, q_] = cs, cs
                Jm[:, p_, q_], Jm[:, q_, p_] = sn, -sn
                A = np.transpose(Jm, (0, 2, 1)) @ A @ Jm
                Vm = Vm @ Jm
    lam = np.clip(np.diagonal(A, axis1=1, axis2=2), 0, None)
    A2 = Vm @ (lam[:, :, None] * np.transpose(Vm, (0, 2, 1)))
    out = B.copy()
    out[:, :3, :3] = A2.reshape(n, 3, 3, 3, 3).transpose(0, 1, 3, 2, 4)
    for j in range(3):
        out[:, 3, j] = -(out[:, 0, j] + out[:, 1, j] + out[:, 2, j])
        out[:, j, 3] = np.transpose(out[:, 3, j], (0, 2, 1))
    out[:, 3, 3] = -(out[:, 0, 3] + out[:, 1, 3] + out[:, 2, 3])
    return out


def process(gt_V, gt_F, V, F, n_iters=5, config=None, dtype=np.float64, trace=None):
    """processing.py:23-108 in FP64: normalise by the GT, run n_iters steps,
    undo the normalisation.  Faces are unchanged.  A list given as `trace`
    receives the Newton trace (Stage3Oracle.trace)."""
    scale, t = normalization(np.asarray(gt_V, np.float64))
    gV = np.asarray(gt_V, np.float64) * scale + t
    sV = np.asarray(V, np.float64) * scale + t
    o = Stage3Oracle(config, dtype)
    o.register(gV, gt_F, sV, F)
    for _ in range(n_iters):
        o.step()
    if trace is not None:
        trace.extend(o.trace)
    return (o.q - t) / scale, np.asarray(F)
