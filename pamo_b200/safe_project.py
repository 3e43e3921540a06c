"""Stage 3 (safe projection) host side; mirrors pamo_safe_project
(simp_cuda/safe_project/src/pamo_safe_project): ``Stage3Config``,
``Stage3System`` and ``process(gt_V, gt_F, V, F, n_iters, system, config)``.

The host does what the reference does on the CPU before its GPU loop: the
normalisation by the ground truth (processing.py:15-20,57-59) in float64, the
unique edges, the hinges (one per interior edge, hinge_energy.py:21-57), the
Voronoi vertex areas (the mixed areas of Meyer et al. 2003, which
igl.massmatrix(VORONOI) computes, system.py:223-225) and the small-angle guard
(system.py:217-221).  Everything after that -- closest points on the ground
truth, contact detection, energies, Jacobi-PCG, CCD, line search -- runs in
libpamo_b200.so (csrc/stage3.cu) through pamo_safe_project().
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import Context, check


class pamo_s3_config(ctypes.Structure):
    _fields_ = [("n_newton_iters", ctypes.c_int), ("n_cg_iters", ctypes.c_int), ("n_line_search_iters", ctypes.c_int),
                ("ccd_max_iters", ctypes.c_int), ("spd_max_iters", ctypes.c_int), ("d_hat", ctypes.c_float),
                ("coll_stiffness", ctypes.c_float), ("contact_detection_radius", ctypes.c_float),
                ("ee_classify_thres", ctypes.c_float), ("ccd_slackness", ctypes.c_float),
                ("ccd_thickness", ctypes.c_float), ("elas_young_modulus", ctypes.c_float),
                ("elas_poisson_ratio", ctypes.c_float), ("hinge_stiffness", ctypes.c_float),
                ("mesh2gt_dist_stiffness", ctypes.c_float), ("max_blocks", ctypes.c_longlong),
                ("reuse_gt", ctypes.c_int)]


class Stage3Config:
    """The reference's Stage3Config defaults (config.py:6-73) for the default
    energy set (GT distance, membrane, bending, contact)."""

    def __init__(self):
        self.debug = False
        self.seed = 0
        self.max_particles = 1 << 20
        self.max_blocks = 1 << 25
        self.reuse_gt = 0  # set per call by Stage3System.project
        self.max_gt_particles = 1 << 24
        self.max_gt_samples = 1 << 14
        self.n_newton_iters = 10
        self.n_cg_iters = 40
        self.cg_precond = "jacobi"
        self.use_cuda_graph = True
        self.n_line_search_iters = 10
        self.detect_contact_every = "newton"
        self.system_scale = 1.0
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
        self.curv_stiffness = 1e-8
        self.hinge_stiffness = 1e-2
        self.mesh2gt_dist_stiffness = 1e3
        self.gt2mesh_dist_stiffness = 1e3
        self.min_angle_thres = 0.0

    def to_c(self) -> pamo_s3_config:
        if self.cg_precond != "jacobi" or self.detect_contact_every != "newton":
            raise NotImplementedError("only the reference's default solver settings are supported")
        c = pamo_s3_config()
        for name, _ in pamo_s3_config._fields_:
            setattr(c, name, getattr(self, name))
        return c


# ------------------------------------------------------------ host preprocessing
def normalization(V):
    """processing.py:15-20.  The extents are exact whichever way they are
    reduced; they are taken over a transposed copy, which numpy reduces much
    faster than the (n, 3) columns."""
    V = np.asarray(V, np.float64)
    center = np.mean(V, axis=0)
    Vt = np.ascontiguousarray(V.T)
    extents = Vt.max(axis=1) - Vt.min(axis=1)
    scale = 1.0 / np.max(extents)
    return scale, -center * scale


def edges_unique(F):
    """Sorted unique edges (a < b), in the order np.unique(axis=0) gives, found as
    unique 64-bit keys a * n + b."""
    F = np.asarray(F, np.int64)
    if len(F) == 0:
        return np.zeros((0, 2), np.int64)
    x = np.concatenate([F[:, 0], F[:, 1], F[:, 2]])
    y = np.concatenate([F[:, 1], F[:, 2], F[:, 0]])
    n = int(F.max()) + 1
    k = np.sort(np.minimum(x, y) * n + np.maximum(x, y))  # np.unique's result, without its slower path
    k = k[np.concatenate([[True], k[1:] != k[:-1]])]
    return np.stack([k // n, k % n], axis=1)


def hinges(F):
    """(x0, x1, x2, x3) per interior edge: the face with directed edge x1->x2
    (x1 < x2) and the face with x2->x1; x0 / x3 their opposite vertices."""
    F = np.asarray(F, np.int64)
    # directed edges a -> b of every face (corner k to k + 1), c the third vertex
    a = np.concatenate([F[:, 0], F[:, 1], F[:, 2]])
    b = np.concatenate([F[:, 1], F[:, 2], F[:, 0]])
    c = np.concatenate([F[:, 2], F[:, 0], F[:, 1]])
    n = int(F.max()) + 1 if len(F) else 1
    mf, mb = a < b, a > b
    af, bf, cf = a[mf], b[mf], c[mf]
    kf = af * n + bf
    kb = b[mb] * n + a[mb]
    cb = c[mb]
    # closed 2-manifold (the usual case): every edge once each way, so the two
    # sorted key lists pair up element by element
    if len(kf) == len(kb):
        of = np.argsort(kf, kind="stable")
        ob = np.argsort(kb, kind="stable")
        kfs = kf[of]
        if np.array_equal(kfs, kb[ob]) and (len(kfs) < 2 or bool((kfs[1:] != kfs[:-1]).all())):
            return np.stack([cf[of], af[of], bf[of], cb[ob]], 1)
    ob = np.argsort(kb, kind="stable")
    kbs = kb[ob]
    pos = np.searchsorted(kbs, kf)
    ok = (pos < len(kbs)) & (kbs[np.minimum(pos, max(len(kbs) - 1, 0))] == kf) if len(kbs) else np.zeros(len(kf), bool)
    H = np.stack([cf[ok], af[ok], bf[ok], cb[ob][pos[ok]]], 1)
    # ordered by (x1, x2): the key x1 * n + x2 orders the same way (stable, as lexsort)
    return H[np.argsort(kf[ok], kind="stable")]


def edges_and_hinges(F):
    """(edges_unique(F), hinges(F)).  A closed 2-manifold (every edge in
    exactly two faces, once each way) takes the library's linear-time host
    builder (pamo_mesh_hinges); otherwise one sort of the 3 m directed face
    edges by undirected key pairs them up, and meshes where that fails take the
    two separate functions.  The builder's arrays are int32, the others int64."""
    if len(F) == 0:
        return edges_unique(F), hinges(F)
    F32 = np.ascontiguousarray(F, np.int32)
    n_pts = int(F32.max()) + 1
    cap = (3 * len(F)) // 2 + 1
    E32, H32 = np.empty((cap, 2), np.int32), np.empty((cap, 4), np.int32)
    ne = ctypes.c_int(0)
    rc = _lib.lib().pamo_mesh_hinges(F32.ctypes.data, len(F32), n_pts, E32.ctypes.data, H32.ctypes.data,
                                     ctypes.byref(ne))
    if rc == 0:
        return E32[:ne.value], H32[:ne.value]
    F = np.asarray(F, np.int64)
    a = np.concatenate([F[:, 0], F[:, 1], F[:, 2]])
    b = np.concatenate([F[:, 1], F[:, 2], F[:, 0]])
    c = np.concatenate([F[:, 2], F[:, 0], F[:, 1]])
    n = int(F.max()) + 1
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    key = lo * n + hi
    o = np.argsort(key, kind="stable")
    ks = key[o]
    if len(ks) % 2 == 0:
        k0, k1 = ks[0::2], ks[1::2]
        o0, o1 = o[0::2], o[1::2]
        fwd0 = a[o0] < b[o0]
        if (np.array_equal(k0, k1) and (len(k0) < 2 or bool((k0[1:] != k0[:-1]).all()))
                and bool((fwd0 != (a[o1] < b[o1])).all())):
            of = np.where(fwd0, o0, o1)
            ob = np.where(fwd0, o1, o0)
            E = np.stack([k0 // n, k0 % n], axis=1)
            H = np.stack([c[of], a[of], b[of], c[ob]], 1)
            return E, H
    return edges_unique(F), hinges(F)


def voronoi_areas(V, F):
    """Mixed Voronoi vertex areas (Meyer, Desbrun, Schroeder, Barr 2003)."""
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    ea, eb, ec = c - b, a - c, b - a
    la2, lb2, lc2 = (ea * ea).sum(1), (eb * eb).sum(1), (ec * ec).sum(1)
    area = 0.5 * np.linalg.norm(np.cross(ec, -eb), axis=1)
    with np.errstate(divide="ignore", invalid="ignore"):
        cos_a = -(eb * ec).sum(1) / np.sqrt(lb2 * lc2)
        cos_b = -(ec * ea).sum(1) / np.sqrt(lc2 * la2)
        cos_c = -(ea * eb).sum(1) / np.sqrt(la2 * lb2)
        cot = lambda cs: cs / np.sqrt(np.maximum(1 - cs * cs, 0))
        ca, cb, cc = cot(cos_a), cot(cos_b), cot(cos_c)
    vor = np.stack([(lb2 * cb + lc2 * cc) / 8, (lc2 * cc + la2 * ca) / 8, (la2 * ca + lb2 * cb) / 8], 1)
    mix = np.stack([np.where(cos_a < 0, area / 2, area / 4), np.where(cos_b < 0, area / 2, area / 4),
                    np.where(cos_c < 0, area / 2, area / 4)], 1)
    obtuse = (cos_a < 0) | (cos_b < 0) | (cos_c < 0)
    w = np.where(obtuse[:, None], mix, vor)
    # per-vertex sums in face order (what np.add.at over the three corners does)
    idx = np.asarray(F, np.int64).T.reshape(-1)
    return np.bincount(idx, weights=w.T.reshape(-1), minlength=len(V))[:len(V)]


def min_internal_angle_deg(V, F):
    # the smallest angle has the largest cosine (arccos and the clip are monotone)
    if not len(F):
        return 180.0
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    cmax = None
    for p, q, r in ((a, b, c), (b, c, a), (c, a, b)):
        u, v = q - p, r - p
        cs = (u * v).sum(1) / np.sqrt((u * u).sum(1) * (v * v).sum(1))
        cmax = cs if cmax is None else np.fmax(cmax, cs)
    if np.isnan(cmax).any():
        return float("nan")
    return float(np.arccos(np.clip(cmax.max(), -1, 1)) * 180 / np.pi)


def device_edges_and_hinges(d_f, n_pts, stream):
    """edges_and_hinges on the device (pamo_mesh_hinges_device): int32 CUDA
    tensors (edges [ne,2], hinges [ne,4]) with the host builder's rows and
    order, or (None, None) when the faces are not a closed 2-manifold."""
    import torch

    m = int(d_f.shape[0])
    if m == 0 or (3 * m) % 2:
        return None, None
    cap = (3 * m) // 2
    d_e = torch.empty((cap, 2), dtype=torch.int32, device=d_f.device)
    d_h = torch.empty((cap, 4), dtype=torch.int32, device=d_f.device)
    ne = ctypes.c_int(0)
    rc = _lib.lib().pamo_mesh_hinges_device(d_f.data_ptr(), m, int(n_pts), d_e.data_ptr(), d_h.data_ptr(),
                                            ctypes.byref(ne), stream)
    if rc == 6:  # PAMO_ERR_CAPACITY: an edge not shared by exactly two faces, once each way
        return None, None
    check("pamo_mesh_hinges_device", rc)
    return d_e[:ne.value], d_h[:ne.value]


def has_duplicate_vertices(d_points):
    """Whether merge_vertices would merge anything in the CUDA float32 points
    [n,3] (pamo_merge_check_device: equal after rounding to 8 decimals)."""
    import torch

    d_points = d_points.contiguous()
    out = ctypes.c_int(0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(d_points.device).cuda_stream)
    check("pamo_merge_check_device", _lib.lib().pamo_merge_check_device(d_points.data_ptr(), int(d_points.shape[0]),
                                                                         ctypes.byref(out), stream))
    return bool(out.value)


def merge_vertices(V, F, digits=8):
    """trimesh.Trimesh(process=True) merging (PaMO.run's stage2_mesh,
    pamo/__init__.py:194): vertices equal after rounding to `digits` decimals
    become one; unreferenced vertices are kept in order like trimesh keeps them
    after merging."""
    V = np.asarray(V, np.float64)
    key = np.round(V, digits)
    # no two rows equal (the usual case): nothing merges, nothing moves.  Equal
    # rows have equal x, so only runs of equal x need a full comparison.
    if len(key) < 2:
        return V, np.asarray(F)
    ox = np.argsort(key[:, 0], kind="stable")
    kx = key[ox]
    same_x = kx[1:, 0] == kx[:-1, 0]
    if not same_x.any():
        return V, np.asarray(F)
    # the rows in runs of equal x, sorted by (x, y, z): equal rows are adjacent
    in_run = np.zeros(len(kx), bool)
    in_run[1:] |= same_x
    in_run[:-1] |= same_x
    sub_rows = kx[in_run]
    k3 = sub_rows[np.lexsort((sub_rows[:, 2], sub_rows[:, 1], sub_rows[:, 0]))]
    if not ((k3[1:] == k3[:-1]).all(axis=1)).any():
        return V, np.asarray(F)
    _, first, inv = np.unique(key, axis=0, return_index=True, return_inverse=True)
    order = np.argsort(first)
    rank = np.empty_like(order)
    rank[order] = np.arange(len(order))
    newF = rank[inv.reshape(-1)][np.asarray(F)]
    return V[first[order]], newF


class Stage3System:
    """Device state for stage 3 (one pamo_ctx)."""

    def __init__(self, config: Stage3Config | None = None, device=0):
        self.config = config or Stage3Config()
        if isinstance(device, str):
            device = int(device.split(":")[1]) if ":" in device else 0
        self.device = device
        self.ctx = Context(device)
        self.last_stats = None
        self.last_trace = None
        # a ground truth that stays the same from call to call (PaMO.run's):
        # its device copies, normalisation and the library's hierarchy are kept
        self._gt_raw = None   # ((gt_V, gt_F), raw device points, scale, t)
        self._gt_norm = None  # ((raw points, gt_F, scale, t, system_scale), normalised points, faces)

    def clear(self):
        self.last_stats = None

    def project(self, gt_V, gt_F, V, F, n_steps, gt_affine=None, gt_static=False):
        """Normalised-frame arrays in, projected vertices (float32) out.  With
        gt_affine = (scale, t), gt_V holds the raw ground-truth points and the
        normalisation gt_V * scale + t is applied on the device (float64, then
        rounded to float32 as the host path does).  gt_static: the caller
        promises that gt_V / gt_F are the same objects with the same contents
        as in its earlier calls, so their device forms are kept."""
        import torch

        c = self.config
        dev = torch.device("cuda", self.device)
        V64 = np.asarray(V, np.float64) * c.system_scale
        F = np.asarray(F, np.int64)
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(dev)
        stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        d_f = t(F, np.int32)
        d_e, d_h = device_edges_and_hinges(d_f, len(V64), stream)
        if d_e is None:  # not a closed 2-manifold: the general host method
            E, H = edges_and_hinges(F)
            if len(H) != len(E):
                raise ValueError(f"number of hinges {len(H)} != number of edges {len(E)} (mesh not closed 2-manifold)")
            d_e, d_h = t(E, np.int32), t(H, np.int32)
        # Voronoi areas and the smallest angle, on the device in double from the
        # double vertices (voronoi_areas / min_internal_angle_deg are the host forms)
        d_v64 = t(V64, np.float64)
        d_w = torch.empty(len(V64), dtype=torch.float32, device=dev)
        min_ang = ctypes.c_double()
        check("pamo_voronoi_areas", _lib.lib().pamo_voronoi_areas(
            d_v64.data_ptr(), d_f.data_ptr(), len(V64), len(F), d_w.data_ptr(), ctypes.byref(min_ang), stream))
        do_nothing = min_ang.value <= c.min_angle_thres
        reuse = 0
        key = None
        if gt_static and gt_affine is not None:
            key = (gt_V, gt_F, float(gt_affine[0]), tuple(float(x) for x in gt_affine[1]), float(c.system_scale))
            old = self._gt_norm
            if old is not None and old[0][0] is key[0] and old[0][1] is key[1] and old[0][2:] == key[2:]:
                reuse = 1
        if reuse:
            _, d_gv, d_gf = self._gt_norm
        elif gt_affine is None:
            d_gv = t(np.asarray(gt_V, np.float64) * c.system_scale, np.float32)
        else:
            raw = gt_V if isinstance(gt_V, torch.Tensor) else t(gt_V, np.float32)
            raw = raw.to(dev, torch.float32).contiguous()
            d_gv = torch.empty_like(raw)
            sc, tr = gt_affine
            check("pamo_affine_points", _lib.lib().pamo_affine_points(
                raw.data_ptr(), int(raw.shape[0]), float(sc), float(tr[0]), float(tr[1]), float(tr[2]),
                float(c.system_scale), d_gv.data_ptr(), stream))
        if not reuse:
            d_gf = gt_F.to(dev, torch.int32).contiguous() if isinstance(gt_F, torch.Tensor) else t(gt_F, np.int32)
            self._gt_norm = (key, d_gv, d_gf) if key is not None else None
        d_v = d_v64.to(torch.float32)
        out = torch.empty((len(V64), 3), dtype=torch.float32, device=dev)
        cfg = c.to_c()
        cfg.reuse_gt = reuse
        check("pamo_safe_project", _lib.lib().pamo_safe_project(
            self.ctx.handle, d_gv.data_ptr(), d_gf.data_ptr(), len(d_gv), len(d_gf), d_v.data_ptr(), d_f.data_ptr(),
            len(V64), len(F), d_e.data_ptr(), len(d_e), d_h.data_ptr(), len(d_h), d_w.data_ptr(), int(n_steps),
            int(do_nothing), ctypes.byref(cfg), stream, out.data_ptr()))
        st = (ctypes.c_double * 3)()
        _lib.lib().pamo_safe_project_stats(self.ctx.handle, st)
        self.last_stats = {"energy": st[0], "contacts": int(st[1]), "newton_iters": int(st[2]),
                           "do_nothing": bool(do_nothing)}
        rows = ctypes.c_int(0)
        cap = max(1, int(n_steps) * c.n_newton_iters)
        tr = np.zeros((cap, 6), np.float64)
        check("pamo_safe_project_trace", _lib.lib().pamo_safe_project_trace(
            self.ctx.handle, tr.ctypes.data, cap, ctypes.byref(rows)))
        # per Newton iteration: energy at the iterate, energy after the line
        # search, CCD step, last halving tried, contact blocks, blocks within d_hat
        self.last_trace = tr[:min(rows.value, cap)]
        return out.cpu().numpy() / c.system_scale


def process(gt_V, gt_F, stage2_V, stage2_F, n_iters, system: Stage3System | None = None,
            config: Stage3Config | None = None, eval=False, return_curve=False, gt_static=False):
    """processing.py:23-108: normalise by the ground truth, project, undo the
    normalisation.  Faces are returned unchanged."""
    if system is None:
        system = Stage3System(config or Stage3Config())
    else:
        system.clear()
    import torch

    on_device = isinstance(gt_V, torch.Tensor) or np.asarray(gt_V).dtype == np.float32
    if on_device:
        # float32 ground truth: its mean and extents, the normalisation and the
        # cast to float32 all run on the device (the mean is a fixed-order
        # double sum, which rounds differently from numpy's by ~1e-16)
        dev = torch.device("cuda", system.device)
        old = system._gt_raw if gt_static else None
        if old is not None and old[0][0] is gt_V and old[0][1] is gt_F:
            _, d_gt, scale, t = old
        else:
            d_gt = gt_V if isinstance(gt_V, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(gt_V))
            d_gt = d_gt.to(dev, torch.float32, non_blocking=True).contiguous()
            st = (ctypes.c_double * 6)()
            check("pamo_point_stats", _lib.lib().pamo_point_stats(
                d_gt.data_ptr(), int(d_gt.shape[0]), st, ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
            center = np.array(st[0:3])
            scale = 1.0 / max(st[3], st[4], st[5])
            t = -center * scale
            system._gt_raw = ((gt_V, gt_F), d_gt, scale, t) if gt_static else None
        gt_in = d_gt
    else:  # float64 ground truth: normalised on the host, as processing.py does
        scale, t = normalization(gt_V)
        gt_in = np.asarray(gt_V, np.float64) * scale + t
    sV = np.asarray(stage2_V, np.float64) * scale + t
    q = system.project(gt_in, gt_F, sV, stage2_F, n_iters, gt_affine=(scale, t) if on_device else None,
                       gt_static=gt_static and on_device)
    return (q.astype(np.float64) - t) / scale, np.asarray(stage2_F)


def __getattr__(name):  # the reference exposes the defaults through .config / .system
    raise AttributeError(name)
