"""The stage-3 FP64 oracle (oracle/s3_oracle.py) checked on its own, on the CPU:
its gradients against central differences of its energy, its distance
gradients against differences of the distances, the symmetry of its CG
operator, the SPD projection's invariants, and the property the reference's
own stage-3 test relies on (safe_project/tests/test_dummy_energy.py:1-40: on a
quadratic energy the CG solve gives the Newton step exactly)."""
import numpy as np
import pytest

from oracle import s3_oracle as S
from pamo_b200 import meshgen as mg


def _system(level=2, seed=0, amplitude=0.05, shift=0.01):
    """A displaced icosphere projected towards the undisplaced one: the mesh
    moves, so the distance, membrane and hinge terms are all away from rest."""
    gV, gF = mg.displaced_icosphere(level, seed, amplitude)
    gV = np.asarray(gV, np.float64)
    rng = np.random.default_rng(seed + 1)
    V = gV + shift * rng.standard_normal(gV.shape)
    o = S.Stage3Oracle()
    o.register(gV, gF, gV, gF)  # rest shape = ground truth
    o.q = V.copy()
    o.update_target()
    return o


def _dir_derivative(f, q, v, h=1e-6):
    return (f(q + h * v) - f(q - h * v)) / (2 * h)


@pytest.mark.parametrize("seed", [0, 1])
def test_gradient_matches_energy_differences(seed):
    o = _system(seed=seed)
    g, dg = o.diff(o.q)  # g is minus the gradient
    rng = np.random.default_rng(10 + seed)
    for _ in range(4):
        v = rng.standard_normal(o.q.shape)
        fd = _dir_derivative(o.energy, o.q, v)
        an = -np.sum(g * v)
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)
    assert np.all(dg >= 0)


def test_gradient_matches_energy_differences_with_contacts():
    """Two shells closer than d_hat: the barrier terms are active.  Facing edges
    of the two shells are nearly parallel, where the edge-edge distance takes
    the smallest of its point-edge candidates and a difference step can cross
    a tie, so the differences hold each block's distance type fixed at q."""
    V, F = mg.thin_shell_pair(800, 5e-4, 0)
    V = np.asarray(V, np.float64)
    V = V + 2e-5 * np.random.default_rng(8).standard_normal(V.shape)
    o = S.Stage3Oracle()
    o.register(V, F, V, F)
    o.update_target()
    o.detect()
    g, _ = o.diff(o.q)
    G, b2c = o.coll
    assert np.count_nonzero(b2c) > 0
    _, ty0 = o._classify_blocks(o.q)
    blocks, kinds = o.blocks, o.kinds
    dh, kappa = o.c.d_hat, o.c.coll_stiffness

    def energy_fixed_types(q):
        d, _ = S.pair_distance_grad(q[blocks], kinds, ty0, want_grad=False)
        ec = np.sum(np.where(d < dh, S.Stage3Oracle.barrier(d, dh), 0.0)) * kappa
        o.blocks = blocks[:0]
        try:
            return o.energy(q) + ec
        finally:
            o.blocks = blocks

    rng = np.random.default_rng(7)
    for _ in range(4):
        v = rng.standard_normal(o.q.shape)
        fd = _dir_derivative(energy_fixed_types, o.q, v, h=1e-8)
        an = -np.sum(g * v)
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)


def test_barrier_derivatives_match_differences():
    dh = 1e-3
    d = np.linspace(1e-5, 0.999e-3, 50)
    h = 1e-9
    b1 = (S.Stage3Oracle.barrier(d + h, dh) - S.Stage3Oracle.barrier(d - h, dh)) / (2 * h)
    b2 = (S.Stage3Oracle.barrier_d1(d + h, dh) - S.Stage3Oracle.barrier_d1(d - h, dh)) / (2 * h)
    np.testing.assert_allclose(S.Stage3Oracle.barrier_d1(d, dh), b1, rtol=1e-5, atol=1e-12)
    np.testing.assert_allclose(S.Stage3Oracle.barrier_d2(d, dh), b2, rtol=1e-5, atol=1e-9)
    assert np.all(S.Stage3Oracle.barrier(np.array([dh, 2 * dh]), dh) == 0)


@pytest.mark.parametrize("kind", ["pt", "ee"])
def test_distance_gradient_matches_differences(kind):
    """Every sub-type (vertex, edge, face / parallel or not) the classification
    reaches on random blocks, with the type held fixed for the differences."""
    rng = np.random.default_rng(3 if kind == "pt" else 4)
    X = rng.standard_normal((4000, 4, 3))
    if kind == "pt":
        bk = np.full(len(X), S.BLOCK_PT)
        ty = S.pt_classify(X[:, 0], X[:, 1], X[:, 2], X[:, 3])
    else:
        # some nearly parallel pairs, to reach the parallel branch
        X[:500, 3] = X[:500, 2] + (X[:500, 1] - X[:500, 0]) * 0.7 + 1e-4 * rng.standard_normal((500, 3))
        bk = np.full(len(X), S.BLOCK_EE)
        ty = S.ee_classify(X[:, 0], X[:, 1], X[:, 2], X[:, 3], 1e-3)
    assert len(np.unique(ty)) >= 3
    d, G = S.pair_distance_grad(X, bk, ty)
    V = rng.standard_normal(X.shape)
    h = 1e-7
    dp, _ = S.pair_distance_grad(X + h * V, bk, ty, want_grad=False)
    dm, _ = S.pair_distance_grad(X - h * V, bk, ty, want_grad=False)
    fd = (dp - dm) / (2 * h)
    an = np.einsum("nij,nij->n", G, V)
    assert np.all(d >= 0)
    np.testing.assert_allclose(an, fd, rtol=1e-4, atol=1e-6)


def test_cg_operator_is_symmetric():
    o = _system(level=2, seed=2)
    o.diff(o.q)
    rng = np.random.default_rng(5)
    u = rng.standard_normal(o.q.shape)
    v = rng.standard_normal(o.q.shape)
    a = np.sum(u * o.hess_dx(o.q, v))
    b = np.sum(v * o.hess_dx(o.q, u))
    assert abs(a - b) <= 1e-10 * max(abs(a), abs(b))


def test_cg_gives_the_newton_step_on_a_small_system():
    """An icosahedron at rest (membrane and hinge terms positive semidefinite,
    the distance term positive definite): 40 Jacobi-PCG iterations on 36
    unknowns solve K p = g to rounding."""
    V, F = mg.icosahedron()
    V = np.asarray(V, np.float64)
    o = S.Stage3Oracle()
    o.register(V, F, V, F)
    o.update_target()
    rng = np.random.default_rng(6)
    o.target = o.target + 0.01 * rng.standard_normal(o.target.shape)
    g, dg = o.diff(o.q)
    p = o.cg(g, dg)
    res = o.hess_dx(o.q, p) - g
    assert np.linalg.norm(res) <= 1e-8 * np.linalg.norm(g)


def _spd_symmetric_form(B, sweeps):
    """Cyclic Jacobi with each rotation applied to rows and columns p, q in the
    symmetric form (a_pq -> 0, a_pp and a_qq move by -/+ t a_pq), the form the
    CUDA projection uses; the oracle applies J^T A J as matrices."""
    n = len(B)
    A = B[:, :3, :3].transpose(0, 1, 3, 2, 4).reshape(n, 9, 9).copy()
    A = 0.5 * (A + np.transpose(A, (0, 2, 1)))
    Vm = np.tile(np.eye(9), (n, 1, 1))
    for _ in range(sweeps):
        for p_ in range(8):
            for q_ in range(p_ + 1, 9):
                apq = A[:, p_, q_].copy()
                nz = np.abs(apq) > 1e-30
                theta = np.where(nz, (A[:, q_, q_] - A[:, p_, p_]) / (2 * np.where(nz, apq, 1)), 0)
                t = np.where(nz, np.sign(theta + (theta == 0)) / (np.abs(theta) + np.sqrt(theta * theta + 1)), 0)
                c = 1 / np.sqrt(t * t + 1)
                s = t * c
                for k in range(9):
                    if k in (p_, q_):
                        continue
                    akp, akq = A[:, k, p_].copy(), A[:, k, q_].copy()
                    A[:, k, p_] = A[:, p_, k] = c * akp - s * akq
                    A[:, k, q_] = A[:, q_, k] = s * akp + c * akq
                A[:, p_, p_] -= t * apq
                A[:, q_, q_] += t * apq
                A[:, p_, q_] = A[:, q_, p_] = 0
                vp, vq = Vm[:, :, p_].copy(), Vm[:, :, q_].copy()
                Vm[:, :, p_] = c[:, None] * vp - s[:, None] * vq
                Vm[:, :, q_] = s[:, None] * vp + c[:, None] * vq
    lam = np.clip(np.diagonal(A, axis1=1, axis2=2), 0, None)
    return Vm @ (lam[:, :, None] * np.transpose(Vm, (0, 2, 1)))


def test_spd_projection_invariants_and_symmetric_form():
    o = _system(level=2, seed=3, shift=0.03)
    Hb, _ = o._hinge_blocks(o.q)
    out = S.spd_project(Hb, 3)
    n = len(Hb)
    full = out.transpose(0, 1, 3, 2, 4).reshape(n, 12, 12)
    scale = np.abs(full).max()
    # symmetric, translation invariant (block rows sum to zero)
    assert np.abs(full - np.transpose(full, (0, 2, 1))).max() <= 1e-12 * scale
    assert np.abs(out.sum(axis=1)).max() <= 1e-12 * scale
    # positive semidefinite up to what three sweeps leave off the diagonal
    assert np.linalg.eigvalsh(full).min() >= -1e-6 * scale
    # the unprojected blocks were indefinite somewhere, so the clamp did work
    raw = Hb.transpose(0, 1, 3, 2, 4).reshape(n, 12, 12)
    assert np.linalg.eigvalsh(0.5 * (raw + np.transpose(raw, (0, 2, 1)))).min() < -1e-3 * scale
    # the symmetric rotation form gives the oracle's result to rounding
    sym = _spd_symmetric_form(Hb, 3)
    np.testing.assert_allclose(sym, full[:, :9, :9], rtol=0, atol=1e-10 * scale)
