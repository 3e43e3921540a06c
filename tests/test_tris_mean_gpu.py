"""The centring offset (PaMO.run's tris_mean) on the device, pamo_tris_mean,
against the oracle's sequential float32 chain (itself pinned to numpy in
test_oracle.py), bit for bit, on inputs that stress a float32 chain: sums that
hover around zero, values on coarse dyadic grids (round-half-even ties), mixed
magnitudes, subnormals, signed zeros and non-finite coordinates."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _device(torch, V, F):
    from pamo_b200 import _lib

    pv = torch.from_numpy(np.ascontiguousarray(V, np.float32)).cuda()
    pf = torch.from_numpy(np.ascontiguousarray(F, np.int32)).cuda()
    out = np.zeros(3, np.float32)
    rc = _lib.lib().pamo_tris_mean(pv.data_ptr(), pf.data_ptr(), len(V), len(F), out.ctypes.data_as(ctypes.c_void_p),
                                   None)
    assert rc == 0, rc
    return out


def _same(a, b):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    both_nan = np.isnan(a) & np.isnan(b)
    return bool(np.all(both_nan | (a.view(np.uint32) == b.view(np.uint32))))


def _cases(rng):
    from pamo_b200 import meshgen as mg

    yield "torus-1024", *mg.noisy_torus(1024, 1024, 0)
    for m in (4095, 4096, 4097, 4129, 100003, 262144 + 17):
        n = max(m // 2, 8)
        F = rng.integers(0, n, (m, 3)).astype(np.int32)
        yield f"normal-{m}", rng.standard_normal((n, 3)).astype(np.float32), F
        # symmetric about zero: the running sums keep crossing binades
        H = rng.standard_normal(((n + 1) // 2, 3)).astype(np.float32)
        yield f"hover-{m}", np.concatenate([H, -H])[:n], F
        # coarse dyadic grid: many steps are ties
        yield f"ties-{m}", (rng.integers(-64, 64, (n, 3)) * 0.375).astype(np.float32), F
        yield f"ties-small-{m}", (rng.integers(-8, 8, (n, 3)) * 2.0 ** -20).astype(np.float32), F
        # a large offset with small increments, positive and negative
        yield f"drift-{m}", (1e4 + rng.random((n, 3))).astype(np.float32), F
        yield f"drift-neg-{m}", (-3e3 - rng.random((n, 3)) * 1e-3).astype(np.float32), F
        # magnitudes from 1e-30 to 1e30, subnormals, zeros of both signs
        W = (rng.standard_normal((n, 3)) * 10.0 ** rng.integers(-30, 30, (n, 3))).astype(np.float32)
        W[rng.random((n, 3)) < 0.05] = np.float32(1e-40)
        W[rng.random((n, 3)) < 0.05] = 0.0
        W[rng.random((n, 3)) < 0.05] = -0.0
        yield f"mixed-{m}", W, F
        yield f"subnormal-{m}", (rng.standard_normal((n, 3)) * 1e-40).astype(np.float32), F
    # non-finite coordinates part way through
    V, F = mg.noisy_torus(256, 256, 1)
    V = V.astype(np.float32).copy()
    V[1000, 0] = np.inf
    V[2000, 1] = -np.inf
    V[3000, 2] = np.nan
    yield "nonfinite", V, F


def test_tris_mean_matches_oracle_bit_for_bit(torch_cuda):
    from oracle import oracle as O

    rng = np.random.default_rng(7)
    bad = []
    n_cases = 0
    for name, V, F in _cases(rng):
        n_cases += 1
        got, want = _device(torch_cuda, V, F), O.tris_mean(V, F)
        if not _same(got, want):
            bad.append((name, got, want))
    assert not bad, bad
    assert n_cases >= 50


def test_tris_mean_rejects_bad_indices(torch_cuda):
    from pamo_b200 import _lib

    V = np.zeros((10, 3), np.float32)
    F = np.array([[0, 1, 2], [3, 4, 10]], np.int32)
    pv = torch_cuda.from_numpy(V).cuda()
    pf = torch_cuda.from_numpy(F).cuda()
    out = np.zeros(3, np.float32)
    assert _lib.lib().pamo_tris_mean(pv.data_ptr(), pf.data_ptr(), 10, 2, out.ctypes.data_as(ctypes.c_void_p),
                                     None) == 1
