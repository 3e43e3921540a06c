"""Parity of the CUDA stage-2 path (libpamo_b200.so through its C ABI) with the
CPU oracle: bit-exact per round (points as float bits, faces, occupancy, map,
undo list) over the normal, undo and stuck paths, and for the whole
device-resident PaMO.run loop."""
import ctypes

import numpy as np
import pytest

from helpers import bits, compact, next_state, prepare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _drive_rounds(torch, V, F, ratio, max_rounds, threshold=1e-3):
    """Runs the same round sequence through the oracle and CUDSP_Free.forward,
    asserting bit equality after every round."""
    import pamo_b200
    from oracle import oracle as O

    P, F0, scale, _ = prepare(V, F)
    Fs = O.shuffle_faces(F0)
    orc = O.Stage2Oracle()
    gpu = pamo_b200.CUDSP_Free()
    undo = np.zeros(0, np.int32)
    stuck = 0
    count = 0
    target = int(ratio * len(F0))
    Pc, Tc = P, Fs
    Tg = F0  # the GPU applies the init permutation itself
    n_rounds = 0
    saw = {"undo": 0, "stuck": 0}
    for r in range(max_rounds):
        prev = len(Tc)
        op, ot, oo, om, ou = orc.forward(Pc, Tc, undo, len(undo), scale, threshold, stuck)
        g = gpu.forward(torch.from_numpy(Pc).cuda(), torch.from_numpy(np.ascontiguousarray(Tg)).cuda(),
                        torch.from_numpy(undo).cuda(), len(undo), float(scale), threshold, bool(stuck), r == 0)
        gv, gt, go, gm, gu = [x.cpu().numpy() for x in g]
        assert np.array_equal(bits(gv), bits(op)), f"round {r}: points differ"
        assert np.array_equal(gt, ot), f"round {r}: faces differ"
        assert np.array_equal(go, oo), f"round {r}: occupancy differs"
        assert np.array_equal(gm, om), f"round {r}: vertex map differs"
        assert np.array_equal(gu, ou), f"round {r}: undo list differs"
        st = orc.stats()
        saw["undo"] += st["n_undo_passes"] > 0
        saw["stuck"] += stuck
        n_rounds += 1
        undo = ou
        Pc, Tc = compact(op, ot, oo, om)
        Tg = Tc
        cur = len(Tc)
        if cur <= target or cur <= 10:
            break
        count, stuck, stop = next_state(cur, prev, count, stuck)
        if stop:
            break
    return n_rounds, saw


def test_rounds_sphere_to_stuck(torch_cuda):
    from pamo_b200 import meshgen as mg

    V, F = mg.displaced_icosphere(3, 0)
    n, saw = _drive_rounds(torch_cuda, V, F, 0.001, 80)
    assert n > 10
    assert saw["stuck"] > 0  # the run ends through the stuck / tolerance path


def test_rounds_thin_shell_undo(torch_cuda):
    from pamo_b200 import meshgen as mg

    V, F = mg.thin_shell_pair(4000, 2e-3, 2)
    n, saw = _drive_rounds(torch_cuda, V, F, 0.01, 12)
    assert saw["undo"] > 0  # collapses pushed one shell through the other and were undone


def test_rounds_c1_sphere(torch_cuda):
    from pamo_b200 import meshgen as mg

    V, F = mg.displaced_icosphere(5, 0)
    _drive_rounds(torch_cuda, V, F, 0.05, 6)


def test_rounds_noisy_torus(torch_cuda):
    from pamo_b200 import meshgen as mg

    V, F = mg.noisy_torus(96, 96, 3)
    _drive_rounds(torch_cuda, V, F, 0.01, 8)


def test_device_loop_matches_oracle_c1(torch_cuda):
    """The whole stage-2 loop of PaMO.run on config 1 (ratio 0.05, min_verts 0)."""
    import pamo_b200
    from oracle import oracle as O
    from pamo_b200 import meshgen as mg

    V, F = mg.displaced_icosphere(5, 0)
    ov, of, orounds = O.pamo_run_stage2(V, F, 0.05, min_verts=0)
    ctx = pamo_b200.Context(0)
    target = max(int(0.05 * len(F)), 0)
    gv, gf, grounds = pamo_b200.stage2_run(ctx, torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda(),
                                           target)
    assert grounds == orounds
    assert np.array_equal(bits(gv.cpu().numpy()), bits(ov))
    assert np.array_equal(gf.cpu().numpy(), of)
    assert len(of) <= target


def test_pamo_run_drop_in(torch_cuda):
    """PaMO(...).run(...) with stage 1 and 3 off returns host numpy like the reference."""
    import pamo_b200
    from oracle import oracle as O
    from pamo_b200 import meshgen as mg

    V, F = mg.displaced_icosphere(4, 1)
    pm = pamo_b200.PaMO((V, F), use_stage1=False, use_stage3=False, verbose=False)
    v, f = pm.run(torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda(), 0.1, min_verts=0)
    assert isinstance(v, np.ndarray) and isinstance(f, np.ndarray)
    ov, of, _ = O.pamo_run_stage2(V, F, 0.1, min_verts=0)
    assert np.array_equal(bits(v), bits(ov)) and np.array_equal(f, of)
    # the reference's default min_verts=1e10 stops after one round
    pm2 = pamo_b200.PaMO((V, F), use_stage1=False, use_stage3=False, verbose=False)
    v2, f2 = pm2.run(torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda(), 0.1)
    assert pm2.last_rounds == 1


def _oracle_blender_loop(V, F, threshold):
    """The reference's pamo_simplify loop (pamo_blender/cusimpinterface.cu:57-161)
    on the oracle: no centring, host bbox scale, undo list passed back in place."""
    from oracle import oracle as O

    L = O.lib()
    c = L.s2o_create()
    P = np.ascontiguousarray(V, np.float32)
    T = O.shuffle_faces(F)
    bb_hi = np.max(np.vstack([P, np.full((1, 3), -1e30, np.float32)]), 0)
    bb_lo = np.min(np.vstack([P, np.full((1, 3), 1e30, np.float32)]), 0)
    scale = np.float32(max((bb_hi - bb_lo).astype(np.float32)))
    n_undo, same, stuck = 0, 0, 0
    try:
        for _ in range(100000):
            n, m = len(P), len(T)
            op = np.empty((n, 3), np.float32)
            ot = np.empty((m, 3), np.int32)
            oo = np.empty(n, np.int32)
            om = np.empty(n, np.int32)
            nu = ctypes.c_int(0)
            undo_ptr = ctypes.cast(L.s2o_undo_list(c), ctypes.c_void_p).value if n_undo else None
            rc = L.s2o_forward(c, P, T, undo_ptr, n_undo, n, m, float(scale), float(threshold), stuck, op, ot, oo, om,
                               ctypes.byref(nu))
            assert rc == 0
            n_undo = nu.value
            P, T = compact(op, ot, oo, om)
            if len(T) == m:
                same += 1
            else:
                same = 0
                stuck = 0
            if same >= 2:
                stuck = 1
            if same >= 4:
                break
    finally:
        L.s2o_destroy(c)
    return P, T


def test_pamo_simplify_c_abi(torch_cuda):
    """Blender-style host C ABI (same signature as the reference's pamo_simplify)."""
    from pamo_b200 import _lib
    from pamo_b200 import meshgen as mg

    V, F = mg.displaced_icosphere(3, 4)
    ov, of = _oracle_blender_loop(V, F, 1e-3)
    inv = np.ascontiguousarray(V, np.float32).copy()
    inf = np.ascontiguousarray(F, np.int32).copy()
    outv = np.zeros_like(inv)
    outf = np.zeros_like(inf)
    nvni = np.array([len(V), len(F)], np.int32)
    _lib.lib().pamo_simplify(inv.ctypes.data, inf.ctypes.data, outv.ctypes.data, outf.ctypes.data, nvni.ctypes.data,
                             1e-3)
    n, m = int(nvni[0]), int(nvni[1])
    assert (n, m) == (len(ov), len(of))
    assert np.array_equal(bits(outv[:n]), bits(ov))
    assert np.array_equal(outf[:m], of)


def test_self_intersect_matches_reference_fixtures(torch_cuda):
    """LBVH + pair test on whole meshes against the reference's own
    selfx::self_intersect flags (tests/golden/isect.npz)."""
    import os

    import pamo_b200

    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "isect.npz"))
    ctx = pamo_b200.Context(0)
    for name in ("two_spheres", "crumpled", "folded_grids", "soup"):
        V, F, want = g[f"{name}_V"], g[f"{name}_F"], g[f"{name}_flags"]
        got, npairs = pamo_b200.self_intersect(ctx, torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda())
        got = got.cpu().numpy()
        assert npairs > 0
        if name == "soup":  # beyond the reference's pair capacity: a superset of its flags
            assert np.all(got[want == 1] == 1) and got.sum() > want.sum()
        else:
            assert np.array_equal(got, want), name


def test_self_intersect_clean_meshes_report_nothing(torch_cuda):
    import pamo_b200
    from pamo_b200 import meshgen as mg

    ctx = pamo_b200.Context(0)
    for V, F in (mg.displaced_icosphere(5, 0), mg.noisy_torus(128, 128, 1), mg.thin_shell_pair(20000, 2e-3, 1)):
        got, _ = pamo_b200.self_intersect(ctx, torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda())
        assert int(got.sum()) == 0
