"""Stage 3 (safe projection) on the GPU: FP32 Newton-PCG with FP64 barrier /
CCD terms against the FP64 oracle of the same algorithm (oracle/s3_oracle.py),
and the invariants the reference relies on (energy decreases, no
self-intersection, faces unchanged)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# FP32 solve vs FP64 solve of the same steps: max vertex deviation allowed, as a
# fraction of the ground truth's bounding-box diagonal
TOL_DIAG = 1e-3


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def c1_stage2():
    from oracle import oracle as O
    from pamo_b200 import meshgen as mg

    V, F = mg.displaced_icosphere(5, 0)
    v, f, _ = O.pamo_run_stage2(V, F, 0.05, min_verts=0)
    return V, F, v, f


def _diag(V):
    V = np.asarray(V, np.float64)
    return float(np.linalg.norm(V.max(0) - V.min(0)))


def test_stage3_c1_matches_fp64_oracle(torch_cuda, c1_stage2):
    from oracle import s3_oracle as S
    from pamo_b200 import safe_project as SP

    V, F, v, f = c1_stage2
    want, _ = S.process(V, F, v.astype(np.float64), f, n_iters=5)
    sysm = SP.Stage3System()
    got, gf = SP.process(V, F, v, f, 5, system=sysm)
    assert np.array_equal(gf, f)
    err = np.abs(got - want).max() / _diag(V)
    moved = np.abs(want - v).max() / _diag(V)
    print(f"stage3 C1: max |fp32 - fp64| = {err:.3e} of bbox diag (moved {moved:.3e}), {sysm.last_stats}")
    assert moved > 10 * err  # the projection does move the mesh
    assert err < TOL_DIAG


def test_stage3_reduces_distance_to_gt(torch_cuda, c1_stage2):
    from oracle import s3_oracle as S
    from pamo_b200 import safe_project as SP

    V, F, v, f = c1_stage2
    got, _ = SP.process(V, F, v, f, 5)
    d0 = np.linalg.norm(S.closest_points_on_mesh(v.astype(np.float64), V.astype(np.float64), F) - v, axis=1).mean()
    d1 = np.linalg.norm(S.closest_points_on_mesh(got, V.astype(np.float64), F) - got, axis=1).mean()
    assert d1 < d0


def test_stage3_output_has_no_self_intersections(torch_cuda, c1_stage2):
    import pamo_b200
    from pamo_b200 import safe_project as SP

    V, F, v, f = c1_stage2
    got, _ = SP.process(V, F, v, f, 5)
    ctx = pamo_b200.Context(0)
    flags, _ = pamo_b200.self_intersect(ctx, torch_cuda.from_numpy(got.astype(np.float32)).cuda(),
                                        torch_cuda.from_numpy(f.astype(np.int32)).cuda())
    assert int(flags.sum()) == 0


def test_stage3_thin_shell_contacts(torch_cuda):
    """Two concentric shells 2e-3 apart, simplified, then projected: the contact
    barrier is active and the result stays intersection-free."""
    import pamo_b200
    from oracle import oracle as O
    from pamo_b200 import meshgen as mg
    from pamo_b200 import safe_project as SP

    V, F = mg.thin_shell_pair(8000, 2e-3, 3)
    v, f, _ = O.pamo_run_stage2(V, F, 0.2, min_verts=0)
    sysm = SP.Stage3System()
    got, _ = SP.process(V, F, v, f, 2, system=sysm)
    assert sysm.last_stats["contacts"] > 0
    assert np.isfinite(got).all()
    ctx = pamo_b200.Context(0)
    flags, _ = pamo_b200.self_intersect(ctx, torch_cuda.from_numpy(got.astype(np.float32)).cuda(),
                                        torch_cuda.from_numpy(f.astype(np.int32)).cuda())
    assert int(flags.sum()) == 0


def test_pamo_run_all_stages_but_remesh(torch_cuda):
    """PaMO(..., use_stage1=False, use_stage3=True).run returns host arrays with the
    stage-2 faces and projected vertices."""
    import pamo_b200
    from pamo_b200 import meshgen as mg

    V, F = mg.displaced_icosphere(4, 2)
    pm = pamo_b200.PaMO((V, F), use_stage1=False, use_stage3=True, verbose=False)
    v, f = pm.run(torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda(), 0.1, min_verts=0)
    assert v.shape[1] == 3 and f.shape[1] == 3 and len(f) <= int(0.1 * len(F))
    assert np.isfinite(v).all()


def test_pamo_run_keeps_ground_truth_between_runs(torch_cuda):
    """A PaMO object keeps its ground truth on the device after the first run
    (its normalisation, copies and hierarchy); later runs give what a fresh
    object gives, within the CG's summation-order noise."""
    import pamo_b200
    from pamo_b200 import meshgen as mg

    V, F = mg.displaced_icosphere(4, 2)
    V = V.astype(np.float32)
    args = (torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda(), 0.1)
    pm = pamo_b200.PaMO((V, F), use_stage1=False, use_stage3=True, verbose=False)
    v1, f1 = pm.run(*args, min_verts=0)
    assert pm.system._gt_norm is not None
    v2, f2 = pm.run(*args, min_verts=0)  # the kept ground truth
    fresh = pamo_b200.PaMO((V, F), use_stage1=False, use_stage3=True, verbose=False)
    v3, f3 = fresh.run(*args, min_verts=0)
    diag = float(np.linalg.norm(V.max(0) - V.min(0)))
    assert np.array_equal(f1, f2) and np.array_equal(f1, f3)
    assert np.abs(v2 - v3).max() / diag < 1e-6
    assert np.abs(v1 - v2).max() / diag < 1e-6
