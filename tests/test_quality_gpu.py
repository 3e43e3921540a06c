"""Quality mode of stage 2 (pamo_set_quality: FP64 quadrics, the quadric's
minimiser as collapse position, self-intersection undo by exact predicates):
on configs 1 and 2 its results reach the target, pass the exact-predicate
checker and the watertight / manifold checks, and their Hausdorff distance to
the input is reported next to the parity mode's and the unmodified
reference's; two runs give the same result."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _run(torch, V, F, ratio, quality):
    import pamo_b200
    from pamo_b200 import _lib

    ctx = pamo_b200.Context(0)
    if quality:
        pamo_b200.check("pamo_set_quality", _lib.lib().pamo_set_quality(ctx.handle, 1))
    v, f, rounds = pamo_b200.stage2_run(ctx, torch.from_numpy(V).cuda(), torch.from_numpy(F).cuda(),
                                        int(ratio * len(F)))
    return v.cpu().numpy(), f.cpu().numpy(), rounds


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_quality_mode_passes_acceptance(torch_cuda, name):
    from pamo_b200 import meshgen as mg
    from pamo_b200 import metrics

    if name == "c1":
        V, F = mg.displaced_icosphere(5, 0)
        ratio, k_in, k_out = 0.05, 2, 16
    else:
        V, F = mg.noisy_torus(1024, 1024, 0)
        ratio, k_in, k_out = 0.01, 1, 24
    vq, fq, rq = _run(torch_cuda, V, F, ratio, True)
    vq2, fq2, _ = _run(torch_cuda, V, F, ratio, True)
    assert np.array_equal(fq, fq2) and np.array_equal(vq.view(np.uint32), vq2.view(np.uint32))
    vp, fp, rp = _run(torch_cuda, V, F, ratio, False)
    chk = metrics.check_mesh(vq, fq)
    assert chk["intersection_free"] and chk["watertight_manifold"], chk
    assert len(fq) <= int(ratio * len(F))
    ref = np.load(os.path.join(GOLDEN, f"refrun_{name}.npz"))
    hq = metrics.hausdorff(V, F, vq, fq, k_in, k_out)
    hp = metrics.hausdorff(V, F, vp, fp, k_in, k_out)
    hr = metrics.hausdorff(V, F, ref["v"], ref["f"], k_in, k_out)
    diag = float(np.linalg.norm(V.astype(np.float64).max(0) - V.astype(np.float64).min(0)))
    print(f"quality {name}: {len(fq)} faces in {rq} rounds, Hausdorff {hq['hausdorff'] / diag:.3e} of diag "
          f"(parity mode {hp['hausdorff'] / diag:.3e} with {len(fp)} faces, reference {hr['hausdorff'] / diag:.3e}), "
          f"chamfer {hq['chamfer']:.3e} vs {hp['chamfer']:.3e}")
    assert hq["hausdorff"] <= hr["hausdorff"] + 1e-3 * diag
