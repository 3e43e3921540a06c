"""Stage 1 (remeshing) on the GPU: pamo_remesh against its CPU restatement
(oracle/s1_oracle.py) bit for bit -- vertices, faces and the centring offset --
and PaMO.run with all three stages: the result is intersection-free under
exact predicates, watertight and manifold, at or below the target, and within
about one voxel of the input (the remesh offsets the surface by 0.9 / R)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _cases():
    from pamo_b200 import meshgen as mg

    yield "icosphere3 R32", mg.displaced_icosphere(3, 0), 32
    yield "icosphere5 R64", mg.displaced_icosphere(5, 0), 64
    yield "torus48 R48", mg.noisy_torus(48, 48, 2), 48
    yield "shell R40", mg.thin_shell_pair(4000, 2e-2, 1), 40


def test_remesh_matches_oracle(torch_cuda):
    import pamo_b200
    from oracle import s1_oracle as S1

    ctx = pamo_b200.Context(0)
    for name, (V, F), R in _cases():
        v, f, off = pamo_b200.remesh(ctx, torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda(), R)
        ov, of, om = S1.remesh(V, F, R)
        v, f = v.cpu().numpy(), f.cpu().numpy()
        assert np.array_equal(off.view(np.uint32), om.view(np.uint32)), name
        assert len(v) == len(ov) and len(f) == len(of), (name, len(v), len(ov), len(f), len(of))
        assert np.array_equal(f, of), name
        assert np.array_equal(v.view(np.uint32), ov.view(np.uint32)), (name, np.abs(v - ov).max())


def test_remesh_matches_oracle_at_benchmark_resolution(torch_cuda):
    """R = 256, config 2's resolution, on config 1's 20,480-face mesh (583,556
    faces out): the same bits as the CPU restatement (about 20 s of numpy)."""
    import pamo_b200
    from oracle import s1_oracle as S1
    from pamo_b200 import meshgen as mg

    V, F = mg.displaced_icosphere(5, 0)
    ctx = pamo_b200.Context(0)
    v, f, off = pamo_b200.remesh(ctx, torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda(), 256)
    ov, of, om = S1.remesh(V, F, 256)
    v, f = v.cpu().numpy(), f.cpu().numpy()
    assert np.array_equal(off.view(np.uint32), om.view(np.uint32))
    assert len(f) == len(of) == 583556
    assert np.array_equal(f, of)
    assert np.array_equal(v.view(np.uint32), ov.view(np.uint32))


def test_config2_stage2_after_remesh_matches_oracle(torch_cuda):
    """Config 2 as benchmarked: stage 1 on the 2,097,152-face torus on the
    device, then the stage-2 loop on its output as PaMO.run runs it with stage 1
    on (no second centring, the offset added back at the end), on the device
    and in the C restatement: the same rounds, faces and vertex bits."""
    import pamo_b200
    from oracle import oracle as O
    from pamo_b200 import meshgen as mg

    V, F = mg.noisy_torus(1024, 1024, 0)
    ctx = pamo_b200.Context(0)
    v1, f1, off = pamo_b200.remesh(ctx, torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda(), 256)
    target = int(0.01 * len(F))
    v2, f2, rounds = pamo_b200.stage2_run(pamo_b200.Context(0), v1, f1, target, offset=off)
    ov, of, orounds = O.Stage2Oracle().run(v1.cpu().numpy(), O.shuffle_faces(f1.cpu().numpy()), target, 4, 1e-3,
                                           1000000)
    assert rounds == orounds
    assert np.array_equal(f2.cpu().numpy(), of)
    assert np.array_equal(v2.cpu().numpy().view(np.uint32), (ov + off).astype(np.float32).view(np.uint32))


def test_remesh_output_is_closed_and_clean(torch_cuda):
    import pamo_b200
    from pamo_b200 import meshgen as mg

    ctx = pamo_b200.Context(0)
    V, F = mg.noisy_torus(256, 256, 0)
    v, f, off = pamo_b200.remesh(ctx, torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda(), 256)
    chk = pamo_b200.metrics.check_mesh(v, f)
    assert chk["intersection_free"] and chk["watertight_manifold"], chk
    assert chk["unreferenced_vertices"] == 0


@pytest.mark.parametrize("ratio", [0.05])
def test_pamo_run_all_three_stages(torch_cuda, ratio):
    import pamo_b200
    from pamo_b200 import meshgen as mg

    V, F = mg.displaced_icosphere(5, 0)
    pm = pamo_b200.PaMO((V, F), use_stage1=True, use_stage3=True, verbose=False)
    v, f = pm.run(torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda(), ratio, min_verts=0)
    target = int(ratio * len(F))
    assert len(f) <= target and pm.stage1_faces > len(f)
    chk = pamo_b200.metrics.check_mesh(v, f)
    assert chk["intersection_free"] and chk["watertight_manifold"], chk
    hd = pamo_b200.metrics.hausdorff(V, F, v, f, 2, 16)
    # the same run without stage 1
    pm2 = pamo_b200.PaMO((V, F), use_stage1=False, use_stage3=True, verbose=False)
    v2, f2 = pm2.run(torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda(), ratio, min_verts=0)
    hd2 = pamo_b200.metrics.hausdorff(V, F, v2, f2, 2, 16)
    R = pamo_b200.stage1_resolution(target)
    extent = float((V.max(0) - V.min(0)).max())
    voxel = extent * (1 + 6.0 / R) / R  # one grid step in the input's units
    print(f"stage 1+2+3 on config 1: {pm.stage1_faces} remeshed faces -> {len(f)}, Hausdorff "
          f"{hd['hausdorff'] / voxel:.2f} voxels (stages 2+3 alone: {hd2['hausdorff'] / voxel:.2f})")
    # the remesh moves the surface out by 0.9 voxel, plus up to one voxel of
    # sampling error: the result stays within that of the stage-1-free run
    assert hd["hausdorff"] < hd2["hausdorff"] + 2.0 * voxel
