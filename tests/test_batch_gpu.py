"""Batched stage 2 (pamo_batch_*): every mesh's result in a batch equals the
plain device loop's result for that mesh on a fresh context, bit for bit --
alone, in a mix of families and sizes, with meshes joining while others run,
and with admission held back by the packed capacity and the memory budget.
The plain loop itself is checked against the oracle in test_stage2_gpu.py."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _plain(torch, V, F, target, tolerance=4, threshold=1e-3, iters=1000000):
    import pamo_b200

    ctx = pamo_b200.Context(0)  # fresh context: no state from earlier runs
    v, f, rounds = pamo_b200.stage2_run(ctx, torch.from_numpy(V).cuda(), torch.from_numpy(F).cuda(), target,
                                        tolerance, threshold, iters)
    return v.cpu().numpy(), f.cpu().numpy(), rounds


def _mix():
    from pamo_b200 import meshgen as mg

    meshes = [
        (mg.displaced_icosphere(4, 1), 0.05),
        (mg.noisy_torus(48, 40, 2), 0.01),
        (mg.thin_shell_pair(6000, 2e-3, 3), 0.05),  # undo passes in most rounds
        (mg.displaced_geodesic(9000, 4), 0.001),
        (mg.icosphere(3), 0.2),  # regular sphere: reaches the stuck / tolerance path
        (mg.noisy_torus(16, 12, 5), 0.05),
    ]
    return [(V.astype(np.float32), F.astype(np.int32), r) for (V, F), r in meshes]


def _same(a, b):
    return a[0].shape == b[0].shape and a[1].shape == b[1].shape and np.array_equal(
        a[0].view(np.uint32), b[0].view(np.uint32)) and np.array_equal(a[1], b[1])


def test_batch_matches_plain_on_a_mix(torch_cuda):
    from pamo_b200.batch import BatchEngine, target_faces

    mix = _mix()
    want = [_plain(torch_cuda, V, F, target_faces(len(F), r, 0)) for V, F, r in mix]
    eng = BatchEngine(max_faces=sum(len(F) for _, F, _ in mix), max_meshes=16)
    jobs = [eng.submit(V, F, r, min_verts=0) for V, F, r in mix]
    eng.run()
    for (V, F, r), j, w in zip(mix, jobs, want):
        info = eng.job(j)
        got = eng.result(j)
        assert info["rounds"] == w[2], (len(F), info["rounds"], w[2])
        assert _same(got, w[:2]), f"{len(F)} faces: batch result differs from the plain loop"


def test_batch_alone_equals_in_the_mix(torch_cuda):
    from pamo_b200.batch import BatchEngine

    mix = _mix()
    eng = BatchEngine(max_faces=sum(len(F) for _, F, _ in mix), max_meshes=16)
    jobs = [eng.submit(V, F, r, min_verts=0) for V, F, r in mix]
    eng.run()
    together = [eng.result(j) for j in jobs]
    for (V, F, r), t in zip(mix, together):
        j = eng.submit(V, F, r, min_verts=0)
        eng.run()
        assert _same(eng.result(j), t)


def test_batch_admits_while_running(torch_cuda):
    """Continuous batching: meshes submitted between rounds join the running
    ones; a capacity that holds only part of the mix keeps the rest pending
    until room frees up.  Every result still equals the plain loop's."""
    from pamo_b200.batch import BatchEngine, target_faces

    mix = _mix()
    want = [_plain(torch_cuda, V, F, target_faces(len(F), r, 0)) for V, F, r in mix]
    biggest = max(len(F) for _, F, _ in mix)
    eng = BatchEngine(max_faces=biggest + 3000, max_meshes=3)
    jobs = {}
    saw_pending = False
    for k, (V, F, r) in enumerate(mix):
        jobs[k] = eng.submit(V, F, r, min_verts=0)
        running, pending = eng.step()
        saw_pending = saw_pending or pending > 0
    eng.run()
    assert saw_pending
    for k, w in enumerate(want):
        assert _same(eng.result(jobs[k]), w[:2]), f"mesh {k}"


def test_batch_memory_budget_and_errors(torch_cuda):
    from pamo_b200 import _lib
    from pamo_b200 import meshgen as mg
    from pamo_b200.batch import BatchEngine, target_faces

    V, F = mg.displaced_icosphere(3, 0)
    V, F = V.astype(np.float32), F.astype(np.int32)
    want = _plain(torch_cuda, V, F, target_faces(len(F), 0.1, 0))
    # a budget for one mesh's round state (plus the queued inputs) at a time:
    # per mesh the engine holds edge costs, vertex map, invalid table and three
    # undo lists of 16 (n + 1) + 6 m + 16 entries
    n0, m0 = len(V), len(F)
    al = lambda b: (b + 255) // 256 * 256
    region = al(64) + al((3 * m0 + 1) * 4) + al((n0 + 1) * 4) + 3 * al((16 * (n0 + 1) + 6 * m0 + 16) * 4) + al(n0 + 1)
    eng = BatchEngine(max_faces=100_000, max_meshes=8, memory_budget=int(1.5 * region) + 3 * 12 * (n0 + m0))
    jobs = [eng.submit(V, F, 0.1, min_verts=0) for _ in range(3)]
    running, pending = eng.step()
    assert running == 1 and pending == 2
    eng.run()
    for j in jobs:
        assert _same(eng.result(j), want[:2])
    bad = F.copy()
    bad[5, 1] = len(V)  # index out of range: rejected before anything runs
    with pytest.raises(_lib.PamoError):
        eng.submit(V, bad, 0.1, min_verts=0)
    with pytest.raises(_lib.PamoError):
        eng.submit(np.zeros((10, 3), np.float32), np.zeros((200_000, 3), np.int32), 0.1)  # beyond max_faces
