"""The library's device waits are bounded: a prefix scan in which one tile
never publishes, and the persistent CG solve in which one block never
publishes its partial sums, both give up after a short poll limit, record the
fault and return, and the call reports PAMO_ERR_DEVICE (what a real fault of
that kind reports).  Nothing hangs, and the same context then runs normal work
correctly.  The failure is a flag that nothing sets; no kernel faults."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PAMO_ERR_DEVICE = 4
SPIN_LIMIT = 4096  # polls per wait (~ms) instead of the production ~seconds


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _stream(torch):
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def test_scan_wait_runs_out_and_context_recovers(torch_cuda):
    import time

    import pamo_b200
    from oracle import oracle as O
    from pamo_b200 import _lib
    from pamo_b200 import meshgen as mg

    ctx = pamo_b200.Context(0)
    t0 = time.time()
    rc = _lib.lib().pamo_debug_wait_timeout(ctx.handle, 0, SPIN_LIMIT, _stream(torch_cuda))
    assert rc == PAMO_ERR_DEVICE
    assert time.time() - t0 < 30
    # the same context and the scans it uses still give the oracle's result
    V, F = mg.displaced_icosphere(4, 0)
    v, f, rounds = pamo_b200.stage2_run(ctx, torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda(),
                                        int(0.1 * len(F)))
    ov, of, orounds = O.pamo_run_stage2(V, F, 0.1, min_verts=0)
    assert rounds == orounds and np.array_equal(f.cpu().numpy(), of)


def test_cg_wait_runs_out_and_context_recovers(torch_cuda):
    import time

    import pamo_b200
    from pamo_b200 import _lib

    ctx = pamo_b200.Context(0)
    t0 = time.time()
    rc = _lib.lib().pamo_debug_wait_timeout(ctx.handle, 1, SPIN_LIMIT, _stream(torch_cuda))
    if rc == 1:
        pytest.skip("the device runs the CG without the persistent solve: no waits")
    assert rc == PAMO_ERR_DEVICE
    assert time.time() - t0 < 30
    # a normal solve on the same context: diagonal system 2 x = 1
    n = 64
    dev = torch_cuda.device("cuda", 0)
    row_ptr = torch_cuda.arange(n + 1, dtype=torch_cuda.int32, device=dev)
    col = torch_cuda.arange(n, dtype=torch_cuda.int32, device=dev)
    blocks = torch_cuda.zeros((n, 9), dtype=torch_cuda.float32, device=dev)
    blocks[:, [0, 4, 8]] = 2.0
    diag = torch_cuda.full((3 * n,), 2.0, dtype=torch_cuda.float32, device=dev)
    rhs = torch_cuda.ones(3 * n, dtype=torch_cuda.float32, device=dev)
    out = torch_cuda.empty(3 * n, dtype=torch_cuda.float32, device=dev)
    rc = _lib.lib().pamo_bsr_pcg(ctx.handle, n, row_ptr.data_ptr(), col.data_ptr(), blocks.data_ptr(), n,
                                 diag.data_ptr(), rhs.data_ptr(), 5, out.data_ptr(), _stream(torch_cuda))
    assert rc == 0
    assert np.allclose(out.cpu().numpy(), 0.5, atol=1e-6)
