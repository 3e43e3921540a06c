"""pamo_self_intersect_noalloc: the self-intersection check for callers that
cannot allocate device memory (a host application owning all device memory
through its own pool, or a latency-critical loop that must not let cudaMalloc
synchronise the device).  It keeps its scratch in a fixed device array inside
the library.  Through the C ABI its flags and candidate-pair counts must equal
those of pamo_self_intersect, which allocates its buffers in a context, on two
calls in a row (the array keeps the previous call's contents)."""
import ctypes
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


def _noalloc(torch, V, F):
    from pamo_b200 import _lib

    pv = torch.from_numpy(np.ascontiguousarray(V, np.float32)).cuda()
    pf = torch.from_numpy(np.ascontiguousarray(F, np.int32)).cuda()
    out = torch.full((len(F),), 7, dtype=torch.uint8, device="cuda")  # stale garbage must be cleared
    n = ctypes.c_longlong(-1)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = _lib.lib().pamo_self_intersect_noalloc(pv.data_ptr(), pf.data_ptr(), len(V), len(F), out.data_ptr(),
                                                ctypes.byref(n), stream)
    return rc, out.cpu().numpy(), n.value


def _meshes():
    from pamo_b200 import meshgen as mg

    g = np.load(os.path.join(GOLDEN, "isect.npz"))
    cases = [(g[f"{k}_V"], g[f"{k}_F"]) for k in ("two_spheres", "crumpled", "folded_grids", "soup")]
    cases.append(mg.displaced_icosphere(5, 0))
    cases.append(mg.thin_shell_pair(20000, 2e-3, 1))
    # removed faces (-1, -1, -1) spread through an intersecting mesh
    V, F = cases[1]
    F = np.array(F, np.int32)
    F[::7] = -1
    cases.append((V, F))
    return cases


def test_noalloc_matches_allocating_entry_point(torch_cuda):
    import pamo_b200

    ctx = pamo_b200.Context(0)
    for V, F in _meshes():
        want, want_pairs = pamo_b200.self_intersect(ctx, torch_cuda.from_numpy(np.ascontiguousarray(V)).cuda(),
                                                    torch_cuda.from_numpy(np.ascontiguousarray(F)).cuda())
        want = want.cpu().numpy()
        for call in range(2):  # two calls in a row share the device array
            rc, got, pairs = _noalloc(torch_cuda, V, F)
            assert rc == 0, f"status {rc}"
            assert np.array_equal(got, want), f"call {call}: {np.sum(got != want)} flags differ"
            assert pairs == want_pairs


def test_noalloc_empty_mesh(torch_cuda):
    """No faces: status OK and no candidate pairs, with or without points."""
    from pamo_b200 import _lib

    n = ctypes.c_longlong(-1)
    stream = ctypes.c_void_p(torch_cuda.cuda.current_stream().cuda_stream)
    assert _lib.lib().pamo_self_intersect_noalloc(None, None, 0, 0, None, ctypes.byref(n), stream) == 0
    assert n.value == 0
    pv = torch_cuda.zeros((4, 3), dtype=torch_cuda.float32, device="cuda")
    n.value = -1
    assert _lib.lib().pamo_self_intersect_noalloc(pv.data_ptr(), None, 4, 0, None, ctypes.byref(n), stream) == 0
    assert n.value == 0


def test_noalloc_rejects_sizes_beyond_its_limit(torch_cuda):
    from pamo_b200 import meshgen as mg

    V, F = mg.displaced_icosphere(6, 0)  # 81,920 faces > 32,768
    rc, _, _ = _noalloc(torch_cuda, V, F)
    assert rc == 6  # PAMO_ERR_CAPACITY
