"""Stage 3's mesh preparation on the device: pamo_mesh_hinges_device against the
host builder (pamo_mesh_hinges, itself checked against the oracle's
edges_unique / hinges on the CPU), and pamo_merge_check_device against the host
merge (merge_vertices, trimesh's process=True rounding to 8 decimals)."""
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


def _device_hinges(torch, F, n_pts):
    from pamo_b200 import _lib

    d_f = torch.from_numpy(np.ascontiguousarray(F, np.int32)).cuda()
    cap = max((3 * len(F)) // 2, 1)
    d_e = torch.empty((cap, 2), dtype=torch.int32, device="cuda")
    d_h = torch.empty((cap, 4), dtype=torch.int32, device="cuda")
    ne = ctypes.c_int(0)
    rc = _lib.lib().pamo_mesh_hinges_device(d_f.data_ptr(), len(F), n_pts, d_e.data_ptr(), d_h.data_ptr(),
                                            ctypes.byref(ne), None)
    return rc, d_e[:ne.value].cpu().numpy(), d_h[:ne.value].cpu().numpy()


def _host_hinges(F, n_pts):
    from pamo_b200 import _lib

    F32 = np.ascontiguousarray(F, np.int32)
    cap = (3 * len(F)) // 2 + 1
    E, H = np.empty((cap, 2), np.int32), np.empty((cap, 4), np.int32)
    ne = ctypes.c_int(0)
    rc = _lib.lib().pamo_mesh_hinges(F32.ctypes.data, len(F32), n_pts, E.ctypes.data, H.ctypes.data, ctypes.byref(ne))
    return rc, E[:ne.value], H[:ne.value]


def test_device_hinges_equal_host_builder(torch_cuda):
    from pamo_b200 import meshgen as mg

    rng = np.random.default_rng(0)
    for V, F in (mg.displaced_icosphere(3, 0), mg.noisy_torus(48, 40, 1), mg.noisy_torus(101, 102, 1),
                 mg.thin_shell_pair(4000, 2e-2, 1)):
        # shuffled faces and vertex numbers: the rows must still match
        perm = rng.permutation(len(V))
        F2 = perm[F][rng.permutation(len(F))]
        for FF in (F, F2):
            rd, Ed, Hd = _device_hinges(torch_cuda, FF, len(V))
            rh, Eh, Hh = _host_hinges(FF, len(V))
            assert rd == 0 and rh == 0
            assert np.array_equal(Ed, Eh) and np.array_equal(Hd, Hh)
            assert len(Ed) == 3 * len(FF) // 2


def test_device_hinges_reject_what_the_host_rejects(torch_cuda):
    from pamo_b200 import meshgen as mg

    V, F = mg.displaced_icosphere(2, 0)
    open_mesh = F[1:]  # a hole: boundary edges
    assert _device_hinges(torch_cuda, open_mesh[:-1], len(V))[0] == 6
    doubled = np.concatenate([F, F[:2]])  # two edges in four faces
    assert _device_hinges(torch_cuda, doubled, len(V))[0] == 6
    flipped = F.copy()
    flipped[0] = flipped[0, ::-1]  # an edge used twice the same way
    assert _device_hinges(torch_cuda, flipped, len(V))[0] == _host_hinges(flipped, len(V))[0] == 6
    bad = F.copy()
    bad[3, 1] = len(V)
    assert _device_hinges(torch_cuda, bad, len(V))[0] == 1


def test_merge_check_matches_host_merge(torch_cuda):
    from pamo_b200 import meshgen as mg
    from pamo_b200.safe_project import has_duplicate_vertices, merge_vertices

    V, F = mg.noisy_torus(64, 64, 0)
    assert not has_duplicate_vertices(torch_cuda.from_numpy(V).cuda())
    v2, _ = merge_vertices(V.astype(np.float64), F)
    assert len(v2) == len(V)
    # a copy of a vertex, and a point that rounds to the same 8 decimals as
    # another: each merges on the host and is reported on the device
    W0 = np.concatenate([V, np.array([[0.01, 0.2, 0.3]], np.float32)])
    near = np.nextafter(np.float32(0.01), np.float32(1.0))  # 0.01 + 9e-10: the same after rounding
    for extra in (V[5], np.array([near, 0.2, 0.3], np.float32)):
        W = np.concatenate([W0, extra[None]]).astype(np.float32)
        merged, _ = merge_vertices(W.astype(np.float64), F)
        assert len(merged) < len(W)
        assert has_duplicate_vertices(torch_cuda.from_numpy(W).cuda())
    # signed zeros compare equal: reported (the host merge then decides)
    W = np.concatenate([V, np.array([[0.0, 1.0, 2.0], [-0.0, 1.0, 2.0]], np.float32)])
    assert has_duplicate_vertices(torch_cuda.from_numpy(W).cuda())
    # differing in the 8th decimal after rounding: kept apart on both sides
    W = np.concatenate([V, (V[9] + np.float32(3e-6))[None]]).astype(np.float32)
    merged, _ = merge_vertices(W.astype(np.float64), F)
    assert len(merged) == len(W)
    assert not has_duplicate_vertices(torch_cuda.from_numpy(W).cuda())
