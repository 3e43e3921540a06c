"""Stage-3 host preparation (pamo_b200/safe_project.py and the library's
pamo_mesh_hinges): the unique edges, the hinges and trimesh-style vertex
merging give exactly what the plain numpy forms (np.unique with axis /
return_index / return_inverse, lexsort) give, on closed meshes, on meshes with
duplicated and near-duplicated vertices, on grids with many equal coordinates
and on an open patch (where the builder declines and numpy takes over)."""
import numpy as np
import pytest

from pamo_b200 import meshgen as mg
from pamo_b200 import safe_project as sp


def _edges_ref(F):
    F = np.asarray(F, np.int64)
    x = np.concatenate([F[:, 0], F[:, 1], F[:, 2]])
    y = np.concatenate([F[:, 1], F[:, 2], F[:, 0]])
    n = int(F.max()) + 1
    k = np.unique(np.minimum(x, y) * n + np.maximum(x, y))
    return np.stack([k // n, k % n], axis=1)


def _hinges_ref(F):
    F = np.asarray(F, np.int64)
    D = np.concatenate([np.stack([F[:, k], F[:, (k + 1) % 3], F[:, (k + 2) % 3]], 1) for k in range(3)])
    n = int(F.max()) + 1
    fwd, bwd = D[D[:, 0] < D[:, 1]], D[D[:, 0] > D[:, 1]]
    kf, kb = fwd[:, 0] * n + fwd[:, 1], bwd[:, 1] * n + bwd[:, 0]
    ob = np.argsort(kb, kind="stable")
    kbs = kb[ob]
    pos = np.searchsorted(kbs, kf)
    ok = (pos < len(kbs)) & (kbs[np.minimum(pos, len(kbs) - 1)] == kf)
    H = np.stack([fwd[ok, 2], fwd[ok, 0], fwd[ok, 1], bwd[ob][pos[ok], 2]], 1)
    return H[np.lexsort((H[:, 2], H[:, 1]))]


def _merge_ref(V, F, digits=8):
    V = np.asarray(V, np.float64)
    _, first, inv = np.unique(np.round(V, digits), axis=0, return_index=True, return_inverse=True)
    order = np.argsort(first)
    rank = np.empty_like(order)
    rank[order] = np.arange(len(order))
    return V[first[order]], rank[inv.reshape(-1)][np.asarray(F)]


def _cases():
    out = [mg.icosphere(3), mg.noisy_torus(40, 30, 1), mg.thin_shell_pair(3000, 2e-3, 3), mg.displaced_icosphere(3, 2)]
    V, F = mg.icosphere(2)
    n0 = len(V)
    V2, F2 = np.concatenate([V, V[:5]]), F.copy()  # five duplicated vertices, each used by one face
    for k in range(5):
        F2[np.where(F2[:, 0] == k)[0][:1], 0] = n0 + k
    out.append((V2, F2))
    V3 = V.copy()
    V3[:, 0] = np.round(V3[:, 0], 1)  # many equal x, no equal rows
    out.append((V3, F))
    V4 = V3.copy()
    V4[30] = V4[31]
    V4[40] = V4[41] + 1e-10  # equal after rounding to 8 digits
    out.append((V4, F))
    Vo, Fo = mg.icosphere(2)
    out.append((Vo, Fo[:60]))  # an open patch: boundary edges have one face
    return out


def test_mesh_hinges_rejects_bad_input():
    import ctypes

    from pamo_b200 import _lib

    F = np.ascontiguousarray(mg.icosphere(1)[1], np.int32)
    E, H, ne = np.empty((100, 2), np.int32), np.empty((100, 4), np.int32), ctypes.c_int()
    L = _lib.lib()
    assert L.pamo_mesh_hinges(F.ctypes.data, len(F), int(F.max()), E.ctypes.data, H.ctypes.data, ctypes.byref(ne)) \
        == 1  # PAMO_ERR_INVALID_ARG: an index equal to n_pts
    assert L.pamo_mesh_hinges(F.ctypes.data, 10, int(F.max()) + 1, E.ctypes.data, H.ctypes.data, ctypes.byref(ne)) \
        == 6  # PAMO_ERR_CAPACITY: open, edges with one face


@pytest.mark.parametrize("case", range(8))
def test_host_prep_matches_numpy_forms(case):
    V, F = _cases()[case]
    assert np.array_equal(sp.edges_unique(F), _edges_ref(F))
    assert np.array_equal(sp.hinges(F), _hinges_ref(F))
    E, H = sp.edges_and_hinges(F)  # the library's host builder on closed meshes
    assert np.array_equal(E, _edges_ref(F))
    assert np.array_equal(H, _hinges_ref(F))
    a, b = sp.merge_vertices(V, F), _merge_ref(V, F)
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(np.asarray(a[1]), np.asarray(b[1]))
