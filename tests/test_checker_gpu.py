"""The device acceptance checker (pamo_check_mesh, pamo_mesh_distance) against
the rational / brute-force oracle (oracle/check_oracle.py), then the acceptance
criteria on config 1 and config 2: every output intersection-free under exact
predicates, watertight and manifold, at or below the target face count, and
with a two-sided Hausdorff distance to the input no worse than that of the
unmodified reference's own output (tests/golden/refrun_c{1,2}.npz) plus 1e-3 of
the bounding-box diagonal.  Config 2's stage-2 result is also compared bit for
bit with the oracle's run of the whole loop (tests/golden/c2_oracle.npz)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
HD_SLACK = 1e-3  # of the input's bounding-box diagonal


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _cases():
    from pamo_b200 import meshgen as mg
    from helpers import crafted_mesh

    g = np.load(os.path.join(GOLDEN, "isect.npz"))
    out = [("crafted", *crafted_mesh())]
    out += [(k, g[f"{k}_V"].astype(np.float32), g[f"{k}_F"].astype(np.int32))
            for k in ("two_spheres", "crumpled", "folded_grids", "soup")]
    V, F = mg.displaced_icosphere(3, 1)
    out.append(("icosphere3", V.astype(np.float32), F.astype(np.int32)))
    # an open grid (boundary edges), a duplicated face and a removed face
    n = 6
    xs, ys = np.meshgrid(np.arange(n, dtype=np.float32), np.arange(n, dtype=np.float32))
    Vg = np.stack([xs.ravel(), ys.ravel(), np.zeros(n * n, np.float32)], 1)
    q = [[i * n + j, i * n + j + 1, (i + 1) * n + j + 1] for i in range(n - 1) for j in range(n - 1)]
    q += [[i * n + j, (i + 1) * n + j + 1, (i + 1) * n + j] for i in range(n - 1) for j in range(n - 1)]
    Fg = np.array(q + [q[3], [-1, -1, -1]], np.int32)
    out.append(("grid_dup", Vg, Fg))
    return out


def test_checker_matches_rational_oracle(torch_cuda):
    from oracle import check_oracle as C
    from pamo_b200 import metrics

    keys = {"pairs": "intersecting_pairs", "degenerate": "degenerate_faces",
            "boundary_half_edges": "boundary_half_edges", "nonmanifold_half_edges": "nonmanifold_half_edges",
            "nonmanifold_vertices": "nonmanifold_vertices", "unreferenced_vertices": "unreferenced_vertices",
            "candidates": "candidate_pairs"}
    for name, V, F in _cases():
        want = C.check_mesh(V, F)
        got, flags = metrics.check_mesh(V, F, return_flags=True)
        for ko, kg in keys.items():
            assert got[kg] == want[ko], (name, kg, got[kg], want[ko])
        assert np.array_equal(flags, want["flags"]), (name, np.nonzero(flags != want["flags"])[0][:10])
        assert got["traversal_errors"] == 0
    # the intersecting fixtures are caught, the clean sphere passes
    res = {name: metrics.check_mesh(V, F) for name, V, F in _cases()}
    assert res["crumpled"]["intersecting_pairs"] > 0 and res["two_spheres"]["intersecting_pairs"] > 0
    assert res["icosphere3"]["intersection_free"] and res["icosphere3"]["watertight_manifold"]
    assert res["grid_dup"]["boundary_half_edges"] > 0 and res["grid_dup"]["nonmanifold_half_edges"] > 0


def test_checker_rejects_bad_indices(torch_cuda):
    from pamo_b200 import PamoError, metrics

    V = np.zeros((3, 3), np.float32)
    with pytest.raises(PamoError):
        metrics.check_mesh(V, np.array([[0, 1, 3]], np.int32))


def test_mesh_distance_matches_brute_force(torch_cuda):
    from oracle import check_oracle as C
    from pamo_b200 import meshgen as mg
    from pamo_b200 import metrics

    VA, FA = mg.displaced_icosphere(3, 1)
    VB, FB = mg.displaced_icosphere(2, 5)
    VB = VB * 1.05
    for k in (1, 3):
        got = metrics.mesh_distance(VA, FA, VB, FB, subdiv=k)
        P = C.face_samples(VA.astype(np.float32), FA, k)
        d = C.point_mesh_distances(P, VB.astype(np.float32), FB)
        assert got["samples"] == len(P)
        assert abs(got["max"] - d.max()) <= 1e-9 * max(1.0, d.max())
        assert abs(got["mean_sq"] - np.mean(d * d)) <= 1e-9 * max(1.0, np.mean(d * d))
        assert got["upper"] >= got["max"]
    # identical meshes are at distance 0
    same = metrics.hausdorff(VA, FA, VA, FA, 2, 2)
    assert same["hausdorff"] < 1e-6


def _diag(V):
    V = np.asarray(V, np.float64)
    return float(np.linalg.norm(V.max(0) - V.min(0)))


def _accept(V_in, F_in, v, f, ref_v, ref_f, target, subdiv_in, subdiv_out, label):
    from pamo_b200 import metrics

    chk = metrics.check_mesh(v, f)
    assert chk["intersection_free"], (label, chk)
    assert chk["watertight_manifold"], (label, chk)
    assert len(f) <= target, (label, len(f), target)
    ours = metrics.hausdorff(V_in, F_in, v, f, subdiv_in, subdiv_out)
    ref = metrics.hausdorff(V_in, F_in, ref_v, ref_f, subdiv_in, subdiv_out)
    diag = _diag(V_in)
    print(f"{label}: {len(f)} faces, Hausdorff {ours['hausdorff'] / diag:.3e} of diag "
          f"(reference {ref['hausdorff'] / diag:.3e}), upper {ours['upper'] / diag:.3e}")
    assert ours["hausdorff"] <= ref["hausdorff"] + HD_SLACK * diag, (label, ours, ref)
    return chk, ours, ref


def test_config1_outputs_pass_acceptance(torch_cuda):
    """Config 1 (level-5 displaced icosphere, ratio 0.05): stage 2 alone and
    stages 2 + 3, against the unmodified reference's stage-2 output."""
    import pamo_b200
    from pamo_b200 import meshgen as mg

    V, F = mg.displaced_icosphere(5, 0)
    ref = np.load(os.path.join(GOLDEN, "refrun_c1.npz"))
    target = int(0.05 * len(F))
    r_chk = pamo_b200.metrics.check_mesh(ref["v"], ref["f"])
    assert r_chk["intersection_free"]
    ctx = pamo_b200.Context(0)
    v2, f2, _ = pamo_b200.stage2_run(ctx, torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda(), target)
    _accept(V, F, v2.cpu().numpy(), f2.cpu().numpy(), ref["v"], ref["f"], target, 2, 16, "c1 stage 2")
    pm = pamo_b200.PaMO((V, F), use_stage1=False, use_stage3=True, verbose=False)
    v3, f3 = pm.run(torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda(), 0.05, min_verts=0)
    _accept(V, F, v3, f3, ref["v"], ref["f"], target, 2, 16, "c1 stages 2+3")


def test_config2_stage2_matches_oracle_and_passes_acceptance(torch_cuda):
    """Config 2 (1024 x 1024 noisy torus, 2,097,152 faces, ratio 0.01): the GPU
    loop equals the oracle's whole run bit for bit, and the result passes the
    checks against the unmodified reference's output."""
    import pamo_b200
    from pamo_b200 import meshgen as mg

    V, F = mg.noisy_torus(1024, 1024, 0)
    want = np.load(os.path.join(GOLDEN, "c2_oracle.npz"))
    target = int(0.01 * len(F))
    ctx = pamo_b200.Context(0)
    v, f, rounds = pamo_b200.stage2_run(ctx, torch_cuda.from_numpy(V).cuda(), torch_cuda.from_numpy(F).cuda(), target)
    v, f = v.cpu().numpy(), f.cpu().numpy()
    assert rounds == int(want["rounds"])
    assert np.array_equal(f, want["f"])
    assert np.array_equal(v.view(np.uint32), want["v"].view(np.uint32))
    ref = np.load(os.path.join(GOLDEN, "refrun_c2.npz"))
    _accept(V, F, v, f, ref["v"], ref["f"], target, 1, 24, "c2 stage 2")
