"""Acceptance checks of a result mesh on the device (libpamo_b200.so):

* ``check_mesh(V, F)`` -- exact-predicate self-intersection test of every pair
  of faces with overlapping boxes, degenerate faces, and the manifold /
  watertight checks (pamo_check_mesh).  It takes the role of the reference's
  CGAL self-intersection script
  (simp_cuda/safe_project/scripts/cgal_intersect/main.cpp:19-111).
* ``hausdorff(VA, FA, VB, FB)`` -- two-sided surface distance by dense
  sampling, with upper bounds (pamo_mesh_distance); the reference's
  metrics.py:31-51 computes the same terms with igl and trimesh.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check

CHECK_KEYS = ["intersecting_pairs", "intersecting_faces", "degenerate_faces", "boundary_half_edges",
              "nonmanifold_half_edges", "nonmanifold_vertices", "unreferenced_vertices", "candidate_pairs",
              "dead_faces", "traversal_errors", "bad_indices"]


def _dev(x, dtype, device):
    import torch

    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(x, dtype={torch.float32: np.float32, torch.int32: np.int32}[dtype])
                            ).to(device)


def _stream(device):
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def check_mesh(V, F, device=0, return_flags=False):
    """Counts of the checks (CHECK_KEYS) for mesh (V [n,3], F [m,3]); with
    return_flags also the per-face intersection flags (numpy uint8)."""
    import torch

    dev = torch.device("cuda", device)
    v = _dev(V, torch.float32, dev)
    f = _dev(F, torch.int32, dev)
    flags = torch.zeros(int(f.shape[0]), dtype=torch.uint8, device=dev)
    out = (ctypes.c_longlong * len(CHECK_KEYS))()
    check("pamo_check_mesh", _lib.lib().pamo_check_mesh(v.data_ptr(), f.data_ptr(), int(v.shape[0]), int(f.shape[0]),
                                                        flags.data_ptr(), out, _stream(dev)))
    res = {k: int(out[i]) for i, k in enumerate(CHECK_KEYS)}
    res["watertight_manifold"] = all(res[k] == 0 for k in CHECK_KEYS[2:6])
    res["intersection_free"] = res["intersecting_pairs"] == 0
    if return_flags:
        return res, flags.cpu().numpy()
    return res


def mesh_distance(VA, FA, VB, FB, subdiv=4, device=0):
    """One-sided distance A -> B: {max, upper, mean_sq, samples}."""
    import torch

    dev = torch.device("cuda", device)
    va, fa = _dev(VA, torch.float32, dev), _dev(FA, torch.int32, dev)
    vb, fb = _dev(VB, torch.float32, dev), _dev(FB, torch.int32, dev)
    out = (ctypes.c_double * 4)()
    check("pamo_mesh_distance", _lib.lib().pamo_mesh_distance(
        va.data_ptr(), fa.data_ptr(), int(va.shape[0]), int(fa.shape[0]), vb.data_ptr(), fb.data_ptr(),
        int(vb.shape[0]), int(fb.shape[0]), int(subdiv), out, _stream(dev)))
    return {"max": out[0], "upper": out[1], "mean_sq": out[2], "samples": int(out[3])}


def hausdorff(VA, FA, VB, FB, subdiv_a=4, subdiv_b=4, device=0):
    """Two-sided Hausdorff distance between the surfaces of A and B by sampling:
    {"hausdorff": max of both directions, "upper": its bound, "a_to_b", "b_to_a",
    "chamfer": sum of the two mean squared distances}."""
    ab = mesh_distance(VA, FA, VB, FB, subdiv_a, device)
    ba = mesh_distance(VB, FB, VA, FA, subdiv_b, device)
    return {"hausdorff": max(ab["max"], ba["max"]), "upper": max(ab["upper"], ba["upper"]), "a_to_b": ab,
            "b_to_a": ba, "chamfer": ab["mean_sq"] + ba["mean_sq"]}
