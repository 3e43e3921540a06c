"""Generates the golden vectors in tests/golden/ by running the REFERENCE's own
stage-2 build (oracle/_ref/, compiled from the reference sources by
oracle/build_ref.sh) on a CUDA device.

    python tests/golden/make_golden.py --out <directory>

Cases (each in a fresh process, so the reference's persistent state starts
empty as it does for a new CUDSP_Free object):
  * round sequences driven like PaMO.run (simp_cuda/pamo/__init__.py:148-185)
    through ref_round_canonical (the reference kernels with the per-vertex face
    lists sorted), recording every round's outputs;
  * selfx::self_intersect face flags on meshes that do intersect;
  * pow(float,2) as the reference kernels evaluate it, against the single
    rounding of x*x;
  * timing and output statistics of the unmodified reference (PaMO.run-style
    loop over CUSimp_Free::forward, and the pamo_simplify C-ABI).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from oracle import ref as R  # noqa: E402
from pamo_b200 import meshgen as mg  # noqa: E402


def meshes():
    return {
        "ico3": (lambda: mg.displaced_icosphere(3, 0), 0.001, 60),
        "shell4k": (lambda: mg.thin_shell_pair(4000, 2e-3, 2), 0.01, 12),
        "c1": (lambda: mg.displaced_icosphere(5, 0), 0.05, 1),
    }


def prepare(V, F):
    tm = O.tris_mean(V, F)
    P = (V - tm).astype(np.float32)
    T = O.shuffle_faces(F)
    sx = P[:, 0].max() - P[:, 0].min()
    sy = P[:, 1].max() - P[:, 1].min()
    sz = P[:, 2].max() - P[:, 2].min()
    scale = np.float32(max(max(sx, sy), sz))
    return P, T, scale


def run_sequence(name, out_dir):
    gen, ratio, max_rounds = meshes()[name]
    V, F = gen()
    P, T, scale = prepare(V, F)
    rec = {"P0": P, "T0": T, "scale": np.float32(scale), "threshold": np.float32(1e-3), "ratio": np.float32(ratio)}
    undo = np.zeros(0, np.int32)
    stuck = 0
    count = 0
    target = int(ratio * len(F))
    r = 0
    for r in range(max_rounds):
        prev = len(T)
        o = R.round_canonical(P, T, undo, scale, 1e-3, stuck)
        rec[f"r{r}_stuck"] = np.int32(stuck)
        for k in ("pts", "tris", "occ", "map", "undo", "cost", "collapsed", "isect0"):
            rec[f"r{r}_{k}"] = o[k]
        rec[f"r{r}_stats"] = np.array([o["n_edges"], o["n_main"], o["n_total"], o["undo_passes"], len(o["undo"]),
                                       o["undo0"]], np.int32)
        undo = o["undo"]
        P = o["pts"][o["occ"].astype(bool)]
        keep = o["tris"][:, 0] >= 0
        T = o["map"][o["tris"][keep]].astype(np.int32)
        cur = len(T)
        if cur <= target or cur <= 10:
            break
        if cur == prev:
            count += 1
        else:
            count = 0
            stuck = 0
        if count >= 2:
            stuck = 1
        if count == 4:
            break
    rec["n_rounds"] = np.int32(r + 1)
    np.savez_compressed(os.path.join(out_dir, f"seq_{name}.npz"), **rec)
    print(name, "rounds", r + 1, "faces", len(T), flush=True)


def isect_cases():
    rng = np.random.default_rng(5)
    cases = {}
    # two interpenetrating displaced spheres
    a = mg.displaced_icosphere(3, 1)
    b = mg.displaced_icosphere(3, 2)
    V = np.concatenate([a[0], b[0] + np.float32([0.6, 0.1, 0.0])]).astype(np.float32)
    F = np.concatenate([a[1], b[1] + len(a[0])]).astype(np.int32)
    cases["two_spheres"] = (V, F)
    # crumpled sphere: strong per-vertex noise folds the surface through itself
    V, F = mg.displaced_icosphere(3, 3)
    V = (V * (1.0 + 0.35 * rng.standard_normal((len(V), 1)))).astype(np.float32)
    cases["crumpled"] = (V, F)
    # small grid in the z=0 plane folded back onto itself (coplanar and shared-vertex pairs)
    n = 12
    xs, ys = np.meshgrid(np.arange(n, dtype=np.float32), np.arange(n, dtype=np.float32), indexing="ij")
    G = np.stack([xs.ravel() * 0.1, ys.ravel() * 0.1, np.zeros(n * n, np.float32)], 1)
    G2 = G.copy()
    G2[:, 2] = 0.05 * np.sin(G2[:, 0] * 20.0)
    G2[:, 0] += 0.03
    V = np.concatenate([G, G2]).astype(np.float32)
    quads = []
    for i in range(n - 1):
        for j in range(n - 1):
            p = i * n + j
            quads += [[p, p + n, p + n + 1], [p, p + n + 1, p + 1]]
    Q = np.array(quads, np.int32)
    F = np.concatenate([Q, Q + n * n]).astype(np.int32)
    cases["folded_grids"] = (V, F)
    # triangle soup in a unit box, with vertex reuse so shared-vertex paths occur
    V = rng.uniform(-0.5, 0.5, (300, 3)).astype(np.float32)
    F = rng.integers(0, 300, (600, 3)).astype(np.int32)
    F = F[(F[:, 0] != F[:, 1]) & (F[:, 1] != F[:, 2]) & (F[:, 0] != F[:, 2])]
    cases["soup"] = (V, F)
    return cases


def run_isect(out_dir):
    rec = {}
    for name, (V, F) in isect_cases().items():
        flags = R.self_intersect_flags(V, F)
        rec[f"{name}_V"] = V
        rec[f"{name}_F"] = F
        rec[f"{name}_flags"] = flags
        print(name, "faces", len(F), "flagged", int(flags.sum()), flush=True)
    np.savez_compressed(os.path.join(out_dir, "isect.npz"), **rec)


def run_pow2(out_dir):
    rng = np.random.default_rng(7)
    x = np.concatenate([
        np.exp(rng.uniform(np.log(1e-8), np.log(1e3), 4_000_000)),
        rng.uniform(0.0, 1.0, 2_000_000),
        np.array([0.0, 1.0, 2.0, 3.0, 1e-20, 1e19, 7.25, 0.1, 0.3], np.float64),
    ]).astype(np.float32)
    y = R.pow2(x)
    sq = (x * x).astype(np.float32)
    bad = y.view(np.uint32) != sq.view(np.uint32)
    mism = int(np.sum(bad))
    res = {"n": int(len(x)), "mismatch_vs_single_rounded_square": mism,
           "x": [float(v) for v in x[bad][:200]], "x_bits": [int(v) for v in x[bad][:200].view(np.uint32)],
           "pow_bits": [int(v) for v in y[bad][:200].view(np.uint32)],
           "sq_bits": [int(v) for v in sq[bad][:200].view(np.uint32)]}
    json.dump(res, open(os.path.join(out_dir, "pow2_probe.json"), "w"))
    print("pow2", res, flush=True)


def run_ref_timing(out_dir):
    import torch

    res = {}
    for name, gen, ratio in (("c1", lambda: mg.displaced_icosphere(5, 0), 0.05),
                             ("c2", lambda: mg.noisy_torus(1024, 1024, 0), 0.01)):
        V, F = gen()
        P = torch.from_numpy(V).cuda()
        T = torch.from_numpy(F).cuda()
        times = []
        st = {}
        for rep in range(2 if name == "c2" else 3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            v, f = R.pamo_run_stage2_torch(P, T, ratio, min_verts=0, stats=st)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        res[name] = {"faces_in": int(len(F)), "faces_out": int(len(f)), "verts_out": int(len(v)),
                     "rounds": st.get("rounds"), "seconds": times}
        np.savez_compressed(os.path.join(out_dir, f"refrun_{name}.npz"), v=v.astype(np.float32), f=f.astype(np.int32))
        print(name, res[name], flush=True)
    json.dump(res, open(os.path.join(out_dir, "ref_timing.json"), "w"), indent=1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory for the generated fixtures")
    ap.add_argument("--case", default=None)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    if args.case is None:
        for case in ["pow2", "isect", *meshes().keys(), "timing"]:
            subprocess.run([sys.executable, __file__, "--out", args.out, "--case", case], check=True)
        return
    if args.case == "pow2":
        run_pow2(args.out)
    elif args.case == "isect":
        run_isect(args.out)
    elif args.case == "timing":
        run_ref_timing(args.out)
    else:
        run_sequence(args.case, args.out)
    # the reference keeps thrust vectors in a static object whose destructor
    # runs after the CUDA runtime unloads; leave without running it
    sys.stdout.flush()
    os._exit(0)


if __name__ == "__main__":
    main()
