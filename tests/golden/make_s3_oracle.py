"""Generates the stage-3 golden fixtures: the FP64 oracle (oracle/s3_oracle.py)
run of pamo_safe_project.process on stage-2 results computed by the stage-2
oracle (bit-identical to the CUDA stage 2, tests/test_stage2_gpu.py):

  s3_c1.npz        config 1: level-5 displaced icosphere, ratio 0.05, 5 steps
                   (no contact within reach)
  s3_shell8k.npz   thin-shell pair, 7,840 faces, gap 2e-3, ratio 0.2, 2 steps:
                   ~30,000 contact blocks within d_hat, CCD steps below 1
  s3_shell500k.npz config 3's thin-shell pair: two concentric displaced spheres
                   of 250k faces each (500,000 faces), gap 2e-3, ratio 0.05,
                   5 steps
  s3_c2step.npz    config 2's stage-3 input: the 20,604-face stage-2 result of
                   the 2,097,152-face torus (c2_oracle.npz, the same oracle),
                   one step (10 Newton iterations, ~790,000 contact blocks)

Each holds the stage-2 result (v float32, f), the projected vertices q
(float64) and the Newton trace (energy at the iterate, energy after the line
search, CCD step, last halving tried, contact blocks, blocks within d_hat).

    python tests/golden/make_s3_oracle.py --out tests/golden [--case c1|shell8k|shell500k|c2step]
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

CASES = {
    "c1": ("icosphere", 5, 0, 0.05, 5),
    "shell8k": ("shell", 8000, 3, 0.2, 2),
    "shell500k": ("shell", 500_000, 0, 0.05, 5),
    "c2step": ("torus", 1024, 0, 0.01, 1),
}


def case_input(name):
    from pamo_b200 import meshgen as mg

    kind, size, seed, ratio, steps = CASES[name]
    if kind == "icosphere":
        V, F = mg.displaced_icosphere(size, seed)
    elif kind == "torus":
        V, F = mg.noisy_torus(size, size, seed)
    else:
        V, F = mg.thin_shell_pair(size, 2e-3, seed)
    return V, F, ratio, steps


def run(name, out_dir):
    from oracle import oracle as O
    from oracle import s3_oracle as S

    V, F, ratio, steps = case_input(name)
    t0 = time.time()
    if name == "c2step":  # the stage-2 oracle's result for this input is already a fixture
        fx = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "c2_oracle.npz"))
        v, f = fx["v"], fx["f"]
    else:
        v, f, rounds = O.pamo_run_stage2(V, F, ratio, min_verts=0)
    t1 = time.time()
    trace = []
    q, _ = S.process(V, F, v.astype(np.float64), f, n_iters=steps, trace=trace)
    t2 = time.time()
    np.savez_compressed(os.path.join(out_dir, f"s3_{name}.npz"), v=v.astype(np.float32), f=f.astype(np.int32),
                        q=q.astype(np.float64), trace=np.array(trace, np.float64), steps=np.int64(steps))
    print(f"{name}: {len(F)} -> {len(f)} faces ({t1 - t0:.1f} s), stage 3 {len(trace)} Newton iterations "
          f"({t2 - t1:.1f} s), max blocks within d_hat {max([r[5] for r in trace] or [0])}", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--case", default=None, choices=list(CASES))
    a = ap.parse_args()
    for name in [a.case] if a.case else list(CASES):
        run(name, a.out)


if __name__ == "__main__":
    main()
