"""Generates tests/golden/c2_oracle.npz: the whole stage-2 loop of PaMO.run on
the 1024 x 1024 noisy torus (2,097,152 faces, ratio 0.01, min_verts 0) run by
the CPU oracle (oracle/s2_oracle.c, pinned to the reference's own kernels by
tests/test_golden.py).  The GPU path must reproduce it bit for bit
(tests/test_checker_gpu.py).  Takes about 80 s on 8 host threads.

    python tests/golden/make_c2_oracle.py --out tests/golden/c2_oracle.npz
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    from oracle import oracle as O
    from pamo_b200 import meshgen as mg

    V, F = mg.noisy_torus(1024, 1024, 0)
    t0 = time.time()
    v, f, rounds = O.pamo_run_stage2(V, F, 0.01, min_verts=0)
    print(f"{len(F)} -> {len(f)} faces in {rounds} rounds, {time.time() - t0:.1f} s")
    np.savez_compressed(a.out, v=v.astype(np.float32), f=f.astype(np.int32), rounds=np.int64(rounds))


if __name__ == "__main__":
    main()
