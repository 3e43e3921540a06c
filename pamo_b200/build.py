"""Builds pamo_b200/libpamo_b200.so from pamo_b200/csrc/*.cu for sm_100a.

    python -m pamo_b200.build [--force] [-j N]

Every translation unit that feeds a stage-2 decision is compiled with
--fmad=false (no multiply-add contraction): the reference is built that way
(simp_cuda/setup.py:34) and its collapse/intersection decisions depend on the
exact fp32/fp64 rounding sequence.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpamo_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", os.path.join(ROOT, "include")]
# translation units whose arithmetic must round exactly like the reference
# (checker.cu: its exact predicates' error-free sums need one rounding per operation;
# stage1.cu: its FP64 distances follow the CPU restatement's operation order)
NO_FMA = {"stage2.cu", "lbvh.cu", "scan.cu", "abi.cu", "shuffle.cu", "noalloc.cu", "checker.cu", "stage1.cu"}


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _deps_mtime():
    hdr = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hdr.append(os.path.join(ROOT, "include", "pamo_b200.h"))
    return max(os.path.getmtime(h) for h in hdr if os.path.exists(h))


def _compile(src: str, force: bool) -> str:
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(path), _deps_mtime()):
        return obj
    if src.endswith(".cpp"):  # host-only code
        cmd = [CXX, "-O3", "-std=c++17", "-fPIC", "-pthread", "-I", os.path.join(ROOT, "include"), "-c", path, "-o", obj]
    else:
        flags = list(COMMON)
        if src in NO_FMA:
            flags.append("--fmad=false")
        cmd = [NVCC, *ARCH, *flags, "-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int = 8, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(LIB)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    a = ap.parse_args()
    build(force=a.force, jobs=a.j, verbose=True)


if __name__ == "__main__":
    sys.exit(main())
