#!/usr/bin/env bash
# Compiles the reference's own stage-2 CUDA sources (read in place from the
# reference tree; nothing is copied) into oracle/_ref/ with the reference's nvcc
# flags (simp_cuda/setup.py:34) for sm_100a:
#   oracle/_ref/libref_harness.so   ref_harness.cu + cusimp_free.cu + bvh/*.cuh
#   oracle/_ref/libpamo_ref_cabi.so pamo_blender/cusimpinterface.cu (pamo_simplify)
# --expt-relaxed-constexpr is needed because the kernels call
# std::numeric_limits<>::max() in device code (torch's extension build adds it).
set -euo pipefail
REF=${PAMO_REFERENCE:-/root/reference}
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
mkdir -p "$OUT"
if [ ! -f "$REF/simp_cuda/src/cusimp_free.cu" ]; then
  echo "reference sources not found under $REF; keeping existing $OUT" >&2
  exit 0
fi
if [ -f "$OUT/libref_harness.so" ] && [ -f "$OUT/libpamo_ref_cabi.so" ] \
   && [ "$OUT/libref_harness.so" -nt "$HERE/ref_harness.cu" ] && [ "$OUT/libref_harness.so" -nt "$0" ]; then
  exit 0  # up to date
fi
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
FLAGS="-O3 --extended-lambda --expt-relaxed-constexpr --fmad=false -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -shared -w"
"$NVCC" $FLAGS -I"$REF/simp_cuda/src" "$HERE/ref_harness.cu" -o "$OUT/libref_harness.so"
"$NVCC" $FLAGS "$REF/pamo_blender/cusimpinterface.cu" -o "$OUT/libpamo_ref_cabi.so"
echo "built $OUT"
