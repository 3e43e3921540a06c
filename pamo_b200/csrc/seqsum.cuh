// The float32 chain sum of numpy's mean(axis=0) over a C-contiguous (n, 3)
// float32 array: per column s = x[0], then s = fl(s + x[k]) for k = 1 .. n-1
// (round to nearest even), divided by n -- evaluated exactly, in parallel.
#pragma once

#include <cuda_runtime.h>

namespace pamo {

// Rows below which seq_mean3 runs the plain one-thread chain (its scratch need
// is then 0).
constexpr long long kSeqMeanBlockedMin = 4096;

// Device scratch bytes seq_mean3 needs for n rows.
size_t seq_mean_scratch_bytes(long long n);

// out[c] = fl(chain sum of x_c[0 .. n-1]) / n for c = 0, 1, 2 (device arrays of
// n floats; out: 3 device floats).  scratch: seq_mean_scratch_bytes(n) bytes of
// device memory, 16-byte aligned.  n <= 0 writes nothing.
cudaError_t seq_mean3(const float *x0, const float *x1, const float *x2, long long n, void *scratch, float *out,
                      cudaStream_t s);

}  // namespace pamo
