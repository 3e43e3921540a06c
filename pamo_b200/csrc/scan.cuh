// Device-wide exclusive prefix sums and block-level scan helpers.
//
// One launch per scan: tiles of 2048 items take their index from a counter in
// the order their blocks start, and each adds the totals of the tiles before it
// as they publish them (decoupled look-back: a tile publishes its own sum at
// once and its inclusive prefix when it has it, so a tile waits only on tiles
// that started earlier).  The waits spin with a limit and record a fault when
// it runs out.  Results are deterministic.  The item count may live in device
// memory (d_n), in which case n_max only sizes the grid.
//
// The scratch (scan_scratch_ints(n_max) ints) must be all zero before its first
// scan (scan_scratch_init); every scan leaves its counters zero again.  Scans
// on one scratch must not overlap.
#pragma once

#include "common.cuh"

namespace pamo {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int warp_incl_scan(int v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Exclusive scan of one int per thread across a block of BLOCK threads; the
// block total is returned in `total` (all threads).
template <int BLOCK>
__device__ __forceinline__ int block_excl_scan(int v, int &total)
{
    __shared__ int warp_sums[BLOCK / 32];
    __shared__ int s_total;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = warp_incl_scan(v);
    if (lane == 31) warp_sums[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int s = lane < BLOCK / 32 ? warp_sums[lane] : 0;
        int si = warp_incl_scan(s);
        if (lane < BLOCK / 32) warp_sums[lane] = si - s;
        if (lane == 31) s_total = si;
    }
    __syncthreads();
    int excl = warp_sums[wid] + inc - v;
    total = s_total;
    __syncthreads();  // shared slots may be reused by the next call
    return excl;
}

template <int BLOCK>
__device__ __forceinline__ int block_reduce_sum(int v)
{
    __shared__ int ws[BLOCK / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) ws[wid] = v;
    __syncthreads();
    int r = 0;
    if (wid == 0) {
        r = lane < BLOCK / 32 ? ws[lane] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;  // valid in thread 0
}

__global__ void k_scan_reduce(const int *__restrict__ in, long long n_max, const int *d_n, int *__restrict__ tile_sums);
__global__ void k_scan_tile_sums(int *tile_sums, long long n_tiles_max, long long n_max, const int *d_n, int *d_total);
__global__ void k_scan_down(const int *in, int *out, long long n_max, const int *d_n, const int *__restrict__ tile_sums);

// Scratch needed by exclusive_scan for up to n_max items (ints): a header of
// kScanHeader ints, then one 64-bit status word per tile.
constexpr int kScanHeader = 8;
constexpr long long scan_scratch_ints(long long n_max) { return kScanHeader + 2 * ((n_max + kScanTile - 1) / kScanTile) + 2; }

// Zeroes a freshly allocated scratch of `ints` ints.
inline cudaError_t scan_scratch_init(int *scratch, long long ints, cudaStream_t s = 0)
{
    return cudaMemsetAsync(scratch, 0, (size_t)ints * sizeof(int), s);
}

// out[i] = sum_{j<i} in[i] for i < n, with n = d_n ? *d_n : n_max.  in may equal
// out.  If d_total is non-null the grand total is written there.  If fault is
// non-null, 1 is written there when a wait ran out (the scratch header keeps a
// copy in any case).
cudaError_t exclusive_scan(const int *in, int *out, long long n_max, const int *d_n, int *scratch, int *d_total,
                           cudaStream_t s, int *fault = nullptr);

// exclusive_scan with each look-back wait bounded by `spin_limit` polls, and
// tile `absent_tile` (>= 0) never publishing -- for the test that makes the
// waits run out (pamo_debug_wait_timeout); -1 for a normal scan.
cudaError_t exclusive_scan_waits(const int *in, int *out, long long n_max, const int *d_n, int *scratch, int *d_total,
                                 cudaStream_t s, int *fault, long long spin_limit, long long absent_tile);

}  // namespace pamo
