#include "scan.cuh"

namespace pamo {

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const int *__restrict__ in, long long n_max,
                                                              const int *d_n, int *__restrict__ tile_sums)
{
    long long n = d_n ? (long long)*d_n : n_max;
    long long base = (long long)blockIdx.x * kScanTile;
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        long long i = base + (long long)k * kScanThreads + threadIdx.x;
        if (i < n) sum += in[i];
    }
    int r = block_reduce_sum<kScanThreads>(sum);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = r;
}

// One block: exclusive scan of the tile sums in place, in chunks of 1024.
__global__ void __launch_bounds__(1024) k_scan_tile_sums(int *tile_sums, long long n_tiles_max, long long n_max,
                                                         const int *d_n, int *d_total)
{
    long long n = d_n ? (long long)*d_n : n_max;
    long long n_tiles = (n + kScanTile - 1) / kScanTile;
    if (n_tiles > n_tiles_max) n_tiles = n_tiles_max;
    int carry = 0;
    for (long long c = 0; c < n_tiles; c += 1024) {
        long long i = c + threadIdx.x;
        int v = i < n_tiles ? tile_sums[i] : 0;
        int tot;
        int ex = block_excl_scan<1024>(v, tot);
        if (i < n_tiles) tile_sums[i] = ex + carry;
        carry += tot;
    }
    if (threadIdx.x == 0 && d_total) *d_total = carry;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_down(const int *in, int *out, long long n_max, const int *d_n,
                                                            const int *__restrict__ tile_sums)
{
    __shared__ int tile[kScanTile];
    long long n = d_n ? (long long)*d_n : n_max;
    long long base = (long long)blockIdx.x * kScanTile;
    if (base >= n) return;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        long long i = base + (long long)k * kScanThreads + threadIdx.x;
        tile[k * kScanThreads + threadIdx.x] = i < n ? in[i] : 0;
    }
    __syncthreads();
    int local[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        local[k] = s;
        s += tile[threadIdx.x * kScanItems + k];
    }
    int tot;
    int ex = block_excl_scan<kScanThreads>(s, tot);
    int off = tile_sums[blockIdx.x] + ex;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) tile[threadIdx.x * kScanItems + k] = local[k] + off;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        long long i = base + (long long)k * kScanThreads + threadIdx.x;
        if (i < n) out[i] = tile[k * kScanThreads + threadIdx.x];
    }
}

// Small inputs: one block, 16 consecutive items per thread.
constexpr int kSingleThreads = 1024;
constexpr int kSingleItems = 16;

__global__ void __launch_bounds__(kSingleThreads) k_scan_single(const int *in, int *out, long long n_max,
                                                                const int *d_n, int *d_total)
{
    const long long n = d_n ? (long long)*d_n : n_max;
    const long long base = (long long)threadIdx.x * kSingleItems;
    int v[kSingleItems];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kSingleItems; ++k) {
        long long i = base + k;
        v[k] = i < n ? in[i] : 0;
        sum += v[k];
    }
    int tot;
    int ex = block_excl_scan<kSingleThreads>(sum, tot);
#pragma unroll
    for (int k = 0; k < kSingleItems; ++k) {
        long long i = base + k;
        if (i < n) out[i] = ex;
        ex += v[k];
    }
    if (threadIdx.x == 0 && d_total) *d_total = tot;
}

cudaError_t exclusive_scan(const int *in, int *out, long long n_max, const int *d_n, int *scratch, int *d_total,
                           cudaStream_t s)
{
    if (n_max <= 0) {
        if (d_total) return cudaMemsetAsync(d_total, 0, sizeof(int), s);
        return cudaSuccess;
    }
    if (n_max <= (long long)kSingleThreads * kSingleItems) {
        launch(k_scan_single, 1, kSingleThreads, 0, s, in, out, n_max, d_n, d_total);
        return cudaGetLastError();
    }
    long long tiles = (n_max + kScanTile - 1) / kScanTile;
    launch(k_scan_reduce, (unsigned)tiles, kScanThreads, 0, s, in, n_max, d_n, scratch);
    launch(k_scan_tile_sums, 1, 1024, 0, s, scratch, tiles, n_max, d_n, d_total);
    launch(k_scan_down, (unsigned)tiles, kScanThreads, 0, s, in, out, n_max, d_n, scratch);
    return cudaGetLastError();
}

}  // namespace pamo
