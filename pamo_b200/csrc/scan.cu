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

// Single pass with decoupled look-back (see scan.cuh).  Header: [0] next tile,
// [1] finished blocks, [2] fault.  Status word of a tile: high half the call's
// epoch (30 bits) and a flag (1: the tile's own sum, 2: its inclusive prefix),
// low half the value; a word from an earlier call (another epoch) reads as not
// yet published.
constexpr unsigned kFlagSum = 1, kFlagPrefix = 2;

__device__ __forceinline__ unsigned long long status_word(unsigned epoch, unsigned flag, int value)
{
    return ((unsigned long long)((epoch << 2) | flag) << 32) | (unsigned)value;
}

// spin_limit bounds each wait (polls); absent_tile >= 0 makes that tile never
// publish (only the wait-timeout test passes one: its waiters must give up).
__global__ void __launch_bounds__(kScanThreads) k_scan_lookback(const int *in, int *out, long long n_max,
                                                                const int *d_n, int *scratch, int *d_total,
                                                                int *fault, unsigned epoch, long long spin_limit,
                                                                long long absent_tile)
{
    __shared__ int tile[kScanTile];
    __shared__ long long s_t;
    __shared__ int s_prefix;
    volatile unsigned long long *status = reinterpret_cast<volatile unsigned long long *>(scratch + kScanHeader);
    const long long n = d_n ? (long long)*d_n : n_max;
    const long long n_tiles = (n + kScanTile - 1) / kScanTile;
    if (threadIdx.x == 0) s_t = atomicAdd(&scratch[0], 1);
    __syncthreads();
    const long long t = s_t;
    if (t < n_tiles) {
        const long long base = t * kScanTile;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            long long i = base + (long long)k * kScanThreads + threadIdx.x;
            tile[k * kScanThreads + threadIdx.x] = i < n ? in[i] : 0;
        }
        __syncthreads();
        int local[kScanItems];
        int sum = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            local[k] = sum;
            sum += tile[threadIdx.x * kScanItems + k];
        }
        int agg;
        const int ex = block_excl_scan<kScanThreads>(sum, agg);
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            if (lane == 0 && t != absent_tile) status[t] = status_word(epoch, t == 0 ? kFlagPrefix : kFlagSum, agg);
            int prefix = 0;
            bool timed_out = false;
            for (long long top = t - 1; top >= 0 && !timed_out;) {
                // lane l looks at tile top - l (lane 0 the nearest)
                const long long j = top - lane;
                unsigned flag = kFlagPrefix;
                int val = 0;
                if (j >= 0) {
                    unsigned long long w = status[j];
                    for (long long spins = 0;; ++spins) {
                        const unsigned hi = (unsigned)(w >> 32);
                        if ((hi >> 2) == (epoch & 0x3FFFFFFFu) && (hi & 3u) != 0) {
                            flag = hi & 3u;
                            val = (int)(unsigned)w;
                            break;
                        }
                        if (spins > spin_limit) {  // a tile that started earlier never published
                            timed_out = true;
                            break;
                        }
                        __nanosleep(20);
                        w = status[j];
                    }
                }
                timed_out = __any_sync(0xffffffffu, timed_out);
                // the nearest tile with its prefix ends the look-back (a lane past
                // tile 0 counts as one, with value 0); before it, the tiles' sums
                const unsigned stops = __ballot_sync(0xffffffffu, flag == kFlagPrefix);
                const int stop = stops ? __ffs(stops) - 1 : 31;
                int v = lane <= stop ? val : 0;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                prefix += v;
                if (stops) break;
                top -= 32;
            }
            if (lane == 0) {
                if (timed_out) {
                    atomicExch(&scratch[2], 1);
                    if (fault) atomicExch(fault, 1);
                }
                if (t != absent_tile) status[t] = status_word(epoch, kFlagPrefix, prefix + agg);
                s_prefix = prefix;
                if (t == n_tiles - 1 && d_total) *d_total = prefix + agg;
            }
        }
        __syncthreads();
        const int off = s_prefix + ex;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) tile[threadIdx.x * kScanItems + k] = local[k] + off;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            long long i = base + (long long)k * kScanThreads + threadIdx.x;
            if (i < n) out[i] = tile[k * kScanThreads + threadIdx.x];
        }
    } else if (n_tiles == 0 && t == 0 && threadIdx.x == 0 && d_total) {
        *d_total = 0;
    }
    // the last block to finish leaves the header at zero for the next scan
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&scratch[1], 1) == (int)gridDim.x - 1) {
            scratch[0] = 0;
            scratch[1] = 0;
        }
    }
}

constexpr long long kScanSpinLimit = 1LL << 22;  // ~0.1 s of polls: far beyond any real wait

cudaError_t exclusive_scan(const int *in, int *out, long long n_max, const int *d_n, int *scratch, int *d_total,
                           cudaStream_t s, int *fault)
{
    return exclusive_scan_waits(in, out, n_max, d_n, scratch, d_total, s, fault, kScanSpinLimit, -1);
}

cudaError_t exclusive_scan_waits(const int *in, int *out, long long n_max, const int *d_n, int *scratch, int *d_total,
                                 cudaStream_t s, int *fault, long long spin_limit, long long absent_tile)
{
    static std::atomic<unsigned> epochs{0};
    if (n_max <= 0) {
        if (d_total) return cudaMemsetAsync(d_total, 0, sizeof(int), s);
        return cudaSuccess;
    }
    if (n_max <= (long long)kSingleThreads * kSingleItems) {
        launch(k_scan_single, 1, kSingleThreads, 0, s, in, out, n_max, d_n, d_total);
        return cudaGetLastError();
    }
    const long long tiles = (n_max + kScanTile - 1) / kScanTile;
    const unsigned epoch = (epochs.fetch_add(1, std::memory_order_relaxed) + 1) & 0x3FFFFFFFu;
    launch(k_scan_lookback, (unsigned)tiles, kScanThreads, 0, s, in, out, n_max, d_n, scratch, d_total, fault, epoch,
           spin_limit, absent_tile);
    return cudaGetLastError();
}

}  // namespace pamo
