// Exact parallel form of the float32 chain sum s = x[0], s = fl(s + x[k]).
//
// While every partial sum of a run of steps lies strictly inside one binade
// [2^e, 2^(e+1)) of one sign, each of them is a multiple of u = 2^(e-23), and
// fl(s + x) = s + u * rne(x / u): the rounding of x to the grid does not depend
// on s, except for a tie (x / u = a + 1/2), which goes to whichever of a, a + 1
// makes the new s / u even -- a function of the parity of s / u.  A run of steps
// is then an integer sum whose ties read the running parity: a transducer with
// two states (entry parity 0 or 1 -> total increment, exit parity), and
// composing two of them is associative, so a warp scans 32 steps at once.  The
// minimum and maximum of the running increments decide, from the entry state
// alone, whether every step of the run stays strictly inside the binade (the
// condition for the integer form to hold step by step).
//
// Passes, for blocks of 32 elements of x[1 ..]:
//   k_sm_block_sums  the double-precision sum of each block;
//   k_sm_predict     their exclusive scan from x[0]: an estimate of the value the
//                    chain enters each block with, whose binade is the one the
//                    block's summary is made for;
//   k_sm_summaries   per block the transducer relative to that binade (total
//                    increment and exit parity for either entry parity, the
//                    running increments' minimum and maximum), or "none" when an
//                    element cannot be one step inside it (too large, not finite);
//   k_sm_walk        one thread per column walks the blocks: a block whose binade
//                    is the running state's and whose bounds hold is one integer
//                    add; any other block is added element by element in float32.
// The estimate only chooses which binade a summary is made for: the walk's checks
// make the result the chain's, bit for bit, whatever the estimate was.
#include <cstdint>

#include "common.cuh"
#include "seqsum.cuh"

namespace pamo {
namespace {

constexpr int kSmBlock = 32;            // elements per summary block (one warp)
constexpr int kSmChunk = 512;           // blocks per shared-memory chunk of the walk
constexpr int kSmWalkThreads = 1024;
constexpr int kSmPredictThreads = 1024;
constexpr int kT23 = 1 << 23, kT24 = 1 << 24;

// ecode of a block: sign << 8 | biased exponent of the binade; < 0: no summary
struct __align__(16) SumBlock {
    int ecode, inc0, inc1, outs;  // outs: bit 0 exit parity from entry parity 0, bit 1 from 1
    int mn0, mx0, mn1, mx1;       // minimum / maximum running increment, entry parity 0 / 1
};

inline long long n_blocks(long long n) { return n > 1 ? (n - 1 + kSmBlock - 1) / kSmBlock : 0; }

inline size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

// Element k of column c's blocks (k >= 1); -0.0 past the end, which leaves any
// float32 sum unchanged (s + -0 == s for every s, signed zeros included).
__device__ __forceinline__ float elem(const float *x, long long n, long long k) { return k < n ? x[k] : -0.0f; }

__global__ void k_sm_block_sums(const float *x0, const float *x1, const float *x2, long long n, long long nb,
                                double *D)
{
    const int lane = threadIdx.x & 31;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < 3 * nb; w += warps) {
        const int c = (int)(w / nb);
        const long long b = w - (long long)c * nb;
        const float *x = c == 0 ? x0 : (c == 1 ? x1 : x2);
        double d = (double)elem(x, n, 1 + b * kSmBlock + lane);
#pragma unroll
        for (int off = 16; off; off >>= 1) d += __shfl_xor_sync(0xffffffffu, d, off);
        if (lane == 0) D[w] = d;
    }
}

// One block per column: E[b] = x[0] + D[0] + ... + D[b-1] in double, in place.
__global__ void __launch_bounds__(kSmPredictThreads) k_sm_predict(const float *x0, const float *x1, const float *x2,
                                                                 long long nb, double *D)
{
    __shared__ double warp_tot[kSmPredictThreads / 32];
    const int c = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const float *x = c == 0 ? x0 : (c == 1 ? x1 : x2);
    double *E = D + (long long)c * nb;
    const long long per = (nb + kSmPredictThreads - 1) / kSmPredictThreads;
    const long long lo = (long long)t * per, hi = lo + per < nb ? lo + per : nb;
    double mine = 0.0;
    for (long long b = lo; b < hi; ++b) mine += E[b];
    double incl = mine;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double o = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += o;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    double before = (double)x[0];
    for (int w = 0; w < warp; ++w) before += warp_tot[w];
    before += incl - mine;
    for (long long b = lo; b < hi; ++b) {
        const double d = E[b];
        E[b] = before;
        before += d;
    }
}

// x relative to u = 2^(e - 23): kind 0: x / u rounds to a (exactly or not);
// kind 1: x / u = a + 1/2 exactly (a tie); kind 2: no step inside the binade
// can add it (|x| >= 2^(e+2), or not finite).
__device__ __forceinline__ int classify(float x, int e, int &a)
{
    const unsigned bits = __float_as_uint(x);
    const int E = (int)((bits >> 23) & 0xFFu);
    const unsigned man = bits & 0x7FFFFFu;
    a = 0;
    if (E == 255) return 2;
    if (E == 0 && man == 0) return 0;
    const int M = (int)(E ? (man | 0x800000u) : man);
    const int q = E ? E - 150 : -149;  // |x| = M * 2^q
    const int sh = q - (e - 23);
    const bool neg = bits >> 31;
    if (sh >= 2) return 2;
    if (sh >= 0) {
        a = neg ? -(M << sh) : (M << sh);
        return 0;
    }
    const int d = -sh;
    if (d >= 26) return 0;  // |x / u| < 1/4: rounds to 0
    const int fl = M >> d, rem = M & ((1 << d) - 1), half = 1 << (d - 1);
    if (rem == half) {
        a = neg ? -(fl + 1) : fl;  // candidates a, a + 1
        return 1;
    }
    const int r = fl + (rem > half ? 1 : 0);
    a = neg ? -r : r;
    return 0;
}

__global__ void k_sm_summaries(const float *x0, const float *x1, const float *x2, long long n, long long nb,
                               const double *E, SumBlock *S)
{
    const int lane = threadIdx.x & 31;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < 3 * nb; w += warps) {
        const int c = (int)(w / nb);
        const long long b = w - (long long)c * nb;
        const float *x = c == 0 ? x0 : (c == 1 ? x1 : x2);
        const unsigned eb = __float_as_uint((float)E[w]);
        const int E8 = (int)((eb >> 23) & 0xFFu);
        bool none = E8 == 0 || E8 == 255;
        int a = 0, kind = 0;
        if (!none) kind = classify(elem(x, n, 1 + b * kSmBlock + lane), E8 - 127, a);
        none = __any_sync(0xffffffffu, none || kind == 2);
        if (none) {
            if (lane == 0) S[w] = SumBlock{-1, 0, 0, 0, 0, 0, 0, 0};
            continue;
        }
        // this element's transducer: increment and exit parity per entry parity p
        int i0, i1, o0, o1;
        if (kind == 1) {
            i0 = (a & 1) ? a + 1 : a;  // N + a even with N even
            i1 = (a & 1) ? a : a + 1;  // N + a even with N odd
            o0 = o1 = 0;
        } else {
            i0 = i1 = a;
            o0 = a & 1;
            o1 = o0 ^ 1;
        }
        // inclusive scan: earlier steps first
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int pi0 = __shfl_up_sync(0xffffffffu, i0, off), pi1 = __shfl_up_sync(0xffffffffu, i1, off);
            const int po = __shfl_up_sync(0xffffffffu, o0 | (o1 << 1), off);
            if (lane >= off) {
                const int po0 = po & 1, po1 = po >> 1;
                const int n0 = pi0 + (po0 ? i1 : i0), n1 = pi1 + (po1 ? i1 : i0);
                const int q0 = po0 ? o1 : o0, q1 = po1 ? o1 : o0;
                i0 = n0;
                i1 = n1;
                o0 = q0;
                o1 = q1;
            }
        }
        int mn0 = i0, mx0 = i0, mn1 = i1, mx1 = i1;
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            mn0 = min(mn0, __shfl_xor_sync(0xffffffffu, mn0, off));
            mx0 = max(mx0, __shfl_xor_sync(0xffffffffu, mx0, off));
            mn1 = min(mn1, __shfl_xor_sync(0xffffffffu, mn1, off));
            mx1 = max(mx1, __shfl_xor_sync(0xffffffffu, mx1, off));
        }
        if (lane == 31) S[w] = SumBlock{(int)((eb >> 31) << 8) | E8, i0, i1, o0 | (o1 << 1), mn0, mx0, mn1, mx1};
    }
}

// One block per column.  Thread 0 walks; the other warps copy the next chunk of
// elements and summaries into the other shared-memory buffer meanwhile.
__global__ void __launch_bounds__(kSmWalkThreads) k_sm_walk(const float *x0, const float *x1, const float *x2,
                                                            long long n, long long nb, const SumBlock *S, float *out)
{
    extern __shared__ float4 sm4[];  // 2 x (kSmChunk * kSmBlock floats, then kSmChunk summaries)
    const int c = blockIdx.x;
    const float *x = c == 0 ? x0 : (c == 1 ? x1 : x2);
    const SumBlock *Sc = S + (long long)c * nb;
    constexpr int kBufFloats = kSmChunk * kSmBlock + kSmChunk * (int)(sizeof(SumBlock) / 4);
    float *smf = reinterpret_cast<float *>(sm4);
    const long long n_chunks = (nb + kSmChunk - 1) / kSmChunk;
    auto load = [&](long long q, int buf) {
        float *xs = smf + buf * kBufFloats;
        SumBlock *ss = reinterpret_cast<SumBlock *>(xs + kSmChunk * kSmBlock);
        const long long b0 = q * kSmChunk;
        const int nbk = (int)(nb - b0 < kSmChunk ? nb - b0 : kSmChunk);
        const long long k0 = 1 + b0 * kSmBlock;
        for (int i = threadIdx.x - 32; i < nbk * kSmBlock; i += kSmWalkThreads - 32) xs[i] = elem(x, n, k0 + i);
        for (int i = threadIdx.x - 32; i < nbk; i += kSmWalkThreads - 32) ss[i] = Sc[b0 + i];
    };
    if (threadIdx.x >= 32) load(0, 0);
    __syncthreads();
    float s = x[0];
    bool imode = false;  // the state is (ec, N): |s| = N * 2^(e - 23), N in [2^23, 2^24)
    int ec = 0, N = 0;
    for (long long q = 0; q < n_chunks; ++q) {
        const int buf = (int)(q & 1);
        if (threadIdx.x >= 32) {
            if (q + 1 < n_chunks) load(q + 1, buf ^ 1);
        } else if (threadIdx.x == 0) {
            const float *xs = smf + buf * kBufFloats;
            const int4 *ss4 = reinterpret_cast<const int4 *>(xs + kSmChunk * kSmBlock);
            const int nbk = (int)(nb - q * kSmChunk < kSmChunk ? nb - q * kSmChunk : kSmChunk);
            int4 h0 = ss4[0], h1 = ss4[1];
            for (int i = 0; i < nbk; ++i) {
                const int j = i + 1 < nbk ? i + 1 : i;  // the next summary, loaded ahead
                const int4 g0 = ss4[2 * j], g1 = ss4[2 * j + 1];
                if (!imode) {
                    const unsigned bits = __float_as_uint(s);
                    const int E8 = (int)((bits >> 23) & 0xFFu);
                    if (E8 != 0 && E8 != 255) {
                        imode = true;
                        ec = (int)((bits >> 31) << 8) | E8;
                        N = (int)((bits & 0x7FFFFFu) | 0x800000u);
                    }
                }
                bool jumped = false;
                if (imode && h0.x == ec) {
                    const bool p = N & 1;
                    const int inc = p ? h0.z : h0.y, mn = p ? h1.z : h1.x, mx = p ? h1.w : h1.y;
                    const bool neg = ec & 0x100;
                    // every step's |s| / u stays in [2^23 + 1, 2^24 - 1]
                    const int lo = neg ? N - mx : N + mn, hi = neg ? N - mn : N + mx;
                    if (lo >= kT23 + 1 && hi <= kT24 - 1) {
                        N = neg ? N - inc : N + inc;
                        jumped = true;
                    }
                }
                if (!jumped) {
                    if (imode) {
                        s = __uint_as_float(((unsigned)(ec >> 8) << 31) | ((unsigned)(ec & 0xFF) << 23) |
                                            ((unsigned)N & 0x7FFFFFu));
                        imode = false;
                    }
                    const float4 *x4 = reinterpret_cast<const float4 *>(xs + i * kSmBlock);
#pragma unroll
                    for (int v = 0; v < kSmBlock / 4; ++v) {
                        const float4 t = x4[v];
                        s = __fadd_rn(s, t.x);
                        s = __fadd_rn(s, t.y);
                        s = __fadd_rn(s, t.z);
                        s = __fadd_rn(s, t.w);
                    }
                }
                h0 = g0;
                h1 = g1;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (imode)
            s = __uint_as_float(((unsigned)(ec >> 8) << 31) | ((unsigned)(ec & 0xFF) << 23) | ((unsigned)N & 0x7FFFFFu));
        out[c] = __fdiv_rn(s, (float)n);
    }
}

// The plain chain for short columns: one thread per column.
__global__ void k_sm_chain(const float *x0, const float *x1, const float *x2, long long n, float *out)
{
    const int c = threadIdx.x;
    if (c >= 3) return;
    const float *x = c == 0 ? x0 : (c == 1 ? x1 : x2);
    float s = x[0];
    for (long long k = 1; k < n; ++k) s = __fadd_rn(s, x[k]);
    out[c] = __fdiv_rn(s, (float)n);
}

}  // namespace

size_t seq_mean_scratch_bytes(long long n)
{
    if (n < kSeqMeanBlockedMin) return 0;
    const long long nb = n_blocks(n);
    return align16((size_t)(3 * nb) * sizeof(double)) + (size_t)(3 * nb) * sizeof(SumBlock);
}

cudaError_t seq_mean3(const float *x0, const float *x1, const float *x2, long long n, void *scratch, float *out,
                      cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    if (n < kSeqMeanBlockedMin) {
        launch(k_sm_chain, 1, 32, 0, s, x0, x1, x2, n, out);
        return cudaGetLastError();
    }
    const long long nb = n_blocks(n);
    double *D = static_cast<double *>(scratch);
    SumBlock *S = reinterpret_cast<SumBlock *>(static_cast<char *>(scratch) + align16((size_t)(3 * nb) * sizeof(double)));
    const int warps_grid = grid_for(3 * nb * 32);
    launch(k_sm_block_sums, warps_grid, kThreads, 0, s, x0, x1, x2, n, nb, D);
    launch(k_sm_predict, 3, kSmPredictThreads, 0, s, x0, x1, x2, nb, D);
    launch(k_sm_summaries, warps_grid, kThreads, 0, s, x0, x1, x2, n, nb, (const double *)D, S);
    const int smem = 2 * (kSmChunk * kSmBlock * (int)sizeof(float) + kSmChunk * (int)sizeof(SumBlock));
    cudaError_t e = cudaFuncSetAttribute(k_sm_walk, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    launch(k_sm_walk, 3, kSmWalkThreads, smem, s, x0, x1, x2, n, nb, (const SumBlock *)S, out);
    return cudaGetLastError();
}

}  // namespace pamo
