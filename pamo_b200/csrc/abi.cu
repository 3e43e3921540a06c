// C ABI entry points (include/pamo_b200.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "scan.cuh"
#include "stage1.cuh"
#include "stage2.cuh"
#include "stage3.cuh"

namespace pamo {
int s3_validate(const int *a, long long count, int hi, int *d_bad, int *h_bad, cudaStream_t st);
int s3_fetch(const float4 *q, float *out, int n, cudaStream_t st);
}  // namespace pamo

struct pamo_ctx {
    int device = 0;
    pamo::Stage2 s2;
    pamo::s3::Stage3 s3;
    pamo::s1::Stage1 s1;
    double s3_stats[3] = {0, 0, 0};
    int *undo_prev = nullptr;  // copy of the previous round's undo list (PaMO.run passes a clone)
    long long undo_prev_cap = 0;
    float *stage = nullptr;  // [n*3] staging for host transfers
    long long stage_cap = 0;
    int *istage = nullptr;
    long long istage_cap = 0;
};

namespace pamo {
namespace {

__global__ void k_aos3_to_f4(const float *in, float4 *out, int n)
{
    PAMO_GRID_STRIDE(i, n) out[i] = make_float4(in[3 * i], in[3 * i + 1], in[3 * i + 2], 0.f);
}

__global__ void k_aos3_to_i4(const int *in, int4 *out, int n)
{
    PAMO_GRID_STRIDE(i, n) out[i] = make_int4(in[3 * i], in[3 * i + 1], in[3 * i + 2], 0);
}

__global__ void k_f4_to_aos3(const float4 *in, float *out, int n, float ox, float oy, float oz, int add)
{
    PAMO_GRID_STRIDE(i, n)
    {
        float4 p = in[i];
        if (add) {
            p.x = p.x + ox;
            p.y = p.y + oy;
            p.z = p.z + oz;
        }
        out[3 * i] = p.x;
        out[3 * i + 1] = p.y;
        out[3 * i + 2] = p.z;
    }
}

__global__ void k_i4_to_aos3(const int4 *in, int *out, int n)
{
    PAMO_GRID_STRIDE(i, n)
    {
        int4 t = in[i];
        out[3 * i] = t.x;
        out[3 * i + 1] = t.y;
        out[3 * i + 2] = t.z;
    }
}

// Per-face vertex mean as numpy computes points[tris].mean(axis=1) in float32:
// ((a0 + a1) + a2) / 3, stored per coordinate.
__global__ void k_face_means(const float *pts, const int *tris, int m, float *mx, float *my, float *mz)
{
    PAMO_GRID_STRIDE(f, m)
    {
        int a = tris[3 * f], b = tris[3 * f + 1], c = tris[3 * f + 2];
        mx[f] = ((pts[3 * a] + pts[3 * b]) + pts[3 * c]) / 3.0f;
        my[f] = ((pts[3 * a + 1] + pts[3 * b + 1]) + pts[3 * c + 1]) / 3.0f;
        mz[f] = ((pts[3 * a + 2] + pts[3 * b + 2]) + pts[3 * c + 2]) / 3.0f;
    }
}

// numpy's .mean(axis=0) of a C-contiguous (F,3) float32 array adds the rows one
// after another into a float32 accumulator (no pairwise split on this axis), then
// divides by F.  Each coordinate's chain is inherently sequential, so the bound
// is the latency of F dependent adds.  One block: lane 0 of warps 0, 1, 2 runs
// the x, y, z chains (reading four values per shared-memory load) while warps
// 3..31 stream the next chunk into the other shared buffer.
constexpr int kMeanChunk = 8192;
constexpr int kMeanLoadFirst = 3 * 32;

__global__ void __launch_bounds__(1024) k_sequential_mean(const float *mx, const float *my, const float *mz, int m,
                                                          float *out)
{
    extern __shared__ float4 sm4[];  // 2 buffers x 3 coordinates x kMeanChunk floats
    float *sm = reinterpret_cast<float *>(sm4);
    if (m <= 0) return;
    const int n_chunks = (m + kMeanChunk - 1) / kMeanChunk;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto load = [&](int c, int buf) {
        float *dst = sm + buf * 3 * kMeanChunk;
        int base = c * kMeanChunk;
        int cnt = min(kMeanChunk, m - base);
        for (int i = threadIdx.x - kMeanLoadFirst; i < cnt; i += blockDim.x - kMeanLoadFirst) {
            dst[i] = mx[base + i];
            dst[kMeanChunk + i] = my[base + i];
            dst[2 * kMeanChunk + i] = mz[base + i];
        }
    };
    if (threadIdx.x >= kMeanLoadFirst) load(0, 0);
    __syncthreads();
    float acc = 0.f;
    for (int c = 0; c < n_chunks; ++c) {
        const int buf = c & 1;
        if (threadIdx.x >= kMeanLoadFirst) {
            if (c + 1 < n_chunks) load(c + 1, buf ^ 1);
        } else if (lane == 0) {
            const float *bs = sm + (buf * 3 + warp) * kMeanChunk;
            const float4 *b4 = reinterpret_cast<const float4 *>(bs);
            const int cnt = min(kMeanChunk, m - c * kMeanChunk);
            int i = 0;
            if (c == 0) {  // the accumulator starts from the first row
                acc = bs[0];
                i = 1;
            }
            for (; i < cnt && (i & 3); ++i) acc += bs[i];
            const int n4 = cnt >> 2;
            int q = i >> 2;
            // sixteen values per step, the next sixteen loaded while these are
            // added (the clamped loads stay inside the buffer and are unused at
            // the end), so the chain waits on the adds alone
            if (q + 4 <= n4) {
                float4 c0 = b4[q], c1 = b4[q + 1], c2 = b4[q + 2], c3 = b4[q + 3];
                for (; q + 4 <= n4; q += 4) {
                    const int nq = min(q + 4, n4 - 4);
                    const float4 d0 = b4[nq], d1 = b4[nq + 1], d2 = b4[nq + 2], d3 = b4[nq + 3];
                    acc += c0.x; acc += c0.y; acc += c0.z; acc += c0.w;
                    acc += c1.x; acc += c1.y; acc += c1.z; acc += c1.w;
                    acc += c2.x; acc += c2.y; acc += c2.z; acc += c2.w;
                    acc += c3.x; acc += c3.y; acc += c3.z; acc += c3.w;
                    c0 = d0; c1 = d1; c2 = d2; c3 = d3;
                }
            }
            for (; q < n4; ++q) {
                const float4 v = b4[q];
                acc += v.x;
                acc += v.y;
                acc += v.z;
                acc += v.w;
            }
            for (i = max(i, n4 * 4); i < cnt; ++i) acc += bs[i];
        }
        __syncthreads();
    }
    if (threadIdx.x < kMeanLoadFirst && lane == 0) out[warp] = acc / (float)m;
}

__global__ void k_centre(const float *pts, int n, const float *mean, float4 *out, int *bounds)
{
    const float ox = mean[0], oy = mean[1], oz = mean[2];
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    PAMO_GRID_STRIDE(i, n)
    {
        float x = pts[3 * i] - ox, y = pts[3 * i + 1] - oy, z = pts[3 * i + 2] - oz;
        out[i] = make_float4(x, y, z, 0.f);
        lo[0] = fminf(lo[0], x); lo[1] = fminf(lo[1], y); lo[2] = fminf(lo[2], z);
        hi[0] = fmaxf(hi[0], x); hi[1] = fmaxf(hi[1], y); hi[2] = fmaxf(hi[2], z);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            lo[k] = fminf(lo[k], __shfl_down_sync(0xffffffffu, lo[k], o));
            hi[k] = fmaxf(hi[k], __shfl_down_sync(0xffffffffu, hi[k], o));
        }
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            atomicMin(&bounds[k], float_to_ordered(lo[k]));
            atomicMax(&bounds[3 + k], float_to_ordered(hi[k]));
        }
}

// Per-block partial sums (double) and exact min / max of points [n,3]; a fixed
// grid and a fixed final order make the sums deterministic.
constexpr int kStatBlocks = 296;

__global__ void __launch_bounds__(256) k_point_stats(const float *pts, int n, double *part)
{
    double s[3] = {0.0, 0.0, 0.0};
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    PAMO_GRID_STRIDE(i, n)
    {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float x = pts[3 * i + k];
            s[k] += (double)x;
            lo[k] = fminf(lo[k], x);
            hi[k] = fmaxf(hi[k], x);
        }
    }
    __shared__ double ss[3][8];
    __shared__ float sl[3][8], sh[3][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            s[k] += __shfl_down_sync(0xffffffffu, s[k], o);
            lo[k] = fminf(lo[k], __shfl_down_sync(0xffffffffu, lo[k], o));
            hi[k] = fmaxf(hi[k], __shfl_down_sync(0xffffffffu, hi[k], o));
        }
        if (lane == 0) {
            ss[k][w] = s[k];
            sl[k][w] = lo[k];
            sh[k][w] = hi[k];
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        const int k = threadIdx.x;
        double a = 0.0;
        float l = INFINITY, h = -INFINITY;
        for (int j = 0; j < (int)(blockDim.x >> 5); ++j) {
            a += ss[k][j];
            l = fminf(l, sl[k][j]);
            h = fmaxf(h, sh[k][j]);
        }
        part[9 * blockIdx.x + k] = a;
        part[9 * blockIdx.x + 3 + k] = (double)l;
        part[9 * blockIdx.x + 6 + k] = (double)h;
    }
}

__global__ void k_point_stats_finish(const double *part, int nblocks, int n, double *out)
{
    if (threadIdx.x >= 3) return;
    const int k = threadIdx.x;
    double a = 0.0, l = INFINITY, h = -INFINITY;
    for (int b = 0; b < nblocks; ++b) {
        a += part[9 * b + k];
        l = fmin(l, part[9 * b + 3 + k]);
        h = fmax(h, part[9 * b + 6 + k]);
    }
    out[k] = a / (double)n;  // mean
    out[3 + k] = h - l;      // extent
}

__global__ void k_f64_to_f32(const double *in, int n, float *out)
{
    PAMO_GRID_STRIDE(i, n) out[i] = (float)in[i];
}

// Mixed Voronoi vertex areas (Meyer, Desbrun, Schroeder, Barr 2003) in double
// from double vertices [n,3], summed per vertex, and each face's largest
// corner cosine (the smallest angle), for stage 3's registration.
__global__ void k_voronoi(const double *v, const int *f, int nf, double *area, double *cmax_part)
{
    double cm = -2.0;
    bool nan_seen = false;
    PAMO_GRID_STRIDE(t, nf)
    {
        const int i0 = f[3 * t], i1 = f[3 * t + 1], i2 = f[3 * t + 2];
        double a[3], b[3], c[3];
        for (int k = 0; k < 3; ++k) {
            a[k] = v[3 * i0 + k];
            b[k] = v[3 * i1 + k];
            c[k] = v[3 * i2 + k];
        }
        double ea[3], eb[3], ec[3];
        for (int k = 0; k < 3; ++k) {
            ea[k] = c[k] - b[k];
            eb[k] = a[k] - c[k];
            ec[k] = b[k] - a[k];
        }
        auto dotd = [](const double *x, const double *y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
        const double la2 = dotd(ea, ea), lb2 = dotd(eb, eb), lc2 = dotd(ec, ec);
        // cross(ec, -eb)
        const double cx = -(ec[1] * eb[2] - ec[2] * eb[1]), cy = -(ec[2] * eb[0] - ec[0] * eb[2]),
                     cz = -(ec[0] * eb[1] - ec[1] * eb[0]);
        const double ar = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
        const double cos_a = -dotd(eb, ec) / sqrt(lb2 * lc2);
        const double cos_b = -dotd(ec, ea) / sqrt(lc2 * la2);
        const double cos_c = -dotd(ea, eb) / sqrt(la2 * lb2);
        auto cot = [](double cs) { return cs / sqrt(fmax(1.0 - cs * cs, 0.0)); };
        const double ca = cot(cos_a), cb = cot(cos_b), cc = cot(cos_c);
        double w0, w1, w2;
        if (cos_a < 0 || cos_b < 0 || cos_c < 0) {
            w0 = cos_a < 0 ? ar / 2 : ar / 4;
            w1 = cos_b < 0 ? ar / 2 : ar / 4;
            w2 = cos_c < 0 ? ar / 2 : ar / 4;
        } else {
            w0 = (lb2 * cb + lc2 * cc) / 8;
            w1 = (lc2 * cc + la2 * ca) / 8;
            w2 = (la2 * ca + lb2 * cb) / 8;
        }
        atomicAdd(&area[i0], w0);
        atomicAdd(&area[i1], w1);
        atomicAdd(&area[i2], w2);
        // corner cosines for the smallest-angle test (at a, b, c; as vectors from the corner)
        const double ka = dotd(ec, eb) * -1.0 / sqrt(lc2 * lb2), kb = -dotd(ea, ec) / sqrt(la2 * lc2),
                     kc = -dotd(eb, ea) / sqrt(lb2 * la2);
        for (double k : {ka, kb, kc}) {
            if (k != k) nan_seen = true;
            else cm = fmax(cm, k);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        cm = fmax(cm, __shfl_down_sync(0xffffffffu, cm, o));
        nan_seen = __shfl_down_sync(0xffffffffu, (int)nan_seen, o) || nan_seen;
    }
    __shared__ double s_cm[32];
    __shared__ int s_nan[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        s_cm[w] = cm;
        s_nan[w] = nan_seen;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = -2.0;
        int nn = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            r = fmax(r, s_cm[k]);
            nn |= s_nan[k];
        }
        cmax_part[blockIdx.x] = nn ? NAN : r;
    }
}

// out = float((in * scale + t) * post), each step one double rounding
__global__ void k_affine_points(const float *in, int n, double scale, double tx, double ty, double tz, double post,
                                float *out)
{
    PAMO_GRID_STRIDE(i, 3LL * n)
    {
        const int k = (int)(i % 3);
        const double t = k == 0 ? tx : (k == 1 ? ty : tz);
        out[i] = (float)__dmul_rn(__dadd_rn(__dmul_rn((double)in[i], scale), t), post);
    }
}

__global__ void k_bounds_init(int *b)
{
    int i = threadIdx.x;
    if (i < 3) b[i] = 0x7FFFFFFF;
    else if (i < 6) b[i] = (int)0x80000000;
}

__global__ void k_bounds_to_float(const int *b, float *out)
{
    int i = threadIdx.x;
    if (i < 6) out[i] = ordered_to_float(b[i]);
}

int set_device(pamo_ctx *ctx)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return PAMO_ERR_NO_DEVICE;
    if (ctx->device < 0 || ctx->device >= count) return PAMO_ERR_INVALID_ARG;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return PAMO_ERR_DEVICE;
    return PAMO_OK;
}

int ensure_undo_prev(pamo_ctx *ctx, long long n)
{
    if (n <= ctx->undo_prev_cap && ctx->undo_prev) return PAMO_OK;
    if (ctx->undo_prev) cudaFree(ctx->undo_prev);
    ctx->undo_prev = nullptr;
    long long c = n > 1024 ? n : 1024;
    if (cudaMalloc((void **)&ctx->undo_prev, c * 4) != cudaSuccess) return PAMO_ERR_OOM;
    ctx->undo_prev_cap = c;
    return PAMO_OK;
}

int ensure_stage(pamo_ctx *ctx, long long nf, long long ni)
{
    if (nf > ctx->stage_cap) {
        if (ctx->stage) cudaFree(ctx->stage);
        ctx->stage = nullptr;
        ctx->stage_cap = 0;
        if (cudaMalloc((void **)&ctx->stage, nf * 4) != cudaSuccess) return PAMO_ERR_OOM;
        ctx->stage_cap = nf;
    }
    if (ni > ctx->istage_cap) {
        if (ctx->istage) cudaFree(ctx->istage);
        ctx->istage = nullptr;
        ctx->istage_cap = 0;
        if (cudaMalloc((void **)&ctx->istage, ni * 4) != cudaSuccess) return PAMO_ERR_OOM;
        ctx->istage_cap = ni;
    }
    return PAMO_OK;
}

// reference host-side threshold conversion (cusimp_free.cu:923): clamp then a
// float->u32 conversion whose out-of-range case keeps the low 32 bits (x86-64)
}  // namespace
}  // namespace pamo

using namespace pamo;

#define RET_IF(x)             \
    do {                      \
        int _rc = (x);        \
        if (_rc) return _rc;  \
    } while (0)
#define CU_RET(x)                                          \
    do {                                                   \
        cudaError_t _e = (x);                              \
        if (_e != cudaSuccess) return map_cuda_error(_e); \
    } while (0)

// tris_mean of PaMO.run: each face's corner mean, then the rows added one by
// one in float32 (numpy's order); scratch holds 3 m floats
static int centring_mean(const float *d_points, const int *d_tris, int m, float *scratch, float *mean_dev,
                         cudaStream_t s)
{
    launch(k_face_means, grid_for(m), kThreads, 0, s, d_points, d_tris, m, scratch, scratch + m, scratch + 2LL * m);
    const int smem = 2 * 3 * kMeanChunk * (int)sizeof(float);
    CU_RET(cudaFuncSetAttribute(k_sequential_mean, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    launch(k_sequential_mean, 1, 1024, smem, s, scratch, scratch + m, scratch + 2LL * m, m, mean_dev);
    CU_RET(cudaGetLastError());
    return PAMO_OK;
}

extern "C" {

int pamo_version(void) { return 100; }

long long pamo_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

const char *pamo_status_string(int status)
{
    switch (status) {
    case PAMO_OK: return "ok";
    case PAMO_ERR_INVALID_ARG: return "invalid argument";
    case PAMO_ERR_OOM: return "out of device memory";
    case PAMO_ERR_BUDGET_EXCEEDED: return "budget exceeded";
    case PAMO_ERR_DEVICE: return "CUDA device error";
    case PAMO_ERR_NO_DEVICE: return "no CUDA device";
    case PAMO_ERR_CAPACITY: return "internal capacity exceeded";
    default: return "unknown status";
    }
}

int pamo_ctx_create(int device, pamo_ctx **out)
{
    if (!out) return PAMO_ERR_INVALID_ARG;
    *out = nullptr;
    pamo_ctx *c = new (std::nothrow) pamo_ctx();
    if (!c) return PAMO_ERR_OOM;
    c->device = device;
    c->s2.device = device;
    c->s3.prof = &c->s2.prof;  // one phase timer for all stages
    c->s1.prof = &c->s2.prof;
    int rc = set_device(c);
    if (rc) {
        delete c;
        return rc;
    }
    *out = c;
    return PAMO_OK;
}

int pamo_ctx_destroy(pamo_ctx *ctx)
{
    if (!ctx) return PAMO_ERR_INVALID_ARG;
    if (set_device(ctx) == PAMO_OK) {
        cudaDeviceSynchronize();
        ctx->s2.release();
        ctx->s3.release();
        ctx->s1.release();
        if (ctx->undo_prev) cudaFree(ctx->undo_prev);
        if (ctx->stage) cudaFree(ctx->stage);
        if (ctx->istage) cudaFree(ctx->istage);
    }
    delete ctx;
    return PAMO_OK;
}

int pamo_free_forward(pamo_ctx *ctx, const float *d_points, const int *d_tris, const int *d_verts_undo,
                      int n_verts_undo, int n_pts, int n_tris, float scale, float threshold, int is_stuck, int init,
                      void *stream, float *d_out_points, int *d_out_tris, int *d_out_occ, int *d_out_map,
                      int *n_out_undo)
{
    if (!ctx || n_pts < 0 || n_tris < 0 || n_verts_undo < 0 || !n_out_undo) return PAMO_ERR_INVALID_ARG;
    if ((n_pts && !d_points) || (n_tris && !d_tris) || (n_verts_undo && !d_verts_undo)) return PAMO_ERR_INVALID_ARG;
    RET_IF(set_device(ctx));
    cudaStream_t s = (cudaStream_t)stream;
    Stage2 &S = ctx->s2;
    RET_IF(S.ensure(n_pts, n_tris));
    if (n_verts_undo > S.cap_undo) return PAMO_ERR_CAPACITY;
    RET_IF(S.validate(d_tris, n_pts, n_tris, d_verts_undo, n_verts_undo, (int)S.cap_pts, s));
    launch(k_aos3_to_f4, grid_for(n_pts), kThreads, 0, s, d_points, S.opts, n_pts);
    launch(k_aos3_to_i4, grid_for(n_tris), kThreads, 0, s, d_tris, S.otris, n_tris);
    if (init) RET_IF(stage2_shuffle_faces(S.otris, n_tris, s));
    int nvu = 0;
    RET_IF(S.round(n_pts, n_tris, scale, threshold, is_stuck != 0, d_verts_undo, n_verts_undo, &nvu, s));
    if (d_out_points) launch(k_f4_to_aos3, grid_for(n_pts), kThreads, 0, s, S.pts, d_out_points, n_pts, 0, 0, 0, 0);
    if (d_out_tris) launch(k_i4_to_aos3, grid_for(n_tris), kThreads, 0, s, S.tris, d_out_tris, n_tris);
    if (d_out_occ && n_pts) CU_RET(cudaMemcpyAsync(d_out_occ, S.occ, (size_t)n_pts * 4, cudaMemcpyDeviceToDevice, s));
    if (d_out_map && n_pts)
        CU_RET(cudaMemcpyAsync(d_out_map, S.pts_map, (size_t)n_pts * 4, cudaMemcpyDeviceToDevice, s));
    CU_RET(cudaGetLastError());
    CU_RET(cudaStreamSynchronize(s));
    *n_out_undo = nvu;
    return PAMO_OK;
}

int pamo_free_copy_undo(pamo_ctx *ctx, int *d_out, int n, void *stream)
{
    if (!ctx || n < 0 || (n && !d_out) || n > ctx->s2.cap_undo) return PAMO_ERR_INVALID_ARG;
    RET_IF(set_device(ctx));
    cudaStream_t s = (cudaStream_t)stream;
    if (n) CU_RET(cudaMemcpyAsync(d_out, ctx->s2.undo_list, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
    CU_RET(cudaStreamSynchronize(s));
    return PAMO_OK;
}

// The stage-2 loop of PaMO.run.  offset3 == nullptr: the points are centred
// here (tris_mean in numpy's float32 order) as PaMO.run does without stage 1;
// otherwise they are already centred (stage 1's output) and offset3 is the
// tris_mean added back at the end.
static int stage2_loop(pamo_ctx *ctx, const float *d_points, const int *d_tris, int n_pts, int n_tris,
                       const float *offset3, long long target_faces, int tolerance, float threshold, int iters,
                       void *stream, int *out_n_pts, int *out_n_tris, int *out_rounds)
{
    if (!ctx || n_pts <= 0 || n_tris <= 0 || !d_points || !d_tris || !out_n_pts || !out_n_tris || !out_rounds)
        return PAMO_ERR_INVALID_ARG;
    RET_IF(set_device(ctx));
    cudaStream_t s = (cudaStream_t)stream;
    Stage2 &S = ctx->s2;
    RET_IF(S.ensure(n_pts, n_tris));
    RET_IF(ensure_undo_prev(ctx, S.cap_undo));
    RET_IF(S.validate(d_tris, n_pts, n_tris, nullptr, 0, 0, s));
    // centring (tris_mean in numpy's float32 order) and scale, as PaMO.run does
    float *mxyz = reinterpret_cast<float *>(S.plane);  // 3*m floats of scratch (plane has 4*m)
    float *mean_dev = reinterpret_cast<float *>(S.dev_misc);
    int *bounds = S.dev_misc + 8;
    float *bounds_f = reinterpret_cast<float *>(S.dev_misc + 16);
    if (offset3) {
        CU_RET(cudaMemsetAsync(mean_dev, 0, 3 * sizeof(float), s));  // already centred
    } else {
        RET_IF(centring_mean(d_points, d_tris, n_tris, mxyz, mean_dev, s));
    }
    launch(k_bounds_init, 1, 32, 0, s, bounds);
    launch(k_centre, grid_for(n_pts), kThreads, 0, s, d_points, n_pts, mean_dev, S.opts, bounds);
    launch(k_bounds_to_float, 1, 32, 0, s, bounds, bounds_f);
    launch(k_aos3_to_i4, grid_for(n_tris), kThreads, 0, s, d_tris, S.otris, n_tris);
    RET_IF(stage2_shuffle_faces(S.otris, n_tris, s));
    CU_RET(cudaMemcpyAsync(S.h_scalars, mean_dev, 3 * 4, cudaMemcpyDeviceToHost, s));
    CU_RET(cudaMemcpyAsync(S.h_scalars + 4, bounds_f, 6 * 4, cudaMemcpyDeviceToHost, s));
    CU_RET(cudaStreamSynchronize(s));
    for (int k = 0; k < 3; ++k) S.offset[k] = offset3 ? offset3[k] : S.h_scalars[k];
    const float *bf = S.h_scalars + 4;
    float sx = bf[3] - bf[0], sy = bf[4] - bf[1], sz = bf[5] - bf[2];
    float scale = sy > sx ? sy : sx;  // Python max() keeps the first maximal argument
    scale = sz > scale ? sz : scale;

    int n = n_pts, m = n_tris, count = 0, rounds = 0, n_undo = 0;
    bool stuck = false;
    S.round_faces.clear();
    for (int it = 0; it < iters; ++it) {
        int prev = m;
        S.round_faces.push_back(m);
        int nvu = 0;
        RET_IF(S.round(n, m, scale, threshold, stuck, n_undo ? ctx->undo_prev : nullptr, n_undo, &nvu, s, it > 0));
        rounds++;
        if (nvu > ctx->undo_prev_cap) return PAMO_ERR_CAPACITY;
        if (nvu) CU_RET(cudaMemcpyAsync(ctx->undo_prev, S.undo_list, (size_t)nvu * 4, cudaMemcpyDeviceToDevice, s));
        n_undo = nvu;
        RET_IF(S.compact(n, m, s));
        n = S.hcnt->n_pts_next;
        m = S.hcnt->n_tris_next;
        S.last_stats[7] = m;
        if ((long long)m <= target_faces || m <= 10) break;
        if (m == prev) count++;
        else {
            count = 0;
            stuck = false;
        }
        if (count >= 2) stuck = true;
        if (count == tolerance) break;
    }
    S.res_n_pts = n;
    S.res_n_tris = m;
    S.res_rounds = rounds;
    *out_n_pts = n;
    *out_n_tris = m;
    *out_rounds = rounds;
    return PAMO_OK;
}

int pamo_tris_mean(const float *d_points, const int *d_tris, int n_pts, int n_tris, float *h_out3, void *stream)
{
    if (!h_out3 || n_pts <= 0 || n_tris <= 0 || !d_points || !d_tris) return PAMO_ERR_INVALID_ARG;
    int dev;
    if (cudaGetDevice(&dev) != cudaSuccess) return PAMO_ERR_NO_DEVICE;
    cudaStream_t s = (cudaStream_t)stream;
    CU_RET(retain_pool_memory());
    // 3 n_tris floats of face means, then the bad-index flag and the result
    const size_t cb = ((size_t)3 * n_tris * sizeof(float) + 15) & ~(size_t)15;
    char *scratch = nullptr;
    if (cudaMallocAsync((void **)&scratch, cb + 32, s) != cudaSuccess) return PAMO_ERR_OOM;
    int *d_bad = reinterpret_cast<int *>(scratch + cb);
    float *d_mean = reinterpret_cast<float *>(scratch + cb + 16);
    int h_bad = 0;
    int rc = s3_validate(d_tris, 3LL * n_tris, n_pts, d_bad, &h_bad, s);
    if (rc == PAMO_OK) rc = centring_mean(d_points, d_tris, n_tris, reinterpret_cast<float *>(scratch), d_mean, s);
    if (rc == PAMO_OK && cudaMemcpyAsync(h_out3, d_mean, 3 * sizeof(float), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        rc = PAMO_ERR_DEVICE;
    cudaFreeAsync(scratch, s);
    if (cudaStreamSynchronize(s) != cudaSuccess && rc == PAMO_OK) rc = PAMO_ERR_DEVICE;
    return rc;
}

int pamo_set_quality(pamo_ctx *ctx, int on)
{
    if (!ctx) return PAMO_ERR_INVALID_ARG;
    ctx->s2.quality = on != 0;
    return PAMO_OK;
}

int pamo_stage2_run(pamo_ctx *ctx, const float *d_points, const int *d_tris, int n_pts, int n_tris,
                    long long target_faces, int tolerance, float threshold, int iters, void *stream, int *out_n_pts,
                    int *out_n_tris, int *out_rounds)
{
    return stage2_loop(ctx, d_points, d_tris, n_pts, n_tris, nullptr, target_faces, tolerance, threshold, iters, stream,
                       out_n_pts, out_n_tris, out_rounds);
}

int pamo_stage2_run_centred(pamo_ctx *ctx, const float *d_points, const int *d_tris, int n_pts, int n_tris,
                            const float *h_offset3, long long target_faces, int tolerance, float threshold, int iters,
                            void *stream, int *out_n_pts, int *out_n_tris, int *out_rounds)
{
    if (!h_offset3) return PAMO_ERR_INVALID_ARG;
    return stage2_loop(ctx, d_points, d_tris, n_pts, n_tris, h_offset3, target_faces, tolerance, threshold, iters,
                       stream, out_n_pts, out_n_tris, out_rounds);
}

int pamo_remesh(pamo_ctx *ctx, const float *d_points, const int *d_tris, int n_pts, int n_tris, int resolution,
                void *stream, int *out_n_verts, int *out_n_tris)
{
    if (!ctx || n_pts <= 0 || n_tris <= 0 || !d_points || !d_tris || !out_n_verts || !out_n_tris || resolution < 4 ||
        resolution > 1024)
        return PAMO_ERR_INVALID_ARG;
    RET_IF(set_device(ctx));
    cudaStream_t s = (cudaStream_t)stream;
    pamo::s1::Stage1 &S = ctx->s1;
    RET_IF(S.ensure(n_tris, resolution));
    int h_bad = 0;
    RET_IF(s3_validate(d_tris, 3LL * n_tris, n_pts, S.dev + 15, &h_bad, s));
    // tris_mean of the input (the scratch: the normalised-triangle buffer, 9 m floats)
    RET_IF(centring_mean(d_points, d_tris, n_tris, S.tris, S.mean_dev, s));
    CU_RET(cudaMemcpyAsync(S.offset, S.mean_dev, 3 * sizeof(float), cudaMemcpyDeviceToHost, s));
    RET_IF(pamo::s1::remesh(S, d_points, d_tris, n_pts, n_tris, S.mean_dev, resolution, s));
    CU_RET(cudaStreamSynchronize(s));
    if (S.prof) S.prof->collect();
    *out_n_verts = S.n_verts;
    *out_n_tris = S.n_tris;
    return PAMO_OK;
}

int pamo_remesh_fetch(pamo_ctx *ctx, float *d_out_verts, int *d_out_tris, float *h_offset3, void *stream)
{
    if (!ctx || !d_out_verts || !d_out_tris) return PAMO_ERR_INVALID_ARG;
    RET_IF(set_device(ctx));
    cudaStream_t s = (cudaStream_t)stream;
    pamo::s1::Stage1 &S = ctx->s1;
    if (S.n_tris <= 0) return PAMO_ERR_INVALID_ARG;
    CU_RET(cudaMemcpyAsync(d_out_verts, S.verts, (size_t)S.n_verts * 12, cudaMemcpyDeviceToDevice, s));
    CU_RET(cudaMemcpyAsync(d_out_tris, S.faces, (size_t)S.n_tris * 12, cudaMemcpyDeviceToDevice, s));
    if (h_offset3)
        for (int k = 0; k < 3; ++k) h_offset3[k] = S.offset[k];
    CU_RET(cudaStreamSynchronize(s));
    return PAMO_OK;
}

int pamo_stage2_fetch(pamo_ctx *ctx, float *out_points, int *out_tris, int to_host, void *stream)
{
    if (!ctx || !out_points || !out_tris) return PAMO_ERR_INVALID_ARG;
    RET_IF(set_device(ctx));
    cudaStream_t s = (cudaStream_t)stream;
    Stage2 &S = ctx->s2;
    int n = S.res_n_pts, m = S.res_n_tris;
    if (to_host) {
        RET_IF(ensure_stage(ctx, 3LL * n + 3, 3LL * m + 3));
        launch(k_f4_to_aos3, grid_for(n), kThreads, 0, s, S.opts, ctx->stage, n, S.offset[0], S.offset[1], S.offset[2], 1);
        launch(k_i4_to_aos3, grid_for(m), kThreads, 0, s, S.otris, ctx->istage, m);
        CU_RET(cudaMemcpyAsync(out_points, ctx->stage, (size_t)n * 12, cudaMemcpyDeviceToHost, s));
        CU_RET(cudaMemcpyAsync(out_tris, ctx->istage, (size_t)m * 12, cudaMemcpyDeviceToHost, s));
    } else {
        launch(k_f4_to_aos3, grid_for(n), kThreads, 0, s, S.opts, out_points, n, S.offset[0], S.offset[1], S.offset[2], 1);
        launch(k_i4_to_aos3, grid_for(m), kThreads, 0, s, S.otris, out_tris, m);
    }
    CU_RET(cudaGetLastError());
    CU_RET(cudaStreamSynchronize(s));
    return PAMO_OK;
}

int pamo_stage2_offset(pamo_ctx *ctx, float *h_out3)
{
    if (!ctx || !h_out3) return PAMO_ERR_INVALID_ARG;
    for (int k = 0; k < 3; ++k) h_out3[k] = ctx->s2.offset[k];
    return PAMO_OK;
}

int pamo_stage2_last_round_stats(pamo_ctx *ctx, long long *h_out8)
{
    if (!ctx || !h_out8) return PAMO_ERR_INVALID_ARG;
    for (int k = 0; k < 8; ++k) h_out8[k] = ctx->s2.last_stats[k];
    return PAMO_OK;
}

int pamo_self_intersect(pamo_ctx *ctx, const float *d_points, const int *d_tris, int n_pts, int n_tris,
                        unsigned char *d_out_flags, long long *out_n_pairs, void *stream)
{
    if (!ctx || n_pts <= 0 || n_tris < 0 || !d_points || (n_tris && (!d_tris || !d_out_flags))) return PAMO_ERR_INVALID_ARG;
    RET_IF(set_device(ctx));
    cudaStream_t s = (cudaStream_t)stream;
    Stage2 &S = ctx->s2;
    RET_IF(S.ensure(n_pts, n_tris));
    RET_IF(S.validate(d_tris, n_pts, n_tris, nullptr, 0, 0, s));
    launch(k_aos3_to_f4, grid_for(n_pts), kThreads, 0, s, d_points, S.opts, n_pts);
    launch(k_aos3_to_i4, grid_for(n_tris), kThreads, 0, s, d_tris, S.otris, n_tris);
    RET_IF(S.self_intersect_all(n_pts, n_tris, s));
    if (n_tris) CU_RET(cudaMemcpyAsync(d_out_flags, S.isect, (size_t)n_tris, cudaMemcpyDeviceToDevice, s));
    CU_RET(cudaStreamSynchronize(s));
    if (out_n_pairs) *out_n_pairs = S.hcnt->n_pairs;
    return PAMO_OK;
}

int pamo_profile_enable(pamo_ctx *ctx, int enable)
{
    if (!ctx) return PAMO_ERR_INVALID_ARG;
    ctx->s2.prof.on = enable != 0;
    ctx->s2.prof.reset();
    return PAMO_OK;
}

int pamo_profile_read(pamo_ctx *ctx, double *h_ms, long long *h_calls, int cap)
{
    if (!ctx || cap < 0) return PAMO_ERR_INVALID_ARG;
    int n = cap < PH_COUNT ? cap : PH_COUNT;
    for (int i = 0; i < n; ++i) {
        if (h_ms) h_ms[i] = ctx->s2.prof.ms[i];
        if (h_calls) h_calls[i] = ctx->s2.prof.calls[i];
    }
    return PH_COUNT;
}

int pamo_stage2_round_sizes(pamo_ctx *ctx, int *h_out, int cap)
{
    if (!ctx || cap < 0 || (cap && !h_out)) return -PAMO_ERR_INVALID_ARG;
    int n = (int)ctx->s2.round_faces.size();
    for (int i = 0; i < n && i < cap; ++i) h_out[i] = ctx->s2.round_faces[i];
    return n;
}

void pamo_s3_default_config(pamo_s3_config *c)
{
    if (!c) return;
    c->n_newton_iters = 10;
    c->n_cg_iters = 40;
    c->n_line_search_iters = 10;
    c->ccd_max_iters = 100;
    c->spd_max_iters = 3;
    c->d_hat = 1e-3f;
    c->coll_stiffness = 1e2f;
    c->contact_detection_radius = 1e-2f;
    c->ee_classify_thres = 1e-3f;
    c->ccd_slackness = 0.7f;
    c->ccd_thickness = 1e-6f;
    c->elas_young_modulus = 1e-1f;
    c->elas_poisson_ratio = 0.0f;
    c->hinge_stiffness = 1e-2f;
    c->mesh2gt_dist_stiffness = 1e3f;
    c->max_blocks = 1LL << 25;
    c->reuse_gt = 0;
}

int pamo_safe_project(pamo_ctx *ctx, const float *d_gt_v, const int *d_gt_f, int n_gt_v, int n_gt_f,
                      const float *d_v, const int *d_f, int n_v, int n_f, const int *d_e, int n_e, const int *d_h,
                      int n_h, const float *d_vor, int n_steps, int do_nothing, const pamo_s3_config *cfg,
                      void *stream, float *d_out_v)
{
    if (!ctx || n_gt_v <= 0 || n_gt_f <= 0 || n_v <= 0 || n_f <= 0 || n_e < 0 || n_h < 0 || n_steps < 0 || !d_gt_v ||
        !d_gt_f || !d_v || !d_f || (n_e && !d_e) || (n_h && !d_h) || !d_vor || !d_out_v)
        return PAMO_ERR_INVALID_ARG;
    RET_IF(set_device(ctx));
    cudaStream_t s = (cudaStream_t)stream;
    pamo::s3::Stage3 &S = ctx->s3;
    if (cfg) S.cfg = *cfg;
    else pamo_s3_default_config(&S.cfg);
    if (S.cfg.n_newton_iters < 0 || S.cfg.n_cg_iters < 0 || S.cfg.n_line_search_iters < 0 || S.cfg.ccd_max_iters < 0 ||
        S.cfg.spd_max_iters < 0 || !(S.cfg.d_hat > 0.f) || S.cfg.max_blocks <= 0)
        return PAMO_ERR_INVALID_ARG;
    RET_IF(S.ensure(n_v, n_f, n_e, n_h, n_gt_v, n_gt_f));
    RET_IF(S.ensure_trace((long long)n_steps * S.cfg.n_newton_iters));
    int *bad = S.iscal + 8;
    RET_IF(s3_validate(d_f, 3LL * n_f, n_v, bad, S.h_iscal, s));
    RET_IF(s3_validate(d_e, 2LL * n_e, n_v, bad, S.h_iscal, s));
    RET_IF(s3_validate(d_h, 4LL * n_h, n_v, bad, S.h_iscal, s));
    RET_IF(s3_validate(d_gt_f, 3LL * n_gt_f, n_gt_v, bad, S.h_iscal, s));
    S.do_nothing = do_nothing != 0;
    // the solve runs on the context's own stream, ordered after the caller's
    // stream and before whatever the caller queues next
    if (!S.work) CU_RET(cudaStreamCreateWithFlags(&S.work, cudaStreamNonBlocking));
    if (!S.ev_in) CU_RET(cudaEventCreateWithFlags(&S.ev_in, cudaEventDisableTiming));
    if (!S.ev_out) CU_RET(cudaEventCreateWithFlags(&S.ev_out, cudaEventDisableTiming));
    for (int b = 0; b < 2; ++b) {
        if (!S.side[b]) CU_RET(cudaStreamCreateWithFlags(&S.side[b], cudaStreamNonBlocking));
        if (!S.ev_join[b]) CU_RET(cudaEventCreateWithFlags(&S.ev_join[b], cudaEventDisableTiming));
    }
    if (!S.ev_fork) CU_RET(cudaEventCreateWithFlags(&S.ev_fork, cudaEventDisableTiming));
    CU_RET(cudaEventRecord(S.ev_in, s));
    CU_RET(cudaStreamWaitEvent(S.work, S.ev_in, 0));
    cudaStream_t caller = s;
    s = S.work;
    RET_IF(S.register_mesh(d_gt_v, d_gt_f, n_gt_v, n_gt_f, d_v, d_f, n_v, n_f, d_e, n_e, d_h, n_h, d_vor, s));
    int newton = 0;
    for (int k = 0; k < n_steps; ++k) {
        RET_IF(S.step(s));
        if (!S.do_nothing) newton += S.cfg.n_newton_iters;
    }
    RET_IF(s3_fetch(S.q, d_out_v, n_v, s));
    double e = 0;
    RET_IF(S.energy_now(&e, s));
    CU_RET(cudaMemcpyAsync(S.h_iscal, S.iscal, 4, cudaMemcpyDeviceToHost, s));
    CU_RET(cudaStreamSynchronize(s));
    CU_RET(cudaEventRecord(S.ev_out, s));
    CU_RET(cudaStreamWaitEvent(caller, S.ev_out, 0));
    ctx->s3_stats[0] = e;
    ctx->s3_stats[1] = S.h_iscal[0];
    ctx->s3_stats[2] = newton;
    return PAMO_OK;
}

int pamo_voronoi_areas(const double *d_v, const int *d_f, int nv, int nf, float *d_out, double *h_min_angle_deg,
                       void *stream)
{
    if (nv <= 0 || nf < 0 || !d_v || (nf && !d_f) || !d_out || !h_min_angle_deg) return PAMO_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = 296;
    double *scratch = nullptr;
    CU_RET(retain_pool_memory());
    CU_RET(cudaMallocAsync((void **)&scratch, ((size_t)nv + nb + 1) * sizeof(double), s));
    cudaError_t e = cudaMemsetAsync(scratch, 0, (size_t)nv * sizeof(double), s);
    if (e == cudaSuccess) {
        if (nf) launch(k_voronoi, nb, 256, 0, s, d_v, d_f, nf, scratch, scratch + nv);
        launch(k_f64_to_f32, grid_for(nv), kThreads, 0, s, (const double *)scratch, nv, d_out);
        std::vector<double> host(nb, -2.0);
        if (nf) e = cudaMemcpyAsync(host.data(), scratch + nv, nb * sizeof(double), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        double cm = -2.0;
        bool nan_seen = false;
        for (double x : host) {
            if (x != x) nan_seen = true;
            else cm = std::max(cm, x);
        }
        if (!nf) *h_min_angle_deg = 180.0;
        else if (nan_seen) *h_min_angle_deg = NAN;
        else *h_min_angle_deg = std::acos(std::min(std::max(cm, -1.0), 1.0)) * 180.0 / M_PI;
    }
    cudaFreeAsync(scratch, s);
    CU_RET(e);
    CU_RET(cudaGetLastError());
    return PAMO_OK;
}

int pamo_point_stats(const float *d_pts, int n, double *h_out6, void *stream)
{
    if (n <= 0 || !d_pts || !h_out6) return PAMO_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    double *scratch = nullptr;
    CU_RET(retain_pool_memory());
    CU_RET(cudaMallocAsync((void **)&scratch, (9 * kStatBlocks + 8) * sizeof(double), s));
    launch(k_point_stats, kStatBlocks, 256, 0, s, d_pts, n, scratch);
    launch(k_point_stats_finish, 1, 32, 0, s, (const double *)scratch, kStatBlocks, n, scratch + 9 * kStatBlocks);
    cudaError_t e = cudaMemcpyAsync(h_out6, scratch + 9 * kStatBlocks, 6 * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(scratch, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    CU_RET(e);
    return PAMO_OK;
}

int pamo_mesh_hinges(const int *h_tris, int n_tris, int n_pts, int *h_edges, int *h_hinges, int *out_n_edges)
{
    if (!h_tris || n_tris < 0 || n_pts < 0 || !out_n_edges || (n_tris && (!h_edges || !h_hinges)))
        return PAMO_ERR_INVALID_ARG;
    *out_n_edges = 0;
    if (n_tris == 0) return PAMO_OK;
    const long long nd = 3LL * n_tris;  // directed edges: corner k -> k + 1 of every face, k-major
    for (long long i = 0; i < nd; ++i)
        if (h_tris[i] < 0 || h_tris[i] >= n_pts) return PAMO_ERR_INVALID_ARG;
    if (nd % 2) return PAMO_ERR_CAPACITY;
    std::vector<int> from((size_t)nd), to((size_t)nd), opp((size_t)nd);
    for (int k = 0; k < 3; ++k)
        for (int f = 0; f < n_tris; ++f) {
            const size_t e = (size_t)k * n_tris + f;
            from[e] = h_tris[3 * (size_t)f + k];
            to[e] = h_tris[3 * (size_t)f + (k + 1) % 3];
            opp[e] = h_tris[3 * (size_t)f + (k + 2) % 3];
        }
    // bucket by the smaller vertex (counting sort, stable), then order each
    // bucket by the larger vertex: keys ascend as lo * n + hi
    std::vector<int> start((size_t)n_pts + 1, 0), order((size_t)nd), hi((size_t)nd);
    for (size_t e = 0; e < (size_t)nd; ++e) {
        start[(size_t)std::min(from[e], to[e]) + 1]++;
        hi[e] = std::max(from[e], to[e]);
    }
    for (int v = 0; v < n_pts; ++v) start[(size_t)v + 1] += start[(size_t)v];
    {
        std::vector<int> cur(start.begin(), start.end() - 1);
        for (size_t e = 0; e < (size_t)nd; ++e) order[(size_t)cur[(size_t)std::min(from[e], to[e])]++] = (int)e;
    }
    for (int v = 0; v < n_pts; ++v) {
        const int a = start[(size_t)v], b = start[(size_t)v + 1];
        for (int i = a + 1; i < b; ++i) {  // insertion sort by the larger vertex (stable)
            const int x = order[(size_t)i], kx = hi[(size_t)x];
            int j = i - 1;
            while (j >= a && hi[(size_t)order[(size_t)j]] > kx) {
                order[(size_t)j + 1] = order[(size_t)j];
                --j;
            }
            order[(size_t)j + 1] = x;
        }
    }
    // every key exactly twice, once each way
    long long ne = 0;
    for (long long i = 0; i < nd; i += 2) {
        const size_t e0 = (size_t)order[(size_t)i], e1 = (size_t)order[(size_t)i + 1];
        const int lo = std::min(from[e0], to[e0]), h = hi[e0];
        if (lo == h || std::min(from[e1], to[e1]) != lo || hi[e1] != h || (from[e0] < to[e0]) == (from[e1] < to[e1]))
            return PAMO_ERR_CAPACITY;
        if (i + 2 < nd) {  // the next key must differ
            const size_t e2 = (size_t)order[(size_t)i + 2];
            if (std::min(from[e2], to[e2]) == lo && hi[e2] == h) return PAMO_ERR_CAPACITY;
        }
        const size_t ef = from[e0] < to[e0] ? e0 : e1, eb = from[e0] < to[e0] ? e1 : e0;
        h_edges[2 * ne] = lo;
        h_edges[2 * ne + 1] = h;
        h_hinges[4 * ne] = opp[ef];
        h_hinges[4 * ne + 1] = lo;
        h_hinges[4 * ne + 2] = h;
        h_hinges[4 * ne + 3] = opp[eb];
        ++ne;
    }
    *out_n_edges = (int)ne;
    return PAMO_OK;
}

int pamo_affine_points(const float *d_in, int n, double scale, double tx, double ty, double tz, double post,
                       float *d_out, void *stream)
{
    if (n < 0 || (n && (!d_in || !d_out))) return PAMO_ERR_INVALID_ARG;
    if (n == 0) return PAMO_OK;
    launch(k_affine_points, grid_for(3LL * n), kThreads, 0, (cudaStream_t)stream, d_in, n, scale, tx, ty, tz, post,
           d_out);
    CU_RET(cudaGetLastError());
    return PAMO_OK;
}

int pamo_safe_project_stats(pamo_ctx *ctx, double *h_out3)
{
    if (!ctx || !h_out3) return PAMO_ERR_INVALID_ARG;
    for (int k = 0; k < 3; ++k) h_out3[k] = ctx->s3_stats[k];
    return PAMO_OK;
}

int pamo_safe_project_trace(pamo_ctx *ctx, double *h_out, int cap_rows, int *out_rows)
{
    if (!ctx || cap_rows < 0 || (cap_rows && !h_out) || !out_rows) return PAMO_ERR_INVALID_ARG;
    pamo::s3::Stage3 &S = ctx->s3;
    *out_rows = 0;
    if (!S.trace || !S.iscal) return PAMO_OK;
    RET_IF(set_device(ctx));
    int rows = 0;
    CU_RET(cudaMemcpy(&rows, S.iscal + 13, sizeof(int), cudaMemcpyDeviceToHost));  // the trace's row counter
    if (rows > S.cap_trace) rows = (int)S.cap_trace;
    const int n = rows < cap_rows ? rows : cap_rows;
    if (n > 0) CU_RET(cudaMemcpy(h_out, S.trace, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost));
    *out_rows = rows;
    return PAMO_OK;
}

int pamo_debug_wait_timeout(pamo_ctx *ctx, int which, long long spin_limit, void *stream)
{
    if (!ctx || (which != 0 && which != 1) || spin_limit < 0 || spin_limit > (1LL << 24)) return PAMO_ERR_INVALID_ARG;
    RET_IF(set_device(ctx));
    cudaStream_t s = (cudaStream_t)stream;
    if (which == 0) {
        // a 32-tile scan whose tile 3 never publishes: the tiles after it wait
        // on it, give up after spin_limit polls and record the fault
        const long long n = 32LL * pamo::kScanTile;
        const long long sc = pamo::scan_scratch_ints(n);
        int *buf = nullptr;
        CU_RET(cudaMalloc((void **)&buf, (size_t)(2 * n + sc + 1) * 4));
        int *in = buf, *out = buf + n, *scratch = buf + 2 * n, *fault = scratch + sc;
        int h_fault = 0;
        cudaError_t e = cudaMemsetAsync(buf, 0, (size_t)(2 * n + sc + 1) * 4, s);
        if (e == cudaSuccess) e = pamo::exclusive_scan_waits(in, out, n, nullptr, scratch, nullptr, s, fault, spin_limit, 3);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h_fault, fault, 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaFree(buf);
        if (e != cudaSuccess) return map_cuda_error(e);
        return h_fault ? PAMO_ERR_DEVICE : PAMO_OK;
    }
    // the persistent CG with block 1 never publishing its partial sums: every
    // block's wait on that slot gives up, the solve returns with the error
    // recorded and the call reports PAMO_ERR_DEVICE
    const int n = 4096;
    std::vector<int> rp(n + 1), cl(n);
    std::vector<float> blk(9 * (size_t)n, 0.f), dg(3 * (size_t)n, 2.f), rhs(3 * (size_t)n, 1.f);
    for (int i = 0; i < n; ++i) {
        rp[i] = i;
        cl[i] = i;
        blk[9 * (size_t)i] = blk[9 * (size_t)i + 4] = blk[9 * (size_t)i + 8] = 2.f;
    }
    rp[n] = n;
    int *d_i = nullptr;
    float *d_f = nullptr;
    CU_RET(cudaMalloc((void **)&d_i, (size_t)(2 * n + 1) * 4));
    if (cudaMalloc((void **)&d_f, (size_t)(9 + 3 + 3 + 3) * n * 4) != cudaSuccess) {
        cudaFree(d_i);
        return PAMO_ERR_OOM;
    }
    float *d_blk = d_f, *d_dg = d_f + 9 * (size_t)n, *d_rhs = d_dg + 3 * (size_t)n, *d_out = d_rhs + 3 * (size_t)n;
    cudaError_t e = cudaMemcpy(d_i, rp.data(), (size_t)(n + 1) * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_i + n + 1, cl.data(), (size_t)n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_blk, blk.data(), blk.size() * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_dg, dg.data(), dg.size() * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_rhs, rhs.data(), rhs.size() * 4, cudaMemcpyHostToDevice);
    int rc = e == cudaSuccess ? PAMO_OK : map_cuda_error(e);
    pamo::s3::Stage3 &S = ctx->s3;
    if (rc == PAMO_OK) {
        const long long keep_limit = S.cg_spin_limit;
        S.cg_spin_limit = spin_limit;
        S.cg_absent_block = 1;
        rc = S.solve_bsr(n, d_i, d_i + n + 1, d_blk, n, d_dg, d_rhs, 4, d_out, s);
        S.cg_spin_limit = keep_limit;
        S.cg_absent_block = -1;
        if (rc == PAMO_OK && S.cg_persistent != 1) rc = PAMO_ERR_INVALID_ARG;  // no waits to test here
    }
    cudaFree(d_i);
    cudaFree(d_f);
    return rc;
}

int pamo_bsr_pcg(pamo_ctx *ctx, int n, const int *d_row_ptr, const int *d_col, const float *d_blocks,
                 long long n_blocks, const float *d_diag, const float *d_rhs, int iters, float *d_out, void *stream)
{
    if (!ctx || n <= 0 || n_blocks <= 0 || iters < 0 || !d_row_ptr || !d_col || !d_blocks || !d_diag || !d_rhs ||
        !d_out)
        return PAMO_ERR_INVALID_ARG;
    RET_IF(set_device(ctx));
    cudaStream_t s = (cudaStream_t)stream;
    pamo::s3::Stage3 &S = ctx->s3;
    RET_IF(S.ensure(n, 1, 1, 1, 1, 1));
    int *bad = S.iscal + 8;
    RET_IF(s3_validate(d_col, n_blocks, n, bad, S.h_iscal, s));
    return S.solve_bsr(n, d_row_ptr, d_col, d_blocks, n_blocks, d_diag, d_rhs, iters, d_out, s);
}

int pamo_simplify_ctx(pamo_ctx *ctx, const float *h_in_verts, const int *h_in_tris, float *h_out_verts,
                      int *h_out_tris, int *in_out_nv_ni, float threshold)
{
    if (!ctx || !h_in_verts || !h_in_tris || !h_out_verts || !h_out_tris || !in_out_nv_ni) return PAMO_ERR_INVALID_ARG;
    int n = in_out_nv_ni[0], m = in_out_nv_ni[1];
    if (n <= 0 || m <= 0) return PAMO_ERR_INVALID_ARG;
    RET_IF(set_device(ctx));
    cudaStream_t s = 0;
    Stage2 &S = ctx->s2;
    RET_IF(S.ensure(n, m));
    RET_IF(ensure_stage(ctx, 3LL * n + 3, 3LL * m + 3));
    // scale from the host bounding box, as the reference computes it (cusimpinterface.cu:64-77)
    float bbox[6] = {-1e30f, -1e30f, -1e30f, 1e30f, 1e30f, 1e30f};
    for (int i = 0; i < n; i++) {
        bbox[0] = std::max(bbox[0], h_in_verts[i * 3]);
        bbox[1] = std::max(bbox[1], h_in_verts[i * 3 + 1]);
        bbox[2] = std::max(bbox[2], h_in_verts[i * 3 + 2]);
        bbox[3] = std::min(bbox[3], h_in_verts[i * 3]);
        bbox[4] = std::min(bbox[4], h_in_verts[i * 3 + 1]);
        bbox[5] = std::min(bbox[5], h_in_verts[i * 3 + 2]);
    }
    float scale = std::max({bbox[0] - bbox[3], bbox[1] - bbox[4], bbox[2] - bbox[5]});
    CU_RET(cudaMemcpyAsync(ctx->stage, h_in_verts, (size_t)n * 12, cudaMemcpyHostToDevice, s));
    CU_RET(cudaMemcpyAsync(ctx->istage, h_in_tris, (size_t)m * 12, cudaMemcpyHostToDevice, s));
    RET_IF(S.validate(ctx->istage, n, m, nullptr, 0, 0, s));
    launch(k_aos3_to_f4, grid_for(n), kThreads, 0, s, ctx->stage, S.opts, n);
    launch(k_aos3_to_i4, grid_for(m), kThreads, 0, s, ctx->istage, S.otris, m);
    const int tolerance = 4;
    int same = 0, n_undo = 0;
    bool stuck = false, init = true;
    for (int it = 0; it < 1000000; it++) {
        if (init) RET_IF(stage2_shuffle_faces(S.otris, m, s));
        init = false;
        int nvu = 0;
        // the reference passes its own undo list back in (cusimpinterface.cu:103-105)
        RET_IF(S.round(n, m, scale, threshold, stuck, n_undo ? S.undo_list : nullptr, n_undo, &nvu, s, it > 0));
        n_undo = nvu;
        RET_IF(S.compact(n, m, s));
        int old_m = m;
        n = S.hcnt->n_pts_next;
        m = S.hcnt->n_tris_next;
        in_out_nv_ni[0] = n;
        in_out_nv_ni[1] = m;
        if (old_m == m) same++;
        else {
            same = 0;
            stuck = false;
        }
        if (same >= 2) stuck = true;
        if (same >= tolerance) break;
    }
    launch(k_f4_to_aos3, grid_for(n), kThreads, 0, s, S.opts, ctx->stage, n, 0, 0, 0, 0);
    launch(k_i4_to_aos3, grid_for(m), kThreads, 0, s, S.otris, ctx->istage, m);
    CU_RET(cudaMemcpyAsync(h_out_verts, ctx->stage, (size_t)n * 12, cudaMemcpyDeviceToHost, s));
    CU_RET(cudaMemcpyAsync(h_out_tris, ctx->istage, (size_t)m * 12, cudaMemcpyDeviceToHost, s));
    CU_RET(cudaStreamSynchronize(s));
    return PAMO_OK;
}

void pamo_simplify(float *in_verts, int *in_tris, float *out_verts, int *out_tris, int *in_out_nv_ni, float threshold)
{
    static pamo_ctx *g_ctx = nullptr;
    if (!g_ctx && pamo_ctx_create(0, &g_ctx) != PAMO_OK) {
        fprintf(stderr, "pamo_simplify: no CUDA device\n");
        return;
    }
    int rc = pamo_simplify_ctx(g_ctx, in_verts, in_tris, out_verts, out_tris, in_out_nv_ni, threshold);
    if (rc != PAMO_OK) fprintf(stderr, "pamo_simplify: %s\n", pamo_status_string(rc));
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched simplification engine (pamo_batch_*): many meshes of any sizes are
// packed into the rounds of one Stage2 (see SlotInfo), admitted while the packed
// capacity and the device-memory budget allow, and retired as soon as their own
// loop (PaMO.run's termination rules) ends, so new meshes join between rounds.

namespace pamo {
namespace {

struct JobHeader {  // device scalars of one mesh
    float mean[4];    // centring offset (numpy's tris mean)
    float scale;      // max bounding-box extent after centring
    float pad[3];
    int bounds[8];    // ordered-int box of the centred points
};

__global__ void k_scale_from_bounds(JobHeader *h)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float b[6];
    for (int k = 0; k < 6; ++k) b[k] = ordered_to_float(h->bounds[k]);
    float sx = b[3] - b[0], sy = b[4] - b[1], sz = b[5] - b[2];
    float scale = sy > sx ? sy : sx;  // Python max() keeps the first maximal argument
    h->scale = sz > scale ? sz : scale;
}

__global__ void k_aos3_to_i4_off(const int *in, int4 *out, int n, int off)
{
    PAMO_GRID_STRIDE(i, n) out[i] = make_int4(in[3 * i] + off, in[3 * i + 1] + off, in[3 * i + 2] + off, 0);
}

// a finished mesh out of the packed arrays: points + centring offset, faces rebased
__global__ void k_b_extract(const float4 *opts, const int4 *otris, int voff, int n, int foff, int m,
                            const JobHeader *h, float *out_p, int *out_t)
{
    const float ox = h->mean[0], oy = h->mean[1], oz = h->mean[2];
    PAMO_GRID_STRIDE(i, (long long)(n > m ? n : m))
    {
        if (i < n) {
            float4 p = opts[voff + i];
            out_p[3 * i] = p.x + ox;
            out_p[3 * i + 1] = p.y + oy;
            out_p[3 * i + 2] = p.z + oz;
        }
        if (i < m) {
            int4 t = otris[foff + i];
            out_t[3 * i] = t.x - voff;
            out_t[3 * i + 1] = t.y - voff;
            out_t[3 * i + 2] = t.z - voff;
        }
    }
}

struct Move {
    int src_v, dst_v, n, src_f, dst_f, m;
};

// kept meshes moved down to close the gaps of retired ones (into the other buffer)
__global__ void k_b_repack(const Move *moves, const float4 *src_p, const int4 *src_t, float4 *dst_p, int4 *dst_t)
{
    const Move mv = moves[blockIdx.y];
    const int shift = mv.src_v - mv.dst_v;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (mv.n > mv.m ? mv.n : mv.m);
         i += (long long)blockDim.x * gridDim.x) {
        if (i < mv.n) dst_p[mv.dst_v + i] = src_p[mv.src_v + i];
        if (i < mv.m) {
            int4 t = src_t[mv.src_f + i];
            dst_t[mv.dst_f + i] = make_int4(t.x - shift, t.y - shift, t.z - shift, 0);
        }
    }
}

struct BatchJob {
    long long id = 0;
    int state = PAMO_JOB_PENDING;
    int n0 = 0, m0 = 0;
    float *raw_p = nullptr;  // device copy of the input until admission
    int *raw_t = nullptr;
    long long target = 0;
    int tolerance = 4, iters = 1000000;
    float threshold = 1e-3f;
    uint32_t collapse_t = 0;
    // while running
    int n = 0, m = 0, vert_off = 0, face_off = 0;
    int rounds = 0, count = 0, n_undo = 0;
    bool stuck = false;
    unsigned char *region = nullptr;
    long long region_bytes = 0;
    SlotInfo tmpl{};
    JobHeader *hdr = nullptr;
    // finished
    float *out_p = nullptr;
    int *out_t = nullptr;
    int n_out = 0, m_out = 0;
};

long long region_bytes_for(long long n0, long long m0, long long *cap_undo)
{
    long long cu = 16 * (n0 + 1) + 6 * m0 + 16;
    *cap_undo = cu;
    auto al = [](long long b) { return (b + 255) / 256 * 256; };
    return al(sizeof(JobHeader)) + al((3 * m0 + 1) * 4) + al((n0 + 1) * 4) + 3 * al(cu * 4) + al(n0 + 1);
}

}  // namespace
}  // namespace pamo

struct pamo_batch {
    int device = 0;
    cudaStream_t s = nullptr;
    pamo::Stage2 S;
    long long cap_v = 0, cap_f = 0, budget = 0, in_use = 0;
    int max_meshes = 0;
    int n_packed = 0, m_packed = 0;
    long long next_id = 1;
    std::vector<pamo::BatchJob *> pending, running;
    std::vector<pamo::BatchJob *> all;  // every job not yet released
    pamo::Move *d_moves = nullptr;
    pamo::Move *h_moves = nullptr;
    std::vector<int> nvu;
    long long rounds_run = 0;
    std::vector<long long> done_ids;  // jobs that finished or failed in the last step
    // The jobs' device memory (inputs, per-mesh regions, results) comes from the
    // engine's own stream-ordered pool, which keeps what it has mapped until the
    // engine is destroyed: a device pool that hands memory back at each
    // synchronisation stalled single rounds for up to 0.7 s remapping it.
    cudaMemPool_t pool = nullptr;
};

namespace pamo {
namespace {

BatchJob *find_job(pamo_batch *b, long long id)
{
    for (BatchJob *j : b->all)
        if (j->id == id) return j;
    return nullptr;
}

int batch_admit(pamo_batch *b, BatchJob *j)
{
    cudaStream_t s = b->s;
    Stage2 &S = b->S;
    long long cu = 0;
    j->region_bytes = region_bytes_for(j->n0, j->m0, &cu);
    CU_RET(cudaMallocFromPoolAsync((void **)&j->region, (size_t)j->region_bytes, b->pool, s));
    CU_RET(cudaMemsetAsync(j->region, 0, (size_t)j->region_bytes, s));
    auto al = [](long long x) { return (x + 255) / 256 * 256; };
    unsigned char *p = j->region;
    j->hdr = reinterpret_cast<JobHeader *>(p);
    p += al(sizeof(JobHeader));
    SlotInfo &t = j->tmpl;
    t = SlotInfo{};
    t.edge_cost = reinterpret_cast<uint32_t *>(p);
    p += al((3LL * j->m0 + 1) * 4);
    t.pts_map = reinterpret_cast<int *>(p);
    p += al((j->n0 + 1LL) * 4);
    t.undo_list = reinterpret_cast<int *>(p);
    p += al(cu * 4);
    t.tmp_undo = reinterpret_cast<int *>(p);
    p += al(cu * 4);
    t.undo_prev = reinterpret_cast<int *>(p);
    p += al(cu * 4);
    t.invalid = p;
    t.cap_v = j->n0 + 1;
    t.cap_undo = cu;
    t.scale = &j->hdr->scale;
    t.collapse_t = j->collapse_t;
    t.tres = j->threshold;
    // centring and scale as the single-mesh loop does, written at the packed tail
    const int voff = b->n_packed, foff = b->m_packed, n = j->n0, m = j->m0;
    float *mxyz = reinterpret_cast<float *>(S.plane);  // 3*m floats of scratch
    launch(k_face_means, grid_for(m), kThreads, 0, s, (const float *)j->raw_p, (const int *)j->raw_t, m, mxyz,
           mxyz + m, mxyz + 2LL * m);
    const int smem = 2 * 3 * kMeanChunk * (int)sizeof(float);
    CU_RET(cudaFuncSetAttribute(k_sequential_mean, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    launch(k_sequential_mean, 1, 1024, smem, s, (const float *)mxyz, (const float *)(mxyz + m),
           (const float *)(mxyz + 2LL * m), m, j->hdr->mean);
    launch(k_bounds_init, 1, 32, 0, s, j->hdr->bounds);
    launch(k_centre, grid_for(n), kThreads, 0, s, (const float *)j->raw_p, n, (const float *)j->hdr->mean,
           S.opts + voff, j->hdr->bounds);
    launch(k_scale_from_bounds, 1, 32, 0, s, j->hdr);
    launch(k_aos3_to_i4_off, grid_for(m), kThreads, 0, s, (const int *)j->raw_t, S.otris + foff, m, voff);
    RET_IF(stage2_shuffle_faces(S.otris + foff, m, s));
    CU_RET(cudaFreeAsync(j->raw_p, s));
    CU_RET(cudaFreeAsync(j->raw_t, s));
    j->raw_p = nullptr;
    j->raw_t = nullptr;
    b->in_use -= 12LL * (n + m);
    b->in_use += j->region_bytes;
    j->n = n;
    j->m = m;
    j->vert_off = voff;
    j->face_off = foff;
    j->state = PAMO_JOB_RUNNING;
    b->n_packed += n;
    b->m_packed += m;
    CU_RET(cudaGetLastError());
    return PAMO_OK;
}

int batch_finish(pamo_batch *b, BatchJob *j)
{
    cudaStream_t s = b->s;
    CU_RET(cudaMallocFromPoolAsync((void **)&j->out_p, (size_t)(j->n > 0 ? j->n : 1) * 12, b->pool, s));
    CU_RET(cudaMallocFromPoolAsync((void **)&j->out_t, (size_t)(j->m > 0 ? j->m : 1) * 12, b->pool, s));
    launch(k_b_extract, grid_for(j->n > j->m ? j->n : j->m), kThreads, 0, s, (const float4 *)b->S.opts,
           (const int4 *)b->S.otris, j->vert_off, j->n, j->face_off, j->m, (const JobHeader *)j->hdr, j->out_p,
           j->out_t);
    CU_RET(cudaFreeAsync(j->region, s));
    b->in_use -= j->region_bytes;
    b->in_use += 12LL * (j->n + j->m);
    j->region = nullptr;
    j->hdr = nullptr;
    j->n_out = j->n;
    j->m_out = j->m;
    j->state = PAMO_JOB_DONE;
    CU_RET(cudaGetLastError());
    return PAMO_OK;
}

void batch_fail(pamo_batch *b, BatchJob *j, int rc)
{
    if (j->region) cudaFreeAsync(j->region, b->s);
    if (j->raw_p) cudaFreeAsync(j->raw_p, b->s);
    if (j->raw_t) cudaFreeAsync(j->raw_t, b->s);
    j->region = nullptr;
    j->raw_p = nullptr;
    j->raw_t = nullptr;
    j->state = -rc;
}

}  // namespace
}  // namespace pamo

extern "C" {

int pamo_batch_create(int device, long long max_verts, long long max_faces, int max_meshes,
                      long long memory_budget, void *stream, pamo_batch **out)
{
    if (!out || max_verts <= 0 || max_faces <= 0 || max_meshes <= 0 || memory_budget < 0) return PAMO_ERR_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return PAMO_ERR_NO_DEVICE;
    if (device < 0 || device >= count) return PAMO_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return PAMO_ERR_DEVICE;
    pamo_batch *b = new (std::nothrow) pamo_batch();
    if (!b) return PAMO_ERR_OOM;
    {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        unsigned long long keep = ~0ull;
        if (cudaMemPoolCreate(&b->pool, &props) != cudaSuccess ||
            cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
            if (b->pool) cudaMemPoolDestroy(b->pool);
            delete b;
            return PAMO_ERR_DEVICE;
        }
    }
    b->device = device;
    b->s = (cudaStream_t)stream;
    b->cap_v = max_verts;
    b->cap_f = max_faces;
    b->max_meshes = max_meshes;
    b->budget = memory_budget;
    int rc = b->S.ensure(max_verts, max_faces);
    if (!rc) rc = b->S.ensure_batch(max_meshes);
    if (!rc && (cudaMalloc((void **)&b->d_moves, (size_t)max_meshes * sizeof(Move)) != cudaSuccess ||
                cudaMallocHost((void **)&b->h_moves, (size_t)max_meshes * sizeof(Move)) != cudaSuccess))
        rc = PAMO_ERR_OOM;
    if (rc) {
        pamo_batch_destroy(b);
        return rc;
    }
    b->nvu.resize(max_meshes);
    *out = b;
    return PAMO_OK;
}

int pamo_batch_destroy(pamo_batch *b)
{
    if (!b) return PAMO_ERR_INVALID_ARG;
    cudaSetDevice(b->device);
    if (b->s) cudaStreamSynchronize(b->s);
    for (BatchJob *j : b->all) {
        if (j->raw_p) cudaFree(j->raw_p);
        if (j->raw_t) cudaFree(j->raw_t);
        if (j->region) cudaFree(j->region);
        if (j->out_p) cudaFree(j->out_p);
        if (j->out_t) cudaFree(j->out_t);
        delete j;
    }
    b->S.release();
    if (b->S.slots) cudaFree(b->S.slots);
    if (b->S.scnt) cudaFree(b->S.scnt);
    if (b->S.roots) cudaFree(b->S.roots);
    if (b->S.vslot) cudaFree(b->S.vslot);
    if (b->S.gmap) cudaFree(b->S.gmap);
    if (b->S.line_list) cudaFree(b->S.line_list);
    if (b->S.cand) cudaFree(b->S.cand);
    if (b->S.hslots) cudaFreeHost(b->S.hslots);
    if (b->S.hscnt) cudaFreeHost(b->S.hscnt);
    if (b->d_moves) cudaFree(b->d_moves);
    if (b->h_moves) cudaFreeHost(b->h_moves);
    if (b->pool) cudaMemPoolDestroy(b->pool);
    delete b;
    return PAMO_OK;
}

int pamo_batch_submit(pamo_batch *b, const float *points, const int *tris, int n_pts, int n_tris, int on_host,
                      long long target_faces, int tolerance, float threshold, int iters, long long *out_job)
{
    if (!b || !points || !tris || n_pts <= 0 || n_tris <= 0 || !out_job || iters < 0) return PAMO_ERR_INVALID_ARG;
    if (n_pts > b->cap_v || n_tris > b->cap_f) return PAMO_ERR_CAPACITY;
    if (cudaSetDevice(b->device) != cudaSuccess) return PAMO_ERR_DEVICE;
    cudaStream_t s = b->s;
    if (on_host) {  // reject faces with indices outside [0, n) before anything reaches the device
        for (long long i = 0; i < 3LL * n_tris; ++i)
            if (tris[i] < 0 || tris[i] >= n_pts) return PAMO_ERR_INVALID_ARG;
    }
    BatchJob *j = new (std::nothrow) BatchJob();
    if (!j) return PAMO_ERR_OOM;
    j->n0 = n_pts;
    j->m0 = n_tris;
    j->target = target_faces;
    j->tolerance = tolerance;
    j->threshold = threshold;
    j->iters = iters;
    float ct = (0.0f > threshold) ? 0.0f : threshold;
    ct = (ct < 10.0f) ? ct : 10.0f;
    j->collapse_t = (uint32_t)(unsigned long long)(ct / 10.0f * 4294967296.0f);
    if (cudaMallocFromPoolAsync((void **)&j->raw_p, (size_t)n_pts * 12, b->pool, s) != cudaSuccess ||
        cudaMallocFromPoolAsync((void **)&j->raw_t, (size_t)n_tris * 12, b->pool, s) != cudaSuccess) {
        batch_fail(b, j, PAMO_ERR_OOM);
        delete j;
        return PAMO_ERR_OOM;
    }
    cudaMemcpyKind kind = on_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    if (cudaMemcpyAsync(j->raw_p, points, (size_t)n_pts * 12, kind, s) != cudaSuccess ||
        cudaMemcpyAsync(j->raw_t, tris, (size_t)n_tris * 12, kind, s) != cudaSuccess) {
        batch_fail(b, j, PAMO_ERR_DEVICE);
        delete j;
        return PAMO_ERR_DEVICE;
    }
    if (!on_host) {  // device input: check the indices on the device before admitting
        int rc = b->S.validate(j->raw_t, n_pts, n_tris, nullptr, 0, 0, s);
        if (rc) {
            batch_fail(b, j, rc);
            delete j;
            return rc;
        }
    } else if (cudaStreamSynchronize(s) != cudaSuccess) {  // the caller may reuse its host buffers now
        batch_fail(b, j, PAMO_ERR_DEVICE);
        delete j;
        return PAMO_ERR_DEVICE;
    }
    b->in_use += 12LL * (n_pts + n_tris);
    j->id = b->next_id++;
    b->pending.push_back(j);
    b->all.push_back(j);
    *out_job = j->id;
    return PAMO_OK;
}

int pamo_batch_step(pamo_batch *b, int *out_running, int *out_pending)
{
    if (!b) return PAMO_ERR_INVALID_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess) return PAMO_ERR_DEVICE;
    cudaStream_t s = b->s;
    Stage2 &S = b->S;
    b->done_ids.clear();
    // admission: every pending mesh that fits the packed capacity, the mesh
    // count and the memory budget, in submission order
    for (size_t k = 0; k < b->pending.size();) {
        BatchJob *j = b->pending[k];
        long long cu = 0;
        long long need = region_bytes_for(j->n0, j->m0, &cu);
        bool fits = b->n_packed + (long long)j->n0 <= b->cap_v && b->m_packed + (long long)j->m0 <= b->cap_f &&
                    (int)b->running.size() < b->max_meshes &&
                    (b->budget == 0 || b->in_use + need - 12LL * (j->n0 + j->m0) <= b->budget);
        if (!fits) {
            ++k;
            continue;
        }
        int rc = batch_admit(b, j);
        b->pending.erase(b->pending.begin() + k);
        if (rc) {
            batch_fail(b, j, rc);
            b->done_ids.push_back(j->id);
            continue;
        }
        if (j->iters == 0) {  // no round: the centred, permuted input comes back, as from the plain loop
            rc = batch_finish(b, j);
            if (rc) batch_fail(b, j, rc);
            b->done_ids.push_back(j->id);
            b->n_packed -= j->n0;  // it was the last one packed
            b->m_packed -= j->m0;
            continue;
        }
        b->running.push_back(j);
    }
    const int K = (int)b->running.size();
    if (K > 0) {
        for (int r = 0; r < K; ++r) {
            BatchJob *j = b->running[r];
            SlotInfo &h = S.hslots[r];
            h = j->tmpl;
            h.vert_off = j->vert_off;
            h.n = j->n;
            h.face_off = j->face_off;
            h.m = j->m;
            h.is_stuck = j->stuck ? 1 : 0;
            h.n_undo_in = j->n_undo;
            h.clear_invalid = (!j->stuck && j->n_undo != 0) ? 1 : 0;
        }
        int rc = S.round_batch(b->n_packed, b->m_packed, K, b->nvu.data(), s);
        if (!rc) rc = S.compact_batch(b->n_packed, b->m_packed, K, s);
        if (rc) {  // a device or capacity error fails every mesh of the round
            for (BatchJob *j : b->running) {
                batch_fail(b, j, rc);
                b->done_ids.push_back(j->id);
            }
            b->running.clear();
            b->n_packed = b->m_packed = 0;
            return rc;
        }
        b->rounds_run++;
        // PaMO.run's loop per mesh (simp_cuda/pamo/__init__.py:169-185)
        std::vector<BatchJob *> keep;
        int n_moves = 0, dst_v = 0, dst_f = 0;
        bool moved = false;
        for (int r = 0; r < K; ++r) {
            BatchJob *j = b->running[r];
            const SlotCounters &c = S.hscnt[r];
            const int prev = j->m;
            j->rounds++;
            j->n_undo = b->nvu[r];
            j->n = c.n_next;
            j->m = c.m_next;
            j->vert_off = c.vert_off_next;
            j->face_off = c.face_off_next;
            bool done = (long long)j->m <= j->target || j->m <= 10;
            if (!done) {
                if (j->m == prev) j->count++;
                else {
                    j->count = 0;
                    j->stuck = false;
                }
                if (j->count >= 2) j->stuck = true;
                if (j->count == j->tolerance) done = true;
            }
            if (j->rounds >= j->iters) done = true;
            if (done) {
                int frc = batch_finish(b, j);
                if (frc) batch_fail(b, j, frc);
                b->done_ids.push_back(j->id);
                moved = true;
                continue;
            }
            if (j->vert_off != dst_v || j->face_off != dst_f) moved = true;
            b->h_moves[n_moves++] = Move{j->vert_off, dst_v, j->n, j->face_off, dst_f, j->m};
            j->vert_off = dst_v;
            j->face_off = dst_f;
            dst_v += j->n;
            dst_f += j->m;
            keep.push_back(j);
        }
        if (moved && n_moves > 0) {
            int max_len = 0;
            for (int k = 0; k < n_moves; ++k) {
                int l = b->h_moves[k].n > b->h_moves[k].m ? b->h_moves[k].n : b->h_moves[k].m;
                max_len = l > max_len ? l : max_len;
            }
            CU_RET(cudaMemcpyAsync(b->d_moves, b->h_moves, (size_t)n_moves * sizeof(Move), cudaMemcpyHostToDevice, s));
            long long gx = (max_len + kThreads - 1) / kThreads;
            gx = gx < 1 ? 1 : (gx > 64 ? 64 : gx);
            launch(k_b_repack, dim3((unsigned)gx, (unsigned)n_moves), kThreads, 0, s, (const Move *)b->d_moves,
                   (const float4 *)S.opts, (const int4 *)S.otris, S.pts, S.tris);
            std::swap(S.opts, S.pts);
            std::swap(S.otris, S.tris);
            CU_RET(cudaGetLastError());
            CU_RET(cudaStreamSynchronize(s));  // h_moves is rewritten by the next step
        }
        b->running.swap(keep);
        b->n_packed = dst_v;
        b->m_packed = dst_f;
    }
    if (out_running) *out_running = (int)b->running.size();
    if (out_pending) *out_pending = (int)b->pending.size();
    return PAMO_OK;
}

int pamo_batch_finished(pamo_batch *b, long long *h_out, int cap)
{
    if (!b || cap < 0 || (cap && !h_out)) return -PAMO_ERR_INVALID_ARG;
    const int n = (int)b->done_ids.size();
    for (int i = 0; i < n && i < cap; ++i) h_out[i] = b->done_ids[i];
    return n;
}

int pamo_batch_job(pamo_batch *b, long long job, int *state, int *n_pts, int *n_tris, int *rounds)
{
    if (!b) return PAMO_ERR_INVALID_ARG;
    BatchJob *j = find_job(b, job);
    if (!j) return PAMO_ERR_INVALID_ARG;
    if (state) *state = j->state;
    if (n_pts) *n_pts = j->state == PAMO_JOB_DONE ? j->n_out : j->n;
    if (n_tris) *n_tris = j->state == PAMO_JOB_DONE ? j->m_out : j->m;
    if (rounds) *rounds = j->rounds;
    return PAMO_OK;
}

int pamo_batch_fetch(pamo_batch *b, long long job, float *out_points, int *out_tris, int to_host)
{
    if (!b || !out_points || !out_tris) return PAMO_ERR_INVALID_ARG;
    BatchJob *j = find_job(b, job);
    if (!j || j->state != PAMO_JOB_DONE) return PAMO_ERR_INVALID_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess) return PAMO_ERR_DEVICE;
    cudaMemcpyKind kind = to_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    CU_RET(cudaMemcpyAsync(out_points, j->out_p, (size_t)j->n_out * 12, kind, b->s));
    CU_RET(cudaMemcpyAsync(out_tris, j->out_t, (size_t)j->m_out * 12, kind, b->s));
    CU_RET(cudaStreamSynchronize(b->s));
    return PAMO_OK;
}

int pamo_batch_release(pamo_batch *b, long long job)
{
    if (!b) return PAMO_ERR_INVALID_ARG;
    for (size_t k = 0; k < b->all.size(); ++k) {
        BatchJob *j = b->all[k];
        if (j->id != job) continue;
        if (j->state == PAMO_JOB_PENDING || j->state == PAMO_JOB_RUNNING) return PAMO_ERR_INVALID_ARG;
        cudaSetDevice(b->device);
        if (j->out_p) cudaFreeAsync(j->out_p, b->s);
        if (j->out_t) cudaFreeAsync(j->out_t, b->s);
        b->in_use -= 12LL * (j->n_out + j->m_out);
        b->all.erase(b->all.begin() + k);
        delete j;
        return PAMO_OK;
    }
    return PAMO_ERR_INVALID_ARG;
}

int pamo_batch_profile(pamo_batch *b, int enable, double *h_ms, long long *h_calls, int cap)
{
    if (!b || cap < 0) return -PAMO_ERR_INVALID_ARG;
    Profiler &P = b->S.prof;
    int n = cap < PH_COUNT ? cap : PH_COUNT;
    for (int i = 0; i < n; ++i) {
        if (h_ms) h_ms[i] = P.ms[i];
        if (h_calls) h_calls[i] = P.calls[i];
    }
    if (enable >= 0) {
        P.on = enable != 0;
        P.reset();
    }
    return PH_COUNT;
}

int pamo_batch_stats(pamo_batch *b, long long *h_out8)
{
    if (!b || !h_out8) return PAMO_ERR_INVALID_ARG;
    h_out8[0] = (long long)b->running.size();
    h_out8[1] = (long long)b->pending.size();
    h_out8[2] = b->n_packed;
    h_out8[3] = b->m_packed;
    h_out8[4] = b->in_use;
    h_out8[5] = b->rounds_run;
    h_out8[6] = b->cap_f;
    h_out8[7] = b->budget;
    return PAMO_OK;
}

}  // extern "C"
