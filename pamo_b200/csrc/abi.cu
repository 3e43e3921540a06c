// C ABI entry points (include/pamo_b200.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>

#include "scan.cuh"
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
// divides by F.  That chain is inherently sequential.  One block: warps 1..31
// stream the next chunk into shared memory while thread 0 runs the three
// coordinate chains (interleaved, so the FADD latency is the bound) on the
// current chunk.
constexpr int kMeanChunk = 4096;

__global__ void __launch_bounds__(1024) k_sequential_mean(const float *mx, const float *my, const float *mz, int m,
                                                          float *out)
{
    extern __shared__ float sm[];  // 2 buffers x 3 coordinates x kMeanChunk
    if (m <= 0) return;
    const int n_chunks = (m + kMeanChunk - 1) / kMeanChunk;
    auto load = [&](int c, int buf) {
        float *dst = sm + buf * 3 * kMeanChunk;
        int base = c * kMeanChunk;
        int cnt = min(kMeanChunk, m - base);
        for (int i = threadIdx.x - 32; i < cnt; i += blockDim.x - 32) {
            dst[i] = mx[base + i];
            dst[kMeanChunk + i] = my[base + i];
            dst[2 * kMeanChunk + i] = mz[base + i];
        }
    };
    if (threadIdx.x >= 32) load(0, 0);
    __syncthreads();
    float sx = 0.f, sy = 0.f, sz = 0.f;
    for (int c = 0; c < n_chunks; ++c) {
        const int buf = c & 1;
        if (threadIdx.x >= 32) {
            if (c + 1 < n_chunks) load(c + 1, buf ^ 1);
        } else if (threadIdx.x == 0) {
            const float *b = sm + buf * 3 * kMeanChunk;
            int cnt = min(kMeanChunk, m - c * kMeanChunk);
            int i = 0;
            if (c == 0) {  // the accumulator starts from the first row
                sx = b[0];
                sy = b[kMeanChunk];
                sz = b[2 * kMeanChunk];
                i = 1;
            }
#pragma unroll 8
            for (; i < cnt; ++i) {
                sx += b[i];
                sy += b[kMeanChunk + i];
                sz += b[2 * kMeanChunk + i];
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sx / (float)m;
        out[1] = sy / (float)m;
        out[2] = sz / (float)m;
    }
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

extern "C" {

int pamo_version(void) { return 100; }

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
    k_aos3_to_f4<<<grid_for(n_pts), kThreads, 0, s>>>(d_points, S.opts, n_pts);
    k_aos3_to_i4<<<grid_for(n_tris), kThreads, 0, s>>>(d_tris, S.otris, n_tris);
    if (init) RET_IF(stage2_shuffle_faces(S.otris, n_tris, s));
    int nvu = 0;
    RET_IF(S.round(n_pts, n_tris, scale, threshold, is_stuck != 0, d_verts_undo, n_verts_undo, &nvu, s));
    if (d_out_points) k_f4_to_aos3<<<grid_for(n_pts), kThreads, 0, s>>>(S.pts, d_out_points, n_pts, 0, 0, 0, 0);
    if (d_out_tris) k_i4_to_aos3<<<grid_for(n_tris), kThreads, 0, s>>>(S.tris, d_out_tris, n_tris);
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

int pamo_stage2_run(pamo_ctx *ctx, const float *d_points, const int *d_tris, int n_pts, int n_tris,
                    long long target_faces, int tolerance, float threshold, int iters, void *stream, int *out_n_pts,
                    int *out_n_tris, int *out_rounds)
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
    k_face_means<<<grid_for(n_tris), kThreads, 0, s>>>(d_points, d_tris, n_tris, mxyz, mxyz + n_tris,
                                                       mxyz + 2LL * n_tris);
    {
        const int smem = 2 * 3 * kMeanChunk * (int)sizeof(float);
        CU_RET(cudaFuncSetAttribute(k_sequential_mean, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        k_sequential_mean<<<1, 1024, smem, s>>>(mxyz, mxyz + n_tris, mxyz + 2LL * n_tris, n_tris, mean_dev);
    }
    k_bounds_init<<<1, 32, 0, s>>>(bounds);
    k_centre<<<grid_for(n_pts), kThreads, 0, s>>>(d_points, n_pts, mean_dev, S.opts, bounds);
    k_bounds_to_float<<<1, 32, 0, s>>>(bounds, bounds_f);
    k_aos3_to_i4<<<grid_for(n_tris), kThreads, 0, s>>>(d_tris, S.otris, n_tris);
    RET_IF(stage2_shuffle_faces(S.otris, n_tris, s));
    CU_RET(cudaMemcpyAsync(S.h_scalars, mean_dev, 3 * 4, cudaMemcpyDeviceToHost, s));
    CU_RET(cudaMemcpyAsync(S.h_scalars + 4, bounds_f, 6 * 4, cudaMemcpyDeviceToHost, s));
    CU_RET(cudaStreamSynchronize(s));
    for (int k = 0; k < 3; ++k) S.offset[k] = S.h_scalars[k];
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
        RET_IF(S.round(n, m, scale, threshold, stuck, n_undo ? ctx->undo_prev : nullptr, n_undo, &nvu, s));
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

int pamo_stage2_fetch(pamo_ctx *ctx, float *out_points, int *out_tris, int to_host, void *stream)
{
    if (!ctx || !out_points || !out_tris) return PAMO_ERR_INVALID_ARG;
    RET_IF(set_device(ctx));
    cudaStream_t s = (cudaStream_t)stream;
    Stage2 &S = ctx->s2;
    int n = S.res_n_pts, m = S.res_n_tris;
    if (to_host) {
        RET_IF(ensure_stage(ctx, 3LL * n + 3, 3LL * m + 3));
        k_f4_to_aos3<<<grid_for(n), kThreads, 0, s>>>(S.opts, ctx->stage, n, S.offset[0], S.offset[1], S.offset[2], 1);
        k_i4_to_aos3<<<grid_for(m), kThreads, 0, s>>>(S.otris, ctx->istage, m);
        CU_RET(cudaMemcpyAsync(out_points, ctx->stage, (size_t)n * 12, cudaMemcpyDeviceToHost, s));
        CU_RET(cudaMemcpyAsync(out_tris, ctx->istage, (size_t)m * 12, cudaMemcpyDeviceToHost, s));
    } else {
        k_f4_to_aos3<<<grid_for(n), kThreads, 0, s>>>(S.opts, out_points, n, S.offset[0], S.offset[1], S.offset[2], 1);
        k_i4_to_aos3<<<grid_for(m), kThreads, 0, s>>>(S.otris, out_tris, m);
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
    k_aos3_to_f4<<<grid_for(n_pts), kThreads, 0, s>>>(d_points, S.opts, n_pts);
    k_aos3_to_i4<<<grid_for(n_tris), kThreads, 0, s>>>(d_tris, S.otris, n_tris);
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
    int *bad = S.iscal + 8;
    RET_IF(s3_validate(d_f, 3LL * n_f, n_v, bad, S.h_iscal, s));
    RET_IF(s3_validate(d_e, 2LL * n_e, n_v, bad, S.h_iscal, s));
    RET_IF(s3_validate(d_h, 4LL * n_h, n_v, bad, S.h_iscal, s));
    RET_IF(s3_validate(d_gt_f, 3LL * n_gt_f, n_gt_v, bad, S.h_iscal, s));
    S.do_nothing = do_nothing != 0;
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
    ctx->s3_stats[0] = e;
    ctx->s3_stats[1] = S.h_iscal[0];
    ctx->s3_stats[2] = newton;
    return PAMO_OK;
}

int pamo_safe_project_stats(pamo_ctx *ctx, double *h_out3)
{
    if (!ctx || !h_out3) return PAMO_ERR_INVALID_ARG;
    for (int k = 0; k < 3; ++k) h_out3[k] = ctx->s3_stats[k];
    return PAMO_OK;
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
    k_aos3_to_f4<<<grid_for(n), kThreads, 0, s>>>(ctx->stage, S.opts, n);
    k_aos3_to_i4<<<grid_for(m), kThreads, 0, s>>>(ctx->istage, S.otris, m);
    const int tolerance = 4;
    int same = 0, n_undo = 0;
    bool stuck = false, init = true;
    for (int it = 0; it < 1000000; it++) {
        if (init) RET_IF(stage2_shuffle_faces(S.otris, m, s));
        init = false;
        int nvu = 0;
        // the reference passes its own undo list back in (cusimpinterface.cu:103-105)
        RET_IF(S.round(n, m, scale, threshold, stuck, n_undo ? S.undo_list : nullptr, n_undo, &nvu, s));
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
    k_f4_to_aos3<<<grid_for(n), kThreads, 0, s>>>(S.opts, ctx->stage, n, 0, 0, 0, 0);
    k_i4_to_aos3<<<grid_for(m), kThreads, 0, s>>>(S.otris, ctx->istage, m);
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
