// Stage-3 safe projection kernels and driver (see stage3.cuh).
//
// Energy terms (default configuration of the reference, config.py:27-38):
//   GT attraction   0.5 * w_i * k * |x_i - t_i|^2, t_i = closest GT point
//                   (distance_energy.py:6-46, geometry_kernels.py:82-94)
//   membrane        StVK in each triangle's 2-D frame, mu = E/2(1+nu), lambda
//                   (elastic_energy.py:8-220; its Hessian product holds the frame
//                   fixed, as the reference's does)
//   bending         0.5 * k * (theta - theta0)^2 * l0 per interior edge
//                   (hinge_energy.py:5-274); Hessian blocks of Tamstorf &
//                   Grinspun (2013), SPD-projected
//   contact         kappa * b(d), b(d) = -(d - dh)^2 ln(d / dh) for d < dh
//                   (collision_energy.py:8-99,192-254,379-411), Gauss-Newton
//                   Hessian kappa b''(d) grad(d) grad(d)^T
#include <cooperative_groups.h>
#include <cstdio>
#include <cstring>

#include "distance.cuh"
#include "scan.cuh"
#include "stage3.cuh"

namespace cg = cooperative_groups;

namespace pamo {
namespace s3 {

namespace {

constexpr int kRedBlocks = 296;  // fixed grid for deterministic reductions (2 x 148 SMs)
constexpr int kStack = 96;

enum { D_ENERGY = 0, D_ENERGY_PREV, D_ZR, D_ZR_LAST, D_VAV };
enum { I_NB = 0, I_OVERFLOW, I_STACK, I_NACT, I_NCAND_PT, I_NCAND_EE, I_TICKET, I_DISP, I_BAR_ERR, I_BAR_COUNT,
       I_BAR_GEN, I_ETICKET, I_LS, I_TRACE };

__device__ __forceinline__ F3 ld(const float4 *a, int i) { return f3(a[i]); }
__device__ __forceinline__ void st(float4 *a, int i, F3 v) { a[i] = make_float4(v.x, v.y, v.z, 0.f); }
// one vector reduction (sm_90+, global memory) instead of three scalar ones
__device__ __forceinline__ void atomic_add3(float4 *a, int i, F3 v)
{
    atomicAdd(&a[i], make_float4(v.x, v.y, v.z, 0.f));
}

// ---------------------------------------------------------------- barrier (FP64)
__device__ __forceinline__ double barrier(double d, double dh) { return -(d - dh) * (d - dh) * log(d / dh); }
__device__ __forceinline__ double barrier_d1(double d, double dh)
{
    double t = d - dh;
    return -2.0 * t * log(d / dh) - t * t / d;
}
__device__ __forceinline__ double barrier_d2(double d, double dh)
{
    return -2.0 * log(d / dh) - 2.0 * (d - dh) / d - 1.0 + (dh * dh) / (d * d);
}

// --------------------------------------------------------------- reductions
template <int BLOCK>
__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double ws[BLOCK / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) ws[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = lane < BLOCK / 32 ? ws[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;
}

// Each reduction kernel writes one partial per block; the last block to finish
// (a ticket counter, no waiting) adds the partials in a fixed order (32 lanes
// strided over the blocks, then a shuffle tree), so the sums are deterministic
// and a separate finishing launch is not needed.  Returns true in the last block (all its threads).
__device__ __forceinline__ bool last_block_sum(double block_total, double *partials, int *ticket, double *dst)
{
    __shared__ bool s_last;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = block_total;
        __threadfence();
        s_last = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    if (threadIdx.x < 32) {
        double v = 0.0;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) v += __ldcg(&partials[i]);
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) {
            *dst = v;
            *ticket = 0;
        }
    }
    return true;
}

// ------------------------------------------------------------ preprocessing
__global__ void k_aos_to_f4(const float *in, float4 *a, float4 *b, int n)
{
    PAMO_GRID_STRIDE(i, n)
    {
        float4 v = make_float4(in[3 * i], in[3 * i + 1], in[3 * i + 2], 0.f);
        a[i] = v;
        if (b) b[i] = v;
    }
}

__global__ void k_aos_to_i4(const int *in, int4 *out, int n, int stride, int dup_last)
{
    PAMO_GRID_STRIDE(i, n)
    {
        if (stride == 3) out[i] = make_int4(in[3 * i], in[3 * i + 1], in[3 * i + 2], 0);
        else if (stride == 2) out[i] = make_int4(in[2 * i], in[2 * i + 1], dup_last ? in[2 * i + 1] : 0, 0);
        else out[i] = make_int4(in[4 * i], in[4 * i + 1], in[4 * i + 2], in[4 * i + 3]);
    }
}

__device__ __forceinline__ void frame(F3 x01, F3 x02, F3 &b1, F3 &b2)
{
    b1 = normalized(x01);
    b2 = x02 - dot(x02, b1) * b1;
    b2 = normalized(b2);
}

__global__ void k_elastic_pre(const float4 *x, const int4 *tris, int nt, float *area, float4 *inv_dm)
{
    PAMO_GRID_STRIDE(t, nt)
    {
        int4 f = tris[t];
        F3 x0 = ld(x, f.x), x1 = ld(x, f.y), x2 = ld(x, f.z);
        F3 x01 = x1 - x0, x02 = x2 - x0;
        area[t] = 0.5f * len(cross(x01, x02));
        F3 b1, b2;
        frame(x01, x02, b1, b2);
        float a = dot(b1, x01), b = dot(b1, x02), c = dot(b2, x01), d = dot(b2, x02);
        float det = a * d - b * c;
        inv_dm[t] = make_float4(d / det, -b / det, -c / det, a / det);
    }
}

__device__ __forceinline__ float hinge_theta(F3 x0, F3 x1, F3 x2, F3 x3)
{
    F3 e12 = normalized(x2 - x1);
    F3 n1 = normalized(cross(e12, x0 - x1));
    F3 n2 = normalized(cross(x3 - x1, e12));
    return atan2f(dot(cross(n1, n2), e12), dot(n1, n2));
}

__global__ void k_hinge_pre(const float4 *x, const int4 *h, int nh, float *rest_angle, float *rest_elen)
{
    PAMO_GRID_STRIDE(k, nh)
    {
        int4 i = h[k];
        F3 x0 = ld(x, i.x), x1 = ld(x, i.y), x2 = ld(x, i.z), x3 = ld(x, i.w);
        rest_angle[k] = hinge_theta(x0, x1, x2, x3);
        rest_elen[k] = len(x1 - x2);
    }
}

// ------------------------------------------------- closest point on the GT mesh
__device__ F3 closest_on_triangle(F3 p, F3 a, F3 b, F3 c)
{
    // Ericson, Real-Time Collision Detection, section 5.1.5
    F3 ab = b - a, ac = c - a, ap = p - a;
    float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.f && d2 <= 0.f) return a;
    F3 bp = p - b;
    float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.f && d4 <= d3) return b;
    float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) return a + (d1 / (d1 - d3)) * ab;
    F3 cp = p - c;
    float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.f && d5 <= d6) return c;
    float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) return a + (d2 / (d2 - d6)) * ac;
    float va = d3 * d6 - d5 * d4;
    if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) return b + ((d4 - d3) / ((d4 - d3) + (d5 - d6))) * (c - b);
    float den = 1.f / (va + vb + vc);
    return a + (vb * den) * ab + (vc * den) * ac;
}

__device__ __forceinline__ float box_dist2(float4 lo, float4 hi, F3 p)
{
    float dx = fmaxf(fmaxf(lo.x - p.x, 0.f), p.x - hi.x);
    float dy = fmaxf(fmaxf(lo.y - p.y, 0.f), p.y - hi.y);
    float dz = fmaxf(fmaxf(lo.z - p.z, 0.f), p.z - hi.z);
    return dx * dx + dy * dy + dz * dz;
}

__global__ void __launch_bounds__(kThreads) k_closest(const float4 *q, int np, const BvhNode *nodes, const int *vals,
                                                      const int *scene, const float4 *gpts, const int4 *gtris,
                                                      float4 *target, int *iscal)
{
    const int L = scene[7];
    int stack[kStack];
    PAMO_GRID_STRIDE(i, np)
    {
        F3 p = ld(q, (int)i);
        float best = 1e18f;  // max_dist 1e9, squared
        F3 bestp = mk(1e9f, 1e9f, 1e9f);
        if (L == 1) {
            int4 t = gtris[vals[0]];
            bestp = closest_on_triangle(p, ld(gpts, t.x), ld(gpts, t.y), ld(gpts, t.z));
        } else if (L > 1) {
            int sp = 0;
            stack[sp++] = 0;
            int budget = 4 * L + 64;
            while (sp > 0) {
                if (--budget < 0) {
                    atomicAdd(&iscal[I_STACK], 1);
                    break;
                }
                const BvhNode nd = nodes[stack[--sp]];
                float dl = box_dist2(nd.llo, nd.lhi, p), dr = box_dist2(nd.rlo, nd.rhi, p);
                int cl = __float_as_int(nd.llo.w), cr = __float_as_int(nd.rlo.w);
                // visit the nearer child first: push it last
                int first = dl <= dr ? 0 : 1;
                for (int k = 0; k < 2; ++k) {
                    int side = k == 0 ? 1 - first : first;
                    float dd = side ? dr : dl;
                    int child = side ? cr : cl;
                    if (dd >= best) continue;
                    if (child < 0) {
                        int4 t = gtris[vals[~child]];
                        F3 c = closest_on_triangle(p, ld(gpts, t.x), ld(gpts, t.y), ld(gpts, t.z));
                        float d2 = dot(c - p, c - p);
                        if (d2 < best) {
                            best = d2;
                            bestp = c;
                        }
                    } else if (sp < kStack) {
                        stack[sp++] = child;
                    } else {
                        atomicAdd(&iscal[I_STACK], 1);
                    }
                }
            }
        }
        st(target, (int)i, bestp);
    }
}

// ------------------------------------------------------------ contact detection
__device__ __forceinline__ bool overlap(float4 lo, float4 hi, F3 qlo, F3 qhi)
{
    return !(hi.x < qlo.x || qhi.x < lo.x || hi.y < qlo.y || qhi.y < lo.y || hi.z < qlo.z || qhi.z < lo.z);
}

__device__ __forceinline__ void append_block(int4 idx, int kind, int *iscal, long long cap, int4 *bidx, int *bkind)
{
    cg::coalesced_group g = cg::coalesced_threads();
    int base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(&iscal[I_NB], (int)g.size());
    int pos = g.shfl(base, 0) + (int)g.thread_rank();
    if (pos < cap) {
        bidx[pos] = idx;
        bkind[pos] = kind;
    }
}

// Detection runs in two passes.  The traversals (one thread per vertex or edge,
// few threads for a small mesh) only emit candidate pairs whose boxes overlap
// with a margin; the classification and distance test then runs one thread per
// candidate, and a pair is kept when its classified distance is within thr, as
// in contact_detection.py.  The candidates are gathered with thr + extra and
// kept: while no vertex has moved more than extra / 2 since, every pair within
// thr is among them (each of its two primitives moved at most extra / 2), so
// later detections only rerun the test.
__device__ __forceinline__ void append_pair(int a, int b, int *counter, long long cap, int2 *out)
{
    cg::coalesced_group g = cg::coalesced_threads();
    int base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(counter, (int)g.size());
    int pos = g.shfl(base, 0) + (int)g.thread_rank();
    if (pos < cap) out[pos] = make_int2(a, b);
}

// point-triangle candidates (contact_detection.py:120-164)
__global__ void __launch_bounds__(kThreads) k_detect_pt(const float4 *q, int np, const int4 *tris, const BvhNode *nodes,
                                                        const int *vals, const int *scene, float thr, int *iscal,
                                                        long long cap_c, int2 *cand)
{
    const int L = scene[7];
    int stack[kStack];
    PAMO_GRID_STRIDE(ii, np)
    {
        const int i = (int)ii;
        F3 x0 = ld(q, i);
        F3 qlo = mk(x0.x - thr, x0.y - thr, x0.z - thr), qhi = mk(x0.x + thr, x0.y + thr, x0.z + thr);
        int sp = 0;
        int leaf_only = L == 1 ? 1 : 0;
        if (L > 1) stack[sp++] = 0;
        int budget = 2 * L + 16;
        while (sp > 0 || leaf_only) {
            int c2[2] = {-1, -1};
            if (leaf_only) {
                c2[0] = vals[0];
                leaf_only = 0;
            } else {
                if (--budget < 0) {
                    atomicAdd(&iscal[I_STACK], 1);
                    break;
                }
                const BvhNode nd = nodes[stack[--sp]];
                for (int side = 0; side < 2; ++side) {
                    float4 lo = side ? nd.rlo : nd.llo, hi = side ? nd.rhi : nd.lhi;
                    if (!overlap(lo, hi, qlo, qhi)) continue;
                    int child = __float_as_int(lo.w);
                    if (child < 0) c2[side] = vals[~child];
                    else if (sp < kStack) stack[sp++] = child;
                    else atomicAdd(&iscal[I_STACK], 1);
                }
            }
            for (int k = 0; k < 2; ++k) {
                int f = c2[k];
                if (f < 0) continue;
                int4 t = tris[f];
                if (t.x == i || t.y == i || t.z == i) continue;
                append_pair(i, f, &iscal[I_NCAND_PT], cap_c, cand);
            }
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_test_pt(const float4 *q, const int4 *tris, const int2 *cand,
                                                      long long cap_c, float thr, int *iscal, long long cap,
                                                      int4 *bidx, int *bkind)
{
    const long long n = min((long long)iscal[I_NCAND_PT], cap_c);
    PAMO_GRID_STRIDE(k, n)
    {
        int2 c = cand[k];
        int4 t = tris[c.y];
        F3 x[4] = {ld(q, c.x), ld(q, t.x), ld(q, t.y), ld(q, t.z)};
        int ty = pt_classify(x[0], x[1], x[2], x[3]);
        float d = classified_distance(KIND_PT, ty, x);
        if (d <= thr) append_block(make_int4(c.x, t.x, t.y, t.z), KIND_PT, iscal, cap, bidx, bkind);
    }
}

// largest displacement of a vertex since the candidates were gathered (float
// bits of a non-negative value order like ints)
__global__ void k_max_disp(const float4 *q, const float4 *q_gather, int np, int *iscal)
{
    float m = 0.f;
    PAMO_GRID_STRIDE(i, np) m = fmaxf(m, len(ld(q, (int)i) - ld(q_gather, (int)i)));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(&iscal[I_DISP], __float_as_int(m));
}

// edge-edge candidates (contact_detection.py:168-216)
__global__ void __launch_bounds__(kThreads) k_detect_ee(const float4 *q, int ne, const int4 *edges4,
                                                        const BvhNode *nodes, const int *vals, const int *scene,
                                                        float thr, int *iscal, long long cap_c, int2 *cand)
{
    const int L = scene[7];
    int stack[kStack];
    PAMO_GRID_STRIDE(ee, ne)
    {
        const int e0 = (int)ee;
        int4 a = edges4[e0];
        F3 x0 = ld(q, a.x), x1 = ld(q, a.y);
        F3 qlo = mk(fminf(x0.x, x1.x) - thr, fminf(x0.y, x1.y) - thr, fminf(x0.z, x1.z) - thr);
        F3 qhi = mk(fmaxf(x0.x, x1.x) + thr, fmaxf(x0.y, x1.y) + thr, fmaxf(x0.z, x1.z) + thr);
        if (L < 2) continue;
        int sp = 0;
        stack[sp++] = 0;
        int budget = 2 * L + 16;
        while (sp > 0) {
            if (--budget < 0) {
                atomicAdd(&iscal[I_STACK], 1);
                break;
            }
            const BvhNode nd = nodes[stack[--sp]];
            for (int side = 0; side < 2; ++side) {
                float4 lo = side ? nd.rlo : nd.llo, hi = side ? nd.rhi : nd.lhi;
                if (!overlap(lo, hi, qlo, qhi)) continue;
                int child = __float_as_int(lo.w);
                if (child >= 0) {
                    if (sp < kStack) stack[sp++] = child;
                    else atomicAdd(&iscal[I_STACK], 1);
                    continue;
                }
                int e1 = vals[~child];
                if (e1 <= e0) continue;
                int4 b = edges4[e1];
                if (a.x == b.x || a.x == b.y || a.y == b.x || a.y == b.y) continue;
                append_pair(e0, e1, &iscal[I_NCAND_EE], cap_c, cand);
            }
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_test_ee(const float4 *q, const int4 *edges4, const int2 *cand,
                                                      long long cap_c, float thr, float ee_thres, int *iscal,
                                                      long long cap, int4 *bidx, int *bkind)
{
    const long long n = min((long long)iscal[I_NCAND_EE], cap_c);
    PAMO_GRID_STRIDE(k, n)
    {
        int2 c = cand[k];
        int4 a = edges4[c.x], b = edges4[c.y];
        F3 x[4] = {ld(q, a.x), ld(q, a.y), ld(q, b.x), ld(q, b.y)};
        int ty = ee_classify(x[0], x[1], x[2], x[3], ee_thres);
        float d = classified_distance(KIND_EE, ty, x);
        if (d <= thr) append_block(make_int4(a.x, a.y, b.x, b.y), KIND_EE, iscal, cap, bidx, bkind);
    }
}

// ------------------------------------------------------------------- energy
struct EArgs {
    const float4 *q, *target;
    const float *wk;
    int np, nt, nh;
    const int4 *tris;
    const float *area;
    const float4 *inv_dm;
    float mu, la;
    const int4 *hinges;
    const float *rest_angle, *rest_elen;
    float hinge_k;
    const int4 *bidx;
    const int *bkind;
    int *bsub;
    float *bd;
    int *iscal;  // block count; I_ETICKET: the energy sum's ticket
    long long cap_b;
    float d_hat, kappa, ee_thres;
    double *partials;
    // line search: halving n_halves > 0 is skipped once a trial was accepted
    // (energy below the start's), as the reference's loop stops there
    int n_halves;
    double *dscal;  // D_ENERGY: written by the last block
    // line search (n_halves >= 0): the largest step length of a vertex, which
    // bounds how far a block's distance can have moved from the start's bd
    const float *step_bound;
};

__device__ __forceinline__ void elastic_F(const float4 *q, int4 f, float4 im, F3 &b1, F3 &b2, float F[4])
{
    F3 x0 = ld(q, f.x), x1 = ld(q, f.y), x2 = ld(q, f.z);
    F3 x01 = x1 - x0, x02 = x2 - x0;
    frame(x01, x02, b1, b2);
    float d00 = dot(b1, x01), d01 = dot(b1, x02), d10 = dot(b2, x01), d11 = dot(b2, x02);
    F[0] = d00 * im.x + d01 * im.z;
    F[1] = d00 * im.y + d01 * im.w;
    F[2] = d10 * im.x + d11 * im.z;
    F[3] = d10 * im.y + d11 * im.w;
}

// This thread's share (elements first, first + stride, ...) of the energy at
// A.q: the mesh-to-target, membrane, hinge and barrier terms.
__device__ double energy_terms(const EArgs &A, long long first, long long stride)
{
    const long long nb = min((long long)A.iscal[I_NB], A.cap_b);
    const long long total = (long long)A.np + A.nt + A.nh + nb;
    double acc = 0.0;
    for (long long k = first; k < total; k += stride) {
        if (k < A.np) {
            F3 d = ld(A.q, (int)k) - ld(A.target, (int)k);
            acc += (double)(0.5f * dot(d, d) * A.wk[k]);
        } else if (k < (long long)A.np + A.nt) {
            int t = (int)(k - A.np);
            F3 b1, b2;
            float F[4];
            elastic_F(A.q, A.tris[t], A.inv_dm[t], b1, b2, F);
            // E = 0.5 (F^T F - I)
            float e00 = 0.5f * (F[0] * F[0] + F[2] * F[2] - 1.f);
            float e01 = 0.5f * (F[0] * F[1] + F[2] * F[3]);
            float e11 = 0.5f * (F[1] * F[1] + F[3] * F[3] - 1.f);
            float tr = e00 + e11;
            float ee = e00 * e00 + 2.f * e01 * e01 + e11 * e11;
            acc += (double)(A.area[t] * (A.mu * ee + 0.5f * A.la * tr * tr));
        } else if (k < (long long)A.np + A.nt + A.nh) {
            int h = (int)(k - A.np - A.nt);
            int4 i = A.hinges[h];
            float th = hinge_theta(ld(A.q, i.x), ld(A.q, i.y), ld(A.q, i.z), ld(A.q, i.w));
            float dt = th - A.rest_angle[h];
            acc += (double)(0.5f * A.hinge_k * dt * dt * A.rest_elen[h]);
        } else {
            int b = (int)(k - A.np - A.nt - A.nh);
            if (A.n_halves >= 0) {
                // A trial point: every vertex moved at most step_bound from the
                // start, where the block's distance was bd, and a pair distance
                // changes by at most the sum of its two primitives' largest
                // moves.  A block that stays beyond d_hat adds nothing (the
                // margin covers the fp32 evaluation of the distances).
                if (A.bd[b] - 2.f * *A.step_bound > A.d_hat + 1e-5f) continue;
            }
            int4 i = A.bidx[b];
            int kind = A.bkind[b];
            F3 x[4] = {ld(A.q, i.x), ld(A.q, i.y), ld(A.q, i.z), ld(A.q, i.w)};
            int ty = classify(kind, x, A.ee_thres);
            float d = classified_distance(kind, ty, x);
            if (A.n_halves < 0) {  // the start of a Newton iteration: kept for the differentials
                A.bsub[b] = ty;
                A.bd[b] = d;
            }
            if (d < A.d_hat) acc += barrier((double)d, (double)A.d_hat) * (double)A.kappa;
        }
    }
    return acc;
}

__global__ void __launch_bounds__(kThreads) k_energy(EArgs A)
{
    // D_ENERGY then still holds the accepted trial's energy
    if (A.n_halves > 0 && A.dscal[D_ENERGY] < A.dscal[D_ENERGY_PREV]) return;
    const double acc = energy_terms(A, (long long)blockIdx.x * blockDim.x + threadIdx.x,
                                    (long long)blockDim.x * gridDim.x);
    last_block_sum(block_sum<kThreads>(acc), A.partials, A.iscal + I_ETICKET, A.dscal + D_ENERGY);
}

// --------------------------------------------------------------------- diff
// vertex part: grad = -(x - t) w, diag = w (writes, before the atomics)
__global__ void k_diff_vertex(const float4 *q, const float4 *target, const float *wk, int np, float4 *grad,
                              float4 *diag)
{
    PAMO_GRID_STRIDE(i, np)
    {
        float w = wk[i];
        F3 g = ld(q, (int)i) - ld(target, (int)i);
        st(grad, (int)i, (-w) * g);
        diag[i] = make_float4(w, w, w, 0.f);
    }
}

// Hinge gradient and Hessian blocks (Tamstorf & Grinspun 2013, in the form of
// hinge_energy.py:91-254): writes the 16 row-major 3x3 blocks into B.
__device__ void hinge_blocks(F3 x0, F3 x1, F3 x2, F3 x3, float rest_angle, float rest_elen, float k, F3 g[4],
                             float B[16][9], float &dE)
{
    F3 e0 = x2 - x1, e1 = x0 - x2, e2 = x0 - x1, e1_ = x3 - x2, e2_ = x3 - x1;
    float l0 = len(e0), l1 = len(e1), l2 = len(e2), l1_ = len(e1_), l2_ = len(e2_);
    F3 u0 = normalized(e0), u1 = normalized(e1), u2 = normalized(e2), u1_ = normalized(e1_), u2_ = normalized(e2_);
    float ca1 = dot(u2, u0), ca2 = -dot(u1, u0), ca1_ = dot(u2_, u0), ca2_ = -dot(u1_, u0);
    float h0 = len(cross(e1, e2)) / l0, h1 = len(cross(e0, e2)) / l1, h2 = len(cross(e0, e1)) / l2;
    float h0_ = len(cross(e1_, e2_)) / l0, h1_ = len(cross(e0, e2_)) / l1_, h2_ = len(cross(e0, e1_)) / l2_;
    F3 n = normalized(cross(e0, e2)), n_ = normalized(cross(e2_, e0));
    float th = atan2f(dot(cross(n, n_), e0) / l0, dot(n, n_));
    dE = k * (th - rest_angle) * rest_elen;
    float d2E = k * rest_elen;
    g[0] = (-1.f / h0) * n;
    g[3] = (-1.f / h0_) * n_;
    g[1] = (ca2 / h1) * n + (ca2_ / h1_) * n_;
    g[2] = (ca1 / h2) * n + (ca1_ / h2_) * n_;
    F3 m0 = normalized(cross(e0, n)), m1 = normalized(cross(e1, n)), m2 = normalized(cross(n, e2));
    F3 m0_ = normalized(cross(n_, e0)), m1_ = normalized(cross(n_, e1_)), m2_ = normalized(cross(e2_, n_));
    auto outer = [](F3 a, F3 b, float *o) {
        o[0] = a.x * b.x; o[1] = a.x * b.y; o[2] = a.x * b.z;
        o[3] = a.y * b.x; o[4] = a.y * b.y; o[5] = a.y * b.z;
        o[6] = a.z * b.x; o[7] = a.z * b.y; o[8] = a.z * b.z;
    };
    // M = n m^T; P_xy = c * M^T / (h h); Q = M / (h h); N0 = M0 / l0^2
    float M0[9], M1[9], M2[9], M0_[9], M1_[9], M2_[9];
    outer(n, m0, M0); outer(n, m1, M1); outer(n, m2, M2);
    outer(n_, m0_, M0_); outer(n_, m1_, M1_); outer(n_, m2_, M2_);
    const float il0 = 1.f / (l0 * l0);
    float G[9];
    auto T = [](const float *a, int r, int c) { return a[c * 3 + r]; };  // transpose access
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            const int rc = r * 3 + c;
            // block (0,0): -sym(Q0) dE
            float q0 = M0[rc] / (h0 * h0), q0t = T(M0, r, c) / (h0 * h0);
            float q0_ = M0_[rc] / (h0_ * h0_), q0_t = T(M0_, r, c) / (h0_ * h0_);
            B[0][rc] = -(q0 + q0t) * dE;
            B[15][rc] = -(q0_ + q0_t) * dE;
            // block (1,1): (sym(P11) - N0 + sym(P11_) - N0_) dE
            float p11 = ca1 * T(M1, r, c) / (h1 * h1), p11t = ca1 * M1[rc] / (h1 * h1);
            float p11_ = ca1_ * T(M1_, r, c) / (h1_ * h1_), p11_t = ca1_ * M1_[rc] / (h1_ * h1_);
            B[5][rc] = (p11 + p11t - M0[rc] * il0 + p11_ + p11_t - M0_[rc] * il0) * dE;
            // block (2,2): (sym(P22) - N0 + sym(P22_) - N0_) dE
            float p22 = ca2 * T(M2, r, c) / (h2 * h2), p22t = ca2 * M2[rc] / (h2 * h2);
            float p22_ = ca2_ * T(M2_, r, c) / (h2_ * h2_), p22_t = ca2_ * M2_[rc] / (h2_ * h2_);
            B[10][rc] = (p22 + p22t - M0[rc] * il0 + p22_ + p22_t - M0_[rc] * il0) * dE;
            // block (1,0): (P10 - Q1) dE ; (2,0): (P20 - Q2) dE
            B[4][rc] = (ca1 * T(M0, r, c) / (h1 * h0) - M1[rc] / (h0 * h1)) * dE;
            B[8][rc] = (ca2 * T(M0, r, c) / (h2 * h0) - M2[rc] / (h0 * h2)) * dE;
            // block (1,3): (P10_ - Q1_) dE ; (2,3): (P20_ - Q2_) dE
            B[7][rc] = (ca1_ * T(M0_, r, c) / (h1_ * h0_) - M1_[rc] / (h0_ * h1_)) * dE;
            B[11][rc] = (ca2_ * T(M0_, r, c) / (h2_ * h0_) - M2_[rc] / (h0_ * h2_)) * dE;
            // block (1,2): (P12 + P21^T + N0 + P12_ + P21_^T + N0_) dE
            float p12 = ca1 * T(M2, r, c) / (h1 * h2);
            float p21t = ca2 * M1[rc] / (h2 * h1);
            float p12_ = ca1_ * T(M2_, r, c) / (h1_ * h2_);
            float p21_t = ca2_ * M1_[rc] / (h2_ * h1_);
            B[6][rc] = (p12 + p21t + M0[rc] * il0 + p12_ + p21_t + M0_[rc] * il0) * dE;
            B[3][rc] = 0.f;
        }
    // + d2E * outer(g_i, g_j) on the blocks above, block (0,3) is pure outer
    const int pairs[10][2] = {{0, 0}, {3, 3}, {1, 1}, {2, 2}, {1, 0}, {2, 0}, {1, 3}, {2, 3}, {1, 2}, {0, 3}};
    for (int k2 = 0; k2 < 10; ++k2) {
        int i = pairs[k2][0], j = pairs[k2][1];
        outer(g[i], g[j], G);
        for (int e = 0; e < 9; ++e) B[i * 4 + j][e] += d2E * G[e];
    }
    // mirrored blocks
    const int mir[6][2] = {{0, 1}, {0, 2}, {3, 1}, {3, 2}, {2, 1}, {3, 0}};
    for (int k2 = 0; k2 < 6; ++k2) {
        int i = mir[k2][0], j = mir[k2][1];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) B[i * 4 + j][r * 3 + c] = B[j * 4 + i][c * 3 + r];
    }
}

struct DArgs {
    const float4 *q;
    int nt, nh;
    const int4 *tris;
    const float *area;
    const float4 *inv_dm;
    float mu, la;
    const int4 *hinges;
    const float *rest_angle, *rest_elen;
    float hinge_k;
    int spd_iters;
    float4 *kval;
    const int *tri_slot, *hinge_slot;
    float *hblk;  // the unprojected hinge blocks, for k_hinge_spd
    const int4 *bidx;
    const int *bkind, *bsub;
    const float *bd;
    float4 *bg;
    float *bb2;
    int *iscal;
    long long cap_b;
    float d_hat, kappa;
    float4 *grad, *diag;
    int *bact;  // contact blocks with d < d_hat, appended here for the CG products
};

// one 3x3 block (row-major) added into the assembled Hessian
__device__ __forceinline__ void add_block(float4 *kval, int slot, const float *m)
{
    atomicAdd(&kval[3 * (size_t)slot], make_float4(m[0], m[1], m[2], 0.f));
    atomicAdd(&kval[3 * (size_t)slot + 1], make_float4(m[3], m[4], m[5], 0.f));
    atomicAdd(&kval[3 * (size_t)slot + 2], make_float4(m[6], m[7], m[8], 0.f));
}

// The membrane Hessian's action on a displacement of the triangle's edge
// vectors (dx01, dx02): dF, dE = (dF^T F + F^T dF) / 2, dS, dP = dF S + F dS,
// and the forces on vertices 1 and 2 (vertex 0 gets minus their sum).
__device__ __forceinline__ void membrane_apply(F3 b1, F3 b2, const float F[4], float S00, float S01, float S11,
                                               float4 im, float W, float mu, float la, F3 dx01, F3 dx02, F3 &f1, F3 &f2)
{
    float s00 = dot(b1, dx01), s01 = dot(b1, dx02), s10 = dot(b2, dx01), s11 = dot(b2, dx02);
    float dF[4] = {s00 * im.x + s01 * im.z, s00 * im.y + s01 * im.w, s10 * im.x + s11 * im.z, s10 * im.y + s11 * im.w};
    float de00 = dF[0] * F[0] + dF[2] * F[2];
    float de01 = 0.5f * (dF[0] * F[1] + dF[2] * F[3] + F[0] * dF[1] + F[2] * dF[3]);
    float de11 = dF[1] * F[1] + dF[3] * F[3];
    float trd = de00 + de11;
    float T00 = 2.f * mu * de00 + la * trd, T01 = 2.f * mu * de01, T11 = 2.f * mu * de11 + la * trd;
    float dP00 = dF[0] * S00 + dF[1] * S01 + F[0] * T00 + F[1] * T01;
    float dP01 = dF[0] * S01 + dF[1] * S11 + F[0] * T01 + F[1] * T11;
    float dP10 = dF[2] * S00 + dF[3] * S01 + F[2] * T00 + F[3] * T01;
    float dP11 = dF[2] * S01 + dF[3] * S11 + F[2] * T01 + F[3] * T11;
    float H00 = W * (dP00 * im.x + dP01 * im.y), H01 = W * (dP00 * im.z + dP01 * im.w);
    float H10 = W * (dP10 * im.x + dP11 * im.y), H11 = W * (dP10 * im.z + dP11 * im.w);
    f1 = H00 * b1 + H10 * b2;
    f2 = H01 * b1 + H11 * b2;
}

// One kind of element per launch (PART 0 membranes, 1 hinges, 2 contact
// blocks), so the three run as concurrent branches of the iteration and each
// is compiled for its own register count.
template <int PART>
__global__ void __launch_bounds__(128) k_diff_part(DArgs A)
{
    const long long nb = min((long long)A.iscal[I_NB], A.cap_b);
    const long long first = PART == 0 ? 0 : PART == 1 ? (long long)A.nt : (long long)A.nt + A.nh;
    const long long count = PART == 0 ? (long long)A.nt : PART == 1 ? (long long)A.nh : nb;
    PAMO_GRID_STRIDE(j, count)
    {
        const long long k = first + j;
        if (PART == 0) {
            int t = (int)k;
            int4 f = A.tris[t];
            F3 b1, b2;
            float F[4];
            float4 im = A.inv_dm[t];
            elastic_F(A.q, f, im, b1, b2, F);
            float e00 = 0.5f * (F[0] * F[0] + F[2] * F[2] - 1.f);
            float e01 = 0.5f * (F[0] * F[1] + F[2] * F[3]);
            float e11 = 0.5f * (F[1] * F[1] + F[3] * F[3] - 1.f);
            float tr = e00 + e11;
            // S = 2 mu E + la tr(E) I ; P = F S ; H = -W P inv_dm^T
            float s00 = 2.f * A.mu * e00 + A.la * tr, s01 = 2.f * A.mu * e01, s11 = 2.f * A.mu * e11 + A.la * tr;
            float P00 = F[0] * s00 + F[1] * s01, P01 = F[0] * s01 + F[1] * s11;
            float P10 = F[2] * s00 + F[3] * s01, P11 = F[2] * s01 + F[3] * s11;
            float W = -A.area[t];
            float H00 = W * (P00 * im.x + P01 * im.y), H01 = W * (P00 * im.z + P01 * im.w);
            float H10 = W * (P10 * im.x + P11 * im.y), H11 = W * (P10 * im.z + P11 * im.w);
            F3 f1 = H00 * b1 + H10 * b2, f2 = H01 * b1 + H11 * b2;
            F3 f0 = mk(-f1.x - f2.x, -f1.y - f2.y, -f1.z - f2.z);
            atomic_add3(A.grad, f.x, f0);
            atomic_add3(A.grad, f.y, f1);
            atomic_add3(A.grad, f.z, f2);
            // the membrane Hessian: the linear map (dx01, dx02) -> (force 1, force 2)
            // on the six unit displacements gives M (6 x 6); vertex 0's rows and
            // columns follow from dx01 = x1 - x0, dx02 = x2 - x0 and f0 = -f1 - f2
            float M[6][6];  // M[row][col]: rows f1.xyz, f2.xyz; columns dx01.xyz, dx02.xyz
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                F3 e = mk(c % 3 == 0 ? 1.f : 0.f, c % 3 == 1 ? 1.f : 0.f, c % 3 == 2 ? 1.f : 0.f);
                F3 z0 = mk(0.f, 0.f, 0.f), g1, g2;
                membrane_apply(b1, b2, F, s00, s01, s11, im, A.area[t], A.mu, A.la, c < 3 ? e : z0, c < 3 ? z0 : e,
                               g1, g2);
                M[0][c] = g1.x; M[1][c] = g1.y; M[2][c] = g1.z;
                M[3][c] = g2.x; M[4][c] = g2.y; M[5][c] = g2.z;
            }
            const int *slot = A.tri_slot + 9 * (size_t)t;
            float blk[9];
            // K_ab for a, b in {1, 2}: M's 3x3 sub-blocks; K_a0 = -(K_a1 + K_a2); K_0b = -(K_1b + K_2b)
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j) {
                            auto kk = [&](int aa, int bb) { return M[3 * (aa - 1) + i][3 * (bb - 1) + j]; };
                            float val;
                            if (a > 0 && b > 0) val = kk(a, b);
                            else if (a > 0) val = -(kk(a, 1) + kk(a, 2));
                            else if (b > 0) val = -(kk(1, b) + kk(2, b));
                            else val = kk(1, 1) + kk(1, 2) + kk(2, 1) + kk(2, 2);
                            blk[3 * i + j] = val;
                        }
                    add_block(A.kval, slot[3 * a + b], blk);
                }
        } else if (PART == 1) {
            int h = (int)(k - A.nt);
            int4 i = A.hinges[h];
            int idx[4] = {i.x, i.y, i.z, i.w};
            F3 g[4];
            float B[16][9];
            float dE;
            hinge_blocks(ld(A.q, i.x), ld(A.q, i.y), ld(A.q, i.z), ld(A.q, i.w), A.rest_angle[h], A.rest_elen[h],
                         A.hinge_k, g, B, dE);
            for (int a = 0; a < 4; ++a) {
                atomic_add3(A.grad, idx[a], (-dE) * g[a]);
                // diagonal of the unprojected block, as the reference adds it before projecting
                atomic_add3(A.diag, idx[a], mk(B[a * 5][0], B[a * 5][4], B[a * 5][8]));
            }
            float *dst = A.hblk + (size_t)h * 81;  // vertices 0-2: projected and assembled by k_hinge_spd
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    for (int e = 0; e < 9; ++e) dst[(a * 3 + b) * 9 + e] = B[a * 4 + b][e];
        } else {
            int b = (int)(k - A.nt - A.nh);
            float d = A.bd[b];
            if (!(d < A.d_hat)) {
                A.bb2[b] = 0.f;
                continue;
            }
            int4 i = A.bidx[b];
            int idx[4] = {i.x, i.y, i.z, i.w};
            F3 x[4] = {ld(A.q, i.x), ld(A.q, i.y), ld(A.q, i.z), ld(A.q, i.w)};
            F3 g[4];
            distance_grad(A.bkind[b], A.bsub[b], x, g);
            double b1 = barrier_d1((double)d, (double)A.d_hat) * (double)A.kappa;
            double b2 = barrier_d2((double)d, (double)A.d_hat) * (double)A.kappa;
            float b1f = (float)b1, b2f = (float)b2;
            for (int a = 0; a < 4; ++a) {
                A.bg[4 * (size_t)b + a] = make_float4(g[a].x, g[a].y, g[a].z, 0.f);
                atomic_add3(A.grad, idx[a], (-b1f) * g[a]);
                atomic_add3(A.diag, idx[a], mk(b2f * g[a].x * g[a].x, b2f * g[a].y * g[a].y, b2f * g[a].z * g[a].z));
            }
            A.bb2[b] = b2f;
            cg::coalesced_group grp = cg::coalesced_threads();
            int base = 0;
            if (grp.thread_rank() == 0) base = atomicAdd(&A.iscal[I_NACT], (int)grp.size());
            A.bact[grp.shfl(base, 0) + (int)grp.thread_rank()] = b;
        }
    }
}

// The SPD projection of the hinge blocks (block_spd_project_kernel,
// kernels/utils_kernels.py:20-39: the fork-only wp.spd_project_blocks(3, B, 3),
// read as an eigenvalue clamp): `sweeps` cyclic Jacobi sweeps
// on the symmetric part of the 9 x 9 matrix of hinge vertices 0-2, negative
// eigenvalues set to zero, then vertex 3's rows and columns refilled by
// translation invariance.  One thread per hinge with every rotation unrolled,
// so A and V live in registers (a rolled loop indexes them at run time, which
// puts them in local memory).  The projected blocks are added into the
// assembled Hessian.
__global__ void __launch_bounds__(64) k_hinge_spd(const float *hblk, int nh, int sweeps, const int *hinge_slot,
                                                  float4 *kval)
{
    const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nh) return;
    const float *src = hblk + (size_t)h * 81;  // blocks (a, b), a, b < 3, row-major
    float A[9][9], V[9][9];
#pragma unroll
    for (int bi = 0; bi < 3; ++bi)
#pragma unroll
        for (int bj = 0; bj < 3; ++bj)
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) A[bi * 3 + r][bj * 3 + c] = src[(bi * 3 + bj) * 9 + r * 3 + c];
#pragma unroll
    for (int i = 0; i < 9; ++i)
#pragma unroll
        for (int j = i + 1; j < 9; ++j) {
            float s = 0.5f * (A[i][j] + A[j][i]);
            A[i][j] = A[j][i] = s;
        }
#pragma unroll
    for (int i = 0; i < 9; ++i)
#pragma unroll
        for (int j = 0; j < 9; ++j) V[i][j] = i == j ? 1.f : 0.f;
    for (int sw = 0; sw < sweeps; ++sw) {
#pragma unroll
        for (int p = 0; p < 8; ++p)
#pragma unroll
            for (int qq = p + 1; qq < 9; ++qq) {
                float apq = A[p][qq];
                if (fabsf(apq) > 1e-30f) {
                    float theta = (A[qq][qq] - A[p][p]) / (2.f * apq);
                    float sg = theta >= 0.f ? 1.f : -1.f;
                    float t = sg / (fabsf(theta) + sqrtf(theta * theta + 1.f));
                    float c = 1.f / sqrtf(t * t + 1.f), s = t * c;
                    // A <- J^T A J in the symmetric form: rows and columns p and q
                    // (a_pq becomes 0, a_pp and a_qq move by -/+ t a_pq)
#pragma unroll
                    for (int k = 0; k < 9; ++k) {
                        if (k == p || k == qq) continue;
                        const float akp = A[k][p], akq = A[k][qq];
                        const float nkp = c * akp - s * akq, nkq = s * akp + c * akq;
                        A[k][p] = A[p][k] = nkp;
                        A[k][qq] = A[qq][k] = nkq;
                    }
                    A[p][p] -= t * apq;
                    A[qq][qq] += t * apq;
                    A[p][qq] = A[qq][p] = 0.f;
#pragma unroll
                    for (int k = 0; k < 9; ++k) {  // V <- V J
                        float vkp = V[k][p], vkq = V[k][qq];
                        V[k][p] = c * vkp - s * vkq;
                        V[k][qq] = s * vkp + c * vkq;
                    }
                }
            }
    }
    float lam[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) lam[i] = fmaxf(A[i][i], 0.f);
    // S = V diag(lam) V^T, into A
#pragma unroll
    for (int i = 0; i < 9; ++i)
#pragma unroll
        for (int j = 0; j < 9; ++j) {
            float s = 0.f;
#pragma unroll
            for (int k = 0; k < 9; ++k) s += V[i][k] * lam[k] * V[j][k];
            A[i][j] = s;
        }
    const int *sl = hinge_slot + 16 * (size_t)h;
    float blk[9], b3[3][9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) blk[r * 3 + c] = A[a * 3 + r][b * 3 + c];
            add_block(kval, sl[a * 4 + b], blk);
        }
#pragma unroll
    for (int j = 0; j < 3; ++j)  // block (3, j) = -(blocks (0, j) + (1, j) + (2, j))
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                b3[j][r * 3 + c] = -(A[0 + r][j * 3 + c] + A[3 + r][j * 3 + c] + A[6 + r][j * 3 + c]);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        add_block(kval, sl[12 + j], b3[j]);
#pragma unroll
        for (int r = 0; r < 3; ++r)  // block (j, 3) = block (3, j)^T
#pragma unroll
            for (int c = 0; c < 3; ++c) blk[r * 3 + c] = b3[j][c * 3 + r];
        add_block(kval, sl[j * 4 + 3], blk);
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) {  // block (3, 3) = -(blocks (0, 3) + (1, 3) + (2, 3)), block (j, 3) = (3, j)^T
        const int r = e / 3, c = e % 3;
        blk[e] = -(b3[0][c * 3 + r] + b3[1][c * 3 + r] + b3[2][c * 3 + r]);
    }
    add_block(kval, sl[15], blk);
}

// ---------------------------------------------------------------- A * dx
// The operator of the CG: rows of the assembled block matrix (vertex term,
// membrane, hinges) plus the rank-one Gauss-Newton terms of the contact blocks
// with d < d_hat (listed by k_diff_part<2>).
struct OpArgs {
    int np;
    const int *row_ptr, *col;
    const float4 *kval;
    const int4 *bidx;
    const float4 *bg;
    const float *bb2;
    const int *bact;
    const int *iscal;
    long long cap_b;
};

// Rows [first, ...) of K dx, eight rows per warp and four lanes per row (the
// loop bounds are warp-uniform, so the shuffles see the whole warp).  `ldx(j)`
// gives dx at vertex j; `row(i, (K dx)_i)` receives each finished row.
template <class LDX, class ROW>
__device__ __forceinline__ void op_rows(const OpArgs &A, long long warp0, long long nwarps, LDX ldx, ROW row)
{
    const int lane = threadIdx.x & 31, sub = lane & 3;
    for (long long base = warp0 * 8; base < A.np; base += nwarps * 8) {
        const long long i = base + (lane >> 2);
        F3 acc = mk(0.f, 0.f, 0.f);
        if (i < A.np) {
            const int e = A.row_ptr[i + 1];
            int s = A.row_ptr[i] + sub;
            // a lane's first kRowBatch slots with every load issued before any
            // use (the column, then dx there), so a row costs two round trips
            constexpr int kRowBatch = 4;
            int cidx[kRowBatch];
#pragma unroll
            for (int k = 0; k < kRowBatch; ++k) cidx[k] = s + 4 * k < e ? A.col[s + 4 * k] : -1;
            F3 x[kRowBatch];
#pragma unroll
            for (int k = 0; k < kRowBatch; ++k) x[k] = cidx[k] >= 0 ? ldx(cidx[k]) : mk(0.f, 0.f, 0.f);
#pragma unroll
            for (int k = 0; k < kRowBatch; ++k) {
                if (cidx[k] < 0) continue;
                const size_t b = 3 * (size_t)(s + 4 * k);
                const float4 k0 = A.kval[b], k1 = A.kval[b + 1], k2 = A.kval[b + 2];
                acc = acc + mk(k0.x * x[k].x + k0.y * x[k].y + k0.z * x[k].z, k1.x * x[k].x + k1.y * x[k].y + k1.z * x[k].z,
                               k2.x * x[k].x + k2.y * x[k].y + k2.z * x[k].z);
            }
            for (s += 4 * kRowBatch; s < e; s += 4) {  // rows longer than 4 x kRowBatch
                const F3 xx = ldx(A.col[s]);
                const float4 k0 = A.kval[3 * (size_t)s], k1 = A.kval[3 * (size_t)s + 1], k2 = A.kval[3 * (size_t)s + 2];
                acc = acc + mk(k0.x * xx.x + k0.y * xx.y + k0.z * xx.z, k1.x * xx.x + k1.y * xx.y + k1.z * xx.z,
                               k2.x * xx.x + k2.y * xx.y + k2.z * xx.z);
            }
        }
#pragma unroll
        for (int o = 1; o < 4; o <<= 1) {
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
            acc.z += __shfl_xor_sync(0xffffffffu, acc.z, o);
        }
        if (i < A.np && sub == 0) row((int)i, acc);
    }
}

// The contact terms c (g . dx) g of blocks [first, ...), added into out with
// atomics; returns this thread's share of dx . (their sum).
template <class LDX>
__device__ __forceinline__ double op_contacts(const OpArgs &A, long long first, long long stride, LDX ldx, float4 *out,
                                              long long nb)
{
    double dxh = 0.0;
    for (long long k = first; k < nb; k += stride) {
        const int b = A.bact[k];
        const float c = A.bb2[b];
        if (c == 0.f) continue;
        const int4 i = A.bidx[b];
        const int idx[4] = {i.x, i.y, i.z, i.w};
        F3 g[4];
        float s = 0.f;
        for (int a = 0; a < 4; ++a) {
            g[a] = f3(A.bg[4 * (size_t)b + a]);
            s += dot(g[a], ldx(idx[a]));
        }
        for (int a = 0; a < 4; ++a) atomic_add3(out, idx[a], (c * s) * g[a]);
        dxh += (double)(c * s) * (double)s;
    }
    return dxh;
}

// out = K dx (rows), then the contact terms in a second launch
__global__ void __launch_bounds__(kThreads) k_op_rows(OpArgs A, const float4 *dx, float4 *out)
{
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    op_rows(A, t0 >> 5, ((long long)blockDim.x * gridDim.x) >> 5, [&](int j) { return ld(dx, j); },
            [&](int i, F3 r) { st(out, i, r); });
}

__global__ void __launch_bounds__(kThreads) k_op_contacts(OpArgs A, const float4 *dx, float4 *out)
{
    op_contacts(A, (long long)blockIdx.x * blockDim.x + threadIdx.x, (long long)blockDim.x * gridDim.x,
                [&](int j) { return ld(dx, j); }, out, min((long long)A.iscal[I_NACT], A.cap_b));
}

// ------------------------------------------------------- the block pattern
// Built once per registered mesh: every element's ordered vertex pairs (and
// the diagonal) bucketed by row, each row sorted and deduplicated, then the
// position of every element block in its row.
__global__ void k_fill_int(int *a, long long n, int v)
{
    PAMO_GRID_STRIDE(i, n) a[i] = v;
}

__global__ void k_pat_count(const int4 *tris, int nt, const int4 *hinges, int nh, int *cnt)
{
    const long long total = (long long)nt + nh;
    PAMO_GRID_STRIDE(k, total)
    {
        if (k < nt) {
            const int4 t = tris[k];
            atomicAdd(&cnt[t.x], 2);
            atomicAdd(&cnt[t.y], 2);
            atomicAdd(&cnt[t.z], 2);
        } else {
            const int4 h = hinges[k - nt];
            atomicAdd(&cnt[h.x], 3);
            atomicAdd(&cnt[h.y], 3);
            atomicAdd(&cnt[h.z], 3);
            atomicAdd(&cnt[h.w], 3);
        }
    }
}

__global__ void k_pat_fill(const int4 *tris, int nt, const int4 *hinges, int nh, int np, const int *off, int *cur,
                           int *cand)
{
    const long long total = (long long)np + nt + nh;
    auto put = [&](int r, int c) { cand[off[r] + atomicAdd(&cur[r], 1)] = c; };
    PAMO_GRID_STRIDE(k, total)
    {
        if (k < np) {
            put((int)k, (int)k);
        } else if (k < (long long)np + nt) {
            const int4 t = tris[k - np];
            const int v[3] = {t.x, t.y, t.z};
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    if (a != b) put(v[a], v[b]);
        } else {
            const int4 h = hinges[k - np - nt];
            const int v[4] = {h.x, h.y, h.z, h.w};
            for (int a = 0; a < 4; ++a)
                for (int b = 0; b < 4; ++b)
                    if (a != b) put(v[a], v[b]);
        }
    }
}

__global__ void k_pat_sort(const int *off, int np, int *cand, int *ucnt)
{
    PAMO_GRID_STRIDE(v, np)
    {
        const int a = off[v], b = off[v + 1];
        for (int i = a + 1; i < b; ++i) {
            const int x = cand[i];
            int j = i - 1;
            while (j >= a && cand[j] > x) {
                cand[j + 1] = cand[j];
                --j;
            }
            cand[j + 1] = x;
        }
        int u = a;
        for (int i = a; i < b; ++i)
            if (u == a || cand[i] != cand[u - 1]) cand[u++] = cand[i];
        ucnt[v] = u - a;
    }
}

__global__ void k_pat_emit(const int *off, const int *row_ptr, const int *cand, int np, int *col)
{
    PAMO_GRID_STRIDE(v, np)
    {
        const int a = off[v], r = row_ptr[v], n = row_ptr[v + 1] - r;
        for (int k = 0; k < n; ++k) col[r + k] = cand[a + k];
    }
}

// position of column c in row r (present by construction)
__device__ __forceinline__ int find_slot(const int *row_ptr, const int *col, int r, int c)
{
    int lo = row_ptr[r], hi = row_ptr[r + 1] - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (col[mid] < c) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__global__ void k_pat_slots(const int4 *tris, int nt, const int4 *hinges, int nh, int np, const int *row_ptr,
                            const int *col, int *tri_slot, int *hinge_slot, int *diag_slot)
{
    const long long total = (long long)np + nt + nh;
    PAMO_GRID_STRIDE(k, total)
    {
        if (k < np) {
            diag_slot[k] = find_slot(row_ptr, col, (int)k, (int)k);
        } else if (k < (long long)np + nt) {
            const long long t = k - np;
            const int4 f = tris[t];
            const int v[3] = {f.x, f.y, f.z};
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) tri_slot[9 * t + 3 * a + b] = find_slot(row_ptr, col, v[a], v[b]);
        } else {
            const long long h = k - np - nt;
            const int4 f = hinges[h];
            const int v[4] = {f.x, f.y, f.z, f.w};
            for (int a = 0; a < 4; ++a)
                for (int b = 0; b < 4; ++b) hinge_slot[16 * h + 4 * a + b] = find_slot(row_ptr, col, v[a], v[b]);
        }
    }
}

// the vertex term w I on the diagonal blocks (kval zeroed before)
__global__ void k_diag_term(const float *wk, const int *diag_slot, int np, float4 *kval)
{
    PAMO_GRID_STRIDE(i, np)
    {
        const float w = wk[i];
        const size_t s = 3 * (size_t)diag_slot[i];
        kval[s] = make_float4(w, 0.f, 0.f, 0.f);
        kval[s + 1] = make_float4(0.f, w, 0.f, 0.f);
        kval[s + 2] = make_float4(0.f, 0.f, w, 0.f);
    }
}

// -------------------------------------------------------------------- CG

__global__ void __launch_bounds__(kThreads) k_cg_init(const float4 *grad, const float4 *diag, int np, float4 *p,
                                                      float4 *r, float4 *z, float4 *v, double *partials, int *ticket,
                                                      double *dscal)
{
    double acc = 0.0;
    PAMO_GRID_STRIDE(i, np)
    {
        F3 g = ld(grad, (int)i), d = ld(diag, (int)i);
        F3 zz = mk(g.x / (d.x + 1e-6f), g.y / (d.y + 1e-6f), g.z / (d.z + 1e-6f));
        p[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        st(r, (int)i, g);
        st(z, (int)i, zz);
        st(v, (int)i, zz);
        acc += (double)dot(zz, g);
    }
    double s = block_sum<kThreads>(acc);
    last_block_sum(s, partials, ticket, dscal + D_ZR);
}

// v^T A v, then zr_last = zr
__global__ void __launch_bounds__(kThreads) k_cg_dot(const float4 *a, const float4 *b, int np, double *partials,
                                                     int *ticket, double *dscal)
{
    double acc = 0.0;
    PAMO_GRID_STRIDE(i, np) acc += (double)dot(ld(a, (int)i), ld(b, (int)i));
    double s = block_sum<kThreads>(acc);
    if (last_block_sum(s, partials, ticket, dscal + D_VAV) && threadIdx.x == 0) dscal[D_ZR_LAST] = dscal[D_ZR];
}

// start of a CG iteration: v = z + beta v (not in the first)
__global__ void k_cg_pre(const float4 *z, const double *dscal, int np, int first, float4 *v)
{
    if (first) return;
    const float beta = (float)(dscal[D_ZR] / dscal[D_ZR_LAST]);
    PAMO_GRID_STRIDE(i, np) st(v, (int)i, ld(z, (int)i) + beta * ld(v, (int)i));
}

// p += alpha v, r -= alpha Av (if v^T A v > 1e-16); z = r / diag; partial z.r
__global__ void __launch_bounds__(kThreads) k_cg_update(const float4 *v, const float4 *Av, const float4 *diag,
                                                        double *dscal, int np, float4 *p, float4 *r, float4 *z,
                                                        double *partials, int *ticket)
{
    const double vav = dscal[D_VAV];
    const bool upd = vav > 1e-16;
    const float alpha = upd ? (float)(dscal[D_ZR_LAST] / vav) : 0.f;
    double acc = 0.0;
    PAMO_GRID_STRIDE(i, np)
    {
        F3 rr = ld(r, (int)i);
        if (upd) {
            st(p, (int)i, ld(p, (int)i) + alpha * ld(v, (int)i));
            rr = rr - alpha * ld(Av, (int)i);
            st(r, (int)i, rr);
        }
        F3 d = ld(diag, (int)i);
        F3 zz = mk(rr.x / d.x, rr.y / d.y, rr.z / d.z);
        st(z, (int)i, zz);
        acc += (double)dot(zz, rr);
    }
    double s = block_sum<kThreads>(acc);
    last_block_sum(s, partials, ticket, dscal + D_ZR);
}

// The whole Jacobi-PCG solve of a Newton iteration (the 40 iterations of
// cg_solver.py:96-158) in one cooperative launch, one block per SM and one
// grid-wide sum per iteration.  The reference's iteration
//     Av = A v; alpha = (z.r) / (v.Av); p += alpha v; r -= alpha Av;
//     z = r / diag; v = z + ((z.r)_new / (z.r)) v
// needs v.Av before the update and z.r after it: two sums.  Here (the
// single-reduction form of Chronopoulos and Gear, 1989) A v is carried by the
// recurrence A v_i = A z_i + beta A v_{i-1}, and v.Av by the identity
//     v_i.Av_i = z_i.(A z_i) + 2 beta z_i.(A v_{i-1}) + beta^2 v_{i-1}.(A v_{i-1}),
// which holds for any symmetric A whatever the preconditioner, so the first
// iteration's diag + 1e-6 is kept as the reference has it; the guard
// v.Av > 1e-16 and the update order are the reference's.  An iteration is one
// pass: every vertex keeps a record of three float4 per iteration parity --
// z_i (= r_i / diag), the rows of A z_i / diag and A v_{i-1} / diag -- so a
// row gathers one record per column, forms z_{i+1} there
//     z_{i+1} = z_i - alpha (A z_i / diag + beta A v_{i-1} / diag),
// and computes its row of A z_{i+1}; the contact blocks add their rank-one
// terms (scaled by 1 / diag) into a separate buffer (three copies: read,
// accumulated, zeroed for the one after); the three dot products of the next
// iteration, z.r = sum diag z^2, z.(A z) and z.(A v_i), go into one sum.  The
// time of an iteration is the length of its chains of dependent memory
// accesses, so what stays fixed during the solve is read once: each lane keeps
// the columns of its first row slots in registers.
//
// A sum: every block writes its partials into its own slot of the sum's set
// (three sets, used in turn; a slot's first word holds an all-ones pattern
// until written: a negative NaN that no sum produces, since sums and products
// give the positive canonical NaN; the other words are written before the
// first, which is stored with release semantics), then waits for all slots of
// the set with acquire loads, one thread per slot, and adds them in block
// order -- the same order in every block, so every block gets the same totals,
// independent of scheduling, with one hop between the blocks.  A block's
// writes before its partials are visible to every block after the sum.  Once
// a block has seen all partials of sum k, every block has finished reading sum
// k - 1, so it resets its own slot of that set, which sum k + 2 reuses (the
// reset precedes its release of sum k + 1, which every reader of sum k + 2 has
// acquired).  Slots sit one 128-byte line apart.  Waits spin with a limit; on
// timeout the error is recorded and the kernel returns.  The line search uses
// the same sums for its barrier and energy.
constexpr int kCgThreads = 512;
constexpr int kRec = 3;  // float4 per vertex record of the solve
constexpr unsigned long long kSumPending = ~0ull;
constexpr int kSlotStride = 16;  // u64 words per slot
constexpr int kSlotSets = 3;


__device__ __forceinline__ void st_release(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void st_relaxed(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// waits until *p holds a value; false after the spin limit (error recorded)
__device__ __forceinline__ bool wait_value(const unsigned long long *p, unsigned long long &v, int *iscal,
                                           long long spin_limit)
{
    v = ld_acquire(p);
    for (long long spins = 0; v == kSumPending; ++spins) {
        if (spins > spin_limit) {  // a block never arrived
            atomicExch(iscal + I_BAR_ERR, 1);
            return false;
        }
        __nanosleep(32);
        v = ld_acquire(p);
    }
    return true;
}

// Block sum of `acc`, then the grid-wide total (see above) through the slot
// sets at `slots` (gridDim.x <= BLOCK).  Returns false on a wait timeout.
template <int BLOCK>
__device__ __forceinline__ bool grid_sum_slots(double acc, unsigned long long *slots, int *iscal, long long spin_limit,
                                               int absent_block, int k, double &total)
{
    __shared__ double s_val;
    __shared__ double s_part[BLOCK];  // every block's partial, in block order
    const int G = (int)gridDim.x;
    const size_t set_words = (size_t)G * kSlotStride;
    unsigned long long *set = slots + (size_t)(k % kSlotSets) * set_words;
    unsigned long long *prev = slots + (size_t)((k + kSlotSets - 1) % kSlotSets) * set_words;
    const double bs = block_sum<BLOCK>(acc);
    if (threadIdx.x == 0 && (int)blockIdx.x != absent_block)
        st_release(set + (size_t)blockIdx.x * kSlotStride, (unsigned long long)__double_as_longlong(bs));
    int ok = 1;
    if ((int)threadIdx.x < G) {
        unsigned long long bits = 0;
        if (wait_value(set + (size_t)threadIdx.x * kSlotStride, bits, iscal, spin_limit))
            s_part[threadIdx.x] = __longlong_as_double((long long)bits);
        else
            ok = 0;
    }
    ok = __syncthreads_and(ok);
    if (threadIdx.x < 32) {
        double v = 0.0;
        for (int i = threadIdx.x; i < G; i += 32) v += s_part[i];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) {
            s_val = v;
            if (ok) st_relaxed(prev + (size_t)blockIdx.x * kSlotStride, kSumPending);
        }
    }
    __syncthreads();
    total = s_val;
    return ok != 0;
}

struct CGArgs {
    OpArgs op;
    const float4 *grad, *diag;
    float4 *x, *v;
    float4 *rec0, *rec1;      // the records of even and odd iterations, 3 float4 per vertex
    float4 *wc0, *wc1, *wc2;  // contact part of A z / diag, three copies, zero before the solve
    unsigned long long *slots;  // kSlotSets x gridDim slots, kSlotStride apart (all ones before the solve)
    int *iscal;
    int np, n_iters;
    long long spin_limit;  // polls per wait before it gives up
    int absent_block;      // >= 0: that block never publishes its partials (the wait-timeout test); else -1
};

struct D3s {
    double a, b, c;
};

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// three block sums, then the grid-wide totals: a slot's words 1 and 2 are
// written first, word 0 last with a release store; readers acquire word 0
__device__ __forceinline__ bool grid_sum3(D3s acc, const CGArgs &A, int k, D3s &total)
{
    __shared__ double ws[3][kCgThreads / 32];
    __shared__ double s_part[3][kCgThreads];
    __shared__ D3s s_val;
    const int G = (int)gridDim.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        acc.a += __shfl_down_sync(0xffffffffu, acc.a, o);
        acc.b += __shfl_down_sync(0xffffffffu, acc.b, o);
        acc.c += __shfl_down_sync(0xffffffffu, acc.c, o);
    }
    if (lane == 0) {
        ws[0][wid] = acc.a;
        ws[1][wid] = acc.b;
        ws[2][wid] = acc.c;
    }
    __syncthreads();
    const size_t set_words = (size_t)G * kSlotStride;
    unsigned long long *set = A.slots + (size_t)(k % kSlotSets) * set_words;
    unsigned long long *prev = A.slots + (size_t)((k + kSlotSets - 1) % kSlotSets) * set_words;
    if (wid == 0) {
        double ra = lane < kCgThreads / 32 ? ws[0][lane] : 0.0;
        double rb = lane < kCgThreads / 32 ? ws[1][lane] : 0.0;
        double rc = lane < kCgThreads / 32 ? ws[2][lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            ra += __shfl_down_sync(0xffffffffu, ra, o);
            rb += __shfl_down_sync(0xffffffffu, rb, o);
            rc += __shfl_down_sync(0xffffffffu, rc, o);
        }
        if (lane == 0 && (int)blockIdx.x != A.absent_block) {
            unsigned long long *slot = set + (size_t)blockIdx.x * kSlotStride;
            st_relaxed(slot + 1, (unsigned long long)__double_as_longlong(rb));
            st_relaxed(slot + 2, (unsigned long long)__double_as_longlong(rc));
            st_release(slot, (unsigned long long)__double_as_longlong(ra));
        }
    }
    int ok = 1;
    if ((int)threadIdx.x < G) {
        const unsigned long long *slot = set + (size_t)threadIdx.x * kSlotStride;
        unsigned long long bits = 0;
        if (wait_value(slot, bits, A.iscal, A.spin_limit)) {
            s_part[0][threadIdx.x] = __longlong_as_double((long long)bits);
            s_part[1][threadIdx.x] = __longlong_as_double((long long)ld_relaxed_u64(slot + 1));
            s_part[2][threadIdx.x] = __longlong_as_double((long long)ld_relaxed_u64(slot + 2));
        } else {
            ok = 0;
        }
    }
    ok = __syncthreads_and(ok);
    if (threadIdx.x < 32) {
        double va = 0.0, vb = 0.0, vc = 0.0;
        for (int i = threadIdx.x; i < G; i += 32) {
            va += s_part[0][i];
            vb += s_part[1][i];
            vc += s_part[2][i];
        }
        for (int o = 16; o > 0; o >>= 1) {
            va += __shfl_down_sync(0xffffffffu, va, o);
            vb += __shfl_down_sync(0xffffffffu, vb, o);
            vc += __shfl_down_sync(0xffffffffu, vc, o);
        }
        if (threadIdx.x == 0) {
            s_val = D3s{va, vb, vc};
            if (ok) st_relaxed(prev + (size_t)blockIdx.x * kSlotStride, kSumPending);
        }
    }
    __syncthreads();
    total = s_val;
    return ok != 0;
}

__global__ void __launch_bounds__(kCgThreads, 1) k_cg_solve(CGArgs A)
{
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long gs = (long long)blockDim.x * gridDim.x;
    const int lane = threadIdx.x & 31, sub = lane & 3;
    const long long warp0 = t0 >> 5, nwarps = gs >> 5;
    const OpArgs &O = A.op;
    const long long nb = min((long long)A.iscal[I_NACT], O.cap_b);
    constexpr int kRowBatch = 4;
    const long long i0 = warp0 * 8 + (lane >> 2);
    int s0 = 0, e0 = 0, c0[kRowBatch];
    if (i0 < A.np) {
        s0 = O.row_ptr[i0] + sub;
        e0 = O.row_ptr[i0 + 1];
    }
#pragma unroll
    for (int k = 0; k < kRowBatch; ++k) c0[k] = s0 + 4 * k < e0 ? O.col[s0 + 4 * k] : -1;
    const long long tc = gs - 1 - t0;
    const float4 *diag = A.diag;

    // rows of K z (z(k) at column k) into the owner's record, scaled by 1 / diag;
    // contact terms (scaled by 1 / diag at each vertex) into wcout; returns this
    // thread's share of z . (K z + contacts)
    auto pass = [&](auto zn, auto own, float4 *recout, float4 *wcout, bool spmv) -> double {
        double zw = 0.0;
        for (long long base = warp0 * 8, g = 0; base < A.np; base += nwarps * 8, ++g) {
            const long long i = base + (lane >> 2);
            F3 zi = mk(0.f, 0.f, 0.f);
            if (i < A.np && sub == 0) zi = own((int)i);
            if (!spmv) continue;
            int s = s0, e = e0, cidx[kRowBatch];
            if (g == 0) {
#pragma unroll
                for (int k = 0; k < kRowBatch; ++k) cidx[k] = c0[k];
            } else {
                s = 0;
                e = 0;
                if (i < A.np) {
                    s = O.row_ptr[i] + sub;
                    e = O.row_ptr[i + 1];
                }
#pragma unroll
                for (int k = 0; k < kRowBatch; ++k) cidx[k] = s + 4 * k < e ? O.col[s + 4 * k] : -1;
            }
            F3 xz[kRowBatch];
#pragma unroll
            for (int k = 0; k < kRowBatch; ++k) xz[k] = cidx[k] >= 0 ? zn(cidx[k]) : mk(0.f, 0.f, 0.f);
            F3 kv = mk(0.f, 0.f, 0.f);
#pragma unroll
            for (int k = 0; k < kRowBatch; ++k) {
                if (cidx[k] < 0) continue;
                const size_t b = 3 * (size_t)(s + 4 * k);
                const float4 k0 = O.kval[b], k1 = O.kval[b + 1], k2 = O.kval[b + 2];
                kv = kv + mk(k0.x * xz[k].x + k0.y * xz[k].y + k0.z * xz[k].z,
                             k1.x * xz[k].x + k1.y * xz[k].y + k1.z * xz[k].z,
                             k2.x * xz[k].x + k2.y * xz[k].y + k2.z * xz[k].z);
            }
            for (int ss = s + 4 * kRowBatch; ss < e; ss += 4) {
                const F3 xx = zn(O.col[ss]);
                const float4 k0 = O.kval[3 * (size_t)ss], k1 = O.kval[3 * (size_t)ss + 1],
                             k2 = O.kval[3 * (size_t)ss + 2];
                kv = kv + mk(k0.x * xx.x + k0.y * xx.y + k0.z * xx.z, k1.x * xx.x + k1.y * xx.y + k1.z * xx.z,
                             k2.x * xx.x + k2.y * xx.y + k2.z * xx.z);
            }
#pragma unroll
            for (int o = 1; o < 4; o <<= 1) {
                kv.x += __shfl_xor_sync(0xffffffffu, kv.x, o);
                kv.y += __shfl_xor_sync(0xffffffffu, kv.y, o);
                kv.z += __shfl_xor_sync(0xffffffffu, kv.z, o);
            }
            if (i < A.np && sub == 0) {
                const F3 d = ld(diag, (int)i);
                st(recout + kRec * (size_t)i + 1, 0, mk(kv.x / d.x, kv.y / d.y, kv.z / d.z));
                zw += (double)dot(zi, kv);
            }
        }
        if (!spmv) return zw;
        for (long long k = tc; k < nb; k += gs) {
            const int b = O.bact[k];
            const float c = O.bb2[b];
            if (c == 0.f) continue;
            const int4 i4 = O.bidx[b];
            const int idx[4] = {i4.x, i4.y, i4.z, i4.w};
            F3 g[4];
            float sdx = 0.f;
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                g[a] = f3(O.bg[4 * (size_t)b + a]);
                sdx += dot(g[a], zn(idx[a]));
            }
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const F3 d = ld(diag, idx[a]);
                const F3 t = (c * sdx) * g[a];
                atomic_add3(wcout, idx[a], mk(t.x / d.x, t.y / d.y, t.z / d.z));
            }
            zw += (double)(c * sdx) * (double)sdx;
        }
        return zw;
    };

    // pass 0: x = 0; record 0 = (g / diag, rows of K z_0 / diag, 0) with
    // z_0 = g / (diag + 1e-6)
    D3s acc{0.0, 0.0, 0.0};
    {
        auto z0 = [&](int k) -> F3 {
            const F3 g = ld(A.grad, k), d = ld(diag, k);
            return mk(g.x / (d.x + 1e-6f), g.y / (d.y + 1e-6f), g.z / (d.z + 1e-6f));
        };
        auto own0 = [&](int j) -> F3 {
            const F3 g = ld(A.grad, j), d = ld(diag, j);
            A.x[j] = make_float4(0.f, 0.f, 0.f, 0.f);
            st(A.rec0 + kRec * (size_t)j, 0, mk(g.x / d.x, g.y / d.y, g.z / d.z));
            st(A.rec0 + kRec * (size_t)j + 2, 0, mk(0.f, 0.f, 0.f));
            const F3 z = z0(j);
            acc.a += (double)dot(z, g);
            return z;
        };
        acc.b = pass(z0, own0, A.rec0, A.wc0, true);
    }
    D3s sums;
    int nsum = 0;
    if (!grid_sum3(acc, A, nsum++, sums)) return;
    double gam = sums.a, del = sums.b, eps = 0.0, gam_prev = 0.0, vav = 0.0;
    for (int it = 0; it < A.n_iters; ++it) {
        float beta = 0.f;
        if (it == 0) {
            vav = del;
        } else {
            beta = (float)(gam / gam_prev);
            const double bd = (double)beta;
            vav = del + 2.0 * bd * eps + bd * bd * vav;
        }
        const bool upd = vav > 1e-16;
        const float alpha = upd ? (float)(gam / vav) : 0.f;
        const bool odd = it & 1;
        const float4 *rc = odd ? A.rec1 : A.rec0;
        float4 *rn = odd ? A.rec0 : A.rec1;
        const int m3 = it % 3;
        const float4 *wcc = m3 == 0 ? A.wc0 : m3 == 1 ? A.wc1 : A.wc2;
        float4 *wcn = m3 == 0 ? A.wc1 : m3 == 1 ? A.wc2 : A.wc0;
        float4 *wcz = m3 == 0 ? A.wc2 : m3 == 1 ? A.wc0 : A.wc1;
        const bool last = it == A.n_iters - 1;
        const bool contacts = nb > 0;
        // A v_i / diag and z_{i+1} at vertex k from its record
        auto avs = [&](const float4 *R, int k) -> F3 {
            F3 w = f3(R[1]);
            if (contacts) w = w + ld(wcc, k);
            return it == 0 ? w : w + beta * f3(R[2]);
        };
        auto zn = [&](int k) -> F3 {
            const float4 *R = rc + kRec * (size_t)k;
            const F3 r = f3(R[0]);
            return upd ? r - alpha * avs(R, k) : r;
        };
        acc = D3s{0.0, 0.0, 0.0};
        auto own = [&](int j) -> F3 {
            const float4 *R = rc + kRec * (size_t)j;
            const F3 d = ld(diag, j);
            F3 zc;
            if (it == 0) {
                const F3 g = ld(A.grad, j);
                zc = mk(g.x / (d.x + 1e-6f), g.y / (d.y + 1e-6f), g.z / (d.z + 1e-6f));
            } else {
                zc = f3(R[0]);
            }
            const F3 vj = it == 0 ? zc : zc + beta * ld(A.v, j);
            const F3 av = avs(R, j);
            const F3 r0 = f3(R[0]);
            const F3 z = upd ? r0 - alpha * av : r0;
            if (upd) st(A.x, j, ld(A.x, j) + alpha * vj);
            if (!last) {
                st(A.v, j, vj);
                st(rn + kRec * (size_t)j, 0, z);
                st(rn + kRec * (size_t)j + 2, 0, av);
                if (contacts) wcz[j] = make_float4(0.f, 0.f, 0.f, 0.f);
                acc.a += (double)(d.x * z.x * z.x + d.y * z.y * z.y + d.z * z.z * z.z);
                acc.c += (double)(z.x * av.x * d.x + z.y * av.y * d.y + z.z * av.z * d.z);
            }
            return z;
        };
        acc.b = pass(zn, own, rn, wcn, !last);
        if (last) break;
        if (!grid_sum3(acc, A, nsum++, sums)) return;
        gam_prev = gam;
        gam = sums.a;
        del = sums.b;
        eps = sums.c;
    }
}

// ---------------------------------------------------------- clamp, CCD, line search
// largest |p_i| (float bits of a non-negative value order like ints; out zeroed before)
__global__ void k_max_norm(const float4 *p, int np, float *out)
{
    float m = 0.f;
    PAMO_GRID_STRIDE(i, np) m = fmaxf(m, len(ld(p, (int)i)));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(reinterpret_cast<int *>(out), __float_as_int(m));
}

__global__ void k_clamp(float4 *p, const float4 *q_prev, const float4 *q_det, int np, float radius)
{
    PAMO_GRID_STRIDE(i, np)
    {
        F3 pi = ld(p, (int)i), qn = ld(q_prev, (int)i), qd = ld(q_det, (int)i);
        F3 dq = qn + pi - qd;
        float l = len(dq);
        if (l > radius) st(p, (int)i, radius * ((1.f / l) * dq) + qd - qn);
    }
}

// Additive CCD (Li et al. 2021) per block, in FP64 (ccd_kernels.py:8-110).
__global__ void __launch_bounds__(128) k_accd(const float4 *q, const float4 *pv, const int4 *bidx, const int *bkind,
                                              const int *iscal, long long cap_b, float slack, float thick, int max_iters,
                                              float ee_thres, float *ccd_step)
{
    const long long nb = min((long long)iscal[I_NB], cap_b);
    PAMO_GRID_STRIDE(b, nb)
    {
        int4 i = bidx[b];
        int kind = bkind[b];
        int idx[4] = {i.x, i.y, i.z, i.w};
        D3 x[4], v[4];
        for (int a = 0; a < 4; ++a) {
            x[a] = d3(q[idx[a]]);
            v[a] = d3(pv[idx[a]]);
        }
        D3 avg = 0.25 * (v[0] + v[1] + v[2] + v[3]);
        for (int a = 0; a < 4; ++a) v[a] = v[a] - avg;
        double lv;
        if (kind == KIND_PT) lv = len(v[0]) + fmax(len(v[1]), fmax(len(v[2]), len(v[3])));
        else lv = fmax(len(v[0]), len(v[1])) + fmax(len(v[2]), len(v[3]));
        if (lv < 1e-12) continue;
        const double th = thick;
        // Every distance type is the distance between the two primitives or
        // between features of them found by the Voronoi regions, so it is at
        // least the distance between their boxes.  When that bound already
        // gives a first step beyond 1 (the skip below), so does the exact
        // distance, and the classification is not needed; the 1e-9 margins
        // cover the rounding of both evaluations.
        if (max_iters > 0) {
            const int na = kind == KIND_PT ? 1 : 2;  // primitive A: x[0 .. na), primitive B: x[na .. 4)
            double bb = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                auto c = [&](int a) { return k == 0 ? x[a].x : k == 1 ? x[a].y : x[a].z; };
                double alo = c(0), ahi = c(0), blo = c(3), bhi = c(3);
                for (int a = 1; a < na; ++a) {
                    alo = fmin(alo, c(a));
                    ahi = fmax(ahi, c(a));
                }
                for (int a = na; a < 3; ++a) {
                    blo = fmin(blo, c(a));
                    bhi = fmax(bhi, c(a));
                }
                const double gapk = fmax(fmax(blo - ahi, alo - bhi), 0.0);
                bb += gapk * gapk;
            }
            const double lb = sqrt(bb) * (1.0 - 1e-9);
            const double dmt_lb = fmax((lb * lb - th * th) / (lb + th), 0.0);
            if (slack * dmt_lb / lv > 1.0 + 1e-9) continue;
        }
        int ty = classify(kind, x, (double)ee_thres);
        double d = classified_distance(kind, ty, x);
        double dmt = fmax((d * d - th * th) / (sqrt(d * d) + th), 0.0);
        const double gap = (1.0 - slack) * dmt;
        double t = 0.0, tl = slack * dmt / lv;
        // The first pass never records (it > 0 is needed, or max_iters == 0) and
        // leaves with t = tl when tl > 1, so its distance evaluation is skipped.
        if (max_iters > 0 && tl > 1.0) continue;
        for (int it = 0;; ++it) {
            for (int a = 0; a < 4; ++a) x[a] = x[a] + tl * v[a];
            ty = classify(kind, x, (double)ee_thres);
            d = classified_distance(kind, ty, x);
            dmt = fmax((d * d - th * th) / (sqrt(d * d) + th), 0.0);
            if ((it > 0 && dmt <= gap) || it >= max_iters) {
                float tf = (float)t;  // non-negative: integer order equals float order
                atomicMin(reinterpret_cast<int *>(ccd_step), __float_as_int(tf));
                break;
            }
            t = t + tl;
            if (t > 1.0) break;
            tl = 0.8 * dmt / lv;
        }
    }
}

__global__ void k_line_search(const float4 *q_prev, const float4 *p, const float *ccd_step, int n_halves,
                              const double *dscal, int np, float4 *q, int *iscal)
{
    if (n_halves > 0 && dscal[D_ENERGY] < dscal[D_ENERGY_PREV]) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) iscal[I_LS] = n_halves;  // the last trial taken
    const float a = ccd_step[0] * ldexpf(1.f, -n_halves);
    PAMO_GRID_STRIDE(i, np) st(q, (int)i, ld(q_prev, (int)i) + a * ld(p, (int)i));
}

__global__ void k_copy_energy_prev(double *dscal) { dscal[D_ENERGY_PREV] = dscal[D_ENERGY]; }

// The whole line search (system.py:393-409) in one cooperative launch, one
// block per SM: trial nh moves every vertex to q_prev + step 2^-nh p, a
// grid-wide barrier makes the positions visible, and the trial's energy is one
// grid-wide sum; the loop stops at the first trial after the first whose energy
// is below the start's, as the reference's loop does -- so an accepted first
// trial costs two sums and no further launches.  The sums and the barrier are
// the persistent CG's one-hop slot sums (their own slot sets), with the same
// bounded waits: on a timeout the error is recorded and the kernel returns.
constexpr int kLsThreads = 512;

struct LSArgs {
    EArgs e;  // n_halves is set per trial; e.q is the iterate written here
    float4 *q;
    const float4 *q_prev, *p;
    const float *ccd_step;
    int n_trials;
    unsigned long long *slots;  // kSlotSets x gridDim slots, all ones before the launch
    long long spin_limit;
};

__global__ void __launch_bounds__(kLsThreads, 1) k_line_search_all(LSArgs L)
{
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long gs = (long long)blockDim.x * gridDim.x;
    EArgs A = L.e;
    const double e0 = A.dscal[D_ENERGY];  // the energy at the iterate
    double e = e0;
    int nsum = 0, last = -1;
    for (int nh = 0; nh < L.n_trials; ++nh) {
        if (nh > 0 && e < e0) break;
        const float a = L.ccd_step[0] * ldexpf(1.f, -nh);
        for (long long i = t0; i < A.np; i += gs) st(L.q, (int)i, ld(L.q_prev, (int)i) + a * ld(L.p, (int)i));
        double unused;
        if (!grid_sum_slots<kLsThreads>(0.0, L.slots, A.iscal, L.spin_limit, -1, nsum++, unused)) return;
        A.n_halves = nh;
        if (!grid_sum_slots<kLsThreads>(energy_terms(A, t0, gs), L.slots, A.iscal, L.spin_limit, -1, nsum++, e))
            return;
        last = nh;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        A.dscal[D_ENERGY_PREV] = e0;
        A.dscal[D_ENERGY] = e;
        A.iscal[I_LS] = last;
    }
}

// One row of the Newton trace per iteration: energy at the iterate, energy
// after the line search, CCD step, index of the last halving tried, contact
// blocks, blocks within d_hat.
__global__ void k_trace(const double *dscal, const float *fscal, int *iscal, double *trace, long long cap)
{
    const int i = iscal[I_TRACE];
    if (i < cap) {
        double *r = trace + 6LL * i;
        r[0] = dscal[D_ENERGY_PREV];
        r[1] = dscal[D_ENERGY];
        r[2] = fscal[0];
        r[3] = iscal[I_LS];
        r[4] = iscal[I_NB];
        r[5] = iscal[I_NACT];
    }
    iscal[I_TRACE] = i + 1;
}

// 3x3 blocks given as 9 row-major floats -> the solve's three float4 rows
__global__ void k_blocks9_to_rows(const float *b9, long long nb, float4 *kval)
{
    PAMO_GRID_STRIDE(k, nb)
    {
        const float *b = b9 + 9 * k;
        kval[3 * k] = make_float4(b[0], b[1], b[2], 0.f);
        kval[3 * k + 1] = make_float4(b[3], b[4], b[5], 0.f);
        kval[3 * k + 2] = make_float4(b[6], b[7], b[8], 0.f);
    }
}

__global__ void k_set_float(float *f, float v) { *f = v; }

__global__ void k_scale(float *a, int n, float s)
{
    PAMO_GRID_STRIDE(i, n) a[i] *= s;
}

__global__ void k_validate_idx(const int *a, long long count, int hi, int *bad)
{
    int local = 0;
    PAMO_GRID_STRIDE(i, count) local += (a[i] < 0 || a[i] >= hi);
    if (local) atomicAdd(bad, local);
}

__global__ void k_f4_to_aos(const float4 *in, float *out, int n)
{
    PAMO_GRID_STRIDE(i, n)
    {
        float4 v = in[i];
        out[3 * i] = v.x;
        out[3 * i + 1] = v.y;
        out[3 * i + 2] = v.z;
    }
}

}  // namespace

// ------------------------------------------------------------------ host side
#define S3_TRY(expr)                                      \
    do {                                                  \
        cudaError_t _e = (expr);                          \
        if (_e != cudaSuccess) return map_cuda_error(_e); \
    } while (0)

void Stage3::release()
{
    gt_ready = false;
    void *ptrs[] = {q, q_prev, q_det, p, grad, diag, target, r, z, v, v2, Av, Avc, cg_rec, q_gather, wk, tris, area, inv_dm,
                    edges4, hinges, rest_angle, rest_elen, row_ptr, col, kval, tri_slot, hinge_slot, diag_slot, hblk, pat_cnt,
                    pat_cur, pat_off, pat_cand, pat_scan, bidx, bkind, bsub, bd, bb2, bg, bact, gt_pts, gt_tris, dscal, fscal,
                    iscal, partials, trace};
    drop_graph();
    if (cand_pt) cudaFree(cand_pt);
    if (cand_ee) cudaFree(cand_ee);
    cand_pt = cand_ee = nullptr;
    cap_c = 0;
    if (work) cudaStreamDestroy(work);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    work = nullptr;
    ev_in = ev_out = nullptr;
    for (int b = 0; b < 2; ++b) {
        if (side[b]) cudaStreamDestroy(side[b]);
        if (ev_join[b]) cudaEventDestroy(ev_join[b]);
        side[b] = nullptr;
        ev_join[b] = nullptr;
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    ev_fork = nullptr;
    for (void *x : ptrs)
        if (x) cudaFree(x);
    if (h_iscal) cudaFreeHost(h_iscal);
    if (h_dscal) cudaFreeHost(h_dscal);
    q = q_prev = q_det = p = grad = diag = target = r = z = v = v2 = Av = Avc = cg_rec = q_gather = nullptr;
    row_ptr = col = tri_slot = hinge_slot = diag_slot = nullptr;
    hblk = nullptr;
    pat_cnt = pat_cur = pat_off = pat_cand = pat_scan = nullptr;
    kval = nullptr;
    nnz = cap_nnz = cap_cand = 0;
    gathered = false;
    wk = nullptr; tris = nullptr; area = nullptr; inv_dm = nullptr; edges4 = nullptr; hinges = nullptr;
    rest_angle = rest_elen = nullptr; bidx = nullptr; bkind = bsub = nullptr; bd = bb2 = nullptr;
    bg = nullptr; bact = nullptr; gt_pts = nullptr; gt_tris = nullptr; dscal = nullptr; fscal = nullptr; iscal = nullptr;
    partials = nullptr; h_iscal = nullptr; h_dscal = nullptr;
    trace = nullptr;
    cap_trace = 0;
    tri_bvh.release();
    edge_bvh.release();
    gt_bvh.release();
    cap_p = cap_t = cap_e = cap_h = cap_b = cap_gp = cap_gt = 0;
}

int Stage3::ensure(long long np_, long long nt_, long long ne_, long long nh_, long long ngp_, long long ngt_)
{
    if (np_ <= cap_p && nt_ <= cap_t && ne_ <= cap_e && nh_ <= cap_h && ngp_ <= cap_gp && ngt_ <= cap_gt && dscal)
        return PAMO_OK;
    long long cp = np_ > cap_p ? np_ : cap_p, ct = nt_ > cap_t ? nt_ : cap_t;
    long long ce = ne_ > cap_e ? ne_ : cap_e, ch = nh_ > cap_h ? nh_ : cap_h;
    long long cgp = ngp_ > cap_gp ? ngp_ : cap_gp, cgt = ngt_ > cap_gt ? ngt_ : cap_gt;
    long long cb = cap_b;
    release();
    cp += 1; ct += 1; ce += 1; ch += 1; cgp += 1; cgt += 1;
#define A3(ptr, bytes)                                                   \
    do {                                                                 \
        if (cudaMalloc((void **)&ptr, (size_t)(bytes)) != cudaSuccess) { \
            release();                                                   \
            return PAMO_ERR_OOM;                                         \
        }                                                                \
    } while (0)
    A3(q, cp * 16); A3(q_prev, cp * 16); A3(q_det, cp * 16); A3(p, cp * 16); A3(grad, cp * 16);
    A3(diag, cp * 16); A3(target, cp * 16); A3(r, cp * 16); A3(z, cp * 16); A3(v, cp * 16); A3(v2, cp * 16); A3(Av, cp * 16); A3(Avc, cp * 16);
    A3(cg_rec, cp * 16 * 2 * kRec);
    A3(q_gather, cp * 16);
    A3(wk, cp * 4);
    A3(tris, ct * 16); A3(area, ct * 4); A3(inv_dm, ct * 16); A3(tri_slot, ct * 36);
    A3(edges4, ce * 16);
    A3(hinges, ch * 16); A3(rest_angle, ch * 4); A3(rest_elen, ch * 4); A3(hinge_slot, ch * 64); A3(hblk, ch * 81 * 4);
    A3(row_ptr, (cp + 1) * 4); A3(diag_slot, cp * 4); A3(pat_cnt, (cp + 1) * 4); A3(pat_cur, cp * 4);
    A3(pat_off, (cp + 1) * 4); A3(pat_scan, scan_scratch_ints(cp + 1) * 4);
    if (scan_scratch_init(pat_scan, scan_scratch_ints(cp + 1)) != cudaSuccess) {
        release();
        return PAMO_ERR_OOM;
    }
    A3(gt_pts, cgp * 16); A3(gt_tris, cgt * 16);
    A3(dscal, 64); A3(fscal, 64); A3(iscal, 64);
    A3(partials, (size_t)kSlotSets * kRedBlocks * kSlotStride * 8);  // reduction partials; the persistent solve's slots
#undef A3
    if (cudaMallocHost((void **)&h_iscal, 64) != cudaSuccess || cudaMallocHost((void **)&h_dscal, 64) != cudaSuccess) {
        release();
        return PAMO_ERR_OOM;
    }
    cap_p = cp; cap_t = ct; cap_e = ce; cap_h = ch; cap_gp = cgp; cap_gt = cgt;
    if (tri_bvh.ensure(ct) != cudaSuccess || edge_bvh.ensure(ce) != cudaSuccess || gt_bvh.ensure(cgt) != cudaSuccess) {
        release();
        return PAMO_ERR_OOM;
    }
    return ensure_blocks(cb > 0 ? cb : 8 * cp + 1024);
}

int Stage3::ensure_cands(long long n)
{
    if (n <= cap_c && cand_pt) return PAMO_OK;
    if (cand_pt) cudaFree(cand_pt);
    if (cand_ee) cudaFree(cand_ee);
    cand_pt = cand_ee = nullptr;
    cap_c = 0;
    if (cudaMalloc((void **)&cand_pt, n * sizeof(int2)) != cudaSuccess ||
        cudaMalloc((void **)&cand_ee, n * sizeof(int2)) != cudaSuccess)
        return PAMO_ERR_OOM;
    cap_c = n;
    return PAMO_OK;
}

int Stage3::ensure_blocks(long long nb)
{
    if (nb <= cap_b && bidx) return PAMO_OK;
    void *ptrs[] = {bidx, bkind, bsub, bd, bb2, bg, bact};
    for (void *x : ptrs)
        if (x) cudaFree(x);
    bidx = nullptr; bkind = bsub = nullptr; bd = bb2 = nullptr; bg = nullptr; bact = nullptr;
    cap_b = 0;
    if (cudaMalloc((void **)&bidx, nb * 16) != cudaSuccess || cudaMalloc((void **)&bkind, nb * 4) != cudaSuccess ||
        cudaMalloc((void **)&bsub, nb * 4) != cudaSuccess || cudaMalloc((void **)&bd, nb * 4) != cudaSuccess ||
        cudaMalloc((void **)&bb2, nb * 4) != cudaSuccess || cudaMalloc((void **)&bg, nb * 64) != cudaSuccess ||
        cudaMalloc((void **)&bact, nb * 4) != cudaSuccess)
        return PAMO_ERR_OOM;
    cap_b = nb;
    return PAMO_OK;
}

int Stage3::register_mesh(const float *d_gt_v, const int *d_gt_f, int n_gt_v, int n_gt_f, const float *d_v,
                          const int *d_f, int n_v, int n_f, const int *d_e, int n_e, const int *d_h, int n_h,
                          const float *d_vor, cudaStream_t s)
{
    const int prev_gp = ngp, prev_gt = ngt;
    int rc = ensure(n_v, n_f, n_e, n_h, n_gt_v, n_gt_f);  // a reallocation clears gt_ready
    if (rc) return rc;
    const bool keep_gt = cfg.reuse_gt && gt_ready && d_gt_v == gt_src_v && d_gt_f == gt_src_f && n_gt_v == prev_gp &&
                         n_gt_f == prev_gt;
    graph_stale = true;  // sizes and configuration are baked into the captured iteration
    gathered = false;  // new geometry: contact candidates are gathered again
    np = n_v; nt = n_f; ne = n_e; nh = n_h; ngp = n_gt_v; ngt = n_gt_f;
    radius = cfg.contact_detection_radius;
    launch(k_aos_to_f4, grid_for(np), kThreads, 0, s, d_v, q, q_prev, np);
    launch(k_aos_to_i4, grid_for(nt), kThreads, 0, s, d_f, tris, nt, 3, 0);
    launch(k_aos_to_i4, grid_for(ne), kThreads, 0, s, d_e, edges4, ne, 2, 1);
    launch(k_aos_to_i4, grid_for(nh), kThreads, 0, s, d_h, hinges, nh, 4, 0);
    if (!keep_gt) {
        launch(k_aos_to_f4, grid_for(ngp), kThreads, 0, s, d_gt_v, gt_pts, nullptr, ngp);
        launch(k_aos_to_i4, grid_for(ngt), kThreads, 0, s, d_gt_f, gt_tris, ngt, 3, 0);
    }
    // Voronoi areas x GT-distance stiffness
    S3_TRY(cudaMemcpyAsync(wk, d_vor, (size_t)np * 4, cudaMemcpyDeviceToDevice, s));
    launch(k_scale, grid_for(np), kThreads, 0, s, wk, np, cfg.mesh2gt_dist_stiffness);
    launch(k_elastic_pre, grid_for(nt), kThreads, 0, s, q, tris, nt, area, inv_dm);
    launch(k_hinge_pre, grid_for(nh), kThreads, 0, s, q, hinges, nh, rest_angle, rest_elen);
    if (!keep_gt) {
        gt_ready = false;
        S3_TRY(lbvh_build(gt_bvh, gt_pts, gt_tris, ngt, s));
        S3_TRY(lbvh_refit(gt_bvh, gt_pts, gt_tris, ngt, s));
        gt_src_v = d_gt_v;
        gt_src_f = d_gt_f;
        gt_ready = true;
    }
    S3_TRY(lbvh_build(tri_bvh, q, tris, nt, s));
    S3_TRY(lbvh_build(edge_bvh, q, edges4, ne, s));
    S3_TRY(cudaMemsetAsync(iscal, 0, 64, s));
    S3_TRY(cudaMemsetAsync(dscal, 0, 64, s));
    if ((rc = build_pattern(s))) return rc;
    return cudaGetLastError() == cudaSuccess ? PAMO_OK : PAMO_ERR_DEVICE;
}

int Stage3::build_pattern(cudaStream_t s)
{
    const long long cand_n = (long long)np + 6LL * nt + 12LL * nh;
    if (cand_n > cap_cand || !pat_cand) {
        if (pat_cand) cudaFree(pat_cand);
        pat_cand = nullptr;
        cap_cand = 0;
        if (cudaMalloc((void **)&pat_cand, (size_t)cand_n * 4) != cudaSuccess) return PAMO_ERR_OOM;
        cap_cand = cand_n;
    }
    launch(k_fill_int, grid_for(np), kThreads, 0, s, pat_cnt, (long long)np, 1);  // the diagonal
    S3_TRY(cudaMemsetAsync(pat_cnt + np, 0, 4, s));
    launch(k_pat_count, grid_for((long long)nt + nh), kThreads, 0, s, (const int4 *)tris, nt, (const int4 *)hinges, nh,
           pat_cnt);
    S3_TRY(exclusive_scan(pat_cnt, pat_off, (long long)np + 1, nullptr, pat_scan, nullptr, s));
    S3_TRY(cudaMemsetAsync(pat_cur, 0, (size_t)np * 4, s));
    launch(k_pat_fill, grid_for((long long)np + nt + nh), kThreads, 0, s, (const int4 *)tris, nt, (const int4 *)hinges,
           nh, np, (const int *)pat_off, pat_cur, pat_cand);
    launch(k_pat_sort, grid_for(np), kThreads, 0, s, (const int *)pat_off, np, pat_cand, pat_cnt);
    S3_TRY(exclusive_scan(pat_cnt, row_ptr, (long long)np + 1, nullptr, pat_scan, nullptr, s));
    S3_TRY(cudaMemcpyAsync(h_iscal + 15, row_ptr + np, 4, cudaMemcpyDeviceToHost, s));
    S3_TRY(cudaStreamSynchronize(s));
    nnz = h_iscal[15];
    if (nnz <= 0 || nnz > cand_n) return PAMO_ERR_DEVICE;
    if (nnz > cap_nnz || !kval) {
        if (col) cudaFree(col);
        if (kval) cudaFree(kval);
        col = nullptr;
        kval = nullptr;
        cap_nnz = 0;
        const long long c = nnz + nnz / 8 + 64;
        if (cudaMalloc((void **)&col, (size_t)c * 4) != cudaSuccess ||
            cudaMalloc((void **)&kval, (size_t)c * 48) != cudaSuccess)
            return PAMO_ERR_OOM;
        cap_nnz = c;
    }
    launch(k_pat_emit, grid_for(np), kThreads, 0, s, (const int *)pat_off, (const int *)row_ptr,
           (const int *)pat_cand, np, col);
    launch(k_pat_slots, grid_for((long long)np + nt + nh), kThreads, 0, s, (const int4 *)tris, nt,
           (const int4 *)hinges, nh, np, (const int *)row_ptr, (const int *)col, tri_slot, hinge_slot, diag_slot);
    return cudaGetLastError() == cudaSuccess ? PAMO_OK : PAMO_ERR_DEVICE;
}

int Stage3::detect(cudaStream_t s)
{
    if (!cand_pt) {
        int rc = ensure_cands(32LL * (np + ne) + 4096);
        if (rc) return rc;
    }
    for (int attempt = 0; attempt < 64; ++attempt) {
        const float thr = 2.f * radius + cfg.d_hat;
        const float extra = 0.25f * thr;
        bool gather = !gathered || thr > gather_thr;
        if (gather) {
            // refit the hierarchies built at registration (system.py:121-152) and
            // collect the pairs within thr + extra
            S3_TRY(lbvh_refit(tri_bvh, q, tris, nt, s));
            S3_TRY(lbvh_refit(edge_bvh, q, edges4, ne, s));
            S3_TRY(cudaMemsetAsync(iscal, 0, 6 * sizeof(int), s));
            launch(k_detect_pt, grid_for(np), kThreads, 0, s, q, np, tris, tri_bvh.nodes, tri_bvh.vals, tri_bvh.scene,
                   thr + extra, iscal, cap_c, cand_pt);
            launch(k_detect_ee, grid_for(ne), kThreads, 0, s, q, ne, edges4, edge_bvh.nodes, edge_bvh.vals,
                   edge_bvh.scene, thr + extra, iscal, cap_c, cand_ee);
            S3_TRY(cudaMemcpyAsync(q_gather, q, (size_t)np * 16, cudaMemcpyDeviceToDevice, s));
        } else {
            S3_TRY(cudaMemsetAsync(iscal, 0, 3 * sizeof(int), s));
        }
        S3_TRY(cudaMemsetAsync(iscal + I_DISP, 0, sizeof(int), s));
        launch(k_max_disp, grid_for(np), kThreads, 0, s, q, q_gather, np, iscal);
        launch(k_test_pt, grid_for(cap_c), kThreads, 0, s, q, tris, cand_pt, cap_c, thr, iscal, cap_b, bidx, bkind);
        launch(k_test_ee, grid_for(cap_c), kThreads, 0, s, q, edges4, cand_ee, cap_c, thr, cfg.ee_classify_thres,
               iscal, cap_b, bidx, bkind);
        S3_TRY(cudaMemcpyAsync(h_iscal, iscal, 12 * sizeof(int), cudaMemcpyDeviceToHost, s));
        S3_TRY(cudaStreamSynchronize(s));
        if (prof) prof->collect();
        if (h_iscal[I_BAR_ERR]) return PAMO_ERR_DEVICE;  // a solve's grid barrier timed out
        if (h_iscal[I_STACK] > 0) return PAMO_ERR_CAPACITY;
        const long long nc = h_iscal[I_NCAND_PT] > h_iscal[I_NCAND_EE] ? h_iscal[I_NCAND_PT] : h_iscal[I_NCAND_EE];
        if (nc > cap_c) {  // candidate buffers too small: grow and gather again
            int rc = ensure_cands(nc + nc / 4 + 4096);
            if (rc) return rc;
            gathered = false;
            continue;
        }
        float disp;
        memcpy(&disp, &h_iscal[I_DISP], sizeof(float));
        if (!gather && !(2.f * disp <= gather_thr - thr + extra_at_gather)) {
            gathered = false;  // moved too far since the gathering: gather again
            continue;
        }
        if (gather) {
            gathered = true;
            gather_thr = thr;
            extra_at_gather = extra;
        }
        long long n = h_iscal[I_NB];
        if (n > cfg.max_blocks) {  // the reference halves the radius and retries (energy.py:940-948)
            radius *= 0.5f;
            continue;
        }
        if (n > cap_b) {
            int rc = ensure_blocks(n + n / 4 + 1024);
            if (rc) return rc;
            continue;
        }
        return PAMO_OK;
    }
    return PAMO_ERR_CAPACITY;
}

static EArgs energy_args(Stage3 &S, int n_halves)
{
    return EArgs{S.q, S.target, S.wk, S.np, S.nt, S.nh, S.tris, S.area, S.inv_dm,
                 S.cfg.elas_young_modulus / (2.f * (1.f + S.cfg.elas_poisson_ratio)),
                 S.cfg.elas_young_modulus * S.cfg.elas_poisson_ratio /
                     ((1.f + S.cfg.elas_poisson_ratio) * (1.f - 2.f * S.cfg.elas_poisson_ratio)),
                 S.hinges, S.rest_angle, S.rest_elen, S.cfg.hinge_stiffness, S.bidx, S.bkind, S.bsub, S.bd, S.iscal,
                 S.cap_b, S.cfg.d_hat, S.cfg.coll_stiffness, S.cfg.ee_classify_thres, S.partials, n_halves, S.dscal,
                 S.fscal + 1};
}

static int energy_pass(Stage3 &S, cudaStream_t s, int n_halves = -1)
{
    EArgs e = energy_args(S, n_halves);
    launch(k_energy, kRedBlocks, kThreads, 0, s, e);
    return cudaGetLastError() == cudaSuccess ? PAMO_OK : PAMO_ERR_DEVICE;
}

void Stage3::drop_graph()
{
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
    graph_cap_b = -1;
    graph_kernels = 0;
    graph_stale = false;
}

// One Newton iteration (system.py:354-409).  Contact detection ends with a host
// synchronisation (block count, buffer growth); everything after it has fixed
// sizes and pointers and no host decision, so it is captured once as a CUDA
// graph and replayed (recaptured when the contact buffer grows or a new mesh is
// registered).  A recapture updates the executable graph in place when its
// shape is unchanged -- the usual case, as only sizes and pointers move -- which
// costs the host far less than instantiating it again (the device idles
// meanwhile); otherwise the graph is instantiated anew.  With the phase timer
// on, the iteration runs eagerly so its events can be recorded.
int Stage3::newton(cudaStream_t s)
{
    S3_TRY(cudaMemcpyAsync(q_prev, q, (size_t)np * 16, cudaMemcpyDeviceToDevice, s));
    int rc = newton_elements(s);
    if (rc) return rc;
    if (prof) prof->begin(PH_S3_DETECT, s);
    if ((rc = detect(s))) return rc;
    if ((rc = newton_contacts(s))) return rc;
    const bool timed = prof && prof->on;
    if (timed || !use_graph) return newton_body(s);
    if (!graph || graph_stale || graph_cap_b != cap_b) {
        const long long before = g_launches.load();
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();  // e.g. the legacy default stream: run the iteration directly
            use_graph = false;
            return newton_body(s);
        }
        rc = newton_body(s);
        cudaError_t ce = cudaStreamEndCapture(s, &g);
        const long long kernels = g_launches.load() - before;
        g_launches.fetch_sub(kernels);  // captured, not launched
        if (rc || ce != cudaSuccess || !g) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            drop_graph();
            if (rc) return rc;
            use_graph = false;  // this stream cannot be captured: run the iteration directly
            return newton_body(s);
        }
        if (graph) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(graph, g, &info) != cudaSuccess) {  // another shape: instantiate anew
                cudaGetLastError();
                cudaGraphExecDestroy(graph);
                graph = nullptr;
            }
        }
        if (!graph) {
            ce = cudaGraphInstantiate(&graph, g, 0);
            if (ce != cudaSuccess) {
                cudaGraphDestroy(g);
                graph = nullptr;
                drop_graph();
                cudaGetLastError();
                use_graph = false;
                return newton_body(s);
            }
        }
        cudaGraphDestroy(g);
        graph_kernels = kernels;
        graph_cap_b = cap_b;
        graph_stale = false;
    }
    S3_TRY(cudaGraphLaunch(graph, s));
    g_launches.fetch_add(graph_kernels);
    return PAMO_OK;
}

static DArgs diff_args(Stage3 &S)
{
    const pamo_s3_config &c = S.cfg;
    return DArgs{S.q, S.nt, S.nh, S.tris, S.area, S.inv_dm, c.elas_young_modulus / (2.f * (1.f + c.elas_poisson_ratio)),
                 c.elas_young_modulus * c.elas_poisson_ratio /
                     ((1.f + c.elas_poisson_ratio) * (1.f - 2.f * c.elas_poisson_ratio)),
                 S.hinges, S.rest_angle, S.rest_elen, c.hinge_stiffness, c.spd_max_iters, S.kval, S.tri_slot,
                 S.hinge_slot, S.hblk, S.bidx, S.bkind, S.bsub, S.bd, S.bg, S.bb2, S.iscal, S.cap_b, c.d_hat,
                 c.coll_stiffness, S.grad, S.diag, S.bact};
}

// The element terms that do not depend on the contacts -- the vertex term, the
// membranes, and the hinges with their SPD projection -- all adding into grad,
// diag and the Hessian's values by atomics.  They are issued before detection,
// which leaves q, grad, diag and the Hessian alone: the hinge branch runs on
// side[1] while the host waits for detection's counts.
int Stage3::newton_elements(cudaStream_t s)
{
    if (prof) prof->begin(PH_S3_DIFF, s);
    S3_TRY(cudaMemcpyAsync(q_det, q, (size_t)np * 16, cudaMemcpyDeviceToDevice, s));
    // gradient (coefficient -1) and diagonal
    launch(k_diff_vertex, grid_for(np), kThreads, 0, s, q, target, wk, np, grad, diag);
    const DArgs d = diff_args(*this);
    // the Hessian's values: zero and the vertex term, then the elements
    S3_TRY(cudaMemsetAsync(kval, 0, (size_t)nnz * 48, s));
    launch(k_diag_term, grid_for(np), kThreads, 0, s, (const float *)wk, (const int *)diag_slot, np, kval);
    S3_TRY(cudaEventRecord(ev_fork, s));
    S3_TRY(cudaStreamWaitEvent(side[1], ev_fork, 0));
    if (nh > 0) {
        launch(k_diff_part<1>, grid_for(nh, 128), 128, 0, side[1], d);
        launch(k_hinge_spd, (int)((nh + 63) / 64), 64, 0, side[1], (const float *)hblk, nh, cfg.spd_max_iters,
               (const int *)hinge_slot, kval);
    }
    launch(k_diff_part<0>, grid_for(nt, 128), 128, 0, s, d);
    S3_TRY(cudaEventRecord(ev_join[1], side[1]));
    return cudaGetLastError() == cudaSuccess ? PAMO_OK : PAMO_ERR_DEVICE;
}

// After detection: the energy at the iterate (which fixes the contact blocks'
// distances and classes), the contact terms, and the join with the hinge
// branch.
int Stage3::newton_contacts(cudaStream_t s)
{
    int rc;
    if (prof) prof->begin(PH_S3_DIFF, s);
    S3_TRY(cudaMemsetAsync(iscal + I_NACT, 0, sizeof(int), s));
    if ((rc = energy_pass(*this, s))) return rc;
    launch(k_diff_part<2>, grid_for(cap_b, 128), 128, 0, s, diff_args(*this));
    S3_TRY(cudaStreamWaitEvent(s, ev_join[1], 0));
    return cudaGetLastError() == cudaSuccess ? PAMO_OK : PAMO_ERR_DEVICE;
}

// The solve, the CCD and the line search: one CUDA graph per registration.
int Stage3::newton_body(cudaStream_t s)
{
    int rc;
    // Jacobi-preconditioned CG (cg_solver.py:96-158)
    if (prof) prof->begin(PH_S3_CG, s);
    if ((rc = cg_solve(s))) return rc;
    if (prof) prof->begin(PH_S3_CCD, s);
    launch(k_clamp, grid_for(np), kThreads, 0, s, p, q_prev, q_det, np, cfg.contact_detection_radius);
    launch(k_set_float, 1, 1, 0, s, fscal, 1.0f);
    launch(k_set_float, 1, 1, 0, s, fscal + 1, 0.0f);
    launch(k_max_norm, grid_for(np), kThreads, 0, s, (const float4 *)p, np, fscal + 1);
    launch(k_accd, grid_for(cap_b, 128), 128, 0, s, q, p, bidx, bkind, iscal, cap_b, cfg.ccd_slackness, cfg.ccd_thickness,
                                                cfg.ccd_max_iters, cfg.ee_classify_thres, fscal);
    // line search (system.py:393-409)
    if (prof) prof->begin(PH_S3_LINE, s);
    if (cg_persistent == 1 && ls_persistent == 1) {
        EArgs e = energy_args(*this, 0);
        LSArgs la{e, q, q_prev, p, fscal, cfg.n_line_search_iters, reinterpret_cast<unsigned long long *>(partials),
                  cg_spin_limit};
        S3_TRY(cudaMemsetAsync(partials, 0xFF, (size_t)kSlotSets * cg_blocks * kSlotStride * sizeof(unsigned long long), s));
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(cg_blocks);
        lc.blockDim = dim3(kLsThreads);
        lc.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        lc.attrs = attr;
        lc.numAttrs = 1;
        g_launches.fetch_add(1, std::memory_order_relaxed);
        S3_TRY(cudaLaunchKernelEx(&lc, k_line_search_all, la));
    } else {
        launch(k_copy_energy_prev, 1, 1, 0, s, dscal);
        for (int nh_ = 0; nh_ < cfg.n_line_search_iters; ++nh_) {
            launch(k_line_search, grid_for(np), kThreads, 0, s, q_prev, p, fscal, nh_, dscal, np, q, iscal);
            if ((rc = energy_pass(*this, s, nh_))) return rc;
        }
    }
    if (trace) launch(k_trace, 1, 1, 0, s, (const double *)dscal, (const float *)fscal, iscal, trace, cap_trace);
    if (prof) prof->end(s);
    return cudaGetLastError() == cudaSuccess ? PAMO_OK : PAMO_ERR_DEVICE;
}

// The Jacobi-preconditioned CG of one Newton iteration (cg_solver.py:96-158):
// solves K p = grad (grad holds -dE/dx) with the assembled blocks plus the
// active contact terms, diag as the preconditioner, cfg.n_cg_iters iterations.
int Stage3::cg_solve(cudaStream_t s)
{
    if (cg_persistent < 0) {  // first use: can all blocks of the solve be resident at once?
        int dev = 0, coop = 0, per_sm = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg_solve, kCgThreads, 0);
        cg_persistent = (coop && per_sm >= 1 && sms >= 1) ? 1 : 0;
        int per_sm_ls = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_ls, k_line_search_all, kLsThreads, 0);
        ls_persistent = (coop && per_sm_ls >= 1) ? 1 : 0;
        cg_blocks = sms < kRedBlocks ? sms : kRedBlocks;  // one block per SM, all resident
        cudaGetLastError();
    }
    const OpArgs op{np, row_ptr, col, kval, bidx, bg, bb2, bact, iscal, cap_b};
    if (cg_persistent == 1) {
        // partials hold the solve's kSlotSets x cg_blocks slots, all set to kSumPending
        unsigned long long *slots = reinterpret_cast<unsigned long long *>(partials);
        // the records: cg_rec (two copies of kRec float4 per vertex); the contact parts: Avc, r, z
        CGArgs ca{op, grad, diag, p, v, cg_rec, cg_rec + kRec * cap_p, Avc, r, z, slots, iscal, np, cfg.n_cg_iters,
                  cg_spin_limit, cg_absent_block};
        S3_TRY(cudaMemsetAsync(Avc, 0, (size_t)np * sizeof(float4), s));
        S3_TRY(cudaMemsetAsync(r, 0, (size_t)np * sizeof(float4), s));
        S3_TRY(cudaMemsetAsync(z, 0, (size_t)np * sizeof(float4), s));
        S3_TRY(cudaMemsetAsync(slots, 0xFF, (size_t)kSlotSets * cg_blocks * kSlotStride * sizeof(unsigned long long), s));
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(cg_blocks);
        lc.blockDim = dim3(kCgThreads);
        lc.dynamicSmemBytes = 0;
        lc.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        lc.attrs = attr;
        lc.numAttrs = 1;
        g_launches.fetch_add(1, std::memory_order_relaxed);
        S3_TRY(cudaLaunchKernelEx(&lc, k_cg_solve, ca));
    } else {
        int *ticket = iscal + I_TICKET;
        launch(k_cg_init, kRedBlocks, kThreads, 0, s, grad, diag, np, p, r, z, v, partials, ticket, dscal);
        for (int it = 0; it < cfg.n_cg_iters; ++it) {
            launch(k_cg_pre, grid_for(np), kThreads, 0, s, (const float4 *)z, (const double *)dscal, np, it == 0 ? 1 : 0,
                   v);
            launch(k_op_rows, grid_for(4LL * np), kThreads, 0, s, op, (const float4 *)v, Av);
            launch(k_op_contacts, grid_for(cap_b), kThreads, 0, s, op, (const float4 *)v, Av);
            launch(k_cg_dot, kRedBlocks, kThreads, 0, s, (const float4 *)v, (const float4 *)Av, np, partials, ticket,
                   dscal);
            launch(k_cg_update, kRedBlocks, kThreads, 0, s, (const float4 *)v, (const float4 *)Av, (const float4 *)diag,
                   dscal, np, p, r, z, partials, ticket);
        }
    }
    return cudaGetLastError() == cudaSuccess ? PAMO_OK : PAMO_ERR_DEVICE;
}

int Stage3::step(cudaStream_t s)
{
    if (do_nothing) return PAMO_OK;
    S3_TRY(cudaMemsetAsync(iscal + I_STACK, 0, 4, s));
    if (prof) prof->begin(PH_S3_CLOSEST, s);
    launch(k_closest, grid_for(np), kThreads, 0, s, q, np, gt_bvh.nodes, gt_bvh.vals, gt_bvh.scene, gt_pts, gt_tris, target,
                                                iscal);
    for (int it = 0; it < cfg.n_newton_iters; ++it) {
        int rc = newton(s);
        if (rc) return rc;
    }
    return PAMO_OK;
}

int Stage3::ensure_trace(long long rows)
{
    if (rows <= cap_trace && trace) return PAMO_OK;
    if (trace) cudaFree(trace);
    trace = nullptr;
    cap_trace = 0;
    if (rows <= 0) return PAMO_OK;
    if (cudaMalloc((void **)&trace, (size_t)rows * 6 * sizeof(double)) != cudaSuccess) return PAMO_ERR_OOM;
    cap_trace = rows;
    drop_graph();  // the captured iteration holds the trace pointer
    return PAMO_OK;
}

int Stage3::solve_bsr(int n, const int *d_row_ptr, const int *d_col, const float *d_blocks, long long n_blocks,
                      const float *d_diag, const float *d_rhs, int iters, float *d_out, cudaStream_t s)
{
    int rc = ensure(n, 1, 1, 1, 1, 1);
    if (rc) return rc;
    if (n_blocks > cap_nnz || !kval) {
        if (col) cudaFree(col);
        if (kval) cudaFree(kval);
        col = nullptr;
        kval = nullptr;
        cap_nnz = 0;
        if (cudaMalloc((void **)&col, (size_t)n_blocks * 4) != cudaSuccess ||
            cudaMalloc((void **)&kval, (size_t)n_blocks * 48) != cudaSuccess)
            return PAMO_ERR_OOM;
        cap_nnz = n_blocks;
    }
    drop_graph();
    gathered = false;
    gt_ready = false;  // the stage-3 state of this context is replaced
    np = n;
    nnz = n_blocks;
    cfg.n_cg_iters = iters;
    S3_TRY(cudaMemcpyAsync(row_ptr, d_row_ptr, ((size_t)n + 1) * 4, cudaMemcpyDeviceToDevice, s));
    S3_TRY(cudaMemcpyAsync(col, d_col, (size_t)n_blocks * 4, cudaMemcpyDeviceToDevice, s));
    launch(k_blocks9_to_rows, grid_for(n_blocks), kThreads, 0, s, d_blocks, n_blocks, kval);
    launch(k_aos_to_f4, grid_for(np), kThreads, 0, s, d_diag, diag, nullptr, np);
    launch(k_aos_to_f4, grid_for(np), kThreads, 0, s, d_rhs, grad, nullptr, np);
    S3_TRY(cudaMemsetAsync(iscal, 0, 64, s));  // no contact blocks
    S3_TRY(cudaMemsetAsync(dscal, 0, 64, s));
    if ((rc = cg_solve(s))) return rc;
    launch(k_f4_to_aos, grid_for(np), kThreads, 0, s, (const float4 *)p, d_out, np);
    S3_TRY(cudaMemcpyAsync(h_iscal, iscal, 12 * sizeof(int), cudaMemcpyDeviceToHost, s));
    S3_TRY(cudaStreamSynchronize(s));
    return h_iscal[I_BAR_ERR] ? PAMO_ERR_DEVICE : PAMO_OK;
}

int Stage3::energy_now(double *out, cudaStream_t s)
{
    int rc = energy_pass(*this, s);
    if (rc) return rc;
    S3_TRY(cudaMemcpyAsync(h_dscal, dscal, 8, cudaMemcpyDeviceToHost, s));
    S3_TRY(cudaMemcpyAsync(h_iscal, iscal, 12 * sizeof(int), cudaMemcpyDeviceToHost, s));
    S3_TRY(cudaStreamSynchronize(s));
    if (h_iscal[I_BAR_ERR]) return PAMO_ERR_DEVICE;  // a solve's grid barrier timed out
    *out = h_dscal[0];
    return PAMO_OK;
}

}  // namespace s3

int s3_validate(const int *a, long long count, int hi, int *d_bad, int *h_bad, cudaStream_t st)
{
    if (count <= 0) return PAMO_OK;
    if (cudaMemsetAsync(d_bad, 0, 4, st) != cudaSuccess) return PAMO_ERR_DEVICE;
    launch(s3::k_validate_idx, grid_for(count), kThreads, 0, st, a, count, hi, d_bad);
    if (cudaMemcpyAsync(h_bad, d_bad, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) return PAMO_ERR_DEVICE;
    if (cudaStreamSynchronize(st) != cudaSuccess) return PAMO_ERR_DEVICE;
    return *h_bad == 0 ? PAMO_OK : PAMO_ERR_INVALID_ARG;
}

int s3_fetch(const float4 *q, float *out, int n, cudaStream_t st)
{
    launch(s3::k_f4_to_aos, grid_for(n), kThreads, 0, st, q, out, n);
    return cudaGetLastError() == cudaSuccess ? PAMO_OK : PAMO_ERR_DEVICE;
}

}  // namespace pamo
