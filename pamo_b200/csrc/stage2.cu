// Stage-2 collapse round on the device (sm_100a).
//
// One round follows the reference's CUSimp_Free::forward
// (simp_cuda/src/cusimp_free.cu:891-1048) decision for decision, with a B200
// layout and fewer passes:
//   face pass A   plane of every face (fp32, reference order), vertex degrees,
//                 per-face descending-edge counts                 [:276-289,306-317,337-348]
//   2 scans       vertex->face CSR offsets, edge offsets
//   face pass B   CSR fill + edge emission                          [:291-304,319-335]
//   vertex pass   canonical (ascending face) order of each CSR segment, then the
//                 quadric sum in that order                          [:350-366]
//   edge pass     cost (link condition, edge lengths, flip and skinny terms,
//                 quadric at the midpoint, u32 quantisation) fused with the
//                 64-bit key min over each endpoint                  [:382-610]
//   edge pass     independent-set test + collapse + skinny rollback  [:639-774]
//   scan/scatter  collapsed list in edge order
//   face pass     degenerate faces removed                           [:218-232]
//   edge pass     coincident-endpoint collapses                      [:234-274]
//   LBVH          build over the round's faces, refit, query of the faces touched
//                 by collapses, pair tests                           [bvh/self_intersect.cuh]
//   undo passes   candidates, restore, re-check (<= 5)               [:776-878,1015-1040]
//   scan          pts_map = exclusive scan of occupancy              [:1042-1045]
// The key independent set uses a per-vertex minimum: an edge wins iff its key is
// the minimum over every face touching either endpoint (the reference's per-face
// minimum), which equals: key == vmin[u] == vmin[v] and no vertex of those faces
// has a smaller vmin.
#include <cooperative_groups.h>
#include <cstdio>
#include <cstring>

#include "scan.cuh"
#include "exact.cuh"
#include "stage2.cuh"
#include "tritri.cuh"

namespace pamo {

#define S2_TRY_EARLY(expr)                                \
    do {                                                  \
        cudaError_t _e = (expr);                          \
        if (_e != cudaSuccess) return map_cuda_error(_e); \
    } while (0)

namespace cg = cooperative_groups;

namespace {

constexpr float kCostRange = 10.0f;
constexpr double kRebuildFraction = 0.6;

__device__ __forceinline__ uint32_t quantise_cost(float c)
{
    // the reference converts with a saturating float->u32 conversion
    return (uint32_t)(tclamp(c, 0.0f, kCostRange) / kCostRange * 4294967296.0f);
}

__global__ void k_round_init(const float4 *__restrict__ opts, const int4 *__restrict__ otris, float4 *pts,
                             int4 *tris, int *occ, int *deg, int *cursor, unsigned long long *vmin, int n, int m)
{
    long long N = (long long)(n + 1 > m ? n + 1 : m);
    PAMO_GRID_STRIDE(i, N)
    {
        if (i < n) {
            pts[i] = opts[i];
            occ[i] = 1;
            deg[i] = 0;
            cursor[i] = 0;
            vmin[i] = ~0ull;
        } else if (i == n) {
            occ[n] = 0;
            deg[n] = 0;
        }
        if (i < m) tris[i] = otris[i];
    }
}

__global__ void k_face_a(const float4 *__restrict__ pts, const int4 *__restrict__ tris, int m, int *deg,
                         int *ecount, float4 *plane, float4 *elen)
{
    PAMO_GRID_STRIDE(f, m)
    {
        int4 t = tris[f];
        if (face_dead(t)) {
            ecount[f] = 0;
            continue;
        }
        atomicAdd(&deg[t.x], 1);
        atomicAdd(&deg[t.y], 1);
        atomicAdd(&deg[t.z], 1);
        ecount[f] = (t.x > t.y) + (t.y > t.z) + (t.z > t.x);
        V3 v0 = v3(pts[t.x]), v1 = v3(pts[t.y]), v2 = v3(pts[t.z]);
        V3 nrm = vcross(vsub(v1, v0), vsub(v2, v0));
        nrm = vdivs(nrm, vnorm(nrm));
        float d = -vdot(nrm, v0);
        plane[f] = make_float4(nrm.x, nrm.y, nrm.z, d);
        // the three edge lengths in cyclic order, as the cost kernel sums them
        // (cusimp_free.cu:448-485): |P[i]-P[j]|, |P[j]-P[k]|, |P[k]-P[i]|
        elen[f] = make_float4(vnorm(vsub(v0, v1)), vnorm(vsub(v1, v2)), vnorm(vsub(v2, v0)), 0.f);
    }
}

__global__ void k_face_b(const int4 *__restrict__ tris, int m, const int *__restrict__ first_near, int *cursor,
                         int *near_tris, const int *__restrict__ first_edge, int2 *edges)
{
    PAMO_GRID_STRIDE(f, m)
    {
        int4 t = tris[f];
        if (face_dead(t)) continue;
        near_tris[first_near[t.x] + atomicAdd(&cursor[t.x], 1)] = (int)f;
        near_tris[first_near[t.y] + atomicAdd(&cursor[t.y], 1)] = (int)f;
        near_tris[first_near[t.z] + atomicAdd(&cursor[t.z], 1)] = (int)f;
        int e = first_edge[f];
        if (t.x > t.y) edges[e++] = make_int2(t.y, t.x);
        if (t.y > t.z) edges[e++] = make_int2(t.z, t.y);
        if (t.z > t.x) edges[e++] = make_int2(t.x, t.z);
    }
}

// Canonical segment order, then the quadric sum p p^T in that order.
__device__ __forceinline__ int next_after(int4 t, int v);

__global__ void k_vertex_quadric(const int *__restrict__ first_near, int *near_tris,
                                 const float4 *__restrict__ plane, const int4 *__restrict__ tris, float4 *quad,
                                 int *nxt, int n)
{
    PAMO_GRID_STRIDE(v, n)
    {
        int a = first_near[v], b = first_near[v + 1];
        for (int i = a + 1; i < b; ++i) {
            int x = near_tris[i], j = i - 1;
            while (j >= a && near_tris[j] > x) {
                near_tris[j + 1] = near_tris[j];
                --j;
            }
            near_tris[j + 1] = x;
        }
        float q0 = 0.f, q1 = 0.f, q2 = 0.f, q3 = 0.f, q4 = 0.f, q5 = 0.f, q6 = 0.f, q7 = 0.f, q8 = 0.f, q9 = 0.f;
        for (int s = a; s < b; ++s) {
            const int f = near_tris[s];
            nxt[s] = next_after(tris[f], (int)v);  // vertex after v in face f (i->j->k->i)
            float4 p = plane[f];
            q0 += p.x * p.x; q1 += p.x * p.y; q2 += p.x * p.z; q3 += p.x * p.w;
            q4 += p.y * p.y; q5 += p.y * p.z; q6 += p.y * p.w;
            q7 += p.z * p.z; q8 += p.z * p.w; q9 += p.w * p.w;
        }
        quad[3 * v + 0] = make_float4(q0, q1, q2, q3);
        quad[3 * v + 1] = make_float4(q4, q5, q6, q7);
        quad[3 * v + 2] = make_float4(q8, q9, 0.f, 0.f);
    }
}

// Quality mode: each vertex's quadric in FP64, the planes recomputed from the
// positions in FP64 (unit normal n, d = -n . a), summed over the vertex's faces
// in its (sorted) list order, so the result is deterministic.
__global__ void k_vertex_quadric64(const int *__restrict__ first_near, const int *__restrict__ near_tris,
                                   const float4 *__restrict__ pts, const int4 *__restrict__ tris, double *q64, int n)
{
    PAMO_GRID_STRIDE(v, n)
    {
        double q[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int s = first_near[v]; s < first_near[v + 1]; ++s) {
            const int4 t = tris[near_tris[s]];
            const float4 fa = pts[t.x], fb = pts[t.y], fc = pts[t.z];
            const double ax = fa.x, ay = fa.y, az = fa.z;
            const double ux = fb.x - ax, uy = fb.y - ay, uz = fb.z - az;
            const double wx = fc.x - ax, wy = fc.y - ay, wz = fc.z - az;
            double nx = uy * wz - uz * wy, ny = uz * wx - ux * wz, nz = ux * wy - uy * wx;
            const double len = sqrt(nx * nx + ny * ny + nz * nz);
            if (!(len > 0.0)) continue;  // a degenerate face has no plane
            nx /= len;
            ny /= len;
            nz /= len;
            const double d = -(nx * ax + ny * ay + nz * az);
            q[0] += nx * nx; q[1] += nx * ny; q[2] += nx * nz; q[3] += nx * d;
            q[4] += ny * ny; q[5] += ny * nz; q[6] += ny * d;
            q[7] += nz * nz; q[8] += nz * d; q[9] += d * d;
        }
        for (int k = 0; k < 10; ++k) q64[10 * (size_t)v + k] = q[k];
    }
}

// Quality mode: the point minimising v^T (Qu + Qv) v, from the 3 x 3 system
// A x = -b of the summed quadric (Cramer's rule in FP64).  The midpoint is kept
// when the system is close to singular (|det| below 1e-12 of the product of
// A's row norms) or the minimiser lies more than the edge's length from the
// midpoint (a nearly flat, ill-conditioned quadric).
__device__ V3 qem_position(const double *qu, const double *qv, V3 p0, V3 p1)
{
    double q[10];
    for (int k = 0; k < 10; ++k) q[k] = qu[k] + qv[k];
    const double a00 = q[0], a01 = q[1], a02 = q[2], a11 = q[4], a12 = q[5], a22 = q[7];
    const double b0 = -q[3], b1 = -q[6], b2 = -q[8];
    const double c00 = a11 * a22 - a12 * a12, c01 = a02 * a12 - a01 * a22, c02 = a01 * a12 - a02 * a11;
    const double det = a00 * c00 + a01 * c01 + a02 * c02;
    const double r0 = sqrt(a00 * a00 + a01 * a01 + a02 * a02), r1 = sqrt(a01 * a01 + a11 * a11 + a12 * a12);
    const double r2 = sqrt(a02 * a02 + a12 * a12 + a22 * a22);
    const V3 mid = vmid(p0, p1);
    if (!(fabs(det) > 1e-12 * r0 * r1 * r2)) return mid;
    const double c11 = a00 * a22 - a02 * a02, c12 = a01 * a02 - a00 * a12, c22 = a00 * a11 - a01 * a01;
    const double x = (c00 * b0 + c01 * b1 + c02 * b2) / det;
    const double y = (c01 * b0 + c11 * b1 + c12 * b2) / det;
    const double z = (c02 * b0 + c12 * b1 + c22 * b2) / det;
    const double ex = (double)p1.x - p0.x, ey = (double)p1.y - p0.y, ez = (double)p1.z - p0.z;
    const double dx = x - mid.x, dy = y - mid.y, dz = z - mid.z;
    if (!(dx * dx + dy * dy + dz * dz <= ex * ex + ey * ey + ez * ez)) return mid;
    return {(float)x, (float)y, (float)z};
}

__device__ __forceinline__ int next_after(int4 t, int v)
{
    if (t.x == v) return t.y;
    if (t.y == v) return t.z;
    if (t.z == v) return t.x;
    return -2;
}

__device__ __forceinline__ float skinny_term(V3 n0, V3 n1, V3 n2)
{
    // edge_length / triangle_area (cusimp_free.cu:368-380) and the penalty with
    // the reference's precedence: only the first square divides (:533,573)
    float l01 = vnorm(vsub(n0, n1));
    float l12 = vnorm(vsub(n1, n2));
    float l20 = vnorm(vsub(n2, n0));
    float s = (l01 + l12 + l20) / 2.0f;
    float area = sqrtf(s * (s - l01) * (s - l12) * (s - l20));
    // pow(float, 2) in the reference resolves to std::pow's promoting overload:
    // the squares and the sum after the fp32 numerator are doubles, rounded once
    const float c4s3 = 4.0f * sqrtf(3.0f);
    float num = c4s3 * area;
    // Shortcut: every term is non-negative, so the same sum in fp32 (five
    // roundings, relative error < 4e-7 while l01^2 is a normal float; an fp32
    // overflow to +inf only happens when the double sum is far above 1) bounds
    // the double sum from below within 4e-7.  At or above 1 + 2^-18 the double
    // sum is above 1, its float rounding is >= 1, and the clamped penalty is
    // exactly 0 -- the value the double path returns.  Well-shaped triangles
    // (sum near 3) take this path; NaN and near-1 sums fall through.
    const float q01 = l01 * l01;
    if (q01 >= 1.17549435e-38f) {
        float ef = num / q01 + l12 * l12 + l20 * l20 + 0.0000001f;
        if (ef >= 1.0f + 0x1p-18f) return 0.0f;
    }
    // Second shortcut: CUDA's double pow(x, 2.0) is within one double ulp of the
    // exact square x*x for every float x (an exhaustive check over all finite
    // floats on a B200; it differs for ~6% of them).  The same sum with exact
    // squares therefore lies within 8 ulp of the one with pow (each term is
    // non-negative); when a 16-ulp neighbourhood of it rounds to one float, that
    // float is the reference's.  Otherwise (NaN, inf, or a sum next to a float
    // rounding boundary) the pow form is evaluated as the reference writes it.
    const double sq = (double)num / ((double)l01 * (double)l01) + (double)l12 * (double)l12 +
                      (double)l20 * (double)l20 + (double)0.0000001f;
    const double margin = sq * 0x1p-48;
    const float fq = (float)sq;
    if (fq == (float)(sq - margin) && fq == (float)(sq + margin)) return 1.0f - tclamp(fq, 0.0f, 1.0f);
    double e = (double)num / pow((double)l01, 2.0) + pow((double)l12, 2.0) + pow((double)l20, 2.0) +
               (double)0.0000001f;
    return 1.0f - tclamp((float)e, 0.0f, 1.0f);
}

// Whether the moved face's unit normal c / |c| points against `on`, i.e. the
// reference's dot(on, c / |c|) < 0 with c normalised by three divisions.
// Shortcut: with |c|^2 in the normal range and |on . c| well above the
// rounding error of either dot product (1e-5 of sum |on_i c_i|, against a few
// 2^-24 for both forms), the two dot products have the same, non-zero sign, and
// dot(on, c) / |c| stays far from underflow (dc^2 > 1e-30 |c|^2).  Otherwise
// the reference's expression is evaluated.
__device__ __forceinline__ bool normal_flips(V3 on, V3 c)
{
    const float s2 = c.x * c.x + c.y * c.y + c.z * c.z;
    const float dc = vdot(on, c);
    const float mag = fabsf(on.x * c.x) + fabsf(on.y * c.y) + fabsf(on.z * c.z);
    if (s2 > 1e-30f && s2 < 1e30f && fabsf(dc) > 1e-5f * mag && dc * dc > 1e-30f * s2) return dc < 0.f;
    const V3 nn = vdivs(c, vnorm(c));
    return vdot(on, nn) < 0;
}

struct CostArgs {
    const int2 *edges;
    const int *n_edges;
    const float4 *pts;
    const int4 *tris;
    const int *first_near;
    const int *near_tris;
    const int *nxt;
    const float4 *plane;
    const float4 *elen;
    const float4 *quad;
    const uint8_t *invalid;
    uint32_t *edge_cost;
    unsigned long long *vmin;
    float tres, edge_s;
    int is_stuck;
    // batch mode (null otherwise): per-mesh parameters and stale state
    const SlotInfo *slots;
    const SlotCounters *scnt;
    const int *vslot;
    // quality mode (null otherwise): FP64 quadrics in, collapse positions out
    const double *quad64;
    float4 *epos;
};

// Returns true when the reference writes a new cost for the edge.  QUALITY:
// quality mode (FP64 quadric terms and the chosen collapse position in epos);
// compiled separately so the reference's path carries none of it.
template <bool QUALITY>
__device__ bool edge_cost_value(const CostArgs &A, int u, int v, bool inv_u, bool inv_v, float tres, float edge_s,
                                int is_stuck, uint32_t &out, int e = -1)
{
    if constexpr (QUALITY) {  // an edge whose cost is not rewritten collapses to its midpoint
        const V3 m0 = vmid(v3(A.pts[u]), v3(A.pts[v]));
        A.epos[e] = make_float4(m0.x, m0.y, m0.z, 0.f);
    }
    if (inv_u && inv_v) {
        out = 0xFFFFFFFFu;
        return true;
    }
    if (is_stuck) return false;
    const int ua = A.first_near[u], ub = A.first_near[u + 1];
    const int va = A.first_near[v], vb = A.first_near[v + 1];
    int dup = 0;
    for (int a = ua; a < ub; ++a) {
        int iu = A.nxt[a];
        for (int b = va; b < vb; ++b) {
            int iv = A.nxt[b];
            if (iu == iv) dup++;
            if (dup > 2) {
                out = 0xFFFFFFFFu;
                return true;
            }
        }
    }
    if (dup != 2) return false;

    float elen = 0.0f;
    int nedge = 0;
    for (int pass = 0; pass < 2; ++pass) {
        int lo = pass ? va : ua, hi = pass ? vb : ub;
        for (int a = lo; a < hi; ++a) {
            const int f = A.near_tris[a];
            int4 t = A.tris[f];
            float4 l = A.elen[f];
            if (t.x > t.y) { elen += l.x; nedge++; }
            if (t.y > t.z) { elen += l.y; nedge++; }
            if (t.z > t.x) { elen += l.z; nedge++; }
        }
    }
    V3 v0 = v3(A.pts[u]), v1 = v3(A.pts[v]);
    elen = elen / (float)nedge / edge_s * tres;
    elen = elen + vnorm(vsub(v0, v1)) / edge_s * tres;
    // the collapse position: the midpoint (the reference), or in quality mode
    // the FP64 quadric's minimiser
    V3 mid;
    if constexpr (QUALITY) {
        mid = qem_position(A.quad64 + 10 * (size_t)u, A.quad64 + 10 * (size_t)v, v0, v1);
        A.epos[e] = make_float4(mid.x, mid.y, mid.z, 0.f);
    } else {
        mid = vmid(v0, v1);
    }

    float Qa = 0.0f;
    int ntri = 0;
    for (int pass = 0; pass < 2; ++pass) {
        int w = pass ? v : u, other = pass ? u : v;
        int lo = pass ? va : ua, hi = pass ? vb : ub;
        for (int a = lo; a < hi; ++a) {
            const int f = A.near_tris[a];
            int4 t = A.tris[f];
            if (face_has(t, other)) continue;
            V3 o0 = v3(A.pts[t.x]), o1 = v3(A.pts[t.y]), o2 = v3(A.pts[t.z]);
            V3 n0 = t.x == w ? mid : o0;
            V3 n1 = t.y == w ? mid : o1;
            V3 n2 = t.z == w ? mid : o2;
            // the unchanged face's unit normal is the face plane's (same expression)
            V3 on = v3(A.plane[f]);
            const V3 c = vcross(vsub(n1, n0), vsub(n2, n0));
            if (normal_flips(on, c)) {
                out = 0xFFFFFFFFu;
                return true;
            }
            Qa += skinny_term(n0, n1, n2);
            ntri++;
        }
    }
    Qa = 5.0f * Qa;
    if constexpr (QUALITY) {  // the quadric error in FP64 at the chosen position
        const double *qu = A.quad64 + 10 * (size_t)u, *qv = A.quad64 + 10 * (size_t)v;
        double q[10];
        for (int k = 0; k < 10; ++k) q[k] = qu[k] + qv[k];
        const double x = mid.x, y = mid.y, z = mid.z;
        const double qe = x * (q[0] * x + q[1] * y + q[2] * z + q[3]) + y * (q[1] * x + q[4] * y + q[5] * z + q[6]) +
                          z * (q[2] * x + q[5] * y + q[7] * z + q[8]) + (q[3] * x + q[6] * y + q[8] * z + q[9]);
        const float cost = (float)(qe / ((double)edge_s * (double)edge_s));
        out = quantise_cost(cost + elen + Qa / (float)ntri * tres);
        return true;
    }
    float4 a0 = A.quad[3 * u], a1 = A.quad[3 * u + 1], a2 = A.quad[3 * u + 2];
    float4 b0 = A.quad[3 * v], b1 = A.quad[3 * v + 1], b2 = A.quad[3 * v + 2];
    float m00 = a0.x + b0.x, m01 = a0.y + b0.y, m02 = a0.z + b0.z, m03 = a0.w + b0.w;
    float m11 = a1.x + b1.x, m12 = a1.y + b1.y, m13 = a1.z + b1.z, m22 = a1.w + b1.w;
    float m23 = a2.x + b2.x, m33 = a2.y + b2.y;
    float x = mid.x, y = mid.y, z = mid.z, w = 1.0f;
    float r0 = m00 * x + m01 * y + m02 * z + m03 * w;
    float r1 = m01 * x + m11 * y + m12 * z + m13 * w;
    float r2 = m02 * x + m12 * y + m22 * z + m23 * w;
    float r3 = m03 * x + m13 * y + m23 * z + m33 * w;
    float qe = r0 * x + r1 * y + r2 * z + r3 * w;
    float cost = qe / (edge_s * edge_s);
    out = quantise_cost(cost + elen + Qa / (float)ntri * tres);
    return true;
}

// The edge-cost pass runs in the hierarchy's leaf (Morton) order: a block takes
// kChunkFaces consecutive leaves, lists their faces' edges in shared memory
// (each face owns its 0-2 descending edges) and its threads take the list in
// turn, so neighbouring lanes gather neighbouring vertices and every lane has an
// edge.  Costs are indexed by edge, so the order of work does not change them.
constexpr int kChunkFaces = kThreads;
constexpr int kChunkEdges = 3 * kChunkFaces;

__device__ __forceinline__ int chunk_edges(const int *order, const int *first_edge, int L, long long base,
                                           int *s_list)
{
    long long p = base + threadIdx.x;
    int f = p < L ? order[p] : -1;  // -1: past the end, or a face removed since the build
    int fe = f >= 0 ? first_edge[f] : 0;
    int c = f >= 0 ? first_edge[f + 1] - fe : 0;
    int total;
    int off = block_excl_scan<kThreads>(c, total);
    for (int j = 0; j < c; ++j) s_list[off + j] = fe + j;
    __syncthreads();
    return total;
}

template <bool QUALITY>
__global__ void __launch_bounds__(kThreads) k_edge_cost(CostArgs A, const int *order, const int *scene,
                                                        const int *first_edge)
{
    __shared__ int s_list[kChunkEdges];
    const int L = scene[7];
    for (long long base = (long long)blockIdx.x * kChunkFaces; base < L; base += (long long)gridDim.x * kChunkFaces) {
        const int total = chunk_edges(order, first_edge, L, base, s_list);
        for (int q = threadIdx.x; q < total; q += kThreads) {
            const int e = s_list[q];
            int2 ed = A.edges[e];
            uint32_t c;
            if (!A.slots) {
                if (edge_cost_value<QUALITY>(A, ed.x, ed.y, A.invalid[ed.x], A.invalid[ed.y], A.tres, A.edge_s,
                                             A.is_stuck, c, e))
                    A.edge_cost[e] = c;
                else
                    c = A.edge_cost[e];  // the reference keeps the previous round's value
            } else {  // the mesh's own parameters, invalid table and stale costs (mesh-local numbers)
                const int r = A.vslot[ed.x];
                const SlotInfo &S = A.slots[r];
                const int el = e - A.scnt[r].edge_off;
                if (edge_cost_value<QUALITY>(A, ed.x, ed.y, S.invalid[ed.x - S.vert_off], S.invalid[ed.y - S.vert_off],
                                             S.tres, *S.scale, S.is_stuck, c))
                    S.edge_cost[el] = c;
                else
                    c = S.edge_cost[el];
            }
            unsigned long long key = ((unsigned long long)c << 32) | (unsigned)e;
            atomicMin(&A.vmin[ed.x], key);
            atomicMin(&A.vmin[ed.y], key);
        }
        __syncthreads();
    }
}

__device__ __forceinline__ bool is_skinny(V3 p, V3 q, V3 r)
{
    V3 pq = vsub(q, p), pr = vsub(r, p), qr = vsub(r, q);
    float lpq = sqrtf(vdot(pq, pq)), lpr = sqrtf(vdot(pr, pr)), lqr = sqrtf(vdot(qr, qr));
    float ml = fmaxf(lpq, fmaxf(lpr, lqr));
    V3 c = vcross(pq, pr);
    float thr = (float)(1e-6 * (double)ml * (double)ml);
    float area = 0.5f * sqrtf(c.x * c.x + c.y * c.y + c.z * c.z);
    return area < thr;
}

struct CollapseArgs {
    const int2 *edges;
    const int *n_edges;
    const uint32_t *edge_cost;
    const unsigned long long *vmin;
    const int *first_near;
    const int *near_tris;
    const float4 *opts;
    const int4 *otris;
    float4 *pts;
    int4 *tris;
    int *occ;
    int *eflag;
    uint32_t collapse_t;
    const SlotInfo *slots;  // batch mode (null otherwise)
    const SlotCounters *scnt;
    const int *vslot;
    const float4 *epos;  // quality mode: the position the edge cost chose (null: the midpoint)
};

__device__ __forceinline__ bool faces_min_ok(const CollapseArgs &A, int lo, int hi, unsigned long long key)
{
    for (int a = lo; a < hi; ++a) {
        int4 t = A.otris[A.near_tris[a]];  // round input: never written during this pass
        if (A.vmin[t.x] < key || A.vmin[t.y] < key || A.vmin[t.z] < key) return false;
    }
    return true;
}

// The independent set: one thread per edge tests the threshold and the key
// (most edges fail at once) and flags the winners; the collapse list is their
// scan.  The winners' collapses then run one thread per winner
// (k_collapse_apply), so no warp carries idle lanes through a collapse.
// Winners have disjoint one-rings, and the tests read only the round input
// (otris) and the key minima, so splitting the two changes nothing.
__global__ void __launch_bounds__(kThreads) k_collapse(CollapseArgs A)
{
    const int E = *A.n_edges;
    PAMO_GRID_STRIDE(ee, E)
    {
        const int e = (int)ee;
        int win = 0;
        uint32_t c, collapse_t;
        if (!A.slots) {
            c = A.edge_cost[e];
            collapse_t = A.collapse_t;
        } else {
            const int r = A.vslot[A.edges[e].x];
            c = A.slots[r].edge_cost[e - A.scnt[r].edge_off];
            collapse_t = A.slots[r].collapse_t;
        }
        if (c <= collapse_t) {
            const int2 ed = A.edges[e];
            const int u = ed.x, v = ed.y;
            const unsigned long long key = ((unsigned long long)c << 32) | (unsigned)e;
            if (A.vmin[u] == key && A.vmin[v] == key)
                win = faces_min_ok(A, A.first_near[u], A.first_near[u + 1], key) &&
                      faces_min_ok(A, A.first_near[v], A.first_near[v + 1], key);
        }
        A.eflag[e] = win;
    }
}

// Collapse of each winner (list[0, *n_list)): u moves to the midpoint (the
// quality mode's chosen position), v goes, faces holding both die and v's faces
// take u; if a surviving one-ring face is skinny the one-rings are restored from
// the round input, and the edge stays in the collapsed list.
template <bool QUALITY>
__global__ void __launch_bounds__(kThreads) k_collapse_apply(CollapseArgs A, const int *list, const int *n_list)
{
    const int N = *n_list;
    PAMO_GRID_STRIDE(k, N)
    {
        const int e = list[k];
        const int2 ed = A.edges[e];
        const int u = ed.x, v = ed.y;
        const int ua = A.first_near[u], ub = A.first_near[u + 1];
        const int va = A.first_near[v], vb = A.first_near[v + 1];
        V3 mid;
        if constexpr (QUALITY) mid = v3(A.epos[e]);  // the position the edge cost chose
        else mid = vmid(v3(A.opts[u]), v3(A.opts[v]));
        A.pts[u] = make_float4(mid.x, mid.y, mid.z, 0.f);
        A.pts[v] = make_float4(0.f, 0.f, 0.f, 0.f);
        A.occ[v] = 0;
        for (int a = ua; a < ub; ++a) {
            const int f = A.near_tris[a];
            const int4 t = A.tris[f];
            if (face_has(t, v)) A.tris[f] = make_int4(-1, -1, -1, 0);
        }
        for (int a = va; a < vb; ++a) {
            const int f = A.near_tris[a];
            int4 t = A.tris[f];
            if (face_has(t, u)) t = make_int4(-1, -1, -1, 0);
            else if (t.x == v) t.x = u;
            else if (t.y == v) t.y = u;
            else if (t.z == v) t.z = u;
            A.tris[f] = t;
        }
        bool sk = false;
        for (int pass = 0; pass < 2 && !sk; ++pass) {
            const int lo = pass ? va : ua, hi = pass ? vb : ub;
            for (int a = lo; a < hi; ++a) {
                const int4 t = A.tris[A.near_tris[a]];
                if (t.x == -1) continue;
                if (is_skinny(v3(A.pts[t.x]), v3(A.pts[t.y]), v3(A.pts[t.z]))) {
                    sk = true;
                    break;
                }
            }
        }
        if (sk) {  // roll back; the edge stays in the collapsed list
            A.occ[v] = 1;
            A.pts[u] = A.opts[u];
            A.pts[v] = A.opts[v];
            for (int a = ua; a < ub; ++a) A.tris[A.near_tris[a]] = A.otris[A.near_tris[a]];
            for (int a = va; a < vb; ++a) A.tris[A.near_tris[a]] = A.otris[A.near_tris[a]];
        }
    }
}

// list[pos[i]] = i for flagged i (pos = exclusive scan of the flags)
__global__ void k_scatter_flagged(const int *__restrict__ flags, const int *__restrict__ pos, const int *d_n,
                                  int *list, int list_offset)
{
    const int N = *d_n;
    PAMO_GRID_STRIDE(i, N)
    {
        if (flags[i]) list[list_offset + pos[i]] = (int)i;
    }
}

__global__ void k_remove_invalid_faces(int4 *tris, int m)
{
    PAMO_GRID_STRIDE(f, m)
    {
        int4 t = tris[f];
        if (face_dead(t)) continue;
        if (t.x == t.y || t.y == t.z || t.z == t.x) tris[f] = make_int4(-1, -1, -1, 0);
    }
}

__global__ void k_line_flags(const int2 *edges, const int *n_edges, const float4 *pts, int *eflag, int *count)
{
    const int E = *n_edges;
    int local = 0;
    PAMO_GRID_STRIDE(e, E)
    {
        int2 ed = edges[e];
        float4 p = pts[ed.x], q = pts[ed.y];
        int f = (p.x == q.x && p.y == q.y && p.z == q.z);
        eflag[e] = f;
        local += f;
    }
    if (local) atomicAdd(count, local);
}

// Coincident-endpoint collapses: positions were read (k_line_flags) before any
// write; the writes are applied in edge order by one thread.  Flagged edges are
// rare (exactly equal coordinates), so one block of kLineThreads finds them
// chunk by chunk and its thread 0 applies each chunk's edges in order.
constexpr int kLineThreads = 1024;
constexpr int kLinePerThread = 8;

__device__ __forceinline__ void line_collapse(int u, int v, const int *first_near, const int *near_tris, float4 *pts,
                                              int4 *tris, int *occ)
{
    pts[v] = make_float4(0.f, 0.f, 0.f, 0.f);
    occ[v] = 0;
    for (int a = first_near[u]; a < first_near[u + 1]; ++a) {
        int f = near_tris[a];
        if (face_has(tris[f], v)) tris[f] = make_int4(-1, -1, -1, 0);
    }
    for (int a = first_near[v]; a < first_near[v + 1]; ++a) {
        int f = near_tris[a];
        int4 t = tris[f];
        if (face_has(t, u)) t = make_int4(-1, -1, -1, 0);
        else if (t.x == v) t.x = u;
        else if (t.y == v) t.y = u;
        else if (t.z == v) t.z = u;
        tris[f] = t;
    }
}

// Calls on_edge(e) on thread 0 for every flagged e < E, in ascending order.
template <typename OnEdge>
__device__ __forceinline__ void for_flagged_in_order(const int *eflag, int E, OnEdge on_edge)
{
    __shared__ int s_idx[kLineThreads * kLinePerThread];
    for (long long base = 0; base < E; base += kLineThreads * kLinePerThread) {
        int local[kLinePerThread];
        int c = 0;
#pragma unroll
        for (int k = 0; k < kLinePerThread; ++k) {
            long long e = base + (long long)threadIdx.x * kLinePerThread + k;
            if (e < E && eflag[e]) local[c++] = (int)e;
        }
        int total;
        int off = block_excl_scan<kLineThreads>(c, total);
        for (int k = 0; k < c; ++k) s_idx[off + k] = local[k];
        __syncthreads();
        if (threadIdx.x == 0)
            for (int i = 0; i < total; ++i) on_edge(s_idx[i]);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kLineThreads) k_line_apply(const int2 *edges, const int *n_edges, const int *eflag,
                                                             const int *first_near, const int *near_tris, float4 *pts,
                                                             int4 *tris, int *occ, int *collapsed, RoundCounters *cnt)
{
    const int E = *n_edges;
    const int nm = cnt->n_main;
    int k = 0;
    if (cnt->n_line > 0)
        for_flagged_in_order(eflag, E, [&](int e) {
            int u = edges[e].x, v = edges[e].y;
            collapsed[nm + k++] = e;
            line_collapse(u, v, first_near, near_tris, pts, tris, occ);
        });
    if (threadIdx.x != 0) return;
    cnt->n_line = k;
    cnt->n_total = nm + k;
    int window = ((nm + 511) / 512) * 512;  // grid of the reference's undo-candidate launch
    cnt->n_considered = cnt->n_total < window ? cnt->n_total : window;
}

__global__ void k_mark_active(const int *collapsed, const RoundCounters *cnt, const int2 *edges,
                              const int *first_near, const int *near_tris, uint8_t *active)
{
    const int N = cnt->n_considered;
    PAMO_GRID_STRIDE(p, N)
    {
        int2 ed = edges[collapsed[p]];
        for (int a = first_near[ed.x]; a < first_near[ed.x + 1]; ++a) active[near_tris[a]] = 1;
        for (int a = first_near[ed.y]; a < first_near[ed.y + 1]; ++a) active[near_tris[a]] = 1;
    }
}

constexpr int kStack = 96;

__device__ __forceinline__ bool box_overlap(float4 alo, float4 ahi, float3 qlo, float3 qhi)
{
    return !(ahi.x < qlo.x || qhi.x < alo.x || ahi.y < qlo.y || qhi.y < alo.y || ahi.z < qlo.z || qhi.z < alo.z);
}

__device__ __forceinline__ int shared_indices(int4 a, int4 b)
{
    return (a.x == b.x) + (a.x == b.y) + (a.x == b.z) + (a.y == b.x) + (a.y == b.y) + (a.y == b.z) +
           (a.z == b.x) + (a.z == b.y) + (a.z == b.z);
}

// The active live faces in leaf (Morton) order, appended a warp at a time, so
// the query threads that follow all have a face and neighbouring lanes walk
// neighbouring paths.  In a batch, only the faces of meshes whose undo loop
// still runs (a mesh whose last check found nothing would find nothing again
// on its unchanged geometry, and pairs never cross meshes).
__global__ void k_active_list(const int *__restrict__ vals, const int *scene, const uint8_t *__restrict__ active,
                              const int4 *__restrict__ tris, int *qlist, RoundCounters *cnt, const SlotInfo *slots,
                              const int *vslot)
{
    const int L = scene[7];
    const int lane = threadIdx.x & 31;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < L; base += (long long)blockDim.x * gridDim.x) {
        const long long p = base + threadIdx.x;
        int f = p < L ? vals[p] : -1;
        bool ok = f >= 0 && active[f];
        if (ok) {
            const int v0 = tris[f].x;
            ok = v0 != -1 && (!slots || slots[vslot[v0]].in_undo);
        }
        unsigned ball = __ballot_sync(0xffffffffu, ok);
        int first = 0;
        if (lane == 0 && ball) first = atomicAdd(&cnt->n_query, __popc(ball));
        first = __shfl_sync(0xffffffffu, first, 0);
        if (ok) qlist[first + __popc(ball & ((1u << lane) - 1u))] = f;
    }
}

// For each active live face, enumerate overlapping leaves and append candidate
// pairs.  A pair of two active faces is emitted once (by the lower index);
// pairs sharing `skip_shared` or more vertex indices are dropped: 2 for the
// reference's test, which never reports pairs sharing an edge; 4 (none) for
// the exact test of quality mode.
__global__ void __launch_bounds__(kThreads) k_query(const BvhNode *__restrict__ nodes, const int *__restrict__ vals,
                                                    const int *scene, const float4 *__restrict__ pts,
                                                    const int4 *__restrict__ tris, const uint8_t *__restrict__ active,
                                                    int m, uint2 *pairs, long long cap_pairs, RoundCounters *cnt,
                                                    const int *roots, const int *vslot, const int *qlist,
                                                    int skip_shared)
{
    const int L = scene[7];
    int stack[kStack];
    // queries from the list of active faces (k_active_list), or every leaf in
    // leaf order with the inactive ones skipped
    const int N = qlist ? cnt->n_query : L;
    PAMO_GRID_STRIDE(pp, N)
    {
        const int f = qlist ? qlist[pp] : vals[pp];
        if (f < 0 || !active[f] || L < 2) continue;
        int4 t = tris[f];
        if (t.x == -1) continue;
        float4 a = pts[t.x], b = pts[t.y], c = pts[t.z];
        float3 qlo = make_float3(fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)), fminf(a.z, fminf(b.z, c.z)));
        float3 qhi = make_float3(fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)), fmaxf(a.z, fmaxf(b.z, c.z)));
        // a batch starts at the face's own mesh subtree (a leaf: a one-face mesh)
        const int start = roots ? roots[vslot[t.x]] : 0;
        if (start < 0) continue;
        int sp = 0;
        stack[sp++] = start;
        // a tree visits each of its L-1 inner nodes at most once per query; the
        // bound only guards against a corrupted hierarchy
        int budget = 2 * L + 16;
        while (sp > 0) {
            if (--budget < 0) {
                atomicAdd(&cnt->stack_overflow, 1);
                break;
            }
            const BvhNode nd = nodes[stack[--sp]];
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                float4 lo = side ? nd.rlo : nd.llo;
                float4 hi = side ? nd.rhi : nd.lhi;
                if (!box_overlap(lo, hi, qlo, qhi)) continue;
                int child = __float_as_int(lo.w);
                if (child < 0) {
                    int g = vals[~child];
                    if (g < 0 || g == f) continue;  // empty leaves have empty boxes; guard anyway
                    if (active[g] && g < f) continue;
                    int4 tg = tris[g];
                    if (shared_indices(t, tg) >= skip_shared) continue;
                    // one atomic per group of lanes appending together
                    cg::coalesced_group grp = cg::coalesced_threads();
                    int base = 0;
                    if (grp.thread_rank() == 0) base = atomicAdd(&cnt->n_pairs, (int)grp.size());
                    int pos = grp.shfl(base, 0) + (int)grp.thread_rank();
                    if (pos < cap_pairs) pairs[pos] = make_uint2((unsigned)f, (unsigned)g);
                    else atomicAdd(&cnt->pair_overflow, 1);
                } else if (sp < kStack) {
                    stack[sp++] = child;
                } else {
                    atomicAdd(&cnt->stack_overflow, 1);
                }
            }
        }
    }
}

__device__ __forceinline__ void load_face(const float4 *pts, int4 t, float out[3][3], int idx[3])
{
    idx[0] = t.x; idx[1] = t.y; idx[2] = t.z;
    float4 p[3] = {pts[t.x], pts[t.y], pts[t.z]};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        out[a][0] = p[a].x; out[a][1] = p[a].y; out[a][2] = p[a].z;
    }
}

template <bool EXACT>
__global__ void __launch_bounds__(kThreads) k_pairs(const uint2 *pairs, const RoundCounters *cnt,
                                                    long long cap_pairs, const float4 *__restrict__ pts,
                                                    const int4 *__restrict__ tris, uint8_t *isect, float eps)
{
    long long N = cnt->n_pairs < cap_pairs ? cnt->n_pairs : cap_pairs;
    PAMO_GRID_STRIDE(k, N)
    {
        uint2 pr = pairs[k];
        if constexpr (EXACT) {
            // quality mode: the acceptance checker's exact predicate (exact.cuh);
            // a degenerate face counts as intersecting
            exact::P3 P[3], Q[3];
            const int4 ta = tris[pr.x], tb = tris[pr.y];
            const int ia[3] = {ta.x, ta.y, ta.z}, ib[3] = {tb.x, tb.y, tb.z};
            for (int c = 0; c < 3; ++c) {
                const float4 a = pts[ia[c]], b = pts[ib[c]];
                P[c] = {a.x, a.y, a.z};
                Q[c] = {b.x, b.y, b.z};
            }
            const bool da = exact::tri_degenerate(P, ia), db = exact::tri_degenerate(Q, ib);
            if (da) isect[pr.x] = 1;
            if (db) isect[pr.y] = 1;
            if (!da && !db && exact::faces_intersect(P, ia, Q, ib)) {
                isect[pr.x] = 1;
                isect[pr.y] = 1;
            }
            continue;
        }
        float A[3][3], B[3][3];
        int ia[3], ib[3];
        load_face(pts, tris[pr.x], A, ia);
        load_face(pts, tris[pr.y], B, ib);
        if (pair_flag_directed(A, ia, B, ib, eps) || pair_flag_directed(B, ib, A, ia, eps)) {
            isect[pr.x] = 1;
            isect[pr.y] = 1;
        }
    }
}

__global__ void k_undo_flags(const int *collapsed, const RoundCounters *cnt, const int2 *edges,
                             const int *first_near, const int *near_tris, const uint8_t *isect, int *uflag)
{
    const int N = cnt->n_considered;
    PAMO_GRID_STRIDE(p, N)
    {
        int2 ed = edges[collapsed[p]];
        int hit = 0;
        for (int a = first_near[ed.x]; a < first_near[ed.x + 1] && !hit; ++a) hit = isect[near_tris[a]];
        for (int a = first_near[ed.y]; a < first_near[ed.y + 1] && !hit; ++a) hit = isect[near_tris[a]];
        uflag[p] = hit;
    }
}

__global__ void k_undo_scatter(const int *uflag, const int *upos, const RoundCounters *cnt, const int *collapsed,
                               const int2 *edges, int *undo_edges, int *tmp_undo)
{
    const int N = cnt->n_considered;
    PAMO_GRID_STRIDE(p, N)
    {
        if (!uflag[p]) continue;
        int k = upos[p];
        int e = collapsed[p];
        int2 ed = edges[e];
        undo_edges[k] = e;
        tmp_undo[2 * k] = ed.x;
        tmp_undo[2 * k + 1] = ed.y;
    }
}

__global__ void k_undo_apply(const int *undo_edges, const RoundCounters *cnt, const int2 *edges,
                             const int *first_near, const int *near_tris, const float4 *opts, const int4 *otris,
                             float4 *pts, int4 *tris, int *occ)
{
    const int N = cnt->n_undo;
    PAMO_GRID_STRIDE(k, N)
    {
        int2 ed = edges[undo_edges[k]];
        int u = ed.x, v = ed.y;
        occ[v] = 1;
        pts[u] = opts[u];
        pts[v] = opts[v];
        for (int a = first_near[u]; a < first_near[u + 1]; ++a) tris[near_tris[a]] = otris[near_tris[a]];
        for (int a = first_near[v]; a < first_near[v + 1]; ++a) tris[near_tris[a]] = otris[near_tris[a]];
    }
}

// undo_list[first + i] = pts_map[tmp_undo[i]]: the map in pts_map at this point is
// the previous round's (cusimp_free.cu:869-878 runs before :1042-1045).
__global__ void k_rearrange(const int *tmp_undo, const int *pts_map, int *undo_list, int first, int count)
{
    PAMO_GRID_STRIDE(i, count) undo_list[first + i] = pts_map[tmp_undo[i]];
}

__global__ void k_mark_invalid(const int *undo_in, int n, uint8_t *table)
{
    PAMO_GRID_STRIDE(i, n) table[undo_in[i]] = 1;
}

__global__ void k_face_live_flags(const int4 *tris, int m, int *fflag)
{
    PAMO_GRID_STRIDE(f, m) fflag[f] = tris[f].x >= 0;
}

__global__ void k_compact(const float4 *pts, const int *occ, const int *pts_map, int n, const int4 *tris,
                          const int *fflag, const int *fpos, int m, float4 *opts, int4 *otris, RoundCounters *cnt)
{
    long long N = n > m ? n : m;
    PAMO_GRID_STRIDE(i, N)
    {
        if (i < n && occ[i]) opts[pts_map[i]] = pts[i];
        if (i < m && fflag[i]) {
            int4 t = tris[i];
            otris[fpos[i]] = make_int4(pts_map[t.x], pts_map[t.y], pts_map[t.z], 0);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        cnt->n_pts_next = pts_map[n];
        cnt->n_tris_next = fpos[m - 1 >= 0 ? m - 1 : 0] + (m > 0 ? fflag[m - 1] : 0);
    }
}

// After compaction: leaf p's face gets its compacted index, or -1 if removed
// (every surviving face is a leaf, so leaf_of_face is complete again).
__global__ void k_remap_leaves(int *vals, const int *scene, const int *fflag, const int *fpos, int *leaf_of_face)
{
    const int L = scene[7];
    PAMO_GRID_STRIDE(p, L)
    {
        int f = vals[p];
        int nf = (f >= 0 && fflag[f]) ? fpos[f] : -1;
        vals[p] = nf;
        if (nf >= 0) leaf_of_face[nf] = (int)p;
    }
}

// Leaves whose boxes changed since the last refit: the faces of the one-rings of
// the listed edges (collapses, coincident-endpoint collapses and undos only
// change those faces and their vertices).
__global__ void k_mark_dirty(const int *elist, const int *n_list, const int2 *edges, const int *first_near,
                             const int *near_tris, const int *leaf_of_face, const int *parent, int *claim,
                             int *dmask, int *dlist, int *scene)
{
    const int N = *n_list;
    const int L = scene[7];
    if (L < 2) return;
    PAMO_GRID_STRIDE(k, N)
    {
        const int2 ed = edges[elist[k]];
        for (int side = 0; side < 2; ++side) {
            const int w = side ? ed.y : ed.x;
            for (int a = first_near[w]; a < first_near[w + 1]; ++a) {
                const int p = leaf_of_face[near_tris[a]];
                if (p >= 0) lbvh_mark_dirty_leaf(p, L, parent, claim, dmask, dlist, scene);
            }
        }
    }
}

__global__ void k_validate_faces(const int *tris, int m, int n, int *bad)
{
    int local = 0;
    PAMO_GRID_STRIDE(f, m)
    {
        int a = tris[3 * f], b = tris[3 * f + 1], c = tris[3 * f + 2];
        bool dead = a == -1 && b == -1 && c == -1;
        bool ok = a >= 0 && a < n && b >= 0 && b < n && c >= 0 && c < n;
        local += !(dead || ok);
    }
    if (local) atomicAdd(bad, local);
}

__global__ void k_validate_range(const int *v, int count, int hi, int *bad)
{
    int local = 0;
    PAMO_GRID_STRIDE(i, count) local += (v[i] < 0 || v[i] > hi);
    if (local) atomicAdd(bad, local);
}

// ---------------------------------------------------------------------------
// Batch kernels.  Per-mesh loops use blockIdx.y = the mesh's rank and stride
// over the mesh's range with blockIdx.x.
#define SLOT_STRIDE(j, count) \
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < (long long)(count); j += (long long)blockDim.x * gridDim.x)

// Before the round, per mesh, as the single-mesh round does (cusimp_free.cu:899-916):
// stuck: the undo list starts with the previous one mapped through the previous
// vertex map; not stuck with a non-empty list: the invalid table is cleared.
__global__ void k_b_pre_copy(const SlotInfo *slots)
{
    const SlotInfo S = slots[blockIdx.y];
    if (S.is_stuck) {
        SLOT_STRIDE(j, S.n_undo_in)
        {
            int x = S.undo_prev[j];
            S.tmp_undo[j] = x;
            S.undo_list[j] = S.pts_map[x];
        }
    } else if (S.clear_invalid) {
        SLOT_STRIDE(j, S.cap_v) S.invalid[j] = 0;
    }
}

__global__ void k_b_pre_mark(const SlotInfo *slots)
{
    const SlotInfo S = slots[blockIdx.y];
    SLOT_STRIDE(j, S.n_undo_in) S.invalid[S.undo_prev[j]] = 1;
}

__global__ void k_b_vslot(const SlotInfo *slots, int *vslot)
{
    const SlotInfo S = slots[blockIdx.y];
    SLOT_STRIDE(j, S.n) vslot[S.vert_off + j] = (int)blockIdx.y;
}

// first packed edge and edge count of each mesh (first_edge has m + 1 entries)
__global__ void k_b_edge_off(const SlotInfo *slots, const int *first_edge, SlotCounters *scnt, int K)
{
    PAMO_GRID_STRIDE(r, K)
    {
        const SlotInfo &S = slots[r];
        scnt[r].edge_off = first_edge[S.face_off];
        scnt[r].n_edges = first_edge[S.face_off + S.m] - first_edge[S.face_off];
    }
}

// pos = exclusive scan over the packed edges of a flag, total = its sum:
// each mesh's first entry and count in the compacted list.
__device__ __forceinline__ void seg_of_scan(const int *pos, int total, int n_all, int first, int count, int &off,
                                            int &cnt)
{
    off = first < n_all ? pos[first] : total;
    int end = first + count < n_all ? pos[first + count] : total;
    cnt = end - off;
}

__global__ void k_b_main(const int *pos, const RoundCounters *cnt, SlotCounters *scnt, int K)
{
    PAMO_GRID_STRIDE(r, K)
    {
        int off, c;
        seg_of_scan(pos, cnt->n_main, cnt->n_edges, scnt[r].edge_off, scnt[r].n_edges, off, c);
        scnt[r].main_off = off;
        scnt[r].n_main = c;
    }
}

// Coincident-endpoint collapses over the whole batch (the single-mesh version's
// order: positions read before any write, writes in edge order), and each
// mesh's undo-candidate window: its collapsed edges then its coincident ones,
// cut at the reference's launch-grid roundup of its own collapsed count.
__global__ void __launch_bounds__(kLineThreads) k_b_line_apply(const int2 *edges, const int *n_edges,
                                                               const int *eflag, const int *first_near,
                                                               const int *near_tris, float4 *pts, int4 *tris, int *occ,
                                                               int *line_list, const int *vslot, RoundCounters *cnt,
                                                               SlotCounters *scnt, int K)
{
    const int E = *n_edges;
    for (int r = threadIdx.x; r < K; r += blockDim.x) scnt[r].n_line = 0;
    __syncthreads();
    int k = 0;
    if (cnt->n_line > 0)
        for_flagged_in_order(eflag, E, [&](int e) {
            int u = edges[e].x, v = edges[e].y;
            line_list[k++] = e;
            scnt[vslot[u]].n_line++;
            line_collapse(u, v, first_near, near_tris, pts, tris, occ);
        });
    if (threadIdx.x != 0) return;
    cnt->n_line = k;
    cnt->n_total = cnt->n_main + k;
    int line_off = 0, cand_off = 0;
    for (int r = 0; r < K; ++r) {
        SlotCounters &c = scnt[r];
        c.line_off = line_off;
        line_off += c.n_line;
        int total = c.n_main + c.n_line;
        int window = ((c.n_main + 511) / 512) * 512;
        c.n_considered = total < window ? total : window;
        c.cand_off = cand_off;
        cand_off += c.n_considered;
    }
    cnt->n_considered = cand_off;
}

__global__ void k_b_cand_fill(const int *collapsed, const int *line_list, const int2 *edges, const int *vslot,
                              const RoundCounters *cnt, const SlotCounters *scnt, int *cand)
{
    const int nm = cnt->n_main, nl = cnt->n_line;
    PAMO_GRID_STRIDE(p, (long long)nm + nl)
    {
        int e, r, k;
        if (p < nm) {
            e = collapsed[p];
            r = vslot[edges[e].x];
            k = (int)p - scnt[r].main_off;
        } else {
            int q = (int)p - nm;
            e = line_list[q];
            r = vslot[edges[e].x];
            k = scnt[r].n_main + q - scnt[r].line_off;
        }
        if (k < scnt[r].n_considered) cand[scnt[r].cand_off + k] = e;
    }
}

__global__ void k_b_undo_counts(const int *upos, const RoundCounters *cnt, SlotCounters *scnt, int K)
{
    PAMO_GRID_STRIDE(r, K)
    {
        int off, c;
        seg_of_scan(upos, cnt->n_undo, cnt->n_considered, scnt[r].cand_off, scnt[r].n_considered, off, c);
        scnt[r].undo_off = off;
        scnt[r].n_undo = c;
    }
}

// undo edges (packed) and each mesh's undo vertices (mesh-local numbers)
__global__ void k_b_undo_scatter(const int *uflag, const int *upos, const RoundCounters *cnt, const int *cand,
                                 const int2 *edges, const int *vslot, const SlotInfo *slots,
                                 const SlotCounters *scnt, int *undo_edges)
{
    const int N = cnt->n_considered;
    PAMO_GRID_STRIDE(p, N)
    {
        if (!uflag[p]) continue;
        int k = upos[p];
        int e = cand[p];
        int2 ed = edges[e];
        undo_edges[k] = e;
        int r = vslot[ed.x];
        const SlotInfo &S = slots[r];
        int j = k - scnt[r].undo_off;
        S.tmp_undo[2 * j] = ed.x - S.vert_off;
        S.tmp_undo[2 * j + 1] = ed.y - S.vert_off;
    }
}

// undo_list[first + j] = pts_map[tmp_undo[j]] per mesh (the previous round's map)
__global__ void k_b_rearrange(const SlotInfo *slots)
{
    const SlotInfo S = slots[blockIdx.y];
    SLOT_STRIDE(j, S.pass_count) S.undo_list[S.pass_first + j] = S.pts_map[S.tmp_undo[j]];
}

// each mesh's vertex map in its own numbers, and the copy of its undo list
__global__ void k_b_local_map(const SlotInfo *slots, const int *gmap)
{
    const SlotInfo S = slots[blockIdx.y];
    const int base = gmap[S.vert_off];
    SLOT_STRIDE(j, (long long)S.n + 1) S.pts_map[j] = gmap[S.vert_off + j] - base;
    SLOT_STRIDE(j, S.nvu) S.undo_prev[j] = S.undo_list[j];
}

__global__ void k_b_next(const SlotInfo *slots, const int *gmap, const int *fpos, SlotCounters *scnt, int K)
{
    PAMO_GRID_STRIDE(r, K)
    {
        const SlotInfo &S = slots[r];
        scnt[r].vert_off_next = gmap[S.vert_off];
        scnt[r].n_next = gmap[S.vert_off + S.n] - gmap[S.vert_off];
        scnt[r].face_off_next = fpos[S.face_off];
        scnt[r].m_next = fpos[S.face_off + S.m] - fpos[S.face_off];
    }
}

}  // namespace

void Profiler::begin(int phase, cudaStream_t s)
{
    if (!on) return;
    if (open_phase >= 0) end(s);
    if (used + 2 > kPool || n_marks >= kPool / 2) return;  // pool full: drop (collect() frees it)
    for (int k = 0; k < 2; ++k)
        if (!ev[used + k]) cudaEventCreate(&ev[used + k]);
    cudaEventRecord(ev[used], s);
    marks[n_marks][0] = phase;
    marks[n_marks][1] = used;
    open_phase = phase;
    used += 2;
}

void Profiler::end(cudaStream_t s)
{
    if (!on || open_phase < 0) return;
    cudaEventRecord(ev[marks[n_marks][1] + 1], s);
    n_marks++;
    open_phase = -1;
}

void Profiler::collect()
{
    if (!on) return;
    for (int i = 0; i < n_marks; ++i) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, ev[marks[i][1]], ev[marks[i][1] + 1]) == cudaSuccess) {
            ms[marks[i][0]] += t;
            calls[marks[i][0]]++;
        }
    }
    if (open_phase >= 0) {  // a phase still open keeps its start event, moved to slot 0
        const int slot = marks[n_marks][1];
        cudaEvent_t a = ev[0], b = ev[1];
        ev[0] = ev[slot];
        ev[1] = ev[slot + 1];
        ev[slot] = a;
        ev[slot + 1] = b;
        marks[0][0] = marks[n_marks][0];
        marks[0][1] = 0;
        used = 2;
    } else {
        used = 0;
    }
    n_marks = 0;
}

void Profiler::reset()
{
    for (int i = 0; i < PH_COUNT; ++i) {
        ms[i] = 0;
        calls[i] = 0;
    }
    n_marks = used = 0;
    open_phase = -1;
}

void Profiler::release()
{
    for (int i = 0; i < kPool; ++i)
        if (ev[i]) {
            cudaEventDestroy(ev[i]);
            ev[i] = nullptr;
        }
}

int Stage2::validate(const int *d_tris, int n, int m, const int *d_undo, int n_undo, int undo_hi, cudaStream_t s)
{
    int *bad = dev_misc + 32;
    S2_TRY_EARLY(cudaMemsetAsync(bad, 0, 4, s));
    if (m > 0) launch(k_validate_faces, grid_for(m), kThreads, 0, s, d_tris, m, n, bad);
    if (n_undo > 0) launch(k_validate_range, grid_for(n_undo), kThreads, 0, s, d_undo, n_undo, undo_hi, bad);
    S2_TRY_EARLY(cudaMemcpyAsync(hcnt, bad, 4, cudaMemcpyDeviceToHost, s));
    S2_TRY_EARLY(cudaStreamSynchronize(s));
    return hcnt->n_main == 0 ? PAMO_OK : PAMO_ERR_INVALID_ARG;
}

// ---------------------------------------------------------------------------
// buffers

void Stage2::release()
{
    void *p[] = {edge_cost, pts_map, undo_list, tmp_undo, invalid_table, opts, pts, otris, tris, occ,
                 first_near, cursor, near_tris, first_edge, edges, plane, elen4, nxt, quad, vmin, eflag, collapsed,
                 active, isect, uflag, undo_edges, fflag, pairs, scan_scratch, dev_misc, dcnt, quad64, epos};
    for (void *q : p)
        if (q) cudaFree(q);
    quad64 = nullptr;
    epos = nullptr;
    cap_q64 = cap_epos = 0;
    if (hcnt) cudaFreeHost(hcnt);
    if (h_scalars) cudaFreeHost(h_scalars);
    prof.release();
    edge_cost = nullptr; pts_map = nullptr; undo_list = nullptr; tmp_undo = nullptr; invalid_table = nullptr;
    opts = pts = nullptr; otris = tris = nullptr; occ = nullptr;
    first_near = cursor = near_tris = first_edge = nullptr; edges = nullptr; plane = quad = elen4 = nullptr;
    nxt = nullptr;
    vmin = nullptr; eflag = collapsed = nullptr; active = isect = nullptr; uflag = undo_edges = fflag = nullptr;
    pairs = nullptr; scan_scratch = nullptr; dev_misc = nullptr; dcnt = nullptr; hcnt = nullptr; h_scalars = nullptr;
    bvh.release();
    bvh_carried = false;
    bvh_leaves = 0;
    bvh_boxes_valid = false;
    cap_pts = cap_tris = cap_edges = cap_undo = cap_pairs = 0;
}

int Stage2::ensure(long long n, long long m)
{
    if (n <= cap_pts && m <= cap_tris && dcnt) return PAMO_OK;
    long long cp = n > cap_pts ? n : cap_pts;
    long long ct = m > cap_tris ? m : cap_tris;
    release();
    cp = cp > 4 ? cp : 4;
    ct = ct > 4 ? ct : 4;
    long long ce = 3 * ct;
    long long cu = 16 * (cp + 1) + 6 * ct + 16;
    long long big = (cp + 1 > ce + 1 ? cp + 1 : ce + 1);
    big = big > ct + 1 ? big : ct + 1;
    scan_scratch_len = scan_scratch_ints(big);
#define ALLOC(ptr, bytes)                                             \
    do {                                                              \
        if (cudaMalloc((void **)&ptr, (size_t)(bytes)) != cudaSuccess) { \
            release();                                                \
            return PAMO_ERR_OOM;                                      \
        }                                                             \
    } while (0)
    ALLOC(edge_cost, (ce + 1) * 4);
    ALLOC(pts_map, (cp + 1) * 4);
    ALLOC(undo_list, cu * 4);
    ALLOC(tmp_undo, cu * 4);
    ALLOC(invalid_table, cp + 1);
    ALLOC(opts, (cp + 1) * 16);
    ALLOC(pts, (cp + 1) * 16);
    ALLOC(otris, (ct + 1) * 16);
    ALLOC(tris, (ct + 1) * 16);
    ALLOC(occ, (cp + 1) * 4);
    ALLOC(first_near, (cp + 1) * 4);
    ALLOC(cursor, (cp + 1) * 4);
    ALLOC(near_tris, 3 * (ct + 1) * 4);
    ALLOC(first_edge, (ct + 1) * 4);
    ALLOC(edges, (ce + 1) * 8);
    ALLOC(plane, (ct + 1) * 16);
    ALLOC(elen4, (ct + 1) * 16);
    ALLOC(nxt, 3 * (ct + 1) * 4);
    ALLOC(quad, 3 * (cp + 1) * 16);
    ALLOC(vmin, (cp + 1) * 8);
    ALLOC(eflag, (ce + 1) * 4);
    ALLOC(collapsed, (ce + 1) * 4);
    ALLOC(active, ct + 1);
    ALLOC(isect, ct + 1);
    ALLOC(uflag, (ce + 1) * 4);
    ALLOC(undo_edges, (ce + 1) * 4);
    ALLOC(fflag, (ct + 1) * 4);
    ALLOC(scan_scratch, scan_scratch_len * 4);
    ALLOC(dev_misc, 256);
    ALLOC(dcnt, sizeof(RoundCounters));
#undef ALLOC
    if (cudaMallocHost((void **)&hcnt, sizeof(RoundCounters)) != cudaSuccess) {
        release();
        return PAMO_ERR_OOM;
    }
    if (cudaMallocHost((void **)&h_scalars, 64) != cudaSuccess) {
        release();
        return PAMO_ERR_OOM;
    }
    scan_scratch_init(scan_scratch, scan_scratch_len);
    // state the reference reads stale starts at zero
    cudaMemset(edge_cost, 0, (ce + 1) * 4);
    cudaMemset(pts_map, 0, (cp + 1) * 4);
    cudaMemset(undo_list, 0, cu * 4);
    cudaMemset(tmp_undo, 0, cu * 4);
    cudaMemset(invalid_table, 0, cp + 1);
    cap_pts = cp;
    cap_tris = ct;
    cap_edges = ce;
    cap_undo = cu;
    if (bvh.ensure(ct) != cudaSuccess) {
        release();
        return PAMO_ERR_OOM;
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return PAMO_ERR_DEVICE;
    return ensure_pairs(16 * ct);
}

int Stage2::ensure_pairs(long long n)
{
    if (n <= cap_pairs && pairs) return PAMO_OK;
    if (pairs) cudaFree(pairs);
    pairs = nullptr;
    cap_pairs = 0;
    if (cudaMalloc((void **)&pairs, (size_t)n * sizeof(uint2)) != cudaSuccess) return PAMO_ERR_OOM;
    cap_pairs = n;
    return PAMO_OK;
}

// ---------------------------------------------------------------------------
// one round

#define S2_TRY(expr)                                  \
    do {                                              \
        cudaError_t _e = (expr);                      \
        if (_e != cudaSuccess) return map_cuda_error(_e); \
    } while (0)

// dirty_edges / n_dirty: when the boxes were up to date before this round's
// changes, the edges whose one-rings changed since (incremental refit);
// otherwise null (full refit).
static cudaError_t isect_pass(Stage2 &S, int m, cudaStream_t s, const int *dirty_edges = nullptr,
                              const int *n_dirty = nullptr)
{
    cudaError_t e;
    if ((e = cudaMemsetAsync(S.isect, 0, (size_t)m, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(&S.dcnt->n_pairs, 0, 2 * sizeof(int), s)) != cudaSuccess) return e;  // n_pairs, overflow
    S.prof.begin(PH_REFIT, s);
    if (dirty_edges && S.bvh_boxes_valid && S.bvh.leaves_built >= 2) {
        if ((e = cudaMemsetAsync(S.bvh.scene + 9, 0, sizeof(int), s)) != cudaSuccess) return e;
        launch(k_mark_dirty, grid_for(3LL * m), kThreads, 0, s, dirty_edges, n_dirty, (const int2 *)S.edges,
               (const int *)S.first_near, (const int *)S.near_tris, (const int *)S.bvh.leaf_of_face,
               (const int *)S.bvh.parent, S.bvh.claim, S.bvh.dmask, S.bvh.dlist, S.bvh.scene);
        if ((e = lbvh_refit_dirty(S.bvh, S.pts, S.tris, S.bvh.leaves_built, s)) != cudaSuccess) return e;
    } else {
        if ((e = lbvh_refit(S.bvh, S.pts, S.tris, m, s)) != cudaSuccess) return e;
    }
    S.bvh_boxes_valid = true;
    S.prof.begin(PH_QUERY, s);
    const bool batch = S.n_slots > 0;
    if ((e = cudaMemsetAsync(&S.dcnt->n_query, 0, sizeof(int), s)) != cudaSuccess) return e;
    launch(k_active_list, grid_for(m), kThreads, 0, s, (const int *)S.bvh.vals, (const int *)S.bvh.scene,
           (const uint8_t *)S.active, (const int4 *)S.tris, S.fflag, S.dcnt,
           batch ? (const SlotInfo *)S.slots : nullptr, batch ? (const int *)S.vslot : nullptr);
    launch(k_query, grid_for(m), kThreads, 0, s, (const BvhNode *)S.bvh.nodes, (const int *)S.bvh.vals,
           (const int *)S.bvh.scene, (const float4 *)S.pts, (const int4 *)S.tris, (const uint8_t *)S.active, m,
           S.pairs, S.cap_pairs, S.dcnt, batch ? (const int *)S.roots : nullptr,
           batch ? (const int *)S.vslot : nullptr, (const int *)S.fflag, S.quality ? 4 : 2);
    S.prof.begin(PH_PAIRS, s);
    if (S.quality)
        launch(k_pairs<true>, grid_for(S.cap_pairs), kThreads, 0, s, S.pairs, S.dcnt, S.cap_pairs, S.pts, S.tris,
               S.isect, 1e-3f);
    else
        launch(k_pairs<false>, grid_for(S.cap_pairs), kThreads, 0, s, S.pairs, S.dcnt, S.cap_pairs, S.pts, S.tris,
               S.isect, 1e-3f);
    S.prof.end(s);
    return cudaGetLastError();
}

static cudaError_t undo_check(Stage2 &S, cudaStream_t s)
{
    S.prof.begin(PH_UNDO, s);
    const long long NC = S.cap_edges;
    launch(k_undo_flags, grid_for(NC), kThreads, 0, s, S.collapsed, S.dcnt, S.edges, S.first_near, S.near_tris, S.isect,
                                                   S.uflag);
    // positions of the flagged entries (in collapsed-list order)
    cudaError_t e = exclusive_scan(S.uflag, S.eflag, NC, &S.dcnt->n_considered, S.scan_scratch, &S.dcnt->n_undo, s, &S.dcnt->scan_fault);
    if (e != cudaSuccess) return e;
    launch(k_undo_scatter, grid_for(NC), kThreads, 0, s, S.uflag, S.eflag, S.dcnt, S.collapsed, S.edges, S.undo_edges,
                                                     S.tmp_undo);
    S.prof.end(s);
    return cudaGetLastError();
}

int Stage2::round(int n, int m, float scale, float threshold, bool is_stuck, const int *d_undo_in, int n_undo_in,
                  int *n_undo_out, cudaStream_t s, bool keep_bvh)
{
    int nvu = 0, first = 0;
    S2_TRY(cudaMemsetAsync(dcnt, 0, sizeof(RoundCounters), s));
    if (is_stuck) {
        if (n_undo_in > 0) {
            S2_TRY(cudaMemcpyAsync(tmp_undo, d_undo_in, (size_t)n_undo_in * 4, cudaMemcpyDeviceToDevice, s));
            launch(k_rearrange, grid_for(n_undo_in), kThreads, 0, s, tmp_undo, pts_map, undo_list, 0, n_undo_in);
        }
        nvu += n_undo_in;
        first += n_undo_in;
    } else if (n_undo_in != 0) {
        S2_TRY(cudaMemsetAsync(invalid_table, 0, (size_t)cap_pts + 1, s));
    }
    if (n_undo_in > 0) launch(k_mark_invalid, grid_for(n_undo_in), kThreads, 0, s, d_undo_in, n_undo_in, invalid_table);

    const float tres = threshold, edge_s = scale;
    // host-side conversion as in the reference (cusimp_free.cu:923): the
    // template clamp, then float -> u32 keeping the low 32 bits when out of range
    float ct = (0.0f > threshold) ? 0.0f : threshold;
    ct = (ct < kCostRange) ? ct : kCostRange;
    const uint32_t collapse_t = (uint32_t)(unsigned long long)(ct / kCostRange * 4294967296.0f);

    prof.begin(PH_SETUP, s);
    launch(k_round_init, grid_for((n + 1 > m ? n + 1 : m)), kThreads, 0, s, opts, otris, pts, tris, occ, first_near,
                                                                       cursor, vmin, n, m);
    launch(k_face_a, grid_for(m), kThreads, 0, s, pts, tris, m, first_near, first_edge, plane, elen4);
    if (m > 0) S2_TRY(cudaMemsetAsync(first_edge + m, 0, 4, s));
    S2_TRY(exclusive_scan(first_near, first_near, (long long)n + 1, nullptr, scan_scratch, nullptr, s, &dcnt->scan_fault));
    S2_TRY(exclusive_scan(first_edge, first_edge, (long long)m + 1, nullptr, scan_scratch, &dcnt->n_edges, s, &dcnt->scan_fault));
    const int *d_n_edges = &dcnt->n_edges;
    launch(k_face_b, grid_for(m), kThreads, 0, s, tris, m, first_near, cursor, near_tris, first_edge, edges);
    launch(k_vertex_quadric, grid_for(n), kThreads, 0, s, first_near, near_tris, plane, tris, quad, nxt, n);
    if (quality) {
        int rc = ensure_quality(n, 3LL * m);
        if (rc) return rc;
        launch(k_vertex_quadric64, grid_for(n), kThreads, 0, s, (const int *)first_near, (const int *)near_tris,
               (const float4 *)pts, (const int4 *)tris, quad64, n);
    }
    // The hierarchy only needs the round input's faces as leaves: build it, or
    // keep the previous round's (leaves renumbered by compact(), removed faces
    // as empty leaves) while at least kRebuildFraction of its leaves are faces.
    // Queries find every overlapping leaf whatever the tree, so the pairs found
    // do not depend on this choice; the refit before each query sets the boxes.
    prof.begin(PH_LBVH_BUILD, s);
    if (!(keep_bvh && bvh_carried && m <= bvh_leaves && (double)m >= kRebuildFraction * (double)bvh_leaves)) {
        S2_TRY(lbvh_build(bvh, pts, tris, m, s));
        bvh_leaves = m;
        bvh_boxes_valid = false;
    }
    bvh_carried = false;

    const long long EMAX = 3LL * m;
    prof.begin(PH_EDGE_COST, s);
    CostArgs ca{edges, d_n_edges, pts, tris, first_near, near_tris, nxt, plane, elen4, quad, invalid_table,
                edge_cost, vmin, tres, edge_s, is_stuck ? 1 : 0, nullptr, nullptr, nullptr,
                quality ? (const double *)quad64 : nullptr, quality ? epos : nullptr};
    if (quality)
        launch(k_edge_cost<true>, grid_for(m, kChunkFaces), kThreads, 0, s, ca, bvh.vals, bvh.scene, first_edge);
    else
        launch(k_edge_cost<false>, grid_for(m, kChunkFaces), kThreads, 0, s, ca, bvh.vals, bvh.scene, first_edge);
    CollapseArgs cl{edges, d_n_edges, edge_cost, vmin, first_near, near_tris, opts, otris, pts, tris, occ, eflag,
                    collapse_t, nullptr, nullptr, nullptr, quality ? (const float4 *)epos : nullptr};
    prof.begin(PH_COLLAPSE, s);
    launch(k_collapse, grid_for(EMAX), kThreads, 0, s, cl);
    S2_TRY(exclusive_scan(eflag, uflag, EMAX, d_n_edges, scan_scratch, &dcnt->n_main, s, &dcnt->scan_fault));
    launch(k_scatter_flagged, grid_for(EMAX), kThreads, 0, s, eflag, uflag, d_n_edges, collapsed, 0);
    if (quality)
        launch(k_collapse_apply<true>, grid_for(EMAX), kThreads, 0, s, cl, (const int *)collapsed,
               (const int *)&dcnt->n_main);
    else
        launch(k_collapse_apply<false>, grid_for(EMAX), kThreads, 0, s, cl, (const int *)collapsed,
               (const int *)&dcnt->n_main);
    prof.begin(PH_CLEANUP, s);
    launch(k_remove_invalid_faces, grid_for(m), kThreads, 0, s, tris, m);
    launch(k_line_flags, grid_for(EMAX), kThreads, 0, s, edges, d_n_edges, pts, eflag, &dcnt->n_line);
    launch(k_line_apply, 1, kLineThreads, 0, s, edges, d_n_edges, eflag, first_near, near_tris, pts, tris, occ, collapsed,
           dcnt);

    S2_TRY(cudaMemsetAsync(active, 0, (size_t)m, s));
    launch(k_mark_active, grid_for(EMAX), kThreads, 0, s, collapsed, dcnt, edges, first_near, near_tris, active);
    // a full refit: the collapses change too many leaves for the incremental one to pay
    S2_TRY(isect_pass(*this, m, s));
    S2_TRY(undo_check(*this, s));
    S2_TRY(cudaMemcpyAsync(hcnt, dcnt, sizeof(RoundCounters), cudaMemcpyDeviceToHost, s));
    S2_TRY(cudaStreamSynchronize(s));
    prof.collect();
    if (hcnt->pair_overflow > 0) {
        // candidate buffer too small: grow and redo the pass
        long long need = (long long)hcnt->n_pairs + hcnt->n_pairs / 2 + 1024;
        int rc = ensure_pairs(need);
        if (rc) return rc;
        S2_TRY(isect_pass(*this, m, s));
        S2_TRY(undo_check(*this, s));
        S2_TRY(cudaMemcpyAsync(hcnt, dcnt, sizeof(RoundCounters), cudaMemcpyDeviceToHost, s));
        S2_TRY(cudaStreamSynchronize(s));
        if (hcnt->pair_overflow > 0) return PAMO_ERR_CAPACITY;
    }
    if (hcnt->stack_overflow > 0) return PAMO_ERR_CAPACITY;
    if (hcnt->scan_fault) return PAMO_ERR_DEVICE;
    last_stats[0] = hcnt->n_edges;
    last_stats[1] = hcnt->n_main;
    last_stats[2] = hcnt->n_total;
    last_stats[5] = hcnt->n_pairs;
    last_stats[6] = m;
    int cnt_undo = hcnt->n_undo;
    nvu += 2 * cnt_undo;
    if (nvu > cap_undo) return PAMO_ERR_CAPACITY;
    int it = 0;
    while (cnt_undo != 0) {
        it++;
        prof.begin(PH_UNDO, s);
        launch(k_undo_apply, grid_for(cnt_undo), kThreads, 0, s, undo_edges, dcnt, edges, first_near, near_tris, opts,
                                                              otris, pts, tris, occ);
        if (nvu - first > 0)
            launch(k_rearrange, grid_for(nvu - first), kThreads, 0, s, tmp_undo, pts_map, undo_list, first, nvu - first);
        first += 2 * cnt_undo;
        S2_TRY(isect_pass(*this, m, s, undo_edges, &dcnt->n_undo));  // only the undone one-rings changed
        S2_TRY(undo_check(*this, s));
        S2_TRY(cudaMemcpyAsync(hcnt, dcnt, sizeof(RoundCounters), cudaMemcpyDeviceToHost, s));
        S2_TRY(cudaStreamSynchronize(s));
        prof.collect();
        if (hcnt->pair_overflow > 0) {
            long long need = (long long)hcnt->n_pairs + hcnt->n_pairs / 2 + 1024;
            int rc = ensure_pairs(need);
            if (rc) return rc;
            S2_TRY(isect_pass(*this, m, s, undo_edges, &dcnt->n_undo));
            S2_TRY(undo_check(*this, s));
            S2_TRY(cudaMemcpyAsync(hcnt, dcnt, sizeof(RoundCounters), cudaMemcpyDeviceToHost, s));
            S2_TRY(cudaStreamSynchronize(s));
            if (hcnt->pair_overflow > 0) return PAMO_ERR_CAPACITY;
        }
        if (hcnt->stack_overflow > 0) return PAMO_ERR_CAPACITY;
    if (hcnt->scan_fault) return PAMO_ERR_DEVICE;
        cnt_undo = hcnt->n_undo;
        nvu += 2 * cnt_undo;
        if (nvu > cap_undo) return PAMO_ERR_CAPACITY;
        if (it == 5) break;
    }
    last_stats[3] = it;
    last_stats[4] = nvu;
    // pts_map = exclusive scan of occ[0..n]
    prof.begin(PH_COMPACT, s);
    S2_TRY(exclusive_scan(occ, pts_map, (long long)n + 1, nullptr, scan_scratch, nullptr, s, &dcnt->scan_fault));
    prof.end(s);
    *n_undo_out = nvu;
    return PAMO_OK;
}

cudaError_t query_and_test_pairs(const BvhNode *nodes, const int *vals, const int *scene, const float4 *pts,
                                 const int4 *tris, const uint8_t *active, int m, uint2 *pairs, long long cap_pairs,
                                 RoundCounters *cnt, uint8_t *isect, cudaStream_t s)
{
    launch(k_query, grid_for(m), kThreads, 0, s, nodes, vals, scene, pts, tris, active, m, pairs, cap_pairs, cnt,
           (const int *)nullptr, (const int *)nullptr, (const int *)nullptr, 2);
    launch(k_pairs<false>, grid_for(cap_pairs), kThreads, 0, s, pairs, cnt, cap_pairs, pts, tris, isect, 1e-3f);
    return cudaGetLastError();
}

int Stage2::ensure_quality(long long n_pts, long long n_edges)
{
    if (n_pts > cap_q64 || !quad64) {
        if (quad64) cudaFree(quad64);
        quad64 = nullptr;
        cap_q64 = 0;
        const long long c = n_pts > cap_pts ? n_pts : cap_pts;
        if (cudaMalloc((void **)&quad64, (size_t)(c + 1) * 10 * sizeof(double)) != cudaSuccess) return PAMO_ERR_OOM;
        cap_q64 = c;
    }
    if (n_edges > cap_epos || !epos) {
        if (epos) cudaFree(epos);
        epos = nullptr;
        cap_epos = 0;
        const long long c = n_edges > cap_edges ? n_edges : cap_edges;
        if (cudaMalloc((void **)&epos, (size_t)(c + 1) * sizeof(float4)) != cudaSuccess) return PAMO_ERR_OOM;
        cap_epos = c;
    }
    return PAMO_OK;
}

int Stage2::self_intersect_all(int n, int m, cudaStream_t s)
{
    bvh_carried = false;
    bvh_leaves = 0;
    // faces of opts/otris; every live face queries the hierarchy
    launch(k_round_init, grid_for((n + 1 > m ? n + 1 : m)), kThreads, 0, s, opts, otris, pts, tris, occ, first_near,
                                                                       cursor, vmin, n, m);
    S2_TRY(cudaMemsetAsync(dcnt, 0, sizeof(RoundCounters), s));
    S2_TRY(cudaMemsetAsync(active, 1, (size_t)m, s));
    S2_TRY(lbvh_build(bvh, pts, tris, m, s));
    bvh_boxes_valid = false;
    S2_TRY(isect_pass(*this, m, s));
    S2_TRY(cudaMemcpyAsync(hcnt, dcnt, sizeof(RoundCounters), cudaMemcpyDeviceToHost, s));
    S2_TRY(cudaStreamSynchronize(s));
    if (hcnt->pair_overflow > 0) {
        long long need = (long long)hcnt->n_pairs + hcnt->n_pairs / 2 + 1024;
        int rc = ensure_pairs(need);
        if (rc) return rc;
        S2_TRY(isect_pass(*this, m, s));
        S2_TRY(cudaMemcpyAsync(hcnt, dcnt, sizeof(RoundCounters), cudaMemcpyDeviceToHost, s));
        S2_TRY(cudaStreamSynchronize(s));
        if (hcnt->pair_overflow > 0) return PAMO_ERR_CAPACITY;
    }
    if (hcnt->stack_overflow > 0) return PAMO_ERR_CAPACITY;
    if (hcnt->scan_fault) return PAMO_ERR_DEVICE;
    return PAMO_OK;
}

int Stage2::compact(int n, int m, cudaStream_t s)
{
    prof.begin(PH_COMPACT, s);
    launch(k_face_live_flags, grid_for(m), kThreads, 0, s, tris, m, fflag);
    S2_TRY(exclusive_scan(fflag, uflag, m, nullptr, scan_scratch, nullptr, s, &dcnt->scan_fault));
    launch(k_compact, grid_for(n > m ? n : m), kThreads, 0, s, pts, occ, pts_map, n, tris, fflag, uflag, m, opts, otris,
                                                           dcnt);
    if (bvh_leaves > 0 && bvh_leaves >= m) {
        launch(k_remap_leaves, grid_for(bvh_leaves), kThreads, 0, s, bvh.vals, (const int *)bvh.scene,
               (const int *)fflag, (const int *)uflag, bvh.leaf_of_face);
        bvh_carried = true;
    }
    prof.end(s);
    S2_TRY(cudaMemcpyAsync(hcnt, dcnt, sizeof(RoundCounters), cudaMemcpyDeviceToHost, s));
    S2_TRY(cudaStreamSynchronize(s));
    prof.collect();
    if (hcnt->scan_fault) return PAMO_ERR_DEVICE;
    return PAMO_OK;
}

}  // namespace pamo

// ---------------------------------------------------------------------------
// batch rounds

namespace pamo {

int Stage2::ensure_batch(int K)
{
    if (K <= cap_slots && slots) return PAMO_OK;
    if (cap_pts <= 0 || cap_tris <= 0) return PAMO_ERR_INVALID_ARG;  // ensure() first
    if (slots) cudaFree(slots);
    if (scnt) cudaFree(scnt);
    if (roots) cudaFree(roots);
    if (hslots) cudaFreeHost(hslots);
    if (hscnt) cudaFreeHost(hscnt);
    slots = nullptr; scnt = nullptr; roots = nullptr; hslots = nullptr; hscnt = nullptr;
    cap_slots = 0;
    int c = K > 16 ? K : 16;
    if (cudaMalloc((void **)&slots, (size_t)c * sizeof(SlotInfo)) != cudaSuccess ||
        cudaMalloc((void **)&scnt, (size_t)c * sizeof(SlotCounters)) != cudaSuccess ||
        cudaMalloc((void **)&roots, (size_t)c * 4) != cudaSuccess ||
        cudaMallocHost((void **)&hslots, (size_t)c * sizeof(SlotInfo)) != cudaSuccess ||
        cudaMallocHost((void **)&hscnt, (size_t)c * sizeof(SlotCounters)) != cudaSuccess)
        return PAMO_ERR_OOM;
    if (!vslot && cudaMalloc((void **)&vslot, (size_t)(cap_pts + 1) * 4) != cudaSuccess) return PAMO_ERR_OOM;
    if (!gmap && cudaMalloc((void **)&gmap, (size_t)(cap_pts + 1) * 4) != cudaSuccess) return PAMO_ERR_OOM;
    if (!line_list && cudaMalloc((void **)&line_list, (size_t)(cap_edges + 1) * 4) != cudaSuccess) return PAMO_ERR_OOM;
    if (!cand && cudaMalloc((void **)&cand, (size_t)(cap_edges + 1) * 4) != cudaSuccess) return PAMO_ERR_OOM;
    cap_slots = c;
    return PAMO_OK;
}

static cudaError_t undo_check_batch(Stage2 &S, int K, cudaStream_t s)
{
    S.prof.begin(PH_UNDO, s);
    const long long NC = S.cap_edges;
    launch(k_undo_flags, grid_for(NC), kThreads, 0, s, S.cand, S.dcnt, S.edges, S.first_near, S.near_tris, S.isect,
           S.uflag);
    cudaError_t e = exclusive_scan(S.uflag, S.eflag, NC, &S.dcnt->n_considered, S.scan_scratch, &S.dcnt->n_undo, s, &S.dcnt->scan_fault);
    if (e != cudaSuccess) return e;
    launch(k_b_undo_counts, grid_for(K), kThreads, 0, s, S.eflag, S.dcnt, S.scnt, K);
    launch(k_b_undo_scatter, grid_for(NC), kThreads, 0, s, S.uflag, S.eflag, S.dcnt, S.cand, S.edges, S.vslot,
           S.slots, S.scnt, S.undo_edges);
    S.prof.end(s);
    return cudaGetLastError();
}

static dim3 slot_grid(int K, long long per_slot_max)
{
    long long x = (per_slot_max + kThreads - 1) / kThreads;
    x = x < 1 ? 1 : (x > 64 ? 64 : x);
    return dim3((unsigned)x, (unsigned)K);
}

int Stage2::round_batch(int n, int m, int K, int *nvu_out, cudaStream_t s)
{
    if (K <= 0 || K > cap_slots) return PAMO_ERR_INVALID_ARG;
    n_slots = K;
    bvh_carried = false;
    std::vector<int> nvu(K), first(K), cnt_undo(K);
    long long max_n = 0, max_undo_in = 0, max_cap_v = 0;
    for (int r = 0; r < K; ++r) {
        SlotInfo &h = hslots[r];
        nvu[r] = first[r] = h.is_stuck ? h.n_undo_in : 0;
        h.pass_first = h.pass_count = 0;
        h.nvu = 0;
        h.in_undo = 1;
        max_n = h.n > max_n ? h.n : max_n;
        max_undo_in = h.n_undo_in > max_undo_in ? h.n_undo_in : max_undo_in;
        max_cap_v = h.cap_v > max_cap_v ? h.cap_v : max_cap_v;
    }
    S2_TRY(cudaMemsetAsync(dcnt, 0, sizeof(RoundCounters), s));
    S2_TRY(cudaMemsetAsync(scnt, 0, (size_t)K * sizeof(SlotCounters), s));
    S2_TRY(cudaMemcpyAsync(slots, hslots, (size_t)K * sizeof(SlotInfo), cudaMemcpyHostToDevice, s));
    launch(k_b_pre_copy, slot_grid(K, max_undo_in > max_cap_v ? max_undo_in : max_cap_v), kThreads, 0, s,
           (const SlotInfo *)slots);
    launch(k_b_pre_mark, slot_grid(K, max_undo_in), kThreads, 0, s, (const SlotInfo *)slots);
    launch(k_b_vslot, slot_grid(K, max_n), kThreads, 0, s, (const SlotInfo *)slots, vslot);

    prof.begin(PH_SETUP, s);
    launch(k_round_init, grid_for((n + 1 > m ? n + 1 : m)), kThreads, 0, s, opts, otris, pts, tris, occ, first_near,
           cursor, vmin, n, m);
    launch(k_face_a, grid_for(m), kThreads, 0, s, pts, tris, m, first_near, first_edge, plane, elen4);
    S2_TRY(cudaMemsetAsync(first_edge + m, 0, 4, s));
    S2_TRY(exclusive_scan(first_near, first_near, (long long)n + 1, nullptr, scan_scratch, nullptr, s, &dcnt->scan_fault));
    S2_TRY(exclusive_scan(first_edge, first_edge, (long long)m + 1, nullptr, scan_scratch, &dcnt->n_edges, s, &dcnt->scan_fault));
    const int *d_n_edges = &dcnt->n_edges;
    launch(k_face_b, grid_for(m), kThreads, 0, s, tris, m, first_near, cursor, near_tris, first_edge, edges);
    launch(k_vertex_quadric, grid_for(n), kThreads, 0, s, first_near, near_tris, plane, tris, quad, nxt, n);
    launch(k_b_edge_off, grid_for(K), kThreads, 0, s, (const SlotInfo *)slots, (const int *)first_edge, scnt, K);
    prof.begin(PH_LBVH_BUILD, s);
    S2_TRY(lbvh_build(bvh, pts, tris, m, s, vslot, K, roots));
    bvh_boxes_valid = false;
    bvh_leaves = m;

    const long long EMAX = 3LL * m;
    prof.begin(PH_EDGE_COST, s);
    CostArgs ca{edges, d_n_edges, pts, tris, first_near, near_tris, nxt, plane, elen4, quad, nullptr,
                nullptr, vmin, 0.f, 1.f, 0, slots, scnt, vslot, nullptr, nullptr};
    launch(k_edge_cost<false>, grid_for(m, kChunkFaces), kThreads, 0, s, ca, bvh.vals, bvh.scene, first_edge);
    CollapseArgs cl{edges, d_n_edges, nullptr, vmin, first_near, near_tris, opts, otris, pts, tris, occ, eflag,
                    0u, slots, scnt, vslot, nullptr};
    prof.begin(PH_COLLAPSE, s);
    launch(k_collapse, grid_for(EMAX), kThreads, 0, s, cl);
    S2_TRY(exclusive_scan(eflag, uflag, EMAX, d_n_edges, scan_scratch, &dcnt->n_main, s, &dcnt->scan_fault));
    launch(k_scatter_flagged, grid_for(EMAX), kThreads, 0, s, eflag, uflag, d_n_edges, collapsed, 0);
    launch(k_collapse_apply<false>, grid_for(EMAX), kThreads, 0, s, cl, (const int *)collapsed,
           (const int *)&dcnt->n_main);
    launch(k_b_main, grid_for(K), kThreads, 0, s, (const int *)uflag, (const RoundCounters *)dcnt, scnt, K);
    prof.begin(PH_CLEANUP, s);
    launch(k_remove_invalid_faces, grid_for(m), kThreads, 0, s, tris, m);
    launch(k_line_flags, grid_for(EMAX), kThreads, 0, s, edges, d_n_edges, pts, eflag, &dcnt->n_line);
    launch(k_b_line_apply, 1, kLineThreads, 0, s, edges, d_n_edges, eflag, first_near, near_tris, pts, tris, occ,
           line_list, (const int *)vslot, dcnt, scnt, K);
    launch(k_b_cand_fill, grid_for(EMAX), kThreads, 0, s, (const int *)collapsed, (const int *)line_list, edges,
           (const int *)vslot, (const RoundCounters *)dcnt, (const SlotCounters *)scnt, cand);

    S2_TRY(cudaMemsetAsync(active, 0, (size_t)m, s));
    launch(k_mark_active, grid_for(EMAX), kThreads, 0, s, cand, dcnt, edges, first_near, near_tris, active);
    // the first pass refits the round's new hierarchy; the undo passes refit only
    // the one-rings of the edges they undid
    auto pass = [&](bool undo) -> int {
        S2_TRY(isect_pass(*this, m, s, undo ? undo_edges : nullptr, undo ? &dcnt->n_undo : nullptr));
        S2_TRY(undo_check_batch(*this, K, s));
        S2_TRY(cudaMemcpyAsync(hcnt, dcnt, sizeof(RoundCounters), cudaMemcpyDeviceToHost, s));
        S2_TRY(cudaMemcpyAsync(hscnt, scnt, (size_t)K * sizeof(SlotCounters), cudaMemcpyDeviceToHost, s));
        S2_TRY(cudaStreamSynchronize(s));
        prof.collect();
        if (hcnt->pair_overflow > 0) {
            long long need = (long long)hcnt->n_pairs + hcnt->n_pairs / 2 + 1024;
            int rc = ensure_pairs(need);
            if (rc) return rc;
            S2_TRY(isect_pass(*this, m, s, undo ? undo_edges : nullptr, undo ? &dcnt->n_undo : nullptr));
            S2_TRY(undo_check_batch(*this, K, s));
            S2_TRY(cudaMemcpyAsync(hcnt, dcnt, sizeof(RoundCounters), cudaMemcpyDeviceToHost, s));
            S2_TRY(cudaMemcpyAsync(hscnt, scnt, (size_t)K * sizeof(SlotCounters), cudaMemcpyDeviceToHost, s));
            S2_TRY(cudaStreamSynchronize(s));
            if (hcnt->pair_overflow > 0) return PAMO_ERR_CAPACITY;
        }
        if (hcnt->stack_overflow > 0) return PAMO_ERR_CAPACITY;
    if (hcnt->scan_fault) return PAMO_ERR_DEVICE;
        return PAMO_OK;
    };
    int rc = pass(false);
    if (rc) return rc;
    last_stats[0] = hcnt->n_edges;
    last_stats[1] = hcnt->n_main;
    last_stats[2] = hcnt->n_total;
    last_stats[5] = hcnt->n_pairs;
    last_stats[6] = m;
    bool any = false;
    for (int r = 0; r < K; ++r) {
        cnt_undo[r] = hscnt[r].n_undo;
        nvu[r] += 2 * cnt_undo[r];
        if (nvu[r] > hslots[r].cap_undo) return PAMO_ERR_CAPACITY;
        any = any || cnt_undo[r] != 0;
    }
    int it = 0;
    while (any) {
        it++;
        prof.begin(PH_UNDO, s);
        launch(k_undo_apply, grid_for(hcnt->n_undo), kThreads, 0, s, undo_edges, dcnt, edges, first_near, near_tris,
               opts, otris, pts, tris, occ);
        long long max_cnt = 0;
        for (int r = 0; r < K; ++r) {
            hslots[r].pass_first = first[r];
            hslots[r].pass_count = nvu[r] - first[r];
            hslots[r].in_undo = cnt_undo[r] != 0 ? 1 : 0;
            max_cnt = hslots[r].pass_count > max_cnt ? hslots[r].pass_count : max_cnt;
            first[r] += 2 * cnt_undo[r];
        }
        S2_TRY(cudaMemcpyAsync(slots, hslots, (size_t)K * sizeof(SlotInfo), cudaMemcpyHostToDevice, s));
        if (max_cnt > 0) launch(k_b_rearrange, slot_grid(K, max_cnt), kThreads, 0, s, (const SlotInfo *)slots);
        rc = pass(true);
        if (rc) return rc;
        any = false;
        for (int r = 0; r < K; ++r) {
            cnt_undo[r] = hscnt[r].n_undo;
            nvu[r] += 2 * cnt_undo[r];
            if (nvu[r] > hslots[r].cap_undo) return PAMO_ERR_CAPACITY;
            any = any || cnt_undo[r] != 0;
        }
        if (it == 5) break;
    }
    last_stats[3] = it;
    // the packed vertex map, each mesh's own map and undo-list copy
    prof.begin(PH_COMPACT, s);
    S2_TRY(exclusive_scan(occ, gmap, (long long)n + 1, nullptr, scan_scratch, nullptr, s, &dcnt->scan_fault));
    long long max_nvu = 0;
    for (int r = 0; r < K; ++r) {
        hslots[r].nvu = nvu[r];
        max_nvu = nvu[r] > max_nvu ? nvu[r] : max_nvu;
        nvu_out[r] = nvu[r];
    }
    S2_TRY(cudaMemcpyAsync(slots, hslots, (size_t)K * sizeof(SlotInfo), cudaMemcpyHostToDevice, s));
    launch(k_b_local_map, slot_grid(K, (max_n + 1 > max_nvu ? max_n + 1 : max_nvu)), kThreads, 0, s,
           (const SlotInfo *)slots, (const int *)gmap);
    prof.end(s);
    return PAMO_OK;
}

int Stage2::compact_batch(int n, int m, int K, cudaStream_t s)
{
    prof.begin(PH_COMPACT, s);
    launch(k_face_live_flags, grid_for(m), kThreads, 0, s, tris, m, fflag);
    S2_TRY(cudaMemsetAsync(fflag + m, 0, 4, s));
    S2_TRY(exclusive_scan(fflag, uflag, (long long)m + 1, nullptr, scan_scratch, nullptr, s, &dcnt->scan_fault));
    launch(k_compact, grid_for(n > m ? n : m), kThreads, 0, s, pts, occ, gmap, n, tris, fflag, uflag, m, opts, otris,
           dcnt);
    launch(k_b_next, grid_for(K), kThreads, 0, s, (const SlotInfo *)slots, (const int *)gmap, (const int *)uflag, scnt,
           K);
    prof.end(s);
    S2_TRY(cudaMemcpyAsync(hcnt, dcnt, sizeof(RoundCounters), cudaMemcpyDeviceToHost, s));
    S2_TRY(cudaMemcpyAsync(hscnt, scnt, (size_t)K * sizeof(SlotCounters), cudaMemcpyDeviceToHost, s));
    S2_TRY(cudaStreamSynchronize(s));
    prof.collect();
    return PAMO_OK;
}

}  // namespace pamo
