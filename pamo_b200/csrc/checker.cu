// Acceptance checks of a simplified mesh, on the device:
//   * pamo_check_mesh: exact-predicate self-intersection test of every pair of
//     faces whose closed bounding boxes overlap, degenerate faces, and the
//     manifold / watertight checks (edges in exactly two faces, once each way;
//     one closed fan of faces around every vertex);
//   * pamo_mesh_distance: one-sided distance from a mesh's surface to another
//     mesh by dense sampling (the Hausdorff and Chamfer terms of the
//     reference's metrics.py:31-51), with an upper bound from the sampling
//     density.
// The role model of the first is the reference's CGAL self-intersection script
// (simp_cuda/safe_project/scripts/cgal_intersect/main.cpp:19-111): faces that
// share a vertex or an edge intersect only beyond what they share.
//
// Both traverse the faces' LBVH (lbvh.cuh) without a stack: inner nodes keep
// both child boxes, the parent array gives the way up, and a walker that
// returns to a node from its first child goes on to the second.
#include <cfloat>
#include <vector>

#include "exact.cuh"
#include "lbvh.cuh"
#include "scan.cuh"

namespace pamo {
namespace {

using exact::P3;

enum CheckCounter {
    C_PAIRS = 0,       // intersecting pairs
    C_FACES,           // faces in an intersecting pair
    C_DEGENERATE,      // faces with a repeated index or collinear corners
    C_BOUNDARY,        // half-edges without a reverse half-edge
    C_NONMANIFOLD,     // half-edges of an edge in more than two faces or twice one way
    C_BAD_VERTEX,      // vertices whose faces do not form one closed fan
    C_UNREFERENCED,    // vertices in no live face
    C_CANDIDATES,      // face pairs with overlapping boxes
    C_DEAD,            // faces (-1, -1, -1)
    C_ERROR,           // traversal budget exceeded (corrupt hierarchy)
    C_BAD_INDEX,       // an index outside [0, n_pts) in a live face
    C_COUNT
};

__global__ void k_ck_convert(const float *pts, int n, const int *tris, int m, float4 *p4, int4 *t4)
{
    const long long N = n > m ? n : m;
    PAMO_GRID_STRIDE(i, N)
    {
        if (i < n) p4[i] = make_float4(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], 0.f);
        if (i < m) t4[i] = make_int4(tris[3 * i], tris[3 * i + 1], tris[3 * i + 2], 0);
    }
}

__global__ void k_ck_validate(const int4 *tris, int m, int n, unsigned long long *cnt)
{
    PAMO_GRID_STRIDE(f, m)
    {
        const int4 t = tris[f];
        if (face_dead(t)) {
            atomicAdd(&cnt[C_DEAD], 1ULL);
            continue;
        }
        if (t.x < 0 || t.x >= n || t.y < 0 || t.y >= n || t.z < 0 || t.z >= n) atomicAdd(&cnt[C_BAD_INDEX], 1ULL);
    }
}

__device__ __forceinline__ void load_tri(const float4 *p, int4 t, P3 *T, int *idx)
{
    idx[0] = t.x; idx[1] = t.y; idx[2] = t.z;
    for (int k = 0; k < 3; ++k) {
        const float4 q = p[idx[k]];
        T[k] = {q.x, q.y, q.z};
    }
}

// degenerate flag per live face; counts
__global__ void k_ck_degenerate(const float4 *p, const int4 *tris, int m, uint8_t *deg, unsigned long long *cnt)
{
    PAMO_GRID_STRIDE(f, m)
    {
        const int4 t = tris[f];
        uint8_t d = 0;
        if (!face_dead(t)) {
            P3 T[3];
            int idx[3];
            load_tri(p, t, T, idx);
            d = exact::tri_degenerate(T, idx) ? 1 : 0;
            if (d) atomicAdd(&cnt[C_DEGENERATE], 1ULL);
        }
        deg[f] = d;
    }
}

__device__ __forceinline__ bool overlaps(float4 lo, float4 hi, float3 qlo, float3 qhi)
{
    return !(hi.x < qlo.x || qhi.x < lo.x || hi.y < qlo.y || qhi.y < lo.y || hi.z < qlo.z || qhi.z < lo.z);
}

// Every pair f < g of live faces with overlapping closed boxes, one thread per
// leaf (Morton order, so a warp's faces are neighbours and walk similar paths).
__global__ void __launch_bounds__(128) k_ck_pairs(const BvhNode *__restrict__ nodes, const int *__restrict__ parent,
                                                  const int *__restrict__ vals, const int *scene,
                                                  const float4 *__restrict__ p, const int4 *__restrict__ tris,
                                                  const uint8_t *__restrict__ deg, uint8_t *flags,
                                                  unsigned long long *cnt)
{
    const int L = scene[7];
    if (L < 2) return;
    PAMO_GRID_STRIDE(pp, L)
    {
        const int f = vals[pp];
        const int4 tf = tris[f];
        if (deg[f]) continue;
        P3 A[3];
        int ia[3];
        load_tri(p, tf, A, ia);
        const float3 qlo = make_float3(fminf((float)A[0].x, fminf((float)A[1].x, (float)A[2].x)),
                                       fminf((float)A[0].y, fminf((float)A[1].y, (float)A[2].y)),
                                       fminf((float)A[0].z, fminf((float)A[1].z, (float)A[2].z)));
        const float3 qhi = make_float3(fmaxf((float)A[0].x, fmaxf((float)A[1].x, (float)A[2].x)),
                                       fmaxf((float)A[0].y, fmaxf((float)A[1].y, (float)A[2].y)),
                                       fmaxf((float)A[0].z, fmaxf((float)A[1].z, (float)A[2].z)));
        unsigned long long cand = 0;
        bool hit = false;
        auto visit_leaf = [&](int leaf) {
            const int g = vals[leaf];
            if (g <= f || deg[g]) return;
            ++cand;
            P3 B[3];
            int ib[3];
            load_tri(p, tris[g], B, ib);
            if (exact::faces_intersect(A, ia, B, ib)) {
                hit = true;
                flags[g] = 1;
                atomicAdd(&cnt[C_PAIRS], 1ULL);
            }
        };
        // stackless walk: `from` 0 = arrived from the parent, 1 = from the left
        // child, 2 = from the right child
        int node = 0, from = 0;
        long long budget = 4LL * L + 16;
        while (true) {
            if (--budget < 0) {
                atomicAdd(&cnt[C_ERROR], 1ULL);
                break;
            }
            const BvhNode nd = nodes[node];
            int next = -1;
            if (from == 0) {
                if (overlaps(nd.llo, nd.lhi, qlo, qhi)) {
                    const int c = __float_as_int(nd.llo.w);
                    if (c >= 0) next = c;
                    else visit_leaf(~c);
                }
            }
            if (next < 0 && from != 2 && overlaps(nd.rlo, nd.rhi, qlo, qhi)) {
                const int c = __float_as_int(nd.rlo.w);
                if (c >= 0) next = c;
                else visit_leaf(~c);
            }
            if (next >= 0) {
                node = next;
                from = 0;
                continue;
            }
            const int code = parent[node];
            if (code < 0) break;  // back at the root
            node = code >> 2;
            from = (code & 1) ? 2 : 1;
        }
        if (hit) flags[f] = 1;
        if (cand) atomicAdd(&cnt[C_CANDIDATES], cand);
    }
}

__global__ void k_ck_count(const int4 *tris, int m, int *deg_v)
{
    PAMO_GRID_STRIDE(f, m)
    {
        const int4 t = tris[f];
        if (face_dead(t)) continue;
        atomicAdd(&deg_v[t.x], 1);
        atomicAdd(&deg_v[t.y], 1);
        atomicAdd(&deg_v[t.z], 1);
    }
}

__global__ void k_ck_fill(const int4 *tris, int m, const int *first, int *cursor, int *faces_of)
{
    PAMO_GRID_STRIDE(f, m)
    {
        const int4 t = tris[f];
        if (face_dead(t)) continue;
        faces_of[first[t.x] + atomicAdd(&cursor[t.x], 1)] = (int)f;
        faces_of[first[t.y] + atomicAdd(&cursor[t.y], 1)] = (int)f;
        faces_of[first[t.z] + atomicAdd(&cursor[t.z], 1)] = (int)f;
    }
}

__device__ __forceinline__ int corner(int4 t, int k) { return k == 0 ? t.x : (k == 1 ? t.y : t.z); }

// does face t contain the directed edge a -> b
__device__ __forceinline__ bool has_directed(int4 t, int a, int b)
{
    return (t.x == a && t.y == b) || (t.y == a && t.z == b) || (t.z == a && t.x == b);
}

// per half-edge a -> b of every live face: the faces around a holding a -> b
// (itself included) and b -> a
__global__ void k_ck_edges(const int4 *tris, int m, const int *first, const int *faces_of, unsigned long long *cnt)
{
    PAMO_GRID_STRIDE(h, 3LL * m)
    {
        const int f = (int)(h / 3), k = (int)(h % 3);
        const int4 t = tris[f];
        if (face_dead(t)) continue;
        const int a = corner(t, k), b = corner(t, (k + 1) % 3);
        int same = 0, back = 0;
        for (int s = first[a]; s < first[a + 1]; ++s) {
            const int4 u = tris[faces_of[s]];
            same += has_directed(u, a, b);
            back += has_directed(u, b, a);
        }
        if (same > 1 || back > 1) atomicAdd(&cnt[C_NONMANIFOLD], 1ULL);
        else if (back == 0) atomicAdd(&cnt[C_BOUNDARY], 1ULL);
    }
}

// per vertex: following the faces around v across their shared edges (face
// (v, x, y) is followed by the face holding v -> y) must run through all of
// them once and come back
__global__ void k_ck_fans(const int4 *tris, int n, const int *first, const int *faces_of, unsigned long long *cnt)
{
    PAMO_GRID_STRIDE(vv, n)
    {
        const int v = (int)vv;
        const int s0 = first[v], d = first[v + 1] - s0;
        if (d == 0) {
            atomicAdd(&cnt[C_UNREFERENCED], 1ULL);
            continue;
        }
        auto next_of = [&](int4 t) {  // y of the rotation (v, x, y)
            return t.x == v ? t.z : (t.y == v ? t.x : t.y);
        };
        const int start = faces_of[s0];
        int cur = start, steps = 0;
        bool ok = true;
        while (true) {
            const int y = next_of(tris[cur]);
            int nxt = -1, found = 0;
            for (int s = s0; s < s0 + d; ++s) {
                const int g = faces_of[s];
                if (has_directed(tris[g], v, y)) {
                    nxt = g;
                    ++found;
                }
            }
            if (found != 1) {
                ok = false;
                break;
            }
            ++steps;
            cur = nxt;
            if (cur == start || steps > d) break;
        }
        if (!ok || cur != start || steps != d) atomicAdd(&cnt[C_BAD_VERTEX], 1ULL);
    }
}

// ------------------------------------------------------------------ distances
struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 dsub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 dat(float4 p) { return {p.x, p.y, p.z}; }

// squared distance from p to the closed triangle abc: the closest point by the
// Voronoi regions of the triangle's vertices, edges and face (Ericson,
// Real-Time Collision Detection, 2005, sec. 5.1.5)
__device__ double point_tri_d2(D3 p, D3 a, D3 b, D3 c)
{
    const D3 ab = dsub(b, a), ac = dsub(c, a), ap = dsub(p, a);
    const double d1 = ddot(ab, ap), d2 = ddot(ac, ap);
    D3 q;
    if (d1 <= 0.0 && d2 <= 0.0) {
        q = a;
    } else {
        const D3 bp = dsub(p, b);
        const double d3 = ddot(ab, bp), d4 = ddot(ac, bp);
        if (d3 >= 0.0 && d4 <= d3) {
            q = b;
        } else {
            const double vc = d1 * d4 - d3 * d2;
            if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
                const double v = d1 / (d1 - d3);
                q = {a.x + v * ab.x, a.y + v * ab.y, a.z + v * ab.z};
            } else {
                const D3 cp = dsub(p, c);
                const double d5 = ddot(ab, cp), d6 = ddot(ac, cp);
                if (d6 >= 0.0 && d5 <= d6) {
                    q = c;
                } else {
                    const double vb = d5 * d2 - d1 * d6;
                    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
                        const double w = d2 / (d2 - d6);
                        q = {a.x + w * ac.x, a.y + w * ac.y, a.z + w * ac.z};
                    } else {
                        const double va = d3 * d6 - d5 * d4;
                        if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
                            const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
                            q = {b.x + w * (c.x - b.x), b.y + w * (c.y - b.y), b.z + w * (c.z - b.z)};
                        } else {
                            const double den = 1.0 / (va + vb + vc);
                            const double v = vb * den, w = vc * den;
                            q = {a.x + ab.x * v + ac.x * w, a.y + ab.y * v + ac.y * w, a.z + ab.z * v + ac.z * w};
                        }
                    }
                }
            }
        }
    }
    const D3 d = dsub(p, q);
    return ddot(d, d);
}

__device__ __forceinline__ double box_d2(float4 lo, float4 hi, D3 p)
{
    const double dx = fmax(fmax((double)lo.x - p.x, 0.0), p.x - (double)hi.x);
    const double dy = fmax(fmax((double)lo.y - p.y, 0.0), p.y - (double)hi.y);
    const double dz = fmax(fmax((double)lo.z - p.z, 0.0), p.z - (double)hi.z);
    return dx * dx + dy * dy + dz * dz;
}

// squared distance from p to the nearest face of the hierarchy's mesh: a
// stackless walk that enters the nearer child first and the farther one on
// the way back if its box is still closer than the best face so far
__device__ double nearest_d2(D3 p, const BvhNode *__restrict__ nodes, const int *__restrict__ parent,
                             const int *__restrict__ vals, int L, const float4 *__restrict__ pts,
                             const int4 *__restrict__ tris, unsigned long long *err)
{
    double best = DBL_MAX;
    auto leaf = [&](int pos) {
        const int g = vals[pos];
        if (g < 0) return;
        const int4 t = tris[g];
        const double d2 = point_tri_d2(p, dat(pts[t.x]), dat(pts[t.y]), dat(pts[t.z]));
        best = fmin(best, d2);
    };
    if (L == 1) {
        leaf(0);
        return best;
    }
    int node = 0, from = 0;  // from: 0 parent, 1 left child, 2 right child
    long long budget = 4LL * L + 16;
    while (true) {
        if (--budget < 0) {
            atomicAdd(err, 1ULL);
            break;
        }
        const BvhNode nd = nodes[node];
        const double dl = box_d2(nd.llo, nd.lhi, p), dr = box_d2(nd.rlo, nd.rhi, p);
        const int near_side = dl <= dr ? 1 : 2;
        const int cl = __float_as_int(nd.llo.w), cr = __float_as_int(nd.rlo.w);
        int next = -1;
        // from the parent: the nearer side, then the farther; back from the
        // nearer side: the farther; back from the farther side: done here
        if (from == 0 || from == near_side) {
            for (int k = from == 0 ? 0 : 1; k < 2 && next < 0; ++k) {
                const int side = k == 0 ? near_side : 3 - near_side;
                if ((side == 1 ? dl : dr) >= best) continue;
                const int c = side == 1 ? cl : cr;
                if (c >= 0) next = c;
                else leaf(~c);
            }
        }
        if (next >= 0) {
            node = next;
            from = 0;
            continue;
        }
        const int code = parent[node];
        if (code < 0) break;
        node = code >> 2;
        from = (code & 1) ? 2 : 1;
    }
    return best;
}

// One thread per sample (face f of A, barycentric grid point (i/k, j/k)):
// distance to mesh B; the block's largest squared distance and the sum of the
// squared distances go to this block's partials.
__global__ void __launch_bounds__(128) k_hd_samples(const float4 *__restrict__ pa, const int4 *__restrict__ fa,
                                                    int nfa, int k, const BvhNode *__restrict__ nodes,
                                                    const int *__restrict__ parent, const int *__restrict__ vals,
                                                    const int *scene, const float4 *__restrict__ pb,
                                                    const int4 *__restrict__ fb, double *part_max, double *part_sum,
                                                    double *part_edge, unsigned long long *err)
{
    const int L = scene[7];
    const int S = (k + 1) * (k + 2) / 2;
    double mx = 0.0, sum = 0.0, edge = 0.0;
    PAMO_GRID_STRIDE(i, (long long)nfa * S)
    {
        const int f = (int)(i / S);
        int s = (int)(i % S);
        const int4 t = fa[f];
        if (face_dead(t) || L == 0) continue;
        // s -> (u, v) with u + v <= k, rows of u
        int u = 0;
        while (s > k - u) {
            s -= k - u + 1;
            ++u;
        }
        const int v = s;
        const D3 a = dat(pa[t.x]), b = dat(pa[t.y]), c = dat(pa[t.z]);
        const double su = (double)u / k, sv = (double)v / k;
        const D3 q = {a.x + su * (b.x - a.x) + sv * (c.x - a.x), a.y + su * (b.y - a.y) + sv * (c.y - a.y),
                      a.z + su * (b.z - a.z) + sv * (c.z - a.z)};
        const double d2 = nearest_d2(q, nodes, parent, vals, L, pb, fb, err);
        mx = fmax(mx, d2);
        sum += d2;
        if (u == 0 && v == 0) {  // the face's longest edge, once per face
            const D3 e0 = dsub(b, a), e1 = dsub(c, b), e2 = dsub(a, c);
            edge = fmax(edge, fmax(ddot(e0, e0), fmax(ddot(e1, e1), ddot(e2, e2))));
        }
    }
    __shared__ double sm[3][128];
    sm[0][threadIdx.x] = mx;
    sm[1][threadIdx.x] = sum;
    sm[2][threadIdx.x] = edge;
    __syncthreads();
    for (int o = 64; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sm[0][threadIdx.x] = fmax(sm[0][threadIdx.x], sm[0][threadIdx.x + o]);
            sm[1][threadIdx.x] += sm[1][threadIdx.x + o];
            sm[2][threadIdx.x] = fmax(sm[2][threadIdx.x], sm[2][threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part_max[blockIdx.x] = sm[0][0];
        part_sum[blockIdx.x] = sm[1][0];
        part_edge[blockIdx.x] = sm[2][0];
    }
}

constexpr int kHdBlocks = kNumSMs * 8;

struct DeviceBuf {
    void *p = nullptr;
    cudaStream_t s = nullptr;
    DeviceBuf(size_t bytes, cudaStream_t st) : s(st)
    {
        if (bytes && cudaMallocAsync(&p, bytes, st) != cudaSuccess) p = nullptr;
    }
    ~DeviceBuf()
    {
        if (p) cudaFreeAsync(p, s);
    }
    DeviceBuf(const DeviceBuf &) = delete;
    DeviceBuf &operator=(const DeviceBuf &) = delete;
    template <class T> T *as() const { return static_cast<T *>(p); }
};

}  // namespace
}  // namespace pamo

using namespace pamo;

extern "C" int pamo_check_mesh(const float *d_points, const int *d_tris, int n_pts, int n_tris,
                               unsigned char *d_out_flags, long long *h_out, void *stream)
{
    if (!h_out || n_pts < 0 || n_tris < 0 || (n_tris && (!d_points || !d_tris || n_pts == 0))) return PAMO_ERR_INVALID_ARG;
    for (int i = 0; i < C_COUNT; ++i) h_out[i] = 0;
    if (n_tris == 0) {
        h_out[C_UNREFERENCED] = n_pts;
        return PAMO_OK;
    }
    int dev;
    if (cudaGetDevice(&dev) != cudaSuccess) return PAMO_ERR_NO_DEVICE;
    cudaStream_t s = (cudaStream_t)stream;
    PAMO_CUDA_TRY(retain_pool_memory());
    DeviceBuf p4((size_t)n_pts * 16, s), t4((size_t)n_tris * 16, s), cnt(C_COUNT * 8, s), deg((size_t)n_tris, s);
    DeviceBuf flags(d_out_flags ? 0 : (size_t)n_tris, s);
    DeviceBuf degv(((size_t)n_pts + 1) * 4, s), first(((size_t)n_pts + 1) * 4, s), cursor((size_t)n_pts * 4, s);
    DeviceBuf faces_of((size_t)n_tris * 3 * 4, s), scan_tmp((size_t)scan_scratch_ints((long long)n_pts + 1) * 4, s);
    if (!p4.p || !t4.p || !cnt.p || !deg.p || !degv.p || !first.p || !cursor.p || !faces_of.p || !scan_tmp.p ||
        (!d_out_flags && !flags.p))
        return PAMO_ERR_OOM;
    uint8_t *fl = d_out_flags ? d_out_flags : flags.as<uint8_t>();
    unsigned long long *c = cnt.as<unsigned long long>();
    PAMO_CUDA_TRY(cudaMemsetAsync(c, 0, C_COUNT * 8, s));
    PAMO_CUDA_TRY(cudaMemsetAsync(fl, 0, (size_t)n_tris, s));
    launch(k_ck_convert, grid_for(n_pts > n_tris ? n_pts : n_tris), kThreads, 0, s, d_points, n_pts, d_tris, n_tris,
           p4.as<float4>(), t4.as<int4>());
    launch(k_ck_validate, grid_for(n_tris), kThreads, 0, s, (const int4 *)t4.as<int4>(), n_tris, n_pts, c);
    unsigned long long h_bad[C_COUNT];
    PAMO_CUDA_TRY(cudaMemcpyAsync(h_bad, c, C_COUNT * 8, cudaMemcpyDeviceToHost, s));
    PAMO_CUDA_TRY(cudaStreamSynchronize(s));
    if (h_bad[C_BAD_INDEX]) return PAMO_ERR_INVALID_ARG;
    launch(k_ck_degenerate, grid_for(n_tris), kThreads, 0, s, (const float4 *)p4.as<float4>(),
           (const int4 *)t4.as<int4>(), n_tris, deg.as<uint8_t>(), c);
    // self-intersections
    Lbvh b;
    cudaError_t e = lbvh_build(b, p4.as<float4>(), t4.as<int4>(), n_tris, s);
    if (e == cudaSuccess) e = lbvh_refit(b, p4.as<float4>(), t4.as<int4>(), n_tris, s);
    if (e != cudaSuccess) {
        b.release();
        return map_cuda_error(e);
    }
    launch(k_ck_pairs, grid_for(n_tris, 128), 128, 0, s, (const BvhNode *)b.nodes, (const int *)b.parent,
           (const int *)b.vals, (const int *)b.scene, (const float4 *)p4.as<float4>(), (const int4 *)t4.as<int4>(),
           (const uint8_t *)deg.as<uint8_t>(), fl, c);
    // manifold checks over the vertex -> face lists
    PAMO_CUDA_TRY(cudaMemsetAsync(degv.p, 0, ((size_t)n_pts + 1) * 4, s));
    PAMO_CUDA_TRY(cudaMemsetAsync(cursor.p, 0, (size_t)n_pts * 4, s));
    launch(k_ck_count, grid_for(n_tris), kThreads, 0, s, (const int4 *)t4.as<int4>(), n_tris, degv.as<int>());
    PAMO_CUDA_TRY(scan_scratch_init(scan_tmp.as<int>(), scan_scratch_ints((long long)n_pts + 1), s));
    PAMO_CUDA_TRY(exclusive_scan(degv.as<int>(), first.as<int>(), (long long)n_pts + 1, nullptr, scan_tmp.as<int>(),
                                 nullptr, s));
    launch(k_ck_fill, grid_for(n_tris), kThreads, 0, s, (const int4 *)t4.as<int4>(), n_tris,
           (const int *)first.as<int>(), cursor.as<int>(), faces_of.as<int>());
    launch(k_ck_edges, grid_for(3LL * n_tris), kThreads, 0, s, (const int4 *)t4.as<int4>(), n_tris,
           (const int *)first.as<int>(), (const int *)faces_of.as<int>(), c);
    launch(k_ck_fans, grid_for(n_pts), kThreads, 0, s, (const int4 *)t4.as<int4>(), n_pts,
           (const int *)first.as<int>(), (const int *)faces_of.as<int>(), c);
    // faces in intersecting pairs
    unsigned long long h[C_COUNT];
    e = cudaMemcpyAsync(h, c, C_COUNT * 8, cudaMemcpyDeviceToHost, s);
    std::vector<uint8_t> hf((size_t)n_tris);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hf.data(), fl, (size_t)n_tris, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    b.release();
    if (e != cudaSuccess) return map_cuda_error(e);
    long long nf = 0;
    for (uint8_t x : hf) nf += x;
    for (int i = 0; i < C_COUNT; ++i) h_out[i] = (long long)h[i];
    h_out[C_FACES] = nf;
    return h[C_ERROR] ? PAMO_ERR_DEVICE : PAMO_OK;
}

extern "C" int pamo_mesh_distance(const float *d_pa, const int *d_fa, int na, int nfa, const float *d_pb,
                                  const int *d_fb, int nb, int nfb, int subdiv, double *h_out4, void *stream)
{
    if (!h_out4 || na < 0 || nfa < 0 || nb < 0 || nfb < 0 || subdiv < 1 || subdiv > 1024) return PAMO_ERR_INVALID_ARG;
    if ((nfa && (!d_pa || !d_fa || na == 0)) || (nfb && (!d_pb || !d_fb || nb == 0))) return PAMO_ERR_INVALID_ARG;
    for (int i = 0; i < 4; ++i) h_out4[i] = 0.0;
    if (nfa == 0) return PAMO_OK;
    if (nfb == 0) return PAMO_ERR_INVALID_ARG;  // no surface to measure against
    int dev;
    if (cudaGetDevice(&dev) != cudaSuccess) return PAMO_ERR_NO_DEVICE;
    cudaStream_t s = (cudaStream_t)stream;
    PAMO_CUDA_TRY(retain_pool_memory());
    DeviceBuf pa4((size_t)na * 16, s), fa4((size_t)nfa * 16, s), pb4((size_t)nb * 16, s), fb4((size_t)nfb * 16, s);
    DeviceBuf part(3 * kHdBlocks * 8, s), err(8, s), bad(C_COUNT * 8, s);
    if (!pa4.p || !fa4.p || !pb4.p || !fb4.p || !part.p || !err.p || !bad.p) return PAMO_ERR_OOM;
    launch(k_ck_convert, grid_for(na > nfa ? na : nfa), kThreads, 0, s, d_pa, na, d_fa, nfa, pa4.as<float4>(),
           fa4.as<int4>());
    launch(k_ck_convert, grid_for(nb > nfb ? nb : nfb), kThreads, 0, s, d_pb, nb, d_fb, nfb, pb4.as<float4>(),
           fb4.as<int4>());
    PAMO_CUDA_TRY(cudaMemsetAsync(bad.p, 0, C_COUNT * 8, s));
    PAMO_CUDA_TRY(cudaMemsetAsync(err.p, 0, 8, s));
    launch(k_ck_validate, grid_for(nfa), kThreads, 0, s, (const int4 *)fa4.as<int4>(), nfa, na,
           bad.as<unsigned long long>());
    unsigned long long ba[C_COUNT];
    PAMO_CUDA_TRY(cudaMemcpyAsync(ba, bad.p, C_COUNT * 8, cudaMemcpyDeviceToHost, s));
    PAMO_CUDA_TRY(cudaStreamSynchronize(s));
    if (ba[C_BAD_INDEX] || ba[C_DEAD] == (unsigned long long)nfa) return PAMO_ERR_INVALID_ARG;
    const long long live_a = (long long)nfa - (long long)ba[C_DEAD];  // dead faces of A add no samples
    PAMO_CUDA_TRY(cudaMemsetAsync(bad.p, 0, C_COUNT * 8, s));
    launch(k_ck_validate, grid_for(nfb), kThreads, 0, s, (const int4 *)fb4.as<int4>(), nfb, nb,
           bad.as<unsigned long long>());
    PAMO_CUDA_TRY(cudaMemcpyAsync(ba, bad.p, C_COUNT * 8, cudaMemcpyDeviceToHost, s));
    PAMO_CUDA_TRY(cudaStreamSynchronize(s));
    if (ba[C_BAD_INDEX] || ba[C_DEAD] == (unsigned long long)nfb) return PAMO_ERR_INVALID_ARG;
    Lbvh b;
    cudaError_t e = lbvh_build(b, pb4.as<float4>(), fb4.as<int4>(), nfb, s);
    if (e == cudaSuccess) e = lbvh_refit(b, pb4.as<float4>(), fb4.as<int4>(), nfb, s);
    if (e != cudaSuccess) {
        b.release();
        return map_cuda_error(e);
    }
    double *pm = part.as<double>(), *ps = pm + kHdBlocks, *pe = ps + kHdBlocks;
    launch(k_hd_samples, kHdBlocks, 128, 0, s, (const float4 *)pa4.as<float4>(), (const int4 *)fa4.as<int4>(), nfa,
           subdiv, (const BvhNode *)b.nodes, (const int *)b.parent, (const int *)b.vals, (const int *)b.scene,
           (const float4 *)pb4.as<float4>(), (const int4 *)fb4.as<int4>(), pm, ps, pe, err.as<unsigned long long>());
    std::vector<double> h(3 * kHdBlocks);
    unsigned long long herr = 0;
    e = cudaMemcpyAsync(h.data(), pm, 3 * kHdBlocks * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err.p, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    b.release();
    if (e != cudaSuccess) return map_cuda_error(e);
    if (herr) return PAMO_ERR_DEVICE;
    double mx = 0.0, sum = 0.0, edge = 0.0;
    for (int i = 0; i < kHdBlocks; ++i) {  // fixed order: the result does not depend on scheduling
        mx = fmax(mx, h[i]);
        sum += h[kHdBlocks + i];
        edge = fmax(edge, h[2 * kHdBlocks + i]);
    }
    const double samples = (double)live_a * ((subdiv + 1) * (subdiv + 2) / 2);
    h_out4[0] = sqrt(mx);
    // every point of a face lies within (longest edge / k) / sqrt(3) of a sample
    // (a sub-triangle's circumradius, or half its longest edge when obtuse), and
    // the distance to B is 1-Lipschitz
    h_out4[1] = sqrt(mx) + sqrt(edge) / subdiv / sqrt(3.0);
    h_out4[2] = sum / samples;
    h_out4[3] = samples;
    return PAMO_OK;
}
