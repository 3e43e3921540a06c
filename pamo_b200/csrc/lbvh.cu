#include "lbvh.cuh"
#include "scan.cuh"

namespace pamo {

namespace {

constexpr int kSortThreads = kLbvhSortThreads;
constexpr int kSortItems = kLbvhSortItems;
constexpr int kSortTile = kLbvhSortTile;

__device__ __forceinline__ uint32_t expand10(uint32_t v)
{
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__device__ __forceinline__ void face_box(const float4 *pts, int4 t, float3 &lo, float3 &hi)
{
    float4 a = pts[t.x], b = pts[t.y], c = pts[t.z];
    lo = make_float3(fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)), fminf(a.z, fminf(b.z, c.z)));
    hi = make_float3(fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)), fmaxf(a.z, fmaxf(b.z, c.z)));
}

__global__ void k_scene_init(int *scene)
{
    int i = threadIdx.x;
    if (i < 3) scene[i] = 0x7FFFFFFF;
    else if (i < 6) scene[i] = (int)0x80000000;
    else if (i < 16) scene[i] = 0;  // [6] dead faces, [7] leaves, [8] error flag
}

// scene box and dead-face count over the round-start faces
__global__ void __launch_bounds__(kThreads) k_scene_bounds(const float4 *pts, const int4 *tris, int m, int *scene)
{
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    int dead = 0;
    PAMO_GRID_STRIDE(f, m)
    {
        int4 t = tris[f];
        if (face_dead(t)) { dead++; continue; }
        float3 l, h;
        face_box(pts, t, l, h);
        lo[0] = fminf(lo[0], l.x); lo[1] = fminf(lo[1], l.y); lo[2] = fminf(lo[2], l.z);
        hi[0] = fmaxf(hi[0], h.x); hi[1] = fmaxf(hi[1], h.y); hi[2] = fmaxf(hi[2], h.z);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            lo[k] = fminf(lo[k], __shfl_down_sync(0xffffffffu, lo[k], o));
            hi[k] = fmaxf(hi[k], __shfl_down_sync(0xffffffffu, hi[k], o));
        }
        dead += __shfl_down_sync(0xffffffffu, dead, o);
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            atomicMin(&scene[k], float_to_ordered(lo[k]));
            atomicMax(&scene[3 + k], float_to_ordered(hi[k]));
        }
        if (dead) atomicAdd(&scene[6], dead);
    }
}

// Sort key of each face: the Morton code of its box centre over the scene box.
// With vslot (a batch of meshes) the key is rank << 3*bits | Morton code with
// `bits` bits per axis, so each mesh's faces are contiguous and form a subtree.
__global__ void __launch_bounds__(kThreads) k_morton(const float4 *pts, const int4 *tris, int m, const int *scene,
                                                     uint32_t *keys, int *vals, const int *vslot, int bits)
{
    const float res = (float)(1 << bits);
    float slo[3], ext[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        slo[k] = ordered_to_float(scene[k]);
        float e = ordered_to_float(scene[3 + k]) - slo[k];
        ext[k] = e > 0.0f ? e : 1.0f;
    }
    PAMO_GRID_STRIDE(f, m)
    {
        int4 t = tris[f];
        uint32_t key = 0xFFFFFFFFu;
        if (!face_dead(t)) {
            float3 l, h;
            face_box(pts, t, l, h);
            float c[3] = {(l.x + h.x) * 0.5f, (l.y + h.y) * 0.5f, (l.z + h.z) * 0.5f};
            uint32_t q[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float u = (c[k] - slo[k]) / ext[k] * res;
                u = fminf(fmaxf(u, 0.0f), res - 1.0f);
                q[k] = expand10((uint32_t)u);
            }
            key = q[0] * 4 + q[1] * 2 + q[2];
            if (vslot) key |= (uint32_t)vslot[t.x] << (3 * bits);
        }
        keys[f] = key;
        vals[f] = (int)f;
    }
}

__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const uint32_t *keys, int n, int shift, int tiles,
                                                             int *hist)
{
    __shared__ int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    long long base = (long long)blockIdx.x * kSortTile;
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        long long i = base + (long long)k * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1);
    }
    __syncthreads();
    hist[threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: elements keep their input order within each digit.
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const uint32_t *keys, const int *vals, int n,
                                                                int shift, int tiles, const int *hist_scanned,
                                                                uint32_t *keys_out, int *vals_out)
{
    __shared__ int wc[kSortThreads / 32][256];
    __shared__ int base_off[256];
    base_off[threadIdx.x] = hist_scanned[threadIdx.x * tiles + blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    long long base = (long long)blockIdx.x * kSortTile;
    for (int c = 0; c < kSortItems; ++c) {
#pragma unroll
        for (int w = 0; w < kSortThreads / 32; ++w) wc[w][threadIdx.x] = 0;
        __syncthreads();
        long long i = base + (long long)c * kSortThreads + threadIdx.x;
        bool valid = i < n;
        uint32_t key = valid ? keys[i] : 0u;
        int val = valid ? vals[i] : 0;
        int d = valid ? (int)((key >> shift) & 255u) : -1;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        int rank = __popc(peers & lt_mask);
        if (valid && rank == 0) wc[warp][d] = __popc(peers);
        __syncthreads();
        {
            int t = threadIdx.x, run = base_off[t];
#pragma unroll
            for (int w = 0; w < kSortThreads / 32; ++w) {
                int cnt = wc[w][t];
                wc[w][t] = run;
                run += cnt;
            }
            base_off[t] = run;
        }
        __syncthreads();
        if (valid) {
            int pos = wc[warp][d] + rank;
            keys_out[pos] = key;
            vals_out[pos] = val;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ int delta(const uint32_t *keys, int L, int i, int j)
{
    if (j < 0 || j >= L) return -1;
    unsigned long long a = ((unsigned long long)keys[i] << 32) | (unsigned)i;
    unsigned long long b = ((unsigned long long)keys[j] << 32) | (unsigned)j;
    return __clzll(a ^ b);
}

// Karras (2012) hierarchy construction, one thread per internal node.
// roots (batch of meshes, rank in the key bits above `rank_shift`): the child
// of a node spanning several ranks that holds one rank only is that rank's
// whole subtree (keys of one rank are contiguous and share every bit above the
// split), recorded as the start node of the rank's queries.
__global__ void __launch_bounds__(kThreads) k_karras(const uint32_t *keys, const int *scene, BvhNode *nodes,
                                                     int *parent, int *roots, int rank_shift)
{
    const int L = scene[7];
    PAMO_GRID_STRIDE(ii, (long long)L - 1)
    {
        int i = (int)ii;
        int d = (delta(keys, L, i, i + 1) - delta(keys, L, i, i - 1)) >= 0 ? 1 : -1;
        int dmin = delta(keys, L, i, i - d);
        int lmax = 2;
        while (delta(keys, L, i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (delta(keys, L, i, i + (l + t) * d) > dmin) l += t;
        int j = i + l * d;
        int dnode = delta(keys, L, i, j);
        int s = 0;
        int len = l;
        do {
            len = (len + 1) >> 1;
            if (delta(keys, L, i, i + (s + len) * d) > dnode) s += len;
        } while (len > 1);
        int gamma = i + s * d + (d < 0 ? -1 : 0);
        int lo = i < j ? i : j, hi = i < j ? j : i;
        int left = (lo == gamma) ? ~gamma : gamma;
        int right = (hi == gamma + 1) ? ~(gamma + 1) : gamma + 1;
        nodes[i].llo.w = __int_as_float(left);
        nodes[i].rlo.w = __int_as_float(right);
        int lid = left < 0 ? (L - 1) + gamma : gamma;
        int rid = right < 0 ? (L - 1) + gamma + 1 : gamma + 1;
        const int tile = (lo >> kRefitTileShift) == (hi >> kRefitTileShift) ? 2 : 0;
        parent[lid] = (i << 2) | tile | 0;
        parent[rid] = (i << 2) | tile | 1;
        if (i == 0) parent[0] = -1;
        if (roots) {
            const uint32_t rlo = keys[lo] >> rank_shift, rhi = keys[hi] >> rank_shift;
            if (rlo != rhi) {
                if (rlo == (keys[gamma] >> rank_shift)) roots[rlo] = left;
                if (rhi == (keys[gamma + 1] >> rank_shift)) roots[rhi] = right;
            }
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_leaf_map(const int *vals, const int *scene, int *leaf_of_face, int m)
{
    const int L = scene[7];
    PAMO_GRID_STRIDE(p, m) leaf_of_face[vals[p]] = p < L ? (int)p : -1;
}

__device__ __forceinline__ void store_child_box(BvhNode *nodes, int code, int self, float3 lo, float3 hi)
{
    int par = code >> 2;
    if (code & 1) {
        nodes[par].rlo = make_float4(lo.x, lo.y, lo.z, __int_as_float(self));
        nodes[par].rhi = make_float4(hi.x, hi.y, hi.z, 0.0f);
    } else {
        nodes[par].llo = make_float4(lo.x, lo.y, lo.z, __int_as_float(self));
        nodes[par].lhi = make_float4(hi.x, hi.y, hi.z, 0.0f);
    }
}

// Bottom-up refit, one thread per leaf: the second child to arrive at a node
// merges the two boxes; the first arrival exits, so nothing waits.  A block
// holds kRefitTile consecutive leaves; a node whose leaves all lie in the
// block's run (the parent code's tile bit) only ever sees arrivals from this
// block, so it counts them in shared memory with block-scope fences, and only
// the few nodes above the runs use global counters and device-scope fences.
// The node indices of one run's nodes lie in that run (a Karras node's index
// is one end of its leaf range), so `node % kRefitTile` is a free slot.
__global__ void __launch_bounds__(kRefitTile) k_refit(const float4 *pts, const int4 *tris, const int *vals,
                                                      int *scene, const int *parent, BvhNode *nodes, int *flags)
{
    __shared__ int arrived[kRefitTile];
    arrived[threadIdx.x] = 0;
    __syncthreads();
    const int L = scene[7];
    const long long p = (long long)blockIdx.x * kRefitTile + threadIdx.x;
    if (L < 2 || p >= L) return;
    int f = vals[p];
    int4 t = f >= 0 ? tris[f] : make_int4(-1, -1, -1, 0);
    float3 lo, hi;
    if (face_dead(t)) {
        lo = make_float3(INFINITY, INFINITY, INFINITY);
        hi = make_float3(-INFINITY, -INFINITY, -INFINITY);
    } else {
        face_box(pts, t, lo, hi);
    }
    int code = parent[(L - 1) + p];
    store_child_box(nodes, code, ~(int)p, lo, hi);
    // a valid hierarchy is at most 64 levels deep (unique 64-bit keys); the
    // bound only guards against a corrupted parent chain
    for (int depth = 0;; ++depth) {
        if (depth > 256) {
            atomicExch(&scene[8], 1);
            break;
        }
        const int node = code >> 2;
        float4 a, b, c, d;
        if (code & 2) {
            __threadfence_block();
            if (atomicAdd(&arrived[node & (kRefitTile - 1)], 1) == 0) break;
            __threadfence_block();
            a = nodes[node].llo, b = nodes[node].lhi, c = nodes[node].rlo, d = nodes[node].rhi;
        } else {
            __threadfence();
            if (atomicAdd(&flags[node], 1) == 0) break;
            __threadfence();
            a = __ldcg(&nodes[node].llo), b = __ldcg(&nodes[node].lhi);
            c = __ldcg(&nodes[node].rlo), d = __ldcg(&nodes[node].rhi);
        }
        lo = make_float3(fminf(a.x, c.x), fminf(a.y, c.y), fminf(a.z, c.z));
        hi = make_float3(fmaxf(b.x, d.x), fmaxf(b.y, d.y), fmaxf(b.z, d.z));
        code = parent[node];
        if (code < 0) break;  // root
        store_child_box(nodes, code, node, lo, hi);
    }
}

__global__ void __launch_bounds__(kThreads) k_refit_dirty(const float4 *pts, const int4 *tris, const int *vals,
                                                          int *scene, const int *parent, BvhNode *nodes, int *claim,
                                                          int *dmask, int *dcount, const int *dlist)
{
    const int L = scene[7];
    const int n = scene[9];
    PAMO_GRID_STRIDE(k, n)
    {
        const int p = dlist[k];
        claim[p] = 0;
        const int f = vals[p];
        int4 t = f >= 0 ? tris[f] : make_int4(-1, -1, -1, 0);
        float3 lo, hi;
        if (face_dead(t)) {
            lo = make_float3(INFINITY, INFINITY, INFINITY);
            hi = make_float3(-INFINITY, -INFINITY, -INFINITY);
        } else {
            face_box(pts, t, lo, hi);
        }
        int code = parent[(L - 1) + p];
        store_child_box(nodes, code, ~p, lo, hi);
        int node = code >> 2;
        for (int depth = 0;; ++depth) {
            if (depth > 256) {
                atomicExch(&scene[8], 1);
                break;
            }
            // the marks were set by an earlier kernel; read them before arriving,
            // since the last child to arrive clears them
            const int need = __popc(__ldcg(&dmask[node]));
            __threadfence();
            const int old = atomicAdd(&dcount[node], 1);
            if (old + 1 < need) break;  // the other dirty child merges this node
            __threadfence();
            float4 a = __ldcg(&nodes[node].llo), b = __ldcg(&nodes[node].lhi);
            float4 c = __ldcg(&nodes[node].rlo), d = __ldcg(&nodes[node].rhi);
            lo = make_float3(fminf(a.x, c.x), fminf(a.y, c.y), fminf(a.z, c.z));
            hi = make_float3(fmaxf(b.x, d.x), fmaxf(b.y, d.y), fmaxf(b.z, d.z));
            dmask[node] = 0;
            dcount[node] = 0;
            const int pc = parent[node];
            if (pc < 0) break;  // root
            store_child_box(nodes, pc, node, lo, hi);
            node = pc >> 2;
        }
    }
}

__global__ void k_count_leaves(int m, int *scene) { scene[7] = m - scene[6]; }

}  // namespace

cudaError_t Lbvh::ensure(long long n)
{
    if (n <= cap && keys) return cudaSuccess;
    release();
    long long c = n > 16 ? n : 16;
    sort_tiles = (int)((c + kSortTile - 1) / kSortTile);
    cudaError_t e;
#define ALLOC(p, bytes)                                   \
    if ((e = cudaMalloc((void **)&p, (bytes))) != cudaSuccess) { \
        release();                                        \
        return e;                                         \
    }
    ALLOC(keys, c * 4);
    ALLOC(keys2, c * 4);
    ALLOC(vals, c * 4);
    ALLOC(vals2, c * 4);
    ALLOC(hist, (long long)256 * sort_tiles * 4 + 64);
    ALLOC(hist_scratch, scan_scratch_ints((long long)256 * sort_tiles) * 4);
    if ((e = scan_scratch_init(hist_scratch, scan_scratch_ints((long long)256 * sort_tiles))) != cudaSuccess) {
        release();
        return e;
    }
    ALLOC(nodes, c * sizeof(BvhNode));
    ALLOC(parent, 2 * c * 4);
    ALLOC(flags, c * 4);
    ALLOC(leaf_of_face, c * 4);
    ALLOC(scene, 64);
    ALLOC(claim, c * 4);
    ALLOC(dmask, c * 4);
    ALLOC(dcount, c * 4);
    ALLOC(dlist, c * 4);
#undef ALLOC
    if ((e = cudaMemset(claim, 0, c * 4)) != cudaSuccess || (e = cudaMemset(dmask, 0, c * 4)) != cudaSuccess ||
        (e = cudaMemset(dcount, 0, c * 4)) != cudaSuccess) {
        release();
        return e;
    }
    cap = c;
    return cudaSuccess;
}

void Lbvh::release()
{
    void *p[] = {keys, keys2, vals, vals2, hist, hist_scratch, nodes, parent, flags, leaf_of_face, scene, claim, dmask,
                 dcount, dlist};
    for (void *q : p)
        if (q) cudaFree(q);
    keys = keys2 = nullptr;
    vals = vals2 = nullptr;
    hist = hist_scratch = nullptr;
    nodes = nullptr;
    parent = flags = leaf_of_face = scene = nullptr;
    claim = dmask = dcount = dlist = nullptr;
    cap = 0;
    leaves_built = 0;
}

cudaError_t lbvh_build(Lbvh &b, const float4 *pts, const int4 *tris, int m, cudaStream_t s, const int *vslot,
                       int n_ranks, int *roots)
{
    cudaError_t e = b.ensure(m);
    if (e != cudaSuccess) return e;
    b.leaves_built = m;
    launch(k_scene_init, 1, 32, 0, s, b.scene);
    if (m == 0) return cudaGetLastError();
    launch(k_scene_bounds, grid_for(m), kThreads, 0, s, pts, tris, m, b.scene);
    // Morton bits per axis: 10, or fewer to leave room for the rank (keys of live
    // faces stay below 2^31, under the key of removed faces)
    int rank_bits = 0;
    while (vslot && (1 << rank_bits) < n_ranks) ++rank_bits;
    const int bits = vslot ? (31 - rank_bits) / 3 : 10;
    if (roots) {
        e = cudaMemsetAsync(roots, 0, (size_t)n_ranks * 4, s);  // one rank: the whole tree
        if (e != cudaSuccess) return e;
    }
    launch(k_morton, grid_for(m), kThreads, 0, s, pts, tris, m, b.scene, b.keys, b.vals, vslot, bits);
    int tiles = (m + kSortTile - 1) / kSortTile;
    uint32_t *k_in = b.keys, *k_out = b.keys2;
    int *v_in = b.vals, *v_out = b.vals2;
    for (int shift = 0; shift < 32; shift += 8) {
        launch(k_radix_hist, tiles, kSortThreads, 0, s, k_in, m, shift, tiles, b.hist);
        e = exclusive_scan(b.hist, b.hist, (long long)256 * tiles, nullptr, b.hist_scratch, nullptr, s);
        if (e != cudaSuccess) return e;
        launch(k_radix_scatter, tiles, kSortThreads, 0, s, k_in, v_in, m, shift, tiles, b.hist, k_out, v_out);
        uint32_t *tk = k_in; k_in = k_out; k_out = tk;
        int *tv = v_in; v_in = v_out; v_out = tv;
    }
    // after an even number of passes the sorted data is back in keys/vals
    launch(k_count_leaves, 1, 1, 0, s, m, b.scene);
    launch(k_karras, grid_for(m), kThreads, 0, s, b.keys, b.scene, b.nodes, b.parent, vslot ? roots : nullptr,
           3 * bits);
    launch(k_leaf_map, grid_for(m), kThreads, 0, s, b.vals, b.scene, b.leaf_of_face, m);
    return cudaGetLastError();
}

cudaError_t lbvh_refit_dirty(Lbvh &b, const float4 *pts, const int4 *tris, long long max_dirty, cudaStream_t s)
{
    if (b.leaves_built < 2 || max_dirty <= 0) return cudaSuccess;
    launch(k_refit_dirty, grid_for(max_dirty), kThreads, 0, s, pts, tris, (const int *)b.vals, b.scene,
           (const int *)b.parent, b.nodes, b.claim, b.dmask, b.dcount, (const int *)b.dlist);
    return cudaGetLastError();
}

cudaError_t lbvh_refit(Lbvh &b, const float4 *pts, const int4 *tris, int m, cudaStream_t s)
{
    const long long L = b.leaves_built > m ? b.leaves_built : m;
    if (L < 2) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(b.flags, 0, (size_t)L * 4, s);
    if (e != cudaSuccess) return e;
    launch(k_refit, (int)((L + kRefitTile - 1) / kRefitTile), kRefitTile, 0, s, pts, tris, b.vals, b.scene, b.parent,
           b.nodes, b.flags);
    return cudaGetLastError();
}

}  // namespace pamo
