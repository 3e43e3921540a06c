// Mesh preparation for stage 3 on the device: the unique edges and hinges of a
// closed 2-manifold (the device form of pamo_mesh_hinges), and the check for
// vertices that coincide after rounding to 8 decimals (the merge that
// trimesh.Trimesh(process=True) applies to the stage-2 result before stage 3,
// simp_cuda/pamo/__init__.py:193-203).
#include <cstdint>

#include "../../include/pamo_b200.h"
#include "common.cuh"
#include "scan.cuh"

namespace pamo {
namespace {

enum { MP_BAD_INDEX = 0, MP_NOT_MANIFOLD = 1, MP_DUPLICATE = 2, MP_PROBE = 3, MP_COUNT = 4 };

struct Scratch {
    void *p = nullptr;
    cudaStream_t s = nullptr;
    Scratch(size_t bytes, cudaStream_t st) : s(st)
    {
        if (bytes && cudaMallocAsync(&p, bytes, st) != cudaSuccess) p = nullptr;
    }
    ~Scratch()
    {
        if (p) cudaFreeAsync(p, s);
    }
    Scratch(const Scratch &) = delete;
    Scratch &operator=(const Scratch &) = delete;
    template <class T> T *as() const { return static_cast<T *>(p); }
};

// Directed edge e (corner k -> k + 1 of face f, e = k * m + f: the order the
// host builder numbers them in).
__device__ __forceinline__ void half_edge(const int *tris, int m, long long e, int &from, int &to, int &opp)
{
    const int k = (int)(e / m), f = (int)(e - (long long)k * m);
    from = tris[3 * (size_t)f + k];
    to = tris[3 * (size_t)f + (k + 1) % 3];
    opp = tris[3 * (size_t)f + (k + 2) % 3];
}

__global__ void k_mh_count(const int *tris, int m, int n_pts, int *cnt, int *flags)
{
    PAMO_GRID_STRIDE(e, 3LL * m)
    {
        int a, b, c;
        half_edge(tris, m, e, a, b, c);
        if (a < 0 || a >= n_pts || b < 0 || b >= n_pts || c < 0 || c >= n_pts) {
            atomicExch(flags + MP_BAD_INDEX, 1);
            continue;
        }
        atomicAdd(cnt + min(a, b), 1);
    }
}

__global__ void k_mh_fill(const int *tris, int m, int n_pts, const int *start, int *cursor, int *order)
{
    PAMO_GRID_STRIDE(e, 3LL * m)
    {
        int a, b, c;
        half_edge(tris, m, e, a, b, c);
        if (a < 0 || a >= n_pts || b < 0 || b >= n_pts || c < 0 || c >= n_pts) continue;  // flagged by the count
        const int lo = min(a, b);
        order[start[lo] + atomicAdd(cursor + lo, 1)] = (int)e;
    }
}

// One thread per vertex v: its bucket (the directed edges whose smaller vertex
// is v) sorted by (larger vertex, edge number) -- the host builder's stable
// counting sort then stable insertion sort -- and paired: each key exactly
// twice, once each way.  Edge row start[v] / 2 + j of the output is the j-th
// pair of the bucket, so rows ascend by lo * n_pts + hi as the host's do.
__global__ void k_mh_pair(const int *tris, int m, int n_pts, const int *start, int *order, int *edges, int *hinges,
                          int *flags)
{
    PAMO_GRID_STRIDE(vv, n_pts)
    {
        const int v = (int)vv;
        const int a = start[v], b = start[v + 1];
        if (a == b) continue;
        if ((a & 1) || ((b - a) & 1)) {
            atomicExch(flags + MP_NOT_MANIFOLD, 1);
            continue;
        }
        auto hi_of = [&](int e) {
            int x, y, z;
            half_edge(tris, m, e, x, y, z);
            return max(x, y);
        };
        for (int i = a + 1; i < b; ++i) {  // insertion sort by (hi, e)
            const int x = order[i], kx = hi_of(x);
            int j = i - 1;
            while (j >= a) {
                const int y = order[j], ky = hi_of(y);
                if (ky < kx || (ky == kx && y < x)) break;
                order[j + 1] = y;
                --j;
            }
            order[j + 1] = x;
        }
        for (int i = a; i < b; i += 2) {
            int f0, t0, o0, f1, t1, o1;
            half_edge(tris, m, order[i], f0, t0, o0);
            half_edge(tris, m, order[i + 1], f1, t1, o1);
            const int h = max(f0, t0);
            bool ok = v != h && max(f1, t1) == h && (f0 < t0) != (f1 < t1);
            if (ok && i + 2 < b) ok = hi_of(order[i + 2]) != h;  // the next key must differ
            if (!ok) {
                atomicExch(flags + MP_NOT_MANIFOLD, 1);
                break;
            }
            const long long row = a / 2 + (i - a) / 2;
            edges[2 * row] = v;
            edges[2 * row + 1] = h;
            hinges[4 * row] = f0 < t0 ? o0 : o1;
            hinges[4 * row + 1] = v;
            hinges[4 * row + 2] = h;
            hinges[4 * row + 3] = f0 < t0 ? o1 : o0;
        }
    }
}

// numpy's round(x, 8): x * 1e8 rounded to an integer (ties to even), / 1e8;
// -0 becomes +0 so that equal values hash alike
__device__ __forceinline__ double round8(float x)
{
    return rint((double)x * 1e8) / 1e8 + 0.0;
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long h)
{
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdULL;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ULL;
    h ^= h >> 33;
    return h;
}

// Every vertex's rounded position into an open-addressing table (linear
// probing, at most one pass over the table); a vertex meeting an earlier one
// with the same rounded position sets MP_DUPLICATE.
__global__ void k_mc_insert(const float *pts, int n, int *table, unsigned mask, int *flags)
{
    PAMO_GRID_STRIDE(ii, n)
    {
        const int i = (int)ii;
        const double x = round8(pts[3 * (size_t)i]), y = round8(pts[3 * (size_t)i + 1]),
                     z = round8(pts[3 * (size_t)i + 2]);
        unsigned long long h = mix64((unsigned long long)__double_as_longlong(x));
        h = mix64(h ^ (unsigned long long)__double_as_longlong(y));
        h = mix64(h ^ (unsigned long long)__double_as_longlong(z));
        unsigned slot = (unsigned)h & mask;
        bool placed = false;
        for (unsigned probe = 0; probe <= mask; ++probe) {
            const int prev = atomicCAS(table + slot, -1, i);
            if (prev < 0) {
                placed = true;
                break;
            }
            if (round8(pts[3 * (size_t)prev]) == x && round8(pts[3 * (size_t)prev + 1]) == y &&
                round8(pts[3 * (size_t)prev + 2]) == z) {
                atomicExch(flags + MP_DUPLICATE, 1);
                placed = true;
                break;
            }
            slot = (slot + 1) & mask;
        }
        if (!placed) atomicExch(flags + MP_PROBE, 1);  // cannot happen: the table holds 2n slots
    }
}

}  // namespace
}  // namespace pamo

using namespace pamo;

extern "C" int pamo_mesh_hinges_device(const int *d_tris, int n_tris, int n_pts, int *d_edges, int *d_hinges,
                                       int *out_n_edges, void *stream)
{
    if (!out_n_edges || n_tris < 0 || n_pts < 0 || (n_tris && (!d_tris || !d_edges || !d_hinges || n_pts == 0)))
        return PAMO_ERR_INVALID_ARG;
    *out_n_edges = 0;
    if (n_tris == 0) return PAMO_OK;
    const long long nd = 3LL * n_tris;
    if (nd % 2) return PAMO_ERR_CAPACITY;
    int dev;
    if (cudaGetDevice(&dev) != cudaSuccess) return PAMO_ERR_NO_DEVICE;
    cudaStream_t s = (cudaStream_t)stream;
    PAMO_CUDA_TRY(retain_pool_memory());
    const long long n1 = (long long)n_pts + 1;
    Scratch cnt((size_t)n1 * 4, s), start((size_t)n1 * 4, s), cursor((size_t)n_pts * 4, s), order((size_t)nd * 4, s),
        flags(MP_COUNT * 4, s), scan_tmp((size_t)scan_scratch_ints(n1) * 4, s);
    if (!cnt.p || !start.p || !cursor.p || !order.p || !flags.p || !scan_tmp.p) return PAMO_ERR_OOM;
    PAMO_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, (size_t)n1 * 4, s));
    PAMO_CUDA_TRY(cudaMemsetAsync(cursor.p, 0, (size_t)n_pts * 4, s));
    PAMO_CUDA_TRY(cudaMemsetAsync(flags.p, 0, MP_COUNT * 4, s));
    launch(k_mh_count, grid_for(nd), kThreads, 0, s, d_tris, n_tris, n_pts, cnt.as<int>(), flags.as<int>());
    PAMO_CUDA_TRY(scan_scratch_init(scan_tmp.as<int>(), scan_scratch_ints(n1), s));
    PAMO_CUDA_TRY(exclusive_scan(cnt.as<int>(), start.as<int>(), n1, nullptr, scan_tmp.as<int>(), nullptr, s));
    launch(k_mh_fill, grid_for(nd), kThreads, 0, s, d_tris, n_tris, n_pts, (const int *)start.as<int>(),
           cursor.as<int>(), order.as<int>());
    launch(k_mh_pair, grid_for(n_pts), kThreads, 0, s, d_tris, n_tris, n_pts, (const int *)start.as<int>(),
           order.as<int>(), d_edges, d_hinges, flags.as<int>());
    int h_flags[MP_COUNT];
    PAMO_CUDA_TRY(cudaMemcpyAsync(h_flags, flags.p, sizeof(h_flags), cudaMemcpyDeviceToHost, s));
    PAMO_CUDA_TRY(cudaStreamSynchronize(s));
    if (h_flags[MP_BAD_INDEX]) return PAMO_ERR_INVALID_ARG;
    if (h_flags[MP_NOT_MANIFOLD]) return PAMO_ERR_CAPACITY;
    *out_n_edges = (int)(nd / 2);
    return PAMO_OK;
}

extern "C" int pamo_merge_check_device(const float *d_points, int n_pts, int *out_has_duplicates, void *stream)
{
    if (!out_has_duplicates || n_pts < 0 || (n_pts && !d_points)) return PAMO_ERR_INVALID_ARG;
    *out_has_duplicates = 0;
    if (n_pts < 2) return PAMO_OK;
    int dev;
    if (cudaGetDevice(&dev) != cudaSuccess) return PAMO_ERR_NO_DEVICE;
    cudaStream_t s = (cudaStream_t)stream;
    PAMO_CUDA_TRY(retain_pool_memory());
    unsigned size = 1024;
    while (size < 2u * (unsigned)n_pts) size <<= 1;
    Scratch table((size_t)size * 4, s), flags(MP_COUNT * 4, s);
    if (!table.p || !flags.p) return PAMO_ERR_OOM;
    PAMO_CUDA_TRY(cudaMemsetAsync(table.p, 0xFF, (size_t)size * 4, s));
    PAMO_CUDA_TRY(cudaMemsetAsync(flags.p, 0, MP_COUNT * 4, s));
    launch(k_mc_insert, grid_for(n_pts), kThreads, 0, s, d_points, n_pts, table.as<int>(), size - 1, flags.as<int>());
    int h_flags[MP_COUNT];
    PAMO_CUDA_TRY(cudaMemcpyAsync(h_flags, flags.p, sizeof(h_flags), cudaMemcpyDeviceToHost, s));
    PAMO_CUDA_TRY(cudaStreamSynchronize(s));
    if (h_flags[MP_PROBE]) return PAMO_ERR_DEVICE;
    *out_has_duplicates = h_flags[MP_DUPLICATE] ? 1 : 0;
    return PAMO_OK;
}
