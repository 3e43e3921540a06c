// Reference harness -- TEST INFRASTRUCTURE (pins the CPU oracle to the reference).
//
// Compiled by oracle/build_ref.sh against the reference's own stage-2 sources
// (simp_cuda/src/cusimp_free.cu and bvh/*.cuh, included from the reference tree),
// with the reference's nvcc flags (simp_cuda/setup.py:34: -O3 --extended-lambda
// --fmad=false).  The resulting library lives only in oracle/_ref/.
//
// Entry points:
//   ref_round_canonical  one CUSimp_Free::forward round (cusimp_free.cu:891-1048)
//                        driven step by step through the reference's kernels,
//                        with one change: after create_near_tris_kernel the
//                        faces of every vertex are sorted by index, making the
//                        reference deterministic (its atomicAdd slot order,
//                        :291-304, is the only source of run-to-run variation).
//   ref_forward_raw      the unmodified CUSimp_Free::forward (timing, statistics).
//   ref_self_intersect   selfx::self_intersect on a given mesh -> face flags.
//   ref_pow2             pow(float,2) as the reference kernels evaluate it.
#include "cusimp_free.cu"

#include <cub/device/device_scan.cuh>
#include <cstdio>
#include <vector>

using namespace cusimp_free;

namespace {

CUSimp_Free g_sp;  // persistent, like the pybind CUDSP_Free object

// The reference gathers points[-1] for removed faces (bvh/self_intersect.cuh:159-173).
// Every points buffer the harness hands to the reference therefore has one spare
// element in front, so that read stays inside an allocation.
Vertex<float> *g_guard_base = nullptr;

void ensure_pts_guarded(size_t n)
{
    if (n > g_sp.allocated_pts && g_guard_base) {
        cudaFree(g_guard_base);
        g_guard_base = nullptr;
        g_sp.points = nullptr;
    }
    size_t before = g_sp.allocated_pts;
    g_sp.ensure_pts_storage_size(n);
    if (g_sp.allocated_pts != before) {
        cudaFree(g_sp.points);
        cudaMalloc((void **)&g_guard_base, (g_sp.allocated_pts + 2) * sizeof(Vertex<float>));
        cudaMemset(g_guard_base, 0, (g_sp.allocated_pts + 2) * sizeof(Vertex<float>));
        g_sp.points = g_guard_base + 1;
        // state the oracle reads stale starts at zero
        cudaMemset(g_sp.pts_map, 0, (g_sp.allocated_pts + 1) * sizeof(int));
        cudaMemset(g_sp.vertices_undo_list, 0, (g_sp.allocated_pts + 1) * sizeof(int));
        cudaMemset(g_sp.tmp_vertices_undo_list, 0, (g_sp.allocated_pts + 1) * sizeof(int));
        cudaMemset(g_sp.vertices_invalid_table, 0, (g_sp.allocated_pts + 1) * sizeof(bool));
    }
}

__global__ void harness_sort_segments(const int *first, int *near, int n_pts)
{
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_pts) return;
    int a = first[v], b = first[v + 1];
    for (int i = a + 1; i < b; ++i) {
        int x = near[i], j = i - 1;
        while (j >= a && near[j] > x) { near[j + 1] = near[j]; --j; }
        near[j + 1] = x;
    }
}

__global__ void harness_fill_int(int *p, int n, int val)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = val;
}

__global__ void harness_fill_u64(unsigned long long *p, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = ~0ull;
}

__global__ void harness_pow2(const float *x, float *y, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = pow(x[i], 2);
}

inline int nblk(long long n, int b = BLOCK_SIZE) { return (int)((n + b - 1) / b); }

void exclusive_scan(int *data, int n)
{
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, data, data, n);
    g_sp.ensure_temp_storage_size(bytes);
    cub::DeviceScan::ExclusiveSum(g_sp.temp_storage, g_sp.allocated_temp_storage_size, data, data, n);
}

void isect_flags(int n_tris, unsigned char *h_flags)
{
    int n = 0;
    cudaMemcpy(&n, g_sp.n_intersect, sizeof(int), cudaMemcpyDeviceToHost);
    int stored = 2 * n_tris - 2;  // entries the reference actually stores (self_intersect.cuh:213,291)
    if (n > stored) n = stored;
    std::vector<unsigned int> ids(n > 0 ? n : 1);
    if (n > 0) cudaMemcpy(ids.data(), g_sp.intersected_triangle_idx, n * sizeof(unsigned), cudaMemcpyDeviceToHost);
    for (int i = 0; i < n_tris; ++i) h_flags[i] = 0;
    for (int i = 0; i < n; ++i)
        if (ids[i] < (unsigned)n_tris) h_flags[ids[i]] = 1;
}

}  // namespace

extern "C" {

// stats out: [n_edges, n_collapsed_main, n_collapsed_total, n_undo_passes, n_vertices_undo, undo_count0]
int ref_round_canonical(const float *h_pts, const int *h_tris, const int *h_undo, int n_undo, int n_pts, int n_tris,
                        float scale, float threshold, int is_stuck, float *o_pts, int *o_tris, int *o_occ,
                        int *o_map, int *o_undo, int o_undo_cap, unsigned *o_cost, int o_cost_cap, int *o_collapsed,
                        int o_collapsed_cap, unsigned char *o_isect0, int *o_stats)
{
    CUSimp_Free &sp = g_sp;
    const float epsilon = 1e-3f;
    int *d_undo = nullptr;
    cudaMalloc(&d_undo, (n_undo > 0 ? n_undo : 1) * sizeof(int));
    if (n_undo > 0) cudaMemcpy(d_undo, h_undo, n_undo * sizeof(int), cudaMemcpyHostToDevice);

    // sizes first so the undo-list buffers exist (the reference allocates them on
    // the first forward; a first call with an undo list is not meaningful there)
    ensure_pts_guarded(n_pts);
    sp.n_vertices_undo = 0;
    sp.n_invalid_vertices = 0;
    int first_n = 0;
    if (is_stuck) {
        cudaMemcpy(sp.tmp_vertices_undo_list, d_undo, n_undo * sizeof(int), cudaMemcpyDeviceToDevice);
        sp.n_vertices_undo += n_undo;
        if (sp.n_vertices_undo > 0)
            rearrange_index_of_undo_vertices<<<nblk(sp.n_vertices_undo), BLOCK_SIZE>>>(sp, first_n);
        first_n += n_undo;
    } else if (n_undo != 0) {
        cudaMemset(sp.vertices_invalid_table, 0, (sp.allocated_pts + 1) * sizeof(bool));
    }
    if (n_undo != 0) {
        cudaMemcpy(sp.vertices_invalid_list, d_undo, n_undo * sizeof(int), cudaMemcpyDeviceToDevice);
        sp.n_invalid_vertices = n_undo;
        compute_invalid_vertices_table<<<nblk(n_undo), BLOCK_SIZE>>>(sp);
    }
    sp.tres = threshold;
    sp.edge_s = scale;
    sp.collapse_t = uint32_t(cusimp_free::clamp(threshold, 0.0f, COST_RANGE) / COST_RANGE * std::numeric_limits<uint32_t>::max());
    sp.resize(n_pts, n_tris);
    cudaMemcpy(sp.points, h_pts, n_pts * sizeof(Vertex<float>), cudaMemcpyHostToDevice);
    harness_fill_int<<<nblk(n_pts + 1), BLOCK_SIZE>>>(sp.pts_occ, n_pts, 1);
    cudaMemset(sp.pts_occ + n_pts, 0, sizeof(int));
    sp.ensure_tris_storage_size(n_tris);
    cudaMemcpy(sp.triangles, h_tris, n_tris * sizeof(Triangle<int>), cudaMemcpyHostToDevice);
    cudaMemcpy(sp.original_points, sp.points, n_pts * sizeof(Vertex<float>), cudaMemcpyDeviceToDevice);
    cudaMemcpy(sp.original_tris, sp.triangles, n_tris * sizeof(Triangle<int>), cudaMemcpyDeviceToDevice);

    sp.ensure_near_count_storage_size(n_pts);
    cudaMemset(sp.first_near_tris, 0, (n_pts + 1) * sizeof(int));
    count_near_tris_kernel<<<nblk(n_tris), BLOCK_SIZE>>>(sp);
    exclusive_scan(sp.first_near_tris, n_pts + 1);
    cudaMemcpy(&sp.n_near_tris, sp.first_near_tris + n_pts, sizeof(int), cudaMemcpyDeviceToHost);
    sp.ensure_near_tris_storage_size(sp.n_near_tris);
    sp.ensure_near_offset_storage_size(n_pts);
    cudaMemset(sp.near_offset, 0, (n_pts + 1) * sizeof(int));
    create_near_tris_kernel<<<nblk(n_tris), BLOCK_SIZE>>>(sp);
    harness_sort_segments<<<nblk(n_pts, 256), 256>>>(sp.first_near_tris, sp.near_tris, n_pts);  // canonical order

    sp.ensure_edge_count_storage_size(n_tris);
    cudaMemset(sp.first_edge, 0, (n_tris + 1) * sizeof(int));
    count_edge_kernel<<<nblk(n_tris), BLOCK_SIZE>>>(sp);
    exclusive_scan(sp.first_edge, n_tris + 1);
    cudaMemcpy(&sp.n_edges, sp.first_edge + n_tris, sizeof(int), cudaMemcpyDeviceToHost);
    sp.ensure_edge_storage_size(sp.n_edges);
    create_edge_kernel<<<nblk(n_tris), BLOCK_SIZE>>>(sp);

    sp.ensure_vert_Q_storage_size(n_pts);
    compute_vert_Q_kernel<<<nblk(n_pts), BLOCK_SIZE>>>(sp);
    size_t before_cost = sp.allocated_edge_cost;
    sp.ensure_edge_cost_storage_size(sp.n_edges);
    if (sp.allocated_edge_cost != before_cost) cudaMemset(sp.edge_cost, 0, (sp.allocated_edge_cost + 1) * sizeof(uint32_t));
    compute_edge_cost_kernel<<<nblk(sp.n_edges), BLOCK_SIZE>>>(sp, is_stuck != 0);
    sp.ensure_tri_min_cost_storage_size(n_tris);
    harness_fill_u64<<<nblk(n_tris), BLOCK_SIZE>>>(sp.tri_min_cost, n_tris);
    propagate_edge_cost_kernel<<<nblk(sp.n_edges), BLOCK_SIZE>>>(sp);

    cudaMalloc((void **)&sp.n_collapsed, sizeof(int));
    cudaMemset(sp.n_collapsed, 0, sizeof(int));
    cudaMalloc((void **)&sp.collapsed_edge_idx, (sp.n_edges > 0 ? sp.n_edges : 1) * sizeof(int));
    cudaMemset(sp.collapsed_edge_idx, 0, sp.n_edges * sizeof(int));
    if (sp.n_edges > 0) collapse_edge_kernel<<<nblk(sp.n_edges), BLOCK_SIZE>>>(sp);
    cudaMalloc((void **)&sp.n_intersect, sizeof(unsigned int));
    int h_main = 0;
    cudaMalloc(&sp.n_edges_undo, sizeof(int));
    cudaMemset(sp.n_edges_undo, 0, sizeof(int));
    cudaMemcpy(&h_main, sp.n_collapsed, sizeof(int), cudaMemcpyDeviceToHost);
    cudaMalloc(&sp.edges_undo, (2 * h_main > 0 ? 2 * h_main : 1) * sizeof(int));
    if (n_tris > 0) remove_invalid_faces<<<nblk(n_tris), BLOCK_SIZE>>>(sp);
    if (sp.n_edges > 0) remove_line_edge_collapse<<<nblk(sp.n_edges), BLOCK_SIZE>>>(sp);
    int h_total = 0;
    cudaMemcpy(&h_total, sp.n_collapsed, sizeof(int), cudaMemcpyDeviceToHost);
    if (o_cost) {
        int n = sp.n_edges < o_cost_cap ? sp.n_edges : o_cost_cap;
        cudaMemcpy(o_cost, sp.edge_cost, n * sizeof(unsigned), cudaMemcpyDeviceToHost);
    }
    if (o_collapsed) {
        int n = h_total < o_collapsed_cap ? h_total : o_collapsed_cap;
        cudaMemcpy(o_collapsed, sp.collapsed_edge_idx, n * sizeof(int), cudaMemcpyDeviceToHost);
    }

    selfx::self_intersect(&sp, n_pts, n_tris, epsilon);
    if (o_isect0) isect_flags(n_tris, o_isect0);
    cudaMemset(sp.n_edges_undo, 0, sizeof(int));
    if (h_main > 0) get_undo_candidate_kernel<<<nblk(h_main), BLOCK_SIZE>>>(sp);
    cudaDeviceSynchronize();
    int h_nundo = 0;
    cudaMemcpy(&h_nundo, sp.n_edges_undo, sizeof(int), cudaMemcpyDeviceToHost);
    int undo0 = h_nundo;
    sp.n_vertices_undo += 2 * h_nundo;
    int it = 0;
    while (h_nundo != 0) {
        it++;
        undo_collapse_kernel<<<nblk(h_main), BLOCK_SIZE>>>(sp);
        rearrange_index_of_undo_vertices<<<nblk(sp.n_vertices_undo), BLOCK_SIZE>>>(sp, first_n);
        cudaDeviceSynchronize();
        first_n += 2 * h_nundo;
        selfx::self_intersect(&sp, n_pts, n_tris, epsilon);
        cudaDeviceSynchronize();
        cudaMemset(sp.n_edges_undo, 0, sizeof(int));
        get_undo_candidate_kernel<<<nblk(h_main), BLOCK_SIZE>>>(sp);
        cudaDeviceSynchronize();
        cudaMemcpy(&h_nundo, sp.n_edges_undo, sizeof(int), cudaMemcpyDeviceToHost);
        sp.n_vertices_undo += 2 * h_nundo;
        if (it == 5) break;
    }
    cudaMemcpy(sp.pts_map, sp.pts_occ, (n_pts + 1) * sizeof(int), cudaMemcpyDeviceToDevice);
    exclusive_scan(sp.pts_map, n_pts + 1);
    cudaFree(sp.n_intersect);
    sp.n_intersect = nullptr;
    cudaFree(d_undo);

    cudaMemcpy(o_pts, sp.points, n_pts * sizeof(Vertex<float>), cudaMemcpyDeviceToHost);
    cudaMemcpy(o_tris, sp.triangles, n_tris * sizeof(Triangle<int>), cudaMemcpyDeviceToHost);
    cudaMemcpy(o_occ, sp.pts_occ, n_pts * sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(o_map, sp.pts_map, n_pts * sizeof(int), cudaMemcpyDeviceToHost);
    int nu = sp.n_vertices_undo < o_undo_cap ? sp.n_vertices_undo : o_undo_cap;
    if (nu > 0) cudaMemcpy(o_undo, sp.vertices_undo_list, nu * sizeof(int), cudaMemcpyDeviceToHost);
    o_stats[0] = sp.n_edges;
    o_stats[1] = h_main;
    o_stats[2] = h_total;
    o_stats[3] = it;
    o_stats[4] = sp.n_vertices_undo;
    o_stats[5] = undo0;
    cudaError_t err = cudaDeviceSynchronize();
    return err == cudaSuccess ? 0 : (int)err;
}

// The unmodified reference round on device buffers (d_pts/d_tris are device
// pointers, as PaMO.run passes them).  Results stay in the harness's state and
// are read with ref_state().
int ref_forward_raw(const float *d_pts, const int *d_tris, const int *d_undo, int n_undo, int n_pts, int n_tris,
                    float scale, float threshold, int is_stuck, int init)
{
    ensure_pts_guarded(n_pts);
    g_sp.forward((Vertex<float> *)d_pts, (Triangle<int> *)d_tris, (int *)d_undo, n_undo, n_pts, n_tris, scale,
                 threshold, is_stuck != 0, init != 0);
    cudaError_t err = cudaDeviceSynchronize();
    // forward launches get_undo_candidate_kernel with a zero-block grid when no
    // edge collapsed (cusimp_free.cu:1017); that launch only records
    // cudaErrorInvalidConfiguration as the thread's last error.  Clear it so the
    // caller's next launch check does not report it.
    cudaGetLastError();
    return err == cudaSuccess ? 0 : (int)err;
}

// Device pointers of the reference state after a round:
// out[0]=points, [1]=triangles, [2]=pts_occ, [3]=pts_map, [4]=vertices_undo_list; counts in n_out.
void ref_state(void **out, int *n_out)
{
    out[0] = g_sp.points;
    out[1] = g_sp.triangles;
    out[2] = g_sp.pts_occ;
    out[3] = g_sp.pts_map;
    out[4] = g_sp.vertices_undo_list;
    n_out[0] = g_sp.n_pts;
    n_out[1] = g_sp.n_tris;
    n_out[2] = g_sp.n_vertices_undo;
}

// Clones the round outputs into caller buffers, as pybind.cpp:74-100 clones them.
int ref_copy_state(float *d_pts, int *d_tris, int *d_occ, int *d_map, int *d_undo)
{
    cudaMemcpy(d_pts, g_sp.points, g_sp.n_pts * sizeof(Vertex<float>), cudaMemcpyDeviceToDevice);
    cudaMemcpy(d_tris, g_sp.triangles, g_sp.n_tris * sizeof(Triangle<int>), cudaMemcpyDeviceToDevice);
    cudaMemcpy(d_occ, g_sp.pts_occ, g_sp.n_pts * sizeof(int), cudaMemcpyDeviceToDevice);
    cudaMemcpy(d_map, g_sp.pts_map, g_sp.n_pts * sizeof(int), cudaMemcpyDeviceToDevice);
    if (d_undo && g_sp.n_vertices_undo > 0)
        cudaMemcpy(d_undo, g_sp.vertices_undo_list, g_sp.n_vertices_undo * sizeof(int), cudaMemcpyDeviceToDevice);
    cudaError_t err = cudaDeviceSynchronize();
    return err == cudaSuccess ? 0 : (int)err;
}

// selfx::self_intersect (bvh/self_intersect.cuh:151-392) on a host mesh; writes a
// 0/1 flag per face for the faces in the reported pair list.
int ref_self_intersect(const float *h_pts, const int *h_tris, int n_pts, int n_tris, unsigned char *o_flags)
{
    CUSimp_Free &sp = g_sp;
    ensure_pts_guarded(n_pts);
    sp.ensure_tris_storage_size(n_tris);
    sp.resize(n_pts, n_tris);
    cudaMemcpy(sp.points, h_pts, n_pts * sizeof(Vertex<float>), cudaMemcpyHostToDevice);
    cudaMemcpy(sp.triangles, h_tris, n_tris * sizeof(Triangle<int>), cudaMemcpyHostToDevice);
    harness_fill_int<<<nblk(n_pts + 1), BLOCK_SIZE>>>(sp.pts_occ, n_pts, 1);
    int *n_col = nullptr;
    cudaMalloc(&n_col, sizeof(int));
    cudaMemset(n_col, 0, sizeof(int));
    sp.n_collapsed = n_col;
    cudaMalloc((void **)&sp.n_intersect, sizeof(unsigned int));
    selfx::self_intersect(&sp, n_pts, n_tris, 1e-3f);
    isect_flags(n_tris, o_flags);
    cudaFree(sp.n_intersect);
    sp.n_intersect = nullptr;
    cudaFree(n_col);
    cudaError_t err = cudaDeviceSynchronize();
    return err == cudaSuccess ? 0 : (int)err;
}

int ref_pow2(const float *h_x, float *h_y, int n)
{
    float *dx = nullptr, *dy = nullptr;
    cudaMalloc(&dx, n * sizeof(float));
    cudaMalloc(&dy, n * sizeof(float));
    cudaMemcpy(dx, h_x, n * sizeof(float), cudaMemcpyHostToDevice);
    harness_pow2<<<nblk(n, 256), 256>>>(dx, dy, n);
    cudaMemcpy(h_y, dy, n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dy);
    cudaError_t err = cudaDeviceSynchronize();
    return err == cudaSuccess ? 0 : (int)err;
}

}  // extern "C"
