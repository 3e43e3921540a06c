// Stage 1 of PaMO.run on the device (sm_100a): remeshing through a narrow-band
// signed distance field and dual marching cubes
// (simp_cuda/pamo/__init__.py:60-120,130-142; the reference calls
// torchcumesh2sdf.get_sdf and pdmc.DMC, restated here -- see stage1.cu).
#pragma once

#include "common.cuh"
#include "stage2.cuh"  // Profiler

namespace pamo {
namespace s1 {

struct Stage1 {
    int R = 0;
    long long cap_tris = 0, cap_grid = 0, cap_cells = 0, cap_edges = 0, cap_verts = 0, cap_quads = 0, cap_tiles = 0;
    float *tris = nullptr;              // [m][9] normalised triangles (float32, the reference's arithmetic)
    unsigned long long *field = nullptr;  // [R^3]: squared distance bits, then the field as double
    uint8_t *state = nullptr;           // [R^3] flood fill: 0 near the surface, 1 free, 2 outside
    uint8_t *tile_dirty = nullptr;      // [2 x tiles] flood-fill tiles to visit (two sets used in turn)
    int *cell_cnt = nullptr;            // [C^3 + 1] patches per cell, then their first vertex
    int *edge_cnt = nullptr;            // [3 R^3 + 1] quads per grid edge (0/1), then the quad index
    int *scan_cells = nullptr, *scan_edges = nullptr, *scan_quads = nullptr;  // scan scratch
    int4 *quads = nullptr;              // [cap_quads]
    int *q_first = nullptr;             // [cap_quads + 1] first-configuration flags, then their prefix
    float *verts = nullptr;             // [cap_verts][3] in the centred frame
    int *faces = nullptr;               // [2 cap_quads][3]
    int *dev = nullptr;                 // [16] counters: [0] min x [1] min y [2] min z (ordered ints),
                                        // [3] max (ordered), [4] flood changed, [5] flood budget out
    int *h_dev = nullptr;               // pinned copy
    float *mean_dev = nullptr;          // [4] the centring mean (tris_mean)
    int n_verts = 0, n_tris = 0;
    float offset[3] = {0, 0, 0};        // tris_mean of the input (added back after stage 2)
    Profiler *prof = nullptr;           // the context's phase timer (optional)

    int ensure(long long m, int R_);
    int ensure_out(long long nv, long long nq);
    void release();
};

// Runs stage 1 on faces (d_points [n,3], d_tris [m,3]) whose centring mean
// (numpy float32 order) is in mean_dev[3]; resolution R.  The result (in the
// centred frame) is in S.verts / S.faces, sizes in S.n_verts / S.n_tris.
int remesh(Stage1 &S, const float *d_points, const int *d_tris, int n_pts, int m, const float *mean_dev, int R,
           cudaStream_t s);

}  // namespace s1
}  // namespace pamo
