// Linear BVH over the faces of one mesh round (used by the stage-2 undo check).
//
// Build: 30-bit Morton code of each face's box centre (10 bits per axis over the
// scene box) -> stable LSD radix sort (4 x 8-bit digits, hand written) ->
// Karras hierarchy over 64-bit keys (code << 32 | sorted position) -> bottom-up
// refit.  Internal node i (0 <= i < L-1) stores both child boxes inline (64 B),
// so traversal reads one node per step and tests the two children.
//
// The leaf set is fixed per build (faces live at the build, sorted by their
// geometry then); a caller that removes and renumbers faces may keep the tree by
// rewriting the leaves' face indices (-1 for a removed face).  Refit recomputes every leaf box from the current
// geometry (a dead face gets the empty box lo=+inf, hi=-inf, which overlaps
// nothing) and rebuilds the inner boxes, so the undo passes never rebuild the
// hierarchy.
#pragma once

#include "common.cuh"

namespace pamo {

struct __align__(16) BvhNode {
    float4 llo;  // .w = left child (int bits): >= 0 internal node, < 0 leaf ~position
    float4 lhi;
    float4 rlo;  // .w = right child
    float4 rhi;
};

struct Lbvh {
    long long cap = 0;        // faces
    uint32_t *keys = nullptr;  // morton keys (ping)
    uint32_t *keys2 = nullptr;
    int *vals = nullptr;  // face index per sorted position (ping)
    int *vals2 = nullptr;
    int *hist = nullptr;        // radix digit counts [256 * tiles]
    int *hist_scratch = nullptr;
    BvhNode *nodes = nullptr;   // [cap]
    int *parent = nullptr;      // [2*cap]: internal nodes then leaves; (p<<1)|is_right, -1 for root
    int *flags = nullptr;       // [cap] refit arrival counters
    int *leaf_of_face = nullptr;  // [cap]: sorted position of each face, -1 if not a leaf
    int *scene = nullptr;       // 6 ordered ints + n_dead + n_leaves
    int sort_tiles = 0;
    long long leaves_built = 0;  // faces of the last build: bound on the leaf count

    cudaError_t ensure(long long n_faces);
    void release();
};

// Builds the hierarchy for faces [0, m): leaves are the faces live in `tris`
// (the round input), ordered by the Morton code of their box centre.  For a
// batch of meshes, vslot gives each vertex's mesh rank (< n_ranks): each mesh
// gets its own subtree, whose start node (internal index, or ~leaf position for
// a one-face mesh) is written to roots[rank].
cudaError_t lbvh_build(Lbvh &b, const float4 *pts, const int4 *tris, int m, cudaStream_t s,
                       const int *vslot = nullptr, int n_ranks = 0, int *roots = nullptr);

// Recomputes all boxes from the current geometry (pts, tris).  A leaf whose face
// index is negative (a face removed after the build) gets the empty box.
cudaError_t lbvh_refit(Lbvh &b, const float4 *pts, const int4 *tris, int m, cudaStream_t s);

}  // namespace pamo
