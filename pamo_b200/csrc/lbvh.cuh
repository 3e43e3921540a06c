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

#include <cooperative_groups.h>

#include "common.cuh"

namespace pamo {

constexpr int kRefitTile = 256;  // leaves per refit block
// radix-sort tile of lbvh_build (threads x items per thread); Lbvh::hist holds
// 256 counts per tile
constexpr int kLbvhSortThreads = 256;
constexpr int kLbvhSortItems = 8;
constexpr int kLbvhSortTile = kLbvhSortThreads * kLbvhSortItems;
constexpr int kRefitTileShift = 8;
static_assert(kRefitTile == 1 << kRefitTileShift, "refit tile");

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
    // [2*cap]: internal nodes then leaves; (p << 2) | tile << 1 | is_right, -1 for
    // the root, where `tile` says that the parent's leaves all lie in one aligned
    // run of kRefitTile leaves (merged in shared memory by k_refit)
    int *parent = nullptr;
    int *flags = nullptr;       // [cap] refit arrival counters
    int *leaf_of_face = nullptr;  // [cap]: sorted position of each face, -1 if not a leaf
    int *scene = nullptr;       // 6 ordered ints + n_dead + n_leaves
    int sort_tiles = 0;
    long long leaves_built = 0;  // faces of the last build: bound on the leaf count
    // incremental refit (lbvh_mark_dirty_leaf / lbvh_refit_dirty); all zero between refits
    int *claim = nullptr;   // [cap] leaf listed as dirty
    int *dmask = nullptr;   // [cap] per inner node: which children hold a dirty leaf (bit 0 left, 1 right)
    int *dcount = nullptr;  // [cap] per inner node: dirty children merged so far
    int *dlist = nullptr;   // [cap] dirty leaves; their count is scene[9]

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

// Incremental refit, for boxes that were all up to date before some faces
// changed: the caller lists the changed faces' leaves with lbvh_mark_dirty_leaf
// (in a kernel, after zeroing scene[9]); lbvh_refit_dirty then recomputes those
// leaves and, bottom-up, exactly the inner nodes above them (a node is merged by
// the last of its dirty children to arrive).  Leaves the marks zero again.
__device__ __forceinline__ void lbvh_mark_dirty_leaf(int p, int L, const int *parent, int *claim, int *dmask,
                                                     int *dlist, int *scene)
{
    if (atomicExch(&claim[p], 1) != 0) return;  // listed already
    {  // one counter atomic per group of lanes listing together
        cooperative_groups::coalesced_group g = cooperative_groups::coalesced_threads();
        int base = 0;
        if (g.thread_rank() == 0) base = atomicAdd(&scene[9], (int)g.size());
        dlist[g.shfl(base, 0) + (int)g.thread_rank()] = p;
    }
    int code = parent[(L - 1) + p];
    // mark the path to the root; a node already marked has its path marked (or
    // being marked) by the leaf that got there first
    for (int depth = 0; depth < 256 && code >= 0; ++depth) {
        const int node = code >> 2;
        if (atomicOr(&dmask[node], 1 << (code & 1)) != 0) break;
        code = parent[node];
    }
}

cudaError_t lbvh_refit_dirty(Lbvh &b, const float4 *pts, const int4 *tris, long long max_dirty, cudaStream_t s);

}  // namespace pamo
