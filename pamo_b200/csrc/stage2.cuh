// Stage-2 simplification state and round driver (host side).
#pragma once

#include <vector>

#include "common.cuh"
#include "lbvh.cuh"

namespace pamo {

// Device counters of one round (one struct, copied to the host in one go).
struct RoundCounters {
    int n_main;          // collapsed edges chosen by the independent set
    int n_line;          // coincident-endpoint edges collapsed afterwards
    int n_total;         // n_main + n_line
    int n_considered;    // collapsed-list prefix the undo check looks at
    int n_undo;          // undo edges found by the last check
    int n_pairs;         // candidate pairs found by the last query
    int pair_overflow;   // pairs dropped for lack of buffer space
    int stack_overflow;  // traversals that ran out of stack
    int n_pts_next;      // compaction result
    int n_tris_next;
    int n_edges;
    int n_query;         // faces in this pass's query list
    int scan_fault;      // a prefix scan's wait ran out (see scan.cuh)
    int pad[3];
};

// ---------------------------------------------------------------------------
// Batches: several meshes packed into one round.
//
// The meshes of a batch sit one after another in the packed round arrays
// (vertices, faces, and so the edges emitted per face, keep their order), so
// every per-vertex, per-face and per-edge kernel runs unchanged over the packed
// arrays: a mesh never shares a vertex with another one, and the independent
// set, the collapses and the cleanup only look at one-rings.  What the
// reference keeps per simplifier is kept per mesh: the state it reads stale
// from earlier rounds (edge costs, the previous vertex map, the undo lists, the
// invalid-vertex table) lives in a region of the mesh's own (`SlotInfo`
// pointers, indexed by mesh-local numbers), the parameters (scale, threshold,
// stuck mode) are per mesh, the undo check's collapsed-list window is per mesh,
// and the hierarchy keeps each mesh in its own subtree (the mesh's rank is the
// top of the sort key), which each query starts from.
struct SlotInfo {        // uploaded by the host before each round, indexed by rank
    int vert_off, n;     // packed vertex range of the mesh
    int face_off, m;     // packed face range
    int is_stuck;
    int n_undo_in;       // entries of undo_prev from the previous round
    int clear_invalid;   // clear the invalid table before marking (not stuck, list non-empty)
    uint32_t collapse_t;
    float tres;          // threshold
    int pass_first, pass_count;  // undo pass: rearrangement window of the undo list
    int nvu;             // undo-list length at the end of the round
    int in_undo;         // the mesh's undo loop still runs: its faces are queried this pass
    const float *scale;  // device scalar: the mesh's scale (max bbox extent)
    uint32_t *edge_cost; // [3 m0 + 1] edge costs (stale between rounds)
    int *pts_map;        // [n0 + 1] the previous round's vertex map
    int *undo_list;      // [cap_undo]
    int *tmp_undo;       // [cap_undo]
    int *undo_prev;      // [cap_undo] copy of the previous round's undo list
    uint8_t *invalid;    // [n0 + 1] invalid-vertex table
    long long cap_v;     // n0 + 1
    long long cap_undo;  // entries of each undo region
};

struct SlotCounters {    // written on the device during a round, read by the host
    int edge_off, n_edges;
    int main_off, n_main;
    int line_off, n_line;
    int cand_off, n_considered;
    int undo_off, n_undo;
    int vert_off_next, n_next;
    int face_off_next, m_next;
    int pad[2];
};

// Optional per-phase device timing (CUDA events on the round's stream, read at
// the round's synchronisation points).
enum Phase {
    PH_SETUP = 0,   // round init, face pass A, CSR/edge scans, face pass B, quadrics
    PH_LBVH_BUILD,  // Morton codes, radix sort, hierarchy
    PH_EDGE_COST,   // k_edge_cost
    PH_COLLAPSE,    // k_collapse + collapsed-list compaction
    PH_CLEANUP,     // degenerate faces, coincident-endpoint collapses
    PH_REFIT,       // leaf boxes + bottom-up refit
    PH_QUERY,       // hierarchy traversal -> candidate pairs
    PH_PAIRS,       // triangle-pair tests
    PH_UNDO,        // undo candidates, restore, list rearrangement
    PH_COMPACT,     // pts_map scan + compaction for the next round
    PH_S3_CLOSEST,  // stage 3: closest points on the ground truth
    PH_S3_DETECT,   // stage 3: hierarchy refits + contact detection (with its sync)
    PH_S3_DIFF,     // stage 3: energy, gradient, diagonal, hinge / contact blocks
    PH_S3_CG,       // stage 3: Jacobi-PCG iterations
    PH_S3_CCD,      // stage 3: clamp + additive CCD
    PH_S3_LINE,     // stage 3: line-search energies
    PH_S1_PREP,     // stage 1: centring mean, normalisation
    PH_S1_DIST,     // stage 1: narrow-band unsigned distances
    PH_S1_FLOOD,    // stage 1: flood fill of the outside, signed field
    PH_S1_DMC,      // stage 1: dual marching cubes, quad split
    PH_COUNT
};

struct Profiler {
    bool on = false;
    double ms[PH_COUNT] = {0};
    long long calls[PH_COUNT] = {0};
    static constexpr int kPool = 256;
    cudaEvent_t ev[kPool] = {};
    int used = 0;
    int marks[kPool / 2][2] = {};  // (phase, first event index)
    int n_marks = 0;
    int open_phase = -1;

    void begin(int phase, cudaStream_t s);
    void end(cudaStream_t s);
    void collect();  // after the stream was synchronised
    void reset();
    void release();
};

struct Stage2 {
    int device = 0;
    Profiler prof;
    std::vector<int> round_faces;  // faces entering each round of the last loop
    long long cap_pts = 0, cap_tris = 0, cap_edges = 0, cap_undo = 0, cap_pairs = 0;

    // persistent between rounds (the reference reads these stale)
    uint32_t *edge_cost = nullptr;
    int *pts_map = nullptr;
    int *undo_list = nullptr;
    int *tmp_undo = nullptr;
    uint8_t *invalid_table = nullptr;

    // round input ("original" snapshot) and working copies
    float4 *opts = nullptr, *pts = nullptr;
    int4 *otris = nullptr, *tris = nullptr;
    int *occ = nullptr;
    int *first_near = nullptr, *cursor = nullptr, *near_tris = nullptr;
    int *first_edge = nullptr;
    int2 *edges = nullptr;
    float4 *plane = nullptr;
    float4 *elen4 = nullptr;  // per face: lengths of edges (i,j), (j,k), (k,i)
    int *nxt = nullptr;       // per CSR slot: the vertex after the slot's vertex in the face
    float4 *quad = nullptr;   // 3 float4 per vertex (10 used)
    unsigned long long *vmin = nullptr;
    int *eflag = nullptr;
    int *collapsed = nullptr;
    uint8_t *active = nullptr;
    uint8_t *isect = nullptr;
    int *uflag = nullptr;
    int *undo_edges = nullptr;
    int *fflag = nullptr;  // face compaction flags
    uint2 *pairs = nullptr;
    int *scan_scratch = nullptr;
    long long scan_scratch_len = 0;
    int *dev_misc = nullptr;  // scalars: [0] tris_mean-bits etc.
    RoundCounters *dcnt = nullptr;
    RoundCounters *hcnt = nullptr;  // pinned
    float *h_scalars = nullptr;     // pinned: [0..2] offset, [3] scale
    Lbvh bvh;
    // The hierarchy of the previous round, its leaves renumbered by compact():
    // reused (refit only) while enough of its leaves are still faces.
    bool bvh_carried = false;
    long long bvh_leaves = 0;  // faces the hierarchy was built over
    bool bvh_boxes_valid = false;  // every box matches the geometry of the last refit

    // batch mode (see SlotInfo); unused by the single-mesh rounds
    int n_slots = 0, cap_slots = 0;
    SlotInfo *slots = nullptr;       // device [cap_slots]
    SlotInfo *hslots = nullptr;      // pinned host copy
    SlotCounters *scnt = nullptr;    // device [cap_slots]
    SlotCounters *hscnt = nullptr;   // pinned host copy
    int *vslot = nullptr;            // device [cap_pts + 1]: rank of each packed vertex
    int *roots = nullptr;            // device [cap_slots]: subtree of each rank in the hierarchy
    int *line_list = nullptr;        // device [cap_edges + 1]
    int *cand = nullptr;             // device [cap_edges + 1]: per-mesh undo-candidate windows
    int *gmap = nullptr;             // device [cap_pts + 1]: packed vertex map

    // Quality mode (no reference counterpart; off by default): FP64 quadrics,
    // the collapse position from the quadric's minimiser instead of the
    // midpoint, and the self-intersection undo decided with exact predicates.
    bool quality = false;
    double *quad64 = nullptr;  // [10 per vertex] FP64 quadrics
    float4 *epos = nullptr;    // [per edge] the collapse position chosen by the edge cost
    long long cap_q64 = 0, cap_epos = 0;
    int ensure_quality(long long n_pts, long long n_edges);

    // input staging for the per-round ABI ([n,3] layouts)
    // results of the device loop
    int res_n_pts = 0, res_n_tris = 0, res_rounds = 0;
    float offset[3] = {0, 0, 0};
    long long last_stats[8] = {0};

    int ensure(long long n_pts, long long n_tris);
    // Rejects faces whose indices are outside [0, n) (other than removed faces
    // -1,-1,-1) and undo entries outside [0, undo_hi]; nothing else runs on bad input.
    int validate(const int *d_tris_aos3, int n, int m, const int *d_undo, int n_undo, int undo_hi, cudaStream_t s);
    int ensure_pairs(long long n);
    void release();

    // One round on opts/otris (already holding the input; init shuffle applied
    // by the caller).  d_undo_in: device list of n_undo_in entries.
    // keep_bvh: opts/otris are this context's own compact() output, so the
    // hierarchy carried over from the previous round may be reused.
    int round(int n, int m, float scale, float threshold, bool is_stuck, const int *d_undo_in, int n_undo_in,
              int *n_undo_out, cudaStream_t s, bool keep_bvh = false);

    // Batch mode: buffers for up to n_slots meshes (after ensure()).
    int ensure_batch(int n_slots);
    // One round over the packed meshes in opts/otris described by hslots[0..K)
    // (uploaded here).  Per-mesh undo-list lengths come back in nvu_out[K].
    int round_batch(int n, int m, int K, int *nvu_out, cudaStream_t s);
    // Compaction of a batch round; per-mesh next sizes and offsets in hscnt.
    int compact_batch(int n, int m, int K, cudaStream_t s);

    // Whole-mesh self-intersection of opts/otris: isect[f] = 1 for every face of
    // a pair the reference's selfx::self_intersect reports (all pairs, no cap).
    int self_intersect_all(int n, int m, cudaStream_t s);

    // compaction of the round's output into opts/otris for the next round;
    // returns new sizes through hcnt (after a sync).  The hierarchy's leaves
    // are renumbered to the compacted faces (removed faces become empty leaves).
    int compact(int n, int m, cudaStream_t s);
};

int stage2_shuffle_faces(int4 *tris, int m, cudaStream_t s);  // reference init permutation

// Hierarchy query of the faces flagged in `active` and the pair tests, on
// caller-provided buffers (cnt->n_pairs / pair_overflow must be zero).
cudaError_t query_and_test_pairs(const BvhNode *nodes, const int *vals, const int *scene, const float4 *pts,
                                 const int4 *tris, const uint8_t *active, int m, uint2 *pairs, long long cap_pairs,
                                 RoundCounters *cnt, uint8_t *isect, cudaStream_t s);

}  // namespace pamo
