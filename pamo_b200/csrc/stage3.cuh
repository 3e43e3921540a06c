// Stage-3 safe projection on the device (sm_100a): barrier-energy Newton
// iterations with a Jacobi-PCG on the assembled block-sparse Hessian (contact
// terms matrix-free), contact detection on LBVHs, additive CCD and a halving
// line search (simp_cuda/safe_project/src/pamo_safe_project:
// system.py:411-470, cg_solver.py:46-158, energy.py, kernels/*).
//
// Precision: positions, distances, gradients and the CG vectors are FP32; the
// barrier value and its derivatives for d < d_hat, the CCD step search, the
// energy sums and the CG dot products are FP64.
#pragma once

#include "../../include/pamo_b200.h"
#include "common.cuh"
#include "lbvh.cuh"
#include "stage2.cuh"

namespace pamo {
namespace s3 {

struct Stage3 {
    int device = 0;
    pamo_s3_config cfg{};
    long long cap_p = 0, cap_t = 0, cap_e = 0, cap_h = 0, cap_b = 0, cap_gp = 0, cap_gt = 0;
    int np = 0, nt = 0, ne = 0, nh = 0, ngp = 0, ngt = 0;
    float radius = 0.f;
    bool do_nothing = false;

    // per vertex (xyz in float4, w unused)
    float4 *q = nullptr, *q_prev = nullptr, *q_det = nullptr, *p = nullptr, *grad = nullptr, *diag = nullptr;
    float4 *target = nullptr, *r = nullptr, *z = nullptr, *v = nullptr, *v2 = nullptr, *Av = nullptr;
    float *wk = nullptr;  // Voronoi area x GT-distance stiffness
    // per triangle / edge / hinge
    int4 *tris = nullptr;
    float *area = nullptr;
    float4 *inv_dm = nullptr;  // 2x2 row-major
    int4 *edges4 = nullptr;    // (a, b, b, 0): a segment as a degenerate triangle for the LBVH
    int4 *hinges = nullptr;
    float *rest_angle = nullptr, *rest_elen = nullptr;
    // The Hessian as 3x3 blocks in rows of vertices (BSR).  The pattern -- the
    // diagonal, the mesh edges and the hinges' four-vertex couplings -- is fixed
    // for a registered mesh; the values are assembled once per Newton iteration
    // (vertex term, membrane, SPD-projected hinges).  The contact terms stay
    // matrix-free (rank one per active block).
    int *row_ptr = nullptr;     // [np + 1]
    int *col = nullptr;         // [nnz], ascending in each row
    float4 *kval = nullptr;     // [3 nnz]: the rows of each block (w unused)
    int *tri_slot = nullptr;    // [9 nt]: block (a, b) of triangle t at 9 t + 3 a + b
    int *hinge_slot = nullptr;  // [16 nh]: block (a, b) of hinge h at 16 h + 4 a + b
    int *diag_slot = nullptr;   // [np]
    float *hblk = nullptr;      // [81 nh]: the unprojected hinge blocks of vertices 0-2 (current Newton iteration)
    int *pat_cnt = nullptr, *pat_cur = nullptr, *pat_off = nullptr, *pat_cand = nullptr, *pat_scan = nullptr;
    long long nnz = 0, cap_nnz = 0, cap_cand = 0;
    float4 *Avc = nullptr;      // contact terms of A v (the four-launch solve) / A z (the persistent solve)
    float4 *cg_rec = nullptr;   // the persistent solve's vertex records: 2 x 3 float4 per vertex
    // contact blocks
    int4 *bidx = nullptr;
    int *bkind = nullptr, *bsub = nullptr;
    float *bd = nullptr, *bb2 = nullptr;
    float4 *bg = nullptr;  // 4 gradient vectors per block
    int *bact = nullptr;   // blocks with d < d_hat (the CG operator's contact terms)
    int2 *cand_pt = nullptr, *cand_ee = nullptr;  // detection: pairs whose boxes overlap
    long long cap_c = 0;
    float4 *q_gather = nullptr;  // positions when the candidates were gathered
    bool gathered = false;
    float gather_thr = 0.f, extra_at_gather = 0.f;
    // hierarchies
    Lbvh tri_bvh, edge_bvh, gt_bvh;
    float4 *gt_pts = nullptr;
    int4 *gt_tris = nullptr;
    // the ground truth of the last registration (kept when cfg.reuse_gt says so)
    const float *gt_src_v = nullptr;
    const int *gt_src_f = nullptr;
    bool gt_ready = false;
    // scalars and reduction partials
    double *dscal = nullptr;  // [0] energy [1] energy_prev [2] zr [3] zr_last [4] vAv
    float *fscal = nullptr;   // [0] ccd step
    int *iscal = nullptr;     // [0] block count [1] overflow [2] stack overflow
    double *partials = nullptr;
    int *h_iscal = nullptr;   // pinned
    double *h_dscal = nullptr;
    double *trace = nullptr;  // [cap_trace][6] per Newton iteration (k_trace); null: not recorded
    long long cap_trace = 0;
    Profiler *prof = nullptr;  // the context's phase timer (optional)
    cudaGraphExec_t graph = nullptr;  // one Newton iteration after detection
    long long graph_cap_b = -1, graph_kernels = 0;
    // a new registration changed the iteration's sizes and pointers: the next
    // iteration is captured again and the executable graph updated in place
    bool graph_stale = false;
    bool use_graph = true;
    int cg_blocks = 0;   // grid of the persistent solve
    int cg_persistent = -1;  // 1: one cooperative launch per solve; 0: one launch per phase; -1: not decided
    int ls_persistent = -1;  // 1: the line search as one cooperative launch (decided with cg_persistent)
    long long cg_spin_limit = 1LL << 24;  // polls per grid-sum wait (~ seconds) before the solve gives up
    int cg_absent_block = -1;  // the wait-timeout test only: a block that never publishes
    cudaStream_t work = nullptr;  // the solve's own stream (graphs cannot be captured on the legacy stream)
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    // the differentials' two side branches (created with the solve's stream)
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};

    int ensure(long long np_, long long nt_, long long ne_, long long nh_, long long ngp_, long long ngt_);
    int ensure_blocks(long long nb);
    int ensure_cands(long long n);
    int build_pattern(cudaStream_t s);
    void release();

    // Inputs are device arrays in the normalised frame.
    int register_mesh(const float *d_gt_v, const int *d_gt_f, int n_gt_v, int n_gt_f, const float *d_v,
                      const int *d_f, int n_v, int n_f, const int *d_e, int n_e, const int *d_h, int n_h,
                      const float *d_vor, cudaStream_t s);
    int step(cudaStream_t s);
    int newton(cudaStream_t s);
    int newton_elements(cudaStream_t s);
    int newton_contacts(cudaStream_t s);
    int newton_body(cudaStream_t s);
    int detect(cudaStream_t s);
    int cg_solve(cudaStream_t s);
    int ensure_trace(long long rows);
    // K x = rhs by cg_solve for a caller's matrix of 3x3 blocks (BSR over n
    // vertices); replaces the context's stage-3 state
    int solve_bsr(int n, const int *d_row_ptr, const int *d_col, const float *d_blocks, long long n_blocks,
                  const float *d_diag, const float *d_rhs, int iters, float *d_out, cudaStream_t s);
    void drop_graph();
    // diagnostics
    int energy_now(double *out, cudaStream_t s);
};

}  // namespace s3
}  // namespace pamo
