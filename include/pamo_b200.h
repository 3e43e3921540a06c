/*
 * pamo_b200 -- C ABI of the B200 (sm_100a) PaMO mesh-optimization hot path.
 *
 * Conventions
 *   - Every entry point returns an int status (PAMO_OK on success) except
 *     pamo_simplify, whose signature mirrors the reference's void C ABI.
 *   - Pointers named d_* are device pointers on the context's device; h_* are
 *     host pointers.  Buffers are owned by the caller unless stated otherwise.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *     Calls return after the stream work they enqueue has completed unless
 *     stated otherwise.
 *   - A context holds the device state one simplification carries between
 *     rounds (the reference's CUSimp_Free object).  It is not thread safe: use
 *     one context per host thread.
 *   - Failures never fall back to another implementation: a missing device or
 *     a CUDA error is reported as PAMO_ERR_NO_DEVICE / PAMO_ERR_DEVICE.
 */
#ifndef PAMO_B200_H
#define PAMO_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define PAMO_OK 0
#define PAMO_ERR_INVALID_ARG 1
#define PAMO_ERR_OOM 2
#define PAMO_ERR_BUDGET_EXCEEDED 3
#define PAMO_ERR_DEVICE 4
#define PAMO_ERR_NO_DEVICE 5
#define PAMO_ERR_CAPACITY 6

typedef struct pamo_ctx pamo_ctx;

/* Library version (major*10000 + minor*100 + patch). */
int pamo_version(void);

/* Kernels this library has launched in this process, on every device and
   stream (a running total; take the difference around a region of interest).
   No counterpart in the reference. */
long long pamo_launch_count(void);

/* Human-readable name of a status code (static storage). */
const char *pamo_status_string(int status);

/* Creates a context bound to CUDA device `device`. */
int pamo_ctx_create(int device, pamo_ctx **out);

/* Releases the context and all device memory it owns. */
int pamo_ctx_destroy(pamo_ctx *ctx);

/*
 * One stage-2 collapse round.  Replaces CUDSP_Free.forward
 * (simp_cuda/src/pybind.cpp:52-103, which calls CUSimp_Free::forward,
 * simp_cuda/src/cusimp_free.cu:891-1048).
 *
 *   d_points [n_pts*3] f32, d_tris [n_tris*3] i32: the round's input mesh.
 *   d_verts_undo [n_verts_undo] i32: the undo list the previous round returned.
 *   scale, threshold, is_stuck, init: as in the reference (init applies the
 *     reference's round-0 face permutation).
 *   Outputs (caller-allocated): d_out_points [n_pts*3], d_out_tris [n_tris*3],
 *     d_out_occ [n_pts], d_out_map [n_pts]; *n_out_undo receives the length of
 *     the round's undo list, which pamo_free_copy_undo copies out.
 *
 * The adjacency order inside each vertex's face list is ascending face index
 * (the reference fills it in atomicAdd order), which makes every output
 * deterministic.
 */
int pamo_free_forward(pamo_ctx *ctx, const float *d_points, const int *d_tris, const int *d_verts_undo,
                      int n_verts_undo, int n_pts, int n_tris, float scale, float threshold, int is_stuck, int init,
                      void *stream, float *d_out_points, int *d_out_tris, int *d_out_occ, int *d_out_map,
                      int *n_out_undo);

/* Copies the first n entries of the last round's undo list to d_out. */
int pamo_free_copy_undo(pamo_ctx *ctx, int *d_out, int n, void *stream);

/*
 * The whole stage-2 loop of PaMO.run (simp_cuda/pamo/__init__.py:122-189,
 * stage 1 off): centring by the mean face centroid (numpy float32 order),
 * scale = max bbox extent, the init permutation, collapse rounds with the
 * reference's stuck / tolerance / target logic, and compaction between rounds,
 * all resident on the device.
 *   target_faces = max(int(ratio * n_tris), min_verts) as PaMO.run computes it.
 * On success *out_n_pts / *out_n_tris hold the result size and *out_rounds the
 * number of rounds; fetch the mesh with pamo_stage2_fetch.
 */
int pamo_stage2_run(pamo_ctx *ctx, const float *d_points, const int *d_tris, int n_pts, int n_tris,
                    long long target_faces, int tolerance, float threshold, int iters, void *stream, int *out_n_pts,
                    int *out_n_tris, int *out_rounds);

/*
 * Quality mode of the stage-2 rounds of this context (no reference
 * counterpart; off by default, which is the reference's algorithm bit for
 * bit).  On: each vertex's quadric is accumulated in FP64 from FP64 face
 * planes; an edge collapses to the minimiser of the summed quadric (the 3x3
 * system solved in FP64; the midpoint when it is close to singular or the
 * minimiser lies farther than the edge's length from the midpoint), whose FP64
 * quadric error is the cost's QEM term; the candidate pairs of the
 * self-intersection undo include faces sharing an edge, and every pair is
 * decided by the exact-predicate test of pamo_check_mesh (a degenerate face
 * counts as intersecting).  Affects pamo_stage2_run(_centred),
 * pamo_free_forward and pamo_simplify_ctx on this context.  The reference
 * keeps fp32 quadrics and the midpoint (simp_cuda/src/cusimp_free.cu:337-366,
 * 491) and an inexact pair test (simp_cuda/src/bvh/tri_tri_3d.cuh:131-276).
 */
int pamo_set_quality(pamo_ctx *ctx, int on);

/*
 * pamo_stage2_run on points that are already centred -- stage 1's output,
 * which the reference's PaMO.run passes to stage 2 without centring again
 * (simp_cuda/pamo/__init__.py:130-144) -- with h_offset3 (host float[3], the
 * input's tris_mean) added back by pamo_stage2_fetch.
 */
int pamo_stage2_run_centred(pamo_ctx *ctx, const float *d_points, const int *d_tris, int n_pts, int n_tris,
                            const float *h_offset3, long long target_faces, int tolerance, float threshold, int iters,
                            void *stream, int *out_n_pts, int *out_n_tris, int *out_rounds);

/*
 * Stage 1 of PaMO.run, remeshing (replaces PaMO.preprocess_mesh + remesh,
 * simp_cuda/pamo/__init__.py:60-120,130-142, which call torchcumesh2sdf and
 * pdmc): the triangles normalised into the unit cube as preprocess_mesh does,
 * a narrow-band signed distance field on a resolution^3 grid (band 3 /
 * resolution; sign by flood fill from the grid boundary; shifted by
 * -0.9 / resolution), dual marching cubes (one vertex per surface patch of a
 * cell), and each quad split into the triangle pair with the larger smallest
 * angle.  PaMO.run uses resolution 256, 128 when the target is at most 1000
 * faces, 64 at most 50.  The result is in the frame centred on the input's
 * tris_mean; *out_n_verts / *out_n_tris give its size and pamo_remesh_fetch
 * copies it.
 */
int pamo_remesh(pamo_ctx *ctx, const float *d_points, const int *d_tris, int n_pts, int n_tris, int resolution,
                void *stream, int *out_n_verts, int *out_n_tris);

/* Copies the last pamo_remesh result to device buffers (vertices [n,3] in the
   centred frame, faces [m,3]) and the input's tris_mean to h_offset3
   (optional, host float[3]). */
int pamo_remesh_fetch(pamo_ctx *ctx, float *d_out_verts, int *d_out_tris, float *h_offset3, void *stream);

/*
 * Copies the result of the last pamo_stage2_run: vertices with the centring
 * offset added back (float32, as PaMO.run's "verts + tris_mean"), and faces.
 * `to_host` != 0 means out_points/out_tris are host pointers.
 */
int pamo_stage2_fetch(pamo_ctx *ctx, float *out_points, int *out_tris, int to_host, void *stream);

/* Centring offset (tris_mean) of the last pamo_stage2_run, host float[3]. */
int pamo_stage2_offset(pamo_ctx *ctx, float *h_out3);

/*
 * The centring offset PaMO.run subtracts (simp_cuda/pamo/__init__.py:64, the
 * tris_mean of the input): each face's corner mean ((a + b) + c) / 3, then
 * numpy's float32 mean(axis=0) of those rows, whose adds run one after another
 * -- computed on the device, bit for bit.  d_points [n_pts,3] float32, d_tris
 * [n_tris,3] int32 (device); h_out3: host float[3].  Indices outside [0, n_pts)
 * return PAMO_ERR_INVALID_ARG.  Synchronises the stream.
 */
int pamo_tris_mean(const float *d_points, const int *d_tris, int n_pts, int n_tris, float *h_out3, void *stream);

/*
 * Per-round statistics of the last pamo_stage2_run / pamo_free_forward:
 * h_out[0..7] = {n_edges, n_collapsed, n_collapsed_with_coincident,
 *               n_undo_passes, n_undo_vertices, candidate_pairs_pass0,
 *               faces_in, faces_out}
 */
int pamo_stage2_last_round_stats(pamo_ctx *ctx, long long *h_out8);

/*
 * Whole-mesh self-intersection check with the reference's pair predicate
 * (replaces selfx::self_intersect, simp_cuda/src/bvh/self_intersect.cuh:151-392,
 * as a standalone check): d_out_flags[f] = 1 for every face of an intersecting
 * pair.  Unlike the reference the pair list has no capacity cap.  Faces
 * (-1,-1,-1) are ignored.  *out_n_pairs (optional) receives the number of
 * candidate pairs tested.
 */
int pamo_self_intersect(pamo_ctx *ctx, const float *d_points, const int *d_tris, int n_pts, int n_tris,
                        unsigned char *d_out_flags, long long *out_n_pairs, void *stream);

/*
 * Device timing of the stage-2 phases (no reference counterpart; diagnostics).
 * pamo_profile_enable(ctx, 1) resets and starts accumulating CUDA-event times
 * per phase; pamo_profile_read copies up to `cap` phase totals (ms) and call
 * counts and returns the number of phases.  Phase order: setup, lbvh build,
 * edge cost, collapse, cleanup, refit, query, pair tests, undo, compaction.
 */
int pamo_profile_enable(pamo_ctx *ctx, int enable);
int pamo_profile_read(pamo_ctx *ctx, double *h_ms, long long *h_calls, int cap);

/*
 * Faces entering each round of the last pamo_stage2_run (no reference
 * counterpart; PaMO.run prints nothing of the kind).  Writes up to `cap` entries
 * and returns the number of rounds (negative status on bad arguments).
 */
int pamo_stage2_round_sizes(pamo_ctx *ctx, int *h_out, int cap);

/*
 * Stage-3 safe projection settings; field for field the defaults of the
 * reference's Stage3Config (simp_cuda/safe_project/src/pamo_safe_project/
 * config.py:6-73) that the default energy set uses.  pamo_s3_default_config
 * fills them.
 */
typedef struct pamo_s3_config {
    int n_newton_iters;      /* 10 */
    int n_cg_iters;          /* 40 */
    int n_line_search_iters; /* 10 */
    int ccd_max_iters;       /* 100 */
    int spd_max_iters;       /* 3 */
    float d_hat;             /* 1e-3 */
    float coll_stiffness;    /* 1e2 */
    float contact_detection_radius; /* 1e-2 */
    float ee_classify_thres; /* 1e-3 */
    float ccd_slackness;     /* 0.7 */
    float ccd_thickness;     /* 1e-6 */
    float elas_young_modulus;  /* 1e-1 */
    float elas_poisson_ratio;  /* 0.0 */
    float hinge_stiffness;     /* 1e-2 */
    float mesh2gt_dist_stiffness; /* 1e3 */
    long long max_blocks;      /* 2^25: contact blocks before the radius is halved */
    /* 0.  1: the ground truth (pointers, sizes and contents) is the one of the
       context's previous call, so its device copy and hierarchy are kept
       (no reference counterpart: the reference registers it every time) */
    int reuse_gt;
} pamo_s3_config;

void pamo_s3_default_config(pamo_s3_config *cfg);

/*
 * Stage-3 safe projection of a simplified mesh towards its ground truth.
 * Replaces Stage3System.register_mesh + n_steps x Stage3System.step
 * (simp_cuda/safe_project/src/pamo_safe_project/system.py:167-272,411-470) as
 * pamo_safe_project.process calls them (processing.py:62-99), after the
 * caller's normalisation.  All arrays are device arrays in the normalised frame:
 *   d_gt_v [n_gt_v*3] f32, d_gt_f [n_gt_f*3] i32  ground truth
 *   d_v [n_v*3] f32, d_f [n_f*3] i32              mesh to project
 *   d_e [n_e*2] i32                               its unique edges
 *   d_h [n_h*4] i32                               its hinges (x0 | x1 x2 edge | x3)
 *   d_vor [n_v] f32                               Voronoi vertex areas
 * do_nothing != 0 skips the steps (the reference's small-angle guard).
 * The projected vertices are written to d_out_v [n_v*3].
 */
int pamo_safe_project(pamo_ctx *ctx, const float *d_gt_v, const int *d_gt_f, int n_gt_v, int n_gt_f,
                      const float *d_v, const int *d_f, int n_v, int n_f, const int *d_e, int n_e, const int *d_h,
                      int n_h, const float *d_vor, int n_steps, int do_nothing, const pamo_s3_config *cfg,
                      void *stream, float *d_out_v);

/* Mean (double, a fixed-order sum) and bounding-box extent of points [n,3] on
   the device: h_out6 = {mean x, y, z, extent x, y, z} (host memory).  Stage 3's
   normalisation takes these for the ground truth (processing.py:15-20). */
int pamo_point_stats(const float *d_pts, int n, double *h_out6, void *stream);

/* Stage-3 registration inputs on the device (system.py:217-225 computes them on
   the host with libigl): the mixed Voronoi area of each vertex of the mesh
   (double vertices [nv,3], faces [nf,3]; summed in double, stored as float32
   in d_out[nv]) and the mesh's smallest corner angle in degrees (host; NaN if a
   face is degenerate, 180 for no faces). */
int pamo_voronoi_areas(const double *d_v, const int *d_f, int nv, int nf, float *d_out, double *h_min_angle_deg,
                       void *stream);

/* The unique edges and the hinges of a closed 2-manifold triangle mesh, on the
   host (replaces the O(NT^2) face scan of hinge_preprocess_slow_kernel,
   energy_kernels/hinge_energy.py:21-57, and trimesh's edges_unique):
   h_edges [n_edges,2] (a < b, ascending by a * n_pts + b), h_hinges
   [n_edges,4] (x0, x1, x2, x3) in the same order, where x1 < x2 is the edge,
   x0 the third vertex of the face with directed edge x1 -> x2 and x3 that of
   the face with x2 -> x1.  Both output buffers hold 3 * n_tris / 2 rows.
   Returns PAMO_ERR_INVALID_ARG for an index outside [0, n_pts) and
   PAMO_ERR_CAPACITY when an edge is not shared by exactly two faces, once
   each way (the caller then uses a general method). */
int pamo_mesh_hinges(const int *h_tris, int n_tris, int n_pts, int *h_edges, int *h_hinges, int *out_n_edges);

/* pamo_mesh_hinges on device buffers: the same rows in the same order from the
   device faces d_tris [n_tris,3] into d_edges / d_hinges (3 * n_tris / 2 rows
   each), and the same status codes; waits for `stream`.  Stage 3 builds its
   edges and hinges with this when the stage-2 result is a closed 2-manifold. */
int pamo_mesh_hinges_device(const int *d_tris, int n_tris, int n_pts, int *d_edges, int *d_hinges, int *out_n_edges,
                            void *stream);

/* Whether two of the device points d_points [n_pts,3] coincide after rounding
   each coordinate to 8 decimals, numpy's round(x, 8) (*out_has_duplicates 1,
   else 0) -- the merge trimesh.Trimesh(process=True) applies to the stage-2
   result before stage 3 (simp_cuda/pamo/__init__.py:193-203) changes nothing
   when there are none.  Waits for `stream`. */
int pamo_merge_check_device(const float *d_points, int n_pts, int *out_has_duplicates, void *stream);

/* Wavefront OBJ text (host memory, `len` bytes) to vertices [n,3] and
   triangles [m,3] int, on the host, over `n_threads` threads (<= 0: all).
   Replaces trimesh.load(path, force='mesh', process=False) in the reference's
   example.py:24 (float64 vertices, into `verts_f64`) and the `.float()` /
   `.int()` of example.py:31-32 (into `verts`); either vertex buffer may be
   null.  `v` lines give the vertices (read as double; `verts` gets them
   rounded to float), `f` lines their first
   index of each corner (1-based; negative counts back from the vertices read
   so far), polygons split into fans (c0, c_k, c_k+1); other statements are
   skipped.  Always writes the counts to out_n_verts / out_n_tris; returns
   PAMO_ERR_CAPACITY (nothing written) when they exceed the capacities, so a
   first call with zero capacities sizes the buffers.  A malformed `v` or `f`
   line or an index outside the vertices returns PAMO_ERR_INVALID_ARG with the
   line's byte offset in *out_err_offset (if given). */
int pamo_obj_parse(const char *text, long long len, float *verts, double *verts_f64, long long cap_verts, int *tris,
                   long long cap_tris, int n_threads, long long *out_n_verts, long long *out_n_tris,
                   long long *out_err_offset);

/* Vertices and triangles to OBJ text (`v x y z` with the shortest decimal form
   that reads back as the same float, then `f a b c`, 1-based), as the
   reference's example.py:39-43 export does with trimesh.  Writes the length to
   *out_len; PAMO_ERR_CAPACITY (nothing written) when it exceeds `cap`;
   PAMO_ERR_INVALID_ARG for an index outside [0, n_verts). */
int pamo_obj_format(const float *verts, long long n_verts, const int *tris, long long n_tris, char *out,
                    long long cap, int n_threads, long long *out_len);

/* Stanford PLY (ASCII, binary little- or big-endian; host memory) to vertices
   and triangles, with the conventions of pamo_obj_parse: an element `vertex`
   with properties x, y, z (read as double; `verts` rounds them to float), the
   list property `vertex_indices` or `vertex_index` of an element `face` split
   into fans, every other element and property skipped.  A malformed header, a
   truncated body or an index outside the vertices returns
   PAMO_ERR_INVALID_ARG.  Replaces trimesh.load for .ply inputs. */
int pamo_ply_parse(const char *data, long long len, float *verts, double *verts_f64, long long cap_verts, int *tris,
                   long long cap_tris, long long *out_n_verts, long long *out_n_tris);

/* Vertices and triangles as binary little-endian PLY (float x, y, z; list
   uchar int vertex_indices).  Writes the length to *out_len;
   PAMO_ERR_CAPACITY (nothing written) when it exceeds `cap`. */
int pamo_ply_format(const float *verts, long long n_verts, const int *tris, long long n_tris, char *out, long long cap,
                    long long *out_len);

/* Stage-3 input normalisation on the device (processing.py:57-59 applies it
   to the ground truth on the host): out[i] = float((in[i] * scale + t) * post)
   per coordinate of n points [n,3], each step in double with one rounding, so
   the result equals the host float64 computation cast to float32. */
int pamo_affine_points(const float *d_in, int n, double scale, double tx, double ty, double tz, double post,
                       float *d_out, void *stream);

/*
 * Diagnostics of the last pamo_safe_project call (no reference counterpart):
 * h_out[0] total energy at the end, [1] contact blocks of the last detection,
 * [2] Newton iterations run.
 */
int pamo_safe_project_stats(pamo_ctx *ctx, double *h_out3);

/*
 * Per-Newton-iteration record of the last pamo_safe_project call (no
 * reference counterpart; the quantities are those of Stage3System.step,
 * system.py:354-470): six doubles per iteration = {energy at the iterate after
 * contact detection, energy after the line search, CCD step (accd_kernel,
 * ccd_kernels.py:8-110), index of the last line-search halving tried, contact
 * blocks, blocks closer than d_hat}.  Copies up to cap_rows rows to h_out and
 * writes the number of iterations recorded to *out_rows.
 */
int pamo_safe_project_trace(pamo_ctx *ctx, double *h_out, int cap_rows, int *out_rows);

/*
 * The stage-3 Jacobi-preconditioned CG (cg_solver.py:96-158, the solve each
 * Newton iteration runs) on a caller's symmetric matrix of 3x3 blocks over n
 * vertices in block-CSR form: d_row_ptr [n+1], d_col [n_blocks] (ascending per
 * row), d_blocks [n_blocks*9] row-major, preconditioner d_diag [n*3] (the
 * matrix's diagonal), right-hand side d_rhs [n*3]; `iters` CG iterations from
 * x = 0, solution in d_out [n*3].  For tests of the solver against known
 * answers (the reference's tests/test_dummy_energy.py).  Replaces the stage-3
 * state held by the context.
 */
/*
 * Test of the library's bounded device waits (no counterpart in the
 * reference).  which = 0: a prefix scan (the single-pass look-back of every
 * stage-2 round) in which one tile never publishes; which = 1: the persistent
 * CG solve of stage 3 in which one block never publishes its partial sums.
 * The waiting blocks give up after `spin_limit` polls (at most 2^24), record
 * the fault and return; the call then reports what a real run reports for
 * such a fault, PAMO_ERR_DEVICE, and the context stays usable.  Returns
 * PAMO_OK if nothing waited (PAMO_ERR_INVALID_ARG when the device cannot run
 * the persistent solve, so there is no wait to test).
 */
int pamo_debug_wait_timeout(pamo_ctx *ctx, int which, long long spin_limit, void *stream);

int pamo_bsr_pcg(pamo_ctx *ctx, int n, const int *d_row_ptr, const int *d_col, const float *d_blocks,
                 long long n_blocks, const float *d_diag, const float *d_rhs, int iters, float *d_out, void *stream);

/*
 * pamo_self_intersect without any allocation (no counterpart in the reference).
 * For callers that may not allocate device memory themselves or have the
 * library do it: a host application that owns all device memory through its own
 * pool, or a latency-critical loop where cudaMalloc/cudaFree would synchronise
 * the device and stall its other streams.  Same inputs and output as
 * pamo_self_intersect, with no context.  All scratch lives in one ~11 MB
 * file-scope device array that every GPU loading the library holds until the
 * process exits.  Limits: n_tris <= 32768, n_pts <= 65536 and at most 786,432
 * candidate pairs (box-overlapping face pairs) in total; larger inputs return
 * PAMO_ERR_CAPACITY.  An empty mesh (n_tris == 0) returns at once with
 * *out_n_pairs = 0.  Each call looks up the array's device address on the
 * current device, and waits for its stream twice (index validation, then the
 * counters are read back to the host), so no call can be captured into a CUDA
 * graph.  Every call shares the array: calls that overlap on the
 * GPU, on any stream or host thread, race and must be serialised by the
 * caller.
 */
int pamo_self_intersect_noalloc(const float *d_points, const int *d_tris, int n_pts, int n_tris,
                                unsigned char *d_out_flags, long long *out_n_pairs, void *stream);

/*
 * Acceptance checker of a triangle mesh, on the device.  It takes the role of
 * the reference's exact self-intersection script
 * (simp_cuda/safe_project/scripts/cgal_intersect/main.cpp:19-111,
 * CGAL PMP::self_intersections) as a library call.  Every pair of live faces
 * whose closed bounding boxes overlap is decided with exact-sign orientation
 * predicates (a double filter with an exact expansion fallback): faces with
 * no common vertex intersect when the closed triangles share any point, faces
 * sharing one vertex when they share another point, faces sharing an edge when
 * they are coplanar and fold onto each other, and a repeated face always.
 * Degenerate faces (a repeated index or collinear corners) are counted and
 * left out of the pair tests.  Faces (-1,-1,-1) are ignored.
 *   d_out_flags [n_tris] (optional): 1 for each face of an intersecting pair.
 *   h_out[11] (host) = {intersecting pairs, faces in them, degenerate faces,
 *     boundary half-edges (no reverse half-edge), non-manifold half-edges (an
 *     edge in more than two faces or twice in one direction), vertices whose
 *     faces do not form one closed fan, unreferenced vertices, candidate pairs
 *     (box overlaps), dead faces, traversal errors, out-of-range indices}.
 * The mesh is watertight and manifold when h_out[2..5] are all zero.
 * Returns PAMO_ERR_INVALID_ARG for an index outside [0, n_pts).
 */
int pamo_check_mesh(const float *d_points, const int *d_tris, int n_pts, int n_tris, unsigned char *d_out_flags,
                    long long *h_out, void *stream);

/*
 * One-sided surface distance from mesh A to mesh B (device arrays), by dense
 * sampling: every live face of A is sampled on the barycentric grid
 * (i/subdiv, j/subdiv), i + j <= subdiv, and each sample's distance to the
 * closest point of B is found through B's LBVH.  Replaces the Hausdorff and
 * Chamfer terms of the reference's metrics.py:31-51 (igl.hausdorff,
 * igl.point_mesh_squared_distance).
 *   h_out4 = {largest sample distance (a lower bound of the one-sided
 *     Hausdorff distance), an upper bound of it (plus each face's longest
 *     edge / subdiv / sqrt 3: every point of a face lies that close to a
 *     sample), mean squared sample distance, number of samples}.
 * The two-sided Hausdorff distance is the larger of the A->B and B->A values.
 */
int pamo_mesh_distance(const float *d_pa, const int *d_fa, int na, int nfa, const float *d_pb, const int *d_fb,
                       int nb, int nfb, int subdiv, double *h_out4, void *stream);

/*
 * Host-pointer simplifier.  Same signature and meaning as the reference's
 * Blender C ABI pamo_simplify (pamo_blender/cusimpinterface.cu:57): rounds until
 * four rounds without progress, output written to caller buffers sized like the
 * input, in_out_nv_ni = {n_verts, n_tris} in and out.  Uses an internal context
 * on device 0 (like the reference's static simplifier it is not re-entrant).
 */
void pamo_simplify(float *in_verts, int *in_tris, float *out_verts, int *out_tris, int *in_out_nv_ni,
                   float threshold);

/* pamo_simplify with an explicit context and a status code. */
int pamo_simplify_ctx(pamo_ctx *ctx, const float *h_in_verts, const int *h_in_tris, float *h_out_verts,
                      int *h_out_tris, int *in_out_nv_ni, float threshold);

/* ---------------------------------------------------------------------------
 * Batched simplification (no counterpart in the reference, which runs one mesh
 * per CUDSP_Free object).  Many meshes share every collapse round: they are
 * packed one after another into one set of round buffers, each keeps its own
 * parameters and the state the reference carries between rounds, and each ends
 * by PaMO.run's own rules (target, tolerance, iteration cap), so its result is
 * the one pamo_stage2_run gives for it on a fresh context.  Meshes submitted
 * while others run join at the next round, when the packed capacity
 * (max_verts / max_faces / max_meshes) and the device-memory budget allow.
 * One engine per host thread; all work goes to `stream`. */
typedef struct pamo_batch pamo_batch;

#define PAMO_JOB_PENDING 0 /* submitted, waiting for room */
#define PAMO_JOB_RUNNING 1
#define PAMO_JOB_DONE 2 /* result ready for pamo_batch_fetch; a failed job reports -status */

/* memory_budget: bytes of per-mesh device state (inputs waiting, per-mesh
   round state, results not yet released) the engine may hold; 0 = no limit. */
int pamo_batch_create(int device, long long max_verts, long long max_faces, int max_meshes,
                      long long memory_budget, void *stream, pamo_batch **out);
int pamo_batch_destroy(pamo_batch *b);

/* Queues one mesh (points [n,3] f32, faces [m,3] i32, host or device memory;
   host buffers may be reused on return).  target_faces / tolerance / threshold
   / iters mean what they mean for pamo_stage2_run. */
int pamo_batch_submit(pamo_batch *b, const float *points, const int *tris, int n_pts, int n_tris, int on_host,
                      long long target_faces, int tolerance, float threshold, int iters, long long *out_job);

/* Admits what fits, runs one collapse round over every running mesh and
   retires the meshes whose loop ended.  Returns the running / pending counts. */
int pamo_batch_step(pamo_batch *b, int *out_running, int *out_pending);

/* Jobs that finished (or failed) during the last pamo_batch_step: returns how
   many, and writes up to cap of their ids to h_out, so a server need not poll
   every job after every round. */
int pamo_batch_finished(pamo_batch *b, long long *h_out, int cap);

/* State (PAMO_JOB_*), current (or final) sizes and rounds run of a job. */
int pamo_batch_job(pamo_batch *b, long long job, int *state, int *n_pts, int *n_tris, int *rounds);

/* Copies a finished job's result (points [n,3] with the centring undone, faces
   [m,3]) to host (to_host=1) or device buffers of at least that size. */
int pamo_batch_fetch(pamo_batch *b, long long job, float *out_points, int *out_tris, int to_host);

/* Frees a finished or failed job's result. */
int pamo_batch_release(pamo_batch *b, long long job);

/* Per-phase device times (ms) and call counts accumulated since the timer was
   last switched (same phases as pamo_profile_read); then enable (1) or disable
   (0) the timer and reset it, or leave it as it is (-1).  Returns the number of
   phases. */
int pamo_batch_profile(pamo_batch *b, int enable, double *h_ms, long long *h_calls, int cap);

/* {running, pending, packed vertices, packed faces, bytes held, rounds run,
    max_faces, memory budget} */
int pamo_batch_stats(pamo_batch *b, long long *h_out8);

#ifdef __cplusplus
}
#endif

#endif /* PAMO_B200_H */
