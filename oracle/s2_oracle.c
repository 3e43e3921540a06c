/*
 * CPU oracle for the PaMO stage-2 simplification round -- TEST INFRASTRUCTURE.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load
 * this library, and only as the checker / CPU baseline; the product path
 * (pamo_b200/) never calls it.
 *
 * It restates, in plain C, the per-round algorithm of the reference's
 * CUSimp_Free::forward (simp_cuda/src/cusimp_free.cu:891-1048) together with the
 * self-intersection check it calls (simp_cuda/src/bvh/self_intersect.cuh:151-392,
 * bvh/tri_tri_3d.cuh:100-297).  Every floating-point expression keeps the
 * reference's operation order and precision (fp32 with no contraction, fp64
 * where the reference uses double), so that a build with -ffp-contract=off
 * reproduces the device results bit for bit.
 *
 * Determinism.  The reference fills the vertex->face adjacency with atomicAdd
 * slots (cusimp_free.cu:291-304), so its fp32 sums depend on scheduling.  This
 * oracle (and the CUDA product) define the adjacency order canonically: the faces
 * of each vertex in ascending face index.  List outputs that the reference fills
 * with atomicAdd (collapsed edges, undo edges, intersecting pairs) are produced
 * in ascending edge/face order.  The racy coincident-edge pass
 * (remove_line_edge_collapse, cusimp_free.cu:234-274) is given the semantics
 * "all threads read positions before any writes, writes applied in edge order",
 * one legal interleaving of the reference kernel.
 *
 * Persistent state that the reference reads stale across rounds (edge_cost for
 * edges whose cost is not rewritten, cusimp_free.cu:402-403,440-442; pts_map of
 * the previous round, :869-878; the invalid-vertex table, :899-916; the undo
 * list tail, :1036-1040) lives in the context, zero-initialised at allocation.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define COST_RANGE 10.0f
#define S2O_OK 0
#define S2O_ERR_ARG 1
#define S2O_ERR_OOM 3

typedef struct { float x, y, z; } v3;
typedef struct { int i, j, k; } t3;

/* ---------------------------------------------------------------- helpers */
static inline float fmin_t(float a, float b) { return a < b ? a : b; }  /* cusimp_free.cu:29-34 */
static inline float fmax_t(float a, float b) { return a > b ? a : b; }
static inline float fclamp_t(float x, float a, float b) { return fmin_t(fmax_t(a, x), b); }

/* device float->u32 conversion (cvt.rzi.u32.f32): NaN->0, saturating */
static inline uint32_t f2u_sat(float x)
{
    if (!(x == x)) return 0u;
    if (x <= 0.0f) return 0u;
    if (x >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)x;
}

static inline v3 vsub(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline v3 vcross(v3 a, v3 b)
{
    v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static inline float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float vnorm(v3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline v3 vdivs(v3 a, float s) { v3 r = {a.x / s, a.y / s, a.z / s}; return r; }
static inline int tri_dead(t3 t) { return t.i == -1 && t.j == -1 && t.k == -1; }
static inline int tri_has(t3 t, int v) { return t.i == v || t.j == v || t.k == v; }

/* Heron area, cusimp_free.cu:368-375 */
static inline float tri_area(v3 p0, v3 p1, v3 p2)
{
    float a = vnorm(vsub(p0, p1));
    float b = vnorm(vsub(p1, p2));
    float c = vnorm(vsub(p2, p0));
    float s = (a + b + c) / 2;
    return sqrtf(s * (s - a) * (s - b) * (s - c));
}

/* The skinny penalty term of compute_edge_cost_kernel (cusimp_free.cu:533,573),
 * with the reference's operator precedence: only the first square divides.
 * Built with nvcc and libstdc++, pow(float, 2) there is std::pow's promoting
 * overload, so the squares are doubles and everything after the fp32 numerator
 * 4*sqrt(3)*area is evaluated in double, then rounded once by float(...).  The
 * square of a float is exact in double. */
static inline float skinny_term(v3 n0, v3 n1, v3 n2)
{
    float l01 = vnorm(vsub(n0, n1));
    float l12 = vnorm(vsub(n1, n2));
    float l20 = vnorm(vsub(n2, n0));
    const float c4s3 = 4.0f * sqrtf(3.0f);
    float num = c4s3 * tri_area(n0, n1, n2);
    double e = (double)num / ((double)l01 * (double)l01) + (double)l12 * (double)l12 + (double)l20 * (double)l20 +
               (double)0.0000001f;
    return 1.0f - fclamp_t((float)e, 0.0f, 1.0f);
}

/* is_skinny_triangle, cusimp_free.cu:617-637 */
static inline int is_skinny(v3 p, v3 q, v3 r)
{
    v3 pq = vsub(q, p), pr = vsub(r, p), qr = vsub(r, q);
    float lpq = sqrtf(vdot(pq, pq)), lpr = sqrtf(vdot(pr, pr)), lqr = sqrtf(vdot(qr, qr));
    float ml = fmaxf(lpq, fmaxf(lpr, lqr));
    v3 c = vcross(pq, pr);
    float thr = (float)(1e-6 * (double)ml * (double)ml);
    float area = 0.5f * sqrtf(c.x * c.x + c.y * c.y + c.z * c.z);
    return area < thr;
}

/* ------------------------------------------------ tri-tri (parity arithmetic) */
/* translate_coordinates / floor_mean, self_intersect.cuh:124-149 */
static inline int floor_mean6(float a, float b, float c, float d, float e, float f)
{
    float m = (a + b + c + d + e + f) / 6.0f;
    return (int)floorf(m);
}

static inline int near_same(v3 a, v3 b) /* are_vertices_same(eps=1e-6f), self_intersect.cuh:26-31 */
{
    const float eps = 1e-6f;
    return fabsf(a.x - b.x) < eps && fabsf(a.y - b.y) < eps && fabsf(a.z - b.z) < eps;
}

static inline int shared_edge_coord(const v3 *A, const v3 *B) /* self_intersect.cuh:39-48 */
{
    int n = 0;
    for (int a = 0; a < 3; ++a)
        n += near_same(A[a], B[0]) || near_same(A[a], B[1]) || near_same(A[a], B[2]);
    return n >= 2;
}

static inline double ddot3(const double *a, const float *b)
{
    return a[0] * (double)b[0] + a[1] * (double)b[1] + a[2] * (double)b[2];
}
static inline void dplane(const float t[3][3], double pl[4])
{
    double ba[3], bc[3];
    for (int c = 0; c < 3; ++c) {
        ba[c] = (double)t[0][c] - (double)t[1][c];
        bc[c] = (double)t[2][c] - (double)t[1][c];
    }
    pl[0] = ba[1] * bc[2] - ba[2] * bc[1];
    pl[1] = ba[2] * bc[0] - ba[0] * bc[2];
    pl[2] = ba[0] * bc[1] - ba[1] * bc[0];
    pl[3] = -ddot3(pl, t[1]);
}

/* is_coplanar, tri_tri_3d.cuh:100-129 */
static int coplanar(const float a[3][3], const float b[3][3])
{
    float sc = 0.0f;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) sc = fmaxf(sc, fabsf(a[i][j]));
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) sc = fmaxf(sc, fabsf(b[i][j]));
    double pl[4];
    dplane(a, pl);
    double eps = (double)sc * 1e-6;
    for (int j = 0; j < 3; ++j)
        if (!(fabs(ddot3(pl, b[j]) + pl[3]) <= eps)) return 0;
    return 1;
}

static inline int same_sign3(const float s[3])
{
    return (s[0] != 0.0f && s[1] != 0.0f && s[2] != 0.0f) && ((s[0] < 0.0f) == (s[1] < 0.0f)) &&
           ((s[0] < 0.0f) == (s[2] < 0.0f));
}

/* isect_tri_tri_v3_ex, tri_tri_3d.cuh:131-276: plane of each triangle in fp64,
 * signed distances rounded to fp32, interval overlap along the plane-plane line. */
static int tri_tri(const float ta[3][3], const float tb[3][3], float r1[3], float r2[3])
{
    float side[2][3];
    double pa[4], pb[4];
    dplane(ta, pa);
    for (int j = 0; j < 3; ++j) side[1][j] = (float)(ddot3(pa, tb[j]) + pa[3]);
    if (side[1][0] == 0.0f && side[1][1] == 0.0f && side[1][2] == 0.0f) return 0;
    if (same_sign3(side[1])) return 0;
    dplane(tb, pb);
    for (int j = 0; j < 3; ++j) side[0][j] = (float)(ddot3(pb, ta[j]) + pb[3]);
    if (same_sign3(side[0])) return 0;

    double dir[3];
    dir[0] = pa[1] * pb[2] - pa[2] * pb[1];
    dir[1] = pa[2] * pb[0] - pa[0] * pb[2];
    dir[2] = pa[0] * pb[1] - pa[1] * pb[0];

    float rmin[2], rmax[2], loc[2][2][3];
    for (int i = 0; i < 2; ++i) {
        const float(*t)[3] = i == 0 ? ta : tb;
        const float *s = side[i];
        int o[3];
        if ((s[0] != 0.0f && s[1] != 0.0f) && ((s[0] < 0.0f) == (s[1] < 0.0f))) {
            o[0] = 1; o[1] = 2; o[2] = 0;
        } else if ((s[1] != 0.0f && s[2] != 0.0f) && ((s[1] < 0.0f) == (s[2] < 0.0f))) {
            o[0] = 2; o[1] = 0; o[2] = 1;
        } else if (s[1] == 0.0f && ((s[2] < 0.0f) != (s[0] < 0.0f))) {
            o[0] = 1; o[1] = 2; o[2] = 0;
        } else {
            o[0] = 0; o[1] = 1; o[2] = 2;
        }
        double db = ddot3(dir, t[o[1]]);
        float sc = s[o[1]];
        if (sc != 0.0f) {
            double da = ddot3(dir, t[o[0]]);
            double dc = ddot3(dir, t[o[2]]);
            float f0 = sc / (sc - s[o[0]]);
            float f1 = sc / (sc - s[o[2]]);
            double off0 = f0 * (da - db);
            double off1 = f1 * (dc - db);
            if (off0 > off1) {
                double td = off0; off0 = off1; off1 = td;
                float tf = f0; f0 = f1; f1 = tf;
                int ti = o[0]; o[0] = o[2]; o[2] = ti;
            }
            rmin[i] = (float)(db + off0);
            rmax[i] = (float)(db + off1);
            float s0 = 1.0f - f0, s1 = 1.0f - f1;
            for (int c = 0; c < 3; ++c) {
                loc[i][0][c] = s0 * t[o[1]][c] + f0 * t[o[0]][c];
                loc[i][1][c] = s1 * t[o[1]][c] + f1 * t[o[2]][c];
            }
        } else {
            rmin[i] = rmax[i] = (float)db;
            for (int c = 0; c < 3; ++c) loc[i][0][c] = loc[i][1][c] = t[o[1]][c];
        }
    }
    if ((rmax[0] > rmin[1]) && (rmin[0] < rmax[1])) {
        const float *a, *b;
        if (rmin[0] >= rmin[1]) {
            a = loc[0][0];
            b = (rmax[0] <= rmax[1]) ? loc[0][1] : loc[1][1];
        } else {
            if (rmax[0] <= rmax[1]) { a = loc[0][1]; b = loc[1][0]; }
            else { a = loc[1][0]; b = loc[1][1]; }
        }
        for (int c = 0; c < 3; ++c) { r1[c] = a[c]; r2[c] = b[c]; }
        return 1;
    }
    return 0;
}

/* One directed candidate of the reference's pair lambda (self_intersect.cuh:229-378):
 * "cur" is the BVH object, "qry" the querying face.  Returns 1 if the pair is
 * reported as intersecting. */
int s2o_pair_flag(const float *cur9, const int *cur_idx, const float *qry9, const int *qry_idx, float eps)
{
    v3 P[6];
    for (int a = 0; a < 3; ++a) {
        P[a].x = cur9[3 * a]; P[a].y = cur9[3 * a + 1]; P[a].z = cur9[3 * a + 2];
        P[3 + a].x = qry9[3 * a]; P[3 + a].y = qry9[3 * a + 1]; P[3 + a].z = qry9[3 * a + 2];
    }
    int mx = floor_mean6(P[0].x, P[1].x, P[2].x, P[3].x, P[4].x, P[5].x);
    int my = floor_mean6(P[0].y, P[1].y, P[2].y, P[3].y, P[4].y, P[5].y);
    int mz = floor_mean6(P[0].z, P[1].z, P[2].z, P[3].z, P[4].z, P[5].z);
    for (int a = 0; a < 6; ++a) {
        P[a].x -= (float)mx; P[a].y -= (float)my; P[a].z -= (float)mz;
    }
    int shared = 0;
    for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k) shared += cur_idx[j] == qry_idx[k];
    float ta[3][3], tb[3][3];
    for (int a = 0; a < 3; ++a) {
        ta[a][0] = P[a].x; ta[a][1] = P[a].y; ta[a][2] = P[a].z;
        tb[a][0] = P[3 + a].x; tb[a][1] = P[3 + a].y; tb[a][2] = P[3 + a].z;
    }
    if (coplanar(ta, tb)) return 0;
    if (shared == 2) return 0;
    if (shared_edge_coord(P, P + 3)) return 0;
    float r1[3], r2[3];
    if (!tri_tri(ta, tb, r1, r2)) return 0;
    float dx = fabsf(r2[0] - r1[0]), dy = fabsf(r2[1] - r1[1]), dz = fabsf(r2[2] - r1[2]);
    float d = -INFINITY;
    if (dx > d) d = dx;
    if (dy > d) d = dy;
    if (dz > d) d = dz;
    if (d < eps && shared == 1) return 0;
    return 1;
}

/* ------------------------------------------------------------ context */
typedef struct {
    int cap_pts, cap_tris, cap_edges, cap_undo;
    /* persistent across rounds */
    uint32_t *edge_cost;
    int *pts_map;
    int *undo_list;
    int *tmp_undo;
    unsigned char *invalid_table;
    /* per round (sized by capacity) */
    v3 *pts, *opts;
    t3 *tris, *otris;
    int *occ;
    int *first_near, *near;
    int *first_edge;
    int *edges; /* 2 per edge */
    float *Q;   /* 10 per vertex: 00 01 02 03 11 12 13 22 23 33 */
    uint64_t *tri_min;
    int *collapsed;
    unsigned char *isect;
    unsigned char *isect0; /* flags of the round's first intersection pass */
    int *undo_edges;
    unsigned char *line_flag;
    /* round stats */
    int n_pts, n_tris, n_edges, n_main, n_total, n_considered, n_undo_passes;
    int undo_counts[8];
    int n_vertices_undo;
    long long n_cand_pairs[8];
} s2o_ctx;

static void *zalloc(size_t n) { return calloc(n ? n : 1, 1); }

static int ctx_alloc(s2o_ctx *c, int cap_pts, int cap_tris)
{
    c->cap_pts = cap_pts;
    c->cap_tris = cap_tris;
    c->cap_edges = 3 * cap_tris;
    c->cap_undo = 16 * (cap_pts + 1);
    size_t P = (size_t)cap_pts + 1, T = (size_t)cap_tris + 1, E = (size_t)c->cap_edges + 1;
    c->edge_cost = zalloc(E * 4);
    c->pts_map = zalloc(P * 4);
    c->undo_list = zalloc((size_t)c->cap_undo * 4);
    c->tmp_undo = zalloc((size_t)c->cap_undo * 4);
    c->invalid_table = zalloc(P);
    c->pts = zalloc(P * sizeof(v3));
    c->opts = zalloc(P * sizeof(v3));
    c->tris = zalloc(T * sizeof(t3));
    c->otris = zalloc(T * sizeof(t3));
    c->occ = zalloc(P * 4);
    c->first_near = zalloc(P * 4);
    c->near = zalloc(3 * T * 4);
    c->first_edge = zalloc(T * 4);
    c->edges = zalloc(2 * E * 4);
    c->Q = zalloc(10 * P * 4);
    c->tri_min = zalloc(T * 8);
    c->collapsed = zalloc(E * 4);
    c->isect = zalloc(T);
    c->isect0 = zalloc(T);
    c->undo_edges = zalloc(E * 4);
    c->line_flag = zalloc(E);
    return c->edge_cost && c->pts_map && c->undo_list && c->tmp_undo && c->invalid_table && c->pts &&
                   c->opts && c->tris && c->otris && c->occ && c->first_near && c->near && c->first_edge &&
                   c->edges && c->Q && c->tri_min && c->collapsed && c->isect && c->isect0 && c->undo_edges && c->line_flag
               ? S2O_OK
               : S2O_ERR_OOM;
}

static void ctx_free_bufs(s2o_ctx *c)
{
    void *p[] = {c->edge_cost, c->pts_map, c->undo_list, c->tmp_undo, c->invalid_table, c->pts, c->opts,
                 c->tris, c->otris, c->occ, c->first_near, c->near, c->first_edge, c->edges, c->Q,
                 c->tri_min, c->collapsed, c->isect, c->undo_edges, c->line_flag};
    for (size_t i = 0; i < sizeof(p) / sizeof(p[0]); ++i) free(p[i]);
}

s2o_ctx *s2o_create(void) { return (s2o_ctx *)zalloc(sizeof(s2o_ctx)); }
void s2o_destroy(s2o_ctx *c)
{
    if (!c) return;
    ctx_free_bufs(c);
    free(c);
}

static int ensure(s2o_ctx *c, int n_pts, int n_tris)
{
    if (c->cap_pts >= n_pts && c->cap_tris >= n_tris && c->edge_cost) return S2O_OK;
    int cp = n_pts > c->cap_pts ? n_pts : c->cap_pts;
    int ct = n_tris > c->cap_tris ? n_tris : c->cap_tris;
    ctx_free_bufs(c);
    return ctx_alloc(c, cp, ct);
}

/* -------------------------------------------------------- round pieces */
static void build_csr(s2o_ctx *c)
{
    int n = c->n_pts, m = c->n_tris;
    int *fn = c->first_near;
    memset(fn, 0, (size_t)(n + 1) * 4);
    for (int f = 0; f < m; ++f) {
        t3 t = c->tris[f];
        if (tri_dead(t)) continue;
        fn[t.i]++; fn[t.j]++; fn[t.k]++;
    }
    int s = 0;
    for (int v = 0; v <= n; ++v) { int d = fn[v]; fn[v] = s; s += d; }
    int *cur = (int *)malloc((size_t)(n + 1) * 4);
    memcpy(cur, fn, (size_t)(n + 1) * 4);
    for (int f = 0; f < m; ++f) { /* ascending face index within each vertex segment */
        t3 t = c->tris[f];
        if (tri_dead(t)) continue;
        c->near[cur[t.i]++] = f;
        c->near[cur[t.j]++] = f;
        c->near[cur[t.k]++] = f;
    }
    free(cur);
}

static void build_edges(s2o_ctx *c) /* count_edge_kernel / create_edge_kernel, :306-335 */
{
    int m = c->n_tris, e = 0;
    for (int f = 0; f < m; ++f) {
        t3 t = c->tris[f];
        c->first_edge[f] = e;
        if (tri_dead(t)) continue;
        if (t.i > t.j) { c->edges[2 * e] = t.j; c->edges[2 * e + 1] = t.i; e++; }
        if (t.j > t.k) { c->edges[2 * e] = t.k; c->edges[2 * e + 1] = t.j; e++; }
        if (t.k > t.i) { c->edges[2 * e] = t.i; c->edges[2 * e + 1] = t.k; e++; }
    }
    c->first_edge[m] = e;
    c->n_edges = e;
}

/* tri2plane + compute_vert_Q_kernel, :337-366 (10 unique entries of p p^T) */
static void compute_Q(s2o_ctx *c)
{
    int n = c->n_pts;
#pragma omp parallel for schedule(static)
    for (int v = 0; v < n; ++v) {
        float q[10] = {0};
        for (int s = c->first_near[v]; s < c->first_near[v + 1]; ++s) {
            t3 t = c->tris[c->near[s]];
            v3 v0 = c->pts[t.i], v1 = c->pts[t.j], v2 = c->pts[t.k];
            v3 nrm = vcross(vsub(v1, v0), vsub(v2, v0));
            nrm = vdivs(nrm, vnorm(nrm));
            float d = -vdot(nrm, v0);
            float p[4] = {nrm.x, nrm.y, nrm.z, d};
            q[0] += p[0] * p[0]; q[1] += p[0] * p[1]; q[2] += p[0] * p[2]; q[3] += p[0] * p[3];
            q[4] += p[1] * p[1]; q[5] += p[1] * p[2]; q[6] += p[1] * p[3];
            q[7] += p[2] * p[2]; q[8] += p[2] * p[3]; q[9] += p[3] * p[3];
        }
        memcpy(c->Q + 10 * (size_t)v, q, sizeof(q));
    }
}

static inline int next_after(t3 t, int v)
{
    if (t.i == v) return t.j;
    if (t.j == v) return t.k;
    if (t.k == v) return t.i;
    return -2; /* the reference prints "error" and reads an uninitialised value */
}

/* compute_edge_cost_kernel, :382-585.  Returns 1 and sets *out when the reference
 * writes the cost, 0 when it leaves the stale value in place. */
static int edge_cost_one(const s2o_ctx *c, int e, int is_stuck, float tres, float edge_s, uint32_t *out)
{
    int u = c->edges[2 * e], v = c->edges[2 * e + 1];
    const v3 *P = c->pts;
    const t3 *T = c->tris;
    const int *fn = c->first_near, *nr = c->near;
    if (c->invalid_table[u] && c->invalid_table[v]) { *out = 0xFFFFFFFFu; return 1; }
    if (is_stuck) return 0;
    int dup = 0;
    for (int a = fn[u]; a < fn[u + 1]; ++a) {
        int iu = next_after(T[nr[a]], u);
        for (int b = fn[v]; b < fn[v + 1]; ++b) {
            int iv = next_after(T[nr[b]], v);
            if (iu == iv) dup++;
            if (dup > 2) { *out = 0xFFFFFFFFu; return 1; }
        }
    }
    if (dup != 2) return 0;

    float elen = 0.0f;
    int nedge = 0;
    for (int pass = 0; pass < 2; ++pass) {
        int w = pass ? v : u;
        for (int a = fn[w]; a < fn[w + 1]; ++a) {
            t3 t = T[nr[a]];
            if (t.i > t.j) { elen += vnorm(vsub(P[t.i], P[t.j])); nedge++; }
            if (t.j > t.k) { elen += vnorm(vsub(P[t.j], P[t.k])); nedge++; }
            if (t.k > t.i) { elen += vnorm(vsub(P[t.k], P[t.i])); nedge++; }
        }
    }
    v3 v0 = P[u], v1 = P[v];
    elen = elen / (float)nedge / edge_s * tres;
    elen = elen + vnorm(vsub(v0, v1)) / edge_s * tres;
    v3 mid = {(v0.x + v1.x) / 2.0f, (v0.y + v1.y) / 2.0f, (v0.z + v1.z) / 2.0f};

    float Qa = 0.0f;
    int ntri = 0;
    for (int pass = 0; pass < 2; ++pass) {
        int w = pass ? v : u, other = pass ? u : v;
        for (int a = fn[w]; a < fn[w + 1]; ++a) {
            t3 t = T[nr[a]];
            if (tri_has(t, other)) continue;
            v3 o0 = P[t.i], o1 = P[t.j], o2 = P[t.k];
            v3 n0 = o0, n1 = o1, n2 = o2;
            if (t.i == w) n0 = mid;
            if (t.j == w) n1 = mid;
            if (t.k == w) n2 = mid;
            v3 on = vcross(vsub(o1, o0), vsub(o2, o0));
            on = vdivs(on, vnorm(on));
            v3 nn = vcross(vsub(n1, n0), vsub(n2, n0));
            nn = vdivs(nn, vnorm(nn));
            if (vdot(on, nn) < 0) { *out = 0xFFFFFFFFu; return 1; }
            Qa += skinny_term(n0, n1, n2);
            ntri++;
        }
    }
    Qa = 5.0f * Qa;
    const float *qu = c->Q + 10 * (size_t)u, *qv = c->Q + 10 * (size_t)v;
    float q[10];
    for (int k = 0; k < 10; ++k) q[k] = qu[k] + qv[k];
    /* Mat4x4::vTMv with w = 1 (column-major product then dot) */
    float x = mid.x, y = mid.y, z = mid.z, w = 1.0f;
    float m00 = q[0], m01 = q[1], m02 = q[2], m03 = q[3], m11 = q[4], m12 = q[5], m13 = q[6], m22 = q[7],
          m23 = q[8], m33 = q[9];
    float r0 = m00 * x + m01 * y + m02 * z + m03 * w;
    float r1 = m01 * x + m11 * y + m12 * z + m13 * w;
    float r2 = m02 * x + m12 * y + m22 * z + m23 * w;
    float r3 = m03 * x + m13 * y + m23 * z + m33 * w;
    float qe = r0 * x + r1 * y + r2 * z + r3 * w;
    float cost = qe / (edge_s * edge_s);
    float tot = fclamp_t(cost + elen + Qa / (float)ntri * tres, 0.0f, COST_RANGE);
    *out = f2u_sat(tot / COST_RANGE * 4294967296.0f);
    return 1;
}

/* collapse_edge_kernel body for one winning edge, :677-773 */
static void collapse_one(s2o_ctx *c, int e)
{
    int u = c->edges[2 * e], v = c->edges[2 * e + 1];
    v3 *P = c->pts;
    t3 *T = c->tris;
    const int *fn = c->first_near, *nr = c->near;
    v3 v0 = c->opts[u], v1 = c->opts[v];
    v3 mid = {(v0.x + v1.x) / 2.0f, (v0.y + v1.y) / 2.0f, (v0.z + v1.z) / 2.0f};
    P[u] = mid;
    P[v].x = P[v].y = P[v].z = 0.0f;
    c->occ[v] = 0;
    for (int a = fn[u]; a < fn[u + 1]; ++a) {
        t3 *t = &T[nr[a]];
        if (tri_has(*t, v)) t->i = t->j = t->k = -1;
    }
    for (int a = fn[v]; a < fn[v + 1]; ++a) {
        t3 *t = &T[nr[a]];
        if (tri_has(*t, u)) t->i = t->j = t->k = -1;
        else if (t->i == v) t->i = u;
        else if (t->j == v) t->j = u;
        else if (t->k == v) t->k = u;
    }
    int sk = 0;
    for (int pass = 0; pass < 2 && !sk; ++pass) {
        int w = pass ? v : u;
        for (int a = fn[w]; a < fn[w + 1]; ++a) {
            t3 t = T[nr[a]];
            if (t.i == -1) continue;
            if (is_skinny(P[t.i], P[t.j], P[t.k])) { sk = 1; break; }
        }
    }
    if (sk) {
        c->occ[v] = 1;
        P[u] = c->opts[u];
        P[v] = c->opts[v];
        for (int a = fn[u]; a < fn[u + 1]; ++a) T[nr[a]] = c->otris[nr[a]];
        for (int a = fn[v]; a < fn[v + 1]; ++a) T[nr[a]] = c->otris[nr[a]];
    }
}

/* remove_line_edge_collapse body, :234-274 */
static void line_collapse_one(s2o_ctx *c, int e)
{
    int u = c->edges[2 * e], v = c->edges[2 * e + 1];
    t3 *T = c->tris;
    const int *fn = c->first_near, *nr = c->near;
    c->pts[v].x = c->pts[v].y = c->pts[v].z = 0.0f;
    c->occ[v] = 0;
    for (int a = fn[u]; a < fn[u + 1]; ++a) {
        t3 *t = &T[nr[a]];
        if (tri_has(*t, v)) t->i = t->j = t->k = -1;
    }
    for (int a = fn[v]; a < fn[v + 1]; ++a) {
        t3 *t = &T[nr[a]];
        if (tri_has(*t, u)) t->i = t->j = t->k = -1;
        else if (t->i == v) t->i = u;
        else if (t->j == v) t->j = u;
        else if (t->k == v) t->k = u;
    }
}

/* ------------------------------------------------ self intersection */
typedef struct { float lo[3], hi[3]; int f; } box_t;
static int cmp_box(const void *a, const void *b)
{
    const box_t *x = a, *y = b;
    if (x->lo[0] < y->lo[0]) return -1;
    if (x->lo[0] > y->lo[0]) return 1;
    return x->f - y->f;
}

static inline void face_coords(const s2o_ctx *c, int f, float out9[9], int idx[3])
{
    t3 t = c->tris[f];
    int id[3] = {t.i, t.j, t.k};
    for (int a = 0; a < 3; ++a) {
        idx[a] = id[a];
        v3 p = c->pts[id[a]];
        out9[3 * a] = p.x; out9[3 * a + 1] = p.y; out9[3 * a + 2] = p.z;
    }
}

/* Marks isect[f] = 1 for every live face in an intersecting pair.  Candidate
 * pairs are all live face pairs whose (inclusive) AABBs overlap, i.e. exactly the
 * set the reference's LBVH traversal enumerates; each unordered pair is tested
 * in both directions as the reference does. Returns the number of candidate
 * (unordered) pairs. */
static long long self_intersect(s2o_ctx *c, float eps)
{
    int m = c->n_tris;
    memset(c->isect, 0, (size_t)m);
    box_t *bx = (box_t *)malloc(sizeof(box_t) * (size_t)(m ? m : 1));
    int nb = 0;
    for (int f = 0; f < m; ++f) {
        t3 t = c->tris[f];
        if (t.i == -1) continue;
        v3 a = c->pts[t.i], b = c->pts[t.j], d = c->pts[t.k];
        box_t B;
        B.lo[0] = fminf(a.x, fminf(b.x, d.x)); B.hi[0] = fmaxf(a.x, fmaxf(b.x, d.x));
        B.lo[1] = fminf(a.y, fminf(b.y, d.y)); B.hi[1] = fmaxf(a.y, fmaxf(b.y, d.y));
        B.lo[2] = fminf(a.z, fminf(b.z, d.z)); B.hi[2] = fmaxf(a.z, fmaxf(b.z, d.z));
        B.f = f;
        bx[nb++] = B;
    }
    qsort(bx, (size_t)nb, sizeof(box_t), cmp_box);
    long long ncand = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : ncand)
    for (int i = 0; i < nb; ++i) {
        const box_t *A = &bx[i];
        float ca[9], cb[9];
        int ia[3], ib[3];
        int have_a = 0;
        for (int j = i + 1; j < nb && bx[j].lo[0] <= A->hi[0]; ++j) {
            const box_t *B = &bx[j];
            if (A->hi[1] < B->lo[1] || B->hi[1] < A->lo[1]) continue;
            if (A->hi[2] < B->lo[2] || B->hi[2] < A->lo[2]) continue;
            if (A->hi[0] < B->lo[0] || B->hi[0] < A->lo[0]) continue;
            ncand++;
            if (!have_a) { face_coords(c, A->f, ca, ia); have_a = 1; }
            face_coords(c, B->f, cb, ib);
            int hit = s2o_pair_flag(ca, ia, cb, ib, eps) || s2o_pair_flag(cb, ib, ca, ia, eps);
            if (hit) {
#pragma omp atomic write
                c->isect[A->f] = 1;
#pragma omp atomic write
                c->isect[B->f] = 1;
            }
        }
    }
    free(bx);
    return ncand;
}

/* get_undo_candidate_kernel, :776-827 (flag array instead of the list scan) */
static int undo_candidates(s2o_ctx *c)
{
    int cnt = 0;
    const int *fn = c->first_near, *nr = c->near;
    for (int p = 0; p < c->n_considered; ++p) {
        int e = c->collapsed[p];
        int u = c->edges[2 * e], v = c->edges[2 * e + 1];
        int hit = 0;
        for (int a = fn[u]; a < fn[u + 1] && !hit; ++a) hit = c->isect[nr[a]];
        for (int a = fn[v]; a < fn[v + 1] && !hit; ++a) hit = c->isect[nr[a]];
        if (hit) {
            c->undo_edges[cnt] = e;
            c->tmp_undo[2 * cnt] = u;
            c->tmp_undo[2 * cnt + 1] = v;
            cnt++;
        }
    }
    return cnt;
}

/* --------------------------------------------------------------- forward */
int s2o_forward(s2o_ctx *c, const float *pts, const int *tris, const int *undo_in, int n_undo_in, int n_pts,
                int n_tris, float scale, float threshold, int is_stuck, float *out_pts, int *out_tris,
                int *out_occ, int *out_map, int *out_n_undo)
{
    if (!c || n_pts < 0 || n_tris < 0 || n_undo_in < 0) return S2O_ERR_ARG;
    int rc = ensure(c, n_pts, n_tris);
    if (rc) return rc;
    const float eps = 1e-3f;
    c->n_pts = n_pts;
    c->n_tris = n_tris;
    int nvu = 0, first = 0;
    if (is_stuck) {
        memcpy(c->tmp_undo, undo_in, (size_t)n_undo_in * 4);
        nvu += n_undo_in;
        for (int i = 0; i < nvu - first; ++i) c->undo_list[first + i] = c->pts_map[c->tmp_undo[i]];
        first += n_undo_in;
    } else if (n_undo_in != 0) {
        memset(c->invalid_table, 0, (size_t)c->cap_pts + 1);
    }
    for (int i = 0; i < n_undo_in; ++i) c->invalid_table[undo_in[i]] = 1;

    float tres = threshold, edge_s = scale;
    uint32_t collapse_t = (uint32_t)(uint64_t)(fclamp_t(threshold, 0.0f, COST_RANGE) / COST_RANGE * 4294967296.0f);

    memcpy(c->pts, pts, (size_t)n_pts * sizeof(v3));
    for (int i = 0; i < n_pts; ++i) c->occ[i] = 1;
    c->occ[n_pts] = 0;
    memcpy(c->tris, tris, (size_t)n_tris * sizeof(t3));
    memcpy(c->opts, c->pts, (size_t)n_pts * sizeof(v3));
    memcpy(c->otris, c->tris, (size_t)n_tris * sizeof(t3));

    build_csr(c);
    build_edges(c);
    compute_Q(c);
    int E = c->n_edges;
#pragma omp parallel for schedule(dynamic, 1024)
    for (int e = 0; e < E; ++e) {
        uint32_t val;
        if (edge_cost_one(c, e, is_stuck, tres, edge_s, &val)) c->edge_cost[e] = val;
    }
    /* propagate_edge_cost_kernel, :587-610 */
    for (int f = 0; f < n_tris; ++f) c->tri_min[f] = UINT64_MAX;
    const int *fn = c->first_near, *nr = c->near;
    for (int e = 0; e < E; ++e) {
        uint64_t key = ((uint64_t)c->edge_cost[e] << 32) | (uint32_t)e;
        int u = c->edges[2 * e], v = c->edges[2 * e + 1];
        for (int a = fn[u]; a < fn[u + 1]; ++a) if (key < c->tri_min[nr[a]]) c->tri_min[nr[a]] = key;
        for (int a = fn[v]; a < fn[v + 1]; ++a) if (key < c->tri_min[nr[a]]) c->tri_min[nr[a]] = key;
    }
    /* collapse_edge_kernel selection, :639-675 */
    int nmain = 0;
    for (int e = 0; e < E; ++e) {
        if (c->edge_cost[e] > collapse_t) continue;
        uint64_t key = ((uint64_t)c->edge_cost[e] << 32) | (uint32_t)e;
        int u = c->edges[2 * e], v = c->edges[2 * e + 1], ok = 1;
        for (int a = fn[u]; a < fn[u + 1] && ok; ++a) ok = c->tri_min[nr[a]] == key;
        for (int a = fn[v]; a < fn[v + 1] && ok; ++a) ok = c->tri_min[nr[a]] == key;
        if (ok) c->collapsed[nmain++] = e;
    }
    for (int p = 0; p < nmain; ++p) collapse_one(c, c->collapsed[p]);
    c->n_main = nmain;

    /* remove_invalid_faces, :218-232 */
    for (int f = 0; f < n_tris; ++f) {
        t3 *t = &c->tris[f];
        if (tri_dead(*t)) continue;
        if (t->i == t->j || t->j == t->k || t->k == t->i) t->i = t->j = t->k = -1;
    }
    /* remove_line_edge_collapse: snapshot reads, ordered writes */
    for (int e = 0; e < E; ++e) {
        v3 p = c->pts[c->edges[2 * e]], q = c->pts[c->edges[2 * e + 1]];
        c->line_flag[e] = (p.x == q.x && p.y == q.y && p.z == q.z);
    }
    int ntot = nmain;
    for (int e = 0; e < E; ++e)
        if (c->line_flag[e]) { c->collapsed[ntot++] = e; line_collapse_one(c, e); }
    c->n_total = ntot;
    int window = ((nmain + 511) / 512) * 512;
    c->n_considered = ntot < window ? ntot : window;

    memset(c->n_cand_pairs, 0, sizeof(c->n_cand_pairs));
    memset(c->undo_counts, 0, sizeof(c->undo_counts));
    c->n_cand_pairs[0] = self_intersect(c, eps);
    memcpy(c->isect0, c->isect, (size_t)n_tris);
    int cnt = undo_candidates(c);
    c->undo_counts[0] = cnt;
    nvu += 2 * cnt;
    int it = 0;
    while (cnt != 0) {
        it++;
        for (int k = 0; k < cnt; ++k) {
            int e = c->undo_edges[k];
            int u = c->edges[2 * e], v = c->edges[2 * e + 1];
            c->occ[v] = 1;
            c->pts[u] = c->opts[u];
            c->pts[v] = c->opts[v];
            for (int a = fn[u]; a < fn[u + 1]; ++a) c->tris[nr[a]] = c->otris[nr[a]];
            for (int a = fn[v]; a < fn[v + 1]; ++a) c->tris[nr[a]] = c->otris[nr[a]];
        }
        for (int i = 0; i < nvu - first; ++i) c->undo_list[first + i] = c->pts_map[c->tmp_undo[i]];
        first += 2 * cnt;
        c->n_cand_pairs[it < 8 ? it : 7] = self_intersect(c, eps);
        cnt = undo_candidates(c);
        if (it < 8) c->undo_counts[it] = cnt;
        nvu += 2 * cnt;
        if (it == 5) break;
    }
    c->n_undo_passes = it;
    c->n_vertices_undo = nvu;
    /* pts_map = exclusive scan of occ over n_pts + 1 entries, :1042-1045 */
    int s = 0;
    for (int i = 0; i <= n_pts; ++i) { int o = c->occ[i]; c->pts_map[i] = s; s += o; }

    if (out_pts) memcpy(out_pts, c->pts, (size_t)n_pts * sizeof(v3));
    if (out_tris) memcpy(out_tris, c->tris, (size_t)n_tris * sizeof(t3));
    if (out_occ) memcpy(out_occ, c->occ, (size_t)n_pts * 4);
    if (out_map) memcpy(out_map, c->pts_map, (size_t)n_pts * 4);
    if (out_n_undo) *out_n_undo = nvu;
    return S2O_OK;
}

const int *s2o_undo_list(const s2o_ctx *c) { return c->undo_list; }
const unsigned char *s2o_isect0(const s2o_ctx *c) { return c->isect0; }
int s2o_n_edges(const s2o_ctx *c) { return c->n_edges; }
const int *s2o_edges(const s2o_ctx *c) { return c->edges; }
const uint32_t *s2o_edge_cost(const s2o_ctx *c) { return c->edge_cost; }
const int *s2o_collapsed(const s2o_ctx *c) { return c->collapsed; }
const float *s2o_Q(const s2o_ctx *c) { return c->Q; }
const int *s2o_first_near(const s2o_ctx *c) { return c->first_near; }
const int *s2o_near(const s2o_ctx *c) { return c->near; }
/* stats: [n_edges, n_main, n_total, n_considered, n_undo_passes, n_vertices_undo, undo_counts[0..7]] */
void s2o_stats(const s2o_ctx *c, int *out)
{
    out[0] = c->n_edges; out[1] = c->n_main; out[2] = c->n_total; out[3] = c->n_considered;
    out[4] = c->n_undo_passes; out[5] = c->n_vertices_undo;
    for (int i = 0; i < 8; ++i) out[6 + i] = c->undo_counts[i];
}

/* --------------------------------------------------- PaMO.run stage-2 driver */
/* Centring of PaMO.run / preprocess_mesh (simp_cuda/pamo/__init__.py:60-72,144):
 * tris_mean = mean over faces of the per-face vertex mean, both as numpy computes
 * them for float32: ((a0+a1)+a2)/3 per face, then a sequential float32 sum over
 * faces divided by F. */
void s2o_tris_mean(const float *pts, const int *tris, int n_tris, float out[3])
{
    for (int c = 0; c < 3; ++c) {
        float s = 0.0f;
        for (int f = 0; f < n_tris; ++f) {
            float a = pts[3 * tris[3 * f] + c], b = pts[3 * tris[3 * f + 1] + c], d = pts[3 * tris[3 * f + 2] + c];
            float m = ((a + b) + d) / 3.0f;
            s = f == 0 ? m : s + m;
        }
        out[c] = s / (float)n_tris;
    }
}

/* Stage-2 loop of PaMO.run (pamo/__init__.py:148-189) on the CPU.  `tris` must
 * already carry the init shuffle.  Outputs the compacted mesh (vertices still
 * centred, i.e. before "+ tris_mean"). Returns the number of rounds. */
int s2o_run(s2o_ctx *c, const float *pts_c, const int *tris_shuffled, int n_pts, int n_tris, int target_faces,
            int tolerance, float threshold, int iters, float *out_pts, int *out_tris, int *out_n)
{
    float *P = (float *)malloc((size_t)n_pts * 12 + 12), *P2 = (float *)malloc((size_t)n_pts * 12 + 12);
    int *T = (int *)malloc((size_t)n_tris * 12 + 12), *T2 = (int *)malloc((size_t)n_tris * 12 + 12);
    int *occ = (int *)malloc((size_t)n_pts * 4 + 4), *map = (int *)malloc((size_t)n_pts * 4 + 4);
    int *undo = (int *)malloc(4), n_undo = 0;
    memcpy(P, pts_c, (size_t)n_pts * 12);
    memcpy(T, tris_shuffled, (size_t)n_tris * 12);
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < n_pts; ++i)
        for (int k = 0; k < 3; ++k) {
            float x = P[3 * i + k];
            if (x < lo[k]) lo[k] = x;
            if (x > hi[k]) hi[k] = x;
        }
    float sx = hi[0] - lo[0], sy = hi[1] - lo[1], sz = hi[2] - lo[2];
    float scale = sx > sy ? sx : sy; /* Python max() keeps the first on ties */
    scale = scale > sz ? scale : sz;
    int nv = n_pts, nf = n_tris, count = 0, stuck = 0, rounds = 0;
    for (int it = 0; it < iters; ++it) {
        int prev = nf;
        int nu_out = 0;
        s2o_forward(c, P, T, undo, n_undo, nv, nf, scale, threshold, stuck, P2, T2, occ, map, &nu_out);
        rounds++;
        free(undo);
        undo = (int *)malloc((size_t)(nu_out ? nu_out : 1) * 4);
        memcpy(undo, c->undo_list, (size_t)nu_out * 4);
        n_undo = nu_out;
        int k = 0;
        for (int i = 0; i < nv; ++i)
            if (occ[i]) { memcpy(P + 3 * k, P2 + 3 * i, 12); k++; }
        int nfo = 0;
        for (int f = 0; f < nf; ++f)
            if (T2[3 * f] >= 0) {
                for (int a = 0; a < 3; ++a) T[3 * nfo + a] = map[T2[3 * f + a]];
                nfo++;
            }
        nv = k;
        nf = nfo;
        if (nf <= target_faces || nf <= 10) break;
        if (nf == prev) count++;
        else { count = 0; stuck = 0; }
        if (count >= 2) stuck = 1;
        if (count == tolerance) break;
    }
    memcpy(out_pts, P, (size_t)nv * 12);
    memcpy(out_tris, T, (size_t)nf * 12);
    out_n[0] = nv;
    out_n[1] = nf;
    free(P); free(P2); free(T); free(T2); free(occ); free(map); free(undo);
    return rounds;
}

int s2o_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
