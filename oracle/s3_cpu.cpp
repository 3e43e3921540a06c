// Stage 3 (safe projection) restated in C++ for the host cores -- the CPU
// baseline of bench.py (cpu_baseline / --impl reference).  TEST AND BASELINE
// INFRASTRUCTURE: nothing in the product links or calls it.
//
// It follows oracle/s3_oracle.py step for step (itself the restatement of the
// reference's default stage-3 configuration: system.py:354-470,
// cg_solver.py:96-158, energy_kernels/*, ccd_kernels.py:8-110,
// contact_detection.py:120-216, distance_kernels.py), in float32 as the
// reference's Warp kernels compute, with OpenMP over vertices, triangles,
// hinges and contact blocks.  Energies and CG dot products are summed in
// double.  Spatial queries use uniform grids: closest points on the ground
// truth (expanding rings of cells until no unvisited cell can be closer), and
// the contact candidates (boxes grown by the detection threshold).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <omp.h>

namespace {

struct V3 {
    float x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float norm(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 vmin(V3 a, V3 b) { return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)}; }
inline float comp(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

enum { PT = 0, PP01, PP02, PE012, PP03, PE031, PE023 };
enum { EE_PP02 = 0, EE_PP03, EE_PP12, EE_PP13, EE_PE023, EE_PE123, EE_PE201, EE_PE301, EE_EE };
enum { BLOCK_PT = 3, BLOCK_EE = 4 };

struct Cfg {
    int n_newton = 10, n_cg = 40, n_ls = 10, ccd_max = 100, spd_iters = 3;
    float d_hat = 1e-3f, kappa = 1e2f, radius = 1e-2f, ee_thres = 1e-3f, slack = 0.7f, thick = 1e-6f;
    float young = 1e-1f, poisson = 0.f, hinge_k = 1e-2f, gt_k = 1e3f;
    long long max_blocks = 1LL << 25;
};

// --------------------------------------------------------- distances
float pe_distance(V3 x0, V3 x1, V3 x2) { return norm(cross(x1 - x0, x2 - x0)) / norm(x1 - x2); }

int pt_classify(V3 x0, V3 x1, V3 x2, V3 x3)
{
    const V3 x10 = x0 - x1, x12 = x2 - x1, x13 = x3 - x1;
    const V3 cr = cross(x12, x13);
    const float area_sq = dot(cr, cr);
    if (area_sq <= 1e-6f * (dot(x12, x12) * dot(x13, x13)) || area_sq <= 1e-16f) {
        const float d1 = norm(x10), d2 = norm(x0 - x2), d3 = norm(x0 - x3);
        return d1 < d2 ? (d1 < d3 ? PP01 : PP03) : (d2 < d3 ? PP02 : PP03);
    }
    const V3 n = (1.f / std::sqrt(area_sq)) * cr;
    const V3 proj = x0 - dot(n, x10) * n;
    const V3 x10p = proj - x1, x20p = proj - x2, x30p = proj - x3;
    const float a00 = dot(x12, x12), a01 = dot(x12, x13), a11 = dot(x13, x13);
    const float b0 = dot(x10p, x12), b1 = dot(x10p, x13);
    const float det = a00 * a11 - a01 * a01;
    const float beta = b0 * a11 - b1 * a01, gamma = a00 * b1 - b0 * a01, alpha = det - beta - gamma;
    const int neg = (alpha < 0) + (beta < 0) + (gamma < 0);
    if (neg == 0) return PT;
    const V3 x23 = x3 - x2, x31 = x1 - x3;
    if (neg == 1) {
        if (alpha < 0) {
            const float dr = dot(x23, x0 - x2);
            return dr < 0 ? PP02 : (dr > dot(x23, x23) ? PP03 : PE023);
        }
        if (beta < 0) {
            const float dr = dot(x31, x0 - x3);
            return dr < 0 ? PP03 : (dr > dot(x31, x31) ? PP01 : PE031);
        }
        const float dr = dot(x12, x10p);
        return dr < 0 ? PP01 : (dr > dot(x12, x12) ? PP02 : PE012);
    }
    if (alpha >= 0) {
        const float d12 = dot(x12, x10p), d13 = dot(x13, x10p);
        if (d12 > 0 && d13 <= 0) return dot(x12, x20p) > 0 ? PP02 : PE012;
        if (d13 > 0 && d12 <= 0) return dot(x13, x30p) > 0 ? PP03 : PE031;
        return PP01;
    }
    if (beta >= 0) {
        const V3 x21 = x1 - x2;
        const float d23 = dot(x23, x20p), d21 = dot(x21, x20p);
        if (d23 > 0 && d21 <= 0) return dot(x23, x30p) > 0 ? PP03 : PE023;
        if (d21 > 0 && d23 <= 0) return dot(x21, x10p) > 0 ? PP01 : PE012;
        return PP02;
    }
    const V3 x32 = x2 - x3;
    const float d31 = dot(x31, x30p), d32 = dot(x32, x30p);
    if (d31 > 0 && d32 <= 0) return dot(x31, x10p) > 0 ? PP01 : PE031;
    if (d32 > 0 && d31 <= 0) return dot(x32, x20p) > 0 ? PP02 : PE023;
    return PP03;
}

int ee_classify(V3 x0, V3 x1, V3 x2, V3 x3, float sin_thres)
{
    const V3 e0 = x0 - x1, e1 = x2 - x3;
    const float e0_sq = dot(e0, e0), e1_sq = dot(e1, e1);
    const float a00 = e0_sq, a01 = -dot(e0, e1), a10 = dot(e0, e1), a11 = -e1_sq;
    const float b0 = dot(x3 - x1, e0), b1 = dot(x3 - x1, e1);
    const float mu0 = -(b0 * a11 - b1 * a01), mu1 = -(a00 * b1 - a10 * b0), det = -(a00 * a11 - a01 * a10);
    const float s = norm(cross((1.f / norm(e0)) * e0, (1.f / norm(e1)) * e1));
    if (mu0 >= 0 && mu0 <= det && mu1 >= 0 && mu1 <= det && s >= sin_thres && e0_sq > 1e-15f && e1_sq > 1e-15f)
        return EE_EE;
    float best = 1e9f;
    int typ = -1;
    auto endpoint = [&](V3 p, V3 a, V3 b, int t_a, int t_b, int t_e, V3 ev, float ev_sq, V3 ref) {
        const float tt = dot(p - ref, ev);
        float d;
        int t;
        if (tt >= ev_sq) {
            d = norm(a - p);
            t = t_a;
        } else if (tt <= 0) {
            d = norm(b - p);
            t = t_b;
        } else {
            d = pe_distance(p, a, b);
            t = t_e;
        }
        if (d < best) {
            best = d;
            typ = t;
        }
    };
    endpoint(x0, x2, x3, EE_PP02, EE_PP03, EE_PE023, e1, e1_sq, x3);
    endpoint(x1, x2, x3, EE_PP12, EE_PP13, EE_PE123, e1, e1_sq, x3);
    endpoint(x2, x0, x1, EE_PP02, EE_PP12, EE_PE201, e0, e0_sq, x1);
    endpoint(x3, x0, x1, EE_PP03, EE_PP13, EE_PE301, e0, e0_sq, x1);
    return typ;
}

// distance and d(distance)/dx for one classified block (X: the 4 points)
float pair_distance_grad(const V3 *X, int kind, int t, V3 *G)
{
    for (int k = 0; k < 4; ++k) G[k] = {0.f, 0.f, 0.f};
    int idx[4], n = 0;
    char what;
    if (kind == BLOCK_PT) {
        static const int tab[7][4] = {{0, 1, 2, 3}, {0, 1}, {0, 2}, {0, 1, 2}, {0, 3}, {0, 3, 1}, {0, 2, 3}};
        static const char kinds[7] = {'t', 'p', 'p', 'e', 'p', 'e', 'e'};
        static const int cnt[7] = {4, 2, 2, 3, 2, 3, 3};
        what = kinds[t];
        n = cnt[t];
        for (int k = 0; k < n; ++k) idx[k] = tab[t][k];
    } else {
        static const int tab[9][4] = {{0, 2}, {0, 3}, {1, 2}, {1, 3}, {0, 2, 3}, {1, 2, 3}, {2, 0, 1}, {3, 0, 1}, {0, 1, 2, 3}};
        static const char kinds[9] = {'p', 'p', 'p', 'p', 'e', 'e', 'e', 'e', 'E'};
        static const int cnt[9] = {2, 2, 2, 2, 3, 3, 3, 3, 4};
        what = kinds[t];
        n = cnt[t];
        for (int k = 0; k < n; ++k) idx[k] = tab[t][k];
    }
    if (what == 'p') {
        const V3 diff = X[idx[0]] - X[idx[1]];
        const float dd = norm(diff);
        const V3 u = (1.f / dd) * diff;
        G[idx[0]] = u;
        G[idx[1]] = -1.f * u;
        return dd;
    }
    if (what == 'e') {
        const V3 x0 = X[idx[0]], x1 = X[idx[1]], x2 = X[idx[2]];
        const V3 e = x2 - x1;
        const float tt = dot(x0 - x1, e) / dot(e, e);
        const V3 diff = x0 - (x1 + tt * e);
        const V3 u = (1.f / norm(diff)) * diff;
        G[idx[0]] = u;
        G[idx[1]] = -(1.f - tt) * u;
        G[idx[2]] = -tt * u;
        return pe_distance(x0, x1, x2);
    }
    if (what == 't') {
        const V3 x0 = X[0], x1 = X[1], x2 = X[2], x3 = X[3];
        V3 nrm = cross(x2 - x1, x3 - x1);
        nrm = (1.f / norm(nrm)) * nrm;
        const float sd = dot(x0 - x1, nrm);
        const V3 u = (sd > 0 ? 1.f : (sd < 0 ? -1.f : 0.f)) * nrm;
        const V3 proj = x0 - sd * nrm;
        const float a00 = dot(x2 - x1, x2 - x1), a01 = dot(x2 - x1, x3 - x1), a11 = dot(x3 - x1, x3 - x1);
        const float b0 = dot(proj - x1, x2 - x1), b1 = dot(proj - x1, x3 - x1);
        const float det = a00 * a11 - a01 * a01;
        const float be = (b0 * a11 - b1 * a01) / det, ga = (a00 * b1 - b0 * a01) / det, al = 1.f - be - ga;
        G[0] = u;
        G[1] = -al * u;
        G[2] = -be * u;
        G[3] = -ga * u;
        return std::fabs(sd);
    }
    const V3 x0 = X[0], x1 = X[1], x2 = X[2], x3 = X[3];
    V3 nrm = cross(x1 - x0, x3 - x2);
    nrm = (1.f / norm(nrm)) * nrm;
    const float sd = dot(x0 - x2, nrm);
    const V3 u = (sd > 0 ? 1.f : (sd < 0 ? -1.f : 0.f)) * nrm;
    const V3 e0 = x1 - x0, e1 = x3 - x2, w0 = x0 - x2;
    const float a = dot(e0, e0), b = dot(e0, e1), c = dot(e1, e1), dq = dot(e0, w0), eq = dot(e1, w0);
    const float den = a * c - b * b;
    const float s_ = (b * eq - c * dq) / den, t_ = (a * eq - b * dq) / den;
    G[0] = (1.f - s_) * u;
    G[1] = s_ * u;
    G[2] = -(1.f - t_) * u;
    G[3] = -t_ * u;
    return std::fabs(sd);
}

int classify(int kind, const V3 *X, float thres)
{
    return kind == BLOCK_PT ? pt_classify(X[0], X[1], X[2], X[3]) : ee_classify(X[0], X[1], X[2], X[3], thres);
}

// ------------------------------------------------------------ uniform grid
struct Grid {
    V3 lo{0, 0, 0};
    float cs = 1.f;
    int n[3] = {1, 1, 1};
    std::vector<int> first, items;

    void cell_range(V3 a, V3 b, int *c0, int *c1) const
    {
        for (int k = 0; k < 3; ++k) {
            c0[k] = std::clamp((int)std::floor((comp(a, k) - comp(lo, k)) / cs), 0, n[k] - 1);
            c1[k] = std::clamp((int)std::floor((comp(b, k) - comp(lo, k)) / cs), 0, n[k] - 1);
        }
    }
    long long cell(int x, int y, int z) const { return ((long long)z * n[1] + y) * n[0] + x; }

    // boxes [blo[i], bhi[i]] binned into every cell they overlap
    void build(const std::vector<V3> &blo, const std::vector<V3> &bhi, float cell_size)
    {
        V3 l = {1e30f, 1e30f, 1e30f}, h = {-1e30f, -1e30f, -1e30f};
        for (size_t i = 0; i < blo.size(); ++i) {
            l = vmin(l, blo[i]);
            h = vmax(h, bhi[i]);
        }
        lo = l;
        const V3 ext = h - l;
        cs = std::max(cell_size, std::max(ext.x, std::max(ext.y, ext.z)) / 510.f);  // <= 512 cells per axis
        for (int k = 0; k < 3; ++k) n[k] = std::clamp((int)std::floor((comp(h, k) - comp(l, k)) / cs) + 1, 1, 512);
        const long long nc = (long long)n[0] * n[1] * n[2];
        std::vector<int> cnt(nc + 1, 0);
        for (size_t i = 0; i < blo.size(); ++i) {
            int c0[3], c1[3];
            cell_range(blo[i], bhi[i], c0, c1);
            for (int z = c0[2]; z <= c1[2]; ++z)
                for (int y = c0[1]; y <= c1[1]; ++y)
                    for (int x = c0[0]; x <= c1[0]; ++x) cnt[cell(x, y, z)]++;
        }
        first.assign(nc + 1, 0);
        for (long long c = 0; c < nc; ++c) first[c + 1] = first[c] + cnt[c];
        items.assign(first[nc], 0);
        std::vector<int> cur(first.begin(), first.end() - 1);
        for (size_t i = 0; i < blo.size(); ++i) {
            int c0[3], c1[3];
            cell_range(blo[i], bhi[i], c0, c1);
            for (int z = c0[2]; z <= c1[2]; ++z)
                for (int y = c0[1]; y <= c1[1]; ++y)
                    for (int x = c0[0]; x <= c1[0]; ++x) items[cur[cell(x, y, z)]++] = (int)i;
        }
    }
};

V3 closest_on_tri(V3 p, V3 a, V3 b, V3 c)
{
    const V3 ab = b - a, ac = c - a, ap = p - a;
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0 && d2 <= 0) return a;
    const V3 bp = p - b;
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0 && d4 <= d3) return b;
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) return a + (d1 / (d1 - d3)) * ab;
    const V3 cp = p - c;
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0 && d5 <= d6) return c;
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) return a + (d2 / (d2 - d6)) * ac;
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) return b + ((d4 - d3) / ((d4 - d3) + (d5 - d6))) * (c - b);
    const float den = 1.f / (va + vb + vc);
    return a + (vb * den) * ab + (vc * den) * ac;
}

struct System {
    Cfg c;
    int np = 0, nt = 0, ne = 0, nh = 0;
    std::vector<V3> q, q_rest, target, gt_v;
    std::vector<int> F, E, H, gt_f;
    std::vector<float> w, area, rest_angle, rest_elen;
    std::vector<float> inv_dm;  // 4 per triangle
    Grid gt_grid;
    float mu = 0, la = 0, radius = 0;
    std::vector<int> bidx, bkind;  // 4 per block, kind per block
    // per Newton iteration
    std::vector<float> hblk;       // 144 per hinge: [4][4][3][3]
    std::vector<V3> bg;            // 4 per block
    std::vector<float> bb2;
    std::vector<V3> tbuf, hbuf;  // per-element terms of H dx
    std::vector<float> bbuf;

    void frame(V3 x01, V3 x02, V3 &b1, V3 &b2) const
    {
        b1 = (1.f / norm(x01)) * x01;
        b2 = x02 - dot(x02, b1) * b1;
        b2 = (1.f / norm(b2)) * b2;
    }

    static float hinge_angle(V3 x0, V3 x1, V3 x2, V3 x3)
    {
        const V3 e0 = x2 - x1;
        V3 n1 = cross(e0, x0 - x1), n2 = cross(x3 - x1, e0);
        n1 = (1.f / norm(n1)) * n1;
        n2 = (1.f / norm(n2)) * n2;
        const float s = dot(cross(n1, n2), e0) / norm(e0);
        return std::atan2(s, dot(n1, n2));
    }

    void update_target()
    {
#pragma omp parallel for schedule(dynamic, 256)
        for (int i = 0; i < np; ++i) {
            const V3 p = q[i];
            int c[3];
            for (int k = 0; k < 3; ++k)
                c[k] = std::clamp((int)std::floor((comp(p, k) - comp(gt_grid.lo, k)) / gt_grid.cs), 0,
                                  gt_grid.n[k] - 1);
            float best = 3e38f;
            V3 bq = p;
            const int kmax = std::max(gt_grid.n[0], std::max(gt_grid.n[1], gt_grid.n[2]));
            for (int k = 0; k <= kmax; ++k) {
                for (int z = c[2] - k; z <= c[2] + k; ++z)
                    for (int y = c[1] - k; y <= c[1] + k; ++y)
                        for (int x = c[0] - k; x <= c[0] + k; ++x) {
                            if (std::max(std::abs(x - c[0]), std::max(std::abs(y - c[1]), std::abs(z - c[2]))) != k)
                                continue;  // the ring only
                            if (x < 0 || y < 0 || z < 0 || x >= gt_grid.n[0] || y >= gt_grid.n[1] || z >= gt_grid.n[2])
                                continue;
                            const long long cc = gt_grid.cell(x, y, z);
                            for (int s = gt_grid.first[cc]; s < gt_grid.first[cc + 1]; ++s) {
                                const int t = gt_grid.items[s];
                                const V3 cp = closest_on_tri(p, gt_v[gt_f[3 * t]], gt_v[gt_f[3 * t + 1]],
                                                             gt_v[gt_f[3 * t + 2]]);
                                const float d2 = dot(p - cp, p - cp);
                                if (d2 < best) {
                                    best = d2;
                                    bq = cp;
                                }
                            }
                        }
                // every unvisited cell lies farther than k cells from p's cell
                const float reach = (float)k * gt_grid.cs;
                if (best <= reach * reach) break;
            }
            target[i] = bq;
        }
    }

    void detect()
    {
        const float thr = 2.f * radius + c.d_hat;
        // point-triangle: triangle boxes grown by thr, one grid
        std::vector<V3> blo(nt), bhi(nt);
        float avg = 0.f;
        for (int t = 0; t < nt; ++t) {
            const V3 a = q[F[3 * t]], b = q[F[3 * t + 1]], cc = q[F[3 * t + 2]];
            blo[t] = vmin(a, vmin(b, cc)) - V3{thr, thr, thr};
            bhi[t] = vmax(a, vmax(b, cc)) + V3{thr, thr, thr};
            avg += comp(bhi[t] - blo[t], 0);
        }
        Grid g;
        g.build(blo, bhi, std::max(avg / std::max(nt, 1), 1e-6f));
        std::vector<std::vector<int>> local(omp_get_max_threads());
#pragma omp parallel
        {
            std::vector<int> &out = local[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 256)
            for (int v = 0; v < np; ++v) {
                const V3 p = q[v];
                int c0[3], c1[3];
                g.cell_range(p, p, c0, c1);
                const long long cc = g.cell(c0[0], c0[1], c0[2]);
                for (int s = g.first[cc]; s < g.first[cc + 1]; ++s) {
                    const int t = g.items[s];
                    if (p.x < blo[t].x || p.y < blo[t].y || p.z < blo[t].z || p.x > bhi[t].x || p.y > bhi[t].y ||
                        p.z > bhi[t].z)
                        continue;
                    const int a = F[3 * t], b = F[3 * t + 1], e = F[3 * t + 2];
                    if (a == v || b == v || e == v) continue;
                    const V3 X[4] = {p, q[a], q[b], q[e]};
                    V3 G[4];
                    const float d = pair_distance_grad(X, BLOCK_PT, pt_classify(X[0], X[1], X[2], X[3]), G);
                    if (d <= thr) out.insert(out.end(), {v, a, b, e, BLOCK_PT});
                }
            }
        }
        // edge-edge: the grid bins edge boxes grown by thr; a pair is a
        // candidate when a's box grown by thr overlaps b's box
        std::vector<V3> elo(ne), ehi(ne), glo(ne), ghi(ne);
        float eavg = 0.f;
        for (int k = 0; k < ne; ++k) {
            const V3 a = q[E[2 * k]], b = q[E[2 * k + 1]];
            elo[k] = vmin(a, b);
            ehi[k] = vmax(a, b);
            glo[k] = elo[k] - V3{thr, thr, thr};
            ghi[k] = ehi[k] + V3{thr, thr, thr};
            eavg += comp(ghi[k] - glo[k], 0);
        }
        Grid ge;
        ge.build(glo, ghi, std::max(eavg / std::max(ne, 1), 1e-6f));
#pragma omp parallel
        {
            std::vector<int> &out = local[omp_get_thread_num()];
            std::vector<int> cand;
#pragma omp for schedule(dynamic, 256)
            for (int a = 0; a < ne; ++a) {
                int c0[3], c1[3];
                ge.cell_range(glo[a], ghi[a], c0, c1);
                cand.clear();
                for (int z = c0[2]; z <= c1[2]; ++z)
                    for (int y = c0[1]; y <= c1[1]; ++y)
                        for (int x = c0[0]; x <= c1[0]; ++x) {
                            const long long cc = ge.cell(x, y, z);
                            for (int s = ge.first[cc]; s < ge.first[cc + 1]; ++s)
                                if (ge.items[s] > a) cand.push_back(ge.items[s]);
                        }
                std::sort(cand.begin(), cand.end());
                cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
                for (int b : cand) {
                    if (elo[a].x - thr > ehi[b].x || elo[a].y - thr > ehi[b].y || elo[a].z - thr > ehi[b].z ||
                        elo[b].x > ehi[a].x + thr || elo[b].y > ehi[a].y + thr || elo[b].z > ehi[a].z + thr)
                        continue;
                    const int a0 = E[2 * a], a1 = E[2 * a + 1], b0 = E[2 * b], b1 = E[2 * b + 1];
                    if (a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1) continue;
                    const V3 X[4] = {q[a0], q[a1], q[b0], q[b1]};
                    V3 G[4];
                    const float d =
                        pair_distance_grad(X, BLOCK_EE, ee_classify(X[0], X[1], X[2], X[3], c.ee_thres), G);
                    if (d <= thr) out.insert(out.end(), {a0, a1, b0, b1, BLOCK_EE});
                }
            }
        }
        bidx.clear();
        bkind.clear();
        size_t total = 0;
        for (auto &o : local) total += o.size() / 5;
        if (total > (size_t)c.max_blocks) {  // too many contacts: halve the radius for good
            radius *= 0.5f;
            detect();
            return;
        }
        bidx.reserve(4 * total);
        bkind.reserve(total);
        for (auto &o : local)
            for (size_t k = 0; k < o.size(); k += 5) {
                bidx.insert(bidx.end(), o.begin() + k, o.begin() + k + 4);
                bkind.push_back(o[k + 4]);
            }
    }

    static double barrier(double d, double dh) { return d < dh ? -(d - dh) * (d - dh) * std::log(d / dh) : 0.0; }
    static double barrier_d1(double d, double dh)
    {
        const double t = d - dh;
        return d < dh ? -2 * t * std::log(d / dh) - t * t / d : 0.0;
    }
    static double barrier_d2(double d, double dh)
    {
        return d < dh ? -2 * std::log(d / dh) - 2 * (d - dh) / d - 1 + dh * dh / (d * d) : 0.0;
    }

    void elastic_F(const std::vector<V3> &x, int t, float Fm[4], V3 &b1, V3 &b2) const
    {
        const V3 x01 = x[F[3 * t + 1]] - x[F[3 * t]], x02 = x[F[3 * t + 2]] - x[F[3 * t]];
        frame(x01, x02, b1, b2);
        const float D[4] = {dot(b1, x01), dot(b1, x02), dot(b2, x01), dot(b2, x02)};
        const float *im = &inv_dm[4 * t];
        Fm[0] = D[0] * im[0] + D[1] * im[2];
        Fm[1] = D[0] * im[1] + D[1] * im[3];
        Fm[2] = D[2] * im[0] + D[3] * im[2];
        Fm[3] = D[2] * im[1] + D[3] * im[3];
    }

    double energy(const std::vector<V3> &x) const
    {
        double e = 0.0;
#pragma omp parallel for reduction(+ : e) schedule(static)
        for (int i = 0; i < np; ++i) {
            const V3 d = x[i] - target[i];
            e += 0.5 * (double)(dot(d, d) * w[i]);
        }
#pragma omp parallel for reduction(+ : e) schedule(static)
        for (int t = 0; t < nt; ++t) {
            float Fm[4];
            V3 b1, b2;
            elastic_F(x, t, Fm, b1, b2);
            const float e00 = 0.5f * (Fm[0] * Fm[0] + Fm[2] * Fm[2] - 1.f), e01 = 0.5f * (Fm[0] * Fm[1] + Fm[2] * Fm[3]);
            const float e11 = 0.5f * (Fm[1] * Fm[1] + Fm[3] * Fm[3] - 1.f), tr = e00 + e11;
            e += (double)(area[t] * (mu * (e00 * e00 + 2.f * e01 * e01 + e11 * e11) + 0.5f * la * tr * tr));
        }
#pragma omp parallel for reduction(+ : e) schedule(static)
        for (int h = 0; h < nh; ++h) {
            const float th = hinge_angle(x[H[4 * h]], x[H[4 * h + 1]], x[H[4 * h + 2]], x[H[4 * h + 3]]);
            const float dt = th - rest_angle[h];
            e += (double)(0.5f * c.hinge_k * dt * dt * rest_elen[h]);
        }
        const int nb = (int)bkind.size();
#pragma omp parallel for reduction(+ : e) schedule(static)
        for (int b = 0; b < nb; ++b) {
            const V3 X[4] = {x[bidx[4 * b]], x[bidx[4 * b + 1]], x[bidx[4 * b + 2]], x[bidx[4 * b + 3]]};
            V3 G[4];
            const float d = pair_distance_grad(X, bkind[b], classify(bkind[b], X, c.ee_thres), G);
            if (d < c.d_hat) e += barrier(d, c.d_hat) * c.kappa;
        }
        return e;
    }

    // dE/dx (4 x 3) and the 16 3x3 Hessian blocks of one hinge
    // (Tamstorf & Grinspun 2013, the oracle's _hinge_blocks)
    void hinge_blocks(const std::vector<V3> &x, int h, V3 *grad, float *B) const
    {
        const V3 x0 = x[H[4 * h]], x1 = x[H[4 * h + 1]], x2 = x[H[4 * h + 2]], x3 = x[H[4 * h + 3]];
        const V3 e0 = x2 - x1, e1 = x0 - x2, e2 = x0 - x1, e1_ = x3 - x2, e2_ = x3 - x1;
        const float l0 = norm(e0);
        const V3 u0 = (1.f / l0) * e0, u1 = (1.f / norm(e1)) * e1, u2 = (1.f / norm(e2)) * e2;
        const V3 u1_ = (1.f / norm(e1_)) * e1_, u2_ = (1.f / norm(e2_)) * e2_;
        const float ca1 = dot(u2, u0), ca2 = -dot(u1, u0), ca1_ = dot(u2_, u0), ca2_ = -dot(u1_, u0);
        const float h0 = norm(cross(e1, e2)) / l0, h1 = norm(cross(e0, e2)) / norm(e1), h2 = norm(cross(e0, e1)) / norm(e2);
        const float h0_ = norm(cross(e1_, e2_)) / l0, h1_ = norm(cross(e0, e2_)) / norm(e1_);
        const float h2_ = norm(cross(e0, e1_)) / norm(e2_);
        V3 n = cross(e0, e2);
        n = (1.f / norm(n)) * n;
        V3 n_ = cross(e2_, e0);
        n_ = (1.f / norm(n_)) * n_;
        const float th = std::atan2(dot(cross(n, n_), e0) / l0, dot(n, n_));
        const int hh = h;
        const float dE = c.hinge_k * (th - rest_angle[hh]) * rest_elen[hh], d2E = c.hinge_k * rest_elen[hh];
        const V3 g0 = (-1.f / h0) * n, g3 = (-1.f / h0_) * n_;
        const V3 g1 = (ca2 / h1) * n + (ca2_ / h1_) * n_, g2 = (ca1 / h2) * n + (ca1_ / h2_) * n_;
        const V3 gt[4] = {g0, g1, g2, g3};
        for (int k = 0; k < 4; ++k) grad[k] = dE * gt[k];
        auto unit = [](V3 v) { return (1.f / norm(v)) * v; };
        const V3 m0 = unit(cross(e0, n)), m1 = unit(cross(e1, n)), m2 = unit(cross(n, e2));
        const V3 m0_ = unit(cross(n_, e0)), m1_ = unit(cross(n_, e1_)), m2_ = unit(cross(e2_, n_));
        // 3x3 helpers (row-major)
        auto outer = [](V3 a, V3 b, float *M) {
            const float av[3] = {a.x, a.y, a.z}, bv[3] = {b.x, b.y, b.z};
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) M[3 * i + j] = av[i] * bv[j];
        };
        float M0[9], M1[9], M2[9], M0_[9], M1_[9], M2_[9];
        outer(n, m0, M0); outer(n, m1, M1); outer(n, m2, M2);
        outer(n_, m0_, M0_); outer(n_, m1_, M1_); outer(n_, m2_, M2_);
        auto T = [](const float *A, float *R) {
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) R[3 * i + j] = A[3 * j + i];
        };
        float TM0[9], TM1[9], TM2[9], TM0_[9], TM1_[9], TM2_[9];
        T(M0, TM0); T(M1, TM1); T(M2, TM2); T(M0_, TM0_); T(M1_, TM1_); T(M2_, TM2_);
        float *blk[4][4];
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) blk[i][j] = B + 9 * (4 * i + j);
        auto set = [&](float *dst, std::initializer_list<std::pair<float, const float *>> terms, V3 ga, V3 gb) {
            float ggt[9];
            outer(ga, gb, ggt);
            for (int k = 0; k < 9; ++k) {
                float acc = 0.f;
                for (auto &tm : terms) acc += tm.first * tm.second[k];
                dst[k] = acc * dE + d2E * ggt[k];
            }
        };
        const float l02 = l0 * l0;
        // sym(A) = A + A^T expressed through the transposed copies
        set(blk[0][0], {{-1.f / (h0 * h0), M0}, {-1.f / (h0 * h0), TM0}}, g0, g0);
        set(blk[3][3], {{-1.f / (h0_ * h0_), M0_}, {-1.f / (h0_ * h0_), TM0_}}, g3, g3);
        set(blk[1][1], {{ca1 / (h1 * h1), TM1}, {ca1 / (h1 * h1), M1}, {-1.f / l02, M0},
                        {ca1_ / (h1_ * h1_), TM1_}, {ca1_ / (h1_ * h1_), M1_}, {-1.f / l02, M0_}}, g1, g1);
        set(blk[2][2], {{ca2 / (h2 * h2), TM2}, {ca2 / (h2 * h2), M2}, {-1.f / l02, M0},
                        {ca2_ / (h2_ * h2_), TM2_}, {ca2_ / (h2_ * h2_), M2_}, {-1.f / l02, M0_}}, g2, g2);
        set(blk[1][0], {{ca1 / (h1 * h0), TM0}, {-1.f / (h0 * h1), M1}}, g1, g0);
        set(blk[2][0], {{ca2 / (h2 * h0), TM0}, {-1.f / (h0 * h2), M2}}, g2, g0);
        set(blk[1][3], {{ca1_ / (h1_ * h0_), TM0_}, {-1.f / (h0_ * h1_), M1_}}, g1, g3);
        set(blk[2][3], {{ca2_ / (h2_ * h0_), TM0_}, {-1.f / (h0_ * h2_), M2_}}, g2, g3);
        // P12 + P21^T + N0 + P12_ + P21_^T + N0_, with P21^T = (ca2/(h2 h1) M1^T)^T = ca2/(h2 h1) M1
        set(blk[1][2], {{ca1 / (h1 * h2), TM2}, {ca2 / (h2 * h1), M1}, {1.f / l02, M0},
                        {ca1_ / (h1_ * h2_), TM2_}, {ca2_ / (h2_ * h1_), M1_}, {1.f / l02, M0_}}, g1, g2);
        {
            float ggt[9];
            outer(g0, g3, ggt);
            for (int k = 0; k < 9; ++k) blk[0][3][k] = d2E * ggt[k];
        }
        T(blk[1][0], blk[0][1]); T(blk[2][0], blk[0][2]); T(blk[1][3], blk[3][1]);
        T(blk[2][3], blk[3][2]); T(blk[1][2], blk[2][1]); T(blk[0][3], blk[3][0]);
    }

    // eigenvalue clamp of the 9x9 matrix of hinge vertices 0-2 (cyclic Jacobi),
    // vertex 3 refilled by translation invariance (the oracle's spd_project)
    void spd_project(float *B) const
    {
        double A[9][9], V[9][9];
        for (int i = 0; i < 9; ++i)
            for (int j = 0; j < 9; ++j) {
                const int bi = i / 3, ri = i % 3, bj = j / 3, rj = j % 3;
                const int ii = 9 * (4 * bi + bj) + 3 * ri + rj, jj = 9 * (4 * bj + bi) + 3 * rj + ri;
                A[i][j] = 0.5 * ((double)B[ii] + (double)B[jj]);
                V[i][j] = i == j;
            }
        for (int sw = 0; sw < c.spd_iters; ++sw)
            for (int p = 0; p < 8; ++p)
                for (int r = p + 1; r < 9; ++r) {
                    const double apq = A[p][r];
                    if (!(std::fabs(apq) > 1e-30)) continue;
                    const double theta = (A[r][r] - A[p][p]) / (2 * apq);
                    const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                    const double cs = 1 / std::sqrt(t * t + 1), sn = t * cs;
                    for (int k = 0; k < 9; ++k) {  // A J
                        const double akp = A[k][p], akq = A[k][r];
                        A[k][p] = cs * akp - sn * akq;
                        A[k][r] = sn * akp + cs * akq;
                    }
                    for (int k = 0; k < 9; ++k) {  // J^T A
                        const double apk = A[p][k], aqk = A[r][k];
                        A[p][k] = cs * apk - sn * aqk;
                        A[r][k] = sn * apk + cs * aqk;
                    }
                    for (int k = 0; k < 9; ++k) {
                        const double vkp = V[k][p], vkq = V[k][r];
                        V[k][p] = cs * vkp - sn * vkq;
                        V[k][r] = sn * vkp + cs * vkq;
                    }
                }
        double lam[9];
        for (int i = 0; i < 9; ++i) lam[i] = std::max(A[i][i], 0.0);
        for (int i = 0; i < 9; ++i)
            for (int j = 0; j < 9; ++j) {
                double s = 0;
                for (int k = 0; k < 9; ++k) s += V[i][k] * lam[k] * V[j][k];
                const int bi = i / 3, ri = i % 3, bj = j / 3, rj = j % 3;
                B[9 * (4 * bi + bj) + 3 * ri + rj] = (float)s;
            }
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 9; ++k) {
                B[9 * (4 * 3 + j) + k] = -(B[9 * (4 * 0 + j) + k] + B[9 * (4 * 1 + j) + k] + B[9 * (4 * 2 + j) + k]);
            }
        for (int j = 0; j < 3; ++j)
            for (int r = 0; r < 3; ++r)
                for (int s = 0; s < 3; ++s) B[9 * (4 * j + 3) + 3 * r + s] = B[9 * (4 * 3 + j) + 3 * s + r];
        for (int k = 0; k < 9; ++k)
            B[9 * 15 + k] = -(B[9 * (4 * 0 + 3) + k] + B[9 * (4 * 1 + 3) + k] + B[9 * (4 * 2 + 3) + k]);
    }

    void diff(const std::vector<V3> &x, std::vector<V3> &g, std::vector<V3> &dg)
    {
        g.assign(np, {0, 0, 0});
        dg.assign(np, {0, 0, 0});
        for (int i = 0; i < np; ++i) {
            g[i] = -w[i] * (x[i] - target[i]);
            dg[i] = {w[i], w[i], w[i]};
        }
        // membranes (no diagonal term)
        for (int t = 0; t < nt; ++t) {
            float Fm[4];
            V3 b1, b2;
            elastic_F(x, t, Fm, b1, b2);
            const float e00 = 0.5f * (Fm[0] * Fm[0] + Fm[2] * Fm[2] - 1.f), e01 = 0.5f * (Fm[0] * Fm[1] + Fm[2] * Fm[3]);
            const float e11 = 0.5f * (Fm[1] * Fm[1] + Fm[3] * Fm[3] - 1.f), tr = e00 + e11;
            const float S[4] = {2 * mu * e00 + la * tr, 2 * mu * e01, 2 * mu * e01, 2 * mu * e11 + la * tr};
            const float P[4] = {Fm[0] * S[0] + Fm[1] * S[2], Fm[0] * S[1] + Fm[1] * S[3], Fm[2] * S[0] + Fm[3] * S[2],
                                Fm[2] * S[1] + Fm[3] * S[3]};
            const float *im = &inv_dm[4 * t];
            // H = -area P inv_Dm^T
            const float Hm[4] = {-area[t] * (P[0] * im[0] + P[1] * im[1]), -area[t] * (P[0] * im[2] + P[1] * im[3]),
                                 -area[t] * (P[2] * im[0] + P[3] * im[1]), -area[t] * (P[2] * im[2] + P[3] * im[3])};
            const V3 f1 = Hm[0] * b1 + Hm[2] * b2, f2 = Hm[1] * b1 + Hm[3] * b2;
            g[F[3 * t]] = g[F[3 * t]] - (f1 + f2);
            g[F[3 * t + 1]] = g[F[3 * t + 1]] + f1;
            g[F[3 * t + 2]] = g[F[3 * t + 2]] + f2;
        }
        hblk.assign(144 * (size_t)nh, 0.f);
        std::vector<V3> hg(4 * (size_t)nh);
#pragma omp parallel for schedule(static)
        for (int h = 0; h < nh; ++h) hinge_blocks(x, h, &hg[4 * (size_t)h], &hblk[144 * (size_t)h]);
        for (int h = 0; h < nh; ++h)
            for (int k = 0; k < 4; ++k) {
                const int v = H[4 * h + k];
                g[v] = g[v] - hg[4 * (size_t)h + k];
                const float *D = &hblk[144 * (size_t)h + 9 * (4 * k + k)];
                dg[v] = dg[v] + V3{D[0], D[4], D[8]};
            }
#pragma omp parallel for schedule(static)
        for (int h = 0; h < nh; ++h) spd_project(&hblk[144 * (size_t)h]);
        const int nb = (int)bkind.size();
        bg.assign(4 * (size_t)nb, {0, 0, 0});
        bb2.assign(nb, 0.f);
        std::vector<float> b1c(nb, 0.f);
#pragma omp parallel for schedule(static)
        for (int b = 0; b < nb; ++b) {
            const V3 X[4] = {x[bidx[4 * b]], x[bidx[4 * b + 1]], x[bidx[4 * b + 2]], x[bidx[4 * b + 3]]};
            const float d = pair_distance_grad(X, bkind[b], classify(bkind[b], X, c.ee_thres), &bg[4 * (size_t)b]);
            if (d < c.d_hat) {
                b1c[b] = (float)(barrier_d1(d, c.d_hat) * c.kappa);
                bb2[b] = (float)(barrier_d2(d, c.d_hat) * c.kappa);
            }
        }
        for (int b = 0; b < nb; ++b)
            if (bb2[b] != 0.f || b1c[b] != 0.f)
                for (int k = 0; k < 4; ++k) {
                    const V3 G = bg[4 * (size_t)b + k];
                    const int v = bidx[4 * b + k];
                    g[v] = g[v] - b1c[b] * G;
                    dg[v] = dg[v] + bb2[b] * V3{G.x * G.x, G.y * G.y, G.z * G.z};
                }
    }

    // H dx: element terms computed in parallel into per-element buffers, then
    // added to the vertices in element order (deterministic)
    void hess_dx(const std::vector<V3> &x, const std::vector<V3> &dx, std::vector<V3> &out)
    {
        out.resize(np);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < np; ++i) out[i] = w[i] * dx[i];
        tbuf.resize(2 * (size_t)nt);
        hbuf.resize(4 * (size_t)nh);
        const int nb = (int)bkind.size();
        bbuf.resize(nb);
#pragma omp parallel for schedule(static)
        for (int t = 0; t < nt; ++t) {
            float Fm[4];
            V3 b1, b2;
            elastic_F(x, t, Fm, b1, b2);
            const V3 dx01 = dx[F[3 * t + 1]] - dx[F[3 * t]], dx02 = dx[F[3 * t + 2]] - dx[F[3 * t]];
            const float dD[4] = {dot(b1, dx01), dot(b1, dx02), dot(b2, dx01), dot(b2, dx02)};
            const float *im = &inv_dm[4 * t];
            const float dF[4] = {dD[0] * im[0] + dD[1] * im[2], dD[0] * im[1] + dD[1] * im[3],
                                 dD[2] * im[0] + dD[3] * im[2], dD[2] * im[1] + dD[3] * im[3]};
            const float e00 = 0.5f * (Fm[0] * Fm[0] + Fm[2] * Fm[2] - 1.f), e01 = 0.5f * (Fm[0] * Fm[1] + Fm[2] * Fm[3]);
            const float e11 = 0.5f * (Fm[1] * Fm[1] + Fm[3] * Fm[3] - 1.f), tr = e00 + e11;
            // dE = (dF^T F + F^T dF) / 2
            const float d00 = dF[0] * Fm[0] + dF[2] * Fm[2];
            const float d01 = 0.5f * ((dF[0] * Fm[1] + dF[2] * Fm[3]) + (Fm[0] * dF[1] + Fm[2] * dF[3]));
            const float d11 = dF[1] * Fm[1] + dF[3] * Fm[3];
            const float dtr = d00 + d11;
            const float S[4] = {2 * mu * e00 + la * tr, 2 * mu * e01, 2 * mu * e01, 2 * mu * e11 + la * tr};
            const float dS[4] = {2 * mu * d00 + la * dtr, 2 * mu * d01, 2 * mu * d01, 2 * mu * d11 + la * dtr};
            float dP[4];
            for (int r = 0; r < 2; ++r)
                for (int cc = 0; cc < 2; ++cc)
                    dP[2 * r + cc] = dF[2 * r] * S[cc] + dF[2 * r + 1] * S[2 + cc] + Fm[2 * r] * dS[cc] +
                                     Fm[2 * r + 1] * dS[2 + cc];
            const float dH[4] = {area[t] * (dP[0] * im[0] + dP[1] * im[1]), area[t] * (dP[0] * im[2] + dP[1] * im[3]),
                                 area[t] * (dP[2] * im[0] + dP[3] * im[1]), area[t] * (dP[2] * im[2] + dP[3] * im[3])};
            tbuf[2 * (size_t)t] = dH[0] * b1 + dH[2] * b2;
            tbuf[2 * (size_t)t + 1] = dH[1] * b1 + dH[3] * b2;
        }
#pragma omp parallel for schedule(static)
        for (int h = 0; h < nh; ++h) {
            const float *B = &hblk[144 * (size_t)h];
            for (int i = 0; i < 4; ++i) {
                V3 acc{0, 0, 0};
                for (int j = 0; j < 4; ++j) {
                    const float *M = B + 9 * (4 * i + j);
                    const V3 v = dx[H[4 * h + j]];
                    acc = acc + V3{M[0] * v.x + M[1] * v.y + M[2] * v.z, M[3] * v.x + M[4] * v.y + M[5] * v.z,
                                   M[6] * v.x + M[7] * v.y + M[8] * v.z};
                }
                hbuf[4 * (size_t)h + i] = acc;
            }
        }
#pragma omp parallel for schedule(static)
        for (int b = 0; b < nb; ++b) {
            float s = 0.f;
            if (bb2[b] != 0.f)
                for (int k = 0; k < 4; ++k) s += dot(bg[4 * (size_t)b + k], dx[bidx[4 * b + k]]);
            bbuf[b] = bb2[b] * s;
        }
        for (int t = 0; t < nt; ++t) {
            const V3 df1 = tbuf[2 * (size_t)t], df2 = tbuf[2 * (size_t)t + 1];
            out[F[3 * t]] = out[F[3 * t]] - (df1 + df2);
            out[F[3 * t + 1]] = out[F[3 * t + 1]] + df1;
            out[F[3 * t + 2]] = out[F[3 * t + 2]] + df2;
        }
        for (int h = 0; h < nh; ++h)
            for (int i = 0; i < 4; ++i) out[H[4 * h + i]] = out[H[4 * h + i]] + hbuf[4 * (size_t)h + i];
        for (int b = 0; b < nb; ++b)
            if (bbuf[b] != 0.f)
                for (int k = 0; k < 4; ++k)
                    out[bidx[4 * b + k]] = out[bidx[4 * b + k]] + bbuf[b] * bg[4 * (size_t)b + k];
    }

    std::vector<V3> cg(const std::vector<V3> &g, const std::vector<V3> &dg)
    {
        std::vector<V3> p(np, {0, 0, 0}), r = g, z(np), v(np), Av;
        auto vdot = [&](const std::vector<V3> &a, const std::vector<V3> &b) {
            double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
            for (int i = 0; i < np; ++i) s += (double)dot(a[i], b[i]);
            return s;
        };
        for (int i = 0; i < np; ++i) z[i] = V3{r[i].x / (dg[i].x + 1e-6f), r[i].y / (dg[i].y + 1e-6f), r[i].z / (dg[i].z + 1e-6f)};
        v = z;
        double zr = vdot(z, r);
        for (int it = 0; it < c.n_cg; ++it) {
            hess_dx(q, v, Av);
            const double vAv = vdot(v, Av);
            const double zr_last = zr;
            if (vAv > 1e-16) {
                const float alpha = (float)(zr_last / vAv);
                for (int i = 0; i < np; ++i) {
                    p[i] = p[i] + alpha * v[i];
                    r[i] = r[i] - alpha * Av[i];
                }
            }
            for (int i = 0; i < np; ++i) z[i] = V3{r[i].x / dg[i].x, r[i].y / dg[i].y, r[i].z / dg[i].z};
            zr = vdot(z, r);
            const float beta = (float)(zr / zr_last);
            for (int i = 0; i < np; ++i) v[i] = z[i] + beta * v[i];
        }
        return p;
    }

    float accd(const std::vector<V3> &p) const
    {
        const int nb = (int)bkind.size();
        float step = 1.f;
#pragma omp parallel for reduction(min : step) schedule(dynamic, 64)
        for (int b = 0; b < nb; ++b) {
            V3 x[4], v[4];
            for (int k = 0; k < 4; ++k) {
                x[k] = q[bidx[4 * b + k]];
                v[k] = p[bidx[4 * b + k]];
            }
            const V3 avg = 0.25f * (v[0] + v[1] + v[2] + v[3]);
            for (int k = 0; k < 4; ++k) v[k] = v[k] - avg;
            const float lv = bkind[b] == BLOCK_PT ? norm(v[0]) + std::max(norm(v[1]), std::max(norm(v[2]), norm(v[3])))
                                                  : std::max(norm(v[0]), norm(v[1])) + std::max(norm(v[2]), norm(v[3]));
            if (lv < 1e-12f) continue;
            auto dist = [&](const V3 *X) {
                V3 G[4];
                return pair_distance_grad(X, bkind[b], classify(bkind[b], X, c.ee_thres), G);
            };
            auto dminus = [&](float d) { return std::max((d * d - c.thick * c.thick) / (d + c.thick), 0.f); };
            float dmt = dminus(dist(x));
            const float gap = (1.f - c.slack) * dmt;
            float t = 0.f, tl = c.slack * dmt / lv;
            for (int it = 0;; ++it) {
                for (int k = 0; k < 4; ++k) x[k] = x[k] + tl * v[k];
                dmt = dminus(dist(x));
                if ((it > 0 && dmt <= gap) || it >= c.ccd_max) {
                    step = std::min(step, t);
                    break;
                }
                t += tl;
                if (t > 1.f) break;
                tl = 0.8f * dmt / lv;
            }
        }
        return step;
    }

    void newton()
    {
        const std::vector<V3> q_prev = q;
        detect();
        const std::vector<V3> q_det = q;
        const double e0 = energy(q);
        std::vector<V3> g, dg;
        diff(q, g, dg);
        std::vector<V3> p = cg(g, dg);
        for (int i = 0; i < np; ++i) {  // clamp to the detection radius
            const V3 d = q_prev[i] + p[i] - q_det[i];
            const float l = norm(d);
            if (l > c.radius) p[i] = (c.radius / l) * d + q_det[i] - q_prev[i];
        }
        const float step = accd(p);
        double e = e0;
        for (int nh_ = 0; nh_ < c.n_ls; ++nh_) {
            if (nh_ > 0 && e < e0) break;
            const float a = step * std::ldexp(1.f, -nh_);
            for (int i = 0; i < np; ++i) q[i] = q_prev[i] + a * p[i];
            e = energy(q);
        }
    }
};

}  // namespace

extern "C" {

// One pamo_safe_project.process in the normalised frame: ground truth
// (gt_v [ngv,3], gt_f [ngf,3]), the mesh (v, f), its unique edges [ne,2], hinges
// [nh,4] and Voronoi areas; n_steps steps of the default configuration.
// out_v receives the projected vertices.  Returns the number of contact blocks
// of the last detection.
long long s3c_process(const float *gt_v, int ngv, const int *gt_f, int ngf, const float *v, int nv, const int *f,
                      int nf, const int *e, int ne, const int *h, int nh, const float *vor, int n_steps, float *out_v)
{
    System S;
    S.np = nv;
    S.nt = nf;
    S.ne = ne;
    S.nh = nh;
    S.q.resize(nv);
    for (int i = 0; i < nv; ++i) S.q[i] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
    S.q_rest = S.q;
    S.target = S.q;
    S.gt_v.resize(ngv);
    for (int i = 0; i < ngv; ++i) S.gt_v[i] = {gt_v[3 * i], gt_v[3 * i + 1], gt_v[3 * i + 2]};
    S.gt_f.assign(gt_f, gt_f + 3LL * ngf);
    S.F.assign(f, f + 3LL * nf);
    S.E.assign(e, e + 2LL * ne);
    S.H.assign(h, h + 4LL * nh);
    S.w.resize(nv);
    for (int i = 0; i < nv; ++i) S.w[i] = vor[i] * S.c.gt_k;
    S.mu = S.c.young / (2.f * (1.f + S.c.poisson));
    S.la = S.c.young * S.c.poisson / ((1.f + S.c.poisson) * (1.f - 2.f * S.c.poisson));
    S.radius = S.c.radius;
    S.area.resize(nf);
    S.inv_dm.resize(4LL * nf);
    for (int t = 0; t < nf; ++t) {
        const V3 x01 = S.q[f[3 * t + 1]] - S.q[f[3 * t]], x02 = S.q[f[3 * t + 2]] - S.q[f[3 * t]];
        S.area[t] = 0.5f * norm(cross(x01, x02));
        V3 b1, b2;
        S.frame(x01, x02, b1, b2);
        const float D[4] = {dot(b1, x01), dot(b1, x02), dot(b2, x01), dot(b2, x02)};
        const float det = D[0] * D[3] - D[1] * D[2];
        S.inv_dm[4 * t] = D[3] / det;
        S.inv_dm[4 * t + 1] = -D[1] / det;
        S.inv_dm[4 * t + 2] = -D[2] / det;
        S.inv_dm[4 * t + 3] = D[0] / det;
    }
    S.rest_angle.resize(nh);
    S.rest_elen.resize(nh);
    for (int k = 0; k < nh; ++k) {
        S.rest_angle[k] = System::hinge_angle(S.q[h[4 * k]], S.q[h[4 * k + 1]], S.q[h[4 * k + 2]], S.q[h[4 * k + 3]]);
        S.rest_elen[k] = norm(S.q[h[4 * k + 1]] - S.q[h[4 * k + 2]]);
    }
    std::vector<V3> blo(ngf), bhi(ngf);
    V3 glo{1e30f, 1e30f, 1e30f}, ghi{-1e30f, -1e30f, -1e30f};
    for (int t = 0; t < ngf; ++t) {
        const V3 a = S.gt_v[gt_f[3 * t]], b = S.gt_v[gt_f[3 * t + 1]], c = S.gt_v[gt_f[3 * t + 2]];
        blo[t] = vmin(a, vmin(b, c));
        bhi[t] = vmax(a, vmax(b, c));
        glo = vmin(glo, blo[t]);
        ghi = vmax(ghi, bhi[t]);
    }
    // the ground truth's grid: cells twice the mean triangle extent, at most
    // 2^24 cells
    double mean_ext = 0.0;
    for (int t = 0; t < ngf; ++t) {
        const V3 d = bhi[t] - blo[t];
        mean_ext += std::max(d.x, std::max(d.y, d.z));
    }
    mean_ext /= std::max(ngf, 1);
    const V3 ext = ghi - glo;
    const float vol = std::max(ext.x, 1e-6f) * std::max(ext.y, 1e-6f) * std::max(ext.z, 1e-6f);
    S.gt_grid.build(blo, bhi, std::max((float)(2.0 * mean_ext), std::cbrt(vol / (float)(1 << 24))));
    for (int st = 0; st < n_steps; ++st) {
        S.update_target();
        for (int it = 0; it < S.c.n_newton; ++it) S.newton();
    }
    for (int i = 0; i < nv; ++i) {
        out_v[3 * i] = S.q[i].x;
        out_v[3 * i + 1] = S.q[i].y;
        out_v[3 * i + 2] = S.q[i].z;
    }
    return (long long)S.bkind.size();
}

int s3c_num_threads(void) { return omp_get_max_threads(); }
}
