// Exact-sign geometric predicates on float32 coordinates, for host and device.
//
// Method: J. R. Shewchuk, "Adaptive Precision Floating-Point Arithmetic and
// Fast Robust Geometric Predicates", Discrete & Computational Geometry 18
// (1997).  Each predicate is first evaluated in double with Shewchuk's
// forward error bound; when the result is too close to zero for that bound
// to decide its sign, the determinant is evaluated exactly as a nonoverlapping
// floating-point expansion.  The exact path works on the original
// coordinates: a product of two float32 values is exact in double, so the 2x2
// minors x_i*y_j - x_j*y_i start as exact two-term expansions, and only the
// products with the third coordinate need the error-free product (an FMA
// gives its rounding error exactly, the form of Ogita, Rump and Oishi 2005).
//
// orient3d(a, b, c, d) = sign det[a - d; b - d; c - d]: positive when d lies
// below the plane through a, b, c, seen counterclockwise from above.
// orient2d(a, b, c)    = sign det[a - c; b - c]: positive for a
// counterclockwise turn.
//
// Everything here must be compiled without multiply-add contraction
// (--fmad=false / -ffp-contract=off): the error-free sums rely on each
// operation rounding on its own.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define PAMO_HD __host__ __device__ __forceinline__
#else
#define PAMO_HD inline
#endif

namespace pamo {
namespace exact {

// x + y = a + b exactly, x = fl(a + b) (Knuth's branch-free form)
PAMO_HD void two_sum(double a, double b, double &x, double &y)
{
    x = a + b;
    const double bv = x - a;
    const double av = x - bv;
    y = (a - av) + (b - bv);
}

// x + y = a * b exactly, x = fl(a * b)
PAMO_HD void two_prod(double a, double b, double &x, double &y)
{
    x = a * b;
    y = fma(a, b, -x);
}

// h = e + b for a nonoverlapping expansion e (components in increasing
// magnitude); zero components are dropped.  Returns the length of h (<= n + 1).
PAMO_HD int grow_expansion(const double *e, int n, double b, double *h)
{
    int k = 0;
    double q = b;
    for (int i = 0; i < n; ++i) {
        double s, t;
        two_sum(q, e[i], s, t);
        if (t != 0.0) h[k++] = t;
        q = s;
    }
    if (q != 0.0 || k == 0) h[k++] = q;
    return k;
}

// h = e + f (each nonoverlapping): f's components grown into e one by one.
// h needs room for n + m components; tmp as well.
PAMO_HD int sum_expansion(const double *e, int n, const double *f, int m, double *h, double *tmp)
{
    for (int i = 0; i < n; ++i) h[i] = e[i];
    int len = n;
    for (int j = 0; j < m; ++j) {
        len = grow_expansion(h, len, f[j], tmp);
        for (int i = 0; i < len; ++i) h[i] = tmp[i];
    }
    return len;
}

// h = b * e for a nonoverlapping expansion e; h needs room for 2n components.
PAMO_HD int scale_expansion(const double *e, int n, double b, double *h)
{
    int k = 0;
    double q, lo;
    two_prod(e[0], b, q, lo);
    if (lo != 0.0) h[k++] = lo;
    for (int i = 1; i < n; ++i) {
        double p1, p0, s, t;
        two_prod(e[i], b, p1, p0);
        two_sum(q, p0, s, t);
        if (t != 0.0) h[k++] = t;
        two_sum(p1, s, q, t);
        if (t != 0.0) h[k++] = t;
    }
    if (q != 0.0 || k == 0) h[k++] = q;
    return k;
}

// sign of a nonoverlapping expansion: that of its largest (last nonzero) component
PAMO_HD int expansion_sign(const double *e, int n)
{
    for (int i = n - 1; i >= 0; --i)
        if (e[i] != 0.0) return e[i] > 0.0 ? 1 : -1;
    return 0;
}

// exact x_i*y_j - x_j*y_i of float inputs: both products are exact in double
PAMO_HD int minor2(double xi, double yi, double xj, double yj, double *h)
{
    double s, t;
    two_sum(xi * yj, -(xj * yi), s, t);
    int k = 0;
    if (t != 0.0) h[k++] = t;
    h[k++] = s;
    return k;
}

struct P3 {
    double x, y, z;
};

PAMO_HD int orient2d_exact(double ax, double ay, double bx, double by, double cx, double cy)
{
    double mab[2], mac[2], mbc[2], t4[4], h[6], tmp[6];
    const int na = minor2(ax, ay, bx, by, mab);
    int nc = minor2(ax, ay, cx, cy, mac);
    for (int i = 0; i < nc; ++i) mac[i] = -mac[i];
    const int nb = minor2(bx, by, cx, cy, mbc);
    const int n4 = sum_expansion(mab, na, mac, nc, t4, tmp);
    const int n6 = sum_expansion(t4, n4, mbc, nb, h, tmp);
    return expansion_sign(h, n6);
}

// sign det[a - c; b - c] with the double filter first
PAMO_HD int orient2d(double ax, double ay, double bx, double by, double cx, double cy)
{
    const double l = (ax - cx) * (by - cy);
    const double r = (ay - cy) * (bx - cx);
    const double det = l - r;
    const double bound = (3.0 + 16.0 * 1.1102230246251565e-16) * 1.1102230246251565e-16 * (fabs(l) + fabs(r));
    if (det > bound) return 1;
    if (-det > bound) return -1;
    // a difference of doubles is zero only for equal operands, and products of
    // float32 values do not underflow in double: both terms are then exactly 0
    if (l == 0.0 && r == 0.0) return 0;
    return orient2d_exact(ax, ay, bx, by, cx, cy);
}

// c1 * z for the sum of three minors m1 - m2 + m3 (each <= 2 components)
PAMO_HD int minor_sum_times(const double *m1, int n1, const double *m2, int n2, const double *m3, int n3, double z,
                            double *out /* [12] */)
{
    double neg[2], a4[4], a6[6], tmp[6];
    for (int i = 0; i < n2; ++i) neg[i] = -m2[i];
    const int k4 = sum_expansion(m1, n1, neg, n2, a4, tmp);
    const int k6 = sum_expansion(a4, k4, m3, n3, a6, tmp);
    return scale_expansion(a6, k6, z, out);
}

// exact sign det[a - d; b - d; c - d]
//   = az (m_bc - m_bd + m_cd) - bz (m_ac - m_ad + m_cd)
//   + cz (m_ab - m_ad + m_bd) - dz (m_ab - m_ac + m_bc),   m_ij = x_i y_j - x_j y_i
PAMO_HD int orient3d_exact(P3 a, P3 b, P3 c, P3 d)
{
    double mab[2], mac[2], mad[2], mbc[2], mbd[2], mcd[2];
    const int nab = minor2(a.x, a.y, b.x, b.y, mab), nac = minor2(a.x, a.y, c.x, c.y, mac);
    const int nad = minor2(a.x, a.y, d.x, d.y, mad), nbc = minor2(b.x, b.y, c.x, c.y, mbc);
    const int nbd = minor2(b.x, b.y, d.x, d.y, mbd), ncd = minor2(c.x, c.y, d.x, d.y, mcd);
    double ta[12], tb[12], tc[12], td[12], s24[24], s36[36], s48[48], tmp[48];
    const int ka = minor_sum_times(mbc, nbc, mbd, nbd, mcd, ncd, a.z, ta);
    const int kb = minor_sum_times(mac, nac, mad, nad, mcd, ncd, -b.z, tb);
    const int kc = minor_sum_times(mab, nab, mad, nad, mbd, nbd, c.z, tc);
    const int kd = minor_sum_times(mab, nab, mac, nac, mbc, nbc, -d.z, td);
    const int n24 = sum_expansion(ta, ka, tb, kb, s24, tmp);
    const int n36 = sum_expansion(s24, n24, tc, kc, s36, tmp);
    const int n48 = sum_expansion(s36, n36, td, kd, s48, tmp);
    return expansion_sign(s48, n48);
}

PAMO_HD int orient3d(P3 a, P3 b, P3 c, P3 d)
{
    const double adx = a.x - d.x, bdx = b.x - d.x, cdx = c.x - d.x;
    const double ady = a.y - d.y, bdy = b.y - d.y, cdy = c.y - d.y;
    const double adz = a.z - d.z, bdz = b.z - d.z, cdz = c.z - d.z;
    const double bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
    const double cdxady = cdx * ady, adxcdy = adx * cdy;
    const double adxbdy = adx * bdy, bdxady = bdx * ady;
    const double det = adz * (bdxcdy - cdxbdy) + bdz * (cdxady - adxcdy) + cdz * (adxbdy - bdxady);
    const double perm = (fabs(bdxcdy) + fabs(cdxbdy)) * fabs(adz) + (fabs(cdxady) + fabs(adxcdy)) * fabs(bdz) +
                        (fabs(adxbdy) + fabs(bdxady)) * fabs(cdz);
    const double eps = 1.1102230246251565e-16;  // 2^-53
    const double bound = (7.0 + 56.0 * eps) * eps * perm;
    if (det > bound) return 1;
    if (-det > bound) return -1;
    return orient3d_exact(a, b, c, d);
}

// ---------------------------------------------------------------------------
// Closed-set intersection tests built on the two predicates.

PAMO_HD double coord(P3 p, int k) { return k == 0 ? p.x : (k == 1 ? p.y : p.z); }

// A projection (dropping axis `drop`) in which triangle abc is not degenerate,
// and the sign of its orientation there; drop = -1 when the triangle is
// degenerate (collinear or repeated points) in every projection, which means
// in 3-D.  (The orientation in the plane dropping axis k is the k-th component
// of the normal, so some projection keeps a non-degenerate triangle.)
PAMO_HD int tri_projection(P3 a, P3 b, P3 c, int &orient)
{
    for (int k = 2; k >= 0; --k) {
        const int u = (k + 1) % 3, v = (k + 2) % 3;
        const int o = orient2d(coord(a, u), coord(a, v), coord(b, u), coord(b, v), coord(c, u), coord(c, v));
        if (o != 0) {
            orient = o;
            return k;
        }
    }
    orient = 0;
    return -1;
}

struct P2 {
    double x, y;
};

PAMO_HD P2 proj(P3 p, int drop)
{
    const int u = (drop + 1) % 3, v = (drop + 2) % 3;
    return {coord(p, u), coord(p, v)};
}

PAMO_HD int o2(P2 a, P2 b, P2 c) { return orient2d(a.x, a.y, b.x, b.y, c.x, c.y); }

// p on the closed segment ab, given that the three points are collinear
PAMO_HD bool on_segment_collinear(P2 a, P2 b, P2 p)
{
    return fmin(a.x, b.x) <= p.x && p.x <= fmax(a.x, b.x) && fmin(a.y, b.y) <= p.y && p.y <= fmax(a.y, b.y);
}

// closed segments pq and ab in the plane share a point
PAMO_HD bool seg_seg_2d(P2 p, P2 q, P2 a, P2 b)
{
    const int o1 = o2(p, q, a), o2_ = o2(p, q, b), o3 = o2(a, b, p), o4 = o2(a, b, q);
    if (o1 * o2_ < 0 && o3 * o4 < 0) return true;
    if (o1 == 0 && on_segment_collinear(p, q, a)) return true;
    if (o2_ == 0 && on_segment_collinear(p, q, b)) return true;
    if (o3 == 0 && on_segment_collinear(a, b, p)) return true;
    if (o4 == 0 && on_segment_collinear(a, b, q)) return true;
    return false;
}

// p in the closed triangle abc of orientation `orient` (non-zero)
PAMO_HD bool point_in_tri_2d(P2 p, P2 a, P2 b, P2 c, int orient)
{
    return o2(a, b, p) * orient >= 0 && o2(b, c, p) * orient >= 0 && o2(c, a, p) * orient >= 0;
}

// closed segment pq and closed triangle abc, all in one plane; the triangle is
// non-degenerate in projection `drop` with orientation `orient`
PAMO_HD bool seg_tri_coplanar(P3 p3, P3 q3, P3 a3, P3 b3, P3 c3, int drop, int orient)
{
    const P2 p = proj(p3, drop), q = proj(q3, drop), a = proj(a3, drop), b = proj(b3, drop), c = proj(c3, drop);
    if (point_in_tri_2d(p, a, b, c, orient) || point_in_tri_2d(q, a, b, c, orient)) return true;
    return seg_seg_2d(p, q, a, b) || seg_seg_2d(p, q, b, c) || seg_seg_2d(p, q, c, a);
}

// closed segment pq and closed non-degenerate triangle abc in 3-D
PAMO_HD bool seg_tri(P3 p, P3 q, P3 a, P3 b, P3 c)
{
    const int sp = orient3d(a, b, c, p), sq = orient3d(a, b, c, q);
    if (sp * sq > 0) return false;
    if (sp == 0 && sq == 0) {
        int orient;
        const int drop = tri_projection(a, b, c, orient);
        return drop >= 0 && seg_tri_coplanar(p, q, a, b, c, drop, orient);
    }
    // the segment meets the plane in one point; it is in the closed triangle
    // iff the line pq passes each edge on the same side (or through it)
    const int s1 = orient3d(p, q, a, b), s2 = orient3d(p, q, b, c), s3 = orient3d(p, q, c, a);
    return (s1 >= 0 && s2 >= 0 && s3 >= 0) || (s1 <= 0 && s2 <= 0 && s3 <= 0);
}

// closed non-degenerate triangles share a point
PAMO_HD bool tri_tri(const P3 *A, const P3 *B)
{
    int sa[3], sb[3];
    for (int i = 0; i < 3; ++i) sb[i] = orient3d(A[0], A[1], A[2], B[i]);
    if ((sb[0] > 0 && sb[1] > 0 && sb[2] > 0) || (sb[0] < 0 && sb[1] < 0 && sb[2] < 0)) return false;
    for (int i = 0; i < 3; ++i) sa[i] = orient3d(B[0], B[1], B[2], A[i]);
    if ((sa[0] > 0 && sa[1] > 0 && sa[2] > 0) || (sa[0] < 0 && sa[1] < 0 && sa[2] < 0)) return false;
    if (sb[0] == 0 && sb[1] == 0 && sb[2] == 0) {  // coplanar
        int orient;
        const int drop = tri_projection(A[0], A[1], A[2], orient);
        if (drop < 0) return false;
        const P2 a0 = proj(A[0], drop), a1 = proj(A[1], drop), a2 = proj(A[2], drop);
        const P2 b0 = proj(B[0], drop), b1 = proj(B[1], drop), b2 = proj(B[2], drop);
        const int orient_b = o2(b0, b1, b2);  // non-zero: B is non-degenerate and in A's plane
        if (orient_b == 0) return false;
        if (point_in_tri_2d(b0, a0, a1, a2, orient) || point_in_tri_2d(a0, b0, b1, b2, orient_b)) return true;
        const P2 ea[3][2] = {{a0, a1}, {a1, a2}, {a2, a0}}, eb[3][2] = {{b0, b1}, {b1, b2}, {b2, b0}};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                if (seg_seg_2d(ea[i][0], ea[i][1], eb[j][0], eb[j][1])) return true;
        return false;
    }
    // Not coplanar: the intersection, if any, is a segment (or point) on the
    // planes' common line whose ends lie on edges of A or B, so some edge of
    // one triangle meets the other triangle.
    for (int i = 0; i < 3; ++i) {
        if (seg_tri(A[i], A[(i + 1) % 3], B[0], B[1], B[2])) return true;
        if (seg_tri(B[i], B[(i + 1) % 3], A[0], A[1], A[2])) return true;
    }
    return false;
}

// Two faces of one mesh intersect beyond what they share by index:
//   no shared vertex   - the closed triangles share any point;
//   one shared vertex v - they share a point other than v, i.e. the edge of
//     either opposite v meets the other triangle (A n B is convex and holds v,
//     so any other common point q gives the segment vq in both; its far end is
//     on such an edge, or on an edge through v lying along the other
//     triangle, whose far end then lies in the other triangle);
//   a shared edge      - the triangles are coplanar and fold onto each other
//     (third vertices on the same side of the edge);
//   three shared       - the same face twice.
// ia / ib are the vertex indices; both triangles must be non-degenerate.
PAMO_HD bool faces_intersect(const P3 *A, const int *ia, const P3 *B, const int *ib)
{
    int shared = 0, sa[3] = {-1, -1, -1};  // sa[i]: B's corner equal to A's corner i
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (ia[i] == ib[j]) {
                sa[i] = j;
                ++shared;
            }
    if (shared >= 3) return true;
    if (shared == 0) return tri_tri(A, B);
    if (shared == 1) {
        int i = 0;
        while (sa[i] < 0) ++i;
        const int j = sa[i];
        return seg_tri(A[(i + 1) % 3], A[(i + 2) % 3], B[0], B[1], B[2]) ||
               seg_tri(B[(j + 1) % 3], B[(j + 2) % 3], A[0], A[1], A[2]);
    }
    // shared edge (u, w); a and b the third vertices
    int i3 = 0;
    while (sa[i3] >= 0) ++i3;
    int j3 = 0;
    while (j3 == sa[(i3 + 1) % 3] || j3 == sa[(i3 + 2) % 3]) ++j3;
    const P3 u = A[(i3 + 1) % 3], w = A[(i3 + 2) % 3], a = A[i3], b = B[j3];
    if (orient3d(u, w, a, b) != 0) return false;
    int orient;
    const int drop = tri_projection(u, w, a, orient);
    if (drop < 0) return false;
    const int ob = o2(proj(u, drop), proj(w, drop), proj(b, drop));
    return ob == orient;
}

// a triangle is degenerate when it repeats an index or its points are collinear
PAMO_HD bool tri_degenerate(const P3 *T, const int *idx)
{
    if (idx[0] == idx[1] || idx[1] == idx[2] || idx[0] == idx[2]) return true;
    int o;
    return tri_projection(T[0], T[1], T[2], o) < 0;
}

}  // namespace exact
}  // namespace pamo
