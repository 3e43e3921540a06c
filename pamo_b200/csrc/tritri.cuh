// Triangle-pair intersection decision used by the stage-2 undo check.
//
// Decision parity with the reference requires its exact arithmetic: the
// candidate pair is translated by the floored mean of its six vertices
// (simp_cuda/src/bvh/self_intersect.cuh:124-149), tested for coplanarity with an
// fp64 plane and a 1e-6 * max|coord| band (bvh/tri_tri_3d.cuh:100-129), skipped
// when it shares an edge by index or by coordinates within 1e-6
// (self_intersect.cuh:39-48,338-343), and otherwise intersected with the
// plane-interval method: fp64 planes, fp32 signed distances, interval overlap on
// the plane-plane line (tri_tri_3d.cuh:131-276).  A hit whose intersection
// segment is shorter than eps in the L-infinity norm is ignored when the pair
// shares exactly one vertex.  The file is compiled with --fmad=false.
#pragma once

#include "common.cuh"

namespace pamo {

struct Tri9 {
    float v[3][3];
};

__device__ __forceinline__ double tt_ddot(const double *a, const float *b)
{
    return a[0] * (double)b[0] + a[1] * (double)b[1] + a[2] * (double)b[2];
}

__device__ __forceinline__ void tt_plane(const float t[3][3], double pl[4])
{
    double ba[3], bc[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        ba[c] = (double)t[0][c] - (double)t[1][c];
        bc[c] = (double)t[2][c] - (double)t[1][c];
    }
    pl[0] = ba[1] * bc[2] - ba[2] * bc[1];
    pl[1] = ba[2] * bc[0] - ba[0] * bc[2];
    pl[2] = ba[0] * bc[1] - ba[1] * bc[0];
    pl[3] = -tt_ddot(pl, t[1]);
}

__device__ __forceinline__ bool tt_coplanar(const float a[3][3], const float b[3][3])
{
    float sc = 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) sc = fmaxf(sc, fabsf(a[i][j]));
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) sc = fmaxf(sc, fabsf(b[i][j]));
    double pl[4];
    tt_plane(a, pl);
    double eps = (double)sc * 1e-6;
#pragma unroll
    for (int j = 0; j < 3; ++j)
        if (!(fabs(tt_ddot(pl, b[j]) + pl[3]) <= eps)) return false;
    return true;
}

__device__ __forceinline__ bool tt_same_side(const float s[3])
{
    return (s[0] != 0.0f && s[1] != 0.0f && s[2] != 0.0f) && ((s[0] < 0.0f) == (s[1] < 0.0f)) &&
           ((s[0] < 0.0f) == (s[2] < 0.0f));
}

// Returns true and the two ends of the intersection segment when the triangles
// overlap on the plane-plane line.
__device__ __noinline__ bool tt_intersect(const float ta[3][3], const float tb[3][3], float r1[3], float r2[3])
{
    float side[2][3];
    double pa[4], pb[4];
    tt_plane(ta, pa);
#pragma unroll
    for (int j = 0; j < 3; ++j) side[1][j] = (float)(tt_ddot(pa, tb[j]) + pa[3]);
    if (side[1][0] == 0.0f && side[1][1] == 0.0f && side[1][2] == 0.0f) return false;
    if (tt_same_side(side[1])) return false;
    tt_plane(tb, pb);
#pragma unroll
    for (int j = 0; j < 3; ++j) side[0][j] = (float)(tt_ddot(pb, ta[j]) + pb[3]);
    if (tt_same_side(side[0])) return false;

    double dir[3];
    dir[0] = pa[1] * pb[2] - pa[2] * pb[1];
    dir[1] = pa[2] * pb[0] - pa[0] * pb[2];
    dir[2] = pa[0] * pb[1] - pa[1] * pb[0];

    float rmin[2], rmax[2], loc[2][2][3];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const float(*t)[3] = i == 0 ? ta : tb;
        const float *s = side[i];
        int o0, o1, o2;
        if ((s[0] != 0.0f && s[1] != 0.0f) && ((s[0] < 0.0f) == (s[1] < 0.0f))) {
            o0 = 1; o1 = 2; o2 = 0;
        } else if ((s[1] != 0.0f && s[2] != 0.0f) && ((s[1] < 0.0f) == (s[2] < 0.0f))) {
            o0 = 2; o1 = 0; o2 = 1;
        } else if (s[1] == 0.0f && ((s[2] < 0.0f) != (s[0] < 0.0f))) {
            o0 = 1; o1 = 2; o2 = 0;
        } else {
            o0 = 0; o1 = 1; o2 = 2;
        }
        double db = tt_ddot(dir, t[o1]);
        float sc = s[o1];
        if (sc != 0.0f) {
            double da = tt_ddot(dir, t[o0]);
            double dc = tt_ddot(dir, t[o2]);
            float f0 = sc / (sc - s[o0]);
            float f1 = sc / (sc - s[o2]);
            double off0 = (double)f0 * (da - db);
            double off1 = (double)f1 * (dc - db);
            if (off0 > off1) {
                double td = off0; off0 = off1; off1 = td;
                float tf = f0; f0 = f1; f1 = tf;
                int ti = o0; o0 = o2; o2 = ti;
            }
            rmin[i] = (float)(db + off0);
            rmax[i] = (float)(db + off1);
            float s0 = 1.0f - f0, s1 = 1.0f - f1;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                loc[i][0][c] = s0 * t[o1][c] + f0 * t[o0][c];
                loc[i][1][c] = s1 * t[o1][c] + f1 * t[o2][c];
            }
        } else {
            rmin[i] = rmax[i] = (float)db;
#pragma unroll
            for (int c = 0; c < 3; ++c) loc[i][0][c] = loc[i][1][c] = t[o1][c];
        }
    }
    if ((rmax[0] > rmin[1]) && (rmin[0] < rmax[1])) {
        int ia, ja, ib, jb;  // (range, end) of the two reported points
        if (rmin[0] >= rmin[1]) {
            ia = 0; ja = 0;
            if (rmax[0] <= rmax[1]) { ib = 0; jb = 1; }
            else { ib = 1; jb = 1; }
        } else {
            if (rmax[0] <= rmax[1]) { ia = 0; ja = 1; ib = 1; jb = 0; }
            else { ia = 1; ja = 0; ib = 1; jb = 1; }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            r1[c] = loc[ia][ja][c];
            r2[c] = loc[ib][jb][c];
        }
        return true;
    }
    return false;
}

__device__ __forceinline__ bool tt_near(const float *a, const float *b)
{
    const float eps = 1e-6f;
    return fabsf(a[0] - b[0]) < eps && fabsf(a[1] - b[1]) < eps && fabsf(a[2] - b[2]) < eps;
}

// One directed test: `cur` is the BVH object, `qry` the querying face.
__device__ __noinline__ bool pair_flag_directed(const float cur[3][3], const int ci[3], const float qry[3][3],
                                                const int qi[3], float eps)
{
    float ta[3][3], tb[3][3];
    float m[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float s = cur[0][c] + cur[1][c] + cur[2][c] + qry[0][c] + qry[1][c] + qry[2][c];
        m[c] = (float)(int)floorf(s / 6.0f);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            ta[a][c] = cur[a][c] - m[c];
            tb[a][c] = qry[a][c] - m[c];
        }
    int shared = 0;
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int k = 0; k < 3; ++k) shared += ci[j] == qi[k];
    if (tt_coplanar(ta, tb)) return false;
    if (shared == 2) return false;
    int near = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) near += tt_near(ta[a], tb[0]) || tt_near(ta[a], tb[1]) || tt_near(ta[a], tb[2]);
    if (near >= 2) return false;
    float r1[3], r2[3];
    if (!tt_intersect(ta, tb, r1, r2)) return false;
    float dx = fabsf(r2[0] - r1[0]), dy = fabsf(r2[1] - r1[1]), dz = fabsf(r2[2] - r1[2]);
    float d = -INFINITY;
    if (dx > d) d = dx;
    if (dy > d) d = dy;
    if (dz > d) d = dz;
    if (d < eps && shared == 1) return false;
    return true;
}

}  // namespace pamo
