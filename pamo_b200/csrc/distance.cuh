// Point-triangle / edge-edge distance classification, distances and distance
// gradients for the stage-3 contact energy (FP32), plus FP64 variants for the
// CCD step search.
//
// Classification follows the reference's decision logic
// (simp_cuda/safe_project/src/pamo_safe_project/kernels/distance_kernels/
// distance_kernels.py:76-228 point-triangle, :326-442 edge-edge): the projected
// point's barycentric signs choose among point-triangle, point-edge and
// point-point; for edges the closest-point parameters (with a parallel-edge
// guard on the sine of the angle) choose edge-edge, else the best of the eight
// point-edge / point-point candidates.  The distance of each type is the
// unsquared Euclidean distance of the reference (pt_distance, pe_distance,
// pp_distance, ee_distance).  Its gradient is written with the closest-point
// weights: for a distance d = |sum_i w_i x_i| minimised over unconstrained
// weights of the type's affine hull, dd/dx_i = w_i * n (envelope theorem), with n
// the unit vector between the closest points.
#pragma once

#include <cuda_runtime.h>

namespace pamo {
namespace s3 {

enum BlockKind { KIND_PT = 3, KIND_EE = 4 };
enum PtType { PT_PT = 0, PT_PP01, PT_PP02, PT_PE012, PT_PP03, PT_PE031, PT_PE023 };
enum EeType { EE_PP02 = 0, EE_PP03, EE_PP12, EE_PP13, EE_PE023, EE_PE123, EE_PE201, EE_PE301, EE_EE };

template <typename T>
struct Vec3 {
    T x, y, z;
};

template <typename T>
__device__ __forceinline__ Vec3<T> mk(T x, T y, T z) { return {x, y, z}; }
template <typename T>
__device__ __forceinline__ Vec3<T> operator+(Vec3<T> a, Vec3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T>
__device__ __forceinline__ Vec3<T> operator-(Vec3<T> a, Vec3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T>
__device__ __forceinline__ Vec3<T> operator*(T s, Vec3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <typename T>
__device__ __forceinline__ T dot(Vec3<T> a, Vec3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T>
__device__ __forceinline__ Vec3<T> cross(Vec3<T> a, Vec3<T> b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename T>
__device__ __forceinline__ T len(Vec3<T> a) { return sqrt(dot(a, a)); }
template <typename T>
__device__ __forceinline__ Vec3<T> normalized(Vec3<T> a)
{
    T l = len(a);
    return l > T(0) ? (T(1) / l) * a : a;
}

using F3 = Vec3<float>;
using D3 = Vec3<double>;

__device__ __forceinline__ F3 f3(float4 p) { return {p.x, p.y, p.z}; }
__device__ __forceinline__ D3 d3(float4 p) { return {(double)p.x, (double)p.y, (double)p.z}; }

template <typename T>
__device__ __forceinline__ T pp_dist(Vec3<T> a, Vec3<T> b) { return len(b - a); }
template <typename T>
__device__ __forceinline__ T pe_dist(Vec3<T> p, Vec3<T> a, Vec3<T> b) { return len(cross(a - p, b - p)) / len(a - b); }
template <typename T>
__device__ __forceinline__ T pt_dist(Vec3<T> p, Vec3<T> a, Vec3<T> b, Vec3<T> c)
{
    Vec3<T> n = normalized(cross(b - a, c - a));
    T s = dot(p - a, n);
    return s < T(0) ? -s : s;
}
template <typename T>
__device__ __forceinline__ T ee_dist(Vec3<T> a0, Vec3<T> a1, Vec3<T> b0, Vec3<T> b1)
{
    Vec3<T> n = normalized(cross(a1 - a0, b1 - b0));
    T s = dot(a0 - b0, n);
    return s < T(0) ? -s : s;
}

template <typename T>
__device__ int pt_classify(Vec3<T> x0, Vec3<T> x1, Vec3<T> x2, Vec3<T> x3)
{
    Vec3<T> x10 = x0 - x1, x12 = x2 - x1, x13 = x3 - x1;
    T area_sq = dot(cross(x12, x13), cross(x12, x13));
    if (area_sq <= T(1e-6) * (dot(x12, x12) * dot(x13, x13)) || area_sq <= T(1e-16)) {
        T d1 = len(x10), d2 = len(x0 - x2), d3 = len(x0 - x3);
        if (d1 < d2) return d1 < d3 ? PT_PP01 : PT_PP03;
        return d2 < d3 ? PT_PP02 : PT_PP03;
    }
    Vec3<T> n = normalized(cross(x12, x13));
    Vec3<T> proj = x0 - dot(n, x10) * n;
    Vec3<T> p10 = proj - x1, p20 = proj - x2, p30 = proj - x3;
    T a00 = dot(x12, x12), a01 = dot(x12, x13), a11 = dot(x13, x13);
    T b0 = dot(p10, x12), b1 = dot(p10, x13);
    T det = a00 * a11 - a01 * a01;
    T beta = b0 * a11 - b1 * a01;
    T gamma = a00 * b1 - b0 * a01;
    T alpha = det - beta - gamma;
    int neg = (alpha < T(0)) + (beta < T(0)) + (gamma < T(0));
    if (neg == 0) return PT_PT;
    if (neg == 1) {
        if (alpha < T(0)) {
            Vec3<T> x23 = x3 - x2, x20 = x0 - x2;
            T dr = dot(x23, x20);
            if (dr < T(0)) return PT_PP02;
            if (dr > dot(x23, x23)) return PT_PP03;
            return PT_PE023;
        }
        if (beta < T(0)) {
            Vec3<T> x31 = x1 - x3, x30 = x0 - x3;
            T dr = dot(x31, x30);
            if (dr < T(0)) return PT_PP03;
            if (dr > dot(x31, x31)) return PT_PP01;
            return PT_PE031;
        }
        T dr = dot(x12, p10);
        if (dr < T(0)) return PT_PP01;
        if (dr > dot(x12, x12)) return PT_PP02;
        return PT_PE012;
    }
    if (alpha >= T(0)) {
        T d12 = dot(x12, p10), d13 = dot(x13, p10);
        if (d12 > T(0) && d13 <= T(0)) return dot(x12, p20) > T(0) ? PT_PP02 : PT_PE012;
        if (d13 > T(0) && d12 <= T(0)) return dot(x13, p30) > T(0) ? PT_PP03 : PT_PE031;
        return PT_PP01;
    }
    if (beta >= T(0)) {
        Vec3<T> x23 = x3 - x2, x21 = x1 - x2;
        T d23 = dot(x23, p20), d21 = dot(x21, p20);
        if (d23 > T(0) && d21 <= T(0)) return dot(x23, p30) > T(0) ? PT_PP03 : PT_PE023;
        if (d21 > T(0) && d23 <= T(0)) return dot(x21, p10) > T(0) ? PT_PP01 : PT_PE012;
        return PT_PP02;
    }
    Vec3<T> x31 = x1 - x3, x32 = x2 - x3;
    T d31 = dot(x31, p30), d32 = dot(x32, p30);
    if (d31 > T(0) && d32 <= T(0)) return dot(x31, p10) > T(0) ? PT_PP01 : PT_PE031;
    if (d32 > T(0) && d31 <= T(0)) return dot(x32, p20) > T(0) ? PT_PP02 : PT_PE023;
    return PT_PP03;
}

template <typename T>
__device__ int ee_classify(Vec3<T> x0, Vec3<T> x1, Vec3<T> x2, Vec3<T> x3, T sin_thres)
{
    Vec3<T> e0 = x0 - x1, e1 = x2 - x3;
    T e0_sq = dot(e0, e0), e1_sq = dot(e1, e1);
    T a00 = e0_sq, a01 = -dot(e0, e1), a10 = dot(e0, e1), a11 = -e1_sq;
    T b0 = dot(x3 - x1, e0), b1 = dot(x3 - x1, e1);
    T mu0 = -(b0 * a11 - b1 * a01);
    T mu1 = -(a00 * b1 - a10 * b0);
    T det = -(a00 * a11 - a01 * a10);
    T s = len(cross(normalized(e0), normalized(e1)));
    if (mu0 >= T(0) && mu0 <= det && mu1 >= T(0) && mu1 <= det && s >= sin_thres && e0_sq > T(1e-15) &&
        e1_sq > T(1e-15))
        return EE_EE;
    T best = T(1e9);
    int type = -1;
    auto consider = [&](T d, int t) {
        if (d < best) {
            best = d;
            type = t;
        }
    };
    T t0 = dot(x0 - x3, e1);
    if (t0 >= e1_sq) consider(pp_dist(x0, x2), EE_PP02);
    else if (t0 <= T(0)) consider(pp_dist(x0, x3), EE_PP03);
    else consider(pe_dist(x0, x2, x3), EE_PE023);
    T t1 = dot(x1 - x3, e1);
    if (t1 >= e1_sq) consider(pp_dist(x1, x2), EE_PP12);
    else if (t1 <= T(0)) consider(pp_dist(x1, x3), EE_PP13);
    else consider(pe_dist(x1, x2, x3), EE_PE123);
    T t2 = dot(x2 - x1, e0);
    if (t2 >= e0_sq) consider(pp_dist(x2, x0), EE_PP02);
    else if (t2 <= T(0)) consider(pp_dist(x2, x1), EE_PP12);
    else consider(pe_dist(x2, x0, x1), EE_PE201);
    T t3 = dot(x3 - x1, e0);
    if (t3 >= e0_sq) consider(pp_dist(x3, x0), EE_PP03);
    else if (t3 <= T(0)) consider(pp_dist(x3, x1), EE_PP13);
    else consider(pe_dist(x3, x0, x1), EE_PE301);
    return type;
}

// local vertex roles of each classified type: kind of distance + indices
struct TypeInfo {
    int kind;  // 0 pp, 1 pe, 2 pt, 3 ee
    int i0, i1, i2, i3;
};

__device__ __forceinline__ TypeInfo type_info(int block_kind, int t)
{
    if (block_kind == KIND_PT) {
        switch (t) {
        case PT_PT: return {2, 0, 1, 2, 3};
        case PT_PP01: return {0, 0, 1, 0, 0};
        case PT_PP02: return {0, 0, 2, 0, 0};
        case PT_PE012: return {1, 0, 1, 2, 0};
        case PT_PP03: return {0, 0, 3, 0, 0};
        case PT_PE031: return {1, 0, 3, 1, 0};
        default: return {1, 0, 2, 3, 0};  // PT_PE023
        }
    }
    switch (t) {
    case EE_PP02: return {0, 0, 2, 0, 0};
    case EE_PP03: return {0, 0, 3, 0, 0};
    case EE_PP12: return {0, 1, 2, 0, 0};
    case EE_PP13: return {0, 1, 3, 0, 0};
    case EE_PE023: return {1, 0, 2, 3, 0};
    case EE_PE123: return {1, 1, 2, 3, 0};
    case EE_PE201: return {1, 2, 0, 1, 0};
    case EE_PE301: return {1, 3, 0, 1, 0};
    default: return {3, 0, 1, 2, 3};  // EE_EE
    }
}

template <typename T>
__device__ __forceinline__ int classify(int block_kind, const Vec3<T> *x, T ee_thres)
{
    return block_kind == KIND_PT ? pt_classify(x[0], x[1], x[2], x[3]) : ee_classify(x[0], x[1], x[2], x[3], ee_thres);
}

template <typename T>
__device__ __forceinline__ T classified_distance(int block_kind, int t, const Vec3<T> *x)
{
    if (t < 0) return T(1e9);
    TypeInfo ti = type_info(block_kind, t);
    switch (ti.kind) {
    case 0: return pp_dist(x[ti.i0], x[ti.i1]);
    case 1: return pe_dist(x[ti.i0], x[ti.i1], x[ti.i2]);
    case 2: return pt_dist(x[0], x[1], x[2], x[3]);
    default: return ee_dist(x[0], x[1], x[2], x[3]);
    }
}

// distance and its gradient w.r.t. the four block vertices
__device__ inline float distance_grad(int block_kind, int t, const F3 *x, F3 *g)
{
    for (int i = 0; i < 4; ++i) g[i] = mk(0.f, 0.f, 0.f);
    if (t < 0) return 1e9f;
    TypeInfo ti = type_info(block_kind, t);
    if (ti.kind == 0) {
        F3 d = x[ti.i0] - x[ti.i1];
        float l = len(d);
        F3 u = (1.0f / l) * d;
        g[ti.i0] = u;
        g[ti.i1] = mk(-u.x, -u.y, -u.z);
        return l;
    }
    if (ti.kind == 1) {
        F3 p = x[ti.i0], a = x[ti.i1], b = x[ti.i2];
        F3 e = b - a;
        float t_ = dot(p - a, e) / dot(e, e);
        F3 c = a + t_ * e;
        F3 u = normalized(p - c);
        g[ti.i0] = u;
        g[ti.i1] = (-(1.0f - t_)) * u;
        g[ti.i2] = (-t_) * u;
        return pe_dist(p, a, b);
    }
    if (ti.kind == 2) {
        F3 n = normalized(cross(x[2] - x[1], x[3] - x[1]));
        float sd = dot(x[0] - x[1], n);
        F3 u = (sd < 0.f ? -1.f : 1.f) * n;
        F3 proj = x[0] - sd * n;
        F3 e1 = x[2] - x[1], e2 = x[3] - x[1], w = proj - x[1];
        float a00 = dot(e1, e1), a01 = dot(e1, e2), a11 = dot(e2, e2);
        float b0 = dot(w, e1), b1 = dot(w, e2);
        float det = a00 * a11 - a01 * a01;
        float be = (b0 * a11 - b1 * a01) / det;
        float ga = (a00 * b1 - b0 * a01) / det;
        float al = 1.0f - be - ga;
        g[0] = u;
        g[1] = (-al) * u;
        g[2] = (-be) * u;
        g[3] = (-ga) * u;
        return sd < 0.f ? -sd : sd;
    }
    F3 n = normalized(cross(x[1] - x[0], x[3] - x[2]));
    float sd = dot(x[0] - x[2], n);
    F3 u = (sd < 0.f ? -1.f : 1.f) * n;
    F3 e0 = x[1] - x[0], e1 = x[3] - x[2], w0 = x[0] - x[2];
    float a = dot(e0, e0), b = dot(e0, e1), c = dot(e1, e1);
    float dq = dot(e0, w0), eq = dot(e1, w0);
    float den = a * c - b * b;
    float s_ = (b * eq - c * dq) / den;
    float t_ = (a * eq - b * dq) / den;
    g[0] = (1.0f - s_) * u;
    g[1] = s_ * u;
    g[2] = (-(1.0f - t_)) * u;
    g[3] = (-t_) * u;
    return sd < 0.f ? -sd : sd;
}

}  // namespace s3
}  // namespace pamo
