// Host build of the library's exact predicates (pamo_b200/csrc/exact.cuh) for
// the CPU tests, which compare them with rational arithmetic.  Compiled by the
// test itself with -ffp-contract=off.
#include "../../pamo_b200/csrc/exact.cuh"

using pamo::exact::P3;

static P3 at(const float *p, long long i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }

extern "C" {

// out[i] = orient3d(q[4i], q[4i+1], q[4i+2], q[4i+3]) for n quadruples of points
void h_orient3d(const float *q, long long n, int *out)
{
    for (long long i = 0; i < n; ++i) out[i] = pamo::exact::orient3d(at(q, 4 * i), at(q, 4 * i + 1), at(q, 4 * i + 2), at(q, 4 * i + 3));
}

// out[i] = orient2d of points (x, y) pairs t[6i..6i+5]
void h_orient2d(const float *t, long long n, int *out)
{
    for (long long i = 0; i < n; ++i)
        out[i] = pamo::exact::orient2d(t[6 * i], t[6 * i + 1], t[6 * i + 2], t[6 * i + 3], t[6 * i + 4], t[6 * i + 5]);
}

// out[i] = faces_intersect(f[i], g[i]) for faces of one mesh (V [n,3], F [m,3]);
// -1 when either face is degenerate
void h_faces_intersect(const float *V, const int *F, const int *pairs, long long n, int *out)
{
    for (long long i = 0; i < n; ++i) {
        const int f = pairs[2 * i], g = pairs[2 * i + 1];
        P3 A[3], B[3];
        int ia[3], ib[3];
        for (int k = 0; k < 3; ++k) {
            ia[k] = F[3 * f + k];
            ib[k] = F[3 * g + k];
            A[k] = at(V, ia[k]);
            B[k] = at(V, ib[k]);
        }
        if (pamo::exact::tri_degenerate(A, ia) || pamo::exact::tri_degenerate(B, ib)) out[i] = -1;
        else out[i] = pamo::exact::faces_intersect(A, ia, B, ib) ? 1 : 0;
    }
}
}
