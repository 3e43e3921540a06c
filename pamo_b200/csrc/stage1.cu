// Stage 1 of PaMO.run: remeshing (simp_cuda/pamo/__init__.py:60-120,130-142).
//
// The reference normalises the triangles into the unit cube, asks
// torchcumesh2sdf for a narrow-band signed distance field on an R^3 grid,
// shifts it by -0.9/R, extracts quads with pdmc's dual marching cubes and
// splits each quad into the triangle pair with the larger smallest angle.  Both
// libraries are absent, so this file restates their published steps; the CPU
// oracle/s1_oracle.py defines the same semantics and the results agree bit
// for bit (tests/test_stage1_gpu.py):
//
//   1. normalise: ((p - tris_mean) - tris_min) / tris_max + band) / margin in
//      float32, as preprocess_mesh does with numpy (:60-72);
//   2. unsigned distance (double) from every grid sample ((i + 0.5) / R, ...)
//      within `band` of a triangle to the nearest triangle, else `band`: one
//      warp per triangle walks the samples of its box grown by `band` and
//      lowers the sample's squared distance with a 64-bit atomic minimum (the
//      bits of a non-negative double order like the value);
//   3. sign by flood fill: samples farther than half a voxel from every
//      triangle are free, free samples 6-connected to the grid boundary are
//      outside; tiles of 8^3 samples propagate "outside" in shared memory
//      until they settle, and launches repeat until no sample changes
//      (bounded); the field is +-distance - 0.9/R;
//   4. dual marching cubes: a sample is inside where the field is negative.
//      Per cell, the crossed edges pair up on each cube face (an ambiguous face
//      cuts off each outside corner, a rule both cells sharing the face agree
//      on), the pairings split them into cycles, and each cycle (patch) gets
//      one vertex at the mean of its edges' crossing points.  Every crossed
//      grid edge gives one quad through its four cells' patch vertices, wound
//      with the normal towards the outside.  Vertices are numbered by cell and
//      patch, quads by axis and lower sample, through prefix scans;
//   5. each quad is split into (0,1,3),(1,2,3) or (0,1,2),(0,2,3), whichever
//      has the smaller largest corner cosine (double), first-kind quads first
//      (:95-118); vertices are mapped back to the centred frame in double and
//      rounded to float32.
//
// The output is in the frame centred on tris_mean, as the reference's remesh
// returns it; stage 2 then runs without centring again and adds tris_mean
// back at the end (:130-189).
#include <cstring>
#include <vector>

#include "scan.cuh"
#include "stage1.cuh"

namespace pamo {
namespace s1 {
namespace {

// cube corners c = x + 2 y + 4 z; edges 0-3 along x, 4-7 along y, 8-11 along z
constexpr int kEdgeCorners[12][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3},
                                     {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
// the faces as corner cycles
constexpr int kFaceCorners[6][4] = {{0, 2, 6, 4}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 3, 7, 6}, {0, 1, 3, 2}, {4, 5, 7, 6}};

__constant__ signed char c_patch[256][12];  // patch of each edge per sign case, -1: not crossed
__constant__ unsigned char c_npatch[256];

int edge_of(int a, int b)
{
    for (int i = 0; i < 12; ++i)
        if ((kEdgeCorners[i][0] == a && kEdgeCorners[i][1] == b) || (kEdgeCorners[i][0] == b && kEdgeCorners[i][1] == a))
            return i;
    return -1;
}

// The patch table: for each sign case (bit c set: corner c inside), the crossed
// edges linked by their pairings on the cube faces, split into cycles.
void build_patch_table(signed char (*patch)[12], unsigned char *npatch)
{
    for (int cs = 0; cs < 256; ++cs) {
        bool inside[8], crossed[12];
        for (int c = 0; c < 8; ++c) inside[c] = (cs >> c) & 1;
        for (int e = 0; e < 12; ++e) crossed[e] = inside[kEdgeCorners[e][0]] != inside[kEdgeCorners[e][1]];
        int link[12][2], nl[12] = {0};
        auto join = [&](int a, int b) {
            link[a][nl[a]++] = b;
            link[b][nl[b]++] = a;
        };
        for (int f = 0; f < 6; ++f) {
            int es[4], cr[4], n = 0;
            for (int k = 0; k < 4; ++k) {
                es[k] = edge_of(kFaceCorners[f][k], kFaceCorners[f][(k + 1) % 4]);
                if (crossed[es[k]]) cr[n++] = es[k];
            }
            if (n == 2) {
                join(cr[0], cr[1]);
            } else if (n == 4) {  // cut off each outside corner
                for (int k = 0; k < 4; ++k)
                    if (!inside[kFaceCorners[f][k]]) join(es[(k + 3) % 4], es[k]);
            }
        }
        int pid[12];
        for (int e = 0; e < 12; ++e) pid[e] = -1;
        int np = 0;
        for (int e = 0; e < 12; ++e) {
            if (!crossed[e] || pid[e] >= 0) continue;
            int stack[12], sp = 0;
            stack[sp++] = e;
            pid[e] = np;
            while (sp) {
                const int x = stack[--sp];
                for (int k = 0; k < nl[x]; ++k) {
                    const int y = link[x][k];
                    if (pid[y] < 0) {
                        pid[y] = np;
                        stack[sp++] = y;
                    }
                }
            }
            ++np;
        }
        for (int e = 0; e < 12; ++e) patch[cs][e] = (signed char)pid[e];
        npatch[cs] = (unsigned char)np;
    }
}

__device__ __forceinline__ long long gidx(int x, int y, int z, int R) { return ((long long)z * R + y) * R + x; }

// the corners of cube edge e (the order of kEdgeCorners)
__device__ __forceinline__ void edge_corners(int e, int &a, int &b)
{
    if (e < 4) {
        a = 2 * e;
        b = a + 1;
    } else if (e < 8) {
        const int k = e - 4;
        a = (k & 1) | ((k >> 1) << 2);
        b = a + 2;
    } else {
        a = e - 8;
        b = a + 4;
    }
}

// -------------------------------------------------------------- 1. normalise
// per-axis minimum of the centred corners (ordered ints), then the largest
// coordinate after subtracting it
__global__ void k_s1_min(const float *pts, const int *tris, int m, const float *mean, int *dev)
{
    float lo[3] = {INFINITY, INFINITY, INFINITY};
    PAMO_GRID_STRIDE(f, m)
    {
        for (int c = 0; c < 3; ++c) {
            const int v = tris[3 * f + c];
            for (int k = 0; k < 3; ++k) lo[k] = fminf(lo[k], pts[3 * v + k] - mean[k]);
        }
    }
    for (int k = 0; k < 3; ++k) {
        float x = lo[k];
        for (int o = 16; o > 0; o >>= 1) x = fminf(x, __shfl_down_sync(0xffffffffu, x, o));
        if ((threadIdx.x & 31) == 0) atomicMin(&dev[k], float_to_ordered(x));
    }
}

__global__ void k_s1_max(const float *pts, const int *tris, int m, const float *mean, int *dev)
{
    float lo[3];
    for (int k = 0; k < 3; ++k) lo[k] = ordered_to_float(dev[k]);
    float hi = -INFINITY;
    PAMO_GRID_STRIDE(f, m)
    {
        for (int c = 0; c < 3; ++c) {
            const int v = tris[3 * f + c];
            for (int k = 0; k < 3; ++k) hi = fmaxf(hi, (pts[3 * v + k] - mean[k]) - lo[k]);
        }
    }
    for (int o = 16; o > 0; o >>= 1) hi = fmaxf(hi, __shfl_down_sync(0xffffffffu, hi, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&dev[3], float_to_ordered(hi));
}

__global__ void k_s1_normalise(const float *pts, const int *tris, int m, const float *mean, const int *dev,
                               float band, float margin, float *out)
{
    float lo[3];
    for (int k = 0; k < 3; ++k) lo[k] = ordered_to_float(dev[k]);
    const float mx = ordered_to_float(dev[3]);
    PAMO_GRID_STRIDE(f, m)
    {
        for (int c = 0; c < 3; ++c) {
            const int v = tris[3 * f + c];
            for (int k = 0; k < 3; ++k) out[9 * f + 3 * c + k] = (((pts[3 * v + k] - mean[k]) - lo[k]) / mx + band) / margin;
        }
    }
}

// ------------------------------------------------------- 2. unsigned distance
struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 dsub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// squared distance from p to triangle abc; the closest point by the Voronoi
// regions of the triangle (Ericson, Real-Time Collision Detection, 5.1.5), with
// the operation order of oracle/s1_oracle.py _point_tri_d2
__device__ double point_tri_d2(D3 p, D3 a, D3 b, D3 c)
{
    const D3 ab = dsub(b, a), ac = dsub(c, a), ap = dsub(p, a);
    const double d1 = ddot(ab, ap), d2 = ddot(ac, ap);
    const D3 bp = dsub(p, b);
    const double d3 = ddot(ab, bp), d4 = ddot(ac, bp);
    const D3 cp = dsub(p, c);
    const double d5 = ddot(ab, cp), d6 = ddot(ac, cp);
    const double vc = d1 * d4 - d3 * d2;
    const double vb = d5 * d2 - d1 * d6;
    const double va = d3 * d6 - d5 * d4;
    D3 q;
    if (d1 <= 0 && d2 <= 0) {
        q = a;
    } else if (d3 >= 0 && d4 <= d3) {
        q = b;
    } else if (vc <= 0 && d1 >= 0 && d3 <= 0) {
        const double v = d1 / (d1 - d3);
        q = {a.x + v * ab.x, a.y + v * ab.y, a.z + v * ab.z};
    } else if (d6 >= 0 && d5 <= d6) {
        q = c;
    } else if (vb <= 0 && d2 >= 0 && d6 <= 0) {
        const double w = d2 / (d2 - d6);
        q = {a.x + w * ac.x, a.y + w * ac.y, a.z + w * ac.z};
    } else if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        const D3 cb = dsub(c, b);
        q = {b.x + w * cb.x, b.y + w * cb.y, b.z + w * cb.z};
    } else {
        const double den = 1.0 / (va + vb + vc);
        const double v = vb * den, w = vc * den;
        q = {a.x + v * ab.x + w * ac.x, a.y + v * ab.y + w * ac.y, a.z + v * ab.z + w * ac.z};
    }
    const D3 d = dsub(p, q);
    return ddot(d, d);
}

// One warp per triangle over the samples of its box grown by `band`.  Before
// the full closest-point computation a sample is skipped when a lower bound of
// its distance to the triangle -- the distance to the triangle's bounding box,
// and to its plane -- already reaches the sample's current value (the bounds
// hold in exact arithmetic; the 1e-9 relative margin covers their rounding), so
// the minimum, and therefore the field, is the same as without the test.
// (i + 0.5) / R, the coordinate of sample i; for R a power of two (inv_r > 0)
// the product with 1 / R is that same number and spares the FP64 division
__device__ __forceinline__ double s1_coord(int i, int R, double inv_r)
{
    return inv_r > 0.0 ? (i + 0.5) * inv_r : (i + 0.5) / R;
}

__global__ void __launch_bounds__(256, 3) k_s1_udist(const float *tris, int m, int R, double inv_r, double band,
                                                  unsigned long long *field)
{
    const int lane = threadIdx.x & 31;
    const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const double band2 = band * band;
    for (long long t = warp0; t < m; t += nw) {
        const float *T = tris + 9 * t;
        const D3 a = {T[0], T[1], T[2]}, b = {T[3], T[4], T[5]}, c = {T[6], T[7], T[8]};
        int lo[3], n[3];
        const double mn[3] = {fmin(a.x, fmin(b.x, c.x)), fmin(a.y, fmin(b.y, c.y)), fmin(a.z, fmin(b.z, c.z))};
        const double mx[3] = {fmax(a.x, fmax(b.x, c.x)), fmax(a.y, fmax(b.y, c.y)), fmax(a.z, fmax(b.z, c.z))};
        for (int k = 0; k < 3; ++k) {
            // samples (i + 0.5) / R within [mn - band, mx + band]
            int l = (int)floor((mn[k] - band) * R - 0.5), h = (int)ceil((mx[k] + band) * R - 0.5);
            l = max(l, 0);
            h = min(h, R - 1);
            lo[k] = l;
            n[k] = h >= l ? h - l + 1 : 0;
        }
        // the plane's normal (unnormalised) and 1 / |n|^2
        const D3 ab = dsub(b, a), ac = dsub(c, a);
        const D3 nrm = {ab.y * ac.z - ab.z * ac.y, ab.z * ac.x - ab.x * ac.z, ab.x * ac.y - ab.y * ac.x};
        const double nn = ddot(nrm, nrm);
        const double inv_nn = nn > 0.0 ? 1.0 / nn : 0.0;  // degenerate: no plane bound
        const int nxy = n[0] * n[1];
        const int total = nxy * n[2];
        // the lane's sample (ox, oy, oz) in the box, stepped by 32 without divisions
        int ox = 0, oy = 0, oz = 0;
        if (total > 0) {
            ox = lane % n[0];
            oy = (lane / n[0]) % n[1];
            oz = lane / nxy;
        }
        const int qx = total > 0 ? 32 / n[0] : 0, rx = total > 0 ? 32 % n[0] : 0;
        for (int s = lane; s < total; s += 32) {
            const int ix = lo[0] + ox, iy = lo[1] + oy, iz = lo[2] + oz;
            ox += rx;
            oy += qx;
            if (ox >= n[0]) {
                ox -= n[0];
                ++oy;
            }
            while (oy >= n[1]) {
                oy -= n[1];
                ++oz;
            }
            const D3 p = {s1_coord(ix, R, inv_r), s1_coord(iy, R, inv_r), s1_coord(iz, R, inv_r)};
            const double bx = fmax(fmax(mn[0] - p.x, 0.0), p.x - mx[0]);
            const double by = fmax(fmax(mn[1] - p.y, 0.0), p.y - mx[1]);
            const double bz = fmax(fmax(mn[2] - p.z, 0.0), p.z - mx[2]);
            const double box2 = bx * bx + by * by + bz * bz;
            if (box2 >= band2 * (1.0 + 1e-9)) continue;  // the value stays band^2 or lower
            unsigned long long *dst = field + gidx(ix, iy, iz, R);
            const double cur = __longlong_as_double((long long)*dst);
            if (box2 > cur * (1.0 + 1e-9)) continue;
            const double hp = ddot(nrm, dsub(p, a));
            if (hp * hp * inv_nn > cur * (1.0 + 1e-9)) continue;
            const double d2 = point_tri_d2(p, a, b, c);
            const unsigned long long bits = (unsigned long long)__double_as_longlong(d2);
            if (bits < *dst) atomicMin(dst, bits);
        }
    }
}

__global__ void k_s1_fill(unsigned long long *a, long long n, unsigned long long v)
{
    PAMO_GRID_STRIDE(i, n) a[i] = v;
}

// squared distance -> unsigned distance (double), free / near / boundary state
__global__ void k_s1_state(unsigned long long *field, long long n3, int R, double band, uint8_t *state)
{
    PAMO_GRID_STRIDE(i, n3)
    {
        const double ud = sqrt(__longlong_as_double((long long)field[i]));
        field[i] = (unsigned long long)__double_as_longlong(ud);
        const bool free_ = ud > 0.5 / R;
        const int x = (int)(i % R), y = (int)((i / R) % R), z = (int)(i / ((long long)R * R));
        const bool border = x == 0 || y == 0 || z == 0 || x == R - 1 || y == R - 1 || z == R - 1;
        state[i] = free_ ? (border ? 2 : 1) : 0;
    }
}

// ----------------------------------------------------------- 3. flood fill
constexpr int kTile = 8;
constexpr int kHalo = kTile + 2;

// One block per 8^3 tile (one thread per sample): free samples next to an
// outside sample become outside, repeated in shared memory until the tile
// settles (at most 3 * 8^3 sweeps); a change is reported in dev[4].  Only
// tiles marked in `dirty_in` (changed, or next to a tile that changed, in the
// previous launch; all tiles in the first) do the work; a tile that changes
// marks itself and its six neighbours in `dirty_out`.
__global__ void __launch_bounds__(kTile * kTile * kTile) k_s1_flood(uint8_t *state, int R, int *dev,
                                                                   const uint8_t *dirty_in, uint8_t *dirty_out)
{
    __shared__ uint8_t s[kHalo][kHalo][kHalo];
    __shared__ int changed, any_change;
    const int tpr = (R + kTile - 1) / kTile;
    if (!dirty_in[blockIdx.x]) return;
    const int bx = blockIdx.x % tpr, by = (blockIdx.x / tpr) % tpr, bz = blockIdx.x / (tpr * tpr);
    const int tx = threadIdx.x % kTile, ty = (threadIdx.x / kTile) % kTile, tz = threadIdx.x / (kTile * kTile);
    // the tile with its one-sample halo (outside the grid: near, never spreads)
    for (int i = threadIdx.x; i < kHalo * kHalo * kHalo; i += blockDim.x) {
        const int hx = i % kHalo, hy = (i / kHalo) % kHalo, hz = i / (kHalo * kHalo);
        const int gx = bx * kTile + hx - 1, gy = by * kTile + hy - 1, gz = bz * kTile + hz - 1;
        uint8_t v = 0;
        if (gx >= 0 && gy >= 0 && gz >= 0 && gx < R && gy < R && gz < R) v = state[gidx(gx, gy, gz, R)];
        s[hz][hy][hx] = v;
    }
    if (threadIdx.x == 0) any_change = 0;
    const int gx = bx * kTile + tx, gy = by * kTile + ty, gz = bz * kTile + tz;
    const bool in_grid = gx < R && gy < R && gz < R;
    const int x = tx + 1, y = ty + 1, z = tz + 1;
    bool any = false;
    __syncthreads();
    for (int sweep = 0; sweep < 3 * kTile * kTile * kTile; ++sweep) {
        if (threadIdx.x == 0) changed = 0;
        __syncthreads();
        if (in_grid && s[z][y][x] == 1 &&
            (s[z][y][x - 1] == 2 || s[z][y][x + 1] == 2 || s[z][y - 1][x] == 2 || s[z][y + 1][x] == 2 ||
             s[z - 1][y][x] == 2 || s[z + 1][y][x] == 2)) {
            s[z][y][x] = 2;
            changed = 1;
            any = true;
        }
        __syncthreads();
        if (!changed) break;
    }
    if (any) {
        state[gidx(gx, gy, gz, R)] = 2;
        any_change = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0 && any_change) {
        atomicExch(&dev[4], 1);
        dirty_out[blockIdx.x] = 1;
        if (bx > 0) dirty_out[blockIdx.x - 1] = 1;
        if (bx + 1 < tpr) dirty_out[blockIdx.x + 1] = 1;
        if (by > 0) dirty_out[blockIdx.x - tpr] = 1;
        if (by + 1 < tpr) dirty_out[blockIdx.x + tpr] = 1;
        if (bz > 0) dirty_out[blockIdx.x - tpr * tpr] = 1;
        if (bz + 1 < tpr) dirty_out[blockIdx.x + tpr * tpr] = 1;
    }
}

__global__ void k_s1_field(unsigned long long *field, const uint8_t *state, long long n3, int R)
{
    PAMO_GRID_STRIDE(i, n3)
    {
        const double ud = __longlong_as_double((long long)field[i]);
        const double v = (state[i] == 2 ? ud : -ud) - 0.9 / R;
        field[i] = (unsigned long long)__double_as_longlong(v);
    }
}

// ------------------------------------------------------- 4. dual marching cubes
__device__ __forceinline__ double fval(const unsigned long long *field, int x, int y, int z, int R)
{
    return __longlong_as_double((long long)field[gidx(x, y, z, R)]);
}

__device__ __forceinline__ int cell_case(const unsigned long long *field, int x, int y, int z, int R)
{
    int cs = 0;
    for (int c = 0; c < 8; ++c) cs |= (fval(field, x + (c & 1), y + ((c >> 1) & 1), z + ((c >> 2) & 1), R) < 0.0) << c;
    return cs;
}

__global__ void k_s1_cells(const unsigned long long *field, int R, int *cell_cnt)
{
    const int C = R - 1;
    PAMO_GRID_STRIDE(i, (long long)C * C * C)
    {
        const int x = (int)(i % C), y = (int)((i / C) % C), z = (int)(i / ((long long)C * C));
        cell_cnt[i] = c_npatch[cell_case(field, x, y, z, R)];
    }
}

// the patch vertices of each cell: the mean of its edges' crossing points (edge
// order), in sample-index coordinates, mapped to the centred frame
__global__ void k_s1_verts(const unsigned long long *field, int R, const int *cell_first, double band, double margin,
                           double tmax, const int *dev, float *verts)
{
    const int C = R - 1;
    double lo[3];
    for (int k = 0; k < 3; ++k) lo[k] = (double)ordered_to_float(dev[k]);
    PAMO_GRID_STRIDE(i, (long long)C * C * C)
    {
        const int first = cell_first[i], np = cell_first[i + 1] - first;
        if (np == 0) continue;
        const int x = (int)(i % C), y = (int)((i / C) % C), z = (int)(i / ((long long)C * C));
        const int cs = cell_case(field, x, y, z, R);
        double sx[4] = {0, 0, 0, 0}, sy[4] = {0, 0, 0, 0}, sz[4] = {0, 0, 0, 0};
        int cnt[4] = {0, 0, 0, 0};
        for (int e = 0; e < 12; ++e) {
            const int p = c_patch[cs][e];
            if (p < 0) continue;
            int a, b;
            edge_corners(e, a, b);
            const int ax = x + (a & 1), ay = y + ((a >> 1) & 1), az = z + ((a >> 2) & 1);
            const int bx = x + (b & 1), by = y + ((b >> 1) & 1), bz = z + ((b >> 2) & 1);
            const double da = fval(field, ax, ay, az, R), db = fval(field, bx, by, bz, R);
            const double t = da / (da - db);
            sx[p] += ax + t * (double)(bx - ax);
            sy[p] += ay + t * (double)(by - ay);
            sz[p] += az + t * (double)(bz - az);
            cnt[p]++;
        }
        for (int p = 0; p < np; ++p) {
            const double v[3] = {sx[p] / cnt[p], sy[p] / cnt[p], sz[p] / cnt[p]};
            for (int k = 0; k < 3; ++k) {
                const double xn = (v[k] + 0.5) / R;
                verts[3LL * (first + p) + k] = (float)((xn * margin - band) * tmax + lo[k]);
            }
        }
    }
}

// crossed grid edges whose four cells exist (every crossed edge, given the
// grid's outer layer is outside): 1 per axis-major edge slot
__global__ void k_s1_edges(const unsigned long long *field, int R, int *edge_cnt)
{
    const long long n3 = (long long)R * R * R;
    PAMO_GRID_STRIDE(i, 3 * n3)
    {
        const int ax = (int)(i / n3);
        const long long g = i % n3;
        const int x = (int)(g % R), y = (int)((g / R) % R), z = (int)(g / ((long long)R * R));
        int c = 0;
        const int x2 = x + (ax == 0), y2 = y + (ax == 1), z2 = z + (ax == 2);
        // the four cells need the two other coordinates in [1, R - 2]
        const bool room = x2 < R && y2 < R && z2 < R && (ax == 0 || (x >= 1 && x <= R - 2)) &&
                          (ax == 1 || (y >= 1 && y <= R - 2)) && (ax == 2 || (z >= 1 && z <= R - 2));
        if (room) c = (fval(field, x, y, z, R) < 0.0) != (fval(field, x2, y2, z2, R) < 0.0);
        edge_cnt[i] = c;
    }
}

__device__ __forceinline__ double max_cos(const float *v, int i0, int i1, int i2)
{
    const D3 a = {v[3 * i0], v[3 * i0 + 1], v[3 * i0 + 2]};
    const D3 b = {v[3 * i1], v[3 * i1 + 1], v[3 * i1 + 2]};
    const D3 c = {v[3 * i2], v[3 * i2 + 1], v[3 * i2 + 2]};
    auto cosang = [](D3 p, D3 r, D3 s) {
        D3 u = dsub(r, p), w = dsub(s, p);
        const double nu = fmax(sqrt(u.x * u.x + u.y * u.y + u.z * u.z), 1e-12);
        const double nw = fmax(sqrt(w.x * w.x + w.y * w.y + w.z * w.z), 1e-12);
        u = {u.x / nu, u.y / nu, u.z / nu};
        w = {w.x / nw, w.y / nw, w.z / nw};
        return u.x * w.x + u.y * w.y + u.z * w.z;
    };
    return fmax(fmax(cosang(a, b, c), cosang(b, c, a)), cosang(c, a, b));
}

// one quad per crossed edge, through the patch vertices of its four cells
// (counterclockwise seen from the +axis side when the lower sample is inside),
// and whether it splits the first way
__global__ void k_s1_quads(const unsigned long long *field, int R, const int *edge_first, const int *cell_first,
                           const float *verts, int4 *quads, int *q_first)
{
    const long long n3 = (long long)R * R * R;
    const int C = R - 1;
    PAMO_GRID_STRIDE(i, 3 * n3)
    {
        const int q = edge_first[i];
        if (edge_first[i + 1] == q) continue;
        const int ax = (int)(i / n3);
        const long long g = i % n3;
        const int x = (int)(g % R), y = (int)((g / R) % R), z = (int)(g / ((long long)R * R));
        // the other two axes in cyclic order (b, c) with b x c = the edge's axis
        const int bax = (ax + 1) % 3, cax = (ax + 2) % 3;
        const int ob[4] = {0, -1, -1, 0}, oc[4] = {0, 0, -1, -1};
        int vs[4];
        for (int k = 0; k < 4; ++k) {
            int cc[3] = {x, y, z};
            cc[bax] += ob[k];
            cc[cax] += oc[k];
            // the edge's corners inside this cell
            const int l[3] = {x - cc[0], y - cc[1], z - cc[2]};
            const int ca = l[0] + 2 * l[1] + 4 * l[2];
            const int e = ax * 4 + (ax == 0 ? (ca >> 1) : (ax == 1 ? ((ca & 1) | ((ca >> 1) & 2)) : (ca & 3)));
            const long long cell = ((long long)cc[2] * C + cc[1]) * C + cc[0];
            const int cs = cell_case(field, cc[0], cc[1], cc[2], R);
            vs[k] = cell_first[cell] + c_patch[cs][e];
        }
        const bool lower_inside = fval(field, x, y, z, R) < 0.0;
        const int4 qd = lower_inside ? make_int4(vs[0], vs[1], vs[2], vs[3]) : make_int4(vs[3], vs[2], vs[1], vs[0]);
        quads[q] = qd;
        const double a1 = fmax(max_cos(verts, qd.x, qd.y, qd.w), max_cos(verts, qd.y, qd.z, qd.w));
        const double a2 = fmax(max_cos(verts, qd.x, qd.y, qd.z), max_cos(verts, qd.x, qd.z, qd.w));
        q_first[q] = a1 < a2 ? 1 : 0;
    }
}

__global__ void k_s1_faces(const int4 *quads, const int *flag, const int *pos, int nq, int n1, int *faces)
{
    PAMO_GRID_STRIDE(q, nq)
    {
        const int4 d = quads[q];
        int *f;
        int t[6];
        if (flag[q]) {
            f = faces + 6LL * pos[q];
            t[0] = d.x; t[1] = d.y; t[2] = d.w; t[3] = d.y; t[4] = d.z; t[5] = d.w;
        } else {
            f = faces + 6LL * (n1 + (q - pos[q]));
            t[0] = d.x; t[1] = d.y; t[2] = d.z; t[3] = d.x; t[4] = d.z; t[5] = d.w;
        }
        for (int k = 0; k < 6; ++k) f[k] = t[k];
    }
}

__global__ void k_s1_dev_init(int *dev)
{
    if (threadIdx.x < 3) dev[threadIdx.x] = 0x7FFFFFFF;  // min (ordered)
    else if (threadIdx.x == 3) dev[3] = (int)0x80000000;
    else if (threadIdx.x < 16) dev[threadIdx.x] = 0;
}

// k_s1_quads numbers a cell's edge from its lower corner: along x by (y, z),
// along y by (x, z), along z by (x, y) -- the order of kEdgeCorners
static_assert(kEdgeCorners[5][0] == 1 && kEdgeCorners[5][1] == 3 && kEdgeCorners[6][0] == 4, "edge numbering");

}  // namespace

#define S1_TRY(expr)                                      \
    do {                                                  \
        cudaError_t _e = (expr);                          \
        if (_e != cudaSuccess) return map_cuda_error(_e); \
    } while (0)

void Stage1::release()
{
    void *p[] = {tris, field, state, cell_cnt, edge_cnt, scan_cells, scan_edges, scan_quads, quads, q_first, verts,
                 faces, dev, mean_dev, tile_dirty};
    for (void *x : p)
        if (x) cudaFree(x);
    if (h_dev) cudaFreeHost(h_dev);
    tris = nullptr;
    field = nullptr;
    state = nullptr;
    cell_cnt = edge_cnt = scan_cells = scan_edges = scan_quads = nullptr;
    quads = nullptr;
    q_first = nullptr;
    verts = nullptr;
    faces = nullptr;
    dev = h_dev = nullptr;
    mean_dev = nullptr;
    tile_dirty = nullptr;
    cap_tris = cap_grid = cap_cells = cap_edges = cap_verts = cap_quads = cap_tiles = 0;
}

int Stage1::ensure(long long m, int R_)
{
    const long long n3 = (long long)R_ * R_ * R_, c3 = (long long)(R_ - 1) * (R_ - 1) * (R_ - 1);
    const long long tpr = (R_ + kTile - 1) / kTile, nt = tpr * tpr * tpr;
    if (m <= cap_tris && n3 <= cap_grid && nt <= cap_tiles && dev) return PAMO_OK;
    const long long ctl = nt > cap_tiles ? nt : cap_tiles;
    const long long cm = m > cap_tris ? m : cap_tris, cg = n3 > cap_grid ? n3 : cap_grid;
    const long long cc = c3 > cap_cells ? c3 : cap_cells;
    void *keep_v = verts, *keep_f = faces, *keep_q = quads, *keep_qf = q_first, *keep_sq = scan_quads;
    const long long kv = cap_verts, kq = cap_quads;
    verts = nullptr;
    faces = nullptr;
    quads = nullptr;
    q_first = nullptr;
    scan_quads = nullptr;
    release();
    verts = (float *)keep_v;
    faces = (int *)keep_f;
    quads = (int4 *)keep_q;
    q_first = (int *)keep_qf;
    scan_quads = (int *)keep_sq;
    cap_verts = kv;
    cap_quads = kq;
#define S1A(ptr, bytes)                                                    \
    if (cudaMalloc((void **)&ptr, (size_t)(bytes)) != cudaSuccess) {       \
        release();                                                         \
        return PAMO_ERR_OOM;                                               \
    }
    S1A(tris, 9 * 4 * (cm + 1));
    S1A(field, 8 * cg);
    S1A(state, cg);
    S1A(tile_dirty, 2 * ctl);
    S1A(cell_cnt, 4 * (cc + 1));
    S1A(edge_cnt, 4 * (3 * cg + 1));
    S1A(scan_cells, 4 * scan_scratch_ints(cc + 1));
    S1A(scan_edges, 4 * scan_scratch_ints(3 * cg + 1));
    S1A(dev, 64);
    S1A(mean_dev, 16);
#undef S1A
    if (cudaMallocHost((void **)&h_dev, 64) != cudaSuccess) {
        release();
        return PAMO_ERR_OOM;
    }
    if (scan_scratch_init(scan_cells, scan_scratch_ints(cc + 1)) != cudaSuccess ||
        scan_scratch_init(scan_edges, scan_scratch_ints(3 * cg + 1)) != cudaSuccess) {
        release();
        return PAMO_ERR_OOM;
    }
    cap_tris = cm;
    cap_grid = cg;
    cap_tiles = ctl;
    cap_cells = cc;
    cap_edges = 3 * cg;
    return PAMO_OK;
}

int Stage1::ensure_out(long long nv, long long nq)
{
    if (nv > cap_verts || !verts) {
        if (verts) cudaFree(verts);
        verts = nullptr;
        cap_verts = 0;
        const long long c = nv + nv / 8 + 64;
        if (cudaMalloc((void **)&verts, (size_t)c * 12) != cudaSuccess) return PAMO_ERR_OOM;
        cap_verts = c;
    }
    if (nq > cap_quads || !quads) {
        void *p[] = {quads, q_first, faces, scan_quads};
        for (void *x : p)
            if (x) cudaFree(x);
        quads = nullptr;
        q_first = nullptr;
        faces = nullptr;
        scan_quads = nullptr;
        cap_quads = 0;
        const long long c = nq + nq / 8 + 64;
        if (cudaMalloc((void **)&quads, (size_t)c * 16) != cudaSuccess ||
            cudaMalloc((void **)&q_first, (size_t)(c + 1) * 4) != cudaSuccess ||
            cudaMalloc((void **)&faces, (size_t)c * 24) != cudaSuccess ||
            cudaMalloc((void **)&scan_quads, (size_t)scan_scratch_ints(c + 1) * 4) != cudaSuccess)
            return PAMO_ERR_OOM;
        if (scan_scratch_init(scan_quads, scan_scratch_ints(c + 1)) != cudaSuccess) return PAMO_ERR_OOM;
        cap_quads = c;
    }
    return PAMO_OK;
}

int remesh(Stage1 &S, const float *d_points, const int *d_tris, int n_pts, int m, const float *mean_dev, int R,
           cudaStream_t s)
{
    (void)n_pts;
    if (R < 4 || R > 1024 || m <= 0) return PAMO_ERR_INVALID_ARG;
    int rc = S.ensure(m, R);
    if (rc) return rc;
    S.R = R;
    static signed char h_patch[256][12];
    static unsigned char h_npatch[256];
    static bool have_table = false;
    if (!have_table) {  // the same table for every device; built once per process
        build_patch_table(h_patch, h_npatch);
        have_table = true;
    }
    S1_TRY(cudaMemcpyToSymbolAsync(c_patch, h_patch, sizeof(h_patch), 0, cudaMemcpyHostToDevice, s));
    S1_TRY(cudaMemcpyToSymbolAsync(c_npatch, h_npatch, sizeof(h_npatch), 0, cudaMemcpyHostToDevice, s));
    const double band = 3.0 / R, margin = band * 2 + 1;
    const long long n3 = (long long)R * R * R, c3 = (long long)(R - 1) * (R - 1) * (R - 1);
    // 1. normalise
    if (S.prof) S.prof->begin(PH_S1_PREP, s);
    launch(k_s1_dev_init, 1, 32, 0, s, S.dev);
    launch(k_s1_min, grid_for(m), kThreads, 0, s, d_points, d_tris, m, mean_dev, S.dev);
    launch(k_s1_max, grid_for(m), kThreads, 0, s, d_points, d_tris, m, mean_dev, S.dev);
    launch(k_s1_normalise, grid_for(m), kThreads, 0, s, d_points, d_tris, m, mean_dev, (const int *)S.dev,
           (float)band, (float)margin, S.tris);
    // 2. unsigned distance: squared distances start at band^2 (bits of a double)
    if (S.prof) S.prof->begin(PH_S1_DIST, s);
    {
        const double b2 = band * band;
        unsigned long long bits;
        memcpy(&bits, &b2, 8);
        // fill by a kernel: cudaMemset only sets bytes
        launch(k_s1_fill, grid_for(n3), kThreads, 0, s, S.field, n3, bits);
    }
    const double inv_r = (R & (R - 1)) == 0 ? 1.0 / R : 0.0;
    launch(k_s1_udist, grid_for(32LL * m), 256, 0, s, (const float *)S.tris, m, R, inv_r, band, S.field);
    launch(k_s1_state, grid_for(n3), kThreads, 0, s, S.field, n3, R, band, S.state);
    // 3. flood fill from the boundary, until nothing changes
    if (S.prof) S.prof->begin(PH_S1_FLOOD, s);
    const int tpr = (R + kTile - 1) / kTile;
    const int tiles = tpr * tpr * tpr;
    // two dirty-tile flag sets used in turn: every tile is dirty at first
    uint8_t *dirty[2] = {S.tile_dirty, S.tile_dirty + tiles};
    S1_TRY(cudaMemsetAsync(dirty[0], 1, (size_t)tiles, s));
    S1_TRY(cudaMemsetAsync(dirty[1], 0, (size_t)tiles, s));
    int cur = 0;
    bool settled = false;
    for (int round = 0; round < 4 * R + 64 && !settled; round += 8) {
        S1_TRY(cudaMemsetAsync(S.dev + 4, 0, 4, s));
        for (int k = 0; k < 8; ++k) {
            launch(k_s1_flood, tiles, kTile * kTile * kTile, 0, s, S.state, R, S.dev, (const uint8_t *)dirty[cur],
                   dirty[cur ^ 1]);
            S1_TRY(cudaMemsetAsync(dirty[cur], 0, (size_t)tiles, s));
            cur ^= 1;
        }
        S1_TRY(cudaMemcpyAsync(S.h_dev, S.dev, 64, cudaMemcpyDeviceToHost, s));
        S1_TRY(cudaStreamSynchronize(s));
        if (S.prof) S.prof->collect();
        settled = S.h_dev[4] == 0;
    }
    if (!settled) return PAMO_ERR_DEVICE;  // cannot happen within 4 R sweeps of tiles
    launch(k_s1_field, grid_for(n3), kThreads, 0, s, S.field, (const uint8_t *)S.state, n3, R);
    // 4. dual marching cubes: patch vertices
    if (S.prof) S.prof->begin(PH_S1_DMC, s);
    launch(k_s1_cells, grid_for(c3), kThreads, 0, s, (const unsigned long long *)S.field, R, S.cell_cnt);
    S1_TRY(cudaMemsetAsync(S.cell_cnt + c3, 0, 4, s));
    S1_TRY(exclusive_scan(S.cell_cnt, S.cell_cnt, c3 + 1, nullptr, S.scan_cells, nullptr, s, S.dev + 6));
    launch(k_s1_edges, grid_for(3 * n3), kThreads, 0, s, (const unsigned long long *)S.field, R, S.edge_cnt);
    S1_TRY(cudaMemsetAsync(S.edge_cnt + 3 * n3, 0, 4, s));
    S1_TRY(exclusive_scan(S.edge_cnt, S.edge_cnt, 3 * n3 + 1, nullptr, S.scan_edges, nullptr, s, S.dev + 6));
    S1_TRY(cudaMemcpyAsync(S.h_dev + 8, S.cell_cnt + c3, 4, cudaMemcpyDeviceToHost, s));
    S1_TRY(cudaMemcpyAsync(S.h_dev + 9, S.edge_cnt + 3 * n3, 4, cudaMemcpyDeviceToHost, s));
    S1_TRY(cudaMemcpyAsync(S.h_dev + 6, S.dev + 6, 4, cudaMemcpyDeviceToHost, s));
    S1_TRY(cudaStreamSynchronize(s));
    if (S.h_dev[6]) return PAMO_ERR_DEVICE;  // a scan's wait ran out
    const long long nv = S.h_dev[8], nq = S.h_dev[9];
    if (nv <= 0 || nq <= 0 || 2 * nq > 0x7FFFFFFF) return nv <= 0 || nq <= 0 ? PAMO_ERR_INVALID_ARG : PAMO_ERR_CAPACITY;
    if ((rc = S.ensure_out(nv, nq))) return rc;
    float tmax = 0.f;
    {
        // the largest coordinate, an ordered int of a non-negative float: its bits
        const int mx_bits = S.h_dev[3];
        if (mx_bits >= 0) memcpy(&tmax, &mx_bits, 4);
    }
    launch(k_s1_verts, grid_for(c3), kThreads, 0, s, (const unsigned long long *)S.field, R, (const int *)S.cell_cnt,
           band, margin, (double)tmax, (const int *)S.dev, S.verts);
    // quads and their split
    launch(k_s1_quads, grid_for(3 * n3), kThreads, 0, s, (const unsigned long long *)S.field, R,
           (const int *)S.edge_cnt, (const int *)S.cell_cnt, (const float *)S.verts, S.quads, S.q_first);
    S1_TRY(cudaMemsetAsync(S.q_first + nq, 0, 4, s));
    int *qpos = S.edge_cnt;  // the edge slots are no longer needed: the flags' prefix
    S1_TRY(exclusive_scan(S.q_first, qpos, nq + 1, nullptr, S.scan_quads, nullptr, s, S.dev + 6));
    S1_TRY(cudaMemcpyAsync(S.h_dev + 10, qpos + nq, 4, cudaMemcpyDeviceToHost, s));
    S1_TRY(cudaMemcpyAsync(S.h_dev + 6, S.dev + 6, 4, cudaMemcpyDeviceToHost, s));
    S1_TRY(cudaStreamSynchronize(s));
    if (S.h_dev[6]) return PAMO_ERR_DEVICE;
    const int n1 = S.h_dev[10];
    launch(k_s1_faces, grid_for(nq), kThreads, 0, s, (const int4 *)S.quads, (const int *)S.q_first, (const int *)qpos,
           (int)nq, n1, S.faces);
    if (S.prof) S.prof->end(s);
    S1_TRY(cudaGetLastError());
    S.n_verts = (int)nv;
    S.n_tris = (int)(2 * nq);
    return PAMO_OK;
}

}  // namespace s1
}  // namespace pamo
