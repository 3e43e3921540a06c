// pamo_self_intersect_noalloc: the whole-mesh self-intersection check with all
// of its scratch memory in one file-scope device array, for callers that cannot
// allocate device memory (see include/pamo_b200.h).
#include <cstring>

#include "lbvh.cuh"
#include "scan.cuh"
#include "stage2.cuh"

namespace pamo {
namespace {

constexpr int kMaxFaces = 32768;   // limit of this entry point
constexpr int kMaxVerts = 65536;
constexpr int kPairsPerFace = 24;  // sizes the pair buffer: 24 * kMaxFaces candidate pairs in total
constexpr int kTiles = (kMaxFaces + kLbvhSortTile - 1) / kLbvhSortTile;  // lbvh_build's sort tiles

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// byte offsets inside the scratch array
constexpr size_t kOffPts = 0;
constexpr size_t kOffTris = kOffPts + align256(sizeof(float4) * kMaxVerts);
constexpr size_t kOffActive = kOffTris + align256(sizeof(int4) * kMaxFaces);
constexpr size_t kOffKeys = kOffActive + align256(kMaxFaces);
constexpr size_t kOffKeys2 = kOffKeys + align256(4 * (size_t)kMaxFaces);
constexpr size_t kOffVals = kOffKeys2 + align256(4 * (size_t)kMaxFaces);
constexpr size_t kOffVals2 = kOffVals + align256(4 * (size_t)kMaxFaces);
constexpr size_t kOffHist = kOffVals2 + align256(4 * (size_t)kMaxFaces);
constexpr size_t kOffHistScratch = kOffHist + align256(4 * (256 * (size_t)kTiles + 64));
constexpr size_t kOffNodes = kOffHistScratch + align256(4 * (size_t)scan_scratch_ints(256LL * kTiles));
constexpr size_t kOffParent = kOffNodes + align256(sizeof(BvhNode) * kMaxFaces);
constexpr size_t kOffFlags = kOffParent + align256(4 * 2 * (size_t)kMaxFaces);
constexpr size_t kOffLeafOfFace = kOffFlags + align256(4 * (size_t)kMaxFaces);
constexpr size_t kOffScene = kOffLeafOfFace + align256(4 * (size_t)kMaxFaces);
constexpr size_t kOffPairs = kOffScene + align256(64);
constexpr size_t kOffCounters = kOffPairs + align256(sizeof(uint2) * kPairsPerFace * (size_t)kMaxFaces);
constexpr size_t kOffBad = kOffCounters + align256(sizeof(RoundCounters));
constexpr size_t kScratchBytes = kOffBad + 256;  // about 11 MB
static_assert(kOffHistScratch - kOffHist >= 4 * (256 * (size_t)kTiles), "radix histogram area");
static_assert(kOffPairs - kOffScene >= 64, "scene area");

// Held by every GPU that loads the library, until the process exits.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

__global__ void k_na_validate(const int *tris, int m, int n, int *bad)
{
    int local = 0;
    PAMO_GRID_STRIDE(f, m)
    {
        int a = tris[3 * f], b = tris[3 * f + 1], c = tris[3 * f + 2];
        bool dead = a == -1 && b == -1 && c == -1;
        bool ok = a >= 0 && a < n && b >= 0 && b < n && c >= 0 && c < n;
        local += !(dead || ok);
    }
    if (local) atomicAdd(bad, local);
}

__global__ void k_na_convert(const float *pts, int n, const int *tris, int m, float4 *p4, int4 *t4)
{
    long long N = n > m ? n : m;
    PAMO_GRID_STRIDE(i, N)
    {
        if (i < n) p4[i] = make_float4(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], 0.f);
        if (i < m) t4[i] = make_int4(tris[3 * i], tris[3 * i + 1], tris[3 * i + 2], 0);
    }
}

}  // namespace
}  // namespace pamo

using namespace pamo;

extern "C" int pamo_self_intersect_noalloc(const float *d_points, const int *d_tris, int n_pts, int n_tris,
                                           unsigned char *d_out_flags, long long *out_n_pairs, void *stream)
{
    if (n_pts < 0 || n_tris < 0 || (n_tris && (n_pts == 0 || !d_points || !d_tris || !d_out_flags)))
        return PAMO_ERR_INVALID_ARG;
    if (n_tris > kMaxFaces || n_pts > kMaxVerts) return PAMO_ERR_CAPACITY;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PAMO_ERR_NO_DEVICE;
    // The array's name is a host-side stand-in; the kernels need its device
    // address on the current device.  It is looked up on every call (a table
    // lookup in the runtime once the module is loaded), so no cached address
    // can outlive a device reset or belong to another thread's device.  The
    // first call on a device loads the module.
    void *addr = nullptr;
    if (cudaGetSymbolAddress(&addr, g_scratch) != cudaSuccess || !addr) return PAMO_ERR_DEVICE;
    unsigned char *base = static_cast<unsigned char *>(addr);
    cudaStream_t s = (cudaStream_t)stream;
    if (n_tris == 0) {
        if (out_n_pairs) *out_n_pairs = 0;
        return PAMO_OK;
    }
    int *bad = reinterpret_cast<int *>(base + kOffBad);
    int h_bad = 0;
    if (cudaMemsetAsync(bad, 0, sizeof(int), s) != cudaSuccess) return PAMO_ERR_DEVICE;
    launch(k_na_validate, grid_for(n_tris), kThreads, 0, s, d_tris, n_tris, n_pts, bad);
    if (cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return PAMO_ERR_DEVICE;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PAMO_ERR_DEVICE;
    if (h_bad) return PAMO_ERR_INVALID_ARG;

    float4 *p4 = reinterpret_cast<float4 *>(base + kOffPts);
    int4 *t4 = reinterpret_cast<int4 *>(base + kOffTris);
    uint8_t *active = base + kOffActive;
    uint2 *pairs = reinterpret_cast<uint2 *>(base + kOffPairs);
    RoundCounters *cnt = reinterpret_cast<RoundCounters *>(base + kOffCounters);
    Lbvh b;  // views into the scratch array; never released (nothing was allocated)
    b.cap = kMaxFaces;
    b.sort_tiles = kTiles;
    b.keys = reinterpret_cast<uint32_t *>(base + kOffKeys);
    b.keys2 = reinterpret_cast<uint32_t *>(base + kOffKeys2);
    b.vals = reinterpret_cast<int *>(base + kOffVals);
    b.vals2 = reinterpret_cast<int *>(base + kOffVals2);
    b.hist = reinterpret_cast<int *>(base + kOffHist);
    b.hist_scratch = reinterpret_cast<int *>(base + kOffHistScratch);
    b.nodes = reinterpret_cast<BvhNode *>(base + kOffNodes);
    b.parent = reinterpret_cast<int *>(base + kOffParent);
    b.flags = reinterpret_cast<int *>(base + kOffFlags);
    b.leaf_of_face = reinterpret_cast<int *>(base + kOffLeafOfFace);
    b.scene = reinterpret_cast<int *>(base + kOffScene);

    // the array keeps the previous call's contents: reset what must start at zero
    launch(k_na_convert, grid_for(n_pts > n_tris ? n_pts : n_tris), kThreads, 0, s, d_points, n_pts, d_tris, n_tris, p4,
                                                                               t4);
    if (cudaMemsetAsync(active, 1, (size_t)n_tris, s) != cudaSuccess) return PAMO_ERR_DEVICE;
    if (cudaMemsetAsync(cnt, 0, sizeof(RoundCounters), s) != cudaSuccess) return PAMO_ERR_DEVICE;
    if (cudaMemsetAsync(d_out_flags, 0, (size_t)n_tris, s) != cudaSuccess) return PAMO_ERR_DEVICE;
    if (lbvh_build(b, p4, t4, n_tris, s) != cudaSuccess) return PAMO_ERR_DEVICE;
    if (lbvh_refit(b, p4, t4, n_tris, s) != cudaSuccess) return PAMO_ERR_DEVICE;
    const long long cap_pairs = (long long)kPairsPerFace * kMaxFaces;
    if (query_and_test_pairs(b.nodes, b.vals, b.scene, p4, t4, active, n_tris, pairs, cap_pairs, cnt, d_out_flags, s) !=
        cudaSuccess)
        return PAMO_ERR_DEVICE;
    RoundCounters h{};
    if (cudaMemcpyAsync(&h, cnt, sizeof(RoundCounters), cudaMemcpyDeviceToHost, s) != cudaSuccess) return PAMO_ERR_DEVICE;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PAMO_ERR_DEVICE;
    if (h.pair_overflow > 0 || h.stack_overflow > 0) return PAMO_ERR_CAPACITY;
    if (out_n_pairs) *out_n_pairs = h.n_pairs;
    return PAMO_OK;
}
