// Round-0 face permutation.  The reference shuffles the faces with
// thrust::shuffle and a default-constructed thrust::default_random_engine
// (simp_cuda/src/cusimp_free.cu:937-941); every later decision (edge order, key
// tie-breaks, adjacency order) depends on it, so the same open-source CCCL
// routine is called here on the context's stream.
#include <thrust/execution_policy.h>
#include <thrust/random.h>
#include <thrust/shuffle.h>

#include "stage2.cuh"

namespace pamo {

namespace {
// thrust's temporary storage from the stream-ordered pool (no device-wide
// synchronisation, and no fresh mapping once the pool holds the memory)
struct StreamScratch {
    typedef char value_type;
    cudaStream_t s;
    char *allocate(std::ptrdiff_t n)
    {
        void *p = nullptr;
        if (cudaMallocAsync(&p, (size_t)n, s) != cudaSuccess) throw std::bad_alloc();
        return static_cast<char *>(p);
    }
    void deallocate(char *p, size_t) { cudaFreeAsync(p, s); }
};
}  // namespace

int stage2_shuffle_faces(int4 *tris, int m, cudaStream_t s)
{
    if (m <= 1) return PAMO_OK;
    if (retain_pool_memory() != cudaSuccess) return PAMO_ERR_DEVICE;
    try {
        thrust::default_random_engine rng;
        StreamScratch alloc{s};
        thrust::shuffle(thrust::cuda::par_nosync(alloc).on(s), tris, tris + m, rng);
    } catch (...) {
        return PAMO_ERR_DEVICE;
    }
    return cudaGetLastError() == cudaSuccess ? PAMO_OK : PAMO_ERR_DEVICE;
}

}  // namespace pamo
