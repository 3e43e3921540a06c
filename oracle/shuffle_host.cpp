// Init face permutation of the reference (simp_cuda/src/cusimp_free.cu:937-941:
// thrust::shuffle(faces, faces + n, thrust::default_random_engine{})), computed on
// the host with the open-source CCCL thrust headers of the CUDA toolkit.  The
// generic thrust shuffle (a Feistel bijection) is shared by its host and device
// back ends, so this reproduces the device permutation. TEST INFRASTRUCTURE.
#include <thrust/execution_policy.h>
#include <thrust/random.h>
#include <thrust/shuffle.h>

namespace {
struct Tri12 { int i, j, k; };
}

extern "C" void s2o_shuffle_faces(int *tris, int n_tris)
{
    Tri12 *t = reinterpret_cast<Tri12 *>(tris);
    thrust::default_random_engine rng;
    thrust::shuffle(thrust::host, t, t + n_tris, rng);
}
