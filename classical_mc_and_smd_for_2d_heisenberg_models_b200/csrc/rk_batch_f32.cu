// rk_batch_f32.cu -- FP32 precision-form instantiations of the persistent
// batch RK kernel (compiled on their own so the units build in parallel).
#include "rk_cluster_impl.cuh"

namespace smd {

cudaError_t launch_rk_batch_f32(const BatchParams *B, int spt, int zt, int threads, int csh, int nclusters,
                                size_t smem, cudaStream_t st, int *max_clusters)
{
    return launch_batch_prec<float>(B, spt, zt, threads, csh, nclusters, smem, st, max_clusters);
}

}  // namespace smd
