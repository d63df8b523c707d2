// rk_cluster_f32.cu -- FP32 precision-form instantiations of the cluster RK
// kernel (compiled on their own so both precisions build in parallel).
#include "rk_cluster_impl.cuh"

namespace smd {

cudaError_t launch_rk_cluster_f32(const ClusterParams &P, const RKJob &J, int spt, int threads,
                                  size_t smem, cudaStream_t st)
{
    return launch_cluster_prec<float>(P, J, spt, threads, smem, st);
}

}  // namespace smd
