// rk_batch_f64.cu -- FP64 plain-form instantiations of the persistent batch
// RK kernel and the precision dispatch.
#include "rk_cluster_impl.cuh"

namespace smd {

cudaError_t launch_rk_batch_f32(const BatchParams *B, int spt, int zt, int threads, int csh, int nclusters,
                                size_t smem, cudaStream_t st, int *max_clusters);

static cudaError_t batch_dispatch(const BatchParams *B, int precision, int spt, int zt, int threads, int csh,
                                  int nclusters, size_t smem, cudaStream_t st, int *max_clusters)
{
    if (precision == 0)
        return launch_batch_prec<double>(B, spt, zt, threads, csh, nclusters, smem, st, max_clusters);
    return launch_rk_batch_f32(B, spt, zt, threads, csh, nclusters, smem, st, max_clusters);
}

cudaError_t launch_rk_batch(const BatchParams &B, int precision, int spt, int zt, int threads, int csh,
                            int nclusters, size_t smem, cudaStream_t st)
{
    return batch_dispatch(&B, precision, spt, zt, threads, csh, nclusters, smem, st, nullptr);
}

int rk_batch_max_clusters(int precision, int spt, int zt, int threads, int csh, size_t smem)
{
    int n = 0;
    // the occupancy query reads no parameter
    if (batch_dispatch(nullptr, precision, spt, zt, threads, csh, 0, smem, nullptr, &n) != cudaSuccess) return 0;
    return n;
}

int rk_batch_threads(int precision, int spt)
{
    return precision == 0 ? cl_maxt<double>(spt) : cl_maxt<float>(spt);
}

}  // namespace smd
