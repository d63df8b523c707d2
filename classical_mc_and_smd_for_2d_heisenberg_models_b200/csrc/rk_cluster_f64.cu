// rk_cluster_f64.cu -- FP64 plain-form instantiations of the cluster RK
// kernel, the shared-memory size rule and the precision dispatch.
#include "rk_cluster_impl.cuh"

namespace smd {

cudaError_t launch_rk_cluster_f32(const ClusterParams &P, const RKJob &J, int spt, int threads,
                                  size_t smem, cudaStream_t st);

size_t rk_cluster_smem(const ClusterParams &P, int precision)
{
    const size_t v4 = precision == 0 ? 32 : 16;
    const size_t Np = (size_t)P.n_loc_max + 1;
    size_t b = 2 * Np * v4 + (size_t)(P.ZT / 2) * P.n_own_max * 4 + (size_t)P.pmax * P.n_own_max * 4;
    b = (b + 15) & ~size_t(15);
    b += 2 * kMaxClusterCTAs * 8 * sizeof(double) + 32 * 8 * sizeof(double) + 2 * sizeof(uint64_t);
    // FP32 form: FP64 master spins of the own sites
    return b + (precision == 0 ? 0 : (size_t)3 * P.n_own_max * sizeof(double));
}

__global__ void qss_from_parts_kernel(const double *__restrict__ qpart, int W, int n_rec, int CS, int N,
                                      double *__restrict__ qss)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)W * n_rec) return;
    double s = 0.0;
    for (int r = 0; r < CS; r++) s += qpart[e * CS + r];
    qss[e] = (e % n_rec == 0) ? 1.0 : (1.0 / N) * s;
}

cudaError_t launch_qss_from_parts(const double *qpart, int W, int n_rec, int CS, int N, double *qss,
                                  cudaStream_t st)
{
    const size_t n = (size_t)W * n_rec;
    qss_from_parts_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(qpart, W, n_rec, CS, N, qss);
    return cudaGetLastError();
}

int rk_cluster_maxt(int precision, int spt)
{
    return precision == 0 ? cl_maxt<double>(spt) : cl_maxt<float>(spt);
}

cudaError_t launch_rk_cluster(const ClusterParams &P, const RKJob &J, int precision, int spt,
                              int threads, cudaStream_t st)
{
    const size_t smem = rk_cluster_smem(P, precision);
    if (precision == 0) return launch_cluster_prec<double>(P, J, spt, threads, smem, st);
    return launch_rk_cluster_f32(P, J, spt, threads, smem, st);
}

}  // namespace smd
