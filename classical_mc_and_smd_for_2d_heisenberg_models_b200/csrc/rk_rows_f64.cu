// rk_rows_f64.cu -- FP64 plain-form instantiations of the row-band RK
// kernel, its shared-memory and block-size rules and the precision dispatch.
#include "rk_rows_impl.cuh"

namespace smd {

cudaError_t launch_rk_rows_f32(const RowsParams &P, const RKJob &J, int threads, size_t smem,
                               cudaStream_t st);

size_t rk_rows_smem(const RowsParams &P, int precision)
{
    const size_t v4 = precision == 0 ? 32 : 16;
    const size_t Np = (size_t)(P.ny_max + 4) * rows_pitch(P.L, rows_spt(precision));
    return 2 * Np * v4 + 2 * kMaxClusterCTAs * 4 * sizeof(double) + 32 * 4 * sizeof(double);
}

int rk_rows_threads(const RowsParams &P, int precision)
{
    const int t = P.ny_max * (P.L / rows_spt(precision));
    return (t + 31) / 32 * 32;
}

cudaError_t launch_rk_rows(const RowsParams &P, const RKJob &J, int precision, cudaStream_t st)
{
    const size_t smem = rk_rows_smem(P, precision);
    const int threads = rk_rows_threads(P, precision);
    if (precision == 0) return launch_rows_prec<double>(P, J, threads, smem, st);
    return launch_rk_rows_f32(P, J, threads, smem, st);
}

}  // namespace smd
