// rk_rows_f32.cu -- FP32 precision-form instantiations of the row-band RK
// kernel (compiled on their own so both precisions build in parallel).
#include "rk_rows_impl.cuh"

namespace smd {

cudaError_t launch_rk_rows_f32(const RowsParams &P, const RKJob &J, int threads, size_t smem,
                               cudaStream_t st)
{
    return launch_rows_prec<float>(P, J, threads, smem, st);
}

}  // namespace smd
