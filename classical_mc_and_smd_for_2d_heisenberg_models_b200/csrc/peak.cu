// peak.cu -- FMA throughput microbenchmark used as the denominator of the
// RK kernel's roofline (the driver-measured peaks cover HBM and BF16 tensor
// throughput only).  Every thread runs 8 independent FMA chains; the grid
// fills every SM several times over.
#include "../../include/smd_b200.h"

#include <cuda_runtime.h>

namespace {

template <typename T>
__global__ void __launch_bounds__(256) fma_kernel(T *out, int iters, T a, T b)
{
    T x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = T(threadIdx.x + k);
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = fma(x[k], a, b);
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    if (s == T(-1.2345)) out[0] = s;   // keeps the chains alive
}

template <typename T>
double run(int sms, int iters)
{
    T *d = nullptr;
    if (cudaMalloc(&d, sizeof(T)) != cudaSuccess) return -1.0;
    const int blocks = sms * 8, threads = 256;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_kernel<T><<<blocks, threads>>>(d, iters / 8, T(0.999999), T(1e-7));   // warm-up
    cudaEventRecord(e0);
    fma_kernel<T><<<blocks, threads>>>(d, iters, T(0.999999), T(1e-7));
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return -1.0;
    const double flops = 2.0 * 8.0 * (double)iters * blocks * threads;
    return flops / (ms * 1e-3) / 1e12;
}

}  // namespace

extern "C" int smd_measure_fma_peak(int device, int precision, double *tflops)
{
    if (!tflops) return SMD_EINVAL;
    if (cudaSetDevice(device) != cudaSuccess) return SMD_ECUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const double t = precision == SMD_FP64 ? run<double>(sms, 1 << 14) : run<float>(sms, 1 << 15);
    if (t <= 0.0) return SMD_ECUDA;
    *tflops = t;
    return SMD_OK;
}
