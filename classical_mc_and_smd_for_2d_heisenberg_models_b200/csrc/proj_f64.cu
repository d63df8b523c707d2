// proj_f64.cu -- list-q projection of the FP64 plain form on the FP64
// tensor cores (DMMA, mma.sync m8n8k4 f64).
//
// S(q_l) = scale sum_k S_k exp(-i q_l . pos_k) (get_qct_SqData,
// Codes_Folder/subrouts.cpp:8460-8525) for every snapshot row of a sample
// (record, component) is the real GEMM
//
//     C[m][2l + 0/1] = sum_k A[m][k] P[k][2l + 0/1]
//     A = the sample's snapshot rows [rows][N] (m = slot * 3 + c)
//     P = phase table [N][Lq] complex = [N][2 Lq] real, scale folded in
//
// computed in FP64 throughout (the products and sums of the reference's
// direct sum, reordered).  Block tile 64 rows x 64 real columns (32 q), K
// steps of 16 sites staged through shared memory by cp.async (two stages);
// four warps of 32 x 32, each a 4 x 4 grid of 8 x 8 DMMA tiles.  A thread's
// accumulator pair (c0, c1) is one complex value S(q), written straight into
// the q-blocked time series with the record's window weight.
#include "smd_device.cuh"

namespace smd {

namespace dm {

constexpr int BM = 64, BN = 64, BK = 16, APAD = 4, BPAD = 4;

__device__ __forceinline__ void cp8(void *dst, const void *src, bool ok)
{
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(ok ? 8 : 0) : "memory");
}

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

}  // namespace dm

// grid: (column tiles of 2 Lq, row tiles, samples); 128 threads.
__global__ void __launch_bounds__(128) list_proj_dmma_kernel(
    const double *__restrict__ snap, int rows, int N, int R, int rec_begin, int n_rec_total,
    const double *__restrict__ P, int Lq, const double *__restrict__ win, cplx<double> *__restrict__ series,
    int nqb, int qoff)
{
    using namespace dm;
    __shared__ __align__(16) double As[2][BM][BK + APAD];
    __shared__ __align__(16) double Bs[2][BK][BN + BPAD];
    const int n0 = blockIdx.x * BN, m0 = blockIdx.y * BM, s = blockIdx.z;
    const int ncol = 2 * Lq;
    const double *A = snap + (size_t)s * R * 3 * N;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;

    auto load = [&](int stage, int k0) {
        // A tile: BM x BK doubles, 8 per thread; B tile: BK x BN, 8 per thread
#pragma unroll
        for (int u = 0; u < (BM * BK) / 128; u++) {
            const int e = tid + u * 128, mm = e / BK, kk = e % BK;
            const int m = m0 + mm, k = k0 + kk;
            const bool ok = m < rows && k < N;
            cp8(&As[stage][mm][kk], ok ? A + (size_t)m * N + k : A, ok);
        }
#pragma unroll
        for (int u = 0; u < (BK * BN) / 128; u++) {
            const int e = tid + u * 128, kk = e / BN, nn = e % BN;
            const int k = k0 + kk, n = n0 + nn;
            const bool ok = k < N && n < ncol;
            cp8(&Bs[stage][kk][nn], ok ? P + (size_t)k * ncol + n : P, ok);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

    const int nk = (N + BK - 1) / BK;
    load(0, 0);
    for (int kt = 0; kt < nk; kt++) {
        const int st = kt & 1;
        if (kt + 1 < nk) {
            load(st ^ 1, (kt + 1) * BK);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
#pragma unroll
        for (int k4 = 0; k4 < BK; k4 += 4) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[st][wm + i * 8 + g][k4 + t];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[st][k4 + t][wn + j * 8 + g];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) dmma(acc[i][j], a[i], b[j]);
        }
        __syncthreads();   // the stage is refilled by the next iteration's load
    }
    // epilogue: row wm + i*8 + g, columns wn + j*8 + 2t (+1) = one complex q
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int m = m0 + wm + i * 8 + g;
        if (m >= rows) continue;
        const int c = m % 3, rec = rec_begin + m / 3;
        const double w = win[rec];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int l = (n0 + wn + j * 8) / 2 + t;
            if (l < Lq)
                series[series_off<double>(s, c, qoff + l, rec, nqb, n_rec_total)] = {w * acc[i][j][0],
                                                                                   w * acc[i][j][1]};
        }
    }
}

cudaError_t launch_list_proj_f64(const double *snap, int W, int R, int nrec_chunk, int N, int rec_begin,
                                 int n_rec_total, const double *P, int Lq, const double *win, void *series,
                                 int nqb, int qoff, cudaStream_t st)
{
    const int rows = nrec_chunk * 3;
    dim3 grid((2 * Lq + dm::BN - 1) / dm::BN, (rows + dm::BM - 1) / dm::BM, W);
    list_proj_dmma_kernel<<<grid, 128, 0, st>>>(snap, rows, N, R, rec_begin, n_rec_total, P, Lq, win,
                                               (cplx<double> *)series, nqb, qoff);
    return cudaGetLastError();
}

}  // namespace smd
