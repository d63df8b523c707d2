// grid_proj.cu -- projection of the spin snapshots onto the G x G q grid.
//
// get_SqData_iMKL (Codes_Folder/subrouts.cpp:8330-8432): each record's spins
// are embedded into the G x G DFT grid through gridMap (empty grid points
// are zero), transformed by a forward 2D DFT (sign -1, unscaled) and scaled
// by sqrt(1 / G^2).  Here the window weight w[t] of the time transform is
// folded into the same scale, and the values go straight into the q-blocked
// time series (series_off).
//
// Two records share one complex transform: the real grids A(t0), A(t1) of a
// component pack into Z = A(t0) + i A(t1), and
//     X(t0)[q] = (Z[q] + conj Z[-q]) / 2,   X(t1)[q] = (Z[q] - conj Z[-q]) / 2i.
// A block holds NG (3, or 1 for large grids) components, row-interleaved
// with an odd row pitch P = G + 1: element (g, r, col) at (r NG + g) P + col,
// so the row pass sees NG G sequences of stride P and the column pass
// NG P - 1 sequences of stride 1 (element stride NG P; the pad columns
// between components are transformed too and never read), both free of bank
// conflicts.  Each thread holds 16 values per stage.  Common
// grid sizes run a compile-time radix sequence (48 = 16 x 3, 128 = 16 x 8,
// ...), the others the runtime plan.
#include "fft_device.cuh"

namespace smd {

// two-stage transform with compile-time radices P1 then P2 (P2 = 1: none)
template <typename T, int C, int P1, int P2>
__device__ __forceinline__ void smem_fft_fixed(cplx<T> *buf, int n, int nseq, int ss, int es,
                                               const cplx<T> *tw)
{
    stockham_stage<T, P1, (C + P1 - 1) / P1>(buf, n, nseq, ss, es, 1, tw);
    if constexpr (P2 > 1) stockham_stage<T, P2, (C + P2 - 1) / P2>(buf, n, nseq, ss, es, P1, tw);
}

// blockIdx.x = pair * (3 / NG) + component group, blockIdx.y = sample.
// P1 > 0: the plan is (P1, P2) at compile time; else the runtime plan with
// the stage set FL.
template <typename TS, typename T, int FL, int P1, int P2, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) grid_proj_kernel(
    const TS *__restrict__ snap, int N, int R, int nrec_chunk, int rec_begin, int n_rec_total,
    const int *__restrict__ grid_map, FFTPlan plan, const cplx<T> *__restrict__ tw_g,
    double scale, const double *__restrict__ win, cplx<T> *__restrict__ series, int nqb, int NG)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int QB = series_qb<T>();
    const int G = plan.n, GG = G * G, NGG = NG * GG, P = G + 1;
    cplx<T> *buf = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *tw = buf + NG * G * P;
    cplx<T> *scratch = (FL & FK_GEN) ? tw + G : nullptr;
    const int groups = 3 / NG;
    const int pair = blockIdx.x / groups, g0 = (blockIdx.x % groups) * NG, s = blockIdx.y;
    const int slot0 = 2 * pair;
    const bool has1 = slot0 + 1 < nrec_chunk;
    const TS *x0 = snap + ((size_t)(s * R + slot0) * 3 + g0) * N;
    const TS *x1 = x0 + 3 * (size_t)N;   // the next slot
    for (int k = threadIdx.x; k < G; k += blockDim.x) tw[k] = tw_g[k];
#pragma unroll 4
    for (int p = threadIdx.x; p < NGG; p += blockDim.x) {
        const int g = p / GG, rem = p - g * GG;
        const int idx = grid_map[rem];
        T a = T(0), b = T(0);
        if (idx >= 0) {
            a = T(x0[(size_t)g * N + idx]);
            if (has1) b = T(x1[(size_t)g * N + idx]);
        }
        const int r = rem / G, col = rem - r * G;
        buf[(r * NG + g) * P + col] = {a, b};
    }
    __syncthreads();
    if constexpr (P1 > 0) {
        smem_fft_fixed<T, 16, P1, P2>(buf, G, NG * G, P, 1, tw);        // rows
        smem_fft_fixed<T, 16, P1, P2>(buf, G, NG * P - 1, 1, NG * P, tw);   // columns
    } else {
        smem_fft<T, 16, FL>(buf, G, NG * G, P, 1, plan.radix, plan.nst, tw, scratch);
        smem_fft<T, 16, FL>(buf, G, NG * P - 1, 1, NG * P, plan.radix, plan.nst, tw, scratch);
    }
    const int t0 = rec_begin + slot0;
    const T sc0 = T(scale * win[t0]), sc1 = has1 ? T(scale * win[t0 + 1]) : T(0);
    const int nblk = (GG + QB - 1) / QB;
    for (int e = threadIdx.x; e < NG * nblk; e += blockDim.x) {
        const int g = e / nblk, b = e - g * nblk;
        cplx<T> o0[QB], o1[QB];
#pragma unroll
        for (int i = 0; i < QB; i++) {
            const int q = min(b * QB + i, GG - 1);
            const int kr = q / G, kc = q - kr * G;
            const int nr = kr ? G - kr : 0, nc = kc ? G - kc : 0;
            const cplx<T> z = buf[(kr * NG + g) * P + kc], zm = buf[(nr * NG + g) * P + nc];
            o0[i] = {sc0 * T(0.5) * (z.x + zm.x), sc0 * T(0.5) * (z.y - zm.y)};
            o1[i] = {sc1 * T(0.5) * (z.y + zm.y), sc1 * T(-0.5) * (z.x - zm.x)};
        }
        // [t0][QB] then [t0 + 1][QB]: 32 contiguous bytes of the series
        cplx<T> *out = series + ((((size_t)s * 3 + g0 + g) * nqb + b) * n_rec_total + t0) * QB;
        if (b * QB + QB <= GG) {
            if constexpr (QB == 2) {
                *reinterpret_cast<float4 *>(out) = make_float4((float)o0[0].x, (float)o0[0].y,
                                                               (float)o0[QB - 1].x, (float)o0[QB - 1].y);
                if (has1)
                    *reinterpret_cast<float4 *>(out + QB) = make_float4(
                        (float)o1[0].x, (float)o1[0].y, (float)o1[QB - 1].x, (float)o1[QB - 1].y);
            } else {
                *reinterpret_cast<double2 *>(out) = make_double2((double)o0[0].x, (double)o0[0].y);
                if (has1)
                    *reinterpret_cast<double2 *>(out + QB) = make_double2((double)o1[0].x, (double)o1[0].y);
            }
        } else {
            // a block that the grid shares with the first list q
            out[0] = o0[0];
            if (has1) out[QB] = o1[0];
        }
    }
}

// ---------------------------------------------------------- launchers

namespace {

using GridKernelF = void (*)(const float *, int, int, int, int, int, const int *, FFTPlan,
                             const cplx<float> *, double, const double *, cplx<float> *, int, int);
using GridKernelD = void (*)(const double *, int, int, int, int, int, const int *, FFTPlan,
                             const cplx<double> *, double, const double *, cplx<double> *, int, int);

// compile-time plans: (P1, P2) for G = P1 * P2
template <typename T, int P1, int P2>
constexpr auto fixed_kernel()
{
    // FP32 blocks of up to 512 threads run two per SM; FP64 ones keep their
    // 16 values in 128 registers; G = 128 (16 x 8, one component) takes 1024
    constexpr int MAXT = (P1 * P2 > 64) ? 1024 : 512;
    constexpr int MINB = (MAXT == 512 && sizeof(T) == 4) ? 2 : 1;
    return grid_proj_kernel<T, T, FK_R16 | (P2 == 3 ? FK_R3 : 0), P1, P2, MAXT, MINB>;
}

template <typename T>
auto runtime_kernel(int fl)
{
    switch (fl & (FK_R3 | FK_GEN)) {
    case 0: return grid_proj_kernel<T, T, FK_R16, 0, 1, 1024, 1>;
    case FK_R3: return grid_proj_kernel<T, T, FK_R16 | FK_R3, 0, 1, 1024, 1>;
    case FK_GEN: return grid_proj_kernel<T, T, FK_R16 | FK_GEN, 0, 1, 1024, 1>;
    default: return grid_proj_kernel<T, T, FK_R16 | FK_R3 | FK_GEN, 0, 1, 1024, 1>;
    }
}

// the kernel for a plan: a compile-time radix sequence when one matches
template <typename T>
auto pick_kernel(const FFTPlan &p)
{
    const int r1 = p.nst > 0 ? p.radix[0] : 0, r2 = p.nst > 1 ? p.radix[1] : 1;
    if (p.nst <= 2) {
        if (r1 == 16 && r2 == 1) return fixed_kernel<T, 16, 1>();
        if (r1 == 16 && r2 == 2) return fixed_kernel<T, 16, 2>();
        if (r1 == 16 && r2 == 3) return fixed_kernel<T, 16, 3>();
        if (r1 == 16 && r2 == 4) return fixed_kernel<T, 16, 4>();
        if (r1 == 16 && r2 == 8) return fixed_kernel<T, 16, 8>();
        if (r1 == 8 && r2 == 3) return fixed_kernel<T, 8, 3>();
    }
    return runtime_kernel<T>(fft_plan_flags(p));
}

}  // namespace

// values a column pass of NG components transforms
static size_t grid_work(int G, int ng) { return (size_t)G * ((size_t)ng * (G + 1) - 1); }

// Components per block: all three while their values fit 512 threads of
// 16 values and the shared memory of two blocks per SM (FP32) or one (FP64),
// else one.  0: the grid does not fit one block.
int grid_proj_ng(int G, int precision, const FFTPlan &p)
{
    const size_t e = precision == 0 ? sizeof(cplx<double>) : sizeof(cplx<float>);
    const size_t mult = plan_generic(p) ? 2 : 1;
    const size_t GP = (size_t)G * (G + 1);
    const size_t cap3 = (precision == 0 ? 200 : 110) * 1024;
    if (grid_work(G, 3) <= 16 * 512 && 3 * GP * e * mult + G * e <= cap3) return 3;
    if (grid_work(G, 1) <= 16 * 1024 && GP * e * mult + G * e <= 200 * 1024) return 1;
    return 0;
}

size_t grid_proj_smem(int G, int precision, const FFTPlan &p)
{
    const size_t e = precision == 0 ? sizeof(cplx<double>) : sizeof(cplx<float>);
    const int ng = grid_proj_ng(G, precision, p);
    const size_t GP = (size_t)G * (G + 1) * (ng ? ng : 1);
    return (GP + G + (plan_generic(p) ? GP : 0)) * e;
}

cudaError_t launch_grid_proj(const void *snap, int precision, int N, int W, int R, int nrec_chunk,
                             int rec_begin, int n_rec_total, const int *grid_map, const FFTPlan &plan,
                             const void *tw, double scale, const double *win, void *series, int nqb,
                             cudaStream_t st)
{
    const int G = plan.n;
    const int ng = grid_proj_ng(G, precision, plan);
    if (!ng) return cudaErrorInvalidValue;
    const size_t smem = grid_proj_smem(G, precision, plan);
    const int threads = fft_threads((int)grid_work(G, ng), 16);
    dim3 grid(((nrec_chunk + 1) / 2) * (3 / ng), W);
    if (precision == 0) {
        GridKernelD k = pick_kernel<double>(plan);
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<grid, threads, smem, st>>>((const double *)snap, N, R, nrec_chunk, rec_begin, n_rec_total,
                                       grid_map, plan, (const cplx<double> *)tw, scale, win,
                                       (cplx<double> *)series, nqb, ng);
    } else {
        GridKernelF k = pick_kernel<float>(plan);
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<grid, threads, smem, st>>>((const float *)snap, N, R, nrec_chunk, rec_begin, n_rec_total,
                                       grid_map, plan, (const cplx<float> *)tw, scale, win,
                                       (cplx<float> *)series, nqb, ng);
    }
    return cudaGetLastError();
}

}  // namespace smd
