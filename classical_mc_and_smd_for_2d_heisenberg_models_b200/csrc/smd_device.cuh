// smd_device.cuh -- device-side data layout and helpers shared by the SMD
// kernels.
//
// HBM layout (per sample wave of W samples):
//   state    double [W][3][N]   FP64 spins, one SoA row per component
//   s0       double [W][3][N]   initial spins (for the autocorrelation)
//   imp      uint8  [W][N]      impurity flags (disordered lattices only)
//   snap     T      [W][R][3][N] spin snapshots of the R records of a chunk
//   series   cT     [W][3][n_rec][Q] S(q,t), q fastest
//   acc      double [3][Q][n_rec] sum over samples of |S(q,w)|^2
//   qss      double [W][n_rec]  per-sample spin autocorrelation
// Neighbour tables are ELL, [ztot][N] (shell s occupies rows zoff[s] ..
// zoff[s] + zn[s] - 1), so that a warp reading the k-th neighbour of 32
// consecutive sites issues one coalesced 128-byte load.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace smd {

// Most neighbours of one shell: 6 on the crystal lattices, 8 on the
// Ammann-Beenker approximants (Zn1 = ZnX = 8, Zn2 = 3;
// Codes_Folder/subrouts.cpp:1006-1012).
constexpr int kMaxShellNb = 8;

struct LatticeDev {
    int N;
    int zn[3];
    int zoff[3];
    int ztot;
    const int *nbr;          // ELL [ztot][N]
    int shell_on[3];
    double J[3][2][2];
    double lam[3][3];
    double coef[3][3];       // J[s][0][0] * lam[s][.]
    int lieb_delta_on;
    double j2_delta;
    double h;
    float Jf[3][2][2], lamf[3][3], coeff[3][3], j2_deltaf, hf;
    int energy_from_field;   // E = 1/2 sum_i (S_i . h_i - h S_i^z) holds
    int nbonds;              // explicit bond list (used when the identity fails)
    const int4 *bonds;       // (i, j, shell, 0)
};

struct RKJob {
    int n_samples;
    double dt;
    int stride;
    int rec_begin, rec_end;  // records written by this launch
    int n_rec;
    int fix_every;
    double *state;           // [W][3][N]
    const double *s0;        // [W][3][N]
    double *e0;              // [W]
    const uint8_t *imp;      // [W][N] or null
    void *snap;              // [W][R][3][N] of the snapshot type
    int snap_R;
    double *qss;             // [W][n_rec]
    double *stats;           // [W][4]: max drift, last E, E0, sigma_min
    int *status;             // nonzero after a numerical failure
    // FP32 form with a tensor-core list projection: the record also writes
    // the snapshot rows split into bf16 high and low parts, [W][R][3][kp]
    // (null: a separate pass splits the snapshots)
    void *bf_hi, *bf_lo;
    int bf_kp;
    // cluster kernel: per-CTA partial sums of the records' autocorrelation,
    // [W][n_rec][CS], summed into qss by a later launch (null: the cluster
    // reduces them itself with a cluster barrier per record)
    double *qpart;
};

// status bits (1 << k): zero correction denominator; bounded waits that
// expired in the tensor-core projection (2), the time transform (3) and
// the cluster RK kernel's halo exchange (4)
enum { kStatusOK = 0, kStatusBadSigma = 1, kStatusHaloTimeout = 4 };

// Mixed-radix factorisation of a transform length (product of radix = n).
struct FFTPlan {
    int n;
    int nst;
    int radix[16];
};

// Dynamic shared memory of a kernel: the limit is process-wide per kernel,
// so every launcher sets it to the device's opt-in maximum less the
// kernel's static shared memory (one value from every thread) instead of to
// its own launch's size, which a concurrent launch from another thread (the
// serving lanes) could undercut.
template <typename K>
inline cudaError_t allow_dynamic_smem(K kernel)
{
    static int max_optin = 0;
    if (!max_optin) {
        int dev = 0, mx = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&mx, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        max_optin = mx;
    }
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                max_optin - (int)fa.sharedSizeBytes);
}

template <typename T>
struct cplx {
    T x, y;
};

// Layout of a wave's windowed time series w[t] S(q,t): q in blocks of
// QB = 16 / sizeof(cplx<T>) consecutive q (2 in FP32, 1 in FP64), each block
// holding every record t of its q as [t][QB].  One block is a contiguous
// run of n_rec * 16 bytes, so the time transform fetches whole sequences
// with single bulk copies.  nqb = number of q blocks per (sample, component).
template <typename T>
__host__ __device__ constexpr int series_qb() { return 16 / (int)sizeof(cplx<T>); }

template <typename T>
__device__ __forceinline__ size_t series_off(int s, int c, int q, int t, int nqb, int n_rec)
{
    constexpr int QB = series_qb<T>();
    return ((((size_t)s * 3 + c) * nqb + q / QB) * n_rec + t) * QB + q % QB;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Compensated sum (Neumaier): the value is s + c, where c collects the exact
// rounding error of every addition into s (Knuth's TwoSum, exact for any
// operand order), so a sum of many terms carries about twice the working
// precision.  Used for the per-sample energies and the correction's sigma
// (Codes_Folder/subrouts.cpp:5181-5302, 11862-11902), whose difference
// E_ref - E1 sets the correction scale.  csum_add(a, b) and csum_add(b, a)
// are bit-identical, so butterfly (xor) shuffles leave every lane with the
// same total.
struct csum {
    double s, c;
};

__device__ __forceinline__ csum csum_add(csum a, csum b)
{
    const double s = a.s + b.s;
    const double bp = s - a.s;
    const double e = (a.s - (s - bp)) + (b.s - bp);
    return {s, (a.c + b.c) + e};
}

__device__ __forceinline__ void csum_acc(csum &a, double x) { a = csum_add(a, csum{x, 0.0}); }

__device__ __forceinline__ double csum_val(csum a) { return a.s + a.c; }

__device__ __forceinline__ csum warp_sum_c(csum v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = csum_add(v, csum{__shfl_xor_sync(0xffffffffu, v.s, o), __shfl_xor_sync(0xffffffffu, v.c, o)});
    return v;
}

// Block-wide compensated sum of NV values; every thread receives the totals
// (s + c).  red holds two slots of [32][NV][2] doubles (NV <= 4); the order
// of the additions is fixed, so results are deterministic run to run.
template <int NV>
__device__ __forceinline__ void block_sum_c(csum (&v)[NV], double *red, int &slot)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = warp_sum_c(v[k]);
    double *r = red + slot * 32 * 8;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            r[(warp * NV + k) * 2] = v[k].s;
            r[(warp * NV + k) * 2 + 1] = v[k].c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) {
        csum x = (lane < nw) ? csum{r[(lane * NV + k) * 2], r[(lane * NV + k) * 2 + 1]} : csum{0.0, 0.0};
        v[k] = warp_sum_c(x);
    }
    slot ^= 1;
}

// Block-wide sum of NV doubles; every thread receives the totals.  red holds
// two slots of [32][NV]; alternating slots lets consecutive reductions run
// with a single barrier each.  Summation order is fixed, so results are
// deterministic run to run.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *red, int &slot)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
    double *r = red + slot * 32 * NV;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) r[warp * NV + k] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double x = (lane < nw) ? r[lane * NV + k] : 0.0;
        v[k] = warp_sum(x);
    }
    slot ^= 1;
}

}  // namespace smd
