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
// ...), the others the runtime plan, whose kernel calls its stages out of
// line, holds 8 values per thread and transforms the rows (then the
// columns) in batches of at most 8 x blockDim.x values: the sequences
// of a pass are independent, so a grid larger than the threads' registers
// (one component of a 144 x 144 grid, 20736 values) still takes one block.
#include "fft_device.cuh"

#include <algorithm>

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
// the stage set FL, in batches of sequences.
template <typename TS, typename T, int FL, int P1, int P2, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) grid_proj_kernel(
    const TS *__restrict__ snap, int N, int R, int nrec_chunk, int rec_begin, int n_rec_total,
    const int *__restrict__ grid_map, FFTPlan plan, const cplx<T> *__restrict__ tw_g,
    double scale, const double *__restrict__ win, cplx<T> *__restrict__ series, int nqb, int NG,
    int scr_seqs)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int QB = series_qb<T>();
    const int G = plan.n, GG = G * G, P = G + 1;
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
    // one grid-map load serves the NG components of both records
#pragma unroll 4
    for (int rem = threadIdx.x; rem < GG; rem += blockDim.x) {
        const int idx = grid_map[rem];
        const int r = rem / G, col = rem - r * G;
        T a[3], b[3];
#pragma unroll
        for (int g = 0; g < 3; g++) {
            a[g] = T(0);
            b[g] = T(0);
            if (g < NG && idx >= 0) {
                a[g] = T(x0[(size_t)g * N + idx]);
                if (has1) b[g] = T(x1[(size_t)g * N + idx]);
            }
        }
#pragma unroll
        for (int g = 0; g < 3; g++)
            if (g < NG) buf[(r * NG + g) * P + col] = {a[g], b[g]};
    }
    __syncthreads();
    if constexpr (P1 > 0) {
        smem_fft_fixed<T, 16, P1, P2>(buf, G, NG * G, P, 1, tw);        // rows
        smem_fft_fixed<T, 16, P1, P2>(buf, G, NG * P - 1, 1, NG * P, tw);   // columns
    } else {
        const int cap = max(1, 8 * (int)blockDim.x / G);    // sequences per batch
        for (int q0 = 0; q0 < NG * G; q0 += cap)            // rows
            smem_fft<T, 8, FL>(buf + (size_t)q0 * P, G, min(cap, NG * G - q0), P, 1, plan.radix,
                               plan.nst, tw, scratch, scr_seqs);
        for (int q0 = 0; q0 < NG * P - 1; q0 += cap)        // columns
            smem_fft<T, 8, FL>(buf + q0, G, min(cap, NG * P - 1 - q0), 1, NG * P, plan.radix,
                               plan.nst, tw, scratch, scr_seqs);
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

// ---------------------------------------------------------- large grids
//
// Grids too large for one block (G up to 512) take two passes through a
// global scratch Zg [W][pairs][3][G][G] of the packed complex grids:
// rows first (RT rows per block), then columns.  A column block transforms
// CT columns kc and their mirrors (G - kc) % G, which the Hermitian
// separation of the two records needs, and writes the series as the
// one-block kernel does.

// blockIdx.x = (pair * 3 + c) * row_tiles + tile, blockIdx.y = sample
template <typename TS, typename T, int FL>
__global__ void __launch_bounds__(512) grid_rows_kernel(
    const TS *__restrict__ snap, int N, int R, int nrec_chunk, const int *__restrict__ grid_map,
    FFTPlan plan, const cplx<T> *__restrict__ tw_g, cplx<T> *__restrict__ Zg, int RT,
    int scr_seqs)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int G = plan.n, P = G + 1;
    const int tiles = (G + RT - 1) / RT;
    const int tile = blockIdx.x % tiles, pc = blockIdx.x / tiles;
    const int c = pc % 3, pair = pc / 3, s = blockIdx.y;
    const int r0 = tile * RT, nr = min(RT, G - r0);
    cplx<T> *buf = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *tw = buf + (size_t)RT * P;
    cplx<T> *scratch = (FL & FK_GEN) ? tw + G : nullptr;
    const int slot0 = 2 * pair;
    const bool has1 = slot0 + 1 < nrec_chunk;
    const TS *x0 = snap + ((size_t)(s * R + slot0) * 3 + c) * N;
    const TS *x1 = x0 + 3 * (size_t)N;
    for (int k = threadIdx.x; k < G; k += blockDim.x) tw[k] = tw_g[k];
#pragma unroll 4
    for (int e = threadIdx.x; e < RT * G; e += blockDim.x) {
        const int rr = e / G, col = e - rr * G;
        T a = T(0), b = T(0);
        if (rr < nr) {
            const int idx = grid_map[(r0 + rr) * G + col];
            if (idx >= 0) {
                a = T(x0[idx]);
                if (has1) b = T(x1[idx]);
            }
        }
        buf[rr * P + col] = {a, b};
    }
    __syncthreads();
    smem_fft<T, 8, FL>(buf, G, RT, P, 1, plan.radix, plan.nst, tw, scratch, scr_seqs);
    cplx<T> *z = Zg + (((size_t)s * ((R + 1) / 2) + pair) * 3 + c) * G * G;
    for (int e = threadIdx.x; e < nr * G; e += blockDim.x) {
        const int rr = e / G, col = e - rr * G;
        z[(size_t)(r0 + rr) * G + col] = buf[rr * P + col];
    }
}

// blockIdx.x = (pair * 3 + c) * col_tiles + tile, blockIdx.y = sample
template <typename T, int FL>
__global__ void __launch_bounds__(512) grid_cols_kernel(
    int R, int nrec_chunk, int rec_begin, int n_rec_total, FFTPlan plan,
    const cplx<T> *__restrict__ tw_g, const cplx<T> *__restrict__ Zg, double scale,
    const double *__restrict__ win, cplx<T> *__restrict__ series, int nqb, int CT, int scr_seqs)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int QB = series_qb<T>();
    const int G = plan.n, W2 = 2 * CT, Pw = W2 + 1;   // element pitch (odd)
    const int tiles = (G + CT - 1) / CT;
    const int tile = blockIdx.x % tiles, pc = blockIdx.x / tiles;
    const int c = pc % 3, pair = pc / 3, s = blockIdx.y;
    const int c0 = tile * CT;
    cplx<T> *buf = reinterpret_cast<cplx<T> *>(smem_raw);    // [G][Pw]
    cplx<T> *tw = buf + (size_t)G * Pw;
    cplx<T> *scratch = (FL & FK_GEN) ? tw + G : nullptr;
    const int slot0 = 2 * pair;
    const bool has1 = slot0 + 1 < nrec_chunk;
    const cplx<T> *z = Zg + (((size_t)s * ((R + 1) / 2) + pair) * 3 + c) * G * G;
    for (int k = threadIdx.x; k < G; k += blockDim.x) tw[k] = tw_g[k];
    // columns j < CT: kc = c0 + j; columns CT + j: their mirrors
#pragma unroll 4
    for (int e = threadIdx.x; e < G * W2; e += blockDim.x) {
        const int x = e / W2, j = e - x * W2;
        const int jj = j < CT ? j : j - CT;
        int kc = min(c0 + jj, G - 1);
        if (j >= CT) kc = kc ? G - kc : 0;
        buf[x * Pw + j] = z[(size_t)x * G + kc];
    }
    __syncthreads();
    smem_fft<T, 8, FL>(buf, G, W2, 1, Pw, plan.radix, plan.nst, tw, scratch, scr_seqs);
    const int t0 = rec_begin + slot0;
    const T sc0 = T(scale * win[t0]), sc1 = has1 ? T(scale * win[t0 + 1]) : T(0);
    const int nb = (CT + QB - 1) / QB;   // q blocks of a row in this tile
    for (int e = threadIdx.x; e < G * nb; e += blockDim.x) {
        const int kr = e / nb, jb = e - kr * nb;
        const int nr = kr ? G - kr : 0;
        cplx<T> o0[QB], o1[QB];
        bool ok = true;
#pragma unroll
        for (int i = 0; i < QB; i++) {
            const int j = jb * QB + i;
            ok = ok && (j < CT) && (c0 + j < G);
            const int jc = min(j, CT - 1);
            const cplx<T> zz = buf[kr * Pw + jc], zm = buf[nr * Pw + CT + jc];
            o0[i] = {sc0 * T(0.5) * (zz.x + zm.x), sc0 * T(0.5) * (zz.y - zm.y)};
            o1[i] = {sc1 * T(0.5) * (zz.y + zm.y), sc1 * T(-0.5) * (zz.x - zm.x)};
        }
        if (!ok) continue;
        const int q = kr * G + c0 + jb * QB;   // q and q + 1 share a block (G, c0, CT even)
        cplx<T> *out = series + ((((size_t)s * 3 + c) * nqb + q / QB) * n_rec_total + t0) * QB;
#pragma unroll
        for (int i = 0; i < QB; i++) {
            out[i] = o0[i];
            if (has1) out[QB + i] = o1[i];
        }
    }
}

// ---------------------------------------------------------- launchers

namespace {

using GridKernelF = void (*)(const float *, int, int, int, int, int, const int *, FFTPlan,
                             const cplx<float> *, double, const double *, cplx<float> *, int, int,
                             int);
using GridKernelD = void (*)(const double *, int, int, int, int, int, const int *, FFTPlan,
                             const cplx<double> *, double, const double *, cplx<double> *, int, int,
                             int);

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

// Runtime plans: stages out of line, sequences in batches, 64 registers a
// thread; launched with up to 512 threads while two blocks fit an SM's
// shared memory (the blocks' phases overlap), else up to 1024 (measured on
// honeycomb, kagome, square and triangular grids of 36 to 144 points).
constexpr int kRuntimeThreads = 1024;
constexpr size_t kTwoBlockSmem = 113 * 1024;

template <typename T>
auto runtime_kernel(int fl)
{
    constexpr int M = kRuntimeThreads, O = FK_OOL | FK_R16;
    if (fl & FK_R5) return grid_proj_kernel<T, T, O | FK_R3 | FK_R5, 0, 1, M, 1>;
    switch (fl & (FK_R3 | FK_GEN)) {
    case 0: return grid_proj_kernel<T, T, O, 0, 1, M, 1>;
    case FK_R3: return grid_proj_kernel<T, T, O | FK_R3, 0, 1, M, 1>;
    case FK_GEN: return grid_proj_kernel<T, T, O | FK_GEN, 0, 1, M, 1>;
    default: return grid_proj_kernel<T, T, O | FK_R3 | FK_GEN, 0, 1, M, 1>;
    }
}

// whether a plan runs a compile-time radix sequence
static bool fixed_plan(const FFTPlan &p)
{
    const int r1 = p.nst > 0 ? p.radix[0] : 0, r2 = p.nst > 1 ? p.radix[1] : 1;
    if (p.nst > 2) return false;
    return (r1 == 16 && (r2 == 1 || r2 == 2 || r2 == 3 || r2 == 4 || r2 == 8)) || (r1 == 8 && r2 == 3);
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

// sequences of length G the out-of-line stage's copy holds (at most 4096
// values, at least one sequence); 0 for plans without such a stage
static int grid_scratch_seqs(int G, int ng, const FFTPlan &p)
{
    if (!plan_generic(p)) return 0;
    const size_t all = (size_t)ng * (G + 1);
    const size_t cap = std::max<size_t>(1, 4096 / (size_t)G);
    return (int)std::min(all, cap);
}

// Components per block: all three while their values fit 512 threads of
// 16 values and the shared memory of two blocks per SM (FP32) or one (FP64),
// else one while the component's grid fits the shared memory of a block (a
// compile-time plan also needs its values to fit 1024 threads of 16; the
// runtime kernel batches its sequences).  0: the grid does not fit one block.
static size_t grid_smem_ng(int G, int ng, int precision, const FFTPlan &p)
{
    const size_t e = precision == 0 ? sizeof(cplx<double>) : sizeof(cplx<float>);
    return ((size_t)ng * G * (G + 1) + G + (size_t)grid_scratch_seqs(G, ng, p) * G) * e;
}

int grid_proj_ng(int G, int precision, const FFTPlan &p)
{
    const size_t cap3 = (precision == 0 ? 200 : 110) * 1024;
    if (grid_work(G, 3) <= 16 * 512 && grid_smem_ng(G, 3, precision, p) <= cap3) return 3;
    if (fixed_plan(p) && grid_work(G, 1) > 16 * 1024) return 0;
    if (grid_smem_ng(G, 1, precision, p) <= 220 * 1024) return 1;
    return 0;
}

size_t grid_proj_smem(int G, int precision, const FFTPlan &p)
{
    const int ng = grid_proj_ng(G, precision, p);
    return grid_smem_ng(G, ng ? ng : 1, precision, p);
}

// tile sizes of the two-pass path: rows per row block, columns per column
// block (even, with their mirrors 2 CT columns), about 2048 values each,
// transformed with 8 values per thread by at most 512 threads
static int large_rt(int G) { return std::max(1, std::min(G, 2048 / G)); }
static int large_ct(int G) { return std::max(2, std::min(G, 1024 / G) & ~1); }

static size_t large_smem(int G, int n_values, int precision, const FFTPlan &p, int *scr)
{
    const size_t e = precision == 0 ? sizeof(cplx<double>) : sizeof(cplx<float>);
    *scr = plan_generic(p) ? std::max(1, 4096 / G) : 0;
    return ((size_t)n_values + G + (size_t)*scr * G) * e;
}

bool grid_large_ok(int G, int precision, const FFTPlan &p)
{
    if (G > 512 || (G & 1)) return false;
    int scr;
    const size_t a = large_smem(G, large_rt(G) * (G + 1), precision, p, &scr);
    const size_t b = large_smem(G, G * (2 * large_ct(G) + 1), precision, p, &scr);
    return std::max(a, b) <= 200 * 1024 && (size_t)G * (2 * large_ct(G) + 1) <= 8 * 512 &&
           (size_t)large_rt(G) * (G + 1) <= 8 * 512;
}

size_t grid_large_scratch(int G, int R, int precision)
{
    const size_t e = precision == 0 ? sizeof(cplx<double>) : sizeof(cplx<float>);
    return (size_t)((R + 1) / 2) * 3 * G * G * e;   // per sample
}

cudaError_t launch_grid_proj_large(const void *snap, int precision, int N, int W, int R,
                                   int nrec_chunk, int rec_begin, int n_rec_total,
                                   const int *grid_map, const FFTPlan &plan, const void *tw,
                                   double scale, const double *win, void *series, int nqb,
                                   void *Zg, cudaStream_t st)
{
    const int G = plan.n, RT = large_rt(G), CT = large_ct(G);
    const int pairs = (nrec_chunk + 1) / 2;
    int scr_r, scr_c;
    const size_t sm_r = large_smem(G, RT * (G + 1), precision, plan, &scr_r);
    const size_t sm_c = large_smem(G, G * (2 * CT + 1), precision, plan, &scr_c);
    const int thr_r = fft_threads(RT * (G + 1), 8), thr_c = fft_threads(G * (2 * CT + 1), 8);
    const dim3 gr(pairs * 3 * ((G + RT - 1) / RT), W), gc(pairs * 3 * ((G + CT - 1) / CT), W);
    const bool gen = plan_generic(plan), r5 = (fft_plan_flags(plan) & FK_R5) != 0;
    if (precision == 0) {
        auto kr = gen ? grid_rows_kernel<double, double, FK_R16 | FK_R3 | FK_GEN>
                : r5  ? grid_rows_kernel<double, double, FK_R16 | FK_R3 | FK_R5>
                      : grid_rows_kernel<double, double, FK_R16 | FK_R3>;
        auto kc = gen ? grid_cols_kernel<double, FK_R16 | FK_R3 | FK_GEN>
                : r5  ? grid_cols_kernel<double, FK_R16 | FK_R3 | FK_R5>
                      : grid_cols_kernel<double, FK_R16 | FK_R3>;
        allow_dynamic_smem(kr);
        allow_dynamic_smem(kc);
        kr<<<gr, thr_r, sm_r, st>>>((const double *)snap, N, R, nrec_chunk, grid_map, plan,
                                    (const cplx<double> *)tw, (cplx<double> *)Zg, RT, scr_r);
        kc<<<gc, thr_c, sm_c, st>>>(R, nrec_chunk, rec_begin, n_rec_total, plan, (const cplx<double> *)tw,
                                    (const cplx<double> *)Zg, scale, win, (cplx<double> *)series, nqb, CT,
                                    scr_c);
    } else {
        auto kr = gen ? grid_rows_kernel<float, float, FK_R16 | FK_R3 | FK_GEN>
                : r5  ? grid_rows_kernel<float, float, FK_R16 | FK_R3 | FK_R5>
                      : grid_rows_kernel<float, float, FK_R16 | FK_R3>;
        auto kc = gen ? grid_cols_kernel<float, FK_R16 | FK_R3 | FK_GEN>
                : r5  ? grid_cols_kernel<float, FK_R16 | FK_R3 | FK_R5>
                      : grid_cols_kernel<float, FK_R16 | FK_R3>;
        allow_dynamic_smem(kr);
        allow_dynamic_smem(kc);
        kr<<<gr, thr_r, sm_r, st>>>((const float *)snap, N, R, nrec_chunk, grid_map, plan,
                                    (const cplx<float> *)tw, (cplx<float> *)Zg, RT, scr_r);
        kc<<<gc, thr_c, sm_c, st>>>(R, nrec_chunk, rec_begin, n_rec_total, plan, (const cplx<float> *)tw,
                                    (const cplx<float> *)Zg, scale, win, (cplx<float> *)series, nqb, CT,
                                    scr_c);
    }
    return cudaGetLastError();
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
    const int threads = fixed_plan(plan) ? fft_threads((int)grid_work(G, ng), 16)
                                         : std::min(fft_threads((int)grid_work(G, ng), 8),
                                                    smem <= kTwoBlockSmem ? 512 : kRuntimeThreads);
    dim3 grid(((nrec_chunk + 1) / 2) * (3 / ng), W);
    if (precision == 0) {
        GridKernelD k = pick_kernel<double>(plan);
        allow_dynamic_smem(k);
        k<<<grid, threads, smem, st>>>((const double *)snap, N, R, nrec_chunk, rec_begin, n_rec_total,
                                       grid_map, plan, (const cplx<double> *)tw, scale, win,
                                       (cplx<double> *)series, nqb, ng, grid_scratch_seqs(G, ng, plan));
    } else {
        GridKernelF k = pick_kernel<float>(plan);
        allow_dynamic_smem(k);
        k<<<grid, threads, smem, st>>>((const float *)snap, N, R, nrec_chunk, rec_begin, n_rec_total,
                                       grid_map, plan, (const cplx<float> *)tw, scale, win,
                                       (cplx<float> *)series, nqb, ng, grid_scratch_seqs(G, ng, plan));
    }
    return cudaGetLastError();
}

}  // namespace smd
