// fft_kernels.cu -- the time transform
// |S(q,w)|^2 accumulated over samples.
//
// The list-q projections are in proj_f64.cu (FP64, DMMA) and proj_tc.cu
// (FP32 form, tcgen05); the grid q in grid_proj.cu.
//
// Time transform (Codes_Folder/subrouts.cpp:12062-12109): x[t] = w[t] S(q,t)
// (the projections store the window-weighted series), forward FFT of length
// n_rec, |X|^2 / n_rec.  A block owns consecutive q of one component, loops
// over every sample of the wave and keeps the sum over samples in
// registers, so the accumulation needs no atomics and is deterministic.
#include <cuda.h>

#include "fft_device.cuh"

#include <cstdlib>

namespace smd {

// ---------------------------------------------------------- time transform

// Generic lengths.  blockIdx.x = c * ntile + q-tile of QT sequences (QT a
// multiple of the q block).  The series is already windowed.  Sums over the
// W samples of the wave into acc[c][q][n_rec] (added to what acc holds).
template <typename T, int FL>
__global__ void __launch_bounds__(1024) time_fft_kernel(
    const cplx<T> *__restrict__ series, int W, int Q, int nqb, int QT, FFTPlan plan,
    const cplx<T> *__restrict__ tw_g, double *__restrict__ acc, int use_scratch)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int QB = series_qb<T>();
    const int n = plan.n;
    const int ntile = (nqb * QB + QT - 1) / QT;
    const int c = blockIdx.x / ntile, qb0 = (blockIdx.x % ntile) * (QT / QB);
    const int nblk = min(QT / QB, nqb - qb0);
    cplx<T> *buf = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *scratch = use_scratch ? buf + (size_t)QT * n : nullptr;
    constexpr int MAXA = 8;
    double a[MAXA];
#pragma unroll
    for (int u = 0; u < MAXA; u++) a[u] = 0.0;
    const int total = nblk * QB * n;
    const double inv_n = 1.0 / n;
    for (int s = 0; s < W; s++) {
        // the tile's q blocks are one contiguous run: [block][t][QB]
        const cplx<T> *src = series + (((size_t)s * 3 + c) * nqb + qb0) * n * QB;
        for (int e = threadIdx.x; e < total; e += blockDim.x) {
            const int qi = e % QB, t = (e / QB) % n, b = e / (QB * n);
            buf[(b * QB + qi) * n + t] = src[e];
        }
        __syncthreads();
        smem_fft<T, MAXA, FL>(buf, n, QT, n, 1, plan.radix, plan.nst, tw_g, scratch, QT);
#pragma unroll
        for (int u = 0; u < MAXA; u++) {
            const int e = threadIdx.x + u * blockDim.x;
            if (e < total) {
                const double x = (double)buf[e].x, y = (double)buf[e].y;
                a[u] += (x * x + y * y) * inv_n;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < MAXA; u++) {
        const int e = threadIdx.x + u * blockDim.x;
        const int q = qb0 * QB + e / n;
        if (e < total && q < Q) acc[((size_t)c * Q + q) * n + e % n] += a[u];
    }
}

// ---- power-of-two lengths 16 .. 4096: register radix-16 passes
//
// Every thread owns 16 values in each pass: one radix-16 butterfly, or 16/R
// butterflies of the closing radix R in {2, 4, 8} (n = 16^a R).  A pass is
// the Stockham stage of stockham_stage.  The first pass reads the staging
// tile S that one bulk copy filled ([block][t][QB], as in the series) and
// writes the work buffer Wb; each later pass reads and writes Wb in place;
// the last keeps its outputs X[j + r n/R] in registers and adds |X|^2 / n to
// the thread's accumulators.  Wb holds sequence qq at Wb[qq * PS + phys(i)]:
// rows of 16 values whose 16-byte chunks are XOR-swizzled by the row index,
// so the first pass's 16 consecutive values per thread (vector stores) and
// the later passes' runs of consecutive values both spread over all banks;
// FP32 sequences sit 64 bytes apart in bank terms (PS = n + 8) because the
// first pass interleaves the two sequences of a q block across threads.

template <typename T>
__device__ __forceinline__ int p2_phys(int i)
{
    if constexpr (sizeof(T) == 4)   // two values per 16-byte chunk
        return (i & ~15) | ((((i >> 1) & 7) ^ ((i >> 4) & 7)) << 1) | (i & 1);
    else                            // one value per chunk
        return (i & ~15) | ((i & 15) ^ ((i >> 4) & 7));
}

// Twiddles of a pass with Ns > 1: ts[q Ns + k] = w^(2^q k tstep), q < log2 R
// (built once per block, so a warp's loads hit consecutive k); the other
// powers are products of those.
template <typename T, int R>
__device__ __forceinline__ void p2_twiddle(cplx<T> *v, const cplx<T> *ts, int Ns, int k)
{
    cplx<T> w[16];
    w[1] = ts[k];
    if constexpr (R >= 4) {
        w[2] = ts[Ns + k];
        w[3] = cmul(w[1], w[2]);
    }
    if constexpr (R >= 8) {
        w[4] = ts[2 * Ns + k];
#pragma unroll
        for (int r = 5; r < 8; r++) w[r] = cmul(w[r - 4], w[4]);
    }
    if constexpr (R >= 16) {
        w[8] = ts[3 * Ns + k];
#pragma unroll
        for (int r = 9; r < 16; r++) w[r] = cmul(w[r - 8], w[8]);
    }
#pragma unroll
    for (int r = 1; r < R; r++) v[r] = cmul(v[r], w[r]);
}

// loads of a pass over Wb (not the first pass)
template <typename T, int R>
__device__ __forceinline__ void p2_load(cplx<T> (&v)[16], const cplx<T> *Wb, int n, int PS)
{
    const int m = n / R;
#pragma unroll
    for (int u = 0; u < 16 / R; u++) {
        const int beta = threadIdx.x + u * blockDim.x;
        const int j = beta % m, qq = beta / m;
        const cplx<T> *src = Wb + (size_t)qq * PS;
#pragma unroll
        for (int r = 0; r < R; r++) v[u * R + r] = src[p2_phys<T>(j + r * m)];
    }
}

// twiddles and butterflies of a pass with Ns > 1 (ts: the pass's table)
template <typename T, int R>
__device__ __forceinline__ void p2_compute(cplx<T> (&v)[16], const cplx<T> *ts, int n, int Ns)
{
    const int m = n / R;
#pragma unroll
    for (int u = 0; u < 16 / R; u++) {
        const int beta = threadIdx.x + u * blockDim.x;
        const int k = (beta % m) % Ns;
        cplx<T> *x = v + u * R;
        p2_twiddle<T, R>(x, ts, Ns, k);
        cplx<T> y[R];
#pragma unroll
        for (int r = 0; r < R; r++) y[r] = x[r];
        dft_small<T, R>(y, ts, n);   // radix 2..16: no table lookups
#pragma unroll
        for (int r = 0; r < R; r++) x[r] = y[r];
    }
}

// stores of a middle pass (Ns >= 16, so consecutive threads write
// consecutive positions)
template <typename T, int R>
__device__ __forceinline__ void p2_store(const cplx<T> (&v)[16], cplx<T> *Wb, int n, int PS, int Ns)
{
    const int m = n / R;
#pragma unroll
    for (int u = 0; u < 16 / R; u++) {
        const int beta = threadIdx.x + u * blockDim.x;
        const int j = beta % m, qq = beta / m, k = j % Ns;
        const int idx = (j / Ns) * Ns * R + k;
        cplx<T> *dst = Wb + (size_t)qq * PS;
#pragma unroll
        for (int r = 0; r < R; r++) dst[p2_phys<T>(idx + r * Ns)] = v[u * R + r];
    }
}

// |X|^2 / n of the last pass into the accumulators
template <typename T, int R>
__device__ __forceinline__ void p2_accumulate(const cplx<T> (&v)[16], T (&a)[16], T inv_n)
{
#pragma unroll
    for (int e = 0; e < 16; e++) a[e] += (v[e].x * v[e].x + v[e].y * v[e].y) * inv_n;
}

// acc[c][q][f] += a for the outputs f = j + r n/R of the last pass
template <typename T, int R>
__device__ __forceinline__ void p2_flush(const T (&a)[16], double *acc, int c, int Q, int q0, int n)
{
    const int m = n / R;
#pragma unroll
    for (int u = 0; u < 16 / R; u++) {
        const int beta = threadIdx.x + u * blockDim.x;
        const int j = beta % m, q = q0 + beta / m;
        if (q < Q) {
            double *dst = acc + ((size_t)c * Q + q) * n;
#pragma unroll
            for (int r = 0; r < R; r++) dst[j + r * m] += (double)a[u * R + r];
        }
    }
}

// Last pass (radix R, reads Wb): loads, twiddles, butterflies, accumulate.
template <typename T, int R>
__device__ __forceinline__ void p2_last(cplx<T> (&v)[16], T (&a)[16], const cplx<T> *Wb,
                                        const cplx<T> *ts, int n, int PS, int Ns, T inv_n)
{
    p2_load<T, R>(v, Wb, n, PS);
    p2_compute<T, R>(v, ts, n, Ns);
    p2_accumulate<T, R>(v, a, inv_n);
}

// entries of the per-pass twiddle tables for n = 2^log2n
__host__ __device__ inline int p2_table_size(int log2n)
{
    const int n16 = log2n >> 2, lr = log2n & 3;
    int size = 0, Ns = 16;
    for (int st = 1; st < n16; st++, Ns *= 16) size += 4 * Ns;
    if (lr) size += lr * Ns;
    return size;
}

// blockIdx.x = c * ntile + tile; a tile is nseq / QB consecutive q blocks
// (nseq sequences); blockDim.x = nseq * n / 16.  One bulk copy per sample
// brings the tile; the copy of sample s + 1 is issued as soon as the first
// pass of sample s has read S, so it overlaps the remaining passes.  The
// wait on the copy is bounded by poll_limit polls: on expiry thread 0
// records bit 8 in *status, the block stops, and the copy in flight is
// waited for (with the fixed limit kDrainPolls) before the block exits.
constexpr unsigned kDrainPolls = 1u << 26;   // about a second of polling

// INPLACE (the FP32 form): one tile buffer that the passes also work in
// (the copy lands in natural order, the first pass reads it all before
// writing the swizzled layout back), 64 registers a thread, so two blocks
// share an SM and one block's copy overlaps the other's passes; the copy of
// sample s + 1 is issued once the last pass of sample s has read the buffer.
// Otherwise a tile buffer and a work buffer, one block per SM, and the copy
// of sample s + 1 issued after the first pass of sample s.
template <typename T, bool INPLACE>
__global__ void __launch_bounds__(sizeof(T) == 8 ? 256 : 512, INPLACE ? 2 : 1) time_fft_pow2_kernel(
    const cplx<T> *__restrict__ series, int W, int Q, int nqb, int n, int log2n, int nseq,
    const cplx<T> *__restrict__ tw_g, double *__restrict__ acc, int *status, unsigned poll_limit)
{
    constexpr int QB = series_qb<T>();
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int ntile = (nqb * QB + nseq - 1) / nseq;
    const int c = blockIdx.x / ntile, tile = blockIdx.x % ntile;
    const int qb0 = tile * (nseq / QB);
    const int nblk = min(nseq / QB, nqb - qb0);
    const int PS = n + (QB == 2 ? 8 : 0);
    const int n16 = log2n >> 2, rl = 1 << (log2n & 3);
    cplx<T> *S = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *Wb = INPLACE ? S : S + (size_t)nseq * n;
    cplx<T> *ts = Wb + (size_t)nseq * PS;
    uint64_t *bar = reinterpret_cast<uint64_t *>(ts + p2_table_size(log2n));
    __shared__ int abort_flag;
    const uint32_t bar_a = (uint32_t)__cvta_generic_to_shared(bar);
    const uint32_t S_a = (uint32_t)__cvta_generic_to_shared(S);
    const unsigned bytes = (unsigned)((size_t)nblk * n * 16);
    auto issue = [&](int s) {
        const cplx<T> *src = series + (((size_t)s * 3 + c) * nqb + qb0) * n * QB;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(bytes)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(S_a),
            "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(bar_a)
            : "memory");
    };
    auto try_wait = [&](unsigned parity) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar_a), "r"(parity)
            : "memory");
        return done != 0;
    };
    if (threadIdx.x == 0) {
        abort_flag = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        issue(0);
    }
    {
        // per-pass twiddle tables, passes 2 .. nst in order
        cplx<T> *t = ts;
        int Ns = 16;
        for (int st = 1; st <= n16; st++, Ns *= 16) {
            const int R = st < n16 ? 16 : rl;
            if (R == 1) break;
            int nq = 0;
            while ((1 << nq) < R) nq++;
            const int tstep = n / (Ns * R);
            for (int e = threadIdx.x; e < nq * Ns; e += blockDim.x) {
                const int q = e / Ns, k = e - q * Ns;
                t[e] = tw_g[(1 << q) * k * tstep];
            }
            t += nq * Ns;
        }
    }
    const int nst = n16 + (rl > 1 ? 1 : 0);
    const T inv_n = T(1) / T(n);
    T a[16];
#pragma unroll
    for (int e = 0; e < 16; e++) a[e] = T(0);
    cplx<T> v[16];
    int s_abort = 0;
    for (int s = 0; s < W; s++) {
        // thread 0 waits (bounded) and tells the block; the others then
        // observe the completed phase themselves
        if (threadIdx.x == 0) {
            bool done = false;
            for (unsigned it = 0; it < poll_limit && !done; it++) done = try_wait(s & 1);
            if (!done) {
                atomicOr(status, 8);
                abort_flag = 1;
            }
        }
        __syncthreads();
        if (abort_flag) {
            s_abort = s;
            break;
        }
        for (int it = 0; it < (1 << 20) && !try_wait(s & 1); it++) {
        }
        // first pass: radix 16, Ns = 1, reads S
        {
            const int m = n / 16;
            const int qi = threadIdx.x % QB, j = (threadIdx.x / QB) % m, blk = threadIdx.x / (QB * m);
            const cplx<T> *src = S + ((size_t)blk * n + j) * QB + qi;
#pragma unroll
            for (int r = 0; r < 16; r++) v[r] = src[(size_t)r * m * QB];
        }
        __syncthreads();   // S consumed; Wb free (the previous sample's last pass has read it)
        if ((!INPLACE || nst == 1) && threadIdx.x == 0 && s + 1 < W) issue(s + 1);
        dft_small<T, 16>(v, ts, n);   // no table lookups at radix 16
        if (nst == 1) {
            p2_accumulate<T, 16>(v, a, inv_n);
            continue;
        }
        {
            const int m = n / 16;
            const int qi = threadIdx.x % QB, j = (threadIdx.x / QB) % m, blk = threadIdx.x / (QB * m);
            // row j of the swizzled layout: chunk c of the row at c ^ (j & 7)
            cplx<T> *dst = Wb + (size_t)(blk * QB + qi) * PS + 16 * j;
            const int sw = j & 7;
            if constexpr (QB == 2) {
#pragma unroll
                for (int r = 0; r < 16; r += 2)
                    *reinterpret_cast<float4 *>(dst + 2 * ((r >> 1) ^ sw)) = make_float4(
                        (float)v[r].x, (float)v[r].y, (float)v[r + 1].x, (float)v[r + 1].y);
            } else {
#pragma unroll
                for (int r = 0; r < 16; r++)
                    *reinterpret_cast<double2 *>(dst + (r ^ sw)) = make_double2((double)v[r].x, (double)v[r].y);
            }
        }
        __syncthreads();
        int Ns = 16;
        const cplx<T> *tp = ts;   // this pass's twiddle table
        for (int st = 1; st < n16; st++, tp += 4 * Ns, Ns *= 16) {
            if (st == nst - 1) {
                p2_last<T, 16>(v, a, Wb, tp, n, PS, Ns, inv_n);
            } else {
                p2_load<T, 16>(v, Wb, n, PS);
                __syncthreads();
                p2_compute<T, 16>(v, tp, n, Ns);
                p2_store<T, 16>(v, Wb, n, PS, Ns);
                __syncthreads();
            }
        }
        if (rl == 2) p2_last<T, 2>(v, a, Wb, tp, n, PS, Ns, inv_n);
        else if (rl == 4) p2_last<T, 4>(v, a, Wb, tp, n, PS, Ns, inv_n);
        else if (rl == 8) p2_last<T, 8>(v, a, Wb, tp, n, PS, Ns, inv_n);
        if constexpr (INPLACE) {
            __syncthreads();   // the last pass has read the buffer
            if (threadIdx.x == 0 && s + 1 < W) issue(s + 1);
        }
    }
    if (abort_flag) {
        // the copy in flight (sample s_abort) lands before the block exits
        if (threadIdx.x == 0)
            for (unsigned it = 0; it < kDrainPolls && !try_wait(s_abort & 1); it++) {
            }
        return;
    }
    const int q0 = qb0 * QB;
    if (rl == 1) p2_flush<T, 16>(a, acc, c, Q, q0, n);
    else if (rl == 2) p2_flush<T, 2>(a, acc, c, Q, q0, n);
    else if (rl == 4) p2_flush<T, 4>(a, acc, c, Q, q0, n);
    else p2_flush<T, 8>(a, acc, c, Q, q0, n);
}

// ---------------------------------------------------------- small helpers

// AoS [W][N][3] -> SoA [W][3][N]
__global__ void aos_to_soa_kernel(const double *__restrict__ in, double *__restrict__ out, int W,
                                  int N)
{
    const size_t total = (size_t)W * N * 3;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.x * blockDim.x) {
        const size_t s = e / (3 * (size_t)N);
        const size_t r = e - s * 3 * N;
        const size_t i = r / 3, c = r % 3;
        out[(s * 3 + c) * N + i] = in[e];
    }
}

__global__ void soa_to_aos_kernel(const double *__restrict__ in, double *__restrict__ out, int W,
                                  int N)
{
    const size_t total = (size_t)W * N * 3;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.x * blockDim.x) {
        const size_t s = e / (3 * (size_t)N);
        const size_t r = e - s * 3 * N;
        const size_t i = r / 3, c = r % 3;
        out[e] = in[(s * 3 + c) * N + i];
    }
}

// p[e] *= f
__global__ void scale_kernel(double *__restrict__ p, size_t n, double f)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x)
        p[e] *= f;
}

// out[t] += sum_s rows[s][t]
__global__ void sum_rows_kernel(const double *__restrict__ rows, int W, int n,
                                double *__restrict__ out)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < W; w++) s += rows[(size_t)w * n + t];
        out[t] += s;
    }
}

// ---------------------------------------------------------- launchers

// time kernel instance of a stage set (plans of make_plan carry no radix 16 or 8)
template <typename T>
static auto time_kernel(int fl)
{
    if (fl & FK_R5) return time_fft_kernel<T, FK_R3 | FK_R5>;
    switch (fl & (FK_R3 | FK_GEN)) {
    case 0: return time_fft_kernel<T, 0>;
    case FK_R3: return time_fft_kernel<T, FK_R3>;
    case FK_GEN: return time_fft_kernel<T, FK_GEN>;
    default: return time_fft_kernel<T, FK_R3 | FK_GEN>;
    }
}

int series_qblock(int precision) { return precision == 0 ? series_qb<double>() : series_qb<float>(); }

// power-of-two lengths the register-pass transform takes: 16 .. 4096
static int pow2_log2(int n)
{
    if (n < 16 || n > 4096 || (n & (n - 1))) return -1;
    int l = 0;
    while ((1 << l) < n) l++;
    return l;
}

// sequences per block of the register-pass transform: nseq * n = 8192
// values in FP32, 4096 in FP64, at least one q block, at most the q range
static int pow2_nseq(int n, int precision, int Q)
{
    const int qb = series_qblock(precision);
    const int elems = precision == 0 ? 4096 : 8192;
    int nseq = elems / n;
    const int qcap = (Q + qb - 1) / qb * qb;
    if (nseq > qcap) nseq = qcap;
    return nseq < qb ? qb : nseq / qb * qb;
}

// the FP32 form's kernel works in its tile buffer (INPLACE), the FP64 one
// has a tile buffer and a work buffer
static size_t pow2_smem(int n, int nseq, int precision)
{
    const size_t e = precision == 0 ? sizeof(cplx<double>) : sizeof(cplx<float>);
    const int qb = series_qblock(precision);
    const size_t ps = (size_t)n + (qb == 2 ? 8 : 0);
    const size_t tile = precision == 0 ? (size_t)nseq * n : 0;
    return (tile + (size_t)nseq * ps + p2_table_size(pow2_log2(n))) * e + 16;
}

// sequences per block of the generic transform: a multiple of the q block,
// at most 8192 values (8 per thread of a 1024-thread block)
int time_fft_qt(int n, int precision)
{
    const size_t e = precision == 0 ? sizeof(cplx<double>) : sizeof(cplx<float>);
    const int qb = series_qblock(precision);
    int qt = qb;
    while (qt < 64 && (size_t)(qt * 2) * n * e <= 72 * 1024 && qt * 2 * n <= 8192) qt *= 2;
    return qt;
}

size_t time_fft_smem(int n, int qt, int precision, const FFTPlan &p)
{
    if (pow2_log2(n) >= 0) return pow2_smem(n, pow2_nseq(n, precision, 1 << 30), precision);
    const size_t e = precision == 0 ? sizeof(cplx<double>) : sizeof(cplx<float>);
    size_t b = (size_t)qt * n * e;
    if (plan_generic(p)) b *= 2;
    return b;
}

bool time_fft_fits(int n, int precision, const FFTPlan &p)
{
    if (pow2_log2(n) >= 0) return true;
    const int qt = time_fft_qt(n, precision);
    return (size_t)qt * n <= 8192 && time_fft_smem(n, qt, precision, p) <= 200 * 1024;
}

cudaError_t launch_time_fft(const void *series, int precision, int W, int Q, int nqb,
                            const FFTPlan &plan, const void *tw, double *acc, int *status,
                            cudaStream_t st, int ncomp)
{
    const int n = plan.n;
    const int qb = series_qblock(precision);
    const int l2 = pow2_log2(n);
    if (l2 >= 0) {
        // polls of the bounded copy wait (SMD_TFFT_POLL_LIMIT overrides the
        // default; a test sets 0 to make the wait expire)
        unsigned polls = kDrainPolls;
        if (const char *e = std::getenv("SMD_TFFT_POLL_LIMIT")) polls = (unsigned)std::strtoul(e, nullptr, 10);
        const int nseq = pow2_nseq(n, precision, Q);
        const size_t smem = pow2_smem(n, nseq, precision);
        const int threads = nseq * n / 16;
        const int ntile = (nqb * qb + nseq - 1) / nseq;
        if (precision == 0) {
            auto k = time_fft_pow2_kernel<double, false>;
            allow_dynamic_smem(k);
            k<<<ncomp * ntile, threads, smem, st>>>((const cplx<double> *)series, W, Q, nqb, n, l2, nseq,
                                                (const cplx<double> *)tw, acc, status, polls);
        } else {
            auto k = time_fft_pow2_kernel<float, true>;
            allow_dynamic_smem(k);
            k<<<ncomp * ntile, threads, smem, st>>>((const cplx<float> *)series, W, Q, nqb, n, l2, nseq,
                                                (const cplx<float> *)tw, acc, status, polls);
        }
        return cudaGetLastError();
    }
    const int qt = time_fft_qt(n, precision);
    const size_t smem = time_fft_smem(n, qt, precision, plan);
    const int threads = fft_threads(qt * n, 8);
    const int ntile = (nqb * qb + qt - 1) / qt;
    const int fl = fft_plan_flags(plan), gen = (fl & FK_GEN) ? 1 : 0;
    if (precision == 0) {
        auto k = time_kernel<double>(fl);
        allow_dynamic_smem(k);
        k<<<ncomp * ntile, threads, smem, st>>>((const cplx<double> *)series, W, Q, nqb, qt, plan,
                                            (const cplx<double> *)tw, acc, gen);
    } else {
        auto k = time_kernel<float>(fl);
        allow_dynamic_smem(k);
        k<<<ncomp * ntile, threads, smem, st>>>((const cplx<float> *)series, W, Q, nqb, qt, plan,
                                            (const cplx<float> *)tw, acc, gen);
    }
    return cudaGetLastError();
}

cudaError_t launch_aos_to_soa(const double *in, double *out, int W, int N, cudaStream_t st)
{
    aos_to_soa_kernel<<<592, 256, 0, st>>>(in, out, W, N);
    return cudaGetLastError();
}

cudaError_t launch_soa_to_aos(const double *in, double *out, int W, int N, cudaStream_t st)
{
    soa_to_aos_kernel<<<592, 256, 0, st>>>(in, out, W, N);
    return cudaGetLastError();
}

cudaError_t launch_scale(double *p, size_t n, double f, cudaStream_t st)
{
    scale_kernel<<<1184, 256, 0, st>>>(p, n, f);
    return cudaGetLastError();
}

cudaError_t launch_sum_rows(const double *rows, int W, int n, double *out, cudaStream_t st)
{
    sum_rows_kernel<<<(n + 255) / 256, 256, 0, st>>>(rows, W, n, out);
    return cudaGetLastError();
}

}  // namespace smd
