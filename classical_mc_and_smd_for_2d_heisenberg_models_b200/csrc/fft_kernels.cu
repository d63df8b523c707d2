// fft_kernels.cu -- spatial projection S(q,t) and the windowed time
// transform |S(q,w)|^2 accumulated over samples.
//
// Grid q (get_SqData_iMKL, Codes_Folder/subrouts.cpp:8330-8432): each record's
// spins are embedded into the G x G DFT grid through gridMap (empty grid
// points are zero), transformed by a forward 2D DFT (sign -1, unscaled) and
// scaled by sqrt(1 / G^2).  One CTA transforms one (sample, record,
// component) grid in shared memory: G row transforms, then G column
// transforms, each a mixed-radix Stockham FFT (radices 4, 2, 3, 5, and any
// other prime directly).
//
// List q (get_qct_SqData, Codes_Folder/subrouts.cpp:8460-8525): S(q_l) =
// scale sum_k S_k exp(-i q_l . pos_k), a dense contraction of the snapshot
// rows with a phase table; the FP64 form runs it as a tiled SIMT GEMM.
//
// Time transform (Codes_Folder/subrouts.cpp:12062-12109): x[t] = w[t] S(q,t),
// forward FFT of length n_rec, |X|^2 / n_rec.  One CTA owns QT consecutive q
// of one component, loops over every sample of the wave and keeps the sum
// over samples in registers, so the accumulation needs no atomics and is
// deterministic.
#include <cuda.h>

#include "smd_device.cuh"

namespace smd {

template <typename T>
__device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b)
{
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}

template <typename T>
__device__ __forceinline__ cplx<T> cadd(cplx<T> a, cplx<T> b) { return {a.x + b.x, a.y + b.y}; }

template <typename T>
__device__ __forceinline__ cplx<T> csub(cplx<T> a, cplx<T> b) { return {a.x - b.x, a.y - b.y}; }

// Radix-4 DFT (sign -1) of (a, b, c, d) in place: X0..X3 in a..d.
template <typename T>
__device__ __forceinline__ void dft4(cplx<T> &a, cplx<T> &b, cplx<T> &c, cplx<T> &d)
{
    const cplx<T> s0 = cadd(a, c), s1 = csub(a, c), s2 = cadd(b, d), s3 = csub(b, d);
    // -i * s3 = (s3.y, -s3.x)
    a = cadd(s0, s2);
    c = csub(s0, s2);
    b = {s1.x + s3.y, s1.y - s3.x};
    d = {s1.x - s3.y, s1.y + s3.x};
}

// In-register forward DFT of radix R (sign -1).  For R outside
// {2, 3, 4, 8, 16} the twiddle table of the full length n
// (tw[j] = exp(-2 pi i j / n)) gives the R-th roots.
template <typename T, int R>
__device__ __forceinline__ void dft_small(cplx<T> (&v)[R], const cplx<T> *tw, int n)
{
    if constexpr (R == 2) {
        cplx<T> a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        cplx<T> a = v[0], b = v[1], c = v[2], d = v[3];
        cplx<T> s0 = cadd(a, c), s1 = csub(a, c), s2 = cadd(b, d), s3 = csub(b, d);
        // -i * s3 = (s3.y, -s3.x)
        v[0] = cadd(s0, s2);
        v[2] = csub(s0, s2);
        v[1] = {s1.x + s3.y, s1.y - s3.x};
        v[3] = {s1.x - s3.y, s1.y + s3.x};
    } else if constexpr (R == 3) {
        const T h = T(0.86602540378443864676);   // sqrt(3)/2
        cplx<T> a = v[0], b = v[1], c = v[2];
        cplx<T> s = cadd(b, c), d = csub(b, c);
        cplx<T> m = {a.x - T(0.5) * s.x, a.y - T(0.5) * s.y};
        // -i h d = (h d.y, -h d.x)
        v[0] = cadd(a, s);
        v[1] = {m.x + h * d.y, m.y - h * d.x};
        v[2] = {m.x - h * d.y, m.y + h * d.x};
    } else if constexpr (R == 8) {
        // 8 = 2 x 4: radix-4 over r1 (r = r0 + 2 r1), twiddle w8^(r0 p0),
        // radix-2 over r0; X[p0 + 4 p1] lands in v[2 p0 + p1]
        const T h = T(0.70710678118654752440);   // sqrt(1/2)
#pragma unroll
        for (int r0 = 0; r0 < 2; r0++) dft4(v[r0], v[r0 + 2], v[r0 + 4], v[r0 + 6]);
        v[3] = {h * (v[3].x + v[3].y), h * (v[3].y - v[3].x)};    // w8^1
        v[5] = {v[5].y, -v[5].x};                                 // w8^2 = -i
        v[7] = {h * (v[7].y - v[7].x), -h * (v[7].x + v[7].y)};   // w8^3
        cplx<T> u[8];
#pragma unroll
        for (int p0 = 0; p0 < 4; p0++) {
            u[p0] = cadd(v[2 * p0], v[2 * p0 + 1]);
            u[p0 + 4] = csub(v[2 * p0], v[2 * p0 + 1]);
        }
#pragma unroll
        for (int p = 0; p < 8; p++) v[p] = u[p];
    } else if constexpr (R == 16) {
        // 16 = 4 x 4: radix-4 over r1 (r = r0 + 4 r1), twiddle w16^(r0 p0),
        // radix-4 over r0; X[p0 + 4 p1] lands in v[4 p0 + p1]
        const T h = T(0.70710678118654752440);    // sqrt(1/2)
        const T c1 = T(0.92387953251128675613);   // cos(pi/8)
        const T s1 = T(0.38268343236508977173);   // sin(pi/8)
#pragma unroll
        for (int r0 = 0; r0 < 4; r0++) dft4(v[r0], v[r0 + 4], v[r0 + 8], v[r0 + 12]);
        // y[r0][p0] sits in v[r0 + 4 p0]
        v[5] = cmul(v[5], cplx<T>{c1, -s1});                          // w16^1
        v[9] = {h * (v[9].x + v[9].y), h * (v[9].y - v[9].x)};        // w16^2
        v[13] = cmul(v[13], cplx<T>{s1, -c1});                        // w16^3
        v[6] = {h * (v[6].x + v[6].y), h * (v[6].y - v[6].x)};        // w16^2
        v[10] = {v[10].y, -v[10].x};                                  // w16^4 = -i
        v[14] = {h * (v[14].y - v[14].x), -h * (v[14].x + v[14].y)};  // w16^6
        v[7] = cmul(v[7], cplx<T>{s1, -c1});                          // w16^3
        v[11] = {h * (v[11].y - v[11].x), -h * (v[11].x + v[11].y)};  // w16^6
        v[15] = cmul(v[15], cplx<T>{-c1, s1});                        // w16^9
#pragma unroll
        for (int p0 = 0; p0 < 4; p0++) dft4(v[4 * p0], v[4 * p0 + 1], v[4 * p0 + 2], v[4 * p0 + 3]);
        // v[4 p0 + p1] = X[p0 + 4 p1]; reorder to natural order
        cplx<T> u[16];
#pragma unroll
        for (int p0 = 0; p0 < 4; p0++)
#pragma unroll
            for (int p1 = 0; p1 < 4; p1++) u[p0 + 4 * p1] = v[4 * p0 + p1];
#pragma unroll
        for (int p = 0; p < 16; p++) v[p] = u[p];
    } else {
        cplx<T> u[R];
#pragma unroll
        for (int p = 0; p < R; p++) {
            cplx<T> s = v[0];
#pragma unroll
            for (int q = 1; q < R; q++) {
                const cplx<T> w = tw[((q * p) % R) * (n / R)];
                s = cadd(s, cmul(v[q], w));
            }
            u[p] = s;
        }
#pragma unroll
        for (int p = 0; p < R; p++) v[p] = u[p];
    }
}

// One Stockham stage of radix R over nseq sequences of length n held in
// shared memory: element x of sequence q sits at buf[q * ss + x * es].
// Every thread first loads all of its butterflies, then (after a barrier)
// writes them, so the stage runs in place.  NB = butterflies per thread.
template <typename T, int R, int NB>
__device__ __forceinline__ void stockham_stage(cplx<T> *buf, int n, int nseq, int ss, int es,
                                               int Ns, const cplx<T> *tw)
{
    const int m = n / R, nb = nseq * m;
    // Consecutive threads take consecutive elements: along a sequence when
    // its elements are adjacent (es == 1), across sequences otherwise, so
    // shared-memory accesses stay free of bank conflicts.
    const bool qfast = es != 1;
    cplx<T> v[NB][R];
#pragma unroll
    for (int u = 0; u < NB; u++) {
        const int b = threadIdx.x + u * blockDim.x;
        if (b < nb) {
            const int q = qfast ? b % nseq : b / m;
            const int j = qfast ? b / nseq : b - q * m;
#pragma unroll
            for (int r = 0; r < R; r++) v[u][r] = buf[q * ss + (j + r * m) * es];
        }
    }
    __syncthreads();
    const int tstep = n / (Ns * R);
#pragma unroll
    for (int u = 0; u < NB; u++) {
        const int b = threadIdx.x + u * blockDim.x;
        if (b < nb) {
            const int q = qfast ? b % nseq : b / m;
            const int j = qfast ? b / nseq : b - q * m;
            const int k = j % Ns;
#pragma unroll
            for (int r = 1; r < R; r++) v[u][r] = cmul(v[u][r], tw[(r * k) * tstep]);   // index < n
            dft_small<T, R>(v[u], tw, n);
            const int idx = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; r++) buf[q * ss + (idx + r * Ns) * es] = v[u][r];
        }
    }
    __syncthreads();
}

// Any other radix: one butterfly at a time, streaming from a copy of the
// sequences.  Kept out of line so that its register needs stay apart from
// the radix-4 / radix-2 path; thread mapping as in stockham_stage.
template <typename T>
__device__ __noinline__ void stockham_stage_generic(cplx<T> *buf, int n, int nseq, int ss, int es,
                                                    int Ns, int R, const cplx<T> *tw,
                                                    cplx<T> *scratch)
{
    // scratch: a copy of the sequences (same layout), so loads and stores
    // touch different arrays
    const bool qfast = es != 1;
    const int total = nseq * n;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int q = qfast ? e % nseq : e / n;
        const int x = qfast ? e / nseq : e - q * n;
        scratch[q * ss + x * es] = buf[q * ss + x * es];
    }
    __syncthreads();
    const int m = n / R, nb = nseq * m, tstep = n / (Ns * R);
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const int q = qfast ? b % nseq : b / m;
        const int j = qfast ? b / nseq : b - q * m;
        const int k = j % Ns;
        const int idx = (j / Ns) * Ns * R + k;
        for (int p = 0; p < R; p++) {
            cplx<T> s = {T(0), T(0)};
            for (int r = 0; r < R; r++) {
                cplx<T> x = scratch[q * ss + (j + r * m) * es];
                if (r) x = cmul(x, tw[(r * k) * tstep]);   // index < n
                s = cadd(s, cmul(x, tw[((r * p) % R) * (n / R)]));
            }
            buf[q * ss + (idx + p * Ns) * es] = s;
        }
    }
    __syncthreads();
}

// Full transform.  C = values each thread holds in registers during a
// stage (8 keeps a 1024-thread CTA within 64 registers per thread; 16 only
// for the largest grids).  Radices come from the host plan (product = n);
// every stage needs nseq * n <= C * blockDim.x.  KIND selects the stages a
// kernel is built with, so that each plan pays only for the stages it uses:
//   KIND 0: radix 4 and 2 inline (plans of radices 2 and 4);
//   KIND 1: radix 4, 2 and 3 inline (plans of radices 2, 3 and 4);
//   KIND 2: radix 4 and 2 inline, any other radix through the out-of-line
//           streaming stage, whose register needs stay apart from the rest.
template <typename T, int C, int KIND>
__device__ void smem_fft(cplx<T> *buf, int n, int nseq, int ss, int es, const int *radix,
                         int nst, const cplx<T> *tw, cplx<T> *scratch)
{
    int Ns = 1;
    for (int s = 0; s < nst; s++) {
        const int R = radix[s];
        switch (R) {
        case 4: stockham_stage<T, 4, (C + 3) / 4>(buf, n, nseq, ss, es, Ns, tw); break;
        case 2: stockham_stage<T, 2, (C + 1) / 2>(buf, n, nseq, ss, es, Ns, tw); break;
        default:
            if (KIND == 1) stockham_stage<T, 3, (C + 2) / 3>(buf, n, nseq, ss, es, Ns, tw);
            if (KIND == 2) stockham_stage_generic<T>(buf, n, nseq, ss, es, Ns, R, tw, scratch);
            break;
        }
        Ns *= R;
    }
}

// ---------------------------------------------------------- grid projection

// grid 2D FFT of snapshot rows; blockIdx.x = (s * R + slot) * 3 + c.
// C = 8 serves grids up to 64 x 64 with at most 512 threads (128 registers
// each); C = 16 the larger ones with up to 1024 threads.
template <typename TS, typename T, int C, int KIND>
__global__ void __launch_bounds__(C <= 8 ? 512 : 1024) grid_proj_kernel(
    const TS *__restrict__ snap, int N, int R, int rec_begin, int n_rec_total,
    const int *__restrict__ grid_map, FFTPlan plan, const cplx<T> *__restrict__ tw_g,
    double scale, const double *__restrict__ win, cplx<T> *__restrict__ series, int nqb,
    int use_scratch)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int G = plan.n, GG = G * G;
    cplx<T> *buf = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *tw = buf + GG;
    cplx<T> *scratch = use_scratch ? tw + G : nullptr;
    const int row = blockIdx.x, s = blockIdx.y;
    const int c = row % 3, slot = row / 3;
    const TS *x = snap + ((size_t)s * R * 3 + row) * N;
    for (int k = threadIdx.x; k < G; k += blockDim.x) tw[k] = tw_g[k];
    for (int k = threadIdx.x; k < GG; k += blockDim.x) {
        const int idx = grid_map[k];
        buf[k] = {idx < 0 ? T(0) : T(x[idx]), T(0)};
    }
    __syncthreads();
    smem_fft<T, C, KIND>(buf, G, G, G, 1, plan.radix, plan.nst, tw, scratch);   // rows
    smem_fft<T, C, KIND>(buf, G, G, 1, G, plan.radix, plan.nst, tw, scratch);   // columns
    // windowed output, q = k: one 16-byte store per q block
    const int t = rec_begin + slot;
    constexpr int QB = series_qb<T>();
    cplx<T> *out = series + series_off<T>(s, c, 0, t, nqb, n_rec_total);
    const size_t bstride = (size_t)n_rec_total * QB;
    const T sc = T(scale * win[t]);
    for (int b = threadIdx.x; b < GG / QB; b += blockDim.x) {
        cplx<T> v[QB];
#pragma unroll
        for (int i = 0; i < QB; i++) v[i] = {sc * buf[b * QB + i].x, sc * buf[b * QB + i].y};
        if constexpr (QB == 2)
            *reinterpret_cast<float4 *>(out + b * bstride) =
                make_float4((float)v[0].x, (float)v[0].y, (float)v[QB - 1].x, (float)v[QB - 1].y);
        else
            *reinterpret_cast<double2 *>(out + b * bstride) = make_double2((double)v[0].x, (double)v[0].y);
    }
    if (GG % QB && threadIdx.x == 0) {   // a half block shared with the first list q
        const int k = GG - 1;
        out[(k / QB) * bstride + k % QB] = {sc * buf[k].x, sc * buf[k].y};
    }
}

// ---------------------------------------------------------- list projection

// Tiled SIMT GEMM: out[m][l] = sum_k A[m][k] P[k][l], A = snapshot rows
// ([rows][N]), P = phase table ([N][L] complex, scale folded in).
// 64 rows x 32 complex columns per CTA, 256 threads, 4 x 2 outputs each.
template <typename T>
__global__ void __launch_bounds__(256) list_proj_simt_kernel(
    const T *__restrict__ snap, int rows, int N, int R, int rec_begin,
    int n_rec_total, const cplx<T> *__restrict__ P, int Lq, const double *__restrict__ win,
    cplx<T> *__restrict__ series, int nqb, int qoff)
{
    constexpr int BM = 64, BL = 32, BK = 16;
    __shared__ T As[BK][BM + 1];
    __shared__ cplx<T> Ps[BK][BL];
    const int m0 = blockIdx.x * BM, l0 = blockIdx.y * BL, s = blockIdx.z;
    snap += (size_t)s * R * 3 * N;
    const int tid = threadIdx.x;
    const int tm = tid / 16, tl = tid % 16;   // 16 x 16 thread grid
    T ar[4][2][2] = {};
    for (int k0 = 0; k0 < N; k0 += BK) {
        for (int e = tid; e < BM * BK; e += 256) {
            const int mm = e / BK, kk = e % BK;
            const int m = m0 + mm, k = k0 + kk;
            As[kk][mm] = (m < rows && k < N) ? snap[(size_t)m * N + k] : T(0);
        }
        for (int e = tid; e < BK * BL; e += 256) {
            const int kk = e / BL, ll = e % BL;
            const int k = k0 + kk, l = l0 + ll;
            Ps[kk][ll] = (k < N && l < Lq) ? P[(size_t)k * Lq + l] : cplx<T>{T(0), T(0)};
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            T a[4];
            cplx<T> p[2];
#pragma unroll
            for (int u = 0; u < 4; u++) a[u] = As[kk][tm * 4 + u];
#pragma unroll
            for (int v = 0; v < 2; v++) p[v] = Ps[kk][tl * 2 + v];
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int v = 0; v < 2; v++) {
                    ar[u][v][0] = fma(a[u], p[v].x, ar[u][v][0]);
                    ar[u][v][1] = fma(a[u], p[v].y, ar[u][v][1]);
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int m = m0 + tm * 4 + u;
        if (m >= rows) continue;
        const int c = m % 3, slot = m / 3, t = rec_begin + slot;
        const T w = T(win[t]);
#pragma unroll
        for (int v = 0; v < 2; v++) {
            const int l = l0 + tl * 2 + v;
            if (l < Lq)
                series[series_off<T>(s, c, qoff + l, t, nqb, n_rec_total)] = {w * ar[u][v][0], w * ar[u][v][1]};
        }
    }
}

// ---------------------------------------------------------- time transform

// Generic lengths.  blockIdx.x = c * ntile + q-tile of QT sequences (QT a
// multiple of the q block).  The series is already windowed.  Sums over the
// W samples of the wave into acc[c][q][n_rec] (added to what acc holds).
template <typename T, int KIND>
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
        smem_fft<T, MAXA, KIND>(buf, n, QT, n, 1, plan.radix, plan.nst, tw_g, scratch);
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
// the thread's accumulators.  Wb holds sequence qq at Wb[qq * PS + phys(i)]
// with phys(i) = i + QB * (i / 16): the first pass writes 16 consecutive
// values per thread, and the padding spreads those rows over all banks.

template <typename T>
__device__ __forceinline__ int p2_phys(int i)
{
    return i + series_qb<T>() * (i >> 4);
}

// twiddles w^(r k tstep), r = 1 .. R-1, from the loads of w^(k tstep)
// x {1, 2, 4, 8} and products of those
template <typename T, int R>
__device__ __forceinline__ void p2_twiddle(cplx<T> *v, const cplx<T> *tw, int base)
{
    cplx<T> w[16];
    w[1] = tw[base];
    if constexpr (R >= 4) {
        w[2] = tw[2 * base];
        w[3] = cmul(w[1], w[2]);
    }
    if constexpr (R >= 8) {
        w[4] = tw[4 * base];
#pragma unroll
        for (int r = 5; r < 8; r++) w[r] = cmul(w[r - 4], w[4]);
    }
    if constexpr (R >= 16) {
        w[8] = tw[8 * base];
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

// twiddles and butterflies of a pass with Ns > 1
template <typename T, int R>
__device__ __forceinline__ void p2_compute(cplx<T> (&v)[16], const cplx<T> *tw, int n, int Ns)
{
    const int m = n / R, tstep = n / (Ns * R);
#pragma unroll
    for (int u = 0; u < 16 / R; u++) {
        const int beta = threadIdx.x + u * blockDim.x;
        const int k = (beta % m) % Ns;
        cplx<T> *x = v + u * R;
        p2_twiddle<T, R>(x, tw, k * tstep);
        cplx<T> y[R];
#pragma unroll
        for (int r = 0; r < R; r++) y[r] = x[r];
        dft_small<T, R>(y, tw, n);
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
                                        const cplx<T> *tw, int n, int PS, int Ns, T inv_n)
{
    p2_load<T, R>(v, Wb, n, PS);
    p2_compute<T, R>(v, tw, n, Ns);
    p2_accumulate<T, R>(v, a, inv_n);
}

// blockIdx.x = c * ntile + tile; a tile is nseq / QB consecutive q blocks
// (nseq sequences); blockDim.x = nseq * n / 16.  One bulk copy per sample
// brings the tile; the copy of sample s + 1 is issued as soon as the first
// pass of sample s has read S, so it overlaps the remaining passes.  The
// wait on the copy is bounded: on expiry thread 0 records bit 8 in *status,
// the block stops, and the copy in flight is waited for (bounded) before
// the block exits.
template <typename T>
__global__ void __launch_bounds__(sizeof(T) == 8 ? 256 : 512) time_fft_pow2_kernel(
    const cplx<T> *__restrict__ series, int W, int Q, int nqb, int n, int log2n, int nseq,
    const cplx<T> *__restrict__ tw_g, double *__restrict__ acc, int *status)
{
    constexpr int QB = series_qb<T>();
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int ntile = (nqb * QB + nseq - 1) / nseq;
    const int c = blockIdx.x / ntile, tile = blockIdx.x % ntile;
    const int qb0 = tile * (nseq / QB);
    const int nblk = min(nseq / QB, nqb - qb0);
    const int PS = p2_phys<T>(n) + (QB == 2 ? 8 : 0);
    cplx<T> *S = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *Wb = S + (size_t)nseq * n;
    cplx<T> *tw = Wb + (size_t)nseq * PS;
    uint64_t *bar = reinterpret_cast<uint64_t *>(tw + n);
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
    for (int k = threadIdx.x; k < n; k += blockDim.x) tw[k] = tw_g[k];
    const int n16 = log2n >> 2, rl = 1 << (log2n & 3);
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
            for (unsigned it = 0; it < (1u << 26) && !done; it++) done = try_wait(s & 1);
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
        if (threadIdx.x == 0 && s + 1 < W) issue(s + 1);
        dft_small<T, 16>(v, tw, n);
        if (nst == 1) {
            p2_accumulate<T, 16>(v, a, inv_n);
            continue;
        }
        {
            const int m = n / 16;
            const int qi = threadIdx.x % QB, j = (threadIdx.x / QB) % m, blk = threadIdx.x / (QB * m);
            cplx<T> *dst = Wb + (size_t)(blk * QB + qi) * PS + p2_phys<T>(16 * j);
            if constexpr (QB == 2) {
#pragma unroll
                for (int r = 0; r < 16; r += 2)
                    *reinterpret_cast<float4 *>(dst + r) = make_float4(
                        (float)v[r].x, (float)v[r].y, (float)v[r + 1].x, (float)v[r + 1].y);
            } else {
#pragma unroll
                for (int r = 0; r < 16; r++)
                    *reinterpret_cast<double2 *>(dst + r) = make_double2((double)v[r].x, (double)v[r].y);
            }
        }
        __syncthreads();
        int Ns = 16;
        for (int st = 1; st < n16; st++, Ns *= 16) {
            if (st == nst - 1) {
                p2_last<T, 16>(v, a, Wb, tw, n, PS, Ns, inv_n);
            } else {
                p2_load<T, 16>(v, Wb, n, PS);
                __syncthreads();
                p2_compute<T, 16>(v, tw, n, Ns);
                p2_store<T, 16>(v, Wb, n, PS, Ns);
                __syncthreads();
            }
        }
        if (rl == 2) p2_last<T, 2>(v, a, Wb, tw, n, PS, Ns, inv_n);
        else if (rl == 4) p2_last<T, 4>(v, a, Wb, tw, n, PS, Ns, inv_n);
        else if (rl == 8) p2_last<T, 8>(v, a, Wb, tw, n, PS, Ns, inv_n);
    }
    if (abort_flag) {
        // the copy in flight (sample s_abort) lands before the block exits
        if (threadIdx.x == 0)
            for (unsigned it = 0; it < (1u << 26) && !try_wait(s_abort & 1); it++) {
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

static int fft_threads(int elems, int cap)
{
    int t = (elems + cap - 1) / cap;
    t = (t + 31) / 32 * 32;
    if (t < 128) t = 128;
    if (t > 1024) t = 1024;
    return t;
}

// Stage set a plan needs (the KIND of smem_fft); kind 2 runs a stage through
// the streaming stage, which needs a scratch copy of the sequences.
static int plan_kind(const FFTPlan &p)
{
    int kind = 0;
    for (int s = 0; s < p.nst; s++) {
        if (p.radix[s] == 3) kind = kind < 1 ? 1 : kind;
        else if (p.radix[s] != 2 && p.radix[s] != 4) kind = 2;
    }
    return kind;
}

static bool plan_generic(const FFTPlan &p) { return plan_kind(p) == 2; }

// kernel instance of a stage set
template <typename F0, typename F1, typename F2>
static auto by_kind(int kind, F0 k0, F1 k1, F2 k2) { return kind == 0 ? k0 : kind == 1 ? k1 : k2; }

size_t grid_proj_smem(int G, int precision, const FFTPlan &p)
{
    const size_t e = precision == 0 ? sizeof(cplx<double>) : sizeof(cplx<float>);
    size_t b = ((size_t)G * G + G) * e;
    if (plan_generic(p)) b += (size_t)G * G * e;
    return b;
}

cudaError_t launch_grid_proj(const void *snap, int precision, int N, int W, int R, int nrec_chunk,
                             int rec_begin, int n_rec_total, const int *grid_map, const FFTPlan &plan,
                             const void *tw, double scale, const double *win, void *series, int nqb,
                             cudaStream_t st)
{
    const int G = plan.n;
    const size_t smem = grid_proj_smem(G, precision, plan);
    const bool big = G * G > 4096;   // grids up to 128 x 128 hold 16 values per thread
    const int threads = fft_threads(G * G, big ? 16 : 8);
    const int kind = plan_kind(plan), gen = kind == 2 ? 1 : 0;
    // only the first nrec_chunk slots of each sample hold records
    dim3 grid(nrec_chunk * 3, W);
    if (precision == 0) {
        auto k = big ? by_kind(kind, grid_proj_kernel<double, double, 16, 0>,
                               grid_proj_kernel<double, double, 16, 1>, grid_proj_kernel<double, double, 16, 2>)
                     : by_kind(kind, grid_proj_kernel<double, double, 8, 0>,
                               grid_proj_kernel<double, double, 8, 1>, grid_proj_kernel<double, double, 8, 2>);
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<grid, threads, smem, st>>>((const double *)snap, N, R, rec_begin, n_rec_total,
                                       grid_map, plan, (const cplx<double> *)tw, scale, win,
                                       (cplx<double> *)series, nqb, gen);
    } else {
        auto k = big ? by_kind(kind, grid_proj_kernel<float, float, 16, 0>, grid_proj_kernel<float, float, 16, 1>,
                               grid_proj_kernel<float, float, 16, 2>)
                     : by_kind(kind, grid_proj_kernel<float, float, 8, 0>, grid_proj_kernel<float, float, 8, 1>,
                               grid_proj_kernel<float, float, 8, 2>);
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<grid, threads, smem, st>>>((const float *)snap, N, R, rec_begin, n_rec_total,
                                       grid_map, plan, (const cplx<float> *)tw, scale, win,
                                       (cplx<float> *)series, nqb, gen);
    }
    return cudaGetLastError();
}

cudaError_t launch_list_proj_simt(const void *snap, int precision, int W, int R, int nrec_chunk,
                                  int N, int rec_begin, int n_rec_total, const void *P, int Lq,
                                  const double *win, void *series, int nqb, int qoff, cudaStream_t st)
{
    const int rows = nrec_chunk * 3;
    dim3 grid((rows + 63) / 64, (Lq + 31) / 32, W);
    if (precision == 0)
        list_proj_simt_kernel<double><<<grid, 256, 0, st>>>(
            (const double *)snap, rows, N, R, rec_begin, n_rec_total, (const cplx<double> *)P, Lq,
            win, (cplx<double> *)series, nqb, qoff);
    else
        list_proj_simt_kernel<float><<<grid, 256, 0, st>>>(
            (const float *)snap, rows, N, R, rec_begin, n_rec_total, (const cplx<float> *)P, Lq,
            win, (cplx<float> *)series, nqb, qoff);
    return cudaGetLastError();
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

static size_t pow2_smem(int n, int nseq, int precision)
{
    const size_t e = precision == 0 ? sizeof(cplx<double>) : sizeof(cplx<float>);
    const int qb = series_qblock(precision);
    const size_t ps = (size_t)n + (size_t)qb * (n / 16) + (qb == 2 ? 8 : 0);
    return ((size_t)nseq * n + (size_t)nseq * ps + n) * e + 16;
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
                            cudaStream_t st)
{
    const int n = plan.n;
    const int qb = series_qblock(precision);
    const int l2 = pow2_log2(n);
    if (l2 >= 0) {
        const int nseq = pow2_nseq(n, precision, Q);
        const size_t smem = pow2_smem(n, nseq, precision);
        const int threads = nseq * n / 16;
        const int ntile = (nqb * qb + nseq - 1) / nseq;
        if (precision == 0) {
            auto k = time_fft_pow2_kernel<double>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k<<<3 * ntile, threads, smem, st>>>((const cplx<double> *)series, W, Q, nqb, n, l2, nseq,
                                                (const cplx<double> *)tw, acc, status);
        } else {
            auto k = time_fft_pow2_kernel<float>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k<<<3 * ntile, threads, smem, st>>>((const cplx<float> *)series, W, Q, nqb, n, l2, nseq,
                                                (const cplx<float> *)tw, acc, status);
        }
        return cudaGetLastError();
    }
    const int qt = time_fft_qt(n, precision);
    const size_t smem = time_fft_smem(n, qt, precision, plan);
    const int threads = fft_threads(qt * n, 8);
    const int ntile = (nqb * qb + qt - 1) / qt;
    const int kind = plan_kind(plan), gen = kind == 2 ? 1 : 0;
    if (precision == 0) {
        auto k = by_kind(kind, time_fft_kernel<double, 0>, time_fft_kernel<double, 1>, time_fft_kernel<double, 2>);
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<3 * ntile, threads, smem, st>>>((const cplx<double> *)series, W, Q, nqb, qt, plan,
                                            (const cplx<double> *)tw, acc, gen);
    } else {
        auto k = by_kind(kind, time_fft_kernel<float, 0>, time_fft_kernel<float, 1>, time_fft_kernel<float, 2>);
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<3 * ntile, threads, smem, st>>>((const cplx<float> *)series, W, Q, nqb, qt, plan,
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

cudaError_t launch_sum_rows(const double *rows, int W, int n, double *out, cudaStream_t st)
{
    sum_rows_kernel<<<(n + 255) / 256, 256, 0, st>>>(rows, W, n, out);
    return cudaGetLastError();
}

}  // namespace smd
