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

// In-register forward DFT of radix R (sign -1).  For R outside {2,3,4,5}
// the twiddle table of the full length n (tw[j] = exp(-2 pi i j / n)) gives
// the R-th roots.
template <typename T, int R>
__device__ __forceinline__ void dft_small(cplx<T> (&v)[R], const cplx<T> *tw, int n)
{
    if (R == 2) {
        cplx<T> a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if (R == 4) {
        cplx<T> a = v[0], b = v[1], c = v[2], d = v[3];
        cplx<T> s0 = cadd(a, c), s1 = csub(a, c), s2 = cadd(b, d), s3 = csub(b, d);
        // -i * s3 = (s3.y, -s3.x)
        v[0] = cadd(s0, s2);
        v[2] = csub(s0, s2);
        v[1] = {s1.x + s3.y, s1.y - s3.x};
        v[3] = {s1.x - s3.y, s1.y + s3.x};
    } else if (R == 3) {
        const T h = T(0.86602540378443864676);   // sqrt(3)/2
        cplx<T> a = v[0], b = v[1], c = v[2];
        cplx<T> s = cadd(b, c), d = csub(b, c);
        cplx<T> m = {a.x - T(0.5) * s.x, a.y - T(0.5) * s.y};
        // -i h d = (h d.y, -h d.x)
        v[0] = cadd(a, s);
        v[1] = {m.x + h * d.y, m.y - h * d.x};
        v[2] = {m.x - h * d.y, m.y + h * d.x};
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
            for (int r = 1; r < R; r++) v[u][r] = cmul(v[u][r], tw[((r * k) * tstep) % n]);
            dft_small<T, R>(v[u], tw, n);
            const int idx = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; r++) buf[q * ss + (idx + r * Ns) * es] = v[u][r];
        }
    }
    __syncthreads();
}

// Generic prime radix: one butterfly at a time through a local array.
template <typename T>
__device__ void stockham_stage_generic(cplx<T> *buf, int n, int nseq, int ss, int es, int Ns,
                                       int R, const cplx<T> *tw, cplx<T> *scratch)
{
    // scratch: a copy of the sequences (same layout), so loads and stores
    // touch different arrays
    const int total = nseq * n;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int q = e / n, x = e - q * n;
        scratch[q * ss + x * es] = buf[q * ss + x * es];
    }
    __syncthreads();
    const int m = n / R, nb = nseq * m, tstep = n / (Ns * R);
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const int q = b / m, j = b - q * m, k = j % Ns;
        const int idx = (j / Ns) * Ns * R + k;
        for (int p = 0; p < R; p++) {
            cplx<T> s = {T(0), T(0)};
            for (int r = 0; r < R; r++) {
                cplx<T> x = scratch[q * ss + (j + r * m) * es];
                if (r) x = cmul(x, tw[((r * k) * tstep) % n]);
                s = cadd(s, cmul(x, tw[((r * p) % R) * (n / R)]));
            }
            buf[q * ss + (idx + p * Ns) * es] = s;
        }
    }
    __syncthreads();
}

// Values each thread holds in registers during a stage: 8 complex doubles
// or 16 complex floats (32 registers either way), so a CTA of 1024 threads
// transforms up to 8192 FP64 or 16384 FP32 elements.
template <typename T>
struct FFTCap {
    static constexpr int v = sizeof(T) == 8 ? 8 : 16;
};

// Full transform.  Radices come from the host plan (product = n); every
// stage needs nseq * n <= FFTCap<T>::v * blockDim.x.
template <typename T>
__device__ void smem_fft(cplx<T> *buf, int n, int nseq, int ss, int es, const int *radix,
                         int nst, const cplx<T> *tw, cplx<T> *scratch)
{
    constexpr int C = FFTCap<T>::v;
    int Ns = 1;
    for (int s = 0; s < nst; s++) {
        const int R = radix[s];
        switch (R) {
        case 4: stockham_stage<T, 4, (C + 3) / 4>(buf, n, nseq, ss, es, Ns, tw); break;
        case 2: stockham_stage<T, 2, (C + 1) / 2>(buf, n, nseq, ss, es, Ns, tw); break;
        case 3: stockham_stage<T, 3, (C + 2) / 3>(buf, n, nseq, ss, es, Ns, tw); break;
        case 5: stockham_stage<T, 5, (C + 4) / 5>(buf, n, nseq, ss, es, Ns, tw); break;
        default: stockham_stage_generic<T>(buf, n, nseq, ss, es, Ns, R, tw, scratch); break;
        }
        Ns *= R;
    }
}

// ---------------------------------------------------------- grid projection

// grid 2D FFT of snapshot rows; blockIdx.x = (s * R + slot) * 3 + c
template <typename TS, typename T>
__global__ void __launch_bounds__(1024) grid_proj_kernel(
    const TS *__restrict__ snap, int N, int R, int rec_begin, int n_rec_total,
    const int *__restrict__ grid_map, FFTPlan plan, const cplx<T> *__restrict__ tw_g,
    double scale, cplx<T> *__restrict__ series, int Q, int use_scratch)
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
    smem_fft<T>(buf, G, G, G, 1, plan.radix, plan.nst, tw, scratch);   // rows
    smem_fft<T>(buf, G, G, 1, G, plan.radix, plan.nst, tw, scratch);   // columns
    const int t = rec_begin + slot;
    cplx<T> *out = series + (((size_t)s * 3 + c) * n_rec_total + t) * Q;
    const T sc = T(scale);
    for (int k = threadIdx.x; k < GG; k += blockDim.x) {
        cplx<T> v = buf[k];
        out[k] = {sc * v.x, sc * v.y};
    }
}

// ---------------------------------------------------------- list projection

// Tiled SIMT GEMM: out[m][l] = sum_k A[m][k] P[k][l], A = snapshot rows
// ([rows][N]), P = phase table ([N][L] complex, scale folded in).
// 64 rows x 32 complex columns per CTA, 256 threads, 4 x 2 outputs each.
template <typename T>
__global__ void __launch_bounds__(256) list_proj_simt_kernel(
    const T *__restrict__ snap, int rows, int N, int R, int rec_begin,
    int n_rec_total, const cplx<T> *__restrict__ P, int Lq,
    cplx<T> *__restrict__ series, int Q, int qoff)
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
        const int c = m % 3, slot = m / 3;
        cplx<T> *out = series + (((size_t)s * 3 + c) * n_rec_total + rec_begin + slot) * Q + qoff;
#pragma unroll
        for (int v = 0; v < 2; v++) {
            const int l = l0 + tl * 2 + v;
            if (l < Lq) out[l] = {ar[u][v][0], ar[u][v][1]};
        }
    }
}

// ---------------------------------------------------------- time transform

// blockIdx.x = c * (Q / QT) + q-tile.  Sums over the W samples of the wave
// into acc[c][q][n_rec] (added to what acc holds).
template <typename T>
__global__ void __launch_bounds__(1024) time_fft_kernel(
    const cplx<T> *__restrict__ series, int W, int Q, int Qp, int QT, FFTPlan plan,
    const cplx<T> *__restrict__ tw_g, const double *__restrict__ win, double *__restrict__ acc,
    int use_scratch)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = plan.n;
    const int ntile = (Q + QT - 1) / QT;
    const int c = blockIdx.x / ntile, q0 = (blockIdx.x % ntile) * QT;
    const int qt = min(QT, Q - q0);
    cplx<T> *buf = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *scratch = use_scratch ? buf + (size_t)QT * n : nullptr;
    constexpr int MAXA = FFTCap<T>::v;
    double a[MAXA];
#pragma unroll
    for (int u = 0; u < MAXA; u++) a[u] = 0.0;
    const int total = qt * n;
    const double inv_n = 1.0 / n;
    for (int s = 0; s < W; s++) {
        const cplx<T> *src = series + ((size_t)s * 3 + c) * n * Qp + q0;
        for (int e = threadIdx.x; e < total; e += blockDim.x) {
            const int qq = e % qt, t = e / qt;
            const cplx<T> v = src[(size_t)t * Qp + qq];
            const T w = T(win[t]);
            buf[qq * n + t] = {w * v.x, w * v.y};
        }
        __syncthreads();
        smem_fft<T>(buf, n, qt, n, 1, plan.radix, plan.nst, tw_g, scratch);
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
    double *out = acc + ((size_t)c * Q + q0) * n;
#pragma unroll
    for (int u = 0; u < MAXA; u++) {
        const int e = threadIdx.x + u * blockDim.x;
        if (e < total) out[e] += a[u];
    }
}

// Same transform fed by TMA: each sample's [n][QT] tile (all records, QT
// consecutive q) arrives as n / box_rows 2D boxes on one mbarrier, so the
// whole tile is in flight at once.  The tile stays in the [t][q] order it
// lands in (sequence stride 1, element stride QT).  Waits are bounded; on
// expiry the kernel records bit 8 in *status and stops.
template <typename T>
__global__ void __launch_bounds__(1024) time_fft_tma_kernel(
    const __grid_constant__ CUtensorMap smap, int W, int Q, int QT, int box_rows, FFTPlan plan,
    const cplx<T> *__restrict__ tw_g, const double *__restrict__ win, double *__restrict__ acc,
    int use_scratch, int *status)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int n = plan.n;
    const int ntile = (Q + QT - 1) / QT;
    const int c = blockIdx.x / ntile, q0 = (blockIdx.x % ntile) * QT;
    cplx<T> *buf = reinterpret_cast<cplx<T> *>(smem_raw);
    const size_t tile = (size_t)QT * n;
    cplx<T> *scratch = use_scratch ? buf + tile : nullptr;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + (use_scratch ? 2 : 1) * tile * sizeof(cplx<T>));
    const uint32_t bar_a = (uint32_t)__cvta_generic_to_shared(bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    constexpr int MAXA = FFTCap<T>::v;
    double a[MAXA];
#pragma unroll
    for (int u = 0; u < MAXA; u++) a[u] = 0.0;
    const int total = QT * n;
    const double inv_n = 1.0 / n;
    const unsigned bytes = (unsigned)(tile * sizeof(cplx<T>));
    bool ok = true;
    for (int s = 0; s < W && ok; s++) {
        if (threadIdx.x == 0) {
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a),
                         "r"(bytes)
                         : "memory");
            for (int b = 0; b < n / box_rows; b++) {
                const uint32_t dst =
                    (uint32_t)__cvta_generic_to_shared(buf + (size_t)b * box_rows * QT);
                asm volatile(
                    "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
                    "[%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
                    "l"(reinterpret_cast<uint64_t>(&smap)), "r"(bar_a), "r"(2 * q0),
                    "r"((s * 3 + c) * n + b * box_rows)
                    : "memory");
            }
        }
        uint32_t done = 0;
        for (unsigned it = 0; it < (1u << 26) && !done; it++) {
            asm volatile(
                "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                " selp.u32 %0, 1, 0, p;\n}\n"
                : "=r"(done)
                : "r"(bar_a), "r"((unsigned)(s & 1))
                : "memory");
        }
        if (!done) {
            if (threadIdx.x == 0) atomicOr(status, 8);
            ok = false;
            break;
        }
        for (int e = threadIdx.x; e < total; e += blockDim.x) {
            const T w = T(win[e / QT]);
            cplx<T> v = buf[e];
            buf[e] = {w * v.x, w * v.y};
        }
        __syncthreads();
        smem_fft<T>(buf, n, QT, 1, QT, plan.radix, plan.nst, tw_g, scratch);
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
    if (!ok) return;
#pragma unroll
    for (int u = 0; u < MAXA; u++) {
        const int e = threadIdx.x + u * blockDim.x;
        if (e < total) {
            const int om = e / QT, qq = e - om * QT;
            if (q0 + qq < Q) acc[((size_t)c * Q + q0 + qq) * n + om] += a[u];
        }
    }
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

static int fft_threads(int elems, int precision)
{
    const int cap = precision == 0 ? 8 : 16;
    int t = (elems + cap - 1) / cap;
    t = (t + 31) / 32 * 32;
    if (t < 128) t = 128;
    if (t > 1024) t = 1024;
    return t;
}

static bool plan_generic(const FFTPlan &p)
{
    for (int s = 0; s < p.nst; s++)
        if (p.radix[s] != 2 && p.radix[s] != 3 && p.radix[s] != 4 && p.radix[s] != 5) return true;
    return false;
}

size_t grid_proj_smem(int G, int precision, const FFTPlan &p)
{
    const size_t e = precision == 0 ? sizeof(cplx<double>) : sizeof(cplx<float>);
    size_t b = ((size_t)G * G + G) * e;
    if (plan_generic(p)) b += (size_t)G * G * e;
    return b;
}

cudaError_t launch_grid_proj(const void *snap, int precision, int N, int W, int R, int nrec_chunk,
                             int rec_begin, int n_rec_total, const int *grid_map, const FFTPlan &plan,
                             const void *tw, double scale, void *series, int Q, cudaStream_t st)
{
    const int G = plan.n;
    const size_t smem = grid_proj_smem(G, precision, plan);
    const int threads = fft_threads(G * G, precision);
    const int gen = plan_generic(plan) ? 1 : 0;
    // only the first nrec_chunk slots of each sample hold records
    dim3 grid(nrec_chunk * 3, W);
    if (precision == 0) {
        auto k = grid_proj_kernel<double, double>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<grid, threads, smem, st>>>((const double *)snap, N, R, rec_begin, n_rec_total,
                                       grid_map, plan, (const cplx<double> *)tw, scale,
                                       (cplx<double> *)series, Q, gen);
    } else {
        auto k = grid_proj_kernel<float, float>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<grid, threads, smem, st>>>((const float *)snap, N, R, rec_begin, n_rec_total,
                                       grid_map, plan, (const cplx<float> *)tw, scale,
                                       (cplx<float> *)series, Q, gen);
    }
    return cudaGetLastError();
}

cudaError_t launch_list_proj_simt(const void *snap, int precision, int W, int R, int nrec_chunk,
                                  int N, int rec_begin, int n_rec_total, const void *P, int Lq,
                                  void *series, int Q, int qoff, cudaStream_t st)
{
    const int rows = nrec_chunk * 3;
    dim3 grid((rows + 63) / 64, (Lq + 31) / 32, W);
    if (precision == 0)
        list_proj_simt_kernel<double><<<grid, 256, 0, st>>>(
            (const double *)snap, rows, N, R, rec_begin, n_rec_total, (const cplx<double> *)P, Lq,
            (cplx<double> *)series, Q, qoff);
    else
        list_proj_simt_kernel<float><<<grid, 256, 0, st>>>(
            (const float *)snap, rows, N, R, rec_begin, n_rec_total, (const cplx<float> *)P, Lq,
            (cplx<float> *)series, Q, qoff);
    return cudaGetLastError();
}

int time_fft_qt(int n, int precision)
{
    const size_t e = precision == 0 ? sizeof(cplx<double>) : sizeof(cplx<float>);
    const int cap = (precision == 0 ? 8 : 16) * 1024;
    int qt = 1;
    while (qt < 64 && (size_t)(qt * 2) * n * e <= 160 * 1024 && qt * 2 * n <= cap) qt *= 2;
    return qt;
}

size_t time_fft_smem(int n, int qt, int precision, const FFTPlan &p)
{
    const size_t e = precision == 0 ? sizeof(cplx<double>) : sizeof(cplx<float>);
    size_t b = (size_t)qt * n * e;
    if (plan_generic(p)) b *= 2;
    return b;
}

// Rows per TMA box for the time transform: the largest divisor of n up to
// 256 whose box starts on a 128-byte boundary of the tile; 0 when none.
int time_fft_box_rows(int n, int qt, int precision)
{
    const size_t cs = precision == 0 ? sizeof(cplx<double>) : sizeof(cplx<float>);
    if ((size_t)qt * cs < 16) return 0;
    for (int d = n < 256 ? n : 256; d >= 1; d--)
        if (n % d == 0 && ((size_t)d * qt * cs) % 128 == 0) return d;
    return 0;
}

cudaError_t launch_time_fft(const void *series, const CUtensorMap *smap, int precision, int W, int Q,
                            int Qp, const FFTPlan &plan, const void *tw, const double *win,
                            double *acc, int *status, cudaStream_t st)
{
    const int n = plan.n;
    const int qt = time_fft_qt(n, precision);
    size_t smem = time_fft_smem(n, qt, precision, plan);
    const int threads = fft_threads(qt * n, precision);
    const int ntile = (Q + qt - 1) / qt;
    const int gen = plan_generic(plan) ? 1 : 0;
    const int box = smap ? time_fft_box_rows(n, qt, precision) : 0;
    if (box) {
        smem += 16;   // the mbarrier
        if (precision == 0) {
            auto k = time_fft_tma_kernel<double>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k<<<3 * ntile, threads, smem, st>>>(*smap, W, Q, qt, box, plan,
                                                (const cplx<double> *)tw, win, acc, gen, status);
        } else {
            auto k = time_fft_tma_kernel<float>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k<<<3 * ntile, threads, smem, st>>>(*smap, W, Q, qt, box, plan,
                                                (const cplx<float> *)tw, win, acc, gen, status);
        }
        return cudaGetLastError();
    }
    if (precision == 0) {
        auto k = time_fft_kernel<double>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<3 * ntile, threads, smem, st>>>((const cplx<double> *)series, W, Q, Qp, qt, plan,
                                            (const cplx<double> *)tw, win, acc, gen);
    } else {
        auto k = time_fft_kernel<float>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<3 * ntile, threads, smem, st>>>((const cplx<float> *)series, W, Q, Qp, qt, plan,
                                            (const cplx<float> *)tw, win, acc, gen);
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
