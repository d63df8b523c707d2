// fft_device.cuh -- shared-memory mixed-radix FFT stages (Stockham) used by
// the grid projection and the time transform.
#pragma once

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
// {2, 3, 4, 5, 8, 16} the twiddle table of the full length n
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
    } else if constexpr (R == 5) {
        // w = exp(-2 pi i / 5): with t1 = x1 + x4, t2 = x2 + x3,
        // t3 = x1 - x4, t4 = x2 - x3 and c_k = cos(2 pi k / 5),
        // s_k = sin(2 pi k / 5):
        //   X1, X4 = x0 + c1 t1 + c2 t2 -/+ i (s1 t3 + s2 t4)
        //   X2, X3 = x0 + c2 t1 + c1 t2 -/+ i (s2 t3 - s1 t4)
        const T c1 = T(0.30901699437494742410), c2 = T(-0.80901699437494742410);
        const T s1 = T(0.95105651629515357212), s2 = T(0.58778525229247312917);
        const cplx<T> x0 = v[0];
        const cplx<T> t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        const cplx<T> t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        const cplx<T> a1 = {x0.x + c1 * t1.x + c2 * t2.x, x0.y + c1 * t1.y + c2 * t2.y};
        const cplx<T> a2 = {x0.x + c2 * t1.x + c1 * t2.x, x0.y + c2 * t1.y + c1 * t2.y};
        const cplx<T> b1 = {s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y};
        const cplx<T> b2 = {s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y};
        v[0] = {x0.x + t1.x + t2.x, x0.y + t1.y + t2.y};
        // -i b = (b.y, -b.x)
        v[1] = {a1.x + b1.y, a1.y - b1.x};
        v[4] = {a1.x - b1.y, a1.y + b1.x};
        v[2] = {a2.x + b2.y, a2.y - b2.x};
        v[3] = {a2.x - b2.y, a2.y + b2.x};
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
    // Consecutive threads take consecutive elements along a sequence when
    // its elements are adjacent (es == 1) and sequences start at an even
    // stride, else consecutive sequences (element stride es, or an odd
    // sequence stride that spreads them over all banks), so shared-memory
    // accesses stay free of bank conflicts.
    const bool qfast = es != 1 || (ss & 1);
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
// the inline stages.  The copy holds up to scr_seqs sequences ([seq][x],
// compact), so the sequences go through it in batches; thread mapping as in
// stockham_stage.
template <typename T>
__device__ __noinline__ void stockham_stage_generic(cplx<T> *buf, int n, int nseq, int ss, int es,
                                                    int Ns, int R, const cplx<T> *tw,
                                                    cplx<T> *scratch, int scr_seqs)
{
    const bool qfast = es != 1 || (ss & 1);
    const int m = n / R, tstep = n / (Ns * R);
    for (int q0 = 0; q0 < nseq; q0 += scr_seqs) {
        const int nq = min(scr_seqs, nseq - q0);
        for (int e = threadIdx.x; e < nq * n; e += blockDim.x) {
            const int qq = qfast ? e % nq : e / n;
            const int x = qfast ? e / nq : e - qq * n;
            scratch[qq * n + x] = buf[(q0 + qq) * ss + x * es];
        }
        __syncthreads();
        for (int b = threadIdx.x; b < nq * m; b += blockDim.x) {
            const int qq = qfast ? b % nq : b / m;
            const int j = qfast ? b / nq : b - qq * m;
            const int k = j % Ns;
            const int idx = (j / Ns) * Ns * R + k;
            for (int p = 0; p < R; p++) {
                cplx<T> s = {T(0), T(0)};
                for (int r = 0; r < R; r++) {
                    cplx<T> x = scratch[qq * n + j + r * m];
                    if (r) x = cmul(x, tw[(r * k) * tstep]);   // index < n
                    s = cadd(s, cmul(x, tw[((r * p) % R) * (n / R)]));
                }
                buf[(q0 + qq) * ss + (idx + p * Ns) * es] = s;
            }
        }
        __syncthreads();
    }
}

// Stage sets a transform kernel is built with (FL flags), so that each plan
// pays only for the stages it uses: radix 4 and 2 always run inline;
// FK_R16 adds inline radix 16 and 8, FK_R3 inline radix 3, FK_R5 inline
// radix 5 (only in plans that need no out-of-line stage; in the others radix
// 5 runs out of line too, and the instances without radix 5 keep their
// register budgets), and FK_GEN runs
// any other radix through the out-of-line streaming stage (whose register
// needs stay apart from the rest; it needs a scratch copy of the sequences).
enum { FK_R3 = 1, FK_GEN = 2, FK_R16 = 4, FK_R5 = 8, FK_OOL = 16 };

// FK_OOL: the inline stages are called out of line.  A runtime plan's kernel
// holds every stage variant behind one switch; inlined, their registers add
// up and spill, out of line each variant is allocated on its own (one call
// per stage and batch).
template <typename T, int R, int NB>
__device__ __noinline__ void stockham_stage_ool(cplx<T> *buf, int n, int nseq, int ss, int es,
                                                int Ns, const cplx<T> *tw)
{
    stockham_stage<T, R, NB>(buf, n, nseq, ss, es, Ns, tw);
}

template <typename T, int R, int NB, int FL>
__device__ __forceinline__ void run_stage(cplx<T> *buf, int n, int nseq, int ss, int es, int Ns,
                                          const cplx<T> *tw)
{
    if constexpr ((FL & FK_OOL) != 0) stockham_stage_ool<T, R, NB>(buf, n, nseq, ss, es, Ns, tw);
    else stockham_stage<T, R, NB>(buf, n, nseq, ss, es, Ns, tw);
}

// Full transform.  C = values each thread holds in registers during a
// stage.  Radices come from the host plan (product = n); every stage needs
// nseq * n <= C * blockDim.x.
template <typename T, int C, int FL>
__device__ void smem_fft(cplx<T> *buf, int n, int nseq, int ss, int es, const int *radix,
                         int nst, const cplx<T> *tw, cplx<T> *scratch, int scr_seqs)
{
    int Ns = 1;
    for (int s = 0; s < nst; s++) {
        const int R = radix[s];
        switch (R) {
        case 4: run_stage<T, 4, (C + 3) / 4, FL>(buf, n, nseq, ss, es, Ns, tw); break;
        case 2: run_stage<T, 2, (C + 1) / 2, FL>(buf, n, nseq, ss, es, Ns, tw); break;
        case 16:
            if constexpr ((FL & FK_R16) != 0) run_stage<T, 16, (C + 15) / 16, FL>(buf, n, nseq, ss, es, Ns, tw);
            break;
        case 8:
            if constexpr ((FL & FK_R16) != 0) run_stage<T, 8, (C + 7) / 8, FL>(buf, n, nseq, ss, es, Ns, tw);
            break;
        default:
            if constexpr ((FL & FK_R3) != 0) {
                if (R == 3) {
                    run_stage<T, 3, (C + 2) / 3, FL>(buf, n, nseq, ss, es, Ns, tw);
                    break;
                }
            }
            if constexpr ((FL & FK_R5) != 0) {
                if (R == 5) {
                    run_stage<T, 5, (C + 4) / 5, FL>(buf, n, nseq, ss, es, Ns, tw);
                    break;
                }
            }
            if constexpr ((FL & FK_GEN) != 0)
                stockham_stage_generic<T>(buf, n, nseq, ss, es, Ns, R, tw, scratch, scr_seqs);
            break;
        }
        Ns *= R;
    }
}

// threads for a transform of `elems` values with `cap` values per thread
inline int fft_threads(int elems, int cap)
{
    int t = (elems + cap - 1) / cap;
    t = (t + 31) / 32 * 32;
    if (t < 128) t = 128;
    if (t > 1024) t = 1024;
    return t;
}

// Stage set (FK_ flags) a plan needs.
inline int fft_plan_flags(const FFTPlan &p)
{
    int fl = 0;
    for (int s = 0; s < p.nst; s++) {
        const int r = p.radix[s];
        if (r == 16 || r == 8) fl |= FK_R16;
        else if (r == 3) fl |= FK_R3;
        else if (r == 5) fl |= FK_R5;
        else if (r != 2 && r != 4) fl |= FK_GEN;
    }
    // radix 5 runs inline only in plans without an out-of-line radix
    if ((fl & FK_GEN) && (fl & FK_R5)) fl &= ~FK_R5;
    return fl;
}

inline bool plan_generic(const FFTPlan &p) { return (fft_plan_flags(p) & FK_GEN) != 0; }

}  // namespace smd
