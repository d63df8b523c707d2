// rk_cluster_impl.cuh -- the cluster RK kernel template (see rk_cluster.cuh).
//
// Per RK step, with A and B the two stage buffers (own + halo + one zero
// pad slot) and S the FP64 master spins in registers
// (Codes_Folder/subrouts.cpp:11734-11902):
//
//   stage 1  read A    write B = S + K1/2     (local store + halo pushes)  sync
//   stage 2  read B    write A = S + K2/2                                  sync
//   stage 3  read A    write B = S + K3                                    sync
//   stage 4  read B    S = norm(S + (K1 + 2K2 + 2K3 + K4)/6)
//   no fix:  write A = S                                                   sync
//   fix:     FP64 field sweep, cluster reduction of sigma and E, S = norm(S +
//            scale S x (h x S)) for every site from one set of fields, write A
//
// "sync" publishes the halo pushes: with async halo pushes (st.async
// stores that complete bytes on one of two mbarriers of the receiving CTA,
// alternating per publish), the next stage waits for its own CTA's halo
// bytes only; otherwise it is one cluster barrier (release/acquire).  Two
// barriers suffice: a CTA pushes publish p only after it received publish
// p-1 from every CTA it pushes to, and the neighbour relation is symmetric,
// so every reader of a halo copy has read it (and completed its phase p-2)
// before the copy's owner overwrites it.  The FP64 form (T = double) corrects
// every step against the energy at the step's start, as the reference does;
// the FP32 form (T = float) reuses the two FP32 buffers as one FP64 buffer
// for its correction sweep every fix_every steps, against the initial
// energy.  The reference corrects sites in order, each seeing its corrected
// lower-index neighbours; the one-field (Jacobi) update here differs by
// O(scale^2) per step, which is below 1e-20 for energy-conserving models
// (lattices with the Lieb d-wave term are routed to the single-CTA kernel,
// which reproduces the in-place order).
#pragma once

#include <cooperative_groups.h>
#include <cuda_bf16.h>

#include "rk_cluster.cuh"

namespace smd {

namespace cg = cooperative_groups;

template <typename T>
struct alignas(4 * sizeof(T)) Vec4 {
    T x, y, z, w;
};

// FP64 master spins of a thread's own sites, S[k][c].  The FP32 form keeps
// them in shared memory ([3][n_own_max], site-fastest, so a warp's accesses
// are coalesced): they are read only at the RK combination, the corrections
// and the records, and the registers go to the stage values.  The FP64 form
// keeps them in registers, where every stage reads them.
struct MasterRow {
    double *p;
    int stride;
    __device__ __forceinline__ double &operator[](int c) const { return p[c * stride]; }
};
struct MasterSmem {
    double *base;
    int stride, NT;
    __device__ __forceinline__ MasterRow operator[](int k) const
    {
        return {base + threadIdx.x + k * NT, stride};
    }
};
template <int SPT>
struct MasterRegs {
    double v[SPT][3];
    __device__ __forceinline__ double (&operator[](int k))[3] { return v[k]; }
};

__device__ __forceinline__ double cl_coef(const ClusterParams &P, int e, int c, double)
{
    return P.coef64[e][c];
}
__device__ __forceinline__ float cl_coef(const ClusterParams &P, int e, int c, float)
{
    return P.coef32[e][c];
}

// Block sizes per sites-per-thread: each own site keeps in registers its
// FP64 spin, the FP32 copy (FP32 form), stage input, accumulator, mask, up
// to six packed neighbour words and two push codes, so a thread of SPT
// sites needs about 40 SPT + 20 registers.
template <typename T>
__host__ __device__ constexpr int cl_maxt(int spt)
{
    return spt <= 1 ? 768 : spt <= 2 ? 576 : 512;
}

// One RK launch's records for one sample, spread over the CS CTAs of a group
// of the thread-block cluster: this CTA is CTA `rank` of the group, whose
// CTA 0 is the cluster's CTA `vbase` (every distributed-shared-memory access
// and halo push addresses vbase + the group rank).  All CTAs of the
// hardware cluster run this function together on samples of the same
// lattice and record range, so they meet the same cluster barriers.
template <typename T, int SPT, int ZT>
__device__ __forceinline__ void rk_sample(const ClusterParams &P, const RKJob &J, const int smp,
                                          const int rank, const int vbase,
                                          unsigned char *smem_raw)
{
    static_assert(ZT % 2 == 0 && ZT <= kMaxEdgeSlots, "edge slots come in packed pairs");
    cg::cluster_group cl = cg::this_cluster();
    const int CS = P.CS;
    const int NT = blockDim.x, tid = threadIdx.x;
    const int N = P.N;
    const int base = P.own_base[rank], n_own = P.own_cnt[rank], n_halo = P.halo_cnt[rank];
    const int nom = P.n_own_max;
    const int Np = P.n_loc_max + 1;
    const int pad = P.n_loc_max;
    const T zero = T(0);

    Vec4<T> *A = reinterpret_cast<Vec4<T> *>(smem_raw);
    Vec4<T> *B = A + Np;
    uint32_t *idx = reinterpret_cast<uint32_t *>(B + Np);
    int *push = reinterpret_cast<int *>(idx + (ZT / 2) * nom);
    size_t off = (size_t)(reinterpret_cast<unsigned char *>(push + P.pmax * nom) - smem_raw);
    off = (off + 15) & ~size_t(15);
    double *red = reinterpret_cast<double *>(smem_raw + off);   // [2][16][4][2] compensated partials
    double *wpart = red + 2 * kMaxClusterCTAs * 8;                // [32][4][2]
    uint64_t *hbar = reinterpret_cast<uint64_t *>(wpart + 32 * 8);  // [2] halo publish barriers
    double *Sm = reinterpret_cast<double *>(hbar + 2);              // [3][nom], FP32 form only
    double *D = reinterpret_cast<double *>(smem_raw);             // [3][Np], FP32 form only

    // ---- tables
    {
        const uint32_t *gi = P.idx + (size_t)rank * (ZT / 2) * nom;
        for (int e = tid; e < (ZT / 2) * nom; e += NT) idx[e] = gi[e];
        const int *gp = P.push + (size_t)rank * P.pmax * nom;
        for (int e = tid; e < P.pmax * nom; e += NT) push[e] = gp[e];
    }
    const int *halo = P.halo_gid + (size_t)rank * P.n_loc_max;
    const double *st = J.state + (size_t)smp * 3 * N;
    const uint8_t *imp = J.imp ? J.imp + (size_t)smp * N : nullptr;

    constexpr bool SF = sizeof(T) == 4;
    std::conditional_t<SF, MasterSmem, MasterRegs<SPT>> S;
    if constexpr (SF) S = MasterSmem{Sm, nom, NT};
    T mk[SPT];
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        const int li = tid + k * NT;
        if (li < n_own) {
            const int g = base + li;
#pragma unroll
            for (int c = 0; c < 3; c++) S[k][c] = st[c * N + g];
            mk[k] = (imp && imp[g]) ? zero : T(1);
        } else {
            if constexpr (!SF)
#pragma unroll
                for (int c = 0; c < 3; c++) S[k][c] = 0.0;
            mk[k] = zero;
        }
    }
    int slot = 0;
    const double hz = P.h;
    // FP32 copy of the master spins (FP32 form): stage inputs need no
    // conversion from FP64 at every stage
    T Sf[SF ? SPT : 1][3];
    auto spin = [&](int k, int c) -> T {
        if constexpr (SF) return Sf[k][c];
        else return S[k][c];
    };
    auto sync_spin = [&](int k) {
        if constexpr (SF)
#pragma unroll
            for (int c = 0; c < 3; c++) Sf[k][c] = T(S[k][c]);
    };
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        if (tid + k * NT < n_own) sync_spin(k);
        else if constexpr (SF)
            for (int c = 0; c < 3; c++) Sf[k][c] = zero;
    }
    // packed neighbour words and the first two push codes of each own site
    // live in registers (after the table load below); further push codes
    // stay in shared memory
    constexpr bool NBREG = SPT * (ZT / 2) <= 12;
    uint32_t nbw[NBREG ? SPT : 1][NBREG ? ZT / 2 : 1];
    int pc0[SPT], pc1[SPT];
    bool own_[SPT], bnd[SPT];

    // ---- helpers
    auto cl_sync = [&]() { cl.sync(); };
    // Split cluster barrier.  A stage ends with arrive (release: this
    // thread's local stores and halo pushes) and a CTA barrier; the next
    // stage computes the sites whose neighbours are all own sites first,
    // then waits (acquire) and computes the sites that read halo copies.
    // Every thread alternates arrive and wait.
    auto arrive = [&]() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); };
    auto wait = [&]() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); };

    // Async halo publishes: publish p uses barrier hbar[p & 1] (phase p / 2).
    // Thread 0 arms it with the CTA's incoming halo bytes when the CTA starts
    // producing publish p (bytes that arrive first drive the transaction
    // count negative, which the phase tolerates: it also needs the arrival);
    // the consumer waits with a bounded poll, flagging the status on expiry.
    const bool AH = P.async_halo != 0;
    const uint32_t hbar_a = (uint32_t)__cvta_generic_to_shared(hbar);
    constexpr uint32_t kHaloBytes = sizeof(T) == 4 ? 16 : 24;   // x, y, z (+ w in FP32)
    int pub = 0, need = -1;      // next publish; publish the next halo reads need
    uint32_t cur_bar = hbar_a;
    auto begin_pub = [&]() {
        if (!AH) return;
        cur_bar = hbar_a + (uint32_t)(pub & 1) * 8u;
        if (tid == 0)
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(cur_bar),
                         "r"((uint32_t)n_halo * kHaloBytes)
                         : "memory");
    };
    auto end_pub = [&]() {
        if (AH) {
            need = pub++;
        } else {
            arrive();
        }
        __syncthreads();
    };
    bool hfail = false;          // a wait expired: later waits return at once
    auto hwait = [&](int q) {
        if (q < 0 || hfail) return;
        const uint32_t a = hbar_a + (uint32_t)(q & 1) * 8u, par = (uint32_t)(q >> 1) & 1u;
        for (unsigned it = 0; it < (1u << 26); it++) {
            uint32_t ok;
            asm volatile(
                "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
                " selp.u32 %0, 1, 0, p;\n}\n"
                : "=r"(ok)
                : "r"(a), "r"(par)
                : "memory");
            if (ok) return;
        }
        hfail = true;
        atomicOr(J.status, 1 << kStatusHaloTimeout);
    };
    // the barrier half of a stage: the halo bytes of the publish this stage
    // reads, or the cluster barrier's wait
    auto sync_in = [&]() {
        if (AH) hwait(need);
        else wait();
    };

    // Compensated sum (csum) of NV values over every thread of every CTA of
    // the cluster; all threads receive the totals, summed in a fixed order.
    auto cluster_sum = [&](csum *v, int NV) {
        const int lane = tid & 31, warp = tid >> 5, nw = (NT + 31) >> 5;
        for (int q = 0; q < NV; q++) v[q] = warp_sum_c(v[q]);
        if (lane == 0)
            for (int q = 0; q < NV; q++) {
                wpart[(warp * 4 + q) * 2] = v[q].s;
                wpart[(warp * 4 + q) * 2 + 1] = v[q].c;
            }
        __syncthreads();
        if (warp == 0) {
            for (int q = 0; q < NV; q++) {
                csum x = (lane < nw) ? csum{wpart[(lane * 4 + q) * 2], wpart[(lane * 4 + q) * 2 + 1]}
                                     : csum{0.0, 0.0};
                x = warp_sum_c(x);
                if (lane == 0) {
                    for (int r = 0; r < CS; r++) {
                        double *rr = cl.map_shared_rank(red, vbase + r) + ((slot * kMaxClusterCTAs + rank) * 4 + q) * 2;
                        rr[0] = x.s;
                        rr[1] = x.c;
                    }
                }
            }
        }
        cl.sync();
        for (int q = 0; q < NV; q++) {
            csum t{0.0, 0.0};
            for (int r = 0; r < CS; r++) {
                const double *rr = red + ((slot * kMaxClusterCTAs + r) * 4 + q) * 2;
                t = csum_add(t, csum{rr[0], rr[1]});
            }
            v[q] = t;
        }
        slot ^= 1;
    };

    // local store of own site k's value plus the pushes into halo copies
    // (push codes fill from slot 0, so pc0 < 0 means no pushes at all)
    auto push1 = [&](Vec4<T> *buf, int code, const Vec4<T> &v) {
        if (AH) {
            const uint32_t la = (uint32_t)__cvta_generic_to_shared(buf + (code & 0xffff));
            uint32_t ra, rb;
            asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(la), "r"(vbase + (code >> 16)));
            asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(rb) : "r"(cur_bar), "r"(vbase + (code >> 16)));
            if constexpr (sizeof(T) == 4) {
                asm volatile(
                    "st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.f32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(ra),
                    "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "r"(rb)
                    : "memory");
            } else {
                asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];" ::"r"(ra),
                             "d"(v.x), "d"(v.y), "r"(rb)
                             : "memory");
                asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f64 [%0], %1, [%2];" ::"r"(ra + 16u),
                             "d"(v.z), "r"(rb)
                             : "memory");
            }
        } else {
            cl.map_shared_rank(buf, vbase + (code >> 16))[code & 0xffff] = v;
        }
    };
    auto put = [&](Vec4<T> *buf, int k, int li, const Vec4<T> &v) {
        buf[li] = v;
        if (pc0[k] >= 0) {
            push1(buf, pc0[k], v);
            if (pc1[k] >= 0) {
                push1(buf, pc1[k], v);
                for (int p = 2; p < P.pmax; p++) {
                    const int code = push[p * nom + li];
                    if (code >= 0) push1(buf, code, v);
                }
            }
        }
    };
    auto putD = [&](int li, const double v[3]) {
        for (int c = 0; c < 3; c++) D[c * Np + li] = v[c];
        for (int p = 0; p < P.pmax; p++) {
            const int code = push[p * nom + li];
            if (code >= 0) {
                double *rd = cl.map_shared_rank(D, vbase + (code >> 16));
                const int s2 = code & 0xffff;
                for (int c = 0; c < 3; c++) rd[c * Np + s2] = v[c];
            }
        }
    };
    // packed neighbour word j of own site k (local index li)
    auto nbword = [&](int k, int li, int j) -> uint32_t {
        if constexpr (NBREG) return nbw[k][j];
        else return idx[j * nom + li];
    };

    // field of own site k (local index li) from buffer src (mask applied,
    // -h z added)
    auto field = [&](const Vec4<T> *src, int k, int li, T m, T h[3]) {
        T s0 = zero, s1 = zero, s2 = zero;
#pragma unroll
        for (int e = 0; e < ZT; e += 2) {
            const uint32_t w = nbword(k, li, e >> 1);
            const Vec4<T> a = src[w & 0xffffu];
            const Vec4<T> b = src[w >> 16];
            s0 = fma(cl_coef(P, e, 0, zero), a.x, s0);
            s1 = fma(cl_coef(P, e, 1, zero), a.y, s1);
            s2 = fma(cl_coef(P, e, 2, zero), a.z, s2);
            s0 = fma(cl_coef(P, e + 1, 0, zero), b.x, s0);
            s1 = fma(cl_coef(P, e + 1, 1, zero), b.y, s1);
            s2 = fma(cl_coef(P, e + 1, 2, zero), b.z, s2);
        }
        h[0] = m * s0;
        h[1] = m * s1;
        h[2] = m * s2 - T(hz);
    };
    auto field64 = [&](int k, int li, double m, double h[3]) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
        for (int e = 0; e < ZT; e += 2) {
            const uint32_t w = nbword(k, li, e >> 1);
            const int a = w & 0xffffu, b = w >> 16;
            s0 = fma(P.coef64[e][0], D[a], s0);
            s1 = fma(P.coef64[e][1], D[Np + a], s1);
            s2 = fma(P.coef64[e][2], D[2 * Np + a], s2);
            s0 = fma(P.coef64[e + 1][0], D[b], s0);
            s1 = fma(P.coef64[e + 1][1], D[Np + b], s1);
            s2 = fma(P.coef64[e + 1][2], D[2 * Np + b], s2);
        }
        h[0] = m * s0;
        h[1] = m * s1;
        h[2] = m * s2 - hz;
    };
    // own + halo values of the state from global memory (masked)
    auto fill = [&](Vec4<T> *buf) {
        for (int e = tid; e < n_own + n_halo; e += NT) {
            const int g = e < n_own ? base + e : halo[e - n_own];
            const T m = (imp && imp[g]) ? zero : T(1);
            buf[e] = {m * T(st[g]), m * T(st[N + g]), m * T(st[2 * N + g]), zero};
        }
        if (tid == 0) {
            A[pad] = {zero, zero, zero, zero};
            B[pad] = {zero, zero, zero, zero};
        }
    };
    auto fillD = [&]() {
        for (int e = tid; e < n_own + n_halo; e += NT) {
            const int g = e < n_own ? base + e : halo[e - n_own];
            const double m = (imp && imp[g]) ? 0.0 : 1.0;
            for (int c = 0; c < 3; c++) D[c * Np + e] = m * st[c * N + g];
        }
        if (tid == 0)
            for (int c = 0; c < 3; c++) D[c * Np + pad] = 0.0;
    };
    auto normalise = [&](double v[3]) {
        const double n2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (sizeof(T) == 8) {
            const double n = sqrt(n2);       // FP64 form: the reference's v / |v|
            v[0] = v[0] / n;
            v[1] = v[1] / n;
            v[2] = v[2] / n;
        } else {
            const double r = rsqrt(n2);
            v[0] *= r;
            v[1] *= r;
            v[2] *= r;
        }
    };
    // FP64 energy of the state S (A holds it in the FP64 form; the FP32 form
    // fills D from the owners first).  Call after a cluster barrier.
    auto energy = [&]() -> double {
        csum e{0.0, 0.0};
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const int li = tid + k * NT;
            if (li < n_own) {
                double h[3];
                if (sizeof(T) == 8) {
                    T ht[3];
                    field(A, k, li, mk[k], ht);
                    h[0] = ht[0]; h[1] = ht[1]; h[2] = ht[2];
                } else {
                    field64(k, li, (double)mk[k], h);
                }
                csum_acc(e, S[k][0] * h[0] + S[k][1] * h[1] + S[k][2] * h[2] - hz * S[k][2]);
            }
        }
        csum v[1] = {e};
        cluster_sum(v, 1);
        return 0.5 * csum_val(v[0]);
    };
    auto publishD = [&]() {
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const int li = tid + k * NT;
            if (li < n_own) {
                const double m = (double)mk[k];
                const double v[3] = {m * S[k][0], m * S[k][1], m * S[k][2]};
                putD(li, v);
            }
        }
        if (tid == 0)
            for (int c = 0; c < 3; c++) D[c * Np + pad] = 0.0;
    };
    auto publishA = [&]() {
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const int li = tid + k * NT;
            if (li < n_own) {
                const T m = mk[k];
                put(A, k, li, {m * spin(k, 0), m * spin(k, 1), m * spin(k, 2), zero});
            }
        }
        if (tid == 0) {
            A[pad] = {zero, zero, zero, zero};
            B[pad] = {zero, zero, zero, zero};
        }
    };
    using TS = T;
    TS *snap = reinterpret_cast<TS *>(J.snap);
    const double *s0 = J.s0 + (size_t)smp * 3 * N;
    auto record = [&](int r) {
        const size_t sb = ((size_t)smp * J.snap_R + (r - J.rec_begin)) * 3 * N;
        double p = 0.0;
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const int li = tid + k * NT;
            if (li < n_own) {
                const int g = base + li;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    snap[sb + (size_t)c * N + g] = (TS)S[k][c];
                    p += s0[c * N + g] * S[k][c];
                    if constexpr (sizeof(T) == 4) {
                        if (J.bf_hi) {
                            // the tensor-core projection's operand rows
                            const size_t o = ((size_t)smp * J.snap_R * 3 + (size_t)(r - J.rec_begin) * 3 + c) *
                                                 J.bf_kp + g;
                            const float v = (float)S[k][c];
                            const __nv_bfloat16 h = __float2bfloat16_rn(v);
                            reinterpret_cast<__nv_bfloat16 *>(J.bf_hi)[o] = h;
                            reinterpret_cast<__nv_bfloat16 *>(J.bf_lo)[o] = __float2bfloat16_rn(v - __bfloat162float(h));
                        }
                    }
                }
            }
        }
        if (J.qpart) {
            // this CTA's partial, summed over the cluster by a later launch:
            // no cluster barrier at a record
            const int lane = tid & 31, warp = tid >> 5, nw = (NT + 31) >> 5;
            const double x = warp_sum(p);
            if (lane == 0) wpart[warp * 8] = x;
            __syncthreads();
            if (warp == 0) {
                const double y = warp_sum((lane < nw) ? wpart[lane * 8] : 0.0);
                if (lane == 0) J.qpart[((size_t)smp * J.n_rec + r) * CS + rank] = y;
            }
            __syncthreads();   // wpart is read before the next reduction writes it
            return;
        }
        csum v[1] = {csum{p, 0.0}};
        cluster_sum(v, 1);
        if (rank == 0 && tid == 0) J.qss[(size_t)smp * J.n_rec + r] = (r == 0) ? 1.0 : (1.0 / N) * csum_val(v[0]);
    };

    if (AH && tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(hbar_a));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(hbar_a + 8u));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    cl_sync();   // every CTA of the cluster is running (barriers initialised) before any remote access
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        const int li = tid + k * NT;
        const bool own = li < n_own;
        if constexpr (NBREG)
#pragma unroll
            for (int j = 0; j < ZT / 2; j++) nbw[k][j] = own ? idx[j * nom + li] : 0u;
        pc0[k] = (own && P.pmax > 0) ? push[li] : -1;
        pc1[k] = (own && P.pmax > 1) ? push[nom + li] : -1;
        // a site is on the boundary when a neighbour slot is a halo copy
        bool b = false;
        if (own)
            for (int j = 0; j < ZT / 2; j++) {
                const uint32_t w = idx[j * nom + li];
                const int s0 = (int)(w & 0xffffu), s1 = (int)(w >> 16);
                b = b || (s0 >= n_own && s0 < n_own + n_halo) || (s1 >= n_own && s1 < n_own + n_halo);
            }
        own_[k] = own;
        bnd[k] = b;
    }
    // the sites of the thread whose neighbours are all own sites, the
    // barrier wait, then the sites that read halo copies
    auto two_pass = [&](auto &&body) {
#pragma unroll
        for (int k = 0; k < SPT; k++)
            if (own_[k] && !bnd[k]) body(k);
        sync_in();
#pragma unroll
        for (int k = 0; k < SPT; k++)
            if (own_[k] && bnd[k]) body(k);
    };

    double E0, drift = 0.0;
    if (J.rec_begin == 0) {
        if (sizeof(T) == 8) {
            fill(A);
        } else {
            fillD();
        }
        __syncthreads();
        E0 = energy();
        if (rank == 0 && tid == 0) J.e0[smp] = E0;
        record(0);
    } else {
        E0 = J.e0[smp];
        if (rank == 0 && tid == 0) drift = J.stats[smp * 4 + 0];
    }
    fill(A);
    if (!AH) arrive();
    __syncthreads();

    const T dt = T(J.dt);
    const T f1 = T(1.0 / 6.0), f2 = T(2.0 / 6.0);
    const bool per_step = J.fix_every <= 1;
    const int F = J.fix_every < 1 ? 1 : J.fix_every;
    T Pin[SPT][3], acc[SPT][3];
    for (int r = (J.rec_begin > 0 ? J.rec_begin : 1); r < J.rec_end; r++) {
        for (int ss = 0; ss < J.stride; ss++) {
            const int n = (r - 1) * J.stride + ss + 1;
            const bool fix = per_step || (n % F == 0);
            csum eref{0.0, 0.0};
            // ---- stage 1: A -> B
            begin_pub();
            two_pass([&](int k) {
                const int li = tid + k * NT;
                T h[3], Sp[3], Pv[3];
                field(A, k, li, mk[k], h);
                Sp[0] = spin(k, 0);
                Sp[1] = spin(k, 1);
                Sp[2] = spin(k, 2);
                if (sizeof(T) == 8 && per_step)
                    csum_acc(eref, S[k][0] * h[0] + S[k][1] * h[1] + S[k][2] * h[2] - hz * S[k][2]);
                Pv[0] = h[1] * Sp[2] - h[2] * Sp[1];
                Pv[1] = h[2] * Sp[0] - h[0] * Sp[2];
                Pv[2] = h[0] * Sp[1] - h[1] * Sp[0];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const T K = dt * Pv[c];
                    acc[k][c] = f1 * K;
                    Pin[k][c] = Sp[c] + T(0.5) * K;
                }
                const T m = mk[k];
                put(B, k, li, {m * Pin[k][0], m * Pin[k][1], m * Pin[k][2], zero});
            });
            end_pub();
            // ---- stages 2 and 3
#pragma unroll
            for (int stg = 0; stg < 2; stg++) {
                const Vec4<T> *src = stg ? A : B;
                Vec4<T> *dst = stg ? B : A;
                const T cst = stg ? T(1) : T(0.5);
                begin_pub();
                two_pass([&](int k) {
                    const int li = tid + k * NT;
                    T h[3], Pv[3];
                    field(src, k, li, mk[k], h);
                    const T *Sp = Pin[k];
                    Pv[0] = h[1] * Sp[2] - h[2] * Sp[1];
                    Pv[1] = h[2] * Sp[0] - h[0] * Sp[2];
                    Pv[2] = h[0] * Sp[1] - h[1] * Sp[0];
                    T nx[3];
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const T K = dt * Pv[c];
                        acc[k][c] += f2 * K;
                        nx[c] = spin(k, c) + cst * K;
                    }
#pragma unroll
                    for (int c = 0; c < 3; c++) Pin[k][c] = nx[c];
                    const T m = mk[k];
                    put(dst, k, li, {m * nx[0], m * nx[1], m * nx[2], zero});
                });
                end_pub();
            }
            // ---- stage 4 and the FP64 combination (reads B, writes nothing
            // shared, so no barrier follows)
            two_pass([&](int k) {
                T h[3], Pv[3];
                field(B, k, tid + k * NT, mk[k], h);
                const T *Sp = Pin[k];
                Pv[0] = h[1] * Sp[2] - h[2] * Sp[1];
                Pv[1] = h[2] * Sp[0] - h[0] * Sp[2];
                Pv[2] = h[0] * Sp[1] - h[1] * Sp[0];
                double v[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    acc[k][c] += f1 * (dt * Pv[c]);
                    v[c] = S[k][c] + (double)acc[k][c];
                }
                normalise(v);
#pragma unroll
                for (int c = 0; c < 3; c++) S[k][c] = v[c];
                sync_spin(k);
            });
            if (!fix) {
                begin_pub();
                publishA();
                end_pub();
                continue;
            }
            // ---- energy correction
            if (sizeof(T) == 4) {
                cl_sync();      // stage-4 reads of B finish before D (over A and B) is written
                publishD();
                cl_sync();
            } else if (AH) {
                begin_pub();
                publishA();
                end_pub();
                hwait(need);
            } else {
                publishA();
                cl_sync();
            }
            csum sig{0.0, 0.0}, e1{0.0, 0.0};
#pragma unroll
            for (int k = 0; k < SPT; k++) {
                const int li = tid + k * NT;
                if (li < n_own) {
                    double h[3], Pv[3];
                    if (sizeof(T) == 8) {
                        T ht[3];
                        field(A, k, li, mk[k], ht);
                        h[0] = ht[0]; h[1] = ht[1]; h[2] = ht[2];
                    } else {
                        field64(k, li, (double)mk[k], h);
                    }
                    Pv[0] = h[1] * S[k][2] - h[2] * S[k][1];
                    Pv[1] = h[2] * S[k][0] - h[0] * S[k][2];
                    Pv[2] = h[0] * S[k][1] - h[1] * S[k][0];
                    csum_acc(sig, Pv[0] * Pv[0] + Pv[1] * Pv[1] + Pv[2] * Pv[2]);
                    csum_acc(e1, S[k][0] * h[0] + S[k][1] * h[1] + S[k][2] * h[2] - hz * S[k][2]);
#pragma unroll
                    for (int c = 0; c < 3; c++) acc[k][c] = T(Pv[c]);
                }
            }
            csum t3[3] = {eref, sig, e1};
            cluster_sum(t3, 3);
            const double v3[3] = {csum_val(t3[0]), csum_val(t3[1]), csum_val(t3[2])};
            const double Eref = (sizeof(T) == 8 && per_step) ? 0.5 * v3[0] : E0;
            const double E1 = 0.5 * v3[2];
            double scale = (Eref - E1) / v3[1];
            if (!(v3[1] > 0.0)) {
                scale = 0.0;
                if (rank == 0 && tid == 0) atomicOr(J.status, 1 << kStatusBadSigma);
            }
            if (rank == 0 && tid == 0) {
                const double d = fabs(((sizeof(T) == 8 && per_step) ? Eref : E1) - E0);
                drift = d > drift ? d : drift;
            }
#pragma unroll
            for (int k = 0; k < SPT; k++) {
                const int li = tid + k * NT;
                if (li < n_own) {
                    const double Pv[3] = {(double)acc[k][0], (double)acc[k][1], (double)acc[k][2]};
                    double v[3];
                    v[0] = S[k][0] + scale * (S[k][1] * Pv[2] - S[k][2] * Pv[1]);
                    v[1] = S[k][1] + scale * (S[k][2] * Pv[0] - S[k][0] * Pv[2]);
                    v[2] = S[k][2] + scale * (S[k][0] * Pv[1] - S[k][1] * Pv[0]);
                    normalise(v);
#pragma unroll
                    for (int c = 0; c < 3; c++) S[k][c] = v[c];
                    sync_spin(k);
                }
            }
            begin_pub();
            publishA();   // the reduction's cluster barrier ordered every read of A / D before this
            end_pub();
        }
        if (AH) {
            record(r);
        } else {
            wait();   // completes the step's barrier before record's own reduction
            record(r);
            arrive();
            __syncthreads();
        }
    }
    // the last publish has arrived (async pushes: none is left in flight
    // towards this CTA when it reaches the final cluster barrier)
    if (AH) hwait(need);
    else wait();

    double *stw = J.state + (size_t)smp * 3 * N;
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        const int li = tid + k * NT;
        if (li < n_own)
#pragma unroll
            for (int c = 0; c < 3; c++) stw[c * N + base + li] = S[k][c];
    }
    if (J.rec_end >= J.n_rec) {
        if (sizeof(T) == 4) {
            cl_sync();
            publishD();
            cl_sync();
        }
        const double Ef = energy();
        if (rank == 0 && tid == 0) {
            J.stats[smp * 4 + 1] = Ef;
            J.stats[smp * 4 + 2] = E0;
        }
    }
    if (rank == 0 && tid == 0) J.stats[smp * 4 + 0] = drift;
    cl_sync();   // no CTA leaves while others may still touch its shared memory
    if (AH && tid == 0) {
        // every publish to this CTA has completed (the last one was awaited
        // above): the barriers can be set up afresh for the next sample
        asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(hbar_a) : "memory");
        asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(hbar_a + 8u) : "memory");
    }
}

// One sample per cluster of P.CS CTAs: sample blockIdx.x / P.CS.
template <typename T, int SPT, int ZT>
__global__ void __launch_bounds__(cl_maxt<T>(SPT), 1)
    rk_cluster_kernel(const ClusterParams P, const RKJob J)
{
    extern __shared__ __align__(32) unsigned char smem_raw[];
    const int rank = (int)cg::this_cluster().block_rank();
    rk_sample<T, SPT, ZT>(P, J, blockIdx.x / P.CS, rank, 0, smem_raw);
}

// Persistent batch kernel: clusters take items from B.queue until it runs
// dry.  The slot loop runs over a uniform index so that the slot's
// parameters are read from the kernel-parameter bank at a uniform address
// (the coefficients stay constant operands); only the matching slot runs.
template <typename T, int SPT, int ZT>
__global__ void __launch_bounds__(cl_maxt<T>(SPT), 1)
    rk_batch_kernel(const __grid_constant__ BatchParams B)
{
    extern __shared__ __align__(32) unsigned char smem_raw[];
    __shared__ int item_s;
    cg::cluster_group cl = cg::this_cluster();
    const int hw = (int)cl.block_rank(), csh = (int)cl.num_blocks();
    for (;;) {
        if (hw == 0 && threadIdx.x == 0) {
            const int it = atomicAdd(B.queue, 1);
            for (int r = 0; r < csh; r++) *cl.map_shared_rank(&item_s, r) = it;
        }
        cl.sync();
        const int it = item_s;
        if (it >= B.n_items) break;
        const int2 w = B.items[it];
        for (int lu = 0; lu < B.n_slots; lu++) {
            if (lu != w.x) continue;
            const int vcs = B.slot[lu].P.CS, g = hw / vcs;
            rk_sample<T, SPT, ZT>(B.slot[lu].P, B.slot[lu].J, w.y + g, hw - g * vcs, g * vcs, smem_raw);
        }
        cl.sync();   // every CTA has read item_s before rank 0 overwrites it
    }
}

template <typename T, int SPT, int ZT>
cudaError_t launch_batch_t(const BatchParams *B, int threads, int csh, int nclusters, size_t smem,
                           cudaStream_t st, int *max_clusters)
{
    auto k = rk_batch_kernel<T, SPT, ZT>;
    cudaError_t e = allow_dynamic_smem(k);
    if (e != cudaSuccess) return e;
    if (csh > 8) {
        e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(nclusters * csh), 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csh;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (max_clusters) {
        cfg.gridDim = dim3((unsigned)csh, 1, 1);
        return cudaOccupancyMaxActiveClusters(max_clusters, k, &cfg);
    }
    return cudaLaunchKernelEx(&cfg, k, *B);
}

template <typename T, int SPT>
cudaError_t launch_batch_spt(const BatchParams *B, int zt, int threads, int csh, int nclusters, size_t smem,
                             cudaStream_t st, int *max_clusters)
{
    switch (zt) {
    case 8: return launch_batch_t<T, SPT, 8>(B, threads, csh, nclusters, smem, st, max_clusters);
    case 12: return launch_batch_t<T, SPT, 12>(B, threads, csh, nclusters, smem, st, max_clusters);
    case 18: return launch_batch_t<T, SPT, 18>(B, threads, csh, nclusters, smem, st, max_clusters);
    case 20: return launch_batch_t<T, SPT, 20>(B, threads, csh, nclusters, smem, st, max_clusters);
    default: return cudaErrorInvalidValue;
    }
}

template <typename T>
cudaError_t launch_batch_prec(const BatchParams *B, int spt, int zt, int threads, int csh, int nclusters,
                              size_t smem, cudaStream_t st, int *max_clusters)
{
    switch (spt) {
    case 2: return launch_batch_spt<T, 2>(B, zt, threads, csh, nclusters, smem, st, max_clusters);
    case 4: return launch_batch_spt<T, 4>(B, zt, threads, csh, nclusters, smem, st, max_clusters);
    default: return cudaErrorInvalidValue;
    }
}

template <typename T, int SPT, int ZT>
cudaError_t launch_cluster_t(const ClusterParams &P, const RKJob &J, int threads, size_t smem,
                             cudaStream_t st)
{
    auto k = rk_cluster_kernel<T, SPT, ZT>;
    cudaError_t e = allow_dynamic_smem(k);
    if (e != cudaSuccess) return e;
    if (P.CS > 8) {
        e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(J.n_samples * P.CS, 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = P.CS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, P, J);
}

template <typename T, int SPT>
cudaError_t launch_cluster_spt(const ClusterParams &P, const RKJob &J, int threads, size_t smem,
                               cudaStream_t st)
{
    switch (P.ZT) {
    case 4: return launch_cluster_t<T, SPT, 4>(P, J, threads, smem, st);
    case 8: return launch_cluster_t<T, SPT, 8>(P, J, threads, smem, st);
    case 12: return launch_cluster_t<T, SPT, 12>(P, J, threads, smem, st);
    case 14: return launch_cluster_t<T, SPT, 14>(P, J, threads, smem, st);
    case 18: return launch_cluster_t<T, SPT, 18>(P, J, threads, smem, st);
    case 20: return launch_cluster_t<T, SPT, 20>(P, J, threads, smem, st);
    default: return cudaErrorInvalidValue;
    }
}

template <typename T>
cudaError_t launch_cluster_prec(const ClusterParams &P, const RKJob &J, int spt, int threads,
                                size_t smem, cudaStream_t st)
{
    switch (spt) {
    case 1: return launch_cluster_spt<T, 1>(P, J, threads, smem, st);
    case 2: return launch_cluster_spt<T, 2>(P, J, threads, smem, st);
    case 4: return launch_cluster_spt<T, 4>(P, J, threads, smem, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace smd
