// rk_rows_impl.cuh -- the row-band RK kernel template (see rk_rows.cuh).
//
// Same integration as the cluster kernel (Codes_Folder/subrouts.cpp:
// 11734-11902; stage order, FP64 master spins, FP32 or FP64 stages,
// correction every fix_every steps, Jacobi correction update, split cluster
// barrier), with the site records in a padded 2D grid instead of index
// tables.  A thread owns SPT consecutive sites x0 .. x0 + SPT - 1 of one row
// y of its band; their fields come from the five rows y - 2 .. y + 2, each
// row read as one window of consecutive records.
#pragma once

#include "rk_cluster_impl.cuh"
#include "rk_rows.cuh"

namespace smd {

// position xx (relative to the thread's first site) of row offset dy is a
// neighbour of one of the SPT sites through an active shell
template <int GEOM, int SH, int SPT>
__host__ __device__ constexpr bool rows_needed(int dy, int xx)
{
    for (int s = 0; s < 3; s++) {
        if (!((SH >> s) & 1)) continue;
        for (int e = 0; e < stencil_z(GEOM, s); e++) {
            if (stencil_off(GEOM, s, e, 1) != dy) continue;
            const int dx = stencil_off(GEOM, s, e, 0);
            if (xx - dx >= 0 && xx - dx < SPT) return true;
        }
    }
    return false;
}

// shared::cluster address of byte offset `off` of CTA `rank`'s dynamic
// shared memory (the window of a CTA is contiguous, so one mapped base plus
// an offset reaches every buffer)
__device__ __forceinline__ uint32_t rows_map(const void *smem_base, uint32_t rank)
{
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(smem_base);
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}

__device__ __forceinline__ void rows_st(uint32_t addr, const Vec4<float> &v)
{
    asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(v.x), "f"(v.y),
                 "f"(v.z), "f"(v.w)
                 : "memory");
}

__device__ __forceinline__ void rows_st(uint32_t addr, const Vec4<double> &v)
{
    asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(addr), "d"(v.x), "d"(v.y)
                 : "memory");
    asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(addr + 16), "d"(v.z), "d"(v.w)
                 : "memory");
}

__device__ __forceinline__ void rows_st(uint32_t addr, double v)
{
    asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(addr), "d"(v) : "memory");
}

__device__ __forceinline__ double rows_coef(const RowsParams &P, int s, int c, double)
{
    return P.coef64[s][c];
}
__device__ __forceinline__ float rows_coef(const RowsParams &P, int s, int c, float)
{
    return P.coef32[s][c];
}

template <typename T, int SPT, int GEOM, int SH>
__global__ void __launch_bounds__(rows_max_threads(sizeof(T) == 8 ? 0 : 1), 1)
    rk_rows_kernel(const RowsParams P, const RKJob J)
{
    extern __shared__ __align__(32) unsigned char smem_raw[];
    cg::cluster_group cl = cg::this_cluster();
    const int CS = P.CS;
    const int rank = (int)cl.block_rank();
    const int smp = blockIdx.x / CS;
    const int NT = blockDim.x, tid = threadIdx.x;
    const int N = P.N, L = P.L, Pp = rows_pitch(L, SPT);
    const int y0 = P.row0[rank], ny = P.row0[rank + 1] - y0;
    const int Np = (P.ny_max + 4) * Pp;
    const T zero = T(0);

    Vec4<T> *A = reinterpret_cast<Vec4<T> *>(smem_raw);
    Vec4<T> *B = A + Np;
    double *red = reinterpret_cast<double *>(B + Np);             // [2][16][4]
    double *wpart = red + 2 * kMaxClusterCTAs * 4;                // [32][4]
    double *D = reinterpret_cast<double *>(smem_raw);             // [3][Np], FP32 form only

    const int BPR = L / SPT;
    const int y = tid / BPR, x0 = (tid - y * BPR) * SPT;
    const bool own = y < ny;
    const bool bnd = own && (y < 2 || y >= ny - 2);   // reads ghost rows of other bands
    const int base = (y + 2) * Pp + rows_col(x0, SPT); // slot of the first own site
    const int g0 = (y0 + y) * L + x0;                 // its global index
    const double *st = J.state + (size_t)smp * 3 * N;
    const uint8_t *imp = J.imp ? J.imp + (size_t)smp * N : nullptr;

    double S[SPT][3];
    T mk[SPT];
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        const int g = g0 + k;
#pragma unroll
        for (int c = 0; c < 3; c++) S[k][c] = own ? st[c * N + g] : 0.0;
        mk[k] = (own && !(imp && imp[g])) ? T(1) : zero;
    }
    int slot = 0;
    const double hz = P.h;
    constexpr bool SF = sizeof(T) == 4;
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
    for (int k = 0; k < SPT; k++) sync_spin(k);

    // ---- barriers (see rk_cluster_impl.cuh)
    auto cl_sync = [&]() { cl.sync(); };
    auto arrive = [&]() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); };
    auto wait = [&]() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); };
    // a stage: wait for the previous stage's stores and pushes, compute
    // (the boundary rows are a few warps, so they are not deferred behind
    // the wait: that only lengthened each stage's tail)
    auto two_pass = [&](auto &&body) {
        wait();
        if (own) body();
    };
    auto cluster_sum = [&](double *v, int NV) {
        const int lane = tid & 31, warp = tid >> 5, nw = (NT + 31) >> 5;
        for (int q = 0; q < NV; q++) v[q] = warp_sum(v[q]);
        if (lane == 0)
            for (int q = 0; q < NV; q++) wpart[warp * 4 + q] = v[q];
        __syncthreads();
        if (warp == 0) {
            for (int q = 0; q < NV; q++) {
                double x = (lane < nw) ? wpart[lane * 4 + q] : 0.0;
                x = warp_sum(x);
                if (lane == 0) {
                    for (int r = 0; r < CS; r++) {
                        double *rr = cl.map_shared_rank(red, r);
                        rr[slot * kMaxClusterCTAs * 4 + rank * 4 + q] = x;
                    }
                }
            }
        }
        cl.sync();
        for (int q = 0; q < NV; q++) {
            double s = 0.0;
            for (int r = 0; r < CS; r++) s += red[slot * kMaxClusterCTAs * 4 + r * 4 + q];
            v[q] = s;
        }
        slot ^= 1;
    };

    // ---- stores: own record, the ghost-column copy of the two edge
    // columns, and the ghost rows of the bands above and below
    const int rt = rank == 0 ? CS - 1 : rank - 1;        // band above
    const int rn = rank + 1 == CS ? 0 : rank + 1;        // band below
    const int yl_up = P.row0[rt + 1] - P.row0[rt] + y;    // our row y in the band above's frame
    const int yl_dn = y - ny;                             // ... in the band below's frame
    // the bands' shared windows as seen through the cluster (32-bit
    // shared::cluster addresses of their dynamic shared memory)
    const uint32_t win_up = rows_map(smem_raw, rt), win_dn = rows_map(smem_raw, rn);
    // Local stores of own site k: its record and, in the two edge columns
    // of each side, the ghost-column copy.
    auto local_slots = [&](int k, auto &&store) {
        const int x = x0 + k;
        store(base + k);
        if (x < 2 || x >= L - 2) store((y + 2) * Pp + rows_col(x < 2 ? x + L : x - L, SPT));
    };
    auto put = [&](Vec4<T> *buf, int k, const Vec4<T> &v) {
        local_slots(k, [&](int s) { buf[s] = v; });
    };
    auto putD = [&](int k, const double v[3]) {
        local_slots(k, [&](int s) {
            for (int c = 0; c < 3; c++) D[c * Np + s] = v[c];
        });
    };
    // Ghost rows of the neighbouring bands: the two first and two last
    // rows of a band are copied (with their ghost-column copies) after the
    // stage's local stores, reading back the thread's own records, so the
    // compute code carries no remote addressing.
    auto remote_slots = [&](auto &&store) {
        if (!own || !(y < 2 || y >= ny - 2)) return;
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const int x = x0 + k;
            const bool colg = x < 2 || x >= L - 2;
            const int cx = rows_col(x, SPT), cg = rows_col(x < 2 ? x + L : x - L, SPT);
            if (y < 2) {
                store(k, rt, (yl_up + 2) * Pp + cx);
                if (colg) store(k, rt, (yl_up + 2) * Pp + cg);
            }
            if (y >= ny - 2) {
                store(k, rn, (yl_dn + 2) * Pp + cx);
                if (colg) store(k, rn, (yl_dn + 2) * Pp + cg);
            }
        }
    };
    auto push_rows = [&](Vec4<T> *buf) {
        const uint32_t boff = (uint32_t)(reinterpret_cast<unsigned char *>(buf) - smem_raw);
        remote_slots([&](int k, int r, int s) {
            const Vec4<T> v = buf[base + k];
            if (r == rank) buf[s] = v;
            else rows_st((r == rt ? win_up : win_dn) + boff + (uint32_t)s * sizeof(Vec4<T>), v);
        });
    };
    auto push_rowsD = [&]() {
        remote_slots([&](int k, int r, int s) {
            for (int c = 0; c < 3; c++) {
                const double v = D[c * Np + base + k];
                if (r == rank) D[c * Np + s] = v;
                else rows_st((r == rt ? win_up : win_dn) + (uint32_t)(c * Np + s) * 8u, v);
            }
        });
    };

    // ---- fields of the thread's sites (mask applied, -h z added)
    auto field = [&](const Vec4<T> *src, T h[SPT][3]) {
#pragma unroll
        for (int k = 0; k < SPT; k++) h[k][0] = h[k][1] = h[k][2] = zero;
#pragma unroll
        for (int dy = -2; dy <= 2; dy++) {
            const Vec4<T> *row = src + base + dy * Pp;
            Vec4<T> V[SPT + 4];
#pragma unroll
            for (int xx = -2; xx < SPT + 2; xx++)
                if (rows_needed<GEOM, SH, SPT>(dy, xx)) V[xx + 2] = row[xx + rows_fdiv(xx, SPT)];
#pragma unroll
            for (int s = 0; s < 3; s++) {
                if (!((SH >> s) & 1)) continue;
                const T c0 = rows_coef(P, s, 0, zero), c1 = rows_coef(P, s, 1, zero),
                        c2 = rows_coef(P, s, 2, zero);
#pragma unroll
                for (int e = 0; e < stencil_z(GEOM, s); e++) {
                    if (stencil_off(GEOM, s, e, 1) != dy) continue;
                    const int dx = stencil_off(GEOM, s, e, 0);
#pragma unroll
                    for (int k = 0; k < SPT; k++) {
                        const Vec4<T> &w = V[k + dx + 2];
                        h[k][0] = fma(c0, w.x, h[k][0]);
                        h[k][1] = fma(c1, w.y, h[k][1]);
                        h[k][2] = fma(c2, w.z, h[k][2]);
                    }
                }
            }
            // one row window live at a time: keeps the loads of the next
            // row from being hoisted above this row's use (registers)
            asm volatile("" ::: "memory");
        }
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            h[k][0] *= mk[k];
            h[k][1] *= mk[k];
            h[k][2] = mk[k] * h[k][2] - T(hz);
        }
    };
    auto field64 = [&](double h[SPT][3]) {
#pragma unroll
        for (int k = 0; k < SPT; k++) h[k][0] = h[k][1] = h[k][2] = 0.0;
#pragma unroll
        for (int dy = -2; dy <= 2; dy++) {
            const int rb = base + dy * Pp;
            double V[SPT + 4][3];
#pragma unroll
            for (int xx = -2; xx < SPT + 2; xx++)
                if (rows_needed<GEOM, SH, SPT>(dy, xx))
#pragma unroll
                    for (int c = 0; c < 3; c++) V[xx + 2][c] = D[c * Np + rb + xx + rows_fdiv(xx, SPT)];
#pragma unroll
            for (int s = 0; s < 3; s++) {
                if (!((SH >> s) & 1)) continue;
#pragma unroll
                for (int e = 0; e < stencil_z(GEOM, s); e++) {
                    if (stencil_off(GEOM, s, e, 1) != dy) continue;
                    const int dx = stencil_off(GEOM, s, e, 0);
#pragma unroll
                    for (int k = 0; k < SPT; k++)
#pragma unroll
                        for (int c = 0; c < 3; c++)
                            h[k][c] = fma(P.coef64[s][c], V[k + dx + 2][c], h[k][c]);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const double m = (double)mk[k];
            h[k][0] *= m;
            h[k][1] *= m;
            h[k][2] = m * h[k][2] - hz;
        }
    };
    // every slot of the band's frame (own rows, ghost rows, ghost columns)
    // from the state in global memory, masked; pad slots (-1) hold zeros
    auto frame_site = [&](int e) {
        const int yl = e / Pp - 2, pc = e - (e / Pp) * Pp - 3;
        const int q = rows_fdiv(pc, SPT + 1), i = pc - q * (SPT + 1);
        if (i == SPT) return -1;
        const int xl = q * SPT + i;
        int gy = y0 + yl;
        gy = gy < 0 ? gy + L : (gy >= L ? gy - L : gy);
        const int gx = xl < 0 ? xl + L : (xl >= L ? xl - L : xl);
        return gy * L + gx;
    };
    auto fill = [&](Vec4<T> *buf) {
        for (int e = tid; e < (ny + 4) * Pp; e += NT) {
            const int g = frame_site(e);
            if (g < 0) {
                buf[e] = {zero, zero, zero, zero};
                continue;
            }
            const T m = (imp && imp[g]) ? zero : T(1);
            buf[e] = {m * T(st[g]), m * T(st[N + g]), m * T(st[2 * N + g]), zero};
        }
    };
    auto fillD = [&]() {
        for (int e = tid; e < (ny + 4) * Pp; e += NT) {
            const int g = frame_site(e);
            const double m = (g < 0 || (imp && imp[g])) ? 0.0 : 1.0;
            for (int c = 0; c < 3; c++) D[c * Np + e] = g < 0 ? 0.0 : m * st[c * N + g];
        }
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
    // FP64 fields of the own sites from A (FP64 form) or D (FP32 form)
    auto field_fp64 = [&](double h[SPT][3]) {
        if constexpr (sizeof(T) == 8) {
            T ht[SPT][3];
            field(A, ht);
#pragma unroll
            for (int k = 0; k < SPT; k++)
#pragma unroll
                for (int c = 0; c < 3; c++) h[k][c] = ht[k][c];
        } else {
            field64(h);
        }
    };
    auto energy = [&]() -> double {
        double e = 0.0;
        if (own) {
            double h[SPT][3];
            field_fp64(h);
#pragma unroll
            for (int k = 0; k < SPT; k++)
                e += S[k][0] * h[k][0] + S[k][1] * h[k][1] + S[k][2] * h[k][2] - hz * S[k][2];
        }
        double v[1] = {e};
        cluster_sum(v, 1);
        return 0.5 * v[0];
    };
    auto publishD = [&]() {
        if (own)
#pragma unroll
            for (int k = 0; k < SPT; k++) {
                const double m = (double)mk[k];
                const double v[3] = {m * S[k][0], m * S[k][1], m * S[k][2]};
                putD(k, v);
            }
        push_rowsD();
    };
    auto publishA = [&]() {
        if (own)
#pragma unroll
            for (int k = 0; k < SPT; k++) {
                const T m = mk[k];
                put(A, k, {m * spin(k, 0), m * spin(k, 1), m * spin(k, 2), zero});
            }
        push_rows(A);
    };
    T *snap = reinterpret_cast<T *>(J.snap);
    const double *s0 = J.s0 + (size_t)smp * 3 * N;
    auto record = [&](int r) {
        const size_t sb = ((size_t)smp * J.snap_R + (r - J.rec_begin)) * 3 * N;
        double p = 0.0;
        if (own)
#pragma unroll
            for (int k = 0; k < SPT; k++)
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    snap[sb + (size_t)c * N + g0 + k] = (T)S[k][c];
                    p += s0[c * N + g0 + k] * S[k][c];
                }
        double v[1] = {p};
        cluster_sum(v, 1);
        if (rank == 0 && tid == 0) J.qss[(size_t)smp * J.n_rec + r] = (r == 0) ? 1.0 : (1.0 / N) * v[0];
    };

    cl_sync();   // every CTA of the cluster is running before any remote access

    double E0, drift = 0.0;
    if (J.rec_begin == 0) {
        if (sizeof(T) == 8) fill(A);
        else fillD();
        __syncthreads();
        E0 = energy();
        if (rank == 0 && tid == 0) J.e0[smp] = E0;
        record(0);
    } else {
        E0 = J.e0[smp];
        if (rank == 0 && tid == 0) drift = J.stats[smp * 4 + 0];
    }
    cl_sync();   // the FP32 form's D (over A and B) is no longer read
    fill(A);
    arrive();
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
            double eref = 0.0;
            // ---- stage 1: A -> B
            two_pass([&]() {
                T h[SPT][3];
                field(A, h);
#pragma unroll
                for (int k = 0; k < SPT; k++) {
                    T Sp[3], Pv[3];
                    Sp[0] = spin(k, 0);
                    Sp[1] = spin(k, 1);
                    Sp[2] = spin(k, 2);
                    if (sizeof(T) == 8 && per_step)
                        eref += S[k][0] * h[k][0] + S[k][1] * h[k][1] + S[k][2] * h[k][2] -
                                hz * S[k][2];
                    Pv[0] = h[k][1] * Sp[2] - h[k][2] * Sp[1];
                    Pv[1] = h[k][2] * Sp[0] - h[k][0] * Sp[2];
                    Pv[2] = h[k][0] * Sp[1] - h[k][1] * Sp[0];
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const T K = dt * Pv[c];
                        acc[k][c] = f1 * K;
                        Pin[k][c] = Sp[c] + T(0.5) * K;
                    }
                    const T m = mk[k];
                    put(B, k, {m * Pin[k][0], m * Pin[k][1], m * Pin[k][2], zero});
                }
            });
            push_rows(B);
            arrive();
            __syncthreads();
            // ---- stages 2 and 3
#pragma unroll
            for (int stg = 0; stg < 2; stg++) {
                const Vec4<T> *src = stg ? A : B;
                Vec4<T> *dst = stg ? B : A;
                const T cst = stg ? T(1) : T(0.5);
                two_pass([&]() {
                    T h[SPT][3];
                    field(src, h);
#pragma unroll
                    for (int k = 0; k < SPT; k++) {
                        T Pv[3];
                        const T *Sp = Pin[k];
                        Pv[0] = h[k][1] * Sp[2] - h[k][2] * Sp[1];
                        Pv[1] = h[k][2] * Sp[0] - h[k][0] * Sp[2];
                        Pv[2] = h[k][0] * Sp[1] - h[k][1] * Sp[0];
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
                        put(dst, k, {m * nx[0], m * nx[1], m * nx[2], zero});
                    }
                });
                push_rows(dst);
                arrive();
                __syncthreads();
            }
            // ---- stage 4 and the FP64 combination
            two_pass([&]() {
                T h[SPT][3];
                field(B, h);
#pragma unroll
                for (int k = 0; k < SPT; k++) {
                    T Pv[3];
                    const T *Sp = Pin[k];
                    Pv[0] = h[k][1] * Sp[2] - h[k][2] * Sp[1];
                    Pv[1] = h[k][2] * Sp[0] - h[k][0] * Sp[2];
                    Pv[2] = h[k][0] * Sp[1] - h[k][1] * Sp[0];
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
                }
            });
            if (!fix) {
                publishA();
                arrive();
                __syncthreads();
                continue;
            }
            // ---- energy correction
            if (sizeof(T) == 4) {
                cl_sync();      // stage-4 reads of B finish before D (over A and B) is written
                publishD();
            } else {
                publishA();
            }
            cl_sync();
            double sig = 0.0, e1 = 0.0;
            if (own) {
                double h[SPT][3];
                field_fp64(h);
#pragma unroll
                for (int k = 0; k < SPT; k++) {
                    double Pv[3];
                    Pv[0] = h[k][1] * S[k][2] - h[k][2] * S[k][1];
                    Pv[1] = h[k][2] * S[k][0] - h[k][0] * S[k][2];
                    Pv[2] = h[k][0] * S[k][1] - h[k][1] * S[k][0];
                    sig += Pv[0] * Pv[0] + Pv[1] * Pv[1] + Pv[2] * Pv[2];
                    e1 += S[k][0] * h[k][0] + S[k][1] * h[k][1] + S[k][2] * h[k][2] - hz * S[k][2];
#pragma unroll
                    for (int c = 0; c < 3; c++) acc[k][c] = T(Pv[c]);
                }
            }
            double v3[3] = {eref, sig, e1};
            cluster_sum(v3, 3);
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
            if (own)
#pragma unroll
                for (int k = 0; k < SPT; k++) {
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
            publishA();   // the reduction's cluster barrier ordered every read of A / D before this
            arrive();
            __syncthreads();
        }
        wait();   // completes the step's barrier before record's own reduction
        record(r);
        arrive();
        __syncthreads();
    }
    wait();

    double *stw = J.state + (size_t)smp * 3 * N;
    if (own)
#pragma unroll
        for (int k = 0; k < SPT; k++)
#pragma unroll
            for (int c = 0; c < 3; c++) stw[c * N + g0 + k] = S[k][c];
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
}

template <typename T, int GEOM, int SH>
cudaError_t launch_rows_t(const RowsParams &P, const RKJob &J, int threads, size_t smem,
                          cudaStream_t st)
{
    constexpr int SPT = rows_spt(sizeof(T) == 8 ? 0 : 1);
    auto k = rk_rows_kernel<T, SPT, GEOM, SH>;
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

// instances: shells NN (1), NN + NNN (3), all three (7; NN + X runs here
// with zero NNN couplings)
template <typename T>
cudaError_t launch_rows_prec(const RowsParams &P, const RKJob &J, int threads, size_t smem,
                             cudaStream_t st)
{
    const int sh = P.shells == 1 ? 1 : P.shells == 3 ? 3 : 7;
    if (P.geom == kStencilSquare) {
        if (sh == 1) return launch_rows_t<T, kStencilSquare, 1>(P, J, threads, smem, st);
        if (sh == 3) return launch_rows_t<T, kStencilSquare, 3>(P, J, threads, smem, st);
        return launch_rows_t<T, kStencilSquare, 7>(P, J, threads, smem, st);
    }
    if (sh == 1) return launch_rows_t<T, kStencilTriang, 1>(P, J, threads, smem, st);
    if (sh == 3) return launch_rows_t<T, kStencilTriang, 3>(P, J, threads, smem, st);
    return launch_rows_t<T, kStencilTriang, 7>(P, J, threads, smem, st);
}

}  // namespace smd
