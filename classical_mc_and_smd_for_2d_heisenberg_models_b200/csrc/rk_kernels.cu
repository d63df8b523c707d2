// rk_kernels.cu -- persistent RK4 + energy-correction kernels.
//
// One CTA integrates one sample.  The sample's spins stay in shared memory
// for the whole launch as two SoA buffers A and B ([3][N] each); every
// thread owns the sites i = tid + k * blockDim.x and keeps their master
// spins (FP64) and RK accumulator in registers.  Per RK step
// (Codes_Folder/subrouts.cpp:11734-11902):
//
//   stage 1  read A (= S)        write B = S + K1/2     ERef from the same sweep
//   stage 2  read B              write A = S + K2/2
//   stage 3  read A              write B = S + K3
//   stage 4  read B              S = norm(S + (K1 + 2K2 + 2K3 + K4)/6), write A
//   fix      read A: h, P = h x S, sigma = sum |P|^2, E1; one block reduction;
//            S = norm(S + scale S x P), scale = (ERef - E1) / sigma; write A
//
// Kj = dt h(stage input) x (stage input); h_i = -h z + sum_shells sum_nb
// J(a_i, a_nb) lambda (.) S_nb (Codes_Folder/subrouts.cpp:4465-4570).
// Energies come from the field sweeps through E = 1/2 sum_i (S_i . h_i -
// h S_i^z), which equals the reference's bond sum (subrouts.cpp:5181-5302)
// whenever every bond appears once in each direction with one coupling (the
// host checks this per lattice); otherwise the bond list is summed
// explicitly.  The correction uses the sigma sweep's fields for every site
// (a Jacobi update); the reference updates sites in order with fields of
// already-corrected neighbours, which differs by O(scale^2) per step.
//
// Precision form (FP32 kernel): stage fields, cross products and K in FP32
// from FP32 shared buffers; master spins, the RK combination, the
// renormalisation, every energy and the correction in FP64.  The correction
// runs every fix_every steps against the sample's initial energy; at those
// steps the two FP32 buffers are reused as one FP64 buffer so that the
// energy sweep reads FP64 neighbour spins.
#include "field_device.cuh"

#include <algorithm>

namespace smd {

// Local field from the field A with the increments dB already added for the
// neighbours j < i: the state the reference's in-place correction loop sees
// at site i (Codes_Folder/subrouts.cpp:11881-11900), to first order in the
// increments.
template <bool GEN>
__device__ __forceinline__ void local_field_lower(const LatticeDev &L, const double *__restrict__ A,
                                                  const double *__restrict__ dB, int N, int i,
                                                  int ai, const uint8_t *imp, double h[3])
{
    h[0] = 0.0;
    h[1] = 0.0;
    h[2] = (L.h != 0.0) ? -L.h : 0.0;
#pragma unroll
    for (int s = 0; s < 3; s++) {
        if (!L.shell_on[s]) continue;
        const int zs = L.zn[s];
        const int *nb = L.nbr + (size_t)L.zoff[s] * N + i;
#pragma unroll
        for (int k = 0; k < kMaxShellNb; k++) {
            if (k < zs) {
                const int j = __ldg(nb + (size_t)k * N);
                if (j >= 0) {
                    double Jv = L.J[s][0][0];
                    if (GEN) {
                        if (imp) {
                            const int aj = imp[j];
                            Jv = ai ? (aj ? L.J[s][1][1] : L.J[s][1][0])
                                    : (aj ? L.J[s][0][1] : L.J[s][0][0]);
                        }
                        if (s == 1 && L.lieb_delta_on) {
                            const bool neg = ((i & 1) != 0) != ((k & 1) != 0);
                            Jv += neg ? -L.j2_delta : L.j2_delta;
                        }
                    }
                    const double m = (j < i) ? 1.0 : 0.0;
#pragma unroll
                    for (int c = 0; c < 3; c++)
                        h[c] = fma(Jv * L.lam[s][c], A[c * N + j] + m * dB[c * N + j], h[c]);
                }
            }
        }
    }
}

template <typename T>
__device__ __forceinline__ void cross3(const T a[3], const T b[3], T c[3])
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ __forceinline__ void normalise3(double v[3])
{
    const double n = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] = v[0] / n;
    v[1] = v[1] / n;
    v[2] = v[2] / n;
}

// Shared-memory carve-up common to both kernels: two [3][N] stage buffers of
// T, the reduction slots, and the impurity flags.
template <typename T>
__device__ __forceinline__ void carve(unsigned char *raw, int N, T *&A, T *&B, double *&red,
                                      uint8_t *&imp_s)
{
    A = reinterpret_cast<T *>(raw);
    B = A + 3 * N;
    size_t off = (size_t)6 * N * sizeof(T);
    off = (off + 15) & ~size_t(15);
    red = reinterpret_cast<double *>(raw + off);
    imp_s = reinterpret_cast<uint8_t *>(red + 2 * 32 * 8);
}

// ------------------------------------------------------------------ FP64

// Largest CTA for a given number of sites per thread, sized so the
// per-site registers (FP64: spin + accumulator = 12 registers per site; FP32
// form: 9) fit the register file without spills.
__host__ __device__ constexpr int rk_maxt(int prec, int spt)
{
    return prec == 0 ? (spt <= 2 ? 1024 : spt == 3 ? 768 : spt == 4 ? 640 : spt <= 6 ? 512 : 384)
                     : (spt <= 2 ? 1024 : spt == 3 ? 1024 : spt == 4 ? 768 : spt <= 6 ? 640 : 512);
}

template <int MAXSPT, bool GEN>
__global__ void __launch_bounds__(rk_maxt(0, MAXSPT), 1) rk_fp64_kernel(const LatticeDev L, const RKJob J)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N = L.N, T = blockDim.x, tid = threadIdx.x, smp = blockIdx.x;
    double *A, *B, *red;
    uint8_t *imp_s;
    carve<double>(smem_raw, N, A, B, red, imp_s);
    const uint8_t *imp = nullptr;
    if (GEN && J.imp) {
        for (int i = tid; i < N; i += T) imp_s[i] = J.imp[(size_t)smp * N + i];
        imp = imp_s;
    }
    const double *st = J.state + (size_t)smp * 3 * N;
    double S[MAXSPT][3];
#pragma unroll
    for (int k = 0; k < MAXSPT; k++) {
        const int i = tid + k * T;
        if (i < N) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                S[k][c] = st[c * N + i];
                A[c * N + i] = S[k][c];
            }
        }
    }
    __syncthreads();
    int ai[MAXSPT];
#pragma unroll
    for (int k = 0; k < MAXSPT; k++) {
        const int i = tid + k * T;
        ai[k] = (imp && i < N) ? imp[i] : 0;
    }
    int slot = 0;
    const bool efield = L.energy_from_field != 0;
    const double hz = L.h;
    double *snap = reinterpret_cast<double *>(J.snap);
    const double *s0 = J.s0 + (size_t)smp * 3 * N;

    // energy of the state held in A and S (call after a barrier)
    auto energy_of_A = [&]() -> double {
        csum e{0.0, 0.0};
        if (efield) {
#pragma unroll
            for (int k = 0; k < MAXSPT; k++) {
                const int i = tid + k * T;
                if (i < N) {
                    double h[3];
                    local_field<double, GEN>(L, A, N, i, ai[k], imp, h);
                    csum_acc(e, S[k][0] * h[0] + S[k][1] * h[1] + S[k][2] * h[2] - hz * S[k][2]);
                }
            }
        } else {
            e = energy_bonds(L, A, N, imp);
        }
        csum v[1] = {e};
        block_sum_c<1>(v, red, slot);
        return efield ? 0.5 * csum_val(v[0]) : csum_val(v[0]);
    };
    auto record = [&](int r) {
        const size_t base = ((size_t)smp * J.snap_R + (r - J.rec_begin)) * 3 * N;
        double p = 0.0;
#pragma unroll
        for (int k = 0; k < MAXSPT; k++) {
            const int i = tid + k * T;
            if (i < N) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    snap[base + (size_t)c * N + i] = S[k][c];
                    p += s0[c * N + i] * S[k][c];
                }
            }
        }
        csum v[1] = {csum{p, 0.0}};
        block_sum_c<1>(v, red, slot);
        if (tid == 0) J.qss[(size_t)smp * J.n_rec + r] = (r == 0) ? 1.0 : (1.0 / N) * csum_val(v[0]);
    };

    double E0;
    double drift = 0.0;
    if (J.rec_begin == 0) {
        E0 = energy_of_A();
        if (tid == 0) J.e0[smp] = E0;
        record(0);
    } else {
        E0 = J.e0[smp];
        if (tid == 0) drift = J.stats[smp * 4 + 0];
    }

    const double dt = J.dt;
    const double f1 = 1.0 / 6.0, f2 = 2.0 / 6.0;
    const bool per_step = J.fix_every <= 1;
    for (int r = (J.rec_begin > 0 ? J.rec_begin : 1); r < J.rec_end; r++) {
        for (int ss = 0; ss < J.stride; ss++) {
            const int n = (r - 1) * J.stride + ss + 1;
            const bool fix = per_step || (n % J.fix_every == 0);
            double acc[MAXSPT][3];
            csum eref{0.0, 0.0};
            // ---- stage 1: A -> B
#pragma unroll
            for (int k = 0; k < MAXSPT; k++) {
                const int i = tid + k * T;
                if (i < N) {
                    double h[3], P[3];
                    local_field<double, GEN>(L, A, N, i, ai[k], imp, h);
                    if (per_step && efield)
                        csum_acc(eref, S[k][0] * h[0] + S[k][1] * h[1] + S[k][2] * h[2] - hz * S[k][2]);
                    cross3(h, S[k], P);
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const double K = dt * P[c];
                        acc[k][c] = f1 * K;
                        B[c * N + i] = S[k][c] + 0.5 * K;
                    }
                }
            }
            if (per_step && !efield) eref = energy_bonds(L, A, N, imp);
            __syncthreads();
            // ---- stages 2 and 3: B -> A, A -> B
#pragma unroll
            for (int stg = 0; stg < 2; stg++) {
                const double *src = stg ? A : B;
                double *dst = stg ? B : A;
                const double cst = stg ? 1.0 : 0.5;
#pragma unroll
                for (int k = 0; k < MAXSPT; k++) {
                    const int i = tid + k * T;
                    if (i < N) {
                        double h[3], P[3], Sp[3];
                        local_field<double, GEN>(L, src, N, i, ai[k], imp, h);
                        Sp[0] = src[i];
                        Sp[1] = src[N + i];
                        Sp[2] = src[2 * N + i];
                        cross3(h, Sp, P);
#pragma unroll
                        for (int c = 0; c < 3; c++) {
                            const double K = dt * P[c];
                            acc[k][c] += f2 * K;
                            dst[c * N + i] = S[k][c] + cst * K;
                        }
                    }
                }
                __syncthreads();
            }
            // ---- stage 4: B -> combine -> A
#pragma unroll
            for (int k = 0; k < MAXSPT; k++) {
                const int i = tid + k * T;
                if (i < N) {
                    double h[3], P[3], Sp[3];
                    local_field<double, GEN>(L, B, N, i, ai[k], imp, h);
                    Sp[0] = B[i];
                    Sp[1] = B[N + i];
                    Sp[2] = B[2 * N + i];
                    cross3(h, Sp, P);
                    double v[3];
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        acc[k][c] += f1 * (dt * P[c]);
                        v[c] = S[k][c] + acc[k][c];
                    }
                    normalise3(v);
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        S[k][c] = v[c];
                        A[c * N + i] = v[c];
                    }
                }
            }
            __syncthreads();
            if (!fix) continue;
            // ---- energy correction: sigma sweep on A, P kept in acc
            csum sig{0.0, 0.0}, e1{0.0, 0.0};
#pragma unroll
            for (int k = 0; k < MAXSPT; k++) {
                const int i = tid + k * T;
                if (i < N) {
                    double h[3], P[3];
                    local_field<double, GEN>(L, A, N, i, ai[k], imp, h);
                    cross3(h, S[k], P);
                    csum_acc(sig, P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
                    if (efield)
                        csum_acc(e1, S[k][0] * h[0] + S[k][1] * h[1] + S[k][2] * h[2] - hz * S[k][2]);
#pragma unroll
                    for (int c = 0; c < 3; c++) acc[k][c] = P[c];
                }
            }
            if (!efield) e1 = energy_bonds(L, A, N, imp);
            csum t3[3] = {eref, sig, e1};
            block_sum_c<3>(t3, red, slot);
            const double v3[3] = {csum_val(t3[0]), csum_val(t3[1]), csum_val(t3[2])};
            const double Eref = per_step ? (efield ? 0.5 * v3[0] : v3[0]) : E0;
            const double E1 = efield ? 0.5 * v3[2] : v3[2];
            double scale = (Eref - E1) / v3[1];
            if (!(v3[1] > 0.0)) {
                scale = 0.0;
                if (tid == 0) atomicOr(J.status, 1 << kStatusBadSigma);
            }
            if (tid == 0) {
                const double d = fabs((per_step ? Eref : E1) - E0);
                drift = d > drift ? d : drift;
            }
            // A scale above 1e-9 (models whose field is not the gradient of
            // their energy, e.g. the Lieb d-wave term) makes the order of the
            // reference's in-place update visible; a second pass then
            // re-evaluates every field with the lower-index neighbours
            // already corrected, which reproduces that order to O(scale^3).
            // The branch is uniform across the CTA.
            if (fabs(scale) > 1.0e-9) {
#pragma unroll
                for (int k = 0; k < MAXSPT; k++) {
                    const int i = tid + k * T;
                    if (i < N) {
                        double D[3], v[3];
                        cross3(S[k], acc[k], D);
#pragma unroll
                        for (int c = 0; c < 3; c++) v[c] = S[k][c] + scale * D[c];
                        normalise3(v);
#pragma unroll
                        for (int c = 0; c < 3; c++) B[c * N + i] = v[c] - S[k][c];
                    }
                }
                __syncthreads();
#pragma unroll
                for (int k = 0; k < MAXSPT; k++) {
                    const int i = tid + k * T;
                    if (i < N) {
                        double h[3], P[3];
                        local_field_lower<GEN>(L, A, B, N, i, ai[k], imp, h);
                        cross3(h, S[k], P);
#pragma unroll
                        for (int c = 0; c < 3; c++) acc[k][c] = P[c];
                    }
                }
                __syncthreads();
            }
#pragma unroll
            for (int k = 0; k < MAXSPT; k++) {
                const int i = tid + k * T;
                if (i < N) {
                    double D[3], v[3];
                    cross3(S[k], acc[k], D);
#pragma unroll
                    for (int c = 0; c < 3; c++) v[c] = S[k][c] + scale * D[c];
                    normalise3(v);
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        S[k][c] = v[c];
                        A[c * N + i] = v[c];
                    }
                }
            }
            __syncthreads();
        }
        record(r);
    }

    double *stw = J.state + (size_t)smp * 3 * N;
#pragma unroll
    for (int k = 0; k < MAXSPT; k++) {
        const int i = tid + k * T;
        if (i < N)
#pragma unroll
            for (int c = 0; c < 3; c++) stw[c * N + i] = S[k][c];
    }
    if (J.rec_end >= J.n_rec) {
        __syncthreads();
        const double Ef = energy_of_A();
        if (tid == 0) {
            J.stats[smp * 4 + 1] = Ef;
            J.stats[smp * 4 + 2] = E0;
        }
    }
    if (tid == 0) J.stats[smp * 4 + 0] = drift;
}

// ------------------------------------------------------------------ FP32

template <int MAXSPT, bool GEN>
__global__ void __launch_bounds__(rk_maxt(1, MAXSPT), 1) rk_fp32_kernel(const LatticeDev L, const RKJob J)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N = L.N, T = blockDim.x, tid = threadIdx.x, smp = blockIdx.x;
    float *A, *B;
    double *red;
    uint8_t *imp_s;
    carve<float>(smem_raw, N, A, B, red, imp_s);
    double *D = reinterpret_cast<double *>(A);   // FP64 view of A and B together
    const uint8_t *imp = nullptr;
    if (GEN && J.imp) {
        for (int i = tid; i < N; i += T) imp_s[i] = J.imp[(size_t)smp * N + i];
        imp = imp_s;
    }
    const double *st = J.state + (size_t)smp * 3 * N;
    double S[MAXSPT][3];
    int ai[MAXSPT];
#pragma unroll
    for (int k = 0; k < MAXSPT; k++) {
        const int i = tid + k * T;
        if (i < N)
#pragma unroll
            for (int c = 0; c < 3; c++) S[k][c] = st[c * N + i];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < MAXSPT; k++) {
        const int i = tid + k * T;
        ai[k] = (imp && i < N) ? imp[i] : 0;
    }
    int slot = 0;
    const bool efield = L.energy_from_field != 0;
    const double hz = L.h;
    float *snap = reinterpret_cast<float *>(J.snap);
    const double *s0 = J.s0 + (size_t)smp * 3 * N;

    // FP64 copy of S into D (caller guarantees nobody reads A or B)
    auto store_D = [&]() {
#pragma unroll
        for (int k = 0; k < MAXSPT; k++) {
            const int i = tid + k * T;
            if (i < N)
#pragma unroll
                for (int c = 0; c < 3; c++) D[c * N + i] = S[k][c];
        }
    };
    auto store_A = [&]() {
#pragma unroll
        for (int k = 0; k < MAXSPT; k++) {
            const int i = tid + k * T;
            if (i < N)
#pragma unroll
                for (int c = 0; c < 3; c++) A[c * N + i] = (float)S[k][c];
        }
    };
    // FP64 energy of S (D must hold S; call after a barrier)
    auto energy_of_D = [&]() -> double {
        csum e{0.0, 0.0};
        if (efield) {
#pragma unroll
            for (int k = 0; k < MAXSPT; k++) {
                const int i = tid + k * T;
                if (i < N) {
                    double h[3];
                    local_field<double, GEN>(L, D, N, i, ai[k], imp, h);
                    csum_acc(e, S[k][0] * h[0] + S[k][1] * h[1] + S[k][2] * h[2] - hz * S[k][2]);
                }
            }
        } else {
            e = energy_bonds(L, D, N, imp);
        }
        csum v[1] = {e};
        block_sum_c<1>(v, red, slot);
        return efield ? 0.5 * csum_val(v[0]) : csum_val(v[0]);
    };
    auto record = [&](int r) {
        const size_t base = ((size_t)smp * J.snap_R + (r - J.rec_begin)) * 3 * N;
        double p = 0.0;
#pragma unroll
        for (int k = 0; k < MAXSPT; k++) {
            const int i = tid + k * T;
            if (i < N) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    snap[base + (size_t)c * N + i] = (float)S[k][c];
                    p += s0[c * N + i] * S[k][c];
                }
            }
        }
        csum v[1] = {csum{p, 0.0}};
        block_sum_c<1>(v, red, slot);
        if (tid == 0) J.qss[(size_t)smp * J.n_rec + r] = (r == 0) ? 1.0 : (1.0 / N) * csum_val(v[0]);
    };

    double E0;
    double drift = 0.0;
    if (J.rec_begin == 0) {
        store_D();
        __syncthreads();
        E0 = energy_of_D();
        if (tid == 0) J.e0[smp] = E0;
        __syncthreads();
        record(0);
    } else {
        E0 = J.e0[smp];
        if (tid == 0) drift = J.stats[smp * 4 + 0];
    }
    store_A();
    __syncthreads();

    const float dt = (float)J.dt;
    const float f1 = 1.0f / 6.0f, f2 = 2.0f / 6.0f;
    const int F = J.fix_every < 1 ? 1 : J.fix_every;
    for (int r = (J.rec_begin > 0 ? J.rec_begin : 1); r < J.rec_end; r++) {
        for (int ss = 0; ss < J.stride; ss++) {
            const int n = (r - 1) * J.stride + ss + 1;
            const bool fix = (n % F == 0);
            float acc[MAXSPT][3];
            // ---- stage 1: A -> B
#pragma unroll
            for (int k = 0; k < MAXSPT; k++) {
                const int i = tid + k * T;
                if (i < N) {
                    float h[3], P[3], Sf[3];
                    local_field<float, GEN>(L, A, N, i, ai[k], imp, h);
                    Sf[0] = A[i];
                    Sf[1] = A[N + i];
                    Sf[2] = A[2 * N + i];
                    cross3(h, Sf, P);
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const float K = dt * P[c];
                        acc[k][c] = f1 * K;
                        B[c * N + i] = (float)(S[k][c] + 0.5 * (double)K);
                    }
                }
            }
            __syncthreads();
            // ---- stages 2 and 3
#pragma unroll
            for (int stg = 0; stg < 2; stg++) {
                const float *src = stg ? A : B;
                float *dst = stg ? B : A;
                const double cst = stg ? 1.0 : 0.5;
#pragma unroll
                for (int k = 0; k < MAXSPT; k++) {
                    const int i = tid + k * T;
                    if (i < N) {
                        float h[3], P[3], Sp[3];
                        local_field<float, GEN>(L, src, N, i, ai[k], imp, h);
                        Sp[0] = src[i];
                        Sp[1] = src[N + i];
                        Sp[2] = src[2 * N + i];
                        cross3(h, Sp, P);
#pragma unroll
                        for (int c = 0; c < 3; c++) {
                            const float K = dt * P[c];
                            acc[k][c] += f2 * K;
                            dst[c * N + i] = (float)(S[k][c] + cst * (double)K);
                        }
                    }
                }
                __syncthreads();
            }
            // ---- stage 4 and FP64 combine / renormalisation
#pragma unroll
            for (int k = 0; k < MAXSPT; k++) {
                const int i = tid + k * T;
                if (i < N) {
                    float h[3], P[3], Sp[3];
                    local_field<float, GEN>(L, B, N, i, ai[k], imp, h);
                    Sp[0] = B[i];
                    Sp[1] = B[N + i];
                    Sp[2] = B[2 * N + i];
                    cross3(h, Sp, P);
                    double v[3];
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        acc[k][c] += f1 * (dt * P[c]);
                        v[c] = S[k][c] + (double)acc[k][c];
                    }
                    normalise3(v);
#pragma unroll
                    for (int c = 0; c < 3; c++) S[k][c] = v[c];
                }
            }
            __syncthreads();
            if (!fix) {
                store_A();
                __syncthreads();
                continue;
            }
            // ---- FP64 energy correction against E0
            store_D();
            __syncthreads();
            csum sig{0.0, 0.0}, e1{0.0, 0.0};
#pragma unroll
            for (int k = 0; k < MAXSPT; k++) {
                const int i = tid + k * T;
                if (i < N) {
                    double h[3], P[3];
                    local_field<double, GEN>(L, D, N, i, ai[k], imp, h);
                    cross3(h, S[k], P);
                    csum_acc(sig, P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
                    if (efield)
                        csum_acc(e1, S[k][0] * h[0] + S[k][1] * h[1] + S[k][2] * h[2] - hz * S[k][2]);
#pragma unroll
                    for (int c = 0; c < 3; c++) acc[k][c] = (float)P[c];
                }
            }
            if (!efield) e1 = energy_bonds(L, D, N, imp);
            csum t2[2] = {sig, e1};
            block_sum_c<2>(t2, red, slot);
            const double v2[2] = {csum_val(t2[0]), csum_val(t2[1])};
            const double E1 = efield ? 0.5 * v2[1] : v2[1];
            double scale = (E0 - E1) / v2[0];
            if (!(v2[0] > 0.0)) {
                scale = 0.0;
                if (tid == 0) atomicOr(J.status, 1 << kStatusBadSigma);
            }
            if (tid == 0) {
                const double d = fabs(E1 - E0);
                drift = d > drift ? d : drift;
            }
#pragma unroll
            for (int k = 0; k < MAXSPT; k++) {
                const int i = tid + k * T;
                if (i < N) {
                    double P[3] = {acc[k][0], acc[k][1], acc[k][2]};
                    double Dv[3], v[3];
                    cross3(S[k], P, Dv);
#pragma unroll
                    for (int c = 0; c < 3; c++) v[c] = S[k][c] + scale * Dv[c];
                    normalise3(v);
#pragma unroll
                    for (int c = 0; c < 3; c++) S[k][c] = v[c];
                }
            }
            store_A();   // block_sum's barrier ordered every read of D before this
            __syncthreads();
        }
        record(r);
    }

    double *stw = J.state + (size_t)smp * 3 * N;
#pragma unroll
    for (int k = 0; k < MAXSPT; k++) {
        const int i = tid + k * T;
        if (i < N)
#pragma unroll
            for (int c = 0; c < 3; c++) stw[c * N + i] = S[k][c];
    }
    if (J.rec_end >= J.n_rec) {
        __syncthreads();
        store_D();
        __syncthreads();
        const double Ef = energy_of_D();
        if (tid == 0) {
            J.stats[smp * 4 + 1] = Ef;
            J.stats[smp * 4 + 2] = E0;
        }
    }
    if (tid == 0) J.stats[smp * 4 + 0] = drift;
}

// ------------------------------------------------------------ launching

size_t rk_smem_bytes(int N, int precision)
{
    const size_t elem = precision == 0 ? sizeof(double) : sizeof(float);
    size_t off = (size_t)6 * N * elem;
    off = (off + 15) & ~size_t(15);
    return off + 2 * 32 * 8 * sizeof(double) + (size_t)N;
}

template <int MAXSPT, bool GEN>
static cudaError_t launch_one(const LatticeDev &L, const RKJob &J, int precision, int threads,
                              size_t smem, cudaStream_t st)
{
    if (precision == 0) {
        auto k = rk_fp64_kernel<MAXSPT, GEN>;
        cudaError_t e = allow_dynamic_smem(k);
        if (e != cudaSuccess) return e;
        k<<<J.n_samples, threads, smem, st>>>(L, J);
    } else {
        auto k = rk_fp32_kernel<MAXSPT, GEN>;
        cudaError_t e = allow_dynamic_smem(k);
        if (e != cudaSuccess) return e;
        k<<<J.n_samples, threads, smem, st>>>(L, J);
    }
    return cudaGetLastError();
}

template <int MAXSPT>
static cudaError_t launch_spt(const LatticeDev &L, const RKJob &J, int precision, bool gen,
                              int threads, size_t smem, cudaStream_t st)
{
    return gen ? launch_one<MAXSPT, true>(L, J, precision, threads, smem, st)
               : launch_one<MAXSPT, false>(L, J, precision, threads, smem, st);
}

static const int kSptSteps[] = {1, 2, 3, 4, 6, 8};

// Sites per thread for N sites: the smallest instantiated value whose CTA
// limit covers N.  Returns 0 when N exceeds every limit.
static int rk_spt(int N, int precision)
{
    for (int s : kSptSteps)
        if ((long)s * rk_maxt(precision, s) >= N) return s;
    return 0;
}

// Threads per CTA: the fewest warps that cover N at the chosen rate.
int rk_threads(int N, int precision)
{
    const int spt = rk_spt(N, precision);
    if (!spt) return 0;
    int t = (N + spt - 1) / spt;
    t = (t + 31) / 32 * 32;
    return t < 32 ? 32 : t;
}

int rk_max_sites(int precision)
{
    const size_t cap = 227 * 1024;
    int n = 0;
    for (int s : kSptSteps) n = std::max(n, s * rk_maxt(precision, s));
    while (n > 32 && rk_smem_bytes(n, precision) > cap) n -= 32;
    return n;
}

// ------------------------------------------------ local-field histograms

// Histogram of the three components of every site's local field over S
// samples (the static pre-pass of Codes_Folder/smd_code.cpp:2456-2480):
// bin round((h_c + r0) fc) clamped to [0, nh) (get_HistIndex,
// Codes_Folder/subrouts.cpp:795-812).  Counts per block in shared memory,
// then one integer add per bin: the totals do not depend on the order.
template <bool GEN>
__global__ void __launch_bounds__(256) field_hist_kernel(const LatticeDev L, const double *__restrict__ state,
                                                         const uint8_t *__restrict__ imp, int S, double r0,
                                                         double fc, int nh, unsigned long long *hist)
{
    extern __shared__ unsigned int hs[];   // [nh][3]
    for (int e = threadIdx.x; e < nh * 3; e += blockDim.x) hs[e] = 0u;
    __syncthreads();
    const int N = L.N;
    const size_t total = (size_t)S * N;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int s = (int)(e / N), i = (int)(e - (size_t)s * N);
        const uint8_t *im = imp ? imp + (size_t)s * N : nullptr;
        double h[3];
        local_field<double, GEN>(L, state + (size_t)s * 3 * N, N, i, im ? im[i] : 0, im, h);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            int k = (int)round((h[c] + r0) * fc);
            k = k < 0 ? 0 : (k >= nh ? nh - 1 : k);
            atomicAdd(&hs[k * 3 + c], 1u);
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nh * 3; e += blockDim.x)
        if (hs[e]) atomicAdd(&hist[e], (unsigned long long)hs[e]);
}

cudaError_t launch_field_hist(const LatticeDev &L, const double *state, const uint8_t *imp, int S, double r0,
                              double fc, int nh, unsigned long long *hist, bool gen, cudaStream_t st)
{
    const size_t total = (size_t)S * L.N;
    const int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 8);
    const size_t sm = (size_t)nh * 3 * sizeof(unsigned int);
    if (gen) field_hist_kernel<true><<<blocks, 256, sm, st>>>(L, state, imp, S, r0, fc, nh, hist);
    else field_hist_kernel<false><<<blocks, 256, sm, st>>>(L, state, imp, S, r0, fc, nh, hist);
    return cudaGetLastError();
}

cudaError_t launch_rk(const LatticeDev &L, const RKJob &J, int precision, bool gen,
                      cudaStream_t st)
{
    const int spt = rk_spt(L.N, precision);
    const int threads = rk_threads(L.N, precision);
    const size_t smem = rk_smem_bytes(L.N, precision);
    switch (spt) {
    case 1: return launch_spt<1>(L, J, precision, gen, threads, smem, st);
    case 2: return launch_spt<2>(L, J, precision, gen, threads, smem, st);
    case 3: return launch_spt<3>(L, J, precision, gen, threads, smem, st);
    case 4: return launch_spt<4>(L, J, precision, gen, threads, smem, st);
    case 6: return launch_spt<6>(L, J, precision, gen, threads, smem, st);
    case 8: return launch_spt<8>(L, J, precision, gen, threads, smem, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace smd
