// field_device.cuh -- the local exchange field of one site and the
// bond-list energy, shared by the RK kernels (rk_kernels.cu) and the Monte
// Carlo sampler (mc.cu).
#pragma once

#include "smd_device.cuh"

namespace smd {

// kernel-parameter accessors: with s and c fixed after unrolling these
// become constant-bank operands
__device__ __forceinline__ double pcoef(const LatticeDev &L, int s, int c, double) { return L.coef[s][c]; }
__device__ __forceinline__ float pcoef(const LatticeDev &L, int s, int c, float) { return L.coeff[s][c]; }
__device__ __forceinline__ double plam(const LatticeDev &L, int s, int c, double) { return L.lam[s][c]; }
__device__ __forceinline__ float plam(const LatticeDev &L, int s, int c, float) { return L.lamf[s][c]; }
__device__ __forceinline__ double pJ(const LatticeDev &L, int s, int a, int b, double) { return L.J[s][a][b]; }
__device__ __forceinline__ float pJ(const LatticeDev &L, int s, int a, int b, float) { return L.Jf[s][a][b]; }
__device__ __forceinline__ double pdelta(const LatticeDev &L, double) { return L.j2_delta; }
__device__ __forceinline__ float pdelta(const LatticeDev &L, float) { return L.j2_deltaf; }
__device__ __forceinline__ double ph(const LatticeDev &L, double) { return L.h; }
__device__ __forceinline__ float ph(const LatticeDev &L, float) { return L.hf; }

// Local field of site i from SoA buffer b ([3][N]).  GEN handles disorder
// (imp != null) and the Lieb d-wave term; otherwise every shell has one
// coefficient vector.  ai = impurity flag of site i.
template <typename T, bool GEN>
__device__ __forceinline__ void local_field(const LatticeDev &L, const T *__restrict__ b,
                                            int N, int i, int ai, const uint8_t *imp,
                                            T h[3])
{
    const T zero = T(0);
    h[0] = zero;
    h[1] = zero;
    h[2] = (L.h != 0.0) ? -ph(L, zero) : zero;
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
                    T c0, c1, c2;
                    if (GEN) {
                        T Jv;
                        if (imp) {
                            const int aj = imp[j];
                            Jv = ai ? (aj ? pJ(L, s, 1, 1, zero) : pJ(L, s, 1, 0, zero))
                                    : (aj ? pJ(L, s, 0, 1, zero) : pJ(L, s, 0, 0, zero));
                        } else {
                            Jv = pJ(L, s, 0, 0, zero);
                        }
                        if (s == 1 && L.lieb_delta_on) {
                            const bool neg = ((i & 1) != 0) != ((k & 1) != 0);
                            Jv += neg ? -pdelta(L, zero) : pdelta(L, zero);
                        }
                        c0 = Jv * plam(L, s, 0, zero);
                        c1 = Jv * plam(L, s, 1, zero);
                        c2 = Jv * plam(L, s, 2, zero);
                    } else {
                        c0 = pcoef(L, s, 0, zero);
                        c1 = pcoef(L, s, 1, zero);
                        c2 = pcoef(L, s, 2, zero);
                    }
                    h[0] = fma(c0, b[j], h[0]);
                    h[1] = fma(c1, b[N + j], h[1]);
                    h[2] = fma(c2, b[2 * N + j], h[2]);
                }
            }
        }
    }
}


// Bond-list energy for lattices where the field identity does not hold;
// returns this thread's compensated partial sum.  b is an FP64 SoA field.
__device__ inline csum energy_bonds(const LatticeDev &L, const double *b, int N,
                             const uint8_t *imp)
{
    csum e{0.0, 0.0};
    for (int q = threadIdx.x; q < L.nbonds; q += blockDim.x) {
        const int4 bd = L.bonds[q];
        const int i = bd.x, j = bd.y, s = bd.z;
        double Jv = imp ? L.J[s][imp[i]][imp[j]] : L.J[s][0][0];
        if (s == 1 && L.lieb_delta_on)
            Jv += ((i & 1) ? -1 : 1) * ((j & 1) ? -1 : 1) * L.j2_delta;
        csum_acc(e, Jv * L.lam[s][0] * b[i] * b[j] + Jv * L.lam[s][1] * b[N + i] * b[N + j] +
                        Jv * L.lam[s][2] * b[2 * N + i] * b[2 * N + j]);
    }
    if (L.h != 0.0)
        for (int i = threadIdx.x; i < N; i += blockDim.x) csum_acc(e, (-L.h) * b[2 * N + i]);
    return e;
}


}  // namespace smd
