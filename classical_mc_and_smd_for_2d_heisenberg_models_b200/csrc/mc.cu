// mc.cu -- the Monte Carlo stage that produces the SMD sample file, on the
// GPU (smd_mc_run).
//
// The reference samples each temperature on its own MPI rank
// (Codes_Folder/mc_hm_code.cpp).  One MC step is nmicro overrelaxation
// sweeps (each spin reflected about its local field, reflect_aboutVec,
// subrouts.cpp:4956-5004) and ncanon heat-bath sweeps (a new spin drawn
// from exp(-beta S . h) about the field, get_hBathSample and get_rotZ2VMat,
// subrouts.cpp:5095-5178), every sweep visiting the sites in a shuffled
// order (mc_hm_code.cpp:2797-2965); then the total energy and a parallel-
// tempering exchange between neighbouring temperatures, even pairs on even
// steps and odd pairs on odd steps (mc_hm_code.cpp:3010-3125).  A step
// after an accepted exchange uses nmicro2 / ncanon2 sweeps instead.  During
// the measurement stage the configuration of every crSkip-th step is
// appended to MC_Bin_SpinField (mc_hm_code.cpp:5167-5176).
//
// Here every replica (one per temperature and chain) is one CTA holding its
// spins in shared memory as FP64 [3][N] (global memory, L2-resident, when
// they do not fit).  A sweep visits the sites colour class by colour class
// of a proper colouring of the active-shell neighbour graph: sites of one
// class share no bond, so their updates are independent and run in
// parallel.  This visiting order replaces the reference's shuffled order;
// both leave the Boltzmann distribution invariant, so the two samplers agree
// in distribution, not draw by draw.  Random numbers come from a
// counter-based generator (the SplitMix64 finaliser of Steele, Lea and
// Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014,
// applied to a key made of the seed, replica, step, sweep, site and draw),
// so a run is reproducible for a given seed whatever the launch shape.
// Parallel tempering exchanges the temperatures of two replicas (not their
// spins) in a one-thread kernel between MC steps.
#include "host_internal.h"
#include "field_device.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <random>
#include <cmath>
#include <vector>

namespace smd {

// ---------------------------------------------------------------- device

__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Uniform double in [0, 1) from 53 bits of the hashed key.
__device__ __forceinline__ double uniform01(unsigned long long stream, unsigned long long ctr)
{
    return (double)(mix64(stream + mix64(ctr)) >> 11) * 0x1.0p-53;
}

struct McParams {
    LatticeDev L;
    int N;
    const int *order;        // [N] sites grouped by colour class
    const int *cstart;       // [ncol + 1] class offsets in order
    int ncol;
    const uint8_t *imp;      // [R][N] impurity flags or null
    double *spins;           // [R][3][N]
    const double *beta;      // [R] inverse temperature of each replica
    int *longhb;             // [R] 1: this step uses the long sweep counts
    int nmicro, ncanon, nmicro2, ncanon2;
    unsigned long long seed;
    long long step0;         // index of this launch's first MC step
    int nsteps;
    int total_steps;         // steps of the whole run (energy row length)
    double *energy;          // [R][total_steps] total energy after each step
    int smem_spins;          // 1: spins live in shared memory for the launch
};

// Overrelaxation move (reflect_aboutVec): S' = 2 (S . h) h / |h|^2 - S when
// |h|^2 exceeds 1e-12 (the reference's dbleSmall), else S unchanged.
__device__ __forceinline__ void reflect(double S[3], const double h[3])
{
    const double sq = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
    if (sq > 1.0e-12) {
        const double fac = (2.0 / sq) * (S[0] * h[0] + S[1] * h[1] + S[2] * h[2]);
        for (int c = 0; c < 3; c++) S[c] = fac * h[c] - S[c];
    }
}

// Heat-bath move: z = cos of the angle to the field drawn from
// exp(-beta H z) on [-1, 1] by inverting its distribution (get_hBathSample),
// the azimuth uniform, the vector rotated from the pole onto the field's
// direction V by the rotation of get_rotZ2VMat.  A zero field (a vacancy
// with no couplings at h = 0) draws a uniform direction: the reference's
// normalisation of that field divides by zero.
__device__ __forceinline__ void heat_bath(double S[3], const double h[3], double beta, double r1, double r2)
{
    const double H = sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
    double z;
    if (H > 1.0e-12) {
        const double x0 = 1.0 + r2 * (exp(-2.0 * beta * H) - 1.0);
        z = (-1.0 / (beta * H)) * log(x0) - 1.0;
    } else {
        z = 2.0 * r2 - 1.0;
    }
    z = fmin(1.0, fmax(-1.0, z));
    const double w = sqrt(1.0 - z * z);
    double sn, cs;
    sincospi(2.0 * r1, &sn, &cs);
    const double v[3] = {w * cs, w * sn, z};
    if (!(H > 1.0e-12)) {
        for (int c = 0; c < 3; c++) S[c] = v[c];
        return;
    }
    const double V[3] = {h[0] / H, h[1] / H, h[2] / H};
    const double perp = V[0] * V[0] + V[1] * V[1];
    if (perp > 0.0) {
        const double sf = (1.0 - V[2]) / perp;
        const double x11 = 1.0 - sf * V[0] * V[0], x22 = 1.0 - sf * V[1] * V[1];
        const double x33 = x11 + x22 - 1.0, x12 = -sf * V[0] * V[1];
        S[0] = x11 * v[0] + x12 * v[1] + V[0] * v[2];
        S[1] = x12 * v[0] + x22 * v[1] + V[1] * v[2];
        S[2] = -V[0] * v[0] - V[1] * v[1] + x33 * v[2];
    } else {
        // field along +z or -z: the reference's rotation is the identity
        for (int c = 0; c < 3; c++) S[c] = v[c];
    }
}

// Block sum of a compensated value; every thread gets the total.
__device__ double block_sum_c(csum v, double *red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum_c(v);
    if (lane == 0) {
        red[2 * warp] = v.s;
        red[2 * warp + 1] = v.c;
    }
    __syncthreads();
    csum t{0.0, 0.0};
    for (int w = 0; w < nw; w++) t = csum_add(t, csum{red[2 * w], red[2 * w + 1]});
    __syncthreads();
    return csum_val(t);
}

// Total energy of the replica (get_energyValue, subrouts.cpp:5181-5302): the
// field identity E = 1/2 sum_i (S_i . h_i - h S_i^z) where the host found it
// exact for the lattice, else the bond list.
template <bool GEN>
__device__ double replica_energy(const McParams &P, const double *S, const uint8_t *imp, double *red)
{
    const int N = P.N;
    csum e{0.0, 0.0};
    if (P.L.energy_from_field) {
        for (int i = threadIdx.x; i < N; i += blockDim.x) {
            double h[3];
            local_field<double, GEN>(P.L, S, N, i, imp ? imp[i] : 0, imp, h);
            csum_acc(e, 0.5 * (S[i] * h[0] + S[N + i] * h[1] + S[2 * N + i] * h[2] - P.L.h * S[2 * N + i]));
        }
    } else {
        e = energy_bonds(P.L, S, N, imp);
    }
    return block_sum_c(e, red);
}

// P.nsteps MC steps of replica blockIdx.x: per step the overrelaxation and
// heat-bath sweeps colour class by colour class, then the total energy.
template <bool GEN>
__global__ void mc_step_kernel(const McParams P)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int r = blockIdx.x, N = P.N, tid = threadIdx.x, NT = blockDim.x;
    double *red = reinterpret_cast<double *>(smem);            // [64]
    double *S = P.spins + (size_t)r * 3 * N;
    unsigned char *tail = smem + 64 * sizeof(double);
    if (P.smem_spins) {
        double *Ss = reinterpret_cast<double *>(tail);
        for (int e = tid; e < 3 * N; e += NT) Ss[e] = S[e];
        S = Ss;
        tail += (size_t)3 * N * sizeof(double);
    }
    const uint8_t *imp = nullptr;
    if (P.imp) {
        uint8_t *is = reinterpret_cast<uint8_t *>(tail);
        for (int e = tid; e < N; e += NT) is[e] = P.imp[(size_t)r * N + e];
        imp = is;
    }
    __syncthreads();
    const double beta = P.beta[r];
    const unsigned long long stream = mix64(P.seed ^ (0x9e3779b97f4a7c15ull * (unsigned long long)(r + 1)));
    for (int st = 0; st < P.nsteps; st++) {
        const long long gs = P.step0 + st;
        const bool lng = P.longhb[r] != 0;
        __syncthreads();   // every thread has read the flag
        if (tid == 0) P.longhb[r] = 0;
        const int nm = lng ? P.nmicro2 : P.nmicro, nc = lng ? P.ncanon2 : P.ncanon;
        for (int sw = 0; sw < nm + nc; sw++) {
            for (int c = 0; c < P.ncol; c++) {
                for (int q = P.cstart[c] + tid; q < P.cstart[c + 1]; q += NT) {
                    const int i = P.order[q];
                    double h[3], s[3] = {S[i], S[N + i], S[2 * N + i]};
                    local_field<double, GEN>(P.L, S, N, i, imp ? imp[i] : 0, imp, h);
                    if (sw < nm) {
                        reflect(s, h);
                    } else {
                        const unsigned long long ctr = (((unsigned long long)gs * 64 + sw) * N + i) * 2;
                        heat_bath(s, h, beta, uniform01(stream, ctr), uniform01(stream, ctr + 1));
                    }
                    S[i] = s[0];
                    S[N + i] = s[1];
                    S[2 * N + i] = s[2];
                }
                __syncthreads();
            }
        }
        const double E = replica_energy<GEN>(P, S, imp, red);
        if (tid == 0) P.energy[(size_t)r * P.total_steps + gs] = E;
    }
    if (P.smem_spins) {
        double *G = P.spins + (size_t)r * 3 * N;
        for (int e = tid; e < 3 * N; e += NT) G[e] = S[e];
    }
}

// After MC step gs: the energy of each temperature (the replica holding it),
// then, with exchanges on, the parallel-tempering pass of the reference
// (mc_hm_code.cpp:3010-3125): pairs (n0 + 2 iw, n0 + 2 iw + 1), n0 = gs mod
// 2, accepted with probability min(1, exp((beta_2 - beta_1) (E_2 - E_1)))
// while the upper member's acceptance ratio (exchanges + 1) / attempts stays
// at most 50 %; the two replicas swap temperatures and both run the long
// sweep counts next step.  One thread per chain.
__global__ void mc_temper_kernel(double *beta, int *perm, int *longhb, const double *energy, double *energy_t,
                                 int total, long long gs, int T, int chains, int exchange,
                                 unsigned long long seed, int *cnt, int *exc)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= chains) return;
    int *pm = perm + (size_t)c * T;
    for (int t = 0; t < T; t++)
        energy_t[((size_t)c * T + t) * total + gs] = energy[(size_t)pm[t] * total + gs];
    if (!exchange) return;
    const unsigned long long stream = mix64(seed ^ 0x5851f42d4c957f2dull ^ (unsigned long long)c);
    const int n0 = (int)(gs % 2), hw = T / 2;
    const int iw_max = n0 == 0 ? hw - 1 : hw - 2;
    for (int iw = 0; iw <= iw_max; iw++) {
        const int n1 = n0 + 2 * iw, n2 = n1 + 1;
        const int ra = pm[n1], rb = pm[n2];
        int *cn = cnt + (size_t)c * T, *ex = exc + (size_t)c * T;
        cn[n1]++;
        cn[n2]++;
        const double ratio = (ex[n2] + 1) * (100.0 / cn[n2]);
        const double dE = energy[(size_t)rb * total + gs] - energy[(size_t)ra * total + gs];
        const double dB = beta[rb] - beta[ra];
        const double p = fmin(1.0, exp(dB * dE));
        const double u = uniform01(stream, (unsigned long long)gs * 4096 + n1);
        if (u < p && ratio <= 50.0) {
            pm[n1] = rb;
            pm[n2] = ra;
            const double b = beta[ra];
            beta[ra] = beta[rb];
            beta[rb] = b;
            longhb[ra] = longhb[rb] = 1;
            ex[n1]++;
            ex[n2]++;
        }
    }
}

// Configuration of every temperature of every chain into record slot rec of
// out ([chains][T][n_rec][3][N]).
__global__ void mc_record_kernel(const double *spins, const int *perm, int N, int T, int n_rec, int rec,
                                 double *out)
{
    const int ct = blockIdx.x;   // chain * T + t
    const double *src = spins + (size_t)perm[ct] * 3 * N;
    double *dst = out + ((size_t)ct * n_rec + rec) * 3 * N;
    for (int e = threadIdx.x; e < 3 * N; e += blockDim.x) dst[e] = src[e];
}

}  // namespace smd

// ------------------------------------------------------------------ host

using namespace smd;
using namespace smdh;

namespace {

// Greedy colouring of the undirected graph of the active shells' bonds
// (ghost entries skipped): sites in index order take the smallest colour
// none of their coloured neighbours has.  Returns the sites grouped by
// colour and the class offsets.
void colour_classes(const Lattice &L, std::vector<int> &order, std::vector<int> &cstart)
{
    const int N = L.N;
    std::vector<std::vector<int>> adj(N);
    for (int s = 0; s < 3; s++) {
        const std::vector<int> &t = L.nbr_h[s];
        if (t.empty()) continue;
        const int z = L.zn[s];
        for (int i = 0; i < N; i++)
            for (int k = 0; k < z; k++) {
                const int j = t[(size_t)i * z + k];
                if (j >= 0 && j != i) {
                    adj[i].push_back(j);
                    adj[j].push_back(i);
                }
            }
    }
    std::vector<int> col(N, -1);
    int ncol = 0;
    std::vector<char> used;
    for (int i = 0; i < N; i++) {
        used.assign(ncol + 1, 0);
        for (int j : adj[i])
            if (col[j] >= 0) used[col[j]] = 1;
        int c = 0;
        while (used[c]) c++;
        col[i] = c;
        ncol = std::max(ncol, c + 1);
    }
    cstart.assign(ncol + 1, 0);
    for (int i = 0; i < N; i++) cstart[col[i] + 1]++;
    for (int c = 0; c < ncol; c++) cstart[c + 1] += cstart[c];
    order.assign(N, 0);
    std::vector<int> pos(cstart.begin(), cstart.end() - 1);
    for (int i = 0; i < N; i++) order[pos[col[i]]++] = i;
}

}  // namespace

extern "C" int smd_mc_colouring(smd_ctx *ctx, int lattice_id, int *order, int *cstart, int *ncol)
{
    if (!ctx || !order || !cstart || !ncol) return SMD_EINVAL;
    auto L = find_lattice(ctx, lattice_id);
    if (!L) return fail(ctx, SMD_ENOTFOUND, "mc: unknown lattice");
    std::vector<int> o, c;
    colour_classes(*L, o, c);
    if ((int)c.size() - 1 > *ncol) return fail(ctx, SMD_EINVAL, "mc: colour buffer too small");
    std::copy(o.begin(), o.end(), order);
    std::copy(c.begin(), c.end(), cstart);
    *ncol = (int)c.size() - 1;
    return SMD_OK;
}

extern "C" int smd_mc_run(smd_ctx *ctx, const smd_mc_desc *d, const double *spins0, double *samples,
                          double *energy_out, int *pt_counts, smd_report *rep)
{
    if (!ctx || !d || !d->temps) return SMD_EINVAL;
    auto Lp = find_lattice(ctx, d->lattice);
    if (!Lp) return fail(ctx, SMD_ENOTFOUND, "mc: unknown lattice");
    Lattice &L = *Lp;
    const int T = d->n_temps, C = d->chains, N = L.N;
    if (T < 1 || C < 1 || d->n_therm < 0 || d->n_meas < 0 || d->n_therm + d->n_meas < 1)
        return fail(ctx, SMD_EINVAL, "mc: temperatures, chains or step counts");
    if (d->cr_skip < 1 || d->n_micro < 0 || d->n_canon < 0 || d->n_micro2 < 0 || d->n_canon2 < 0 ||
        d->n_micro + d->n_canon > 64 || d->n_micro2 + d->n_canon2 > 64)
        return fail(ctx, SMD_EINVAL, "mc: crSkip or sweep counts");
    for (int t = 0; t < T; t++)
        if (!(d->temps[t] > 0.0)) return fail(ctx, SMD_EINVAL, "mc: temperatures must be positive");
    const int R = T * C;
    const long long total = (long long)d->n_therm + d->n_meas;
    const int n_rec = d->n_meas / d->cr_skip + (d->n_meas % d->cr_skip ? 1 : 0);
    if ((double)R * 3 * N * 8 * (1.0 + n_rec) + (double)R * total * 16 > 0.9 * (double)ctx->budget)
        return fail(ctx, SMD_ENOMEM_ADMIT, "mc: replicas and records exceed the HBM budget");
    cudaStream_t st = ctx->s_rk;
    const auto t_start = std::chrono::steady_clock::now();

    // colour classes of the active shells
    std::vector<int> order, cstart;
    colour_classes(L, order, cstart);
    const int ncol = (int)cstart.size() - 1;
    int max_class = 0;
    for (int c = 0; c < ncol; c++) max_class = std::max(max_class, cstart[c + 1] - cstart[c]);

    // inputs: spins [R][N][3] (host) or seeded random unit vectors
    std::vector<double> h_spins((size_t)R * N * 3);
    if (spins0) {
        std::copy(spins0, spins0 + h_spins.size(), h_spins.begin());
    } else {
        std::mt19937_64 gen(d->seed ^ 0x6a09e667f3bcc909ull);
        std::normal_distribution<double> g(0.0, 1.0);
        for (size_t k = 0; k < (size_t)R * N; k++) {
            double v[3] = {g(gen), g(gen), g(gen)};
            const double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            for (int c = 0; c < 3; c++) h_spins[k * 3 + c] = v[c] / n;
        }
    }
    // Colour-major storage: site order[q] lives at position q, so a class is
    // a contiguous run of positions and its loads and stores are coalesced.
    // Not for the Lieb d-wave term, whose sign follows the site index parity.
    const bool cmaj = !L.dev.lieb_delta_on;
    LatticeDev Ld = L.dev;
    DevBuf dnbr, dbonds;
    if (cmaj) {
        std::vector<int> inv(N);
        for (int q = 0; q < N; q++) inv[order[q]] = q;
        std::vector<int> ell((size_t)std::max(L.ztot, 1) * N, -1);
        for (int s = 0; s < 3; s++) {
            const std::vector<int> &tb = L.nbr_h[s];
            if (tb.empty()) continue;
            const int z = L.zn[s];
            for (int q = 0; q < N; q++)
                for (int k = 0; k < z; k++) {
                    const int j = tb[(size_t)order[q] * z + k];
                    ell[(size_t)(L.zoff[s] + k) * N + q] = j >= 0 ? inv[j] : -1;
                }
        }
        CK(dnbr.ensure(ell.size() * 4), "cudaMalloc");
        CK(cudaMemcpy(dnbr.p, ell.data(), ell.size() * 4, cudaMemcpyHostToDevice), "H2D table");
        Ld.nbr = dnbr.as<int>();
        if (!Ld.energy_from_field && Ld.nbonds > 0) {
            std::vector<int4> b((size_t)Ld.nbonds);
            CK(cudaMemcpy(b.data(), Ld.bonds, b.size() * sizeof(int4), cudaMemcpyDeviceToHost), "D2H bonds");
            for (int4 &e : b) {
                e.x = inv[e.x];
                e.y = inv[e.y];
            }
            CK(dbonds.ensure(b.size() * sizeof(int4)), "cudaMalloc");
            CK(cudaMemcpy(dbonds.p, b.data(), b.size() * sizeof(int4), cudaMemcpyHostToDevice), "H2D bonds");
            Ld.bonds = dbonds.as<int4>();
        }
        std::vector<double> tmp((size_t)N * 3);
        for (int r = 0; r < R; r++) {
            double *row = h_spins.data() + (size_t)r * N * 3;
            for (int q = 0; q < N; q++)
                for (int c = 0; c < 3; c++) tmp[(size_t)q * 3 + c] = row[(size_t)order[q] * 3 + c];
            std::copy(tmp.begin(), tmp.end(), row);
        }
    }
    std::vector<int> pos_order(N);   // the class runs in stored positions
    for (int q = 0; q < N; q++) pos_order[q] = cmaj ? q : order[q];
    std::vector<double> h_beta(R);
    std::vector<int> h_perm(R);
    for (int c = 0; c < C; c++)
        for (int t = 0; t < T; t++) {
            h_beta[c * T + t] = 1.0 / d->temps[t];
            h_perm[c * T + t] = c * T + t;
        }
    DevBuf in, sp, dord, dcst, dbeta, dperm, dlong, den, dent, dcnt, dexc, dimp, drec, dout;
    CK(in.ensure(h_spins.size() * 8), "cudaMalloc");
    CK(sp.ensure(h_spins.size() * 8), "cudaMalloc");
    CK(dord.ensure((size_t)N * 4), "cudaMalloc");
    CK(dcst.ensure((size_t)(ncol + 1) * 4), "cudaMalloc");
    CK(dbeta.ensure((size_t)R * 8), "cudaMalloc");
    CK(dperm.ensure((size_t)R * 4), "cudaMalloc");
    CK(dlong.ensure((size_t)R * 4), "cudaMalloc");
    CK(den.ensure((size_t)R * total * 8), "cudaMalloc");
    CK(dent.ensure((size_t)R * total * 8), "cudaMalloc");
    CK(dcnt.ensure((size_t)R * 4), "cudaMalloc");
    CK(dexc.ensure((size_t)R * 4), "cudaMalloc");
    if (n_rec > 0 && samples) {
        CK(drec.ensure((size_t)R * n_rec * 3 * N * 8), "cudaMalloc");
        CK(dout.ensure((size_t)R * n_rec * 3 * N * 8), "cudaMalloc");
    }
    std::vector<uint8_t> h_imp;
    if (d->imp) {
        h_imp.resize((size_t)R * N);
        for (int r = 0; r < R; r++)
            for (int q = 0; q < N; q++)
                h_imp[(size_t)r * N + q] = d->imp[(size_t)r * N + (cmaj ? order[q] : q)] ? 1 : 0;
        CK(dimp.ensure(h_imp.size()), "cudaMalloc");
        CK(cudaMemcpyAsync(dimp.p, h_imp.data(), h_imp.size(), cudaMemcpyHostToDevice, st), "H2D imp");
    }
    CK(cudaMemcpyAsync(in.p, h_spins.data(), h_spins.size() * 8, cudaMemcpyHostToDevice, st), "H2D spins");
    CK(cudaMemcpyAsync(dord.p, pos_order.data(), (size_t)N * 4, cudaMemcpyHostToDevice, st), "H2D order");
    CK(cudaMemcpyAsync(dcst.p, cstart.data(), cstart.size() * 4, cudaMemcpyHostToDevice, st), "H2D classes");
    CK(cudaMemcpyAsync(dbeta.p, h_beta.data(), (size_t)R * 8, cudaMemcpyHostToDevice, st), "H2D beta");
    CK(cudaMemcpyAsync(dperm.p, h_perm.data(), (size_t)R * 4, cudaMemcpyHostToDevice, st), "H2D perm");
    CK(cudaMemsetAsync(dlong.p, 0, (size_t)R * 4, st), "memset");
    CK(cudaMemsetAsync(dcnt.p, 0, (size_t)R * 4, st), "memset");
    CK(cudaMemsetAsync(dexc.p, 0, (size_t)R * 4, st), "memset");
    CK(launch_aos_to_soa(in.as<double>(), sp.as<double>(), R, N, st), "aos_to_soa");
    int launches = 1;
    // the pipeline: h_spins and h_imp must outlive the copies above
    CK(cudaStreamSynchronize(st), "sync");

    McParams P{};
    P.L = Ld;
    P.N = N;
    P.order = dord.as<int>();
    P.cstart = dcst.as<int>();
    P.ncol = ncol;
    P.imp = d->imp ? dimp.as<uint8_t>() : nullptr;
    P.spins = sp.as<double>();
    P.beta = dbeta.as<double>();
    P.longhb = dlong.as<int>();
    P.nmicro = d->n_micro;
    P.ncanon = d->n_canon;
    P.nmicro2 = d->n_micro2;
    P.ncanon2 = d->n_canon2;
    P.seed = d->seed;
    P.total_steps = (int)total;
    P.energy = den.as<double>();
    const size_t base_smem = 64 * sizeof(double) + (d->imp ? (size_t)N : 0);
    const size_t spin_smem = (size_t)3 * N * sizeof(double);
    P.smem_spins = base_smem + spin_smem <= 200 * 1024 ? 1 : 0;
    const size_t smem = (base_smem + (P.smem_spins ? spin_smem : 0) + 15) & ~size_t(15);
    const bool gen = d->imp || L.dev.lieb_delta_on;
    auto kern = gen ? mc_step_kernel<true> : mc_step_kernel<false>;
    CK(allow_dynamic_smem(kern), "smem attribute");
    // a thread per site of the largest class, within the block size the
    // kernel's registers allow
    cudaFuncAttributes fa{};
    CK(cudaFuncGetAttributes(&fa, kern), "kernel attributes");
    const int tmax = std::max(32, fa.maxThreadsPerBlock / 32 * 32);
    const int threads = std::min(tmax, std::max(64, (max_class + 31) / 32 * 32));

    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0), "event");
    CK(cudaEventCreate(&e1), "event");
    CK(cudaEventRecord(e0, st), "event");
    // steps of a launch: one with exchanges on (the tempering pass follows
    // every step), else up to the next recorded step, at most 64
    const long long kMaxStepsPerLaunch = 64;
    for (long long gs = 0; gs < total;) {
        long long ns = d->pt ? 1 : std::min(kMaxStepsPerLaunch, total - gs);
        long long rec_step = -1;   // a step of this launch whose configuration is recorded
        for (long long s = gs; s < gs + ns; s++)
            if (s >= d->n_therm && (s - d->n_therm) % d->cr_skip == 0) {
                ns = s - gs + 1;
                rec_step = s;
                break;
            }
        P.step0 = gs;
        P.nsteps = (int)ns;
        kern<<<R, threads, smem, st>>>(P);
        CK(cudaGetLastError(), "mc step kernel");
        launches++;
        if (d->pt) {
            // exchanges from step 101 of the thermalization stage and at
            // every measurement step (mc_hm_code.cpp:3015, 5255)
            const int exch = (gs > 100 || gs >= d->n_therm) && T > 1;
            mc_temper_kernel<<<(C + 127) / 128, 128, 0, st>>>(dbeta.as<double>(), dperm.as<int>(), dlong.as<int>(),
                                                              den.as<double>(), dent.as<double>(), (int)total, gs,
                                                              T, C, exch, d->seed, dcnt.as<int>(), dexc.as<int>());
            CK(cudaGetLastError(), "mc tempering kernel");
            launches++;
        }
        if (rec_step >= 0 && drec.p) {
            const int rec = (int)((rec_step - d->n_therm) / d->cr_skip);
            mc_record_kernel<<<R, 256, 0, st>>>(sp.as<double>(), dperm.as<int>(), N, T, n_rec, rec, drec.as<double>());
            CK(cudaGetLastError(), "mc record kernel");
            launches++;
        }
        gs += ns;
    }
    CK(cudaEventRecord(e1, st), "event");
    CK(cudaEventSynchronize(e1), "sync");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);

    // outputs: records [C][T][n_rec][N][3], energies [C][T][total] per
    // temperature, exchange counts [C][T][2]
    if (drec.p) {
        CK(launch_soa_to_aos(drec.as<double>(), dout.as<double>(), R * n_rec, N, st), "soa_to_aos");
        launches++;
        CK(cudaMemcpyAsync(samples, dout.p, (size_t)R * n_rec * 3 * N * 8, cudaMemcpyDeviceToHost, st), "D2H samples");
        CK(cudaStreamSynchronize(st), "sync");
        if (cmaj) {
            // back to the lattice's site order
            std::vector<double> tmp((size_t)N * 3);
            for (size_t w = 0; w < (size_t)R * n_rec; w++) {
                double *row = samples + w * N * 3;
                for (int q = 0; q < N; q++)
                    for (int c = 0; c < 3; c++) tmp[(size_t)order[q] * 3 + c] = row[(size_t)q * 3 + c];
                std::copy(tmp.begin(), tmp.end(), row);
            }
        }
    }
    if (energy_out)
        CK(cudaMemcpyAsync(energy_out, d->pt ? dent.p : den.p, (size_t)R * total * 8, cudaMemcpyDeviceToHost, st),
           "D2H energy");
    std::vector<int> hc(R), he(R);
    CK(cudaMemcpyAsync(hc.data(), dcnt.p, (size_t)R * 4, cudaMemcpyDeviceToHost, st), "D2H counts");
    CK(cudaMemcpyAsync(he.data(), dexc.p, (size_t)R * 4, cudaMemcpyDeviceToHost, st), "D2H counts");
    CK(cudaStreamSynchronize(st), "sync");
    if (pt_counts)
        for (int k = 0; k < R; k++) {
            pt_counts[2 * k] = hc[k];
            pt_counts[2 * k + 1] = he[k];
        }
    if (rep) {
        *rep = smd_report{};
        rep->ms_device = ms;
        rep->ms_rk = ms;
        rep->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
        rep->kernel_launches = launches;
        rep->rk_launches = launches;
        // site updates: every site of every replica once per sweep
        rep->site_steps = (double)R * N * (double)total * (d->n_micro + d->n_canon);
    }
    return SMD_OK;
}
