// prepass.cu -- the static pre-pass over the MC samples (smd_static_prepass).
//
// Before the dynamics the reference's main program reads every sample once
// (Codes_Folder/smd_code.cpp:2289-2726) and
//   * histograms the three components of every site's local field
//     (201 bins over +-maxLocField, get_HistIndex at subrouts.cpp:795-812),
//   * transforms the spins onto the DFT grid (get_SqData_iMKL), caps every
//     amplitude at spec0Max = 10 (smd_code.cpp:2522-2533) and averages the
//     static structure factor max(1e-16, |S_c(q)|^2) (get_StaticSFac,
//     subrouts.cpp:8799-8825) with the factor 1 / max(S - 1, 1).
// Here the samples are the records of one grid projection (the same kernel
// as the dynamics, FP64) in chunks, followed by an accumulation kernel that
// adds the capped |S|^2 of every sample in sample order; the histogram
// kernel evaluates the fields of all samples at once.
#include "host_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

using namespace smd;
using namespace smdh;

namespace smd {

// out[c][q] += sum over the chunk's samples t, in order, of
// max(1e-16, |min(cap, r) S / r|^2), r = |S_c(q, t)|; series [3][nqb][S]
// (FP64, one q per block).  A zero amplitude gives 0/0 in the reference's
// cap, whose square then loses to 1e-16 in max(): 1e-16 here too.
__global__ void static_sf_kernel(const cplx<double> *__restrict__ series, int Q, int nqb, int S, double cap,
                                 double *__restrict__ out)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 3 * Q) return;
    const int c = e / Q, q = e - c * Q;
    const cplx<double> *p = series + ((size_t)c * nqb + q) * S;
    double acc = out[e];
    for (int t = 0; t < S; t++) {
        const cplx<double> z = p[t];
        const double r = hypot(z.x, z.y);
        double v = 1.0e-16;
        if (r > 0.0) {
            const double m = r < cap ? r : cap;
            const double a = m * z.x / r, b = m * z.y / r;
            const double pw = a * a + b * b;
            v = pw > 1.0e-16 ? pw : 1.0e-16;
        }
        acc += v;
    }
    out[e] = acc;
}

cudaError_t launch_static_sf(const void *series, int Q, int nqb, int S, double cap, double *out,
                             cudaStream_t st)
{
    static_sf_kernel<<<(3 * Q + 127) / 128, 128, 0, st>>>(static_cast<const cplx<double> *>(series), Q, nqb, S,
                                                         cap, out);
    return cudaGetLastError();
}

}  // namespace smd

extern "C" int smd_static_prepass(smd_ctx *ctx, int lattice_id, int qset_id, int n_samples, const double *spins0,
                                  const int *imp, double *sf_out, long long *hist_out, double *max_field)
{
    if (!ctx || !spins0 || !sf_out || !hist_out || n_samples < 1) return SMD_EINVAL;
    auto Lp = find_lattice(ctx, lattice_id);
    auto Qp = find_qset(ctx, qset_id);
    if (!Lp || !Qp) return fail(ctx, SMD_ENOTFOUND, "prepass: unknown lattice or q set");
    Lattice &L = *Lp;
    QSet &Qs = *Qp;
    if (Qs.lattice != lattice_id || !Qs.use_grid) return fail(ctx, SMD_EINVAL, "prepass: needs the lattice's grid q set");
    if (!Qs.fp64_ok) return fail(ctx, SMD_EINVAL, "prepass: grid too large for the FP64 transform");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const int N = L.N, G = Qs.G, Qg = G * G, Qt = Qs.Q, S = n_samples;
    cudaStream_t st = ctx->s_rk;
    // maxLocField: sum over the active shells of max|J| times the shell's
    // neighbour count (subrouts.cpp:2081-2091)
    double r0 = 0.0;
    for (int s = 0; s < 3; s++) {
        if (!L.dev.shell_on[s]) continue;
        const double jm = std::max({std::fabs(L.dev.J[s][0][0]), std::fabs(L.dev.J[s][1][1]),
                                    std::fabs(L.dev.J[s][0][1])});
        r0 += jm * L.zn[s];
    }
    const int nh = 201;
    const double box = 2.0 * r0 / (nh - 1), fc = 1.0 / box;
    if (max_field) *max_field = r0;
    DevBuf in, state, impd, series, acc, hist, win;
    CK(in.ensure((size_t)S * N * 3 * 8), "cudaMalloc");
    CK(state.ensure((size_t)S * N * 3 * 8), "cudaMalloc");
    CK(cudaMemcpyAsync(in.p, spins0, (size_t)S * N * 3 * 8, cudaMemcpyHostToDevice, st), "H2D spins");
    CK(launch_aos_to_soa(in.as<double>(), state.as<double>(), S, N, st), "aos_to_soa");
    std::vector<uint8_t> ib;
    if (imp) {
        ib.resize((size_t)S * N);
        for (size_t e = 0; e < ib.size(); e++) ib[e] = imp[e] ? 1 : 0;
        CK(impd.ensure(ib.size()), "cudaMalloc");
        CK(cudaMemcpyAsync(impd.p, ib.data(), ib.size(), cudaMemcpyHostToDevice, st), "H2D imp");
    }
    CK(hist.ensure((size_t)nh * 3 * 8), "cudaMalloc");
    CK(cudaMemsetAsync(hist.p, 0, (size_t)nh * 3 * 8, st), "memset");
    const bool gen = L.lieb_delta || imp;
    if (r0 > 0.0)
        CK(launch_field_hist(L.dev, state.as<double>(), imp ? impd.as<uint8_t>() : nullptr, S, r0, fc, nh,
                             static_cast<unsigned long long *>(hist.p), gen, st),
           "field histogram");
    // grid transforms in chunks of samples, accumulated in sample order
    const int SC = (int)std::max<size_t>(1, std::min<size_t>((size_t)S, ((size_t)1 << 30) / ((size_t)48 * Qt)));
    CK(series.ensure((size_t)3 * Qt * SC * 16), "cudaMalloc");
    CK(acc.ensure((size_t)3 * Qg * 8), "cudaMalloc");
    CK(cudaMemsetAsync(acc.p, 0, (size_t)3 * Qg * 8, st), "memset");
    std::vector<double> ones((size_t)SC, 1.0);
    CK(win.ensure((size_t)SC * 8), "cudaMalloc");
    CK(cudaMemcpyAsync(win.p, ones.data(), (size_t)SC * 8, cudaMemcpyHostToDevice, st), "H2D");
    int launches = 0;
    for (int s0 = 0; s0 < S; s0 += SC) {
        const int n = std::min(SC, S - s0);
        ProjArgs pa{};
        pa.L = &L;
        pa.Qs = &Qs;
        pa.prec = SMD_FP64;
        pa.N = N;
        pa.W = 1;
        pa.R = n;
        pa.rb = 0;
        pa.re = n;
        pa.n_rec = n;
        pa.nqb = Qt;
        pa.snap = state.as<double>() + (size_t)s0 * 3 * N;
        pa.win = win.as<double>();
        pa.series = series.p;
        pa.gscratch = &ctx->gscratch;
        pa.status = nullptr;
        int rc = project_chunk(ctx, pa, st, &launches);
        if (rc) return rc;
        CK(launch_static_sf(series.p, Qg, Qt, n, 10.0 /* spec0Max, subrouts.cpp:393 */, acc.as<double>(), st),
           "static SF");
    }
    CK(launch_scale(acc.as<double>(), (size_t)3 * Qg, 1.0 / std::max(S - 1, 1), st), "scale");
    CK(cudaMemcpyAsync(sf_out, acc.p, (size_t)3 * Qg * 8, cudaMemcpyDeviceToHost, st), "D2H");
    std::vector<unsigned long long> hh((size_t)nh * 3);
    CK(cudaMemcpyAsync(hh.data(), hist.p, hh.size() * 8, cudaMemcpyDeviceToHost, st), "D2H");
    CK(cudaStreamSynchronize(st), "sync");
    for (size_t e = 0; e < hh.size(); e++) hist_out[e] = (long long)hh[e];
    return SMD_OK;
}
