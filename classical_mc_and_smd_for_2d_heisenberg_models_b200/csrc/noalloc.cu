// noalloc.cu -- RK evolution that allocates no device memory.
//
// Who needs this: callers that own every byte of device memory themselves and
// may not call cudaMalloc from our library -- a framework whose memory pool
// holds the whole HBM budget, or a real-time loop that forbids allocation
// (and the device-wide synchronisation cudaMalloc/cudaFree can imply) once it
// has started.  They pass device buffers for the spins and the neighbour
// table; the working memory the RK kernel needs beyond those (SoA spin state,
// initial spins, the two record snapshots, energies, autocorrelation and a
// status word) comes from one file-scope static device array instead of
// cudaMalloc.
//
// The array is SMD_NOALLOC_SCRATCH_BYTES (16 MiB) and lives on every GPU
// that loads the library until the process exits.  Its address is looked up
// with cudaGetSymbolAddress once per device, by the first call on that
// device (with that device current); make that first call before any stream
// capture.  All calls share the array and it keeps the last call's contents,
// so calls whose work overlaps on the GPU (different streams, or several
// host threads) race on it and must be serialised by the caller.
#include "../../include/smd_b200.h"
#include "smd_launch.h"

#include <cuda_runtime.h>

#include <mutex>

using namespace smd;

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[SMD_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_ptr[kMaxDevices] = {};

size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

// Bytes of static scratch a call with S samples of N sites uses.
size_t scratch_bytes(long long S, long long N)
{
    return up256((size_t)S * 3 * N * 8) * 2       // state, initial spins
           + up256((size_t)S * 2 * 3 * N * 8)     // two record snapshots
           + up256((size_t)S * 2 * 8)             // autocorrelation
           + up256((size_t)S * 4 * 8)             // energy statistics
           + up256((size_t)S * 8)                 // initial energies
           + 256;                                 // status word
}

}  // namespace

extern "C" int smd_evolve_fp64_noalloc(const smd_noalloc_model *m, int n_samples, double dt,
                                       int nsteps, const double *d_spins_in, double *d_spins_out,
                                       int *d_status, void *stream)
{
    if (!m || !m->d_nbr || !d_spins_in || !d_spins_out) return SMD_EINVAL;
    if (m->N <= 0 || n_samples <= 0 || nsteps < 1 || !(dt > 0.0)) return SMD_EINVAL;
    int ztot = 0;
    for (int s = 0; s < 3; s++) {
        if (m->zn[s] < 0 || m->zn[s] > kMaxShellNb) return SMD_EINVAL;
        ztot += m->zn[s];
    }
    if (ztot == 0 || m->N > rk_max_sites(SMD_FP64)) return SMD_EINVAL;
    if (n_samples > 65535) return SMD_EINVAL;
    if (scratch_bytes(n_samples, m->N) > (size_t)SMD_NOALLOC_SCRATCH_BYTES) return SMD_ENOMEM_ADMIT;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return SMD_ECUDA;
    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_ptr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return SMD_ECUDA;
            g_ptr[dev] = static_cast<unsigned char *>(p);
        }
        base = g_ptr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t S = n_samples, N = m->N;
    unsigned char *q = base;
    double *state = reinterpret_cast<double *>(q);  q += up256(S * 3 * N * 8);
    double *s0 = reinterpret_cast<double *>(q);     q += up256(S * 3 * N * 8);
    double *snap = reinterpret_cast<double *>(q);   q += up256(S * 2 * 3 * N * 8);
    double *qss = reinterpret_cast<double *>(q);    q += up256(S * 2 * 8);
    double *stats = reinterpret_cast<double *>(q);  q += up256(S * 4 * 8);
    double *e0 = reinterpret_cast<double *>(q);     q += up256(S * 8);
    // the kernel's status bits go to the caller's word when one is given,
    // else to the array's; it is the only word read before it is written
    int *status = d_status ? d_status : reinterpret_cast<int *>(q);
    if (cudaMemsetAsync(status, 0, sizeof(int), st) != cudaSuccess) return SMD_ECUDA;

    LatticeDev L{};
    L.N = m->N;
    int z = 0;
    for (int s = 0; s < 3; s++) {
        L.zn[s] = m->zn[s];
        L.zoff[s] = z;
        z += m->zn[s];
        L.shell_on[s] = m->zn[s] > 0;
        L.J[s][0][0] = m->J[s];
        L.Jf[s][0][0] = (float)m->J[s];
        for (int c = 0; c < 3; c++) {
            L.lam[s][c] = m->lambda[s][c];
            L.lamf[s][c] = (float)m->lambda[s][c];
            L.coef[s][c] = m->J[s] * m->lambda[s][c];
            L.coeff[s][c] = (float)L.coef[s][c];
        }
    }
    L.ztot = z;
    L.nbr = m->d_nbr;
    L.h = (m->h > 1.0e-12 || m->h < -1.0e-12) ? m->h : 0.0;
    L.hf = (float)L.h;
    L.energy_from_field = 1;

    if (launch_aos_to_soa(d_spins_in, state, n_samples, m->N, st) != cudaSuccess) return SMD_ECUDA;
    if (cudaMemcpyAsync(s0, state, S * 3 * N * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return SMD_ECUDA;
    RKJob J{};
    J.n_samples = n_samples;
    J.dt = dt;
    J.stride = nsteps;
    J.rec_begin = 0;
    J.rec_end = 2;
    J.n_rec = 2;
    J.fix_every = 1;
    J.state = state;
    J.s0 = s0;
    J.e0 = e0;
    J.imp = nullptr;
    J.snap = snap;
    J.snap_R = 2;
    J.qss = qss;
    J.stats = stats;
    J.status = status;
    if (launch_rk(L, J, SMD_FP64, false, st) != cudaSuccess) return SMD_ECUDA;
    if (launch_soa_to_aos(state, d_spins_out, n_samples, m->N, st) != cudaSuccess) return SMD_ECUDA;
    return SMD_OK;
}
