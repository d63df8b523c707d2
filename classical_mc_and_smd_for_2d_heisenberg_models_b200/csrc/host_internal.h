// host_internal.h -- host-side objects shared by the library's C++ units
// (host.cu: context, lattices, q sets, single-job pipeline; batch.cu:
// batched multi-lattice jobs; serve.cpp: the serving engine).
#pragma once

#include "../../include/smd_b200.h"
#include "rk_cluster.cuh"
#include "smd_launch.h"

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace smdh {

using smd::ClusterParams;
using smd::FFTPlan;
using smd::LatticeDev;

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    // stream-ordered allocation from a memory pool (serving engine): freed
    // on `st` after the work queued there
    cudaMemPool_t pool = nullptr;
    cudaStream_t st = nullptr;
    ~DevBuf() { release(); }
    void release()
    {
        if (p) {
            if (pool) cudaFreeAsync(p, st);
            else cudaFree(p);
        }
        p = nullptr;
        bytes = 0;
    }
    // exactly b bytes from `pool`, ordered on stream s (no headroom)
    cudaError_t ensure_async(size_t b, cudaMemPool_t mp, cudaStream_t s)
    {
        if (b <= bytes && pool == mp) return cudaSuccess;
        release();
        pool = mp;
        st = s;
        cudaError_t e = cudaMallocFromPoolAsync(&p, b, mp, s);
        if (e == cudaSuccess) bytes = b;
        else p = nullptr;
        return e;
    }
    cudaError_t ensure(size_t b)
    {
        if (b <= bytes) return cudaSuccess;
        release();
        // below 1 GB, a quarter of headroom: a stream of growing jobs then
        // reallocates (and synchronises the device) rarely
        if (b < ((size_t)1 << 30)) b = (b + b / 4 + ((size_t)2 << 20) - 1) & ~(((size_t)2 << 20) - 1);
        cudaError_t e = cudaMalloc(&p, b);
        if (e == cudaSuccess) bytes = b;
        else p = nullptr;
        return e;
    }
    template <typename T>
    T *as() const { return static_cast<T *>(p); }
};

// Partition of one lattice over a cluster of CS CTAs (see rk_cluster.cuh).
struct ClusterTab {
    ClusterParams P{};
    DevBuf own_base, own_cnt, halo_cnt, halo_gid, idx, push;
};

struct Lattice {
    int N = 0, G = 0, zn[3] = {0, 0, 0}, zoff[3] = {0, 0, 0}, ztot = 0;
    bool lieb_delta = false;
    bool vac_only = true;           // impurities (if any) have zero couplings
    LatticeDev dev{};
    DevBuf nbr, grid_map, bonds;
    std::vector<double> pos;
    std::vector<int> nbr_h[3];      // host copies of the active shells' tables
    std::map<std::pair<int, int>, std::unique_ptr<ClusterTab>> ctabs;   // keyed by (CTAs per sample, edge slots)
    std::mutex cache_mu;            // guards ctabs
};

struct QSet {
    int lattice = -1;
    int use_grid = 0;
    int G = 0;
    int n_list = 0;
    int Q = 0;
    double list_scale = 1.0;
    int fp64_ok = 1;           // the FP64 grid transform fits (one block or two passes)
    int large[2] = {0, 0};     // per precision (0 FP64, 1 FP32): two-pass transform
    FFTPlan gplan{};
    DevBuf tw64, tw32;        // grid twiddles
    DevBuf phase64;           // [N][n_list] complex (FP64 list projection)
    // tensor-core operand of the FP32 form: rows 2l / 2l + 1 hold
    // scale cos(q_l . r_k) / -scale sin(q_l . r_k), split into bf16 high and
    // low parts, row pitch kp
    int kp = 0;
    DevBuf bhi, blo;
    CUtensorMap map_bhi{}, map_blo{};
};

struct Plan {
    FFTPlan p{};
    DevBuf tw64, tw32;
};

// Snapshot buffers between the integration and projection streams: the RK
// launch of chunk c reuses the buffer of chunk c - kSnapBufs, so the
// projection has kSnapBufs - 1 RK launches' time to catch up before the
// integration waits for it.
constexpr int kSnapBufs = 3;

struct Batch;   // batch.cu

}  // namespace smdh

struct smd_ctx {
    int device = 0;
    size_t budget = 0;
    cudaStream_t s_rk = nullptr, s_proj = nullptr;
    cudaEvent_t ev_rk[smdh::kSnapBufs]{}, ev_proj[smdh::kSnapBufs]{};
    cudaEvent_t ev_tf[3]{};   // per-component time transforms done (host copy may start)
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    std::string err;
    int next_id = 1;
    // lattices and q sets are shared with the serving lanes' contexts
    // (smd_share_objects); maps_mu guards the maps
    std::mutex maps_mu;
    std::map<int, std::shared_ptr<smdh::Lattice>> lattices;
    std::map<int, std::shared_ptr<smdh::QSet>> qsets;
    std::map<int, std::unique_ptr<smdh::Plan>> tplans;   // keyed by n
    std::map<int, std::shared_ptr<smdh::Batch>> batches;   // batched jobs (batch.cu)
    // job buffers (grow-only)
    smdh::DevBuf state, s0, imp, snap[smdh::kSnapBufs], series, qss, stats, e0, status, win, acc_tmp, in_tmp, out_tmp;
    smdh::DevBuf gscratch;   // packed row-transformed grids of the two-pass grid transform
    smdh::DevBuf qpart;      // cluster kernel: per-CTA autocorrelation partials [W][n_rec][CS]
    int launches = 0;
    std::vector<cudaEvent_t> tev;   // timing events, reused across calls
    // split-BF16 snapshot rows and their tensor maps, one pair per snapshot
    // buffer
    smdh::DevBuf ahi[smdh::kSnapBufs], alo[smdh::kSnapBufs];
    CUtensorMap map_ahi[smdh::kSnapBufs]{}, map_alo[smdh::kSnapBufs]{};
    const void *map_a_base[smdh::kSnapBufs]{};
    int map_a_rows[smdh::kSnapBufs]{}, map_a_kp[smdh::kSnapBufs]{};
};


namespace smdh {

int fail(smd_ctx *c, int code, const std::string &msg);
int cuda_fail(smd_ctx *c, cudaError_t e, const char *where);

#define CK(expr, where)                                          \
    do {                                                         \
        cudaError_t _e = (expr);                                 \
        if (_e != cudaSuccess) return smdh::cuda_fail(ctx, _e, where); \
    } while (0)

// Radices of an FFT of length n (wide: radix 16 and 8 first).
bool make_plan(int n, FFTPlan &p, bool wide);
cudaError_t upload_twiddles(int n, DevBuf &d64, DevBuf &d32);
// Time-transform plan of length n, built once per context.
int time_plan(smd_ctx *ctx, int n, Plan **out);
// Partition of lattice L over CS CTAs with at least zt_min edge slots per
// site (padded with the zero slot); cached per lattice.  Null when the
// lattice does not fit the cluster kernel's limits.
ClusterTab *cluster_tables(Lattice &L, int CS, int zt_min = 0);
// Lattice and q-set objects by id (null when unknown).
std::shared_ptr<Lattice> find_lattice(smd_ctx *ctx, int id);
std::shared_ptr<QSet> find_qset(smd_ctx *ctx, int id);
// Whether the cluster kernel covers the lattice (field-identity energies,
// no Lieb d-wave term, impurities only as vacancies).
bool cluster_ok(const Lattice &L);
// Return the serving engine's pooled device memory that no sample group
// holds (a no-op without an engine), for a context's own jobs when the
// device is short.
void engine_trim(smd_ctx *ctx);
// Cluster partition, sites per thread and block size the single-job path
// takes for a lattice, precision and sample count: the smallest cluster
// that puts about 85 % of the SMs to work within the shared-memory and
// register limits.  Null when the lattice needs the single-CTA kernel.
ClusterTab *cluster_choice(Lattice &L, int prec, int n_samples, int device, int *spt, int *threads);

// Projection of records [rb, re) of W samples from a snapshot buffer
// ([W][R][3][N] of the precision's type) into the windowed time series;
// the FP32 form with list q also reads the split-BF16 rows (written by the
// RK kernel when fused_split, else split here).  Adds its launches to
// *launches.
struct ProjArgs {
    Lattice *L;
    QSet *Qs;
    int prec, N, W, R, rb, re, n_rec, nqb;
    const void *snap;
    void *ahi, *alo;
    const CUtensorMap *map_ahi, *map_alo;
    bool fused_split;
    const double *win;
    void *series;
    DevBuf *gscratch;
    int *status;
};
int project_chunk(smd_ctx *ctx, const ProjArgs &a, cudaStream_t st, int *launches);

}  // namespace smdh
