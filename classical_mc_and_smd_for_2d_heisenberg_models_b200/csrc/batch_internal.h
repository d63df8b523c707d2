// batch_internal.h -- samples of a job resident in HBM between launches,
// shared by the batched form (batch.cu) and the serving engine (engine.cu).
#pragma once

#include "host_internal.h"

namespace smdh {

// One job's samples resident in HBM: a member of a batch, or a sample group
// of a served job.  Carries its job's parameters, so members of different
// jobs (different n_rec, stride, dt, correction period, record chunk) can
// share one persistent RK launch.
struct Member {
    std::shared_ptr<Lattice> L;
    std::shared_ptr<QSet> Qs;
    int prec = 1, n_rec = 0, stride = 1, fix_every = 1, R = 0, nchunks = 0;
    double dt = 0.0;
    Plan *tp = nullptr;
    const double *d_win = nullptr;   // window [n_rec] on the device
    int *d_status = nullptr;         // status word of the member's kernels
    int S = 0, Sp = 0;               // real and padded samples (padding fills the last work item)
    int N = 0, Q = 0, nqb = 0;
    int vcs = 1;                     // CTAs per sample
    bool tc_list = false;            // FP32 list projection on tensor cores (RK writes the bf16 rows)
    std::vector<uint8_t> imp;        // [Sp][N] impurity flags, or empty
    DevBuf state, s0, impd, snap[kSnapBufs], ahi[kSnapBufs], alo[kSnapBufs], series, qss, qpart, stats, e0,
        gscratch;
    CUtensorMap map_ahi[kSnapBufs]{}, map_alo[kSnapBufs]{};
};

// Fill the member's derived fields (N, Q, nqb, tc_list, R when 0, nchunks,
// the time plan) from its lattice, q set and job parameters; EINVAL for
// jobs the batched kernels do not take.
int member_setup(smd_ctx *ctx, Member &mb);
// Device bytes a member of Sp padded samples holds.
size_t member_bytes(const Member &mb, int Sp);
// Allocate the member's buffers (cudaMalloc, or stream-ordered from `pool`
// on stream `st` when pool is set) and upload its impurity flags.
int member_alloc(smd_ctx *ctx, Member &mb, cudaMemPool_t pool, cudaStream_t st);
// RK job of records [rb, re) into snapshot buffer b.
smd::RKJob member_job(const Member &mb, int rb, int re, int b);
// Projection of chunk c (records [c R, min(n_rec, (c + 1) R)), snapshot
// buffer c mod 3) into the member's time series.
int member_project(smd_ctx *ctx, Member &mb, int c, cudaStream_t st, int *launches);
// Time transform and autocorrelation of the member's samples, added into
// acc [3][Q][n_rec] and accq [n_rec].
int member_finish(smd_ctx *ctx, Member &mb, double *acc, double *accq, cudaStream_t st, int *launches);
// Spins [S][N][3] (device) into the member's state and initial spins;
// padded samples repeat the last sample.
int member_load(smd_ctx *ctx, Member &mb, const double *d_spins, cudaStream_t st, int *launches);

// Work items (slot, first sample) of one launch over members with CTAs per
// sample vcs[i] in clusters of csh CTAs (csh / vcs[i] samples per item),
// the costliest members first.
std::vector<int2> make_items(const std::vector<Member *> &m, const std::vector<int> &vcs, int csh);
// One persistent RK launch over members m, member i at its chunk chunk[i]
// (records [chunk R, ...) into snapshot buffer chunk mod 3); every member's
// vcs must divide csh.
int launch_rk_members(smd_ctx *ctx, const std::vector<Member *> &m, const std::vector<int> &chunk, int prec,
                      int zt, int spt, int threads, int csh, int nclusters, size_t smem, const int2 *d_items,
                      int n_items, int *d_queue, cudaStream_t st);
int zt_of(int z);
// Clusters of a persistent RK launch: at most maxc, leaving SMD_RK_RESERVE_SMS
// SMs (default 16) to the projections that run beside it.
int rk_cluster_cap(int maxc, int csh);

// CTAs per sample of a member for a sites-per-thread value: the fewest (a
// power of two) whose share of the sites fits a CTA of the batch kernel and
// the shared memory; 0 when none does.
int member_ctas(Member &mb, int spt, int zt, size_t *smem);

}  // namespace smdh
