// batch.cu -- batched jobs over several lattices (smd_batch_*).
//
// The reference integrates one lattice per run, one sample at a time
// (Codes_Folder/smd_code.cpp:3079-3311, get_dynSpectrum per sample).  A batch
// holds several such jobs ("members", one lattice and q set each) resident
// in HBM and runs every member's samples through one pipeline:
//
//   per chunk of R records
//     stream rk   : ONE persistent RK launch for all members -- thread-block
//                   clusters of CSH CTAs pull (member, first sample) items
//                   from a device queue (largest per-CTA work first); a
//                   member partitioned over CS CTAs runs CSH / CS samples
//                   per item
//     stream proj : per member, the grid / list projection of the chunk
//   after the last chunk, per member: time transform, autocorrelation sums
//
// The job step is captured once into a CUDA graph and replayed.  The
// autotuner (tune()) times the feasible (sites per thread, cluster size)
// configurations on a short integration of the batch's own lattices and
// keeps the fastest per batch shape.
#include "batch_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

using namespace smd;

namespace smdh {

// ------------------------------------------------------------ members

int member_setup(smd_ctx *ctx, Member &mb)
{
    if (!cluster_ok(*mb.L))
        return fail(ctx, SMD_EINVAL, "member lattice needs the single-CTA kernel (use smd_run)");
    if (mb.Qs->use_grid && mb.prec == SMD_FP64 && !mb.Qs->fp64_ok)
        return fail(ctx, SMD_EINVAL, "grid too large for the FP64 transform");
    if (mb.n_rec < 2 || mb.stride < 1 || !(mb.dt > 0.0)) return fail(ctx, SMD_EINVAL, "n_rec, stride or dt");
    if ((long long)(mb.n_rec - 1) * mb.stride > 2000000000LL) return fail(ctx, SMD_EINVAL, "too many steps");
    mb.N = mb.L->N;
    mb.Q = mb.Qs->Q;
    mb.nqb = (mb.Q + series_qblock(mb.prec) - 1) / series_qblock(mb.prec);
    mb.tc_list = mb.Qs->n_list > 0 && mb.prec == SMD_FP32;
    if (mb.fix_every < 1) mb.fix_every = 1;
    if (mb.R <= 0) mb.R = std::min(mb.n_rec, 128);
    mb.R = std::min(mb.R, mb.n_rec);
    mb.nchunks = (mb.n_rec + mb.R - 1) / mb.R;
    int rc = time_plan(ctx, mb.n_rec, &mb.tp);
    if (rc) return rc;
    if (!time_fft_fits(mb.n_rec, mb.prec, mb.tp->p))
        return fail(ctx, SMD_EINVAL, "n_rec too long for the shared-memory time transform");
    return SMD_OK;
}

size_t member_bytes(const Member &mb, int Sp)
{
    const size_t N = mb.N, R = mb.R, n = mb.n_rec, elem = mb.prec == SMD_FP64 ? 8 : 4;
    size_t b = (size_t)Sp * 3 * N * 16 + (size_t)Sp * N;
    b += kSnapBufs * ((size_t)Sp * R * 3 * N * elem + (mb.tc_list ? (size_t)Sp * R * 3 * mb.Qs->kp * 4 : 0));
    b += (size_t)mb.S * 3 * n * mb.nqb * 16 + (size_t)Sp * n * (8 + kMaxClusterCTAs * 8) + (size_t)Sp * 40;
    if (mb.Qs->use_grid && mb.Qs->large[mb.prec == SMD_FP64 ? 0 : 1])
        b += (size_t)mb.S * grid_large_scratch(mb.Qs->G, mb.R, mb.prec == SMD_FP64 ? 0 : 1);
    return b;
}

int member_alloc(smd_ctx *ctx, Member &mb, cudaMemPool_t pool, cudaStream_t st)
{
    const size_t N = mb.N, Sp = mb.Sp, R = mb.R, n = mb.n_rec;
    const size_t elem = mb.prec == SMD_FP64 ? 8 : 4;
    auto get = [&](DevBuf &d, size_t bytes) {
        return pool ? d.ensure_async(bytes, pool, st) : d.ensure(bytes);
    };
    CK(get(mb.state, Sp * 3 * N * 8), "alloc");
    CK(get(mb.s0, Sp * 3 * N * 8), "alloc");
    if (!mb.imp.empty()) {
        CK(get(mb.impd, Sp * N), "alloc");
        CK(cudaMemcpyAsync(mb.impd.p, mb.imp.data(), Sp * N, cudaMemcpyHostToDevice, st), "H2D imp");
        CK(cudaStreamSynchronize(st), "sync");   // the host flags may change after the call
    }
    for (int b = 0; b < kSnapBufs; b++) {
        CK(get(mb.snap[b], Sp * R * 3 * N * elem), "alloc");
        if (mb.tc_list) {
            const size_t ab = Sp * R * 3 * (size_t)mb.Qs->kp * 2;
            CK(get(mb.ahi[b], ab), "alloc");
            CK(get(mb.alo[b], ab), "alloc");
            // the padding columns past N stay zero
            CK(cudaMemsetAsync(mb.ahi[b].p, 0, ab, st), "memset");
            CK(cudaMemsetAsync(mb.alo[b].p, 0, ab, st), "memset");
            if (!make_bf16_map(&mb.map_ahi[b], mb.ahi[b].p, (int)(Sp * R * 3), mb.Qs->kp, tc_bm()) ||
                !make_bf16_map(&mb.map_alo[b], mb.alo[b].p, (int)(Sp * R * 3), mb.Qs->kp, tc_bm()))
                return fail(ctx, SMD_ECUDA, "tensor map encoding failed");
        }
    }
    CK(get(mb.series, (size_t)mb.S * 3 * n * mb.nqb * 16), "alloc series");
    CK(get(mb.qss, Sp * n * 8), "alloc");
    CK(get(mb.qpart, Sp * n * kMaxClusterCTAs * 8), "alloc");
    CK(get(mb.stats, Sp * 4 * 8), "alloc");
    CK(get(mb.e0, Sp * 8), "alloc");
    if (mb.Qs->use_grid && mb.Qs->large[mb.prec == SMD_FP64 ? 0 : 1])
        CK(get(mb.gscratch, (size_t)mb.S * grid_large_scratch(mb.Qs->G, mb.R, mb.prec == SMD_FP64 ? 0 : 1)),
           "alloc");
    return SMD_OK;
}

RKJob member_job(const Member &mb, int rb, int re, int b)
{
    RKJob J{};
    J.n_samples = mb.Sp;
    J.dt = mb.dt;
    J.stride = mb.stride;
    J.rec_begin = rb;
    J.rec_end = re;
    J.n_rec = mb.n_rec;
    J.fix_every = mb.fix_every;
    J.state = mb.state.as<double>();
    J.s0 = mb.s0.as<double>();
    J.e0 = mb.e0.as<double>();
    J.imp = mb.imp.empty() ? nullptr : mb.impd.as<uint8_t>();
    J.snap = mb.snap[b].p;
    J.snap_R = mb.R;
    J.qss = mb.qss.as<double>();
    J.stats = mb.stats.as<double>();
    J.status = mb.d_status;
    J.bf_hi = mb.tc_list ? mb.ahi[b].p : nullptr;
    J.bf_lo = mb.tc_list ? mb.alo[b].p : nullptr;
    J.bf_kp = mb.Qs->kp;
    J.qpart = mb.qpart.as<double>();
    return J;
}

int member_project(smd_ctx *ctx, Member &mb, int c, cudaStream_t st, int *launches)
{
    const int b = c % kSnapBufs;
    ProjArgs pa{};
    pa.L = mb.L.get();
    pa.Qs = mb.Qs.get();
    pa.prec = mb.prec;
    pa.N = mb.N;
    pa.W = mb.S;
    pa.R = mb.R;
    pa.rb = c * mb.R;
    pa.re = std::min(mb.n_rec, (c + 1) * mb.R);
    pa.n_rec = mb.n_rec;
    pa.nqb = mb.nqb;
    pa.snap = mb.snap[b].p;
    pa.ahi = mb.ahi[b].p;
    pa.alo = mb.alo[b].p;
    pa.map_ahi = &mb.map_ahi[b];
    pa.map_alo = &mb.map_alo[b];
    pa.fused_split = mb.tc_list;
    pa.win = mb.d_win;
    pa.series = mb.series.p;
    pa.gscratch = &mb.gscratch;
    pa.status = mb.d_status;
    return project_chunk(ctx, pa, st, launches);
}

int member_finish(smd_ctx *ctx, Member &mb, double *acc, double *accq, cudaStream_t st, int *launches)
{
    const void *tw = mb.prec == SMD_FP64 ? mb.tp->tw64.p : mb.tp->tw32.p;
    CK(launch_time_fft(mb.series.p, mb.prec, mb.S, mb.Q, mb.nqb, mb.tp->p, tw, acc, mb.d_status, st),
       "time fft");
    CK(launch_qss_from_parts(mb.qpart.as<double>(), mb.S, mb.n_rec, mb.vcs, mb.N, mb.qss.as<double>(), st),
       "qss");
    CK(launch_sum_rows(mb.qss.as<double>(), mb.S, mb.n_rec, accq, st), "qss");
    *launches += 3;
    return SMD_OK;
}

int member_load(smd_ctx *ctx, Member &mb, const double *d_spins, cudaStream_t st, int *launches)
{
    const size_t blk = 3 * (size_t)mb.N;
    CK(launch_aos_to_soa(d_spins, mb.state.as<double>(), mb.S, mb.N, st), "aos_to_soa");
    *launches += 1;
    for (int s = mb.S; s < mb.Sp; s++)
        CK(cudaMemcpyAsync(mb.state.as<double>() + (size_t)s * blk, mb.state.as<double>() + (size_t)(mb.S - 1) * blk,
                           blk * 8, cudaMemcpyDeviceToDevice, st),
           "D2D pad");
    CK(cudaMemcpyAsync(mb.s0.p, mb.state.p, (size_t)mb.Sp * blk * 8, cudaMemcpyDeviceToDevice, st), "D2D");
    return SMD_OK;
}

int member_ctas(Member &mb, int spt, int zt, size_t *smem)
{
    const int threads = rk_batch_threads(mb.prec, spt);
    for (int v = 1; v <= kMaxClusterCTAs; v *= 2) {
        if ((mb.N + v - 1) / v > spt * threads || mb.N < v) continue;
        ClusterTab *t = cluster_tables(*mb.L, v, zt);
        if (!t) continue;
        const size_t sm = rk_cluster_smem(t->P, mb.prec);
        if (sm > 227 * 1024) continue;
        if (smem) *smem = sm;
        return v;
    }
    return 0;
}

// Clusters of a persistent RK launch: as many as fit the device at once
// (maxc), less the clusters that would take the last `reserve` SMs.  The
// projections of the previous chunk run on those SMs beside the RK launch,
// as they do beside the single-job cluster kernel (whose samples leave SMs
// free); without them the projections wait for the persistent launch to
// drain.  SMD_RK_RESERVE_SMS sets the reserve (default 16 of 148).
int rk_cluster_cap(int maxc, int csh)
{
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm <= 0) nsm = 148;
    const char *e = std::getenv("SMD_RK_RESERVE_SMS");
    const int reserve = e ? std::max(0, std::atoi(e)) : 16;
    const int cap = std::max(1, (nsm - reserve) / std::max(1, csh));
    return std::min(maxc, cap);
}

// ------------------------------------------------------------ batches

struct Config {
    int spt = 0, threads = 0, csh = 0, nclusters = 0;
    std::vector<int> vcs;   // per member
    size_t smem = 0;
};

struct Batch {
    int prec = SMD_FP32, n_rec = 0, zt = 8, nchunks = 0;
    std::vector<std::unique_ptr<Member>> m;
    std::vector<std::unique_ptr<DevBuf>> acc, accq;   // per member: sums over its samples
    Config cfg;
    smd_batch_tuning info{};
    std::vector<int2> items_h;
    DevBuf items, queue, win, status;
    cudaStream_t s_rk = nullptr, s_proj = nullptr;   // the context's streams
    cudaEvent_t ev_rk[kSnapBufs]{}, ev_proj[kSnapBufs]{}, ev_fork = nullptr, ev_join = nullptr;
    std::vector<cudaEvent_t> tev;   // timing events of an eager run
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int runs = 0, launches_per_step = 0;
    ~Batch()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (int b = 0; b < kSnapBufs; b++) {
            if (ev_rk[b]) cudaEventDestroy(ev_rk[b]);
            if (ev_proj[b]) cudaEventDestroy(ev_proj[b]);
        }
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        for (cudaEvent_t e : tev) cudaEventDestroy(e);
    }
};

static_assert(sizeof(BatchParams) <= 32000, "batch parameters exceed the kernel-parameter limit");

int zt_of(int z) { return z <= 8 ? 8 : z <= 12 ? 12 : z <= 18 ? 18 : z <= 20 ? 20 : -1; }

// Work items of one launch: (slot, first sample) for every member, CSH / CS
// samples per item, members with the most sites per CTA first (their items
// take longest, so the queue ends on short items).
std::vector<int2> make_items(const std::vector<Member *> &m, const std::vector<int> &vcs, int csh)
{
    std::vector<int> order(m.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
    auto cost = [&](int i) {
        return (double)((m[i]->N + vcs[i] - 1) / vcs[i]) * (double)m[i]->R * (double)m[i]->stride;
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    std::vector<int2> it;
    for (int i : order) {
        const int per = csh / vcs[i];
        const int Sp = (m[i]->S + per - 1) / per * per;
        for (int f = 0; f < Sp; f += per) it.push_back(make_int2(i, f));
    }
    return it;
}

// One persistent RK launch over members m, each at its own chunk chunk[i]
// (records [chunk R, ...) into snapshot buffer chunk mod 3).
int launch_rk_members(smd_ctx *ctx, const std::vector<Member *> &m, const std::vector<int> &chunk, int prec,
                      int zt, int spt, int threads, int csh, int nclusters, size_t smem, const int2 *d_items,
                      int n_items, int *d_queue, cudaStream_t st)
{
    BatchParams P{};
    P.n_slots = (int)m.size();
    P.n_items = n_items;
    P.items = d_items;
    P.queue = d_queue;
    for (size_t i = 0; i < m.size(); i++) {
        Member &mb = *m[i];
        ClusterTab *t = cluster_tables(*mb.L, mb.vcs, zt);
        if (!t) return fail(ctx, SMD_EINVAL, "batch: lattice does not fit the cluster kernel");
        const int c = chunk[i], rb = c * mb.R, re = std::min(mb.n_rec, rb + mb.R);
        P.slot[i].P = t->P;
        P.slot[i].J = member_job(mb, rb, re, c % kSnapBufs);
    }
    CK(launch_rk_batch(P, prec, spt, zt, threads, csh, nclusters, smem, st), "batch RK kernel");
    return SMD_OK;
}

namespace {

// Autotuner choices per batch shape (precision, edge slots, record chunk,
// stride and every member's size), kept for the life of the process.
std::mutex g_tune_mu;
std::map<std::string, Config> g_tuned;

std::vector<Member *> raw(const Batch &B)
{
    std::vector<Member *> r;
    for (auto &mp : B.m) r.push_back(mp.get());
    return r;
}

// Feasible configurations: for each sites-per-thread value, every member
// takes the fewest CTAs per sample that fit; the cluster is the largest
// member's CTA count or twice it (more samples of small members per item).
// SMD_BATCH_SPT / SMD_BATCH_CLUSTER restrict the search to one value.
std::vector<Config> candidates(Batch &B)
{
    std::vector<Config> out;
    int f_spt = 0, f_csh = 0;
    if (const char *e = std::getenv("SMD_BATCH_SPT")) f_spt = std::atoi(e);
    if (const char *e = std::getenv("SMD_BATCH_CLUSTER")) f_csh = std::atoi(e);
    for (int spt : {2, 4}) {
        if (f_spt && spt != f_spt) continue;
        Config base;
        base.spt = spt;
        base.threads = rk_batch_threads(B.prec, spt);
        bool ok = true;
        int vmax = 1;
        for (auto &mp : B.m) {
            size_t sm = 0;
            const int v = member_ctas(*mp, spt, B.zt, &sm);
            if (!v) {
                ok = false;
                break;
            }
            base.smem = std::max(base.smem, sm);
            base.vcs.push_back(v);
            vmax = std::max(vmax, v);
        }
        if (!ok) continue;
        std::vector<int> cshs = {vmax, 2 * vmax};
        if (f_csh) cshs = {f_csh};
        for (int csh : cshs) {
            if (csh > kMaxClusterCTAs || csh < vmax || csh % vmax) continue;
            Config c = base;
            c.csh = csh;
            c.nclusters = rk_cluster_cap(rk_batch_max_clusters(B.prec, spt, B.zt, c.threads, csh, c.smem), csh);
            if (c.nclusters > 0) out.push_back(c);
        }
    }
    return out;
}

std::string shape_key(const Batch &B)
{
    std::ostringstream k;
    const char *f1 = std::getenv("SMD_BATCH_SPT"), *f2 = std::getenv("SMD_BATCH_CLUSTER");
    k << B.prec << "/" << B.zt << "/" << B.m[0]->R << "/" << B.m[0]->stride << "/" << (f1 ? f1 : "") << "/"
      << (f2 ? f2 : "");
    for (auto &mp : B.m) k << "|" << mp->N << "x" << mp->S;
    return k.str();
}

void apply(Batch &B, const Config &c)
{
    for (size_t i = 0; i < B.m.size(); i++) B.m[i]->vcs = c.vcs[i];
}

// Valid spins for the autotuner's probe integration: every member's state
// set to a tilted spiral (the probe's results are discarded).
int probe_state(smd_ctx *ctx, Batch &B)
{
    for (auto &mp : B.m) {
        const size_t N = mp->N, Sp = mp->Sp;
        std::vector<double> h(Sp * 3 * N);
        for (size_t s = 0; s < Sp; s++)
            for (size_t i = 0; i < N; i++) {
                const double a = 0.7 * (double)i + 0.3 * (double)s, th = 0.4 + 0.2 * std::sin(0.3 * (double)i);
                h[(s * 3 + 0) * N + i] = std::cos(a) * std::sin(th);
                h[(s * 3 + 1) * N + i] = std::sin(a) * std::sin(th);
                h[(s * 3 + 2) * N + i] = std::cos(th);
            }
        CK(cudaMemcpy(mp->state.p, h.data(), h.size() * 8, cudaMemcpyHostToDevice), "H2D probe");
        CK(cudaMemcpy(mp->s0.p, h.data(), h.size() * 8, cudaMemcpyHostToDevice), "H2D probe");
    }
    return SMD_OK;
}

// Time each candidate's RK launch on the batch's own lattices (a few
// records from the probe state) and keep the fastest; cached per shape.
int tune(smd_ctx *ctx, Batch &B, std::vector<Config> &cands, Config &best)
{
    const std::string key = shape_key(B);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            best = it->second;
            B.info.candidates = 0;
            return SMD_OK;
        }
    }
    auto t0 = std::chrono::steady_clock::now();
    if (cands.size() == 1) {
        best = cands[0];
        B.info.candidates = 1;
    } else {
        int rc = probe_state(ctx, B);
        if (rc) return rc;
        std::vector<Member *> m = raw(B);
        std::vector<int> chunk(m.size(), 0);
        // records [0, rr) of chunk 0: R is shortened for the probe only
        std::vector<int> saveR;
        for (Member *mp : m) {
            saveR.push_back(mp->R);
            mp->R = std::min(mp->R, 9);
        }
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0), "event");
        CK(cudaEventCreate(&e1), "event");
        double best_ms = 1e300;
        for (Config &c : cands) {
            apply(B, c);
            auto it = make_items(m, c.vcs, c.csh);
            DevBuf d;
            CK(d.ensure(it.size() * sizeof(int2)), "cudaMalloc");
            CK(cudaMemcpy(d.p, it.data(), it.size() * sizeof(int2), cudaMemcpyHostToDevice), "H2D items");
            double ms_sum = 0.0;
            for (int rep = 0; rep < 3; rep++) {
                CK(cudaMemsetAsync(B.queue.p, 0, sizeof(int), B.s_rk), "memset");
                CK(cudaEventRecord(e0, B.s_rk), "event");
                rc = launch_rk_members(ctx, m, chunk, B.prec, B.zt, c.spt, c.threads, c.csh, c.nclusters, c.smem,
                                       d.as<int2>(), (int)it.size(), B.queue.as<int>(), B.s_rk);
                if (rc) return rc;
                CK(cudaEventRecord(e1, B.s_rk), "event");
                CK(cudaEventSynchronize(e1), "sync");
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0) ms_sum += ms;   // the first launch warms up
            }
            if (ms_sum < best_ms) {
                best_ms = ms_sum;
                best = c;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        for (size_t i = 0; i < m.size(); i++) m[i]->R = saveR[i];
        B.info.candidates = (int)cands.size();
    }
    B.info.probe_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[key] = best;
    return SMD_OK;
}

// One job step of the batch on the context's streams (eager, or recorded
// into a graph by stream capture).  With timing, events around every RK
// launch and the whole step go to B.tev.
int enqueue_step(smd_ctx *ctx, Batch &B, bool timing)
{
    cudaStream_t srk = B.s_rk, spr = B.s_proj;
    int launches = 0;
    if (timing) CK(cudaEventRecord(B.tev[0], srk), "event");
    CK(cudaMemsetAsync(B.queue.p, 0, (size_t)B.nchunks * sizeof(int), srk), "memset");
    CK(cudaMemsetAsync(B.status.p, 0, sizeof(int), srk), "memset");
    CK(cudaEventRecord(B.ev_fork, srk), "event");
    CK(cudaStreamWaitEvent(spr, B.ev_fork, 0), "wait");
    for (size_t i = 0; i < B.m.size(); i++) {
        CK(cudaMemsetAsync(B.acc[i]->p, 0, 3 * (size_t)B.m[i]->Q * B.n_rec * 8, spr), "memset");
        CK(cudaMemsetAsync(B.accq[i]->p, 0, (size_t)B.n_rec * 8, spr), "memset");
    }
    std::vector<Member *> m = raw(B);
    const Config &c = B.cfg;
    for (int ch = 0; ch < B.nchunks; ch++) {
        const int b = ch % kSnapBufs;
        if (ch >= kSnapBufs) CK(cudaStreamWaitEvent(srk, B.ev_proj[b], 0), "wait");
        if (timing) CK(cudaEventRecord(B.tev[2 + 2 * ch], srk), "event");
        std::vector<int> chunk(m.size(), ch);
        int rc = launch_rk_members(ctx, m, chunk, B.prec, B.zt, c.spt, c.threads, c.csh, c.nclusters, c.smem,
                                   B.items.as<int2>(), (int)B.items_h.size(), B.queue.as<int>() + ch, srk);
        if (rc) return rc;
        launches++;
        if (timing) CK(cudaEventRecord(B.tev[3 + 2 * ch], srk), "event");
        CK(cudaEventRecord(B.ev_rk[b], srk), "event");
        CK(cudaStreamWaitEvent(spr, B.ev_rk[b], 0), "wait");
        for (Member *mp : m) {
            rc = member_project(ctx, *mp, ch, spr, &launches);
            if (rc) return rc;
        }
        CK(cudaEventRecord(B.ev_proj[b], spr), "event");
    }
    CK(cudaStreamWaitEvent(spr, B.ev_rk[(B.nchunks - 1) % kSnapBufs], 0), "wait");
    for (size_t i = 0; i < m.size(); i++) {
        int rc = member_finish(ctx, *m[i], B.acc[i]->as<double>(), B.accq[i]->as<double>(), spr, &launches);
        if (rc) return rc;
    }
    if (timing) CK(cudaEventRecord(B.tev[1], spr), "event");
    CK(cudaEventRecord(B.ev_join, spr), "event");
    CK(cudaStreamWaitEvent(srk, B.ev_join, 0), "wait");
    B.launches_per_step = launches;
    return SMD_OK;
}

std::shared_ptr<Batch> find_batch(smd_ctx *ctx, int id)
{
    std::lock_guard<std::mutex> lk(ctx->maps_mu);
    auto it = ctx->batches.find(id);
    return it == ctx->batches.end() ? nullptr : it->second;
}

}  // namespace

}  // namespace smdh

using namespace smdh;

extern "C" int smd_batch_create(smd_ctx *ctx, const smd_batch_desc *d, int *batch_id)
{
    if (!ctx || !d || !batch_id || !d->members) return SMD_EINVAL;
    if (d->n_members < 1 || d->n_members > kMaxBatchSlots)
        return fail(ctx, SMD_EINVAL, "batch: 1 to 24 members");
    if (d->precision != SMD_FP32 && d->precision != SMD_FP64) return fail(ctx, SMD_EINVAL, "batch: precision");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    auto B = std::make_shared<Batch>();
    B->prec = d->precision;
    B->n_rec = d->n_rec;
    B->s_rk = ctx->s_rk;
    B->s_proj = ctx->s_proj;
    CK(B->status.ensure(sizeof(int)), "cudaMalloc");
    CK(B->win.ensure((size_t)std::max(d->n_rec, 1) * 8), "cudaMalloc");
    int zmax = 0;
    for (int i = 0; i < d->n_members; i++) {
        const smd_batch_member &mm = d->members[i];
        auto mb = std::make_unique<Member>();
        mb->L = find_lattice(ctx, mm.lattice);
        mb->Qs = find_qset(ctx, mm.qset);
        if (!mb->L || !mb->Qs) return fail(ctx, SMD_ENOTFOUND, "batch: unknown lattice or q set");
        if (mb->Qs->lattice != mm.lattice) return fail(ctx, SMD_EINVAL, "batch: q set belongs to another lattice");
        if (mm.n_samples < 1) return fail(ctx, SMD_EINVAL, "batch: n_samples < 1");
        mb->prec = d->precision;
        mb->n_rec = d->n_rec;
        mb->stride = d->stride;
        mb->fix_every = d->fix_every;
        mb->dt = d->dt;
        mb->S = mm.n_samples;
        mb->d_win = B->win.as<double>();
        mb->d_status = B->status.as<int>();
        int rc = member_setup(ctx, *mb);
        if (rc) return fail(ctx, rc, std::string("batch: ") + ctx->err);
        zmax = std::max(zmax, mb->L->zn[0] + mb->L->zn[1] + mb->L->zn[2]);
        if (mm.imp) {
            mb->imp.resize((size_t)mm.n_samples * mb->N);
            for (size_t e = 0; e < mb->imp.size(); e++) mb->imp[e] = mm.imp[e] ? 1 : 0;
        }
        B->m.push_back(std::move(mb));
    }
    B->zt = zt_of(zmax);
    if (B->zt < 0) return fail(ctx, SMD_EINVAL, "batch: more than 18 neighbours per site");
    std::vector<Config> cands = candidates(*B);
    if (cands.empty()) return fail(ctx, SMD_EINVAL, "batch: no cluster configuration fits every member");
    // records per launch: the largest of 128, 64, 32 whose buffers (with the
    // most padding any candidate needs) fit the budget
    int pad_max = 1;
    for (auto &c : cands)
        for (size_t i = 0; i < B->m.size(); i++) pad_max = std::max(pad_max, c.csh / c.vcs[i]);
    size_t need = 0;
    for (int R : {128, 64, 32}) {
        need = (size_t)64 << 20;
        for (auto &mp : B->m) {
            mp->R = std::min(mp->n_rec, R);
            need += member_bytes(*mp, mp->S + pad_max - 1) + 3 * (size_t)mp->Q * mp->n_rec * 8;
        }
        if (need <= ctx->budget) break;
    }
    if (need > ctx->budget) return fail(ctx, SMD_ENOMEM_ADMIT, "batch: members exceed the HBM budget");
    for (auto &mp : B->m) {
        mp->nchunks = (mp->n_rec + mp->R - 1) / mp->R;
        mp->Sp = mp->S + pad_max - 1;
        if (!mp->imp.empty()) {
            // padded samples repeat the last sample's flags
            const size_t N = mp->N;
            mp->imp.resize((size_t)mp->Sp * N);
            for (int s = mp->S; s < mp->Sp; s++)
                std::memcpy(&mp->imp[(size_t)s * N], &mp->imp[(size_t)(mp->S - 1) * N], N);
        }
        int rc = member_alloc(ctx, *mp, nullptr, ctx->s_rk);
        if (rc) return rc;
        B->acc.push_back(std::make_unique<DevBuf>());
        B->accq.push_back(std::make_unique<DevBuf>());
        CK(B->acc.back()->ensure(3 * (size_t)mp->Q * mp->n_rec * 8), "cudaMalloc");
        CK(B->accq.back()->ensure((size_t)mp->n_rec * 8), "cudaMalloc");
    }
    CK(cudaStreamSynchronize(ctx->s_rk), "sync");
    B->nchunks = B->m[0]->nchunks;
    CK(B->queue.ensure((size_t)std::max(B->nchunks, 1) * sizeof(int)), "cudaMalloc");
    for (int b = 0; b < kSnapBufs; b++) {
        CK(cudaEventCreateWithFlags(&B->ev_rk[b], cudaEventDisableTiming), "event");
        CK(cudaEventCreateWithFlags(&B->ev_proj[b], cudaEventDisableTiming), "event");
    }
    CK(cudaEventCreateWithFlags(&B->ev_fork, cudaEventDisableTiming), "event");
    CK(cudaEventCreateWithFlags(&B->ev_join, cudaEventDisableTiming), "event");
    {
        int rc = tune(ctx, *B, cands, B->cfg);
        if (rc) return rc;
    }
    apply(*B, B->cfg);
    B->items_h = make_items(raw(*B), B->cfg.vcs, B->cfg.csh);
    CK(B->items.ensure(B->items_h.size() * sizeof(int2)), "cudaMalloc");
    CK(cudaMemcpy(B->items.p, B->items_h.data(), B->items_h.size() * sizeof(int2), cudaMemcpyHostToDevice),
       "H2D items");
    smd_batch_tuning &t = B->info;
    t.cluster_ctas = B->cfg.csh;
    t.sites_per_thread = B->cfg.spt;
    t.threads = B->cfg.threads;
    t.edge_slots = B->zt;
    t.records_per_launch = B->m[0]->R;
    t.clusters = B->cfg.nclusters;
    t.items = (int)B->items_h.size();
    for (size_t i = 0; i < B->m.size(); i++) t.member_ctas[i] = B->cfg.vcs[i];
    while (B->tev.size() < 2 + 2 * (size_t)B->nchunks) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e), "event");
        B->tev.push_back(e);
    }
    const int id = ctx->next_id++;
    {
        std::lock_guard<std::mutex> lk(ctx->maps_mu);
        ctx->batches[id] = B;
    }
    *batch_id = id;
    return SMD_OK;
}

extern "C" int smd_batch_info(smd_ctx *ctx, int batch_id, smd_batch_tuning *out)
{
    if (!ctx || !out) return SMD_EINVAL;
    auto B = find_batch(ctx, batch_id);
    if (!B) return SMD_ENOTFOUND;
    *out = B->info;
    return SMD_OK;
}

extern "C" int smd_batch_free(smd_ctx *ctx, int batch_id)
{
    if (!ctx) return SMD_EINVAL;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    std::lock_guard<std::mutex> lk(ctx->maps_mu);
    if (!ctx->batches.erase(batch_id)) return SMD_ENOTFOUND;
    return SMD_OK;
}

namespace {

// Inputs into the members' state, then the job step: eagerly with timing on
// the first run, as a replay of the captured graph afterwards
// (SMD_BATCH_GRAPH=0 keeps it eager).
int batch_step(smd_ctx *ctx, Batch &B, const double *const *d_spins0, smd_report *rep)
{
    cudaStream_t st = B.s_rk;
    int launches = 0;
    for (size_t i = 0; i < B.m.size(); i++) {
        int rc = member_load(ctx, *B.m[i], d_spins0[i], st, &launches);
        if (rc) return rc;
    }
    bool graph_ok = true;
    if (const char *e = std::getenv("SMD_BATCH_GRAPH")) graph_ok = std::atoi(e) != 0;
    const bool eager = !graph_ok || B.runs == 0;
    if (eager) {
        int rc = enqueue_step(ctx, B, true);
        if (rc) return rc;
    } else {
        if (!B.exec) {
            CK(cudaStreamSynchronize(st), "sync");
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
            int rc = enqueue_step(ctx, B, false);
            cudaGraph_t g = nullptr;
            cudaError_t ec = cudaStreamEndCapture(st, &g);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            CK(ec, "end capture");
            B.graph = g;
            CK(cudaGraphInstantiate(&B.exec, B.graph, 0), "graph instantiate");
        }
        CK(cudaEventRecord(B.tev[0], st), "event");
        CK(cudaGraphLaunch(B.exec, st), "graph launch");
        CK(cudaEventRecord(B.tev[1], st), "event");
    }
    B.runs++;
    CK(cudaStreamSynchronize(st), "sync");
    int status = 0;
    CK(cudaMemcpy(&status, B.status.p, sizeof(int), cudaMemcpyDeviceToHost), "D2H status");
    if (rep) {
        std::memset(rep, 0, sizeof *rep);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, B.tev[0], B.tev[1]);
        rep->ms_device = ms;
        if (eager)
            for (int c = 0; c < B.nchunks; c++) {
                float m2 = 0.f;
                cudaEventElapsedTime(&m2, B.tev[2 + 2 * c], B.tev[3 + 2 * c]);
                rep->ms_rk += m2;
            }
        rep->rk_launches = B.nchunks;
        rep->rk_kind = 3;
        rep->rk_ctas = B.cfg.csh;
        rep->waves = 1;
        rep->kernel_launches = launches + B.launches_per_step;
        double ss = 0.0, dmax = 0.0, dfin = 0.0;
        for (auto &mp : B.m) {
            ss += (double)mp->N * (double)(mp->n_rec - 1) * mp->stride * mp->S;
            std::vector<double> stt((size_t)mp->S * 4);
            CK(cudaMemcpy(stt.data(), mp->stats.p, stt.size() * 8, cudaMemcpyDeviceToHost), "D2H stats");
            for (int s = 0; s < mp->S; s++) {
                dmax = std::max(dmax, stt[s * 4 + 0] / mp->N);
                dfin = std::max(dfin, std::fabs(stt[s * 4 + 1] - stt[s * 4 + 2]) / mp->N);
            }
        }
        rep->site_steps = ss;
        rep->drift_max = dmax;
        rep->drift_final = dfin;
    }
    if (status & 4) return fail(ctx, SMD_ETIMEOUT, "tensor-core projection: a bounded wait expired");
    if (status & 8) return fail(ctx, SMD_ETIMEOUT, "time transform: a bounded wait expired");
    if (status & 16) return fail(ctx, SMD_ETIMEOUT, "RK halo exchange: a bounded wait expired");
    if (status) return fail(ctx, SMD_ECUDA, "a sample reached a zero correction denominator (sigma = 0)");
    return SMD_OK;
}

}  // namespace

extern "C" int smd_batch_run_device(smd_ctx *ctx, int batch_id, const double *const *d_spins0,
                                    const double *d_window, double *const *d_spec_sum,
                                    double *const *d_qss_sum, smd_report *rep)
{
    if (!ctx || !d_spins0 || !d_window || !d_spec_sum || !d_qss_sum) return SMD_EINVAL;
    auto Bp = find_batch(ctx, batch_id);
    if (!Bp) return fail(ctx, SMD_ENOTFOUND, "batch: unknown id");
    Batch &B = *Bp;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    auto w0 = std::chrono::steady_clock::now();
    CK(cudaMemcpyAsync(B.win.p, d_window, (size_t)B.n_rec * 8, cudaMemcpyDeviceToDevice, B.s_rk), "D2D window");
    int rc = batch_step(ctx, B, d_spins0, rep);
    if (rc) return rc;
    for (size_t i = 0; i < B.m.size(); i++) {
        CK(cudaMemcpyAsync(d_spec_sum[i], B.acc[i]->p, 3 * (size_t)B.m[i]->Q * B.n_rec * 8,
                           cudaMemcpyDeviceToDevice, B.s_rk),
           "D2D spec");
        CK(cudaMemcpyAsync(d_qss_sum[i], B.accq[i]->p, (size_t)B.n_rec * 8, cudaMemcpyDeviceToDevice, B.s_rk),
           "D2D qss");
    }
    CK(cudaStreamSynchronize(B.s_rk), "sync");
    if (rep) rep->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
    return SMD_OK;
}

extern "C" int smd_batch_run(smd_ctx *ctx, int batch_id, const double *const *spins0, const double *window,
                             double *const *spec_out, double *const *qss_out, smd_report *rep)
{
    if (!ctx || !spins0 || !window || !spec_out || !qss_out) return SMD_EINVAL;
    auto Bp = find_batch(ctx, batch_id);
    if (!Bp) return fail(ctx, SMD_ENOTFOUND, "batch: unknown id");
    Batch &B = *Bp;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    auto w0 = std::chrono::steady_clock::now();
    // host spins into the context's input staging, one region per member
    size_t in_b = 0;
    for (auto &mp : B.m) in_b += (size_t)mp->S * mp->N * 3 * 8;
    CK(ctx->in_tmp.ensure(in_b), "cudaMalloc");
    std::vector<const double *> dptr;
    size_t off = 0;
    for (size_t i = 0; i < B.m.size(); i++) {
        const size_t bytes = (size_t)B.m[i]->S * B.m[i]->N * 3 * 8;
        double *dst = reinterpret_cast<double *>(static_cast<char *>(ctx->in_tmp.p) + off);
        CK(cudaMemcpyAsync(dst, spins0[i], bytes, cudaMemcpyHostToDevice, B.s_rk), "H2D spins");
        dptr.push_back(dst);
        off += bytes;
    }
    CK(cudaMemcpyAsync(B.win.p, window, (size_t)B.n_rec * 8, cudaMemcpyHostToDevice, B.s_rk), "H2D window");
    auto w1 = std::chrono::steady_clock::now();
    int rc = batch_step(ctx, B, dptr.data(), rep);
    if (rc) return rc;
    auto w2 = std::chrono::steady_clock::now();
    for (size_t i = 0; i < B.m.size(); i++) {
        Member &mb = *B.m[i];
        const double fc = 1.0 / (double)mb.S;   // sample averages (smd_code.cpp:3596-3611)
        const size_t ns = 3 * (size_t)mb.Q * B.n_rec;
        CK(launch_scale(B.acc[i]->as<double>(), ns, fc, B.s_rk), "scale");
        CK(launch_scale(B.accq[i]->as<double>(), B.n_rec, fc, B.s_rk), "scale");
        CK(cudaMemcpyAsync(spec_out[i], B.acc[i]->p, ns * 8, cudaMemcpyDeviceToHost, B.s_rk), "D2H spec");
        CK(cudaMemcpyAsync(qss_out[i], B.accq[i]->p, (size_t)B.n_rec * 8, cudaMemcpyDeviceToHost, B.s_rk),
           "D2H qss");
    }
    CK(cudaStreamSynchronize(B.s_rk), "sync");
    auto w3 = std::chrono::steady_clock::now();
    if (rep) {
        rep->ms_h2d = std::chrono::duration<double, std::milli>(w1 - w0).count();
        rep->ms_d2h = std::chrono::duration<double, std::milli>(w3 - w2).count();
        rep->ms_total = std::chrono::duration<double, std::milli>(w3 - w0).count();
        rep->kernel_launches += 2 * (int)B.m.size();
    }
    return SMD_OK;
}
