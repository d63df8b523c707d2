// engine.cu -- serving with continuous batching (smd_submit / smd_poll /
// smd_wait / smd_cancel / smd_serve_shutdown).
//
// The reference runs one job per process, one sample at a time
// (Codes_Folder/smd_code.cpp:3079-3311).  Here one engine thread per context
// keeps the samples of many jobs resident in HBM and advances all of them
// together:
//
//   admission  jobs are taken largest first (site-steps; a job waiting over a
//              second goes first, and SMD_SERVE_ORDER=fifo takes them in
//              arrival order); a job's samples are admitted
//              in groups as large as the free HBM budget allows (a group is
//              a Member: spins, snapshots, time series), so a job larger
//              than the budget runs in successive groups and a job arriving
//              while others run joins as soon as slots and memory free up
//   tick       ONE persistent RK launch per precision advances every admitted
//              group by its next chunk of records (each group at its own
//              position, stride, dt and record chunk; thread-block clusters
//              pull (group, sample) items from a device queue), then each
//              group's chunk is projected; a group whose last chunk is done
//              adds its time transform into its job's accumulator, which
//              stays resident until the job's last group lands
//   completion the job's averages go to pinned staging and then to the
//              caller's buffers; smd_poll / smd_wait report it with the
//              latency from submit
//
// Memory comes from a stream-ordered pool (no device-wide synchronisation on
// allocation or release).  A group's arithmetic does not depend on what it
// shares a launch with (its CTAs per sample depend only on its lattice; the
// zero pad slots of a wider edge table add exact zeros), so a job's result
// is the same alone and in any mix.  Jobs whose lattice the batch kernel does
// not take (Lieb d-wave term, bond-list energies, impurities with
// couplings, more sites than 16 CTAs hold) run through smd_run on the
// engine's streams between ticks.
#include "batch_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

using namespace smd;
using namespace smdh;

// host.cu internals shared with the engine
int smd_share_objects(smd_ctx *from, smd_ctx *to, int lattice_id, int qset_id);
void smd_copy_error(smd_ctx *to, const smd_ctx *from, long long job_id);

namespace {

using Clock = std::chrono::steady_clock;

struct Pinned {
    void *p = nullptr;
    size_t bytes = 0;
    bool busy = false;
};

struct SJob {
    long long id = 0;
    smd_job_desc desc{};
    std::vector<double> spins, window;
    std::vector<int> imp;
    double *spec_out = nullptr, *qss_out = nullptr;
    int status = SMD_EBUSY;
    bool cancelled = false;
    Clock::time_point t_submit, t_done;
    double work = 0.0;   // site-steps: N x samples x RK steps
    // engine state
    bool started = false, batched = true, finishing = false;
    std::shared_ptr<Lattice> L;
    std::shared_ptr<QSet> Qs;
    int next_sample = 0, groups_live = 0, vcs = 1, R = 0;
    // streams mode: the single-job cluster configuration of the job, and the
    // event after its last enqueued time transform (groups of one job add
    // into its accumulator one after the other)
    ClusterTab *ctab = nullptr;
    int cspt = 0, cthreads = 0;
    cudaEvent_t ev_fin = nullptr;
    bool fin_recorded = false;
    size_t acc_bytes = 0;
    DevBuf acc, accq, win, stat;
    Pinned *stage = nullptr;       // spectra, autocorrelation, status, then [n_samples][4] energy stats
    cudaEvent_t ev_out = nullptr;
    double drift_max = 0.0, drift_final = 0.0;
};

struct Group {
    std::unique_ptr<Member> m;
    SJob *job = nullptr;
    int chunk = 0;
    int s_begin = 0;   // first sample of the job in this group
    size_t bytes = 0;
    int lane = -1;     // streams mode: the stream pair running the group
};

// streams mode: a stream pair (RK at the highest priority, projections at
// the lowest) with the events that order its three snapshot buffers
struct Lane {
    cudaStream_t rk = nullptr, proj = nullptr;
    cudaEvent_t ev_rk[kSnapBufs]{}, ev_proj[kSnapBufs]{}, done = nullptr;
    bool busy = false;
};
constexpr int kLanes = 16;   // stream pairs (SMD_SERVE_LANES overrides)

struct Engine {
    smd_ctx *parent = nullptr, *ectx = nullptr;
    cudaMemPool_t pool = nullptr;
    size_t budget = 0, used = 0;
    // sites per thread of the batch kernel: 4 (512 threads) measured ahead of
    // 2 on the serving mix, whose large lattices then take fewer CTAs per sample
    int spt = 4, threads = 512;
    std::mutex mu;
    std::condition_variable cv, done_cv;
    std::deque<std::shared_ptr<SJob>> queue;
    std::map<long long, std::shared_ptr<SJob>> jobs;
    std::vector<std::shared_ptr<SJob>> running;
    std::vector<Group> active;
    long long next = 1, tick = 0;
    bool stop = false;
    std::thread th;
    std::vector<std::unique_ptr<Pinned>> pinned;
    DevBuf d_items[kSnapBufs][2], d_queue[kSnapBufs];
    std::vector<int2> h_items[kSnapBufs][2];
    cudaEvent_t ev_rk[kSnapBufs]{}, ev_proj[kSnapBufs]{};
    std::map<long long, int> max_clusters;   // keyed by (prec, zt, csh, smem KiB)
    // Scheduling.  Streams mode (default): every admitted group runs the
    // single-job pipeline -- the cluster RK kernel with its job's own
    // configuration, its projections and its time transform -- enqueued at
    // admission on a stream pair of its own, so the groups of all jobs in
    // flight overlap on the device without a common tick.  Tick mode
    // (SMD_SERVE_MODE=tick): one persistent batch RK launch per tick
    // advances every group by one chunk.
    bool streams = true;
    std::vector<Lane> lanes;
    // Admission order (by_work, the default; SMD_SERVE_ORDER=fifo turns it
    // off): among the jobs not yet started, the one with the most site-steps
    // first, unless a job has waited kAgeLimit, then the oldest such.  A
    // burst then starts its large jobs while the device has the memory for
    // them in few groups, and the small ones fill in beside them (measured
    // on the 12-job serving burst: makespans 4.5-6.1 s in arrival order).
    bool by_work = true;
    static constexpr double kAgeLimit = 1.0;   // seconds
    void reorder_queue();
    int err_rc = SMD_OK;   // a failed enqueue in admit(): the run loop fails the jobs in flight
    int enqueue_group(Group &g);
    int reap_groups();
    // SMD_SERVE_TRACE=1: per-tick host and device times on stderr
    bool trace = false;
    cudaEvent_t tr[kSnapBufs][4]{};
    Clock::time_point t_start = Clock::now();

    void run();
    int admit();
    size_t room();
    int do_tick();
    void reap();
    void finish_job(SJob &j, int rc);
    int start_job(SJob &j);
    int run_alone(SJob &j);
    Pinned *get_pinned(size_t bytes);
    void set_error(const std::string &msg)
    {
        std::lock_guard<std::mutex> lk(parent->maps_mu);
        parent->err = msg;
    }
};

constexpr int kMaxActive = kMaxBatchSlots;

// Moves the job to admit next to the queue's front (mu held, the front not
// started).
void Engine::reorder_queue()
{
    const auto now = Clock::now();
    size_t pick = queue.size();
    double best = -1.0;
    for (size_t i = 0; i < queue.size(); i++) {
        const SJob &q = *queue[i];
        if (q.started || q.cancelled) continue;
        if (std::chrono::duration<double>(now - q.t_submit).count() > kAgeLimit) {
            pick = i;   // the oldest job past the age limit (the queue is in arrival order)
            break;
        }
        if (q.work > best) {
            best = q.work;
            pick = i;
        }
    }
    if (pick == 0 || pick == queue.size()) return;
    auto x = queue[pick];
    queue.erase(queue.begin() + (long)pick);
    queue.push_front(x);
}

// Pinned staging: the smallest free buffer that holds the bytes (best fit,
// so a small job does not take the buffer a large one of the same mix
// reuses, and a repeated mix allocates nothing), else a new one
// (cudaMallocHost of a large lattice's outputs takes ~100 ms).
Pinned *Engine::get_pinned(size_t bytes)
{
    Pinned *best = nullptr;
    for (auto &p : pinned)
        if (!p->busy && p->bytes >= bytes && (!best || p->bytes < best->bytes)) best = p.get();
    if (best) {
        best->busy = true;
        return best;
    }
    auto p = std::make_unique<Pinned>();
    if (cudaMallocHost(&p->p, bytes) != cudaSuccess) return nullptr;
    p->bytes = bytes;
    p->busy = true;
    pinned.push_back(std::move(p));
    return pinned.back().get();
}

void Engine::finish_job(SJob &j, int rc)
{
    {
        std::lock_guard<std::mutex> lk(mu);
        j.status = rc;
        j.t_done = Clock::now();
    }
    done_cv.notify_all();
}

// Lattice lookup, batching decision, accumulator and window for a job.
int Engine::start_job(SJob &j)
{
    smd_ctx *ctx = ectx;
    j.started = true;
    j.L = find_lattice(parent, j.desc.lattice);
    j.Qs = find_qset(parent, j.desc.qset);
    if (!j.L || !j.Qs) return fail(ctx, SMD_ENOTFOUND, "job: unknown lattice or q set");
    if (j.Qs->lattice != j.desc.lattice) return fail(ctx, SMD_EINVAL, "job: q set belongs to another lattice");
    // a probe member decides whether the batch kernel takes the job
    Member probe;
    probe.L = j.L;
    probe.Qs = j.Qs;
    probe.prec = j.desc.precision;
    probe.n_rec = j.desc.n_rec;
    probe.stride = j.desc.stride;
    probe.fix_every = j.desc.fix_every;
    probe.dt = j.desc.dt;
    probe.S = 1;
    if (j.desc.precision != SMD_FP32 && j.desc.precision != SMD_FP64) return fail(ctx, SMD_EINVAL, "job: precision");
    // records per chunk: about 512 RK steps per tick for every job, so the
    // work items of a launch take similar times (tick mode); 128 records
    // per RK launch, the single-job path's chunk (streams mode)
    j.R = streams ? std::min(128, j.desc.n_rec)
                  : std::max(8, std::min(128, 512 / std::max(1, j.desc.stride)));
    probe.R = j.R;
    j.batched = cluster_ok(*j.L) && member_setup(ctx, probe) == SMD_OK;
    if (j.batched && streams) {
        // the configuration the single-job path takes for this job (a
        // function of the lattice, precision and the job's sample count, not
        // of the group sizes, so the job's arithmetic is the same alone and
        // in any mix)
        j.ctab = cluster_choice(*j.L, j.desc.precision, j.desc.n_samples, parent->device, &j.cspt,
                                &j.cthreads);
        if (!j.ctab) j.batched = false;
        else j.vcs = j.ctab->P.CS;
    } else if (j.batched) {
        j.vcs = member_ctas(probe, spt, 18, nullptr);
        if (!j.vcs) j.batched = false;
    }
    if (!j.batched) return SMD_OK;
    const size_t Q = j.Qs->Q, n = j.desc.n_rec;
    j.acc_bytes = 3 * Q * n * 8 + n * 8 + 256;
    cudaStream_t st = ectx->s_rk;
    CK(j.acc.ensure_async(3 * Q * n * 8, pool, st), "alloc");
    CK(j.accq.ensure_async(n * 8, pool, st), "alloc");
    CK(j.win.ensure_async(n * 8, pool, st), "alloc");
    CK(j.stat.ensure_async(sizeof(int), pool, st), "alloc");
    CK(cudaMemsetAsync(j.acc.p, 0, 3 * Q * n * 8, st), "memset");
    CK(cudaMemsetAsync(j.accq.p, 0, n * 8, st), "memset");
    CK(cudaMemsetAsync(j.stat.p, 0, sizeof(int), st), "memset");
    CK(cudaMemcpyAsync(j.win.p, j.window.data(), n * 8, cudaMemcpyHostToDevice, st), "H2D window");
    CK(cudaEventCreateWithFlags(&j.ev_out, cudaEventDisableTiming), "event");
    // staging for the outputs and every sample's energy statistics
    j.stage = get_pinned((3 * Q * n + n) * 8 + 64 + (size_t)j.desc.n_samples * 32);
    if (!j.stage) return fail(ctx, SMD_ECUDA, "serving: pinned staging");
    used += j.acc_bytes;
    if (streams) {
        CK(cudaEventCreateWithFlags(&j.ev_fin, cudaEventDisableTiming), "event");
        // the lanes' streams read the accumulators and window set up above
        CK(cudaStreamSynchronize(st), "sync");
    }
    return SMD_OK;
}

// smd_run on the engine's own context, for jobs the batch kernel does not take.
int Engine::run_alone(SJob &j)
{
    int rc = smd_share_objects(parent, ectx, j.desc.lattice, j.desc.qset);
    if (rc == SMD_OK) {
        smd_job_desc d = j.desc;
        d.imp = j.imp.empty() ? nullptr : j.imp.data();
        rc = smd_run(ectx, &d, j.spins.data(), j.window.data(), j.spec_out, j.qss_out, nullptr, nullptr);
    }
    if (rc != SMD_OK) smd_copy_error(parent, ectx, j.id);
    return rc;
}

// Device memory the pool can still hand out: free device memory plus what
// the pool holds unused, less a margin for the context's own small
// allocations.
size_t Engine::room()
{
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return budget;
    cuuint64_t res = 0, inuse = 0;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &res);
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &inuse);
    const size_t avail = fr + (size_t)(res > inuse ? res - inuse : 0);
    const size_t margin = (size_t)512 << 20;
    return avail > margin ? avail - margin : 0;
}

// Admit sample groups of queued jobs, in arrival order, while slots and the
// HBM budget allow.  Returns the number of groups admitted.
int Engine::admit()
{
    int admitted = 0;
    bool halve_next = false;   // the last group's allocation failed: retry smaller
    int last_S = 0;
    for (;;) {
        std::shared_ptr<SJob> jp;
        {
            std::lock_guard<std::mutex> lk(mu);
            while (!queue.empty() && queue.front()->cancelled) {
                auto c = queue.front();
                queue.pop_front();
                c->status = SMD_ECANCELLED;
                c->t_done = Clock::now();
                done_cv.notify_all();
            }
            if (queue.empty()) return admitted;
            if (by_work && !queue.front()->started) reorder_queue();
            jp = queue.front();
        }
        SJob &j = *jp;
        if (!j.started) {
            {
                std::lock_guard<std::mutex> lk(mu);
                j.started = true;   // smd_cancel no longer drops it
            }
            int rc = start_job(j);
            if (rc != SMD_OK) {
                smd_copy_error(parent, ectx, j.id);
                std::lock_guard<std::mutex> lk(mu);
                queue.pop_front();
                j.status = rc;
                j.t_done = Clock::now();
                done_cv.notify_all();
                continue;
            }
            if (j.batched) running.push_back(jp);
        }
        if (!j.batched) {
            // runs on its own: wait until the launches in flight drain
            if (!active.empty()) return admitted;
            {
                std::lock_guard<std::mutex> lk(mu);
                queue.pop_front();
            }
            finish_job(j, run_alone(j));
            continue;
        }
        if ((int)active.size() >= kMaxActive) return admitted;
        int lane = -1;
        if (streams) {
            for (int k = 0; k < (int)lanes.size() && lane < 0; k++)
                if (!lanes[k].busy) lane = k;
            if (lane < 0) return admitted;   // every stream pair is running a group
        }
        // the largest group of the remaining samples that fits the free budget
        auto make = [&](int S) {
            auto m = std::make_unique<Member>();
            m->L = j.L;
            m->Qs = j.Qs;
            m->prec = j.desc.precision;
            m->n_rec = j.desc.n_rec;
            m->stride = j.desc.stride;
            m->fix_every = j.desc.fix_every;
            m->dt = j.desc.dt;
            m->R = j.R;
            m->S = S;
            m->d_win = j.win.as<double>();
            m->d_status = j.stat.as<int>();
            member_setup(ectx, *m);
            m->vcs = j.vcs;
            const int per = kMaxClusterCTAs / j.vcs;   // samples per item at the widest cluster
            m->Sp = streams ? S : (S + per - 1) / per * per;
            return m;
        };
        const int left = j.desc.n_samples - j.next_sample;
        int S = halve_next ? std::max(1, last_S / 2) : left;
        halve_next = false;
        std::unique_ptr<Member> m = make(S);
        size_t bytes = member_bytes(*m, m->Sp);
        // the group must fit the budget and the memory the device still has
        // (other users of the device, this context's own buffers included)
        const size_t free_now = room();
        auto fits = [&](size_t b) { return used + b <= budget && b <= free_now; };
        while (S > 1 && !fits(bytes)) {
            S = std::max(1, S / 2);
            m = make(S);
            bytes = member_bytes(*m, m->Sp);
        }
        last_S = S;
        if (!fits(bytes)) {
            if (active.empty()) {
                // not even one sample fits with nothing else resident
                std::lock_guard<std::mutex> lk(mu);
                queue.pop_front();
                running.erase(std::find(running.begin(), running.end(), jp));
                j.acc.release();
                j.accq.release();
                j.win.release();
                j.stat.release();
                if (j.stage) j.stage->busy = false;
                used -= j.acc_bytes;
                set_error("job " + std::to_string(j.id) + ": one sample exceeds the HBM budget");
                j.status = SMD_ENOMEM_ADMIT;
                j.t_done = Clock::now();
                done_cv.notify_all();
                continue;
            }
            return admitted;   // wait for memory to free up
        }
        // buffers and inputs of the group
        smd_ctx *ctx = ectx;
        cudaStream_t st = streams ? lanes[lane].rk : ectx->s_rk;
        if (!j.imp.empty()) {
            const size_t N = m->N;
            m->imp.resize((size_t)m->Sp * N);
            for (int s = 0; s < m->Sp; s++) {
                const int src = j.next_sample + std::min(s, S - 1);
                for (size_t i = 0; i < N; i++) m->imp[(size_t)s * N + i] = j.imp[(size_t)src * N + i] ? 1 : 0;
            }
        }
        DevBuf in;
        const size_t in_b = (size_t)S * m->N * 3 * 8;
        if (member_alloc(ectx, *m, pool, st) != SMD_OK || in.ensure_async(in_b, pool, st) != cudaSuccess) {
            cudaGetLastError();   // the failed allocation's error is not sticky
            m.reset();            // returns what was allocated to the pool
            in.release();
            if (!active.empty()) return admitted;   // retry once memory is released
            if (S > 1) {
                // nothing else resident: retry with half the samples
                halve_next = true;
                continue;
            }
            std::lock_guard<std::mutex> lk(mu);
            queue.pop_front();
            set_error("job " + std::to_string(j.id) + ": device allocation failed");
            j.status = SMD_ENOMEM_ADMIT;
            j.t_done = Clock::now();
            done_cv.notify_all();
            if (j.groups_live == 0) {
                running.erase(std::find(running.begin(), running.end(), jp));
                if (j.stage) j.stage->busy = false;
                used -= j.acc_bytes;
            }
            continue;
        }
        CK(cudaMemcpyAsync(in.p, j.spins.data() + (size_t)j.next_sample * m->N * 3, in_b, cudaMemcpyHostToDevice,
                           st),
           "H2D spins");
        int launches = 0;
        if (member_load(ectx, *m, in.as<double>(), st, &launches) != SMD_OK) return admitted;
        in.release();   // stream-ordered after the load
        Group g;
        g.m = std::move(m);
        g.job = &j;
        g.s_begin = j.next_sample;
        g.bytes = bytes;
        g.lane = lane;
        used += bytes;
        j.next_sample += S;
        j.groups_live++;
        active.push_back(std::move(g));
        admitted++;
        if (streams) {
            lanes[lane].busy = true;
            const int rc = enqueue_group(active.back());
            if (rc != SMD_OK) {
                err_rc = rc;
                return admitted;
            }
        }
        if (j.next_sample >= j.desc.n_samples) {
            std::lock_guard<std::mutex> lk(mu);
            queue.pop_front();
        }
    }
}

int Engine::do_tick()
{
    smd_ctx *ctx = ectx;
    cudaStream_t srk = ectx->s_rk, spr = ectx->s_proj;
    const int bt = (int)(tick % kSnapBufs);
    if (tick >= kSnapBufs) {
        // the RK launch of tick - 3 has read this tick's item buffers; the
        // projections of tick - 3 have read the snapshot buffers reused now
        CK(cudaEventSynchronize(ev_rk[bt]), "sync");
        CK(cudaStreamWaitEvent(srk, ev_proj[bt], 0), "wait");
        if (trace) {
            CK(cudaEventSynchronize(tr[bt][3]), "sync");
            float a = 0.f, b = 0.f, c = 0.f;
            cudaEventElapsedTime(&a, tr[bt][0], tr[bt][1]);
            cudaEventElapsedTime(&b, tr[bt][2], tr[bt][3]);
            cudaEventElapsedTime(&c, tr[bt][0], tr[bt][3]);
            std::fprintf(stderr, "[smd serve] tick %lld: rk %.2f ms, projections %.2f ms, tick span %.2f ms\n",
                         tick - kSnapBufs, a, b, c);
        }
    }
    if (trace) {
        std::fprintf(stderr, "[smd serve] tick %lld issued at %.1f ms: %zu groups, %.0f MB in use\n", tick,
                     std::chrono::duration<double, std::milli>(Clock::now() - t_start).count(), active.size(),
                     used / 1e6);
        CK(cudaEventRecord(tr[bt][0], srk), "event");
    }
    CK(cudaMemsetAsync(d_queue[bt].p, 0, 2 * sizeof(int), srk), "memset");
    for (int prec : {SMD_FP32, SMD_FP64}) {
        std::vector<Member *> mm;
        std::vector<int> chunk, vcs;
        int zmax = 0, csh = 1;
        size_t smem = 0;
        for (auto &g : active)
            if (g.m->prec == prec && g.chunk < g.m->nchunks) {
                mm.push_back(g.m.get());
                chunk.push_back(g.chunk);
                vcs.push_back(g.m->vcs);
                zmax = std::max(zmax, g.m->L->zn[0] + g.m->L->zn[1] + g.m->L->zn[2]);
                csh = std::max(csh, g.m->vcs);
            }
        if (mm.empty()) continue;
        const int zt = zt_of(zmax);
        for (Member *m : mm) {
            ClusterTab *t = cluster_tables(*m->L, m->vcs, zt);
            if (!t) return fail(ctx, SMD_EINVAL, "serving: lattice does not fit the cluster kernel");
            smem = std::max(smem, rk_cluster_smem(t->P, prec));
        }
        const long long key = (((long long)prec * 32 + zt) * 32 + csh) * 1024 + (long long)(smem >> 10);
        auto it = max_clusters.find(key);
        if (it == max_clusters.end())
            it = max_clusters.emplace(key, rk_batch_max_clusters(prec, spt, zt, threads, csh, smem)).first;
        if (it->second <= 0) return fail(ctx, SMD_ECUDA, "serving: no cluster of the RK launch fits the device");
        const int ncl = rk_cluster_cap(it->second, csh);
        std::vector<int2> &hi = h_items[bt][prec];
        hi = make_items(mm, vcs, csh);
        CK(d_items[bt][prec].ensure(hi.size() * sizeof(int2)), "cudaMalloc");
        CK(cudaMemcpyAsync(d_items[bt][prec].p, hi.data(), hi.size() * sizeof(int2), cudaMemcpyHostToDevice, srk),
           "H2D items");
        int rc = launch_rk_members(ctx, mm, chunk, prec, zt, spt, threads, csh, ncl, smem,
                                   d_items[bt][prec].as<int2>(), (int)hi.size(), d_queue[bt].as<int>() + prec, srk);
        if (rc) return rc;
    }
    if (trace) CK(cudaEventRecord(tr[bt][1], srk), "event");
    CK(cudaEventRecord(ev_rk[bt], srk), "event");
    CK(cudaStreamWaitEvent(spr, ev_rk[bt], 0), "wait");
    if (trace) CK(cudaEventRecord(tr[bt][2], spr), "event");
    int launches = 0;
    for (auto &g : active) {
        Member &m = *g.m;
        if (g.chunk >= m.nchunks) continue;
        int rc = member_project(ctx, m, g.chunk, spr, &launches);
        if (rc) return rc;
        g.chunk++;
        if (g.chunk == m.nchunks) {
            SJob &j = *g.job;
            rc = member_finish(ctx, m, j.acc.as<double>(), j.accq.as<double>(), spr, &launches);
            if (rc) return rc;
            // the group's energy statistics ([S][4]: max drift, last E, E0, -)
            const size_t Q = j.Qs->Q, n = j.desc.n_rec;
            char *h = static_cast<char *>(j.stage->p) + (3 * Q * n + n) * 8 + 64 + (size_t)g.s_begin * 32;
            CK(cudaMemcpyAsync(h, m.stats.p, (size_t)m.S * 32, cudaMemcpyDeviceToHost, spr), "D2H stats");
        }
    }
    if (trace) CK(cudaEventRecord(tr[bt][3], spr), "event");
    CK(cudaEventRecord(ev_proj[bt], spr), "event");
    // finished groups leave; their buffers are released on the projection
    // stream, after the work that reads them
    for (size_t i = 0; i < active.size();) {
        Group &g = active[i];
        if (g.chunk < g.m->nchunks) {
            i++;
            continue;
        }
        for (DevBuf *d : {&g.m->state, &g.m->s0, &g.m->impd, &g.m->series, &g.m->qss, &g.m->qpart, &g.m->stats,
                          &g.m->e0, &g.m->gscratch})
            d->st = spr;
        for (int b = 0; b < kSnapBufs; b++) {
            g.m->snap[b].st = spr;
            g.m->ahi[b].st = spr;
            g.m->alo[b].st = spr;
        }
        SJob &j = *g.job;
        used -= g.bytes;
        j.groups_live--;
        active.erase(active.begin() + i);   // releases the member's buffers
        if (j.groups_live == 0 && j.next_sample >= j.desc.n_samples) {
            // the job's averages to pinned staging
            const size_t Q = j.Qs->Q, n = j.desc.n_rec, ns = 3 * Q * n;
            const double fc = 1.0 / (double)j.desc.n_samples;   // smd_code.cpp:3596-3611
            CK(launch_scale(j.acc.as<double>(), ns, fc, spr), "scale");
            CK(launch_scale(j.accq.as<double>(), n, fc, spr), "scale");
            char *h = static_cast<char *>(j.stage->p);
            CK(cudaMemcpyAsync(h, j.acc.p, ns * 8, cudaMemcpyDeviceToHost, spr), "D2H spec");
            CK(cudaMemcpyAsync(h + ns * 8, j.accq.p, n * 8, cudaMemcpyDeviceToHost, spr), "D2H qss");
            CK(cudaMemcpyAsync(h + (ns + n) * 8, j.stat.p, sizeof(int), cudaMemcpyDeviceToHost, spr), "D2H status");
            CK(cudaEventRecord(j.ev_out, spr), "event");
            j.finishing = true;
        }
    }
    tick++;
    return SMD_OK;
}

// Streams mode: the group's whole pipeline, enqueued at admission on its
// lane as the single-job path runs it -- per chunk of R records the cluster
// RK kernel on the lane's RK stream, then the chunk's projections on its
// projection stream (three snapshot buffers between the two); after the
// last chunk the time transform adds into the job's accumulator behind the
// job's earlier groups, and the group's energy statistics go to the job's
// staging.
int Engine::enqueue_group(Group &g)
{
    smd_ctx *ctx = ectx;
    Lane &ln = lanes[g.lane];
    Member &m = *g.m;
    SJob &j = *g.job;
    int launches = 0;
    for (int c = 0; c < m.nchunks; c++) {
        const int b = c % kSnapBufs;
        if (c >= kSnapBufs) CK(cudaStreamWaitEvent(ln.rk, ln.ev_proj[b], 0), "wait");
        const int rb = c * m.R, re = std::min(m.n_rec, rb + m.R);
        const RKJob J = member_job(m, rb, re, b);
        CK(launch_rk_cluster(j.ctab->P, J, m.prec, j.cspt, j.cthreads, ln.rk), "rk cluster kernel");
        CK(cudaEventRecord(ln.ev_rk[b], ln.rk), "event");
        CK(cudaStreamWaitEvent(ln.proj, ln.ev_rk[b], 0), "wait");
        const int rc = member_project(ctx, m, c, ln.proj, &launches);
        if (rc) return rc;
        CK(cudaEventRecord(ln.ev_proj[b], ln.proj), "event");
    }
    if (j.fin_recorded) CK(cudaStreamWaitEvent(ln.proj, j.ev_fin, 0), "wait");
    const int rc = member_finish(ctx, m, j.acc.as<double>(), j.accq.as<double>(), ln.proj, &launches);
    if (rc) return rc;
    const size_t Q = j.Qs->Q, n = j.desc.n_rec;
    char *h = static_cast<char *>(j.stage->p) + (3 * Q * n + n) * 8 + 64 + (size_t)g.s_begin * 32;
    CK(cudaMemcpyAsync(h, m.stats.p, (size_t)m.S * 32, cudaMemcpyDeviceToHost, ln.proj), "D2H stats");
    CK(cudaEventRecord(j.ev_fin, ln.proj), "event");
    j.fin_recorded = true;
    CK(cudaEventRecord(ln.done, ln.proj), "event");
    g.chunk = m.nchunks;
    return SMD_OK;
}

// Streams mode: groups whose lane has finished leave (their buffers go back
// to the pool, their lane to the free list); a job whose last group is done
// gets its averages staged for the caller.  Returns the groups reaped, or
// a negative status.
int Engine::reap_groups()
{
    smd_ctx *ctx = ectx;
    int done = 0;
    for (size_t i = 0; i < active.size();) {
        Group &g = active[i];
        Lane &ln = lanes[g.lane];
        const cudaError_t q = cudaEventQuery(ln.done);
        if (q == cudaErrorNotReady) {
            i++;
            continue;
        }
        if (q != cudaSuccess) return -cuda_fail(ctx, q, "serving lane");
        for (DevBuf *d : {&g.m->state, &g.m->s0, &g.m->impd, &g.m->series, &g.m->qss, &g.m->qpart, &g.m->stats,
                          &g.m->e0, &g.m->gscratch})
            d->st = ln.proj;
        for (int b = 0; b < kSnapBufs; b++) {
            g.m->snap[b].st = ln.proj;
            g.m->ahi[b].st = ln.proj;
            g.m->alo[b].st = ln.proj;
        }
        SJob &j = *g.job;
        used -= g.bytes;
        j.groups_live--;
        ln.busy = false;
        active.erase(active.begin() + i);   // releases the member's buffers
        done++;
        if (j.groups_live == 0 && j.next_sample >= j.desc.n_samples) {
            cudaStream_t spr = ectx->s_proj;
            const size_t Q = j.Qs->Q, n = j.desc.n_rec, ns = 3 * Q * n;
            const double fc = 1.0 / (double)j.desc.n_samples;   // smd_code.cpp:3596-3611
            if (launch_scale(j.acc.as<double>(), ns, fc, spr) != cudaSuccess ||
                launch_scale(j.accq.as<double>(), n, fc, spr) != cudaSuccess)
                return -cuda_fail(ctx, cudaGetLastError(), "scale");
            char *h = static_cast<char *>(j.stage->p);
            cudaError_t e = cudaMemcpyAsync(h, j.acc.p, ns * 8, cudaMemcpyDeviceToHost, spr);
            if (e == cudaSuccess) e = cudaMemcpyAsync(h + ns * 8, j.accq.p, n * 8, cudaMemcpyDeviceToHost, spr);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(h + (ns + n) * 8, j.stat.p, sizeof(int), cudaMemcpyDeviceToHost, spr);
            if (e == cudaSuccess) e = cudaEventRecord(j.ev_out, spr);
            if (e != cudaSuccess) return -cuda_fail(ctx, e, "D2H outputs");
            j.finishing = true;
        }
    }
    return done;
}

// Jobs whose outputs have reached the pinned staging: copy to the caller's
// buffers and report.
void Engine::reap()
{
    for (size_t i = 0; i < running.size();) {
        SJob &j = *running[i];
        if (!j.finishing || cudaEventQuery(j.ev_out) != cudaSuccess) {
            i++;
            continue;
        }
        const size_t Q = j.Qs->Q, n = j.desc.n_rec, ns = 3 * Q * n;
        const char *h = static_cast<const char *>(j.stage->p);
        std::memcpy(j.spec_out, h, ns * 8);
        std::memcpy(j.qss_out, h + ns * 8, n * 8);
        int st = 0;
        std::memcpy(&st, h + (ns + n) * 8, sizeof(int));
        const double *stt = reinterpret_cast<const double *>(h + (ns + n) * 8 + 64);
        const double N = (double)j.L->N;
        for (int k = 0; k < j.desc.n_samples; k++) {
            j.drift_max = std::max(j.drift_max, stt[4 * k] / N);
            j.drift_final = std::max(j.drift_final, std::fabs(stt[4 * k + 1] - stt[4 * k + 2]) / N);
        }
        j.stage->busy = false;
        int rc = SMD_OK;
        if (st & 4) rc = SMD_ETIMEOUT;
        else if (st & 8) rc = SMD_ETIMEOUT;
        else if (st & 16) rc = SMD_ETIMEOUT;
        else if (st) rc = SMD_ECUDA;
        if (rc) set_error("job " + std::to_string(j.id) + ": device status " + std::to_string(st));
        for (DevBuf *d : {&j.acc, &j.accq, &j.win, &j.stat}) d->st = ectx->s_proj;
        j.acc.release();
        j.accq.release();
        j.win.release();
        j.stat.release();
        used -= j.acc_bytes;
        cudaEventDestroy(j.ev_out);
        j.ev_out = nullptr;
        if (j.ev_fin) cudaEventDestroy(j.ev_fin);
        j.ev_fin = nullptr;
        j.finishing = false;
        auto keep = running[i];
        running.erase(running.begin() + i);
        finish_job(j, rc);
    }
}

void Engine::run()
{
    cudaSetDevice(parent->device);
    smd_device_opts o{};
    o.device = parent->device;
    o.hbm_budget = parent->budget;
    int crc = smd_ctx_create(&o, &ectx);
    if (crc == SMD_OK) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = parent->device;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) crc = SMD_ECUDA;
        else {
            uint64_t thr = UINT64_MAX;   // keep released memory in the pool
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        for (int b = 0; b < kSnapBufs && crc == SMD_OK; b++) {
            if (cudaEventCreateWithFlags(&ev_rk[b], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&ev_proj[b], cudaEventDisableTiming) != cudaSuccess ||
                d_queue[b].ensure(2 * sizeof(int)) != cudaSuccess)
                crc = SMD_ECUDA;
        }
    }
    budget = parent->budget;
    if (const char *e = std::getenv("SMD_SERVE_TRACE")) trace = std::atoi(e) != 0;
    for (int b = 0; b < kSnapBufs && trace; b++)
        for (int k = 0; k < 4; k++) cudaEventCreate(&tr[b][k]);
    if (const char *e = std::getenv("SMD_SERVE_SPT")) spt = std::atoi(e) == 2 ? 2 : 4;
    threads = rk_batch_threads(SMD_FP32, spt);
    if (const char *e = std::getenv("SMD_SERVE_MODE")) streams = std::strcmp(e, "tick") != 0;
    if (const char *e = std::getenv("SMD_SERVE_ORDER")) by_work = std::strcmp(e, "fifo") != 0;
    if (streams && crc == SMD_OK) {
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        int nl = kLanes;
        if (const char *e = std::getenv("SMD_SERVE_LANES")) nl = std::max(1, std::min(kMaxActive, std::atoi(e)));
        lanes.resize(nl);
        for (Lane &ln : lanes) {
            bool ok = cudaStreamCreateWithPriority(&ln.rk, cudaStreamNonBlocking, hi) == cudaSuccess &&
                      cudaStreamCreateWithPriority(&ln.proj, cudaStreamNonBlocking, lo) == cudaSuccess &&
                      cudaEventCreateWithFlags(&ln.done, cudaEventDisableTiming) == cudaSuccess;
            for (int b = 0; b < kSnapBufs && ok; b++)
                ok = cudaEventCreateWithFlags(&ln.ev_rk[b], cudaEventDisableTiming) == cudaSuccess &&
                     cudaEventCreateWithFlags(&ln.ev_proj[b], cudaEventDisableTiming) == cudaSuccess;
            if (!ok) crc = SMD_ECUDA;
        }
    }
    // a failed launch or copy: every job in flight fails with rc
    auto fail_in_flight = [&](int rc) {
        cudaStreamSynchronize(ectx->s_rk);
        cudaStreamSynchronize(ectx->s_proj);
        for (Lane &ln : lanes) {
            cudaStreamSynchronize(ln.rk);
            cudaStreamSynchronize(ln.proj);
            ln.busy = false;
        }
        smd_copy_error(parent, ectx, 0);
        for (auto &g : active) g.job->groups_live = -1;
        active.clear();
        for (auto &jp : running) {
            used -= jp->acc_bytes;
            finish_job(*jp, rc);
        }
        running.clear();
        used = 0;
    };
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return stop || !queue.empty() || !active.empty() || !running.empty(); });
            if (stop && queue.empty() && active.empty() && running.empty()) break;
        }
        if (crc != SMD_OK) {
            // no device context: every job fails
            std::lock_guard<std::mutex> lk(mu);
            while (!queue.empty()) {
                queue.front()->status = SMD_ECUDA;
                queue.front()->t_done = Clock::now();
                queue.pop_front();
            }
            done_cv.notify_all();
            continue;
        }
        const int admitted = admit();
        if (err_rc != SMD_OK) {
            fail_in_flight(err_rc);
            err_rc = SMD_OK;
            continue;
        }
        if (streams) {
            const int n = reap_groups();
            if (n < 0) {
                fail_in_flight(-n);
                continue;
            }
            reap();
            // nothing finished and nothing new: let the lanes run
            if (n == 0 && admitted == 0) std::this_thread::sleep_for(std::chrono::microseconds(100));
            continue;
        }
        if (!active.empty()) {
            int rc = do_tick();
            if (rc != SMD_OK) fail_in_flight(rc);
        } else if (!running.empty()) {
            // only outputs in flight: wait for the oldest
            for (auto &jp : running)
                if (jp->finishing) {
                    cudaEventSynchronize(jp->ev_out);
                    break;
                }
        }
        reap();
    }
    cudaStreamSynchronize(ectx ? ectx->s_proj : nullptr);
    for (Lane &ln : lanes) {
        if (ln.rk) cudaStreamSynchronize(ln.rk);
        if (ln.proj) cudaStreamSynchronize(ln.proj);
        for (int b = 0; b < kSnapBufs; b++) {
            if (ln.ev_rk[b]) cudaEventDestroy(ln.ev_rk[b]);
            if (ln.ev_proj[b]) cudaEventDestroy(ln.ev_proj[b]);
        }
        if (ln.done) cudaEventDestroy(ln.done);
        if (ln.rk) cudaStreamDestroy(ln.rk);
        if (ln.proj) cudaStreamDestroy(ln.proj);
    }
    for (int b = 0; b < kSnapBufs; b++) {
        for (int p = 0; p < 2; p++) d_items[b][p].release();
        d_queue[b].release();
        if (ev_rk[b]) cudaEventDestroy(ev_rk[b]);
        if (ev_proj[b]) cudaEventDestroy(ev_proj[b]);
        for (int k = 0; k < 4; k++)
            if (tr[b][k]) cudaEventDestroy(tr[b][k]);
    }
    if (ectx) {
        cudaDeviceSynchronize();
        for (auto &p : pinned) cudaFreeHost(p->p);
        pinned.clear();
        if (pool) cudaMemPoolDestroy(pool);
        smd_ctx_destroy(ectx);
    }
}

std::mutex g_mu;
// never destroyed: an engine still running at process exit must not meet a
// destroyed registry (smd_serve_shutdown is the orderly end)
auto &g_engines = *new std::map<smd_ctx *, std::unique_ptr<Engine>>();

Engine *engine_for(smd_ctx *ctx)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_engines.find(ctx);
    if (it != g_engines.end()) return it->second.get();
    auto e = std::make_unique<Engine>();
    e->parent = ctx;
    Engine *p = e.get();
    p->th = std::thread([p] { p->run(); });
    g_engines[ctx] = std::move(e);
    return p;
}

int job_state(Engine *e, long long id, double *latency_ms)
{
    auto it = e->jobs.find(id);
    if (it == e->jobs.end()) return SMD_ENOTFOUND;
    SJob &j = *it->second;
    if (j.status == SMD_EBUSY) return SMD_EBUSY;
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(j.t_done - j.t_submit).count();
    return j.status;
}

}  // namespace

void smdh::engine_trim(smd_ctx *ctx)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_engines.find(ctx);
    if (it == g_engines.end() || !it->second->pool) return;
    cudaMemPoolTrimTo(it->second->pool, 0);
}

extern "C" void smd_serve_shutdown(smd_ctx *ctx)
{
    std::unique_ptr<Engine> e;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_engines.find(ctx);
        if (it == g_engines.end()) return;
        e = std::move(it->second);
        g_engines.erase(it);
    }
    {
        std::lock_guard<std::mutex> lk(e->mu);
        e->stop = true;
    }
    e->cv.notify_all();
    if (e->th.joinable()) e->th.join();
}

extern "C" int smd_submit(smd_ctx *ctx, const smd_job_desc *job, const double *spins0, const double *window,
                          double *spec_out, double *qss_out, long long *job_id)
{
    if (!ctx || !job || !spins0 || !window || !spec_out || !qss_out || !job_id) return SMD_EINVAL;
    int N = 0, Q = 0;
    if (smd_qset_size(ctx, job->qset, &Q) != SMD_OK) return SMD_ENOTFOUND;
    if (smd_lattice_sites(ctx, job->lattice, &N) != SMD_OK) return SMD_ENOTFOUND;
    if (job->n_samples < 1 || job->n_rec < 2 || job->stride < 1 || !(job->dt > 0.0)) return SMD_EINVAL;
    auto j = std::make_shared<SJob>();
    j->desc = *job;
    j->desc.imp = nullptr;
    j->spins.assign(spins0, spins0 + (size_t)job->n_samples * N * 3);
    j->window.assign(window, window + job->n_rec);
    if (job->imp) j->imp.assign(job->imp, job->imp + (size_t)job->n_samples * N);
    j->spec_out = spec_out;
    j->qss_out = qss_out;
    j->t_submit = Clock::now();
    j->work = (double)N * job->n_samples * (double)(job->n_rec - 1) * job->stride;
    Engine *e = engine_for(ctx);
    {
        std::lock_guard<std::mutex> lk(e->mu);
        j->id = e->next++;
        e->jobs[j->id] = j;
        e->queue.push_back(j);
        *job_id = j->id;
    }
    e->cv.notify_all();
    return SMD_OK;
}

extern "C" int smd_poll(smd_ctx *ctx, long long job_id, double *latency_ms)
{
    if (!ctx) return SMD_EINVAL;
    Engine *e = engine_for(ctx);
    std::lock_guard<std::mutex> lk(e->mu);
    return job_state(e, job_id, latency_ms);
}

extern "C" int smd_wait(smd_ctx *ctx, long long job_id, double timeout_ms, double *latency_ms)
{
    if (!ctx) return SMD_EINVAL;
    Engine *e = engine_for(ctx);
    std::unique_lock<std::mutex> lk(e->mu);
    auto pred = [&] { return job_state(e, job_id, nullptr) != SMD_EBUSY; };
    if (timeout_ms < 0) {
        e->done_cv.wait(lk, pred);
    } else if (!e->done_cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), pred)) {
        return SMD_ETIMEOUT;
    }
    return job_state(e, job_id, latency_ms);
}

extern "C" int smd_cancel(smd_ctx *ctx, long long job_id)
{
    if (!ctx) return SMD_EINVAL;
    Engine *e = engine_for(ctx);
    std::lock_guard<std::mutex> lk(e->mu);
    auto it = e->jobs.find(job_id);
    if (it == e->jobs.end()) return SMD_ENOTFOUND;
    SJob &j = *it->second;
    if (j.status != SMD_EBUSY) return j.status;
    if (j.started) return SMD_EBUSY;   // samples already on the device run to completion
    j.cancelled = true;
    return SMD_OK;
}

extern "C" int smd_job_info(smd_ctx *ctx, long long job_id, smd_report *rep)
{
    if (!ctx || !rep) return SMD_EINVAL;
    Engine *e = engine_for(ctx);
    std::lock_guard<std::mutex> lk(e->mu);
    auto it = e->jobs.find(job_id);
    if (it == e->jobs.end()) return SMD_ENOTFOUND;
    SJob &j = *it->second;
    if (j.status == SMD_EBUSY) return SMD_EBUSY;
    std::memset(rep, 0, sizeof *rep);
    rep->ms_total = std::chrono::duration<double, std::milli>(j.t_done - j.t_submit).count();
    rep->site_steps = 0.0;
    if (j.L) rep->site_steps = (double)j.L->N * (double)(j.desc.n_rec - 1) * j.desc.stride * j.desc.n_samples;
    rep->drift_max = j.drift_max;
    rep->drift_final = j.drift_final;
    rep->rk_kind = j.batched ? 3 : 1;
    return j.status;
}
