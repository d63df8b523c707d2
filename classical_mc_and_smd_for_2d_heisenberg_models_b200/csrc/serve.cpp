// serve.cpp -- job submission interface (smd_submit / smd_poll / smd_wait /
// smd_cancel).
//
// Jobs are copied at submit time and taken in arrival order by K worker
// lanes per context (SMD_SERVE_LANES, default 1).  Each lane owns a context
// of its own -- streams, working buffers and an equal share of the HBM
// budget, which admits its jobs -- and shares the parent's lattices and q
// sets, so up to K jobs run on the device at once and small jobs, which
// leave SMs idle on their own, overlap.  On the serving mix of the bench
// (jobs of 256-4096 sites whose RK launches already fill the SMs) four
// lanes measured slower than one (p50 70 vs 56 ms), so one is the default.
// A job's result is that of smd_run of the job alone.  The output buffers named at submit are written when
// the job finishes; smd_poll reports SMD_EBUSY until then and returns the
// job's latency (submit to completion) afterwards.
#include "../../include/smd_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

// host.cu internals shared with the lanes
int smd_share_objects(smd_ctx *from, smd_ctx *to, int lattice_id, int qset_id);
int smd_ctx_device(const smd_ctx *ctx);
size_t smd_ctx_budget(const smd_ctx *ctx);
void smd_copy_error(smd_ctx *to, const smd_ctx *from, long long job_id);

namespace {

struct Job {
    long long id = 0;
    smd_job_desc desc{};
    std::vector<double> spins, window;
    std::vector<int> imp;
    double *spec_out = nullptr, *qss_out = nullptr;
    int status = SMD_EBUSY;
    bool cancelled = false;
    std::chrono::steady_clock::time_point t_submit, t_done;
};

struct Server {
    smd_ctx *ctx = nullptr;
    std::mutex mu;
    std::condition_variable cv, done_cv;
    std::deque<std::shared_ptr<Job>> queue;
    std::map<long long, std::shared_ptr<Job>> jobs;
    long long next = 1;
    bool stop = false;
    std::vector<std::thread> workers;

    void run(int lanes)
    {
        // the lane's own context
        smd_ctx *w = nullptr;
        smd_device_opts o{};
        o.device = smd_ctx_device(ctx);
        size_t fr = 0, tot = 0;
        cudaSetDevice(o.device);
        cudaMemGetInfo(&fr, &tot);
        o.hbm_budget = std::min(smd_ctx_budget(ctx), (size_t)(0.85 * (double)fr)) / (size_t)lanes;
        const int crc = smd_ctx_create(&o, &w);
        for (;;) {
            std::shared_ptr<Job> j;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || !queue.empty(); });
                if (stop && queue.empty()) break;
                j = queue.front();
                queue.pop_front();
                if (j->cancelled) {
                    j->status = SMD_ECANCELLED;
                    j->t_done = std::chrono::steady_clock::now();
                    done_cv.notify_all();
                    continue;
                }
            }
            j->desc.imp = j->imp.empty() ? nullptr : j->imp.data();
            int rc = crc ? SMD_ECUDA : smd_share_objects(ctx, w, j->desc.lattice, j->desc.qset);
            if (rc == SMD_OK)
                rc = smd_run(w, &j->desc, j->spins.data(), j->window.data(), j->spec_out,
                             j->qss_out, nullptr, nullptr);
            if (rc != SMD_OK && w) smd_copy_error(ctx, w, j->id);   // for smd_last_error
            {
                std::lock_guard<std::mutex> lk(mu);
                j->status = rc;
                j->t_done = std::chrono::steady_clock::now();
            }
            done_cv.notify_all();
        }
        if (w) smd_ctx_destroy(w);
    }
};

std::mutex g_mu;
// never destroyed: lanes still blocked at process exit must not meet a
// destroyed registry (smd_serve_shutdown is the orderly end)
auto &g_servers = *new std::map<smd_ctx *, std::unique_ptr<Server>>();

Server *server_for(smd_ctx *ctx)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_servers.find(ctx);
    if (it != g_servers.end()) return it->second.get();
    auto s = std::make_unique<Server>();
    s->ctx = ctx;
    Server *p = s.get();
    int lanes = 1;
    if (const char *e = std::getenv("SMD_SERVE_LANES")) lanes = std::atoi(e);
    lanes = std::max(1, std::min(lanes, 16));
    for (int i = 0; i < lanes; i++) p->workers.emplace_back([p, lanes] { p->run(lanes); });
    g_servers[ctx] = std::move(s);
    return p;
}

}  // namespace

extern "C" void smd_serve_shutdown(smd_ctx *ctx)
{
    std::unique_ptr<Server> s;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_servers.find(ctx);
        if (it == g_servers.end()) return;
        s = std::move(it->second);
        g_servers.erase(it);
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    for (auto &t : s->workers)
        if (t.joinable()) t.join();
}

extern "C" int smd_submit(smd_ctx *ctx, const smd_job_desc *job, const double *spins0,
                          const double *window, double *spec_out, double *qss_out,
                          long long *job_id)
{
    if (!ctx || !job || !spins0 || !window || !spec_out || !qss_out || !job_id) return SMD_EINVAL;
    int N = 0;
    // N comes from the lattice; the q-set size check happens in smd_run
    {
        int Q = 0;
        if (smd_qset_size(ctx, job->qset, &Q) != SMD_OK) return SMD_ENOTFOUND;
    }
    if (smd_lattice_sites(ctx, job->lattice, &N) != SMD_OK) return SMD_ENOTFOUND;
    if (job->n_samples < 1 || job->n_rec < 2) return SMD_EINVAL;
    auto j = std::make_shared<Job>();
    j->desc = *job;
    j->spins.assign(spins0, spins0 + (size_t)job->n_samples * N * 3);
    j->window.assign(window, window + job->n_rec);
    if (job->imp) j->imp.assign(job->imp, job->imp + (size_t)job->n_samples * N);
    j->spec_out = spec_out;
    j->qss_out = qss_out;
    j->t_submit = std::chrono::steady_clock::now();
    Server *s = server_for(ctx);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        j->id = s->next++;
        s->jobs[j->id] = j;
        s->queue.push_back(j);
        *job_id = j->id;
    }
    s->cv.notify_all();
    return SMD_OK;
}

static int job_state(Server *s, long long id, double *latency_ms)
{
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return SMD_ENOTFOUND;
    Job &j = *it->second;
    if (j.status == SMD_EBUSY) return SMD_EBUSY;
    if (latency_ms)
        *latency_ms = std::chrono::duration<double, std::milli>(j.t_done - j.t_submit).count();
    return j.status;
}

extern "C" int smd_poll(smd_ctx *ctx, long long job_id, double *latency_ms)
{
    if (!ctx) return SMD_EINVAL;
    Server *s = server_for(ctx);
    std::lock_guard<std::mutex> lk(s->mu);
    return job_state(s, job_id, latency_ms);
}

extern "C" int smd_wait(smd_ctx *ctx, long long job_id, double timeout_ms, double *latency_ms)
{
    if (!ctx) return SMD_EINVAL;
    Server *s = server_for(ctx);
    std::unique_lock<std::mutex> lk(s->mu);
    auto pred = [&] { return job_state(s, job_id, nullptr) != SMD_EBUSY; };
    if (timeout_ms < 0) {
        s->done_cv.wait(lk, pred);
    } else if (!s->done_cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), pred)) {
        return SMD_ETIMEOUT;
    }
    return job_state(s, job_id, latency_ms);
}

extern "C" int smd_cancel(smd_ctx *ctx, long long job_id)
{
    if (!ctx) return SMD_EINVAL;
    Server *s = server_for(ctx);
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return SMD_ENOTFOUND;
    if (it->second->status != SMD_EBUSY) return it->second->status;
    it->second->cancelled = true;
    return SMD_OK;
}
