// serve.cpp -- job submission interface (smd_submit / smd_poll / smd_wait /
// smd_cancel).
//
// Jobs are copied at submit time and executed by one worker thread per
// context, in arrival order, through smd_run.  The output buffers named at
// submit are written when the job finishes; smd_poll reports SMD_EBUSY until
// then and returns the job's latency (submit to completion) afterwards.
#include "../../include/smd_b200.h"

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

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
    std::thread worker;

    void run()
    {
        for (;;) {
            std::shared_ptr<Job> j;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || !queue.empty(); });
                if (stop && queue.empty()) return;
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
            const int rc = smd_run(ctx, &j->desc, j->spins.data(), j->window.data(), j->spec_out,
                                   j->qss_out, nullptr, nullptr);
            {
                std::lock_guard<std::mutex> lk(mu);
                j->status = rc;
                j->t_done = std::chrono::steady_clock::now();
            }
            done_cv.notify_all();
        }
    }
};

std::mutex g_mu;
std::map<smd_ctx *, std::unique_ptr<Server>> g_servers;

Server *server_for(smd_ctx *ctx)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_servers.find(ctx);
    if (it != g_servers.end()) return it->second.get();
    auto s = std::make_unique<Server>();
    s->ctx = ctx;
    Server *p = s.get();
    p->worker = std::thread([p] { p->run(); });
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
    if (s->worker.joinable()) s->worker.join();
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
