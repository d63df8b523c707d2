// host.cu -- C ABI of the SMD library: context, lattice and q-set upload,
// and the job pipeline.
//
// A job (the reference's RK loop over samples, Codes_Folder/smd_code.cpp:
// 3079-3291, with get_dynSpectrum per sample) runs in waves of W samples that
// fit the context's HBM budget.  Within a wave the records are produced in
// chunks of R records:
//
//   stream rk   : RK kernel (one CTA, or one cluster of CTAs, per sample)
//                 writes the chunk's spin snapshots into one of two
//                 snapshot buffers
//   stream proj : grid projection (2D FFT) and list projection of the chunk,
//                 writing the windowed w[t] S(q,t) into the wave's q-blocked
//                 time series (series_off)
//
// so the projection of chunk c overlaps the integration of chunk c+1 on the
// SMs the RK kernel leaves free.  After the last chunk the time-FFT kernel
// transforms and squares every series and adds the sum over the wave's
// samples into the job's accumulator.
#include "host_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <tuple>
#include <vector>

using namespace smd;
using namespace smdh;

namespace {

const char *kVersion = "smd_b200 0.2 (sm_100a)";

}  // namespace

namespace smdh {

int fail(smd_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg;
    return code;
}

int cuda_fail(smd_ctx *c, cudaError_t e, const char *where)
{
    return fail(c, SMD_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// Radices of an FFT of length n.  wide: radix 16 and 8 first (the grid
// transform, whose stages hold 16 values per thread), else radix 4 first.
bool make_plan(int n, FFTPlan &p, bool wide)
{
    p.n = n;
    p.nst = 0;
    int m = n;
    if (wide) {
        for (int r : {16, 8}) {
            while (m % r == 0 && p.nst < 16) { p.radix[p.nst++] = r; m /= r; }
        }
    }
    while (m % 4 == 0 && m > 4 && p.nst < 16) { p.radix[p.nst++] = 4; m /= 4; }
    for (int r : {4, 2, 3, 5}) {
        while (m % r == 0 && m > 1 && p.nst < 16) { p.radix[p.nst++] = r; m /= r; }
    }
    for (int r = 7; m > 1 && p.nst < 16; r += 2) {
        while (m % r == 0 && p.nst < 16) {
            if (r > 64) return false;   // large primes are not supported
            p.radix[p.nst++] = r;
            m /= r;
        }
    }
    return m == 1;
}

// bf16 bits of x, rounded to nearest even (x finite)
uint16_t bf16_bits(float x)
{
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

float bf16_value(uint16_t h)
{
    const uint32_t u = (uint32_t)h << 16;
    float x;
    std::memcpy(&x, &u, 4);
    return x;
}

// exp(-2 pi i j / n) for j < n, accurate to one rounding
void twiddles(int n, std::vector<double> &w)
{
    w.resize(2 * (size_t)n);
    const double two_pi = 2.0 * std::acos(-1.0);
    for (int j = 0; j < n; j++) {
        const long jj = (2L * j > n) ? (long)j - n : j;
        const double a = two_pi * (double)jj / (double)n;
        w[2 * j] = std::cos(a);
        w[2 * j + 1] = -std::sin(a);
    }
}

cudaError_t upload_twiddles(int n, DevBuf &d64, DevBuf &d32)
{
    std::vector<double> w;
    twiddles(n, w);
    std::vector<float> wf(w.begin(), w.end());
    cudaError_t e = d64.ensure(w.size() * sizeof(double));
    if (e != cudaSuccess) return e;
    e = cudaMemcpy(d64.p, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    e = d32.ensure(wf.size() * sizeof(float));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(d32.p, wf.data(), wf.size() * sizeof(float), cudaMemcpyHostToDevice);
}

}  // namespace smdh

namespace {

// E = 1/2 sum_i (S_i . h_i - h S_i^z) equals the bond sum when every
// neighbour relation is a bond listed once, present in both directions in
// the same shell, with one coupling sign.
bool field_energy_identity(const smd_lattice_desc *d)
{
    const int N = d->N;
    std::map<std::tuple<int, int>, std::pair<int, int>> edges;   // (i,j) -> (shell, count)
    std::map<std::tuple<int, int>, int> sign;                    // Lieb d-wave sign per edge
    for (int s = 0; s < 3; s++) {
        if (!d->shell_on[s]) continue;
        for (int i = 0; i < N; i++)
            for (int k = 0; k < d->zn[s]; k++) {
                const int j = d->nbr[s][i * d->zn[s] + k];
                if (j < 0 || j == i) return false;
                auto key = std::make_tuple(i, j);
                auto it = edges.find(key);
                if (it != edges.end()) return false;   // duplicate neighbour
                edges[key] = {s, 1};
                sign[key] = ((i & 1) ? -1 : 1) * ((k & 1) ? -1 : 1);
            }
    }
    for (auto &e : edges) {
        const int i = std::get<0>(e.first), j = std::get<1>(e.first);
        auto r = edges.find(std::make_tuple(j, i));
        if (r == edges.end() || r->second.first != e.second.first) return false;
        if (d->lieb_delta_on && e.second.first == 1) {
            const int bond_sign = ((i & 1) ? -1 : 1) * ((j & 1) ? -1 : 1);
            if (sign[e.first] != bond_sign || sign[r->first] != bond_sign) return false;
        }
    }
    // the bond list holds every undirected edge once, in its shell
    const int nb = d->nbonds[0] + d->nbonds[1] + d->nbonds[2];
    if ((size_t)nb * 2 != edges.size()) return false;
    int b = 0;
    for (int s = 0; s < 3; s++)
        for (int q = 0; q < d->nbonds[s]; q++, b++) {
            const int i = d->bonds[2 * b], j = d->bonds[2 * b + 1];
            auto it = edges.find(std::make_tuple(i, j));
            if (it == edges.end() || it->second.first != s) return false;
        }
    return true;
}

}  // namespace

// ====================================================================== ABI

extern "C" const char *smd_version(void) { return kVersion; }

extern "C" const char *smd_last_error(const smd_ctx *ctx)
{
    return ctx ? ctx->err.c_str() : "null context";
}

extern "C" int smd_ctx_create(const smd_device_opts *opts, smd_ctx **out)
{
    if (!out) return SMD_EINVAL;
    *out = nullptr;
    std::unique_ptr<smd_ctx> c(new smd_ctx());
    smd_ctx *ctx = c.get();
    c->device = opts ? opts->device : 0;
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (c->device < 0 || c->device >= ndev) return SMD_EINVAL;
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, c->device), "cudaGetDeviceProperties");
    if (prop.major != 10) {
        // the kernels are built for sm_100a only
        return SMD_EINVAL;
    }
    size_t fr = 0, tot = 0;
    CK(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo");
    c->budget = (opts && opts->hbm_budget) ? opts->hbm_budget : (size_t)(0.85 * (double)fr);
    // the integration stream is on the critical path: its launches take SMs
    // ahead of the projection's blocks as they free up
    int prio_lo = 0, prio_hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi), "stream priorities");
    CK(cudaStreamCreateWithPriority(&c->s_rk, cudaStreamNonBlocking, prio_hi), "stream");
    CK(cudaStreamCreateWithPriority(&c->s_proj, cudaStreamNonBlocking, prio_lo), "stream");
    for (int i = 0; i < 3; i++) CK(cudaEventCreateWithFlags(&c->ev_tf[i], cudaEventDisableTiming), "event");
    for (int i = 0; i < kSnapBufs; i++) {
        CK(cudaEventCreateWithFlags(&c->ev_rk[i], cudaEventDisableTiming), "event");
        CK(cudaEventCreateWithFlags(&c->ev_proj[i], cudaEventDisableTiming), "event");
    }
    CK(cudaEventCreate(&c->t0), "event");
    CK(cudaEventCreate(&c->t1), "event");
    *out = c.release();
    return SMD_OK;
}

extern "C" int smd_ctx_destroy(smd_ctx *ctx)
{
    if (!ctx) return SMD_EINVAL;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    ctx->batches.clear();
    ctx->lattices.clear();
    ctx->qsets.clear();
    ctx->tplans.clear();
    for (int i = 0; i < 3; i++) cudaEventDestroy(ctx->ev_tf[i]);
    for (int i = 0; i < kSnapBufs; i++) {
        cudaEventDestroy(ctx->ev_rk[i]);
        cudaEventDestroy(ctx->ev_proj[i]);
    }
    for (cudaEvent_t e : ctx->tev) cudaEventDestroy(e);
    cudaEventDestroy(ctx->t0);
    cudaEventDestroy(ctx->t1);
    cudaStreamDestroy(ctx->s_rk);
    cudaStreamDestroy(ctx->s_proj);
    delete ctx;
    return SMD_OK;
}

extern "C" int smd_lattice_upload(smd_ctx *ctx, const smd_lattice_desc *d, int *lattice_id)
{
    if (!ctx || !d || !lattice_id) return SMD_EINVAL;
    if (d->N <= 0) return fail(ctx, SMD_EINVAL, "lattice: N must be positive");
    for (int s = 0; s < 3; s++) {
        if (d->zn[s] < 0 || d->zn[s] > kMaxShellNb) return fail(ctx, SMD_EINVAL, "lattice: zn must lie in [0, 8]");
        if (d->shell_on[s] && d->zn[s] > 0 && !d->nbr[s])
            return fail(ctx, SMD_EINVAL, "lattice: missing neighbour table");
    }
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    auto L = std::make_unique<Lattice>();
    const int N = d->N;
    L->N = N;
    L->G = d->G;
    int z = 0;
    for (int s = 0; s < 3; s++) {
        L->zn[s] = d->shell_on[s] ? d->zn[s] : 0;
        L->zoff[s] = z;
        z += L->zn[s];
    }
    L->ztot = z;
    // ELL [ztot][N]
    std::vector<int> ell((size_t)std::max(z, 1) * N, -1);
    for (int s = 0; s < 3; s++)
        for (int k = 0; k < L->zn[s]; k++)
            for (int i = 0; i < N; i++) {
                const int j = d->nbr[s][i * d->zn[s] + k];
                if (j >= N) return fail(ctx, SMD_EINVAL, "lattice: neighbour index out of range");
                ell[(size_t)(L->zoff[s] + k) * N + i] = j;
            }
    CK(L->nbr.ensure(ell.size() * sizeof(int)), "cudaMalloc");
    CK(cudaMemcpy(L->nbr.p, ell.data(), ell.size() * sizeof(int), cudaMemcpyHostToDevice), "H2D");
    if (d->G > 0) {
        if (!d->grid_map) return fail(ctx, SMD_EINVAL, "lattice: G > 0 needs grid_map");
        for (int k = 0; k < d->G * d->G; k++)
            if (d->grid_map[k] >= N) return fail(ctx, SMD_EINVAL, "lattice: grid map out of range");
        CK(L->grid_map.ensure((size_t)d->G * d->G * sizeof(int)), "cudaMalloc");
        CK(cudaMemcpy(L->grid_map.p, d->grid_map, (size_t)d->G * d->G * sizeof(int),
                      cudaMemcpyHostToDevice), "H2D");
    }
    const int nb = d->nbonds[0] + d->nbonds[1] + d->nbonds[2];
    std::vector<int4> bonds((size_t)std::max(nb, 1));
    {
        int b = 0;
        for (int s = 0; s < 3; s++)
            for (int q = 0; q < d->nbonds[s]; q++, b++) {
                const int i = d->bonds[2 * b], j = d->bonds[2 * b + 1];
                if (i < 0 || j < 0 || i >= N || j >= N)
                    return fail(ctx, SMD_EINVAL, "lattice: bond index out of range");
                bonds[b] = make_int4(i, j, s, 0);
            }
    }
    CK(L->bonds.ensure(bonds.size() * sizeof(int4)), "cudaMalloc");
    CK(cudaMemcpy(L->bonds.p, bonds.data(), bonds.size() * sizeof(int4), cudaMemcpyHostToDevice), "H2D");
    if (d->pos) L->pos.assign(d->pos, d->pos + 2 * (size_t)N);

    LatticeDev &v = L->dev;
    std::memset(&v, 0, sizeof v);
    v.N = N;
    for (int s = 0; s < 3; s++) {
        v.zn[s] = L->zn[s];
        v.zoff[s] = L->zoff[s];
        v.shell_on[s] = d->shell_on[s] && L->zn[s] > 0;
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) {
                v.J[s][a][b] = d->J[s][a][b];
                v.Jf[s][a][b] = (float)d->J[s][a][b];
            }
        for (int c = 0; c < 3; c++) {
            v.lam[s][c] = d->lambda[s][c];
            v.lamf[s][c] = (float)d->lambda[s][c];
            v.coef[s][c] = d->J[s][0][0] * d->lambda[s][c];
            v.coeff[s][c] = (float)v.coef[s][c];
        }
    }
    v.ztot = z;
    v.nbr = L->nbr.as<int>();
    v.lieb_delta_on = d->lieb_delta_on && std::fabs(d->j2_delta) > 1.0e-12;
    v.j2_delta = d->j2_delta;
    v.j2_deltaf = (float)d->j2_delta;
    v.h = std::fabs(d->h) > 1.0e-12 ? d->h : 0.0;   // extH_ON, subrouts.cpp:1282-1285
    v.hf = (float)v.h;
    v.energy_from_field = field_energy_identity(d) ? 1 : 0;
    v.nbonds = nb;
    v.bonds = L->bonds.as<int4>();
    L->lieb_delta = v.lieb_delta_on;
    for (int s = 0; s < 3; s++) {
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++)
                if ((a || b) && d->J[s][a][b] != 0.0) L->vac_only = false;
        if (v.shell_on[s])
            L->nbr_h[s].assign(d->nbr[s], d->nbr[s] + (size_t)N * d->zn[s]);
    }
    const int id = ctx->next_id++;
    {
        std::lock_guard<std::mutex> lk(ctx->maps_mu);
        ctx->lattices[id] = std::move(L);
    }
    *lattice_id = id;
    return SMD_OK;
}

extern "C" int smd_lattice_free(smd_ctx *ctx, int lattice_id)
{
    if (!ctx) return SMD_EINVAL;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    std::lock_guard<std::mutex> lk(ctx->maps_mu);
    if (!ctx->lattices.erase(lattice_id)) return SMD_ENOTFOUND;
    return SMD_OK;
}

extern "C" int smd_qset_upload(smd_ctx *ctx, int lattice_id, int use_grid, int n_list,
                               const double *qlist, double list_scale, int *qset_id)
{
    if (!ctx || !qset_id) return SMD_EINVAL;
    std::shared_ptr<Lattice> Lp;
    {
        std::lock_guard<std::mutex> lk(ctx->maps_mu);
        auto it = ctx->lattices.find(lattice_id);
        if (it == ctx->lattices.end()) return fail(ctx, SMD_ENOTFOUND, "qset: unknown lattice");
        Lp = it->second;
    }
    Lattice &L = *Lp;
    if (n_list < 0 || (n_list > 0 && !qlist)) return fail(ctx, SMD_EINVAL, "qset: bad q list");
    if (n_list > 0 && L.pos.empty()) return fail(ctx, SMD_EINVAL, "qset: lattice has no positions");
    if (use_grid && L.G <= 0) return fail(ctx, SMD_EINVAL, "qset: lattice has no DFT grid");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    auto Q = std::make_unique<QSet>();
    Q->lattice = lattice_id;
    Q->use_grid = use_grid ? 1 : 0;
    Q->G = use_grid ? L.G : 0;
    Q->n_list = n_list;
    Q->Q = Q->G * Q->G + n_list;
    Q->list_scale = list_scale;
    if (Q->Q <= 0) return fail(ctx, SMD_EINVAL, "qset: empty");
    if (use_grid) {
        if (!make_plan(L.G, Q->gplan, true)) return fail(ctx, SMD_EINVAL, "qset: grid size has a prime factor > 64");
        // SMD_GRID_TWO_PASS=1 sends grids that fit one block through the
        // two-pass transform too (tests compare the two)
        const char *tp = std::getenv("SMD_GRID_TWO_PASS");
        const bool force_two = tp && std::atoi(tp) != 0;
        for (int prec : {0, 1}) {
            if (force_two && grid_large_ok(L.G, prec, Q->gplan)) {
                Q->large[prec] = 1;
                continue;
            }
            if (grid_proj_ng(L.G, prec, Q->gplan)) continue;
            if (!grid_large_ok(L.G, prec, Q->gplan)) {
                if (prec == 1) return fail(ctx, SMD_EINVAL, "qset: grid too large for the shared-memory transforms");
                Q->fp64_ok = 0;
            } else {
                Q->large[prec] = 1;
            }
        }
        CK(upload_twiddles(L.G, Q->tw64, Q->tw32), "twiddles");
    }
    if (n_list > 0) {
        const int N = L.N;
        std::vector<double> ph((size_t)N * n_list * 2);
        for (int k = 0; k < N; k++)
            for (int l = 0; l < n_list; l++) {
                const double a = -(qlist[2 * l] * L.pos[2 * k] + qlist[2 * l + 1] * L.pos[2 * k + 1]);
                ph[2 * ((size_t)k * n_list + l)] = list_scale * std::cos(a);
                ph[2 * ((size_t)k * n_list + l) + 1] = list_scale * std::sin(a);
            }
        CK(Q->phase64.ensure(ph.size() * sizeof(double)), "cudaMalloc");
        CK(cudaMemcpy(Q->phase64.p, ph.data(), ph.size() * sizeof(double), cudaMemcpyHostToDevice), "H2D");
        // split-bf16 operand of the tensor-core projection, [2 n_list][kp]
        const int kp = tc_kpitch(N);
        Q->kp = kp;
        std::vector<uint16_t> bh((size_t)2 * n_list * kp, 0), bl((size_t)2 * n_list * kp, 0);
        for (int l = 0; l < n_list; l++)
            for (int k = 0; k < N; k++)
                for (int part = 0; part < 2; part++) {
                    const double x = ph[2 * ((size_t)k * n_list + l) + part];
                    const uint16_t hi = bf16_bits((float)x);
                    const uint16_t lo = bf16_bits((float)(x - (double)bf16_value(hi)));
                    bh[((size_t)2 * l + part) * kp + k] = hi;
                    bl[((size_t)2 * l + part) * kp + k] = lo;
                }
        CK(Q->bhi.ensure(bh.size() * 2), "cudaMalloc");
        CK(Q->blo.ensure(bl.size() * 2), "cudaMalloc");
        CK(cudaMemcpy(Q->bhi.p, bh.data(), bh.size() * 2, cudaMemcpyHostToDevice), "H2D");
        CK(cudaMemcpy(Q->blo.p, bl.data(), bl.size() * 2, cudaMemcpyHostToDevice), "H2D");
        if (!make_bf16_map(&Q->map_bhi, Q->bhi.p, 2 * n_list, kp, tc_bn()) ||
            !make_bf16_map(&Q->map_blo, Q->blo.p, 2 * n_list, kp, tc_bn()))
            return fail(ctx, SMD_ECUDA, "qset: tensor map encoding failed");
    }
    const int id = ctx->next_id++;
    {
        std::lock_guard<std::mutex> lk(ctx->maps_mu);
        ctx->qsets[id] = std::move(Q);
    }
    *qset_id = id;
    return SMD_OK;
}

extern "C" int smd_qset_size(smd_ctx *ctx, int qset_id, int *Q)
{
    if (!ctx || !Q) return SMD_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->maps_mu);
    auto it = ctx->qsets.find(qset_id);
    if (it == ctx->qsets.end()) return SMD_ENOTFOUND;
    *Q = it->second->Q;
    return SMD_OK;
}

namespace smdh {

std::shared_ptr<Lattice> find_lattice(smd_ctx *ctx, int id)
{
    std::lock_guard<std::mutex> lk(ctx->maps_mu);
    auto it = ctx->lattices.find(id);
    return it == ctx->lattices.end() ? nullptr : it->second;
}

std::shared_ptr<QSet> find_qset(smd_ctx *ctx, int id)
{
    std::lock_guard<std::mutex> lk(ctx->maps_mu);
    auto it = ctx->qsets.find(id);
    return it == ctx->qsets.end() ? nullptr : it->second;
}

int time_plan(smd_ctx *ctx, int n, Plan **out)
{
    auto pi = ctx->tplans.find(n);
    if (pi == ctx->tplans.end()) {
        auto P = std::make_unique<Plan>();
        if (!make_plan(n, P->p, false)) return fail(ctx, SMD_EINVAL, "job: n_rec has a prime factor > 64");
        CK(upload_twiddles(n, P->tw64, P->tw32), "twiddles");
        pi = ctx->tplans.emplace(n, std::move(P)).first;
    }
    *out = pi->second.get();
    return SMD_OK;
}

bool cluster_ok(const Lattice &L)
{
    return L.dev.energy_from_field && !L.lieb_delta && L.vac_only;
}

// Partition of lattice L over CS CTAs: contiguous site ranges, halo lists,
// packed local neighbour slots and halo push lists.  Edge slots beyond the
// lattice's neighbours (up to the kernel's ZT) name the zero pad slot.
// Null when the lattice does not fit the cluster kernel's limits.
ClusterTab *cluster_tables(Lattice &L, int CS, int zt_min)
{
    const int N = L.N;
    if (CS < 1 || CS > kMaxClusterCTAs || N < CS) return nullptr;
    const int zact = L.zn[0] + L.zn[1] + L.zn[2];
    const int zneed = std::max(zact, zt_min);
    const int ZT = zneed <= 4    ? 4
                   : zneed <= 8  ? 8
                   : zneed <= 12 ? 12
                   : zneed <= 14 ? 14
                   : zneed <= 18 ? 18
                   : zneed <= 20 ? 20
                                 : -1;
    if (ZT < 0) return nullptr;
    std::lock_guard<std::mutex> lk(L.cache_mu);
    auto it = L.ctabs.find({CS, ZT});
    if (it != L.ctabs.end()) return it->second.get();
    std::vector<int> base(CS + 1), owner(N);
    for (int r = 0; r <= CS; r++) base[r] = (int)((long long)N * r / CS);
    for (int r = 0; r < CS; r++)
        for (int g = base[r]; g < base[r + 1]; g++) owner[g] = r;
    // neighbours of site g over the active shells, in edge-slot order
    auto edge = [&](int g, int e) -> int {
        for (int s = 0; s < 3; s++) {
            if (e < L.zn[s]) return L.nbr_h[s][(size_t)g * L.zn[s] + e];
            e -= L.zn[s];
        }
        return -1;
    };
    std::vector<std::vector<int>> halo(CS);
    int n_own_max = 0, n_loc_max = 0;
    for (int r = 0; r < CS; r++) {
        std::set<int> hs;
        for (int g = base[r]; g < base[r + 1]; g++)
            for (int e = 0; e < zact; e++) {
                const int j = edge(g, e);
                if (j >= 0 && owner[j] != r) hs.insert(j);
            }
        halo[r].assign(hs.begin(), hs.end());
        const int own = base[r + 1] - base[r];
        n_own_max = std::max(n_own_max, own);
        n_loc_max = std::max(n_loc_max, own + (int)halo[r].size());
    }
    if (n_loc_max + 1 > 65536) return nullptr;
    const int pad = n_loc_max;
    std::vector<uint32_t> idx((size_t)CS * (ZT / 2) * n_own_max, (uint32_t)pad | ((uint32_t)pad << 16));
    std::vector<int> hgid((size_t)CS * n_loc_max, 0);
    std::vector<std::vector<std::vector<int>>> pushes(CS);
    for (int r = 0; r < CS; r++) pushes[r].resize(base[r + 1] - base[r]);
    for (int r = 0; r < CS; r++) {
        const int own = base[r + 1] - base[r];
        std::map<int, int> hslot;
        for (size_t q = 0; q < halo[r].size(); q++) {
            const int j = halo[r][q];
            hslot[j] = own + (int)q;
            hgid[(size_t)r * n_loc_max + q] = j;
            const int o = owner[j];
            pushes[o][j - base[o]].push_back((r << 16) | (own + (int)q));
        }
        for (int li = 0; li < own; li++) {
            const int g = base[r] + li;
            for (int e = 0; e < ZT; e++) {
                int sl = pad;
                const int j = e < zact ? edge(g, e) : -1;
                if (j >= 0) sl = (owner[j] == r) ? j - base[r] : hslot[j];
                uint32_t &w = idx[((size_t)r * (ZT / 2) + e / 2) * n_own_max + li];
                if (e % 2 == 0) w = (w & 0xffff0000u) | (uint32_t)sl;
                else w = (w & 0x0000ffffu) | ((uint32_t)sl << 16);
            }
        }
    }
    // Async halo pushes need a symmetric neighbour relation between CTAs: a
    // site reads a halo copy owned by CTA o exactly when CTA o holds a copy
    // of the site.  A publish's bytes also have to fit one mbarrier
    // transaction count (below 2^20).
    bool sym = true;
    size_t max_halo = 0;
    for (int r = 0; r < CS && sym; r++) {
        max_halo = std::max(max_halo, halo[r].size());
        std::vector<int> reads, held;
        for (int g = base[r]; g < base[r + 1] && sym; g++) {
            reads.clear();
            held.clear();
            for (int e = 0; e < zact; e++) {
                const int j = edge(g, e);
                if (j >= 0 && owner[j] != r) reads.push_back(owner[j]);
            }
            for (int c : pushes[r][g - base[r]]) held.push_back(c >> 16);
            std::sort(reads.begin(), reads.end());
            reads.erase(std::unique(reads.begin(), reads.end()), reads.end());
            std::sort(held.begin(), held.end());
            held.erase(std::unique(held.begin(), held.end()), held.end());
            sym = reads == held;
        }
    }
    const bool async_ok = sym && max_halo * 24 < (1u << 20);
    int pmax = 0;
    for (int r = 0; r < CS; r++)
        for (auto &v : pushes[r]) pmax = std::max(pmax, (int)v.size());
    std::vector<int> push((size_t)CS * std::max(pmax, 1) * n_own_max, -1);
    for (int r = 0; r < CS; r++)
        for (size_t li = 0; li < pushes[r].size(); li++)
            for (size_t p = 0; p < pushes[r][li].size(); p++)
                push[((size_t)r * pmax + p) * n_own_max + li] = pushes[r][li][p];
    std::vector<int> cnt(CS), hc(CS);
    for (int r = 0; r < CS; r++) {
        cnt[r] = base[r + 1] - base[r];
        hc[r] = (int)halo[r].size();
    }

    auto T = std::make_unique<ClusterTab>();
    ClusterParams &P = T->P;
    P.N = N;
    P.CS = CS;
    P.n_own_max = n_own_max;
    P.n_loc_max = n_loc_max;
    P.pmax = pmax;
    P.ZT = ZT;
    P.energy_from_field = L.dev.energy_from_field;
    P.async_halo = async_ok ? 1 : 0;
    P.h = L.dev.h;
    P.hf = (float)L.dev.h;
    for (int e = 0; e < kMaxEdgeSlots; e++)
        for (int c = 0; c < 3; c++) {
            P.coef64[e][c] = 0.0;
            P.coef32[e][c] = 0.0f;
        }
    for (int e = 0; e < zact; e++) {
        int s = 0, k = e;
        while (k >= L.zn[s]) k -= L.zn[s++];
        for (int c = 0; c < 3; c++) {
            P.coef64[e][c] = L.dev.coef[s][c];
            P.coef32[e][c] = (float)L.dev.coef[s][c];
        }
    }
    auto up = [](DevBuf &b, const void *src, size_t bytes) {
        if (b.ensure(std::max<size_t>(bytes, 4)) != cudaSuccess) return false;
        return cudaMemcpy(b.p, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
    };
    if (!up(T->own_base, base.data(), CS * sizeof(int)) || !up(T->own_cnt, cnt.data(), CS * sizeof(int)) ||
        !up(T->halo_cnt, hc.data(), CS * sizeof(int)) ||
        !up(T->halo_gid, hgid.data(), hgid.size() * sizeof(int)) ||
        !up(T->idx, idx.data(), idx.size() * sizeof(uint32_t)) ||
        !up(T->push, push.data(), push.size() * sizeof(int)))
        return nullptr;
    P.own_base = T->own_base.as<int>();
    P.own_cnt = T->own_cnt.as<int>();
    P.halo_cnt = T->halo_cnt.as<int>();
    P.halo_gid = T->halo_gid.as<int>();
    P.idx = T->idx.as<uint32_t>();
    P.push = T->push.as<int>();
    ClusterTab *raw = T.get();
    L.ctabs[{CS, ZT}] = std::move(T);
    return raw;
}

int project_chunk(smd_ctx *ctx, const ProjArgs &a, cudaStream_t st, int *launches)
{
    Lattice &L = *a.L;
    QSet &Qs = *a.Qs;
    const int n = a.re - a.rb;
    const int p32 = a.prec == SMD_FP64 ? 0 : 1;
    if (Qs.use_grid) {
        const double scale = std::sqrt(1.0 / ((double)Qs.G * Qs.G));   // subrouts.cpp:8343
        const void *tw = p32 ? Qs.tw32.p : Qs.tw64.p;
        if (Qs.large[p32]) {
            CK(a.gscratch->ensure((size_t)a.W * grid_large_scratch(Qs.G, a.R, p32)), "cudaMalloc grid scratch");
            CK(launch_grid_proj_large(a.snap, a.prec, a.N, a.W, a.R, n, a.rb, a.n_rec, L.grid_map.as<int>(),
                                      Qs.gplan, tw, scale, a.win, a.series, a.nqb, a.gscratch->p, st),
               "grid projection (two passes)");
            *launches += 2;
        } else {
            CK(launch_grid_proj(a.snap, a.prec, a.N, a.W, a.R, n, a.rb, a.n_rec, L.grid_map.as<int>(), Qs.gplan,
                                tw, scale, a.win, a.series, a.nqb, st),
               "grid projection");
            *launches += 1;
        }
    }
    if (Qs.n_list > 0 && p32) {
        // split-BF16 tensor-core projection of the chunk's rows
        const int rows = a.W * a.R * 3;
        if (!a.fused_split) {
            CK(launch_split_bf16(static_cast<const float *>(a.snap), rows, a.N, Qs.kp, a.ahi, a.alo, st),
               "bf16 split");
            *launches += 1;
        }
        CK(launch_list_proj_tc(*a.map_ahi, *a.map_alo, Qs.map_bhi, Qs.map_blo, rows, Qs.kp, a.R, n, a.rb,
                               a.n_rec, Qs.n_list, a.win, a.series, a.nqb, Qs.G * Qs.G, a.status, st),
           "tensor-core list projection");
        *launches += 1;
    } else if (Qs.n_list > 0) {
        CK(launch_list_proj_f64(static_cast<const double *>(a.snap), a.W, a.R, n, a.N, a.rb, a.n_rec,
                                Qs.phase64.as<double>(), Qs.n_list, a.win, a.series, a.nqb, Qs.G * Qs.G, st),
           "FP64 list projection");
        *launches += 1;
    }
    return SMD_OK;
}

// Estimated RK time of a cluster shape, in units of one site's stage work at
// full SM throughput: the busiest SM runs ceil(CTAs / SMs) CTAs, k at a time
// (k from registers, shared memory and threads); a round of j CTAs of
// w warps each runs at min(1, j w / 20) of the SM's throughput; a CTA's work
// is its own sites plus half a site per halo copy, times 1.2 for four sites a
// thread (128 registers, spills), plus 60 site-units per CTA of the cluster
// (cluster-wide waits).  The constants were fitted to the RK times of every
// shape of twelve serving-mix jobs (five geometries, N 432-6084, 46-253
// samples): the shapes it picks ran within 3 % of the fastest measured per
// job, against 13 % for the fill rule below (9 % leaving each job out of
// the fit in turn).
static double shape_cost(const ClusterParams &P, int prec, int spt, int threads, int n_samples, int sms)
{
    const int regs = spt == 1 ? 80 : spt == 2 ? 96 : 128;   // the instances' register counts
    const int warps = threads / 32;
    const size_t smem = rk_cluster_smem(P, prec) + 1024;
    int k = std::min({65536 / (threads * regs), (int)((228 * 1024) / smem), 2048 / threads});
    k = std::max(k, 1);
    const long long ctas = (long long)n_samples * P.CS;
    long long rem = (ctas + sms - 1) / sms;
    double rounds = 0.0;
    while (rem > 0) {
        const int j = (int)std::min<long long>(k, rem);
        rounds += j / std::min(1.0, j * warps / 20.0);
        rem -= j;
    }
    const double spt_factor = spt == 4 ? 1.2 : 1.0;
    const double work = (P.n_own_max + 0.5 * (P.n_loc_max - P.n_own_max)) * spt_factor + 60.0 * P.CS;
    return rounds * work;
}

// Cluster size and thread shape for a job.  Lattices the cluster kernel does
// not cover (bond-list energies, the Lieb d-wave term, impurities with
// non-zero couplings) keep the single-CTA kernel.  Otherwise the shape of
// least estimated time (shape_cost) over every cluster size and
// sites-per-thread form that fits the shared-memory and register limits.
// SMD_CLUSTER_POLICY=fill takes instead the smallest cluster that puts at
// least ~85% of the SMs to work; SMD_CLUSTER_CTAS forces a size (with
// SMD_RK_SPT forcing the sites per thread).
ClusterTab *cluster_choice(Lattice &L, int prec, int n_samples, int device, int *spt_out, int *threads_out)
{
    if (!cluster_ok(L)) return nullptr;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    int forced = 0;
    if (const char *e = std::getenv("SMD_CLUSTER_CTAS")) forced = std::atoi(e);
    const char *pol = std::getenv("SMD_CLUSTER_POLICY");
    if (!forced && !(pol && std::strcmp(pol, "fill") == 0)) {
        ClusterTab *best = nullptr;
        double best_cost = 0.0;
        for (int CS : {1, 2, 4, 8, 16}) {
            if (CS > 1 && L.N / CS < 96) break;
            ClusterTab *t = cluster_tables(L, CS);
            if (!t || rk_cluster_smem(t->P, prec) > 227 * 1024) continue;
            for (int s : {1, 2, 4}) {
                if (s * rk_cluster_maxt(prec, s) < t->P.n_own_max) continue;
                const int thr = std::min(std::max(32, (t->P.n_own_max + s - 1) / s + 31) / 32 * 32,
                                         rk_cluster_maxt(prec, s));
                const double c = shape_cost(t->P, prec, s, thr, n_samples, sms);
                if (const char *tr = std::getenv("SMD_CLUSTER_TRACE")) {
                    // candidate shapes and their estimates, appended to a file
                    if (FILE *f = std::fopen(tr, "a")) {
                        std::fprintf(f, "N %d S %d CS %d spt %d thr %d own %d loc %d smem %zu cost %.1f\n", L.N,
                                     n_samples, CS, s, thr, t->P.n_own_max, t->P.n_loc_max,
                                     rk_cluster_smem(t->P, prec), c);
                        std::fclose(f);
                    }
                }
                if (!best || c < best_cost * 0.98) {
                    best = t;
                    best_cost = c;
                    *spt_out = s;
                    *threads_out = thr;
                }
            }
        }
        return best;
    }
    ClusterTab *best = nullptr;
    const int sizes[] = {1, 2, 4, 8, 16};
    for (int CS : sizes) {
        if (forced && CS != forced) continue;
        if (!forced && CS > 1 && L.N / CS < 96) break;
        ClusterTab *t = cluster_tables(L, CS);
        if (!t) continue;
        int spt = 0;
        // sites per thread: the fewest that fit a block (SMD_RK_SPT forces one)
        int force_spt = 0;
        if (const char *e = std::getenv("SMD_RK_SPT")) force_spt = std::atoi(e);
        for (int s : {1, 2, 4})
            if ((!force_spt || s == force_spt) && s * rk_cluster_maxt(prec, s) >= t->P.n_own_max) {
                spt = s;
                break;
            }
        if (!spt) continue;
        if (rk_cluster_smem(t->P, prec) > 227 * 1024) continue;
        best = t;
        *spt_out = spt;
        *threads_out = std::min(std::max(32, (t->P.n_own_max + spt - 1) / spt + 31) / 32 * 32,
                                rk_cluster_maxt(prec, spt));
        if (forced || (long long)n_samples * CS >= (long long)(0.85 * sms)) break;
    }
    return best;
}

}  // namespace smdh

namespace {

struct JobGeom {
    Lattice *L;
    QSet *Qs;
    Plan *tp;
    int N, Q, nqb, n_rec, prec, R, W, waves;   // nqb: q blocks of the series layout
    size_t elem, celem;
    ClusterTab *ctab = nullptr;   // cluster kernel partition (null: single-CTA kernel)
    int spt = 0, threads = 0;
};


void choose_cluster(smd_ctx *ctx, JobGeom &g, int n_samples)
{
    g.ctab = cluster_choice(*g.L, g.prec, n_samples, ctx->device, &g.spt, &g.threads);
}

int prepare(smd_ctx *ctx, const smd_job_desc *job, JobGeom &g)
{
    if (!job) return fail(ctx, SMD_EINVAL, "job: null");
    std::unique_lock<std::mutex> mlk(ctx->maps_mu);
    auto li = ctx->lattices.find(job->lattice);
    if (li == ctx->lattices.end()) return fail(ctx, SMD_ENOTFOUND, "job: unknown lattice");
    auto qi = ctx->qsets.find(job->qset);
    if (qi == ctx->qsets.end()) return fail(ctx, SMD_ENOTFOUND, "job: unknown q set");
    mlk.unlock();
    if (qi->second->lattice != job->lattice) return fail(ctx, SMD_EINVAL, "job: q set belongs to another lattice");
    if (job->n_samples < 1) return fail(ctx, SMD_EINVAL, "job: n_samples < 1");
    if (job->n_rec < 2) return fail(ctx, SMD_EINVAL, "job: n_rec < 2");
    if (job->stride < 1) return fail(ctx, SMD_EINVAL, "job: stride < 1");
    if (!(job->dt > 0.0)) return fail(ctx, SMD_EINVAL, "job: dt must be positive");
    if (job->precision != SMD_FP64 && job->precision != SMD_FP32)
        return fail(ctx, SMD_EINVAL, "job: unknown precision");
    if ((long long)(job->n_rec - 1) * job->stride > 2000000000LL)
        return fail(ctx, SMD_EINVAL, "job: too many steps");
    g.L = li->second.get();
    g.Qs = qi->second.get();
    g.N = g.L->N;
    g.Q = g.Qs->Q;
    g.n_rec = job->n_rec;
    g.prec = job->precision;
    g.nqb = (g.Q + series_qblock(g.prec) - 1) / series_qblock(g.prec);
    choose_cluster(ctx, g, job->n_samples);
    if (!g.ctab && g.N > rk_max_sites(g.prec))
        return fail(ctx, SMD_EINVAL, "job: N exceeds the single-CTA capacity of this form");
    if (g.Qs->use_grid && g.prec == SMD_FP64 && !g.Qs->fp64_ok)
        return fail(ctx, SMD_EINVAL, "job: grid too large for the FP64 shared-memory transform");
    g.elem = g.prec == SMD_FP64 ? sizeof(double) : sizeof(float);
    g.celem = 2 * g.elem;
    {
        int rc = time_plan(ctx, g.n_rec, &g.tp);
        if (rc) return rc;
    }
    if (!time_fft_fits(g.n_rec, g.prec, g.tp->p))
        return fail(ctx, SMD_EINVAL, "job: n_rec too long for the shared-memory time transform");
    // chunk of records per RK launch (C2 measured: 128 records 129.4 ms per
    // job step, 64 records 131.1 ms, 32 records 131.3 ms)
    g.R = std::min(g.n_rec, 128);
    // per-sample device bytes
    const size_t N = g.N;
    const bool large = g.Qs->use_grid && g.Qs->large[g.prec == SMD_FP64 ? 0 : 1];
    // FP32 list projection on tensor cores: split-BF16 rows beside every
    // snapshot buffer
    const size_t bf_rows = (g.Qs->n_list > 0 && g.prec == SMD_FP32) ? (size_t)g.R * 3 * g.Qs->kp * 4 : 0;
    const size_t per = 2 * 3 * N * sizeof(double) + N + kSnapBufs * ((size_t)g.R * 3 * N * g.elem + bf_rows) +
                       3 * (size_t)g.n_rec * g.nqb * 16 + (size_t)g.n_rec * sizeof(double) +
                       5 * sizeof(double) + (size_t)g.n_rec * kMaxClusterCTAs * sizeof(double) +
                       (large ? grid_large_scratch(g.Qs->G, g.R, g.prec == SMD_FP64 ? 0 : 1) : 0);
    const size_t fixed = 3 * (size_t)g.Q * g.n_rec * sizeof(double) + (64u << 20);
    // the budget, and no more than the device can give now: its free memory
    // plus the job buffers this context holds (they are reallocated), less
    // a reserve; the serving engine's unused pooled memory is returned first
    // when that is short
    size_t budget = ctx->budget;
    auto avail_now = [&]() -> size_t {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return ctx->budget;
        size_t held = ctx->state.bytes + ctx->s0.bytes + ctx->imp.bytes + ctx->series.bytes + ctx->qss.bytes +
                      ctx->qpart.bytes + ctx->stats.bytes + ctx->e0.bytes + ctx->gscratch.bytes;
        for (int b = 0; b < kSnapBufs; b++) held += ctx->snap[b].bytes + ctx->ahi[b].bytes + ctx->alo[b].bytes;
        const size_t reserve = (size_t)1 << 30;
        return fr + held > reserve ? fr + held - reserve : 0;
    };
    size_t avail = avail_now();
    if (avail < budget) {
        engine_trim(ctx);
        avail = avail_now();
    }
    budget = std::min(budget, avail);
    if (budget <= fixed + per) return fail(ctx, SMD_ENOMEM_ADMIT, "job: one sample exceeds the free HBM");
    size_t W = (budget - fixed) / per;
    W = std::min<size_t>(W, (size_t)job->n_samples);
    W = std::min<size_t>(W, 65535);
    g.W = (int)W;
    g.waves = (job->n_samples + g.W - 1) / g.W;
    // the RK launches run one wave of W samples at a time: shape them for W
    if (g.ctab && g.W < job->n_samples) choose_cluster(ctx, g, g.W);
    return SMD_OK;
}

// The pipeline of one job on device buffers; spec/qss sums accumulate.
int run_device(smd_ctx *ctx, const smd_job_desc *job, const JobGeom &g, const double *d_spins0,
               const double *d_win, double *d_spec_sum, double *d_qss_sum, double *d_final,
               smd_report *rep, double *h_spec = nullptr, double fc = 1.0)
{
    const int N = g.N, Q = g.Q, nqb = g.nqb, n_rec = g.n_rec, R = g.R, W = g.W;
    Lattice &L = *g.L;
    QSet &Qs = *g.Qs;
    // the job's buffers; when the device is short, the serving engine's
    // pooled memory that no group holds is returned to it and the buffers
    // are tried once more
    auto alloc_all = [&]() -> cudaError_t {
        cudaError_t e = ctx->state.ensure((size_t)W * 3 * N * sizeof(double));
        if (e == cudaSuccess) e = ctx->s0.ensure((size_t)W * 3 * N * sizeof(double));
        if (e == cudaSuccess) e = ctx->imp.ensure((size_t)W * N);
        for (int b = 0; b < kSnapBufs && e == cudaSuccess; b++)
            e = ctx->snap[b].ensure((size_t)W * R * 3 * N * g.elem);
        if (e == cudaSuccess) e = ctx->series.ensure((size_t)W * 3 * n_rec * nqb * 16);
        if (e == cudaSuccess) e = ctx->qss.ensure((size_t)W * n_rec * sizeof(double));
        if (e == cudaSuccess && g.ctab) e = ctx->qpart.ensure((size_t)W * n_rec * g.ctab->P.CS * sizeof(double));
        if (e == cudaSuccess) e = ctx->stats.ensure((size_t)W * 4 * sizeof(double));
        if (e == cudaSuccess) e = ctx->e0.ensure((size_t)W * sizeof(double));
        if (e == cudaSuccess) e = ctx->status.ensure(sizeof(int));
        return e;
    };
    cudaError_t ae = alloc_all();
    if (ae == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        engine_trim(ctx);
        ae = alloc_all();
    }
    CK(ae, "cudaMalloc job buffers");
    CK(cudaMemsetAsync(ctx->status.p, 0, sizeof(int), ctx->s_rk), "memset");
    const bool gen = L.lieb_delta || job->imp;
    std::vector<double> stats_h;
    double drift_max = 0.0, drift_final = 0.0;
    double ms_dev = 0.0, ms_rk = 0.0, ms_proj = 0.0, ms_tfft = 0.0;
    int rk_launches = 0;
    const int nchunks = (n_rec + R - 1) / R;
    // event pairs: [0] wave, [1..nchunks] RK launches, then projections, then time FFT
    const size_t nev = 2 * (size_t)(2 + 2 * nchunks);
    while (ctx->tev.size() < nev) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e), "event");
        ctx->tev.push_back(e);
    }
    auto ev = [&](size_t k) { return ctx->tev[k]; };
    auto elapsed = [&](size_t a, size_t b) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev(a), ev(b));
        return (double)ms;
    };

    for (int w = 0; w < g.waves; w++) {
        const int s_begin = w * W;
        const int Ww = std::min(W, job->n_samples - s_begin);
        CK(cudaEventRecord(ev(0), ctx->s_rk), "event");
        CK(launch_aos_to_soa(d_spins0 + (size_t)s_begin * N * 3, ctx->state.as<double>(), Ww, N,
                             ctx->s_rk), "aos_to_soa");
        ctx->launches++;
        CK(cudaMemcpyAsync(ctx->s0.p, ctx->state.p, (size_t)Ww * 3 * N * sizeof(double),
                           cudaMemcpyDeviceToDevice, ctx->s_rk), "D2D");
        if (job->imp) {
            std::vector<uint8_t> ib((size_t)Ww * N);
            for (size_t e = 0; e < ib.size(); e++) ib[e] = job->imp[(size_t)s_begin * N + e] ? 1 : 0;
            CK(cudaMemcpyAsync(ctx->imp.p, ib.data(), ib.size(), cudaMemcpyHostToDevice, ctx->s_rk),
               "H2D imp");
            CK(cudaStreamSynchronize(ctx->s_rk), "sync");
        }
        // the proj stream must not overwrite series of the previous wave
        // before its time transform finished: both run on s_proj in order.
        for (int c = 0; c < nchunks; c++) {
            const int b = c % kSnapBufs;
            const int rb = c * R, re = std::min(n_rec, rb + R);
            if (c >= kSnapBufs) CK(cudaStreamWaitEvent(ctx->s_rk, ctx->ev_proj[b], 0), "wait");
            RKJob J{};
            J.n_samples = Ww;
            J.dt = job->dt;
            J.stride = job->stride;
            J.rec_begin = rb;
            J.rec_end = re;
            J.n_rec = n_rec;
            J.fix_every = job->fix_every < 1 ? 1 : job->fix_every;
            J.state = ctx->state.as<double>();
            J.s0 = ctx->s0.as<double>();
            J.e0 = ctx->e0.as<double>();
            J.imp = job->imp ? ctx->imp.as<uint8_t>() : nullptr;
            J.snap = ctx->snap[b].p;
            J.snap_R = R;
            J.qss = ctx->qss.as<double>();
            J.stats = ctx->stats.as<double>();
            J.status = ctx->status.as<int>();
            J.qpart = g.ctab ? ctx->qpart.as<double>() : nullptr;
            // the cluster kernel writes the tensor-core operand rows itself
            const bool tc_list = Qs.n_list > 0 && g.prec == SMD_FP32;
            const bool fused_split = tc_list && g.ctab;
            if (tc_list) {
                const int rows = Ww * R * 3, kp = Qs.kp;
                const size_t ab = (size_t)W * R * 3 * kp * 2;
                for (DevBuf *d : {&ctx->ahi[b], &ctx->alo[b]}) {
                    const void *old = d->p;
                    CK(d->ensure(ab), "cudaMalloc");
                    if (d->p != old)   // fresh rows: the padding columns past N stay zero
                        CK(cudaMemsetAsync(d->p, 0, d->bytes, ctx->s_rk), "memset");
                }
                if (ctx->map_a_base[b] != ctx->ahi[b].p || ctx->map_a_rows[b] != rows ||
                    ctx->map_a_kp[b] != kp) {
                    if (!make_bf16_map(&ctx->map_ahi[b], ctx->ahi[b].p, rows, kp, tc_bm()) ||
                        !make_bf16_map(&ctx->map_alo[b], ctx->alo[b].p, rows, kp, tc_bm()))
                        return fail(ctx, SMD_ECUDA, "tensor map encoding failed");
                    ctx->map_a_base[b] = ctx->ahi[b].p;
                    ctx->map_a_rows[b] = rows;
                    ctx->map_a_kp[b] = kp;
                }
            }
            J.bf_hi = fused_split ? ctx->ahi[b].p : nullptr;
            J.bf_lo = fused_split ? ctx->alo[b].p : nullptr;
            J.bf_kp = Qs.kp;
            CK(cudaEventRecord(ev(2 + 2 * c), ctx->s_rk), "event");
            if (g.ctab) {
                // SMD_RK_HALO=barrier publishes halos with cluster barriers
                ClusterParams cp = g.ctab->P;
                if (const char *e = std::getenv("SMD_RK_HALO"))
                    if (!std::strcmp(e, "barrier")) cp.async_halo = 0;
                CK(launch_rk_cluster(cp, J, g.prec, g.spt, g.threads, ctx->s_rk), "rk cluster kernel");
            }
            else
                CK(launch_rk(L.dev, J, g.prec, gen, ctx->s_rk), "rk kernel");
            CK(cudaEventRecord(ev(3 + 2 * c), ctx->s_rk), "event");
            ctx->launches++;
            rk_launches++;
            CK(cudaEventRecord(ctx->ev_rk[b], ctx->s_rk), "event");
            CK(cudaStreamWaitEvent(ctx->s_proj, ctx->ev_rk[b], 0), "wait");
            CK(cudaEventRecord(ev(2 + 2 * nchunks + 2 * c), ctx->s_proj), "event");
            ProjArgs pa{};
            pa.L = &L;
            pa.Qs = &Qs;
            pa.prec = g.prec;
            pa.N = N;
            pa.W = Ww;
            pa.R = R;
            pa.rb = rb;
            pa.re = re;
            pa.n_rec = n_rec;
            pa.nqb = nqb;
            pa.snap = ctx->snap[b].p;
            pa.ahi = ctx->ahi[b].p;
            pa.alo = ctx->alo[b].p;
            pa.map_ahi = &ctx->map_ahi[b];
            pa.map_alo = &ctx->map_alo[b];
            pa.fused_split = fused_split;
            pa.win = d_win;
            pa.series = ctx->series.p;
            pa.gscratch = &ctx->gscratch;
            pa.status = ctx->status.as<int>();
            {
                int rc = project_chunk(ctx, pa, ctx->s_proj, &ctx->launches);
                if (rc) return rc;
            }
            CK(cudaEventRecord(ev(3 + 2 * nchunks + 2 * c), ctx->s_proj), "event");
            CK(cudaEventRecord(ctx->ev_proj[b], ctx->s_proj), "event");
        }
        CK(cudaEventRecord(ev(nev - 2), ctx->s_proj), "event");
        const void *tw = g.prec == SMD_FP64 ? g.tp->tw64.p : g.tp->tw32.p;
        if (h_spec && w == g.waves - 1) {
            // last wave with a host destination: one transform per spin
            // component, each scaled by fc and copied to the host on the RK
            // stream (idle by now) while the next component transforms
            const size_t comp_series = (size_t)nqb * n_rec * 16, comp_acc = (size_t)Q * n_rec;
            for (int c = 0; c < 3; c++) {
                CK(launch_time_fft(static_cast<const char *>(ctx->series.p) + c * comp_series, g.prec, Ww, Q,
                                   nqb, g.tp->p, tw, d_spec_sum + c * comp_acc, ctx->status.as<int>(),
                                   ctx->s_proj, 1),
                   "time fft");
                CK(launch_scale(d_spec_sum + c * comp_acc, comp_acc, fc, ctx->s_proj), "scale");
                CK(cudaEventRecord(ctx->ev_tf[c], ctx->s_proj), "event");
                ctx->launches += 2;
            }
            CK(cudaEventRecord(ev(nev - 1), ctx->s_proj), "event");
            for (int c = 0; c < 3; c++) {
                CK(cudaStreamWaitEvent(ctx->s_rk, ctx->ev_tf[c], 0), "wait");
                CK(cudaMemcpyAsync(h_spec + c * comp_acc, d_spec_sum + c * comp_acc, comp_acc * sizeof(double),
                                   cudaMemcpyDeviceToHost, ctx->s_rk),
                   "D2H spec");
            }
        } else {
            CK(launch_time_fft(ctx->series.p, g.prec, Ww, Q, nqb, g.tp->p, tw, d_spec_sum,
                               ctx->status.as<int>(), ctx->s_proj),
               "time fft");
            CK(cudaEventRecord(ev(nev - 1), ctx->s_proj), "event");
            ctx->launches++;
        }
        CK(cudaStreamWaitEvent(ctx->s_proj, ctx->ev_rk[(nchunks - 1) % kSnapBufs], 0), "wait");
        if (g.ctab) {
            CK(launch_qss_from_parts(ctx->qpart.as<double>(), Ww, n_rec, g.ctab->P.CS, N, ctx->qss.as<double>(),
                                     ctx->s_proj),
               "qss");
            ctx->launches++;
        }
        CK(launch_sum_rows(ctx->qss.as<double>(), Ww, n_rec, d_qss_sum, ctx->s_proj), "qss");
        ctx->launches++;
        if (d_final) {
            CK(launch_soa_to_aos(ctx->state.as<double>(), d_final + (size_t)s_begin * N * 3, Ww, N,
                                 ctx->s_proj), "soa_to_aos");
            ctx->launches++;
        }
        CK(cudaEventRecord(ev(1), ctx->s_proj), "event");
        stats_h.resize((size_t)Ww * 4);
        CK(cudaMemcpyAsync(stats_h.data(), ctx->stats.p, stats_h.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, ctx->s_proj), "D2H stats");
        // before the next wave overwrites state / series / qss
        CK(cudaStreamSynchronize(ctx->s_proj), "sync");
        CK(cudaStreamSynchronize(ctx->s_rk), "sync");
        ms_dev += elapsed(0, 1);
        for (int c = 0; c < nchunks; c++) {
            ms_rk += elapsed(2 + 2 * c, 3 + 2 * c);
            ms_proj += elapsed(2 + 2 * nchunks + 2 * c, 3 + 2 * nchunks + 2 * c);
        }
        ms_tfft += elapsed(nev - 2, nev - 1);
        for (int s = 0; s < Ww; s++) {
            drift_max = std::max(drift_max, stats_h[s * 4 + 0] / N);
            drift_final = std::max(drift_final, std::fabs(stats_h[s * 4 + 1] - stats_h[s * 4 + 2]) / N);
        }
    }
    int st = 0;
    CK(cudaMemcpy(&st, ctx->status.p, sizeof(int), cudaMemcpyDeviceToHost), "D2H status");
    if (rep) {
        rep->drift_max = drift_max;
        rep->drift_final = drift_final;
        rep->waves = g.waves;
        rep->ms_device = ms_dev;
        rep->ms_rk = ms_rk;
        rep->ms_proj = ms_proj;
        rep->ms_tfft = ms_tfft;
        rep->rk_launches = rk_launches;
        rep->rk_kind = g.ctab ? 1 : 0;
        rep->rk_ctas = g.ctab ? g.ctab->P.CS : 1;
        rep->site_steps = (double)N * (double)(n_rec - 1) * job->stride * job->n_samples;
    }
    if (st & 4) return fail(ctx, SMD_ETIMEOUT, "tensor-core projection: a bounded wait expired");
    if (st & 8) return fail(ctx, SMD_ETIMEOUT, "time transform: a bounded wait expired");
    if (st & 16) return fail(ctx, SMD_ETIMEOUT, "RK halo exchange: a bounded wait expired");
    if (st) return fail(ctx, SMD_ECUDA, "a sample reached a zero correction denominator (sigma = 0)");
    return SMD_OK;
}

}  // namespace

extern "C" int smd_run_device(smd_ctx *ctx, const smd_job_desc *job, const double *d_spins0,
                              const double *d_window, double *d_spec_sum, double *d_qss_sum,
                              double *d_final, smd_report *rep)
{
    if (!ctx || !job || !d_spins0 || !d_window || !d_spec_sum || !d_qss_sum) return SMD_EINVAL;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    JobGeom g;
    int rc = prepare(ctx, job, g);
    if (rc) return rc;
    ctx->launches = 0;
    auto w0 = std::chrono::steady_clock::now();
    rc = run_device(ctx, job, g, d_spins0, d_window, d_spec_sum, d_qss_sum, d_final, rep);
    auto w1 = std::chrono::steady_clock::now();
    if (rep) {
        rep->ms_total = std::chrono::duration<double, std::milli>(w1 - w0).count();
        rep->ms_h2d = rep->ms_d2h = 0.0;
        rep->kernel_launches = ctx->launches;
    }
    return rc;
}

extern "C" int smd_run(smd_ctx *ctx, const smd_job_desc *job, const double *spins0,
                       const double *window, double *spec_out, double *qss_out, double *final_out,
                       smd_report *rep)
{
    if (!ctx || !job || !spins0 || !window || !spec_out || !qss_out) return SMD_EINVAL;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    JobGeom g;
    int rc = prepare(ctx, job, g);
    if (rc) return rc;
    ctx->launches = 0;
    const size_t S = job->n_samples, N = g.N, Q = g.Q, n = g.n_rec;
    const size_t in_b = S * N * 3 * sizeof(double);
    const size_t acc_b = 3 * Q * n * sizeof(double);
    const size_t out_b = (final_out ? in_b : 0);
    CK(ctx->in_tmp.ensure(in_b + n * sizeof(double)), "cudaMalloc");
    CK(ctx->acc_tmp.ensure(acc_b + n * sizeof(double)), "cudaMalloc");
    if (out_b) CK(ctx->out_tmp.ensure(out_b), "cudaMalloc");
    double *d_in = ctx->in_tmp.as<double>();
    double *d_win = d_in + S * N * 3;
    double *d_acc = ctx->acc_tmp.as<double>();
    double *d_q = d_acc + 3 * Q * n;
    auto w0 = std::chrono::steady_clock::now();
    CK(cudaMemcpyAsync(d_in, spins0, in_b, cudaMemcpyHostToDevice, ctx->s_rk), "H2D spins");
    CK(cudaMemcpyAsync(d_win, window, n * sizeof(double), cudaMemcpyHostToDevice, ctx->s_rk), "H2D window");
    CK(cudaMemsetAsync(d_acc, 0, acc_b + n * sizeof(double), ctx->s_rk), "memset");
    CK(cudaStreamSynchronize(ctx->s_rk), "sync");
    auto w1 = std::chrono::steady_clock::now();
    // averages over samples on the device, as the reference's fc = 1 / evoCnt
    // (smd_code.cpp:3596-3611); the last wave scales each component's
    // spectrum and copies it to spec_out while the next one transforms
    const double fc = 1.0 / (double)S;
    rc = run_device(ctx, job, g, d_in, d_win, d_acc, d_q, out_b ? ctx->out_tmp.as<double>() : nullptr,
                    rep, spec_out, fc);
    if (rc) return rc;
    auto w2 = std::chrono::steady_clock::now();
    CK(launch_scale(d_q, n, fc, ctx->s_rk), "scale");
    CK(cudaMemcpyAsync(qss_out, d_q, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->s_rk), "D2H qss");
    if (out_b)
        CK(cudaMemcpyAsync(final_out, ctx->out_tmp.p, out_b, cudaMemcpyDeviceToHost, ctx->s_rk), "D2H final");
    CK(cudaStreamSynchronize(ctx->s_rk), "sync");
    auto w3 = std::chrono::steady_clock::now();
    if (rep) {
        rep->ms_h2d = std::chrono::duration<double, std::milli>(w1 - w0).count();
        rep->ms_d2h = std::chrono::duration<double, std::milli>(w3 - w2).count();
        rep->ms_total = std::chrono::duration<double, std::milli>(w3 - w0).count();
        rep->kernel_launches = ctx->launches;
    }
    return SMD_OK;
}

extern "C" int smd_dyn_spectrum_ref(smd_ctx *ctx, int lattice_id, int qset_id, double dtm, int ntm,
                                    const double *tWinVec, double *spinField, const int *imp,
                                    double *SqxWVec, double *SqyWVec, double *SqzWVec,
                                    double *qSStVec)
{
    if (!ctx || !tWinVec || !spinField || !SqxWVec || !SqyWVec || !SqzWVec || !qSStVec)
        return SMD_EINVAL;
    smd_job_desc job{};
    job.lattice = lattice_id;
    job.qset = qset_id;
    job.n_samples = 1;
    job.dt = dtm;
    job.n_rec = ntm;
    job.stride = 1;
    job.precision = SMD_FP64;
    job.fix_every = 1;
    job.imp = imp;
    int Q = 0;
    int rc = smd_qset_size(ctx, qset_id, &Q);
    if (rc) return rc;
    std::vector<double> spec((size_t)3 * Q * ntm), fin;
    int N = 0;
    rc = smd_lattice_sites(ctx, lattice_id, &N);
    if (rc) return rc;
    fin.resize((size_t)N * 3);
    rc = smd_run(ctx, &job, spinField, tWinVec, spec.data(), qSStVec, fin.data(), nullptr);
    if (rc) return rc;
    const size_t blk = (size_t)Q * ntm;
    std::memcpy(SqxWVec, spec.data(), blk * sizeof(double));
    std::memcpy(SqyWVec, spec.data() + blk, blk * sizeof(double));
    std::memcpy(SqzWVec, spec.data() + 2 * blk, blk * sizeof(double));
    std::memcpy(spinField, fin.data(), fin.size() * sizeof(double));
    return SMD_OK;
}

extern "C" int smd_evolve(smd_ctx *ctx, int lattice_id, int precision, int n_samples, double dt,
                          int nsteps, int fix_every, const int *imp, double *spins, smd_report *rep)
{
    if (!ctx || !spins || nsteps < 1) return SMD_EINVAL;
    std::shared_ptr<Lattice> Lp;
    {
        std::lock_guard<std::mutex> lk(ctx->maps_mu);
        auto li = ctx->lattices.find(lattice_id);
        if (li == ctx->lattices.end()) return fail(ctx, SMD_ENOTFOUND, "evolve: unknown lattice");
        Lp = li->second;
    }
    // a q set of one list point keeps the pipeline shape; two records
    // (start and end) with stride nsteps give the final state
    int qid = -1;
    double q0[2] = {0.0, 0.0};
    Lattice &L = *Lp;
    std::vector<double> fake_pos;
    if (L.pos.empty()) L.pos.assign(2 * (size_t)L.N, 0.0);
    int rc = smd_qset_upload(ctx, lattice_id, 0, 1, q0, 1.0, &qid);
    if (rc) return rc;
    smd_job_desc job{};
    job.lattice = lattice_id;
    job.qset = qid;
    job.n_samples = n_samples;
    job.dt = dt;
    job.n_rec = 2;
    job.stride = nsteps;
    job.precision = precision;
    job.fix_every = fix_every;
    job.imp = imp;
    std::vector<double> spec(3 * 2), qss(2), win(2, 1.0);
    if (precision == SMD_FP32) {
        // the FP32 form has no list projection yet; use the grid if present
        {
            std::lock_guard<std::mutex> lk(ctx->maps_mu);
            ctx->qsets.erase(qid);
        }
        rc = smd_qset_upload(ctx, lattice_id, 1, 0, nullptr, 1.0, &qid);
        if (rc) return rc;
        int Q = 0;
        smd_qset_size(ctx, qid, &Q);
        spec.assign((size_t)3 * Q * 2, 0.0);
        job.qset = qid;
    }
    rc = smd_run(ctx, &job, spins, win.data(), spec.data(), qss.data(), spins, rep);
    {
        std::lock_guard<std::mutex> lk(ctx->maps_mu);
        ctx->qsets.erase(qid);
    }
    return rc;
}

// ------------------------------------------------------------- serving

// Internal (not exported): serving lanes run jobs on contexts of their own
// (streams and working buffers), sharing the parent's lattice and q set.
int smd_share_objects(smd_ctx *from, smd_ctx *to, int lattice_id, int qset_id)
{
    std::shared_ptr<Lattice> L;
    std::shared_ptr<QSet> Q;
    {
        std::lock_guard<std::mutex> lk(from->maps_mu);
        auto li = from->lattices.find(lattice_id);
        auto qi = from->qsets.find(qset_id);
        if (li == from->lattices.end() || qi == from->qsets.end()) return SMD_ENOTFOUND;
        L = li->second;
        Q = qi->second;
    }
    std::lock_guard<std::mutex> lk(to->maps_mu);
    to->lattices[lattice_id] = L;
    to->qsets[qset_id] = Q;
    return SMD_OK;
}

int smd_ctx_device(const smd_ctx *ctx) { return ctx->device; }

// a lane's failure, reported through the parent's smd_last_error
void smd_copy_error(smd_ctx *to, const smd_ctx *from, long long job_id)
{
    std::lock_guard<std::mutex> lk(to->maps_mu);
    to->err = "job " + std::to_string(job_id) + ": " + from->err;
}
size_t smd_ctx_budget(const smd_ctx *ctx) { return ctx->budget; }
// (smd_submit and the rest: serve.cpp)

extern "C" int smd_lattice_sites(smd_ctx *ctx, int lattice_id, int *N)
{
    if (!ctx || !N) return SMD_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->maps_mu);
    auto it = ctx->lattices.find(lattice_id);
    if (it == ctx->lattices.end()) return SMD_ENOTFOUND;
    *N = it->second->N;
    return SMD_OK;
}
