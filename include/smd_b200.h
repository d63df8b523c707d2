/*
 * smd_b200.h -- C ABI of the B200 semiclassical spin-dynamics (SMD) library.
 *
 * The library replaces the reference's SMD hot path, the per-sample function
 *
 *   void get_dynSpectrum(int procNum, double *tWinVec, double **spinField,
 *                        double **SqxWVec, double **SqyWVec,
 *                        double **SqzWVec, double *qSStVec)
 *   (Codes_Folder/subrouts.cpp:11547-12149)
 *
 * together with the sample loop and accumulation of its caller
 * (Codes_Folder/smd_code.cpp:3079-3291, 3596-3611), with hand-written sm_100a
 * kernels.  Everything the reference reads from process globals (lattice
 * tables, couplings, lambda vectors, field, ntm, dtm, the DFT grid map; see
 * Codes_Folder/subrouts.cpp:65-775) is passed explicitly.
 *
 * Conventions
 *   - plain C types only; host memory belongs to the caller, device memory to
 *     the context;
 *   - every entry point returns an smd_status; smd_last_error() describes the
 *     last failure of a context;
 *   - one context per host thread; a context is not re-entrant;
 *   - spins are [site][3] doubles in the reference's site order, exactly as
 *     the reference's spinField rows and sample files hold them;
 *   - spectra are [3][Q][n_rec] doubles (component, q, frequency bin), the
 *     reference's SqxWVec/SqyWVec/SqzWVec rows stacked by component; grid q
 *     come first in the reference's k = i * Gsz + j order
 *     (Codes_Folder/subrouts.cpp:8421-8431), then the list q.
 */
#ifndef SMD_B200_H
#define SMD_B200_H

#include <stddef.h>

#if defined(__GNUC__)
#define SMD_API __attribute__((visibility("default")))
#else
#define SMD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SMD_OK = 0,
    SMD_EINVAL = 1,        /* invalid argument or unsupported size */
    SMD_ENOMEM_ADMIT = 2,  /* job does not fit the context's HBM budget */
    SMD_ECUDA = 3,         /* CUDA runtime or kernel error */
    SMD_ETIMEOUT = 4,      /* a bounded wait expired */
    SMD_ECANCELLED = 5,    /* job cancelled before completion */
    SMD_ENOTFOUND = 6,     /* unknown lattice, q-set or job id */
    SMD_EBUSY = 7          /* job not finished yet (smd_poll) */
} smd_status;

typedef enum {
    SMD_FP64 = 0,          /* plain form: every step in FP64, correction each step */
    SMD_FP32 = 1           /* precision form: FP32 RK4 stages, FP64 master spins,
                              renormalisation and energy correction */
} smd_precision;

typedef enum {
    SMD_SQUARE = 0, SMD_TRIANG = 1, SMD_HEXAGN = 2, SMD_KAGOME = 3, SMD_LIEB = 4
} smd_geometry;

typedef struct smd_ctx smd_ctx;

typedef struct {
    int device;            /* CUDA device ordinal */
    size_t hbm_budget;     /* bytes the context may hold for job state; 0 = 85% of free */
} smd_device_opts;

/* ------------------------------------------------------------ context */

SMD_API int smd_ctx_create(const smd_device_opts *opts, smd_ctx **out);
SMD_API int smd_ctx_destroy(smd_ctx *ctx);
SMD_API const char *smd_last_error(const smd_ctx *ctx);
SMD_API const char *smd_version(void);

/* -------------------------------------------------- host lattice tables */

/* Geometry constants of convert_inputs2data
 * (Codes_Folder/subrouts.cpp:1028-1067, 1141-1154): N = nSubs L^2,
 * G = gridFac L, zn = (Zn1, Zn2, ZnX).  Also applies the reference's size
 * rules (L even; L a multiple of 3 for the C3 lattices). */
SMD_API int smd_geometry_info(int geom, int L, int *N, int *G, int *nsubs, int zn[3]);

/* Site positions, DFT-grid map and neighbour tables in the reference's exact
 * order, replacing make_rvecList (Codes_Folder/subrouts.cpp:2714-2962) and
 * make_nborsTable (Codes_Folder/subrouts.cpp:2983-3316).  Built in O(N) from
 * cell neighbourhoods instead of the reference's O(N^2) search.
 * rvec[N][2], grid_map[G*G], nb1[N][zn0], nb2[N][zn1], nbx[N][zn2]. */
SMD_API int smd_build_lattice(int geom, int L, double *rvec, int *grid_map, int *nb1,
                      int *nb2, int *nbx);

/* Bond list of make_bondList (Codes_Folder/subrouts.cpp:3426-3570).
 * bonds[max_bonds][2]; nbonds = {total, NN, NNN, Xth}. */
SMD_API int smd_build_bonds(int N, const int zn[3], const int *nb1, const int *nb2,
                    const int *nbx, int j2_on, int jx_on, int *bonds,
                    int max_bonds, int nbonds[4]);

/* Temporal windows of Codes_Folder/aux_code.cpp:249-435, selected by the
 * names of Codes_Folder/smd_code.cpp:2825-2894 (nowin gauss ntall black
 * flatw lancz sincw hann1 hann2 hann3). */
SMD_API int smd_window(const char *name, int n, double *out);

/* ------------------------------------------------------ device objects */

/* Model on one lattice: what get_localField (Codes_Folder/subrouts.cpp:
 * 4465-4570) and get_energyValue (Codes_Folder/subrouts.cpp:5181-5302) read
 * from globals. */
typedef struct {
    int N;                 /* Ns */
    int zn[3];             /* Zn1, Zn2, ZnX */
    const int *nbr[3];     /* nbors1/2/X as [N][zn[s]]; entries < 0 are ghosts */
    int shell_on[3];       /* 1, J2_ON, JX_ON */
    double J[3][2][2];     /* J1Mat, J2Mat, JXMat [a_i][a_j] */
    double lambda[3][3];   /* lambdaVec1..3 */
    int lieb_delta_on;     /* J2ab_ON */
    double j2_delta;       /* J2_delta */
    double h;              /* extH along z */
    int nbonds[3];         /* Nb1, Nb2, NbX */
    const int *bonds;      /* bondList as [Nb][2] */
    int G;                 /* Gsz; 0 = no DFT grid */
    const int *grid_map;   /* gridMap [G*G], -1 = empty grid point */
    const double *pos;     /* [N][2] site positions for list-q projection */
} smd_lattice_desc;

SMD_API int smd_lattice_upload(smd_ctx *ctx, const smd_lattice_desc *desc, int *lattice_id);
SMD_API int smd_lattice_free(smd_ctx *ctx, int lattice_id);

/* q set: the lattice's G x G grid (use_grid = 1) followed by n_list
 * arbitrary points q = qlist[l] ([n_list][2]).  List points use the direct
 * sum of get_qct_SqData (Codes_Folder/subrouts.cpp:8460-8525):
 * list_scale * sum_k S_k exp(-i q . pos_k). */
SMD_API int smd_qset_upload(smd_ctx *ctx, int lattice_id, int use_grid, int n_list,
                    const double *qlist, double list_scale, int *qset_id);
SMD_API int smd_qset_size(smd_ctx *ctx, int qset_id, int *Q);
SMD_API int smd_lattice_sites(smd_ctx *ctx, int lattice_id, int *N);

/* ----------------------------------------------------------------- jobs */

typedef struct {
    int lattice;           /* lattice id */
    int qset;              /* q-set id (on the same lattice) */
    int n_samples;         /* samples in spins0 */
    double dt;             /* dtm */
    int n_rec;             /* records = time-FFT length (the reference's ntm) */
    int stride;            /* RK steps between records (reference: 1) */
    int precision;         /* smd_precision */
    int fix_every;         /* energy-correction period in steps (reference: 1) */
    const int *imp;        /* [n_samples][N] impurity flags, or NULL */
} smd_job_desc;

typedef struct {
    double ms_total;       /* wall time of the call on the device stream */
    double ms_h2d, ms_d2h; /* host <-> device copies inside the call */
    double site_steps;     /* N * RK steps * samples */
    double drift_max;      /* max over samples and checked steps of |E - E0| / N */
    double drift_final;    /* max over samples of |E(final) - E0| / N */
    int waves;             /* sample waves the job was split into */
    int kernel_launches;   /* kernels launched by the call */
    double ms_device;      /* device time of the pipeline (CUDA events, all waves) */
    double ms_rk;          /* summed duration of the RK kernel launches */
    double ms_proj;        /* summed duration of the projection launches */
    double ms_tfft;        /* summed duration of the time-transform launches */
    int rk_launches;       /* RK kernel launches */
    int rk_kind;           /* RK kernel used: 0 single-CTA, 1 cluster, 3 batch (smd_batch_run) */
    int rk_ctas;           /* CTAs per sample (cluster size) */
} smd_report;

/* Run a job end to end from host buffers.
 * spins0      [n_samples][N][3] initial spins (host)
 * window      [n_rec] temporal window (host)
 * spec_out    [3][Q][n_rec] sample average of |S(q,w)|^2 (host), the
 *             reference's CMT_Sq*WVec / evoCnt (Codes_Folder/smd_code.cpp:
 *             3596-3611)
 * qss_out     [n_rec] sample average of the spin autocorrelation (host)
 * final_out   [n_samples][N][3] final spins (host) or NULL */
SMD_API int smd_run(smd_ctx *ctx, const smd_job_desc *job, const double *spins0,
            const double *window, double *spec_out, double *qss_out,
            double *final_out, smd_report *rep);

/* Same job with every buffer already in device memory (pointers from
 * cudaMalloc on the context's device).  Outputs are sample SUMS, not
 * averages: spec_sum[3][Q][n_rec] and qss_sum[n_rec] are accumulated into
 * (caller zeroes them), so several calls can share one accumulator. */
SMD_API int smd_run_device(smd_ctx *ctx, const smd_job_desc *job, const double *d_spins0,
                   const double *d_window, double *d_spec_sum, double *d_qss_sum,
                   double *d_final, smd_report *rep);

/* Reference-equivalent single sample: the data of get_dynSpectrum with flat
 * arrays.  One RK step per record (stride 1), correction every step, FP64.
 * spinField [N][3] is updated to the final state; SqxWVec, SqyWVec,
 * SqzWVec are [Q][ntm] each; qSStVec [ntm]. */
SMD_API int smd_dyn_spectrum_ref(smd_ctx *ctx, int lattice_id, int qset_id, double dtm,
                         int ntm, const double *tWinVec, double *spinField,
                         const int *imp, double *SqxWVec, double *SqyWVec,
                         double *SqzWVec, double *qSStVec);

/* Static pre-pass over the MC samples (Codes_Folder/smd_code.cpp:2289-2726),
 * the reference's first read of the sample file before any dynamics:
 *   sf_out     [3][G*G] average over samples of the static structure factor
 *              max(1e-16, |S_c(q)|^2) on the lattice's DFT grid, each
 *              amplitude capped at spec0Max = 10, with the reference's
 *              factor 1 / max(n_samples - 1, 1) (get_StaticSFac,
 *              subrouts.cpp:8799-8825);
 *   hist_out   [201][3] counts of the local-field components over every
 *              site of every sample in 201 bins over +-max_field
 *              (get_HistIndex, subrouts.cpp:795-812);
 *   max_field  (out, may be NULL) maxLocField = sum over active shells of
 *              max|J| times the shell's neighbours (subrouts.cpp:2081-2091).
 * spins0 [n_samples][N][3] and imp [n_samples][N] (or NULL) on the host;
 * qset_id must be a q set with the lattice's grid. */
SMD_API int smd_static_prepass(smd_ctx *ctx, int lattice_id, int qset_id, int n_samples,
                               const double *spins0, const int *imp, double *sf_out,
                               long long *hist_out, double *max_field);

/* RK evolution only (no projection): nsteps steps of the chosen form,
 * spins [n_samples][N][3] updated in place (host). */
SMD_API int smd_evolve(smd_ctx *ctx, int lattice_id, int precision, int n_samples,
               double dt, int nsteps, int fix_every, const int *imp,
               double *spins, smd_report *rep);

/* ------------------------------------------------------------- batches */

/* Batched form: the sample loops of several jobs on different lattices
 * (the reference runs one lattice per xSMD_run, one sample at a time in
 * Codes_Folder/smd_code.cpp:3079-3311) integrated by one persistent RK
 * launch per chunk of records.  Thread-block clusters take (lattice, sample)
 * work items from a device queue, so lattices of uneven N share the SMs;
 * the projections and time transforms follow per lattice, and the whole
 * job step is replayed as one CUDA graph.  Members share dt, n_rec, stride,
 * precision and correction period; each has its own q set and samples.
 * Every member's lattice must suit the cluster kernel (energies from the
 * field identity, no Lieb d-wave term, impurities only as vacancies).
 * A project-written autotuner picks the cluster size, sites per thread and
 * records per launch for the batch's shape on first use (cached per shape
 * in the process; smd_batch_info reports the choice). */
typedef struct {
    int lattice;           /* lattice id */
    int qset;              /* q set on that lattice */
    int n_samples;         /* samples of this member */
    const int *imp;        /* [n_samples][N] impurity flags, or NULL */
} smd_batch_member;

typedef struct {
    int n_members;                    /* 1 .. 24 */
    const smd_batch_member *members;
    double dt;
    int n_rec, stride, precision, fix_every;
} smd_batch_desc;

typedef struct {
    int cluster_ctas;      /* CTAs per thread-block cluster of the RK launch */
    int sites_per_thread;  /* largest own sites per thread */
    int threads;           /* threads per CTA */
    int edge_slots;        /* neighbour slots per site (padded) */
    int records_per_launch;
    int clusters;          /* persistent clusters of the RK launch */
    int items;             /* work items per RK launch */
    int candidates;        /* configurations timed by the autotuner (0: cached) */
    double probe_ms;       /* autotuner time spent */
    int member_ctas[24];   /* CTAs per sample of each member */
} smd_batch_tuning;

/* Plan, tune and allocate a batch (device buffers for every member: HBM
 * footprint beyond the context's budget gives SMD_ENOMEM_ADMIT). */
SMD_API int smd_batch_create(smd_ctx *ctx, const smd_batch_desc *desc, int *batch_id);
SMD_API int smd_batch_info(smd_ctx *ctx, int batch_id, smd_batch_tuning *out);
/* One job step of every member from host buffers: spins0[m] is
 * [n_samples][N][3] (host), window [n_rec]; spec_out[m] [3][Q_m][n_rec] and
 * qss_out[m] [n_rec] receive the member's sample averages (as smd_run). */
SMD_API int smd_batch_run(smd_ctx *ctx, int batch_id, const double *const *spins0,
                          const double *window, double *const *spec_out,
                          double *const *qss_out, smd_report *rep);
/* The same from device buffers; d_spec_sum[m] / d_qss_sum[m] receive the
 * member's sample SUMS (written, not accumulated). */
SMD_API int smd_batch_run_device(smd_ctx *ctx, int batch_id, const double *const *d_spins0,
                                 const double *d_window, double *const *d_spec_sum,
                                 double *const *d_qss_sum, smd_report *rep);
SMD_API int smd_batch_free(smd_ctx *ctx, int batch_id);

/* ------------------------------------------------------------- serving */

/* Serving with continuous batching: a submitted job is copied and queued;
 * one engine thread per context admits queued jobs' samples in arrival
 * order as launch slots (24) and the context's HBM budget free up (a job
 * larger than the budget runs in successive sample groups), and advances
 * every admitted group with one persistent RK launch per precision per tick,
 * each group at its own record position, stride and dt.  Spin states and each
 * job's partial |S(q,w)|^2 sums stay resident in HBM until the job's last
 * group lands.  A job's result does not depend on the jobs it shares launches
 * with.  Jobs the batched kernel does not take (Lieb d-wave term, bond-list
 * energies, impurities with couplings) run through smd_run between ticks.
 * Outputs go to the host buffers given at submit, valid once smd_poll
 * returns SMD_OK; smd_poll / smd_wait report the latency from submit.
 * smd_cancel drops a job that has not started; a started job returns
 * SMD_EBUSY and runs to completion. */
SMD_API int smd_submit(smd_ctx *ctx, const smd_job_desc *job, const double *spins0,
               const double *window, double *spec_out, double *qss_out,
               long long *job_id);
SMD_API int smd_poll(smd_ctx *ctx, long long job_id, double *latency_ms);
SMD_API int smd_wait(smd_ctx *ctx, long long job_id, double timeout_ms, double *latency_ms);
SMD_API int smd_cancel(smd_ctx *ctx, long long job_id);
/* Report of a finished job: latency (ms_total), site_steps, and the energy
 * drift per site over its samples (drift_max, drift_final); rk_kind 3 when
 * it ran in the shared launches.  Returns the job's status (SMD_EBUSY while
 * it runs). */
SMD_API int smd_job_info(smd_ctx *ctx, long long job_id, smd_report *rep);
/* Stop the context's serving worker after the queued jobs (call before
 * smd_ctx_destroy when smd_submit was used). */
SMD_API void smd_serve_shutdown(smd_ctx *ctx);

/* ---------------------------------------------------------- Monte Carlo */

/* The MC stage that produces the SMD sample file (the reference's xMC_run,
 * Codes_Folder/mc_hm_code.cpp; one MPI rank per temperature there).  Per MC
 * step: n_micro overrelaxation sweeps (reflect_aboutVec, subrouts.cpp:
 * 4956-5004), n_canon heat-bath sweeps (get_hBathSample + get_rotZ2VMat,
 * subrouts.cpp:5095-5178), the total energy (get_energyValue), then with
 * pt set a parallel-tempering exchange between neighbouring temperatures
 * (mc_hm_code.cpp:3010-3125: even pairs on even steps, odd on odd, from step
 * 101 of the thermalization stage and at every measurement step, a step
 * after an accepted exchange running n_micro2 / n_canon2 sweeps).  The
 * measurement stage keeps the configuration of every cr_skip-th step, the
 * records MC_Bin_SpinField holds (mc_hm_code.cpp:5167-5176).  Sweeps visit
 * the sites colour class by colour class (a proper colouring of the active
 * shells' bonds), not in the reference's shuffled order, with a counter-
 * based generator: the sampled distribution is the same, the draws are
 * not. */
typedef struct {
    int lattice;            /* lattice id */
    int n_temps;            /* temperatures */
    const double *temps;    /* [n_temps] */
    int chains;             /* independent replicas per temperature */
    int n_therm;            /* NTerm: thermalization steps */
    int n_meas;             /* NMeas: measurement steps */
    int cr_skip;            /* crSkip: a record every cr_skip measurement steps */
    int pt;                 /* ptON */
    int n_micro, n_canon;   /* 5, 5 in the reference (subrouts.cpp:305-307) */
    int n_micro2, n_canon2; /* 2, 8: after an accepted exchange (subrouts.cpp:321-322) */
    unsigned long long seed;
    const int *imp;         /* [chains][n_temps][N] impurity flags, or NULL */
} smd_mc_desc;

/* Run the sampler.  spins0 [chains][n_temps][N][3] (host) start states, or
 * NULL for seeded random unit vectors (IState high_T).  Outputs (host, each
 * may be NULL):
 *   samples    [chains][n_temps][ceil(n_meas / cr_skip)][N][3] records, by
 *              temperature (the replica holding it at that step)
 *   energy     [chains][n_temps][n_therm + n_meas] total energy after every
 *              step, by temperature
 *   pt_counts  [chains][n_temps][2] exchange attempts and acceptances
 * rep->site_steps counts site updates (replicas x N x steps x sweeps). */
SMD_API int smd_mc_run(smd_ctx *ctx, const smd_mc_desc *desc, const double *spins0,
                       double *samples, double *energy, int *pt_counts, smd_report *rep);

/* The sampler's colour classes of a lattice (active shells as uploaded):
 * order [N] sites grouped by class, cstart [*ncol + 1] class offsets; *ncol
 * holds the capacity of cstart - 1 on entry and the class count on return.
 * No counterpart in the reference (its sweeps are sequential). */
SMD_API int smd_mc_colouring(smd_ctx *ctx, int lattice_id, int *order, int *cstart, int *ncol);

/* ------------------------------------------------- allocation-free entry */

/* Bytes of the static device array behind smd_evolve_fp64_noalloc. */
#define SMD_NOALLOC_SCRATCH_BYTES (16u << 20)

/* Model of smd_evolve_fp64_noalloc: a lattice without disorder or d-wave
 * term, whose neighbour table the caller keeps in device memory. */
typedef struct {
    int N;                 /* sites */
    int zn[3];             /* neighbours per shell; 0 switches a shell off */
    const int *d_nbr;      /* DEVICE table [zn0 + zn1 + zn2][N]: row zoff(s) + k holds
                              the k-th neighbour of shell s of every site (the
                              transpose of smd_build_lattice's [N][zn] tables) */
    double J[3];           /* J1, J2, JX */
    double lambda[3][3];   /* lambdaVec1..3 */
    double h;              /* field along z */
} smd_noalloc_model;

/* FP64 RK4 + energy-correction evolution (nsteps steps, correction every
 * step) of n_samples samples that allocates no device memory: no
 * cudaMalloc, cudaFree or allocating library call.  No counterpart in the
 * reference.  It serves callers that own all device memory themselves (a
 * framework's memory pool, or a real-time loop that may not allocate once
 * running) and so cannot let this library call cudaMalloc.
 *   d_spins_in, d_spins_out: DEVICE [n_samples][N][3] (may be the same buffer)
 *   d_status: DEVICE int owned by the caller, or NULL.  It is set to 0 on the
 *           stream and then receives the RK kernel's status bits: nonzero
 *           (bit 1) when a sample met a zero correction denominator, in which
 *           case that sample's spins are not trustworthy.  Read it once the
 *           stream has completed; smd_evolve reports the same condition as
 *           SMD_ECUDA.
 *   stream: cudaStream_t to enqueue on (NULL = default stream); the call
 *           returns once the work is enqueued.
 * Working memory comes from one static device array of
 * SMD_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * exit; a call needs about n_samples * (96 N + 56) bytes of it and returns
 * SMD_ENOMEM_ADMIT when that exceeds the array.  The first call on a device
 * looks up the array's address (cudaGetSymbolAddress) with that device
 * current: make it before any stream capture.  All calls share the array and
 * it keeps the last call's contents, so calls that overlap on the GPU race:
 * serialise them.  The tables must list every neighbour relation once in
 * each direction (true for smd_build_lattice tables with L >= 4). */
SMD_API int smd_evolve_fp64_noalloc(const smd_noalloc_model *m, int n_samples, double dt,
                                    int nsteps, const double *d_spins_in, double *d_spins_out,
                                    int *d_status, void *stream);

/* ---------------------------------------------------------- diagnostics */

/* Measured FMA throughput (TFLOP/s, 2 flops per FMA) of the device in the
 * given precision; the roofline denominator of the RK kernels.  No
 * counterpart in the reference (it has no device code). */
SMD_API int smd_measure_fma_peak(int device, int precision, double *tflops);

#ifdef __cplusplus
}
#endif

#endif
