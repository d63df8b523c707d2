"""Benchmark of the SMD path: SMD site-steps/s on the triangular-lattice
workload (c2: L=48, N=2304, 64 samples per GPU, FP32 precision form, FP64
correction every 16 steps, 48 x 48 grid + 512-point path, 4096 records).

One bench step = one full job over the batch: RK4 integration of every
sample, the per-record projection onto all q, the windowed time transform
and the sample accumulation of |S(q,w)|^2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c1|c2|c3|c4|c5|mc] [--no-cpu-baseline]

Under torchrun every rank integrates its own 64 samples (weak scaling); the
sample sums are added across ranks with one NCCL all-reduce per step, the
multi-GPU form of the reference's end-of-run MPI reduction
(Codes_Folder/smd_code.cpp:3332-3397).  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SMD site-steps/s"
# c4 bench sample count: 64 of the configuration's 512 samples (one wave of
# the 1.7 GB-per-sample series; site-steps/s is per-sample intensive)
C4_SAMPLES = 64
UNIT = "site-steps/s"


def profile_traffic(name: str, records_per_launch: float = 0.0):
    """DRAM bytes (read + write) per launch of a kernel from its committed
    ncu summary in profiles/ (the `dram_bytes_per_launch:` line), or None.
    A summary with a `records_per_launch:` line was captured on launches of
    that many records; its bytes scale to `records_per_launch` (the traffic
    is the per-record snapshot and operand-row writes)."""
    path = os.path.join(ROOT, "profiles", name)
    traffic, rec = None, 0
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch:"):
                traffic = int(line.split(":")[1])
            elif line.startswith("records_per_launch:"):
                rec = int(line.split(":")[1])
    except OSError:
        return None, None
    if traffic is None:
        return None, None
    src = f"profiles/{name}"
    if rec and records_per_launch and records_per_launch != rec:
        traffic = int(round(traffic * records_per_launch / rec))
        src += f" (captured at {rec} records per launch, scaled to {records_per_launch:g})"
    return traffic, src


def z_active(w, lat) -> int:
    """Active neighbours per site of a workload's lattice."""
    s = w.settings
    return sum(lat.zn[k] for k, on in enumerate([True, s.j2_on, s.jx_on]) if on)


DATA = {"q120": "seeded 120-degree states with Gaussian tilts",
        "stripe": "seeded stripe states with Gaussian tilts",
        "ferro": "seeded ferromagnetic states with Gaussian tilts",
        "relaxed": "seeded random states relaxed by 200 local-field alignment steps, "
                   "then Gaussian tilts"}


def rel_l2(a, b):
    """Relative L2 error ||a - b|| / ||b|| of two spectra."""
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / nb if nb > 0 else None


def flops_per_site_step(z: int) -> int:
    """Algorithmic flops of one site-step of RK4 + energy correction: 6 field
    sweeps x 6z, 4 stages x 18, combine and normalise 24, correction 53,
    energy sums 6z (Codes_Folder/subrouts.cpp:11734-11902)."""
    return 42 * z + 150


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------- serving

def serving_leg(device: int, n_jobs: int, seed: int, fp64: bool = True):
    """A stream of serving-workload jobs (workloads.c5_stream: five
    geometries, N log-uniform in [256, 16384], 16-256 samples, 2^12-2^15 RK
    steps, 1024 records, FP32 form) through the continuous-batching engine
    (smd_submit / smd_wait).  One burst (every job queued at once) gives the
    aggregate service rate (median of five bursts); Poisson arrivals at 70 % of it give p50 / p99
    latency (submit to completion, as the library measures it).  The same
    jobs run one at a time through smd_run in the FP64 plain form give the
    FP64 spectra each served result's DSSF rel-L2 is taken against and one
    denominator of the 4x target (FP64 device time, no serving overhead); the
    same jobs served as one FP64 burst through the engine give the like-for-
    like denominator.  Each phase runs in a context of its own, so the
    buffers one phase grew do not hold device memory the next needs."""
    from classical_mc_and_smd_for_2d_heisenberg_models_b200 import _lib, smd, workloads
    jobs = workloads.c5_stream(n_jobs, seed)
    site_steps = sum(w.settings.N * w.n_samples * w.steps for w in jobs)

    def prepare(ctx):
        out = []
        for w in jobs:
            s = w.settings
            lat = smd.build_lattice(s.geom, s.L)
            lid = ctx.lattice(s, lat)
            qid = ctx.qset(lid)
            spins, imp = workloads.make_inputs(w)
            imp_arr = None if imp is None else np.ascontiguousarray(imp, np.int32)
            out.append((w, lid, qid, spins, imp_arr, smd.window(w.window, w.n_rec)))
        return out

    def fp64_solo(ctx, p, spins=None):
        w, lid, qid, sp, imp_arr, win = p
        return ctx.run(lid, qid, sp if spins is None else spins, w.settings.dtm, w.n_rec,
                       stride=w.stride, precision=_lib.SMD_FP64, fix_every=1, win=win, imp=imp_arr,
                       want_final=False)

    # the FP64 plain form one job at a time through smd_run: device time and spectra
    ms64, spec64 = 0.0, []
    if fp64:
        with smd.Context(device) as c64:
            for p in prepare(c64):
                r = fp64_solo(c64, p)
                ms64 += r.report["ms_device"]
                spec64.append(r.spec)

    out = {}
    with smd.Context(device) as ctx:
        prepared = prepare(ctx)

        def submit(p, fp64_plain=False):
            w, lid, qid, spins, imp_arr, win = p
            prec, fix = (_lib.SMD_FP64, 1) if fp64_plain else (w.precision, w.fix_every)
            return ctx.submit(lid, qid, spins, w.settings.dtm, w.n_rec, stride=w.stride,
                              precision=prec, fix_every=fix, win=win, imp=imp_arr)

        # warm-up burst (untimed): the engine's memory pool, lattice tables,
        # time plans and pinned staging are set up on first use
        for j in [submit(p) for p in prepared]:
            ctx.wait(j)
        # bursts: every job queued at once; the median makespan of five
        # gives the service rate (one burst's makespan moves by up to 30 %
        # from burst to burst, the first after the warm-up most)
        spans = []
        for _ in range(5):
            t0 = time.perf_counter()
            ids = [submit(p) for p in prepared]
            burst = [ctx.wait(j) for j in ids]
            spans.append(time.perf_counter() - t0)
            infos = [ctx.job_info(j) for j in ids]
        makespan = float(np.median(spans))
        rate = 0.7 * len(prepared) / makespan
        rng = np.random.default_rng(seed + 1)
        gaps = rng.exponential(1.0 / rate, size=len(prepared))
        t0 = time.perf_counter()
        ids, t_next = [], 0.0
        for p, g in zip(prepared, gaps):
            t_next += g
            dt = t0 + t_next - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            ids.append(submit(p))
        lat = np.array([ctx.wait(j)[2] for j in ids])
        wall = time.perf_counter() - t0
        out = {"jobs": len(prepared), "arrivals": "Poisson", "rate_jobs_per_s": rate,
               "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
               "max_ms": float(lat.max()), "site_steps": float(site_steps),
               "burst_makespan_s": makespan, "burst_makespans_s": spans,
               "served_site_steps_per_s": site_steps / makespan,
               "energy_drift_per_site": {"max": max(i["drift_max"] for i in infos),
                                         "final": max(i["drift_final"] for i in infos)},
               "sample": f"{len(prepared)} jobs of the serving mix (5 geometries, N log-uniform in "
                         f"[256, 16384], 16-256 samples, 2^12-2^15 RK steps at the stride giving "
                         f"1024 records, 0-10 % vacancies, grid q, FP32 form), Poisson at 70 % of "
                         f"the burst service rate; stream wall time {wall:.1f} s",
               "job_shapes": [f"{w.settings.geom} N={w.settings.N} S={w.n_samples} "
                              f"steps={w.steps}" for w, *_ in prepared]}
    if fp64:
        # the FP64 plain form served the same way (one burst through the
        # engine, in a context of its own): the like-for-like denominator of
        # the served form, in both admission orders (largest job first, the
        # default, and arrival order), the faster one kept
        rates = {}
        old = os.environ.get("SMD_SERVE_ORDER")
        for order in ("work", "fifo"):
            os.environ["SMD_SERVE_ORDER"] = order
            with smd.Context(device) as c64s:
                prep64 = prepare(c64s)
                # untimed warm-up: each job on its first sample at stride 1
                # (kernels, lattice tables, time plans and pinned staging)
                for j in [c64s.submit(lid, qid, sp[:1], w.settings.dtm, w.n_rec, stride=1,
                                      precision=_lib.SMD_FP64, fix_every=1, win=win,
                                      imp=None if imp_arr is None else imp_arr[:1])
                          for w, lid, qid, sp, imp_arr, win in prep64]:
                    c64s.wait(j)
                t0 = time.perf_counter()
                ids64 = [c64s.submit(lid, qid, sp, w.settings.dtm, w.n_rec, stride=w.stride,
                                     precision=_lib.SMD_FP64, fix_every=1, win=win, imp=imp_arr)
                         for w, lid, qid, sp, imp_arr, win in prep64]
                for j in ids64:
                    c64s.wait(j)
                rates[order] = site_steps / (time.perf_counter() - t0)
        if old is None:
            os.environ.pop("SMD_SERVE_ORDER", None)
        else:
            os.environ["SMD_SERVE_ORDER"] = old
        out["fp64_plain_served_site_steps_per_s"] = max(rates.values())
        out["fp64_plain_served_by_order"] = rates
        out["speedup_vs_fp64_plain_served"] = (out["served_site_steps_per_s"] /
                                               out["fp64_plain_served_site_steps_per_s"])
    if fp64:
        rels = [rel_l2(spec, s64) for (spec, _, _), s64 in zip(burst, spec64)]
        floors = [None] * len(rels)
        if max(rels) > 1e-3:
            # chaotic jobs: the FP64 form's own difference under one FP32
            # rounding of its inputs
            with smd.Context(device) as cf:
                for k, p in enumerate(prepare(cf)):
                    if rels[k] > 1e-3:
                        pert = workloads.tangent_perturb(p[3], workloads.FP32_ROUNDOFF, 11)
                        floors[k] = rel_l2(fp64_solo(cf, p, pert).spec, spec64[k])
        out["fp64_plain_site_steps_per_s"] = site_steps / (ms64 / 1e3)
        out["speedup_vs_fp64_plain"] = out["served_site_steps_per_s"] / out["fp64_plain_site_steps_per_s"]
        out["dssf_rel_l2_vs_fp64"] = {
            "max": float(max(rels)), "median": float(np.median(rels)),
            "per_job": [float(x) for x in rels],
            "chaos_floor_per_job": floors,
            "note": "chaos_floor: rel-L2 of the FP64 form from inputs moved by one FP32 rounding "
                    "(2^-24) against the unperturbed FP64 run, taken for jobs above 1e-3"}
    return out


# --------------------------------------------------------- CPU reference

def reference_runner_step(w, procs: int, ntm: int, workdir: str):
    """The reference's own SMD code (oracle/_ref/smd_ref_run, built from
    Codes_Folder/subrouts.cpp) on `procs` host cores: one single-rank process
    per core, each integrating one sample of the workload's lattice for
    ntm - 1 steps (every step recorded, as the reference does), like the
    reference's MPI sample decomposition (Codes_Folder/smd_code.cpp:3130-3180).
    Returns (site_steps, max_ms)."""
    runner = os.path.join(ROOT, "oracle", "_ref", "smd_ref_run")
    jobs = []
    for p in range(procs):
        args = [runner, workdir, os.path.join(workdir, "samples.bin"), str(p), "1",
                "--no-dwf-guard"]
        jobs.append(subprocess.Popen(args, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                     text=True))
    ms = []
    for j in jobs:
        out, err = j.communicate()
        if j.returncode != 0:
            raise RuntimeError(f"reference runner failed: {err.strip()[-300:]}")
        ms.append(json.loads(out.strip().splitlines()[-1])["rk_loop_ms"])
    N = w.settings.N
    return procs * N * (ntm - 1), max(ms)


def prepare_reference(w, procs: int, ntm: int):
    from classical_mc_and_smd_for_2d_heisenberg_models_b200 import samples as smp
    import dataclasses
    s = dataclasses.replace(w.settings, ntm=ntm, window=w.window,
                            NMeas=1000 * max(2, procs), crSkip=1000, imp_ratio=0.0)
    wd = tempfile.mkdtemp(prefix="smd_ref_")
    s.write(wd)
    if w.state == "relaxed":
        from classical_mc_and_smd_for_2d_heisenberg_models_b200 import smd, workloads
        lat = smd.build_lattice(s.geom, s.L)
        spins, _ = workloads.relaxed_samples(s, lat, procs, 200, w.sigma, w.seed)
    else:
        spins, _ = smp.make_samples(s, procs, w.state, w.sigma, w.seed)
    smp.write_sample_file(os.path.join(wd, "samples.bin"), s, spins, None)
    return wd


def reference_available() -> bool:
    return os.access(os.path.join(ROOT, "oracle", "_ref", "smd_ref_run"), os.X_OK)


def ref_procs() -> int:
    return max(1, min(os.cpu_count() or 1, 64))


# ------------------------------------------------------------------ ours

def run_ours(args, w, rank, world):
    import torch
    from classical_mc_and_smd_for_2d_heisenberg_models_b200 import _lib, smd, workloads
    import ctypes as C

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    s = w.settings
    lat = smd.build_lattice(s.geom, s.L)
    spins, imp = workloads.make_inputs(w, rank)
    win = smd.window(w.window, w.n_rec)
    ql = workloads.path_points(s.geom, w.qpath_points) if w.qpath_points else None
    ctx = smd.Context(local)
    lid = ctx.lattice(s, lat)
    qid = ctx.qset(lid, use_grid=True, qlist=ql)
    Q = ctx.qset_size(qid)
    S, N, n = w.n_samples, s.N, w.n_rec
    lib = ctx.lib

    # device-resident inputs and accumulators
    d_spins = torch.from_numpy(spins).to(f"cuda:{local}")
    d_win = torch.from_numpy(win).to(f"cuda:{local}")
    d_spec = torch.zeros((3, Q, n), dtype=torch.float64, device=f"cuda:{local}")
    d_qss = torch.zeros(n, dtype=torch.float64, device=f"cuda:{local}")
    imp_arr = None if imp is None else np.ascontiguousarray(imp, np.int32)

    def device_step(precision, fix_every):
        d_spec.zero_()
        d_qss.zero_()
        torch.cuda.synchronize()
        j = ctx.job(lid, qid, S, s.dtm, n, w.stride, precision, fix_every, imp_arr)
        rep = _lib.Report()
        rc = lib.smd_run_device(ctx.h, C.byref(j), C.c_void_p(d_spins.data_ptr()),
                                C.c_void_p(d_win.data_ptr()), C.c_void_p(d_spec.data_ptr()),
                                C.c_void_p(d_qss.data_ptr()), None, C.byref(rep))
        if rc:
            raise _lib.SMDError(rc, lib.smd_last_error(ctx.h).decode())
        if dist is not None:
            dist.all_reduce(d_spec)
            dist.all_reduce(d_qss)
        torch.cuda.synchronize()
        return rep

    # ---- precision form, device-resident (value)
    for _ in range(args.warmup):
        device_step(w.precision, w.fix_every)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    reps = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            reps.append(device_step(w.precision, w.fix_every))
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ms_dev = sum(r.ms_device for r in reps)
    ms_rk = sum(r.ms_rk for r in reps)
    rk_launches = sum(r.rk_launches for r in reps)
    rk_kind = {0: "rk_fp32_kernel" if w.precision == _lib.SMD_FP32 else "rk_fp64_kernel",
               1: "rk_cluster_kernel"}[reps[-1].rk_kind]
    launches = sum(r.kernel_launches for r in reps)
    drift_max = max(r.drift_max for r in reps)
    drift_final = max(r.drift_final for r in reps)
    t = torch.tensor([ms_dev], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    site_steps_rank = float(S) * N * w.steps
    total_site_steps = site_steps_rank * world * args.steps
    value = total_site_steps / (ms_max / 1e3)
    samples_per_s = (S * world * args.steps) / (ms_max / 1e3)

    # ---- e2e through the C ABI with pinned host buffers (smd_run)
    pin_in = torch.from_numpy(spins).pin_memory()
    pin_win = torch.from_numpy(win).pin_memory()
    pin_spec = torch.zeros((3, Q, n), dtype=torch.float64).pin_memory()
    pin_qss = torch.zeros(n, dtype=torch.float64).pin_memory()
    dp = lambda tns: C.cast(C.c_void_p(tns.data_ptr()), C.POINTER(C.c_double))

    def e2e_step():
        j = ctx.job(lid, qid, S, s.dtm, n, w.stride, w.precision, w.fix_every, imp_arr)
        rep = _lib.Report()
        t0 = time.perf_counter()
        rc = lib.smd_run(ctx.h, C.byref(j), dp(pin_in), dp(pin_win), dp(pin_spec), dp(pin_qss),
                         None, C.byref(rep))
        t1 = time.perf_counter()
        if rc:
            raise _lib.SMDError(rc, lib.smd_last_error(ctx.h).decode())
        return t1 - t0

    # K steps, each from the host buffers to the host result; the mean step
    # time (one step's wall time moves by tens of ms with the host's load:
    # the 277 MB spectrum crosses PCIe every step)
    e2e_steps = max(1, args.steps)
    e2e_step()
    e2e_t = [e2e_step() for _ in range(e2e_steps)]
    tt = torch.tensor([sum(e2e_t) / len(e2e_t)], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    e2e_value = site_steps_rank * world / float(tt.item())
    # the precision form's spectrum of this workload (sample sums), kept for
    # its DSSF error against the FP64 form below
    spec32 = d_spec.double().cpu().numpy().copy()

    # ---- serving: bounded job stream with p50 / p99 latency (rank 0's queue)
    h2d = spins.nbytes + win.nbytes
    d2h = 3 * Q * n * 8 + n * 8

    # ---- FP64 plain form on the same workload (the 4x target's denominator)
    fp64 = None
    dssf = None
    z = z_active(w, lat)
    fpss = flops_per_site_step(z)
    peak64 = C.c_double()
    ok64 = lib.smd_measure_fma_peak(local, _lib.SMD_FP64, C.byref(peak64)) == 0
    if not args.no_fp64 and w.precision != _lib.SMD_FP64:
        device_step(_lib.SMD_FP64, 1)
        r64 = [device_step(_lib.SMD_FP64, 1) for _ in range(max(1, min(args.steps, 2)))]
        ms64 = sum(r.ms_device for r in r64)
        t64 = torch.tensor([ms64], dtype=torch.float64, device=f"cuda:{local}")
        if dist is not None:
            dist.all_reduce(t64, op=dist.ReduceOp.MAX)
        fp64_value = site_steps_rank * world * len(r64) / (float(t64.item()) / 1e3)
        spec64 = d_spec.double().cpu().numpy().copy()
        # chaos floor: the FP64 form from inputs moved by one FP32 rounding
        d_spins.copy_(torch.from_numpy(
            workloads.tangent_perturb(spins, workloads.FP32_ROUNDOFF, 11)).to(d_spins.device))
        device_step(_lib.SMD_FP64, 1)
        spec64p = d_spec.double().cpu().numpy()
        d_spins.copy_(torch.from_numpy(spins).to(d_spins.device))
        G2 = Q - (0 if ql is None else len(ql))   # grid q first, then the path

        def parts(a, b):
            return {"grid": rel_l2(a[:, :G2, :], b[:, :G2, :]),
                    "path": rel_l2(a[:, G2:, :], b[:, G2:, :]) if ql is not None else None,
                    "all": rel_l2(a, b)}

        dssf = parts(spec32, spec64)
        dssf["chaos_floor"] = parts(spec64p, spec64)
        dssf["reference"] = ("FP64 plain form (correction every step) on the same samples; that "
                             "form equals the reference per spin to 1e-10 over 200 steps")
        dssf["chaos_floor_note"] = (
            "rel-L2 of the FP64 form run from the same samples moved by one FP32 rounding "
            "(2^-24 tangent perturbation) against the unperturbed FP64 run: the trajectories "
            "are chaotic over this length, so this is the least DSSF difference any FP32 "
            "arithmetic can reach on this run")
        fp64 = {"value": fp64_value, "unit": UNIT,
                "ms_per_step": float(t64.item()) / len(r64),
                "ms_rk_per_step": sum(r.ms_rk for r in r64) / len(r64),
                "ms_proj_per_step": sum(r.ms_proj for r in r64) / len(r64),
                "ms_tfft_per_step": sum(r.ms_tfft for r in r64) / len(r64),
                "drift_max_per_site": max(r.drift_max for r in r64)}
        ach64 = fpss * site_steps_rank * len(r64) / (sum(r.ms_rk for r in r64) / 1e3) / 1e12
        fp64["rk_roofline"] = {"kernel": "rk_cluster_kernel<double>", "bound": "fp64",
                               "achieved": ach64, "unit": "TFLOP/s",
                               "peak": peak64.value if ok64 else None,
                               "frac": ach64 / peak64.value if ok64 and peak64.value > 0 else None,
                               "peak_source": "smd_measure_fma_peak (FP64 FMA chains on every SM)"}

    # ---- roofline of the dominant kernel (RK4 + correction)
    peak = C.c_double()
    prec_peak = lib.smd_measure_fma_peak(local, w.precision, C.byref(peak))
    rk_flops = fpss * site_steps_rank * args.steps
    achieved = rk_flops / (ms_rk / 1e3) / 1e12
    waves = max(1, reps[-1].waves)
    traffic, traffic_src = profile_traffic(f"{rk_kind}_{w.name}.md",
                                           w.n_rec * waves * args.steps / max(1, rk_launches))
    roof = {"kernel": rk_kind,
            "bound": "fp32" if w.precision == _lib.SMD_FP32 else "fp64",
            "achieved": achieved, "peak": peak.value if prec_peak == 0 else None,
            "unit": "TFLOP/s",
            "frac": (achieved / peak.value) if prec_peak == 0 and peak.value > 0 else None,
            "peak_source": "smd_measure_fma_peak (FMA chains on every SM)",
            "algorithmic_flops_per_site_step": fpss,
            "avg_launch_ms": ms_rk / max(1, rk_launches),
            "traffic": traffic, "traffic_unit": "bytes per launch (DRAM read + write)",
            "traffic_source": traffic_src}

    if dist is not None:
        dist.destroy_process_group()
    ctx.close()

    # ---- serving: the C5-shaped job stream (rank 0), in contexts of its own
    serving = None
    if rank == 0 and not args.no_serving:
        serving = serving_leg(local, args.serving_jobs, 0x5eed05)

    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 stages / f64 master+energy" if w.precision == _lib.SMD_FP32 else "f64",
            "data": f"synthetic ({DATA.get(w.state, w.state)}, sigma {w.sigma} rad)",
            "config": {"workload": w.describe(), "samples_per_gpu": S,
                       "rk_steps": w.steps, "records": n, "Q": Q,
                       "l2": "inputs larger than L2 (time series %.1f GB per GPU)" %
                             (S * 3 * n * Q * (8 if w.precision == _lib.SMD_FP32 else 16) / 1e9)
                             if S * 3 * n * Q * 8 > 126e6 else
                             "inputs smaller than L2 (126 MB): a latency-bound small case",
                       "parallelism": f"samples sharded over {world} GPU(s)"},
            "dssf_samples_per_s": samples_per_s,
            "breakdown_ms_per_step": {"device": ms_dev / args.steps, "rk": ms_rk / args.steps,
                                      "proj": sum(r.ms_proj for r in reps) / args.steps,
                                      "tfft": sum(r.ms_tfft for r in reps) / args.steps},
            "energy_drift_per_site": {"max": drift_max, "final": drift_final},
            "dssf_rel_l2": dssf,
            "fp64_plain": fp64,
            "speedup_vs_fp64_plain": (value / fp64["value"]) if fp64 else None,
            "serving": serving,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": float(tt.item()) * 1e3},
            "roofline": roof,
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
    return line


def run_batch(args, bw, rank, world):
    """The batched form (smd_batch_*): every member lattice's samples in one
    persistent RK launch per chunk of records, the job step replayed as one
    CUDA graph.  One bench step = one job step of the whole batch."""
    import torch
    from classical_mc_and_smd_for_2d_heisenberg_models_b200 import _lib, smd, workloads
    import ctypes as C

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ctx = smd.Context(local)
    lib = ctx.lib
    mem = []
    for k, w in enumerate(bw.members):
        s = w.settings
        lat = smd.build_lattice(s.geom, s.L)
        lid = ctx.lattice(s, lat)
        ql = workloads.bz_points(lat, bw.n_q, w.seed + 1)
        qid = ctx.qset(lid, use_grid=False, qlist=ql)
        spins, imp = workloads.make_inputs(w, rank, lat=lat)
        mem.append((w, lat, lid, qid, spins, imp, ctx.qset_size(qid)))
    m0 = bw.members[0]
    n = m0.n_rec
    win = smd.window(m0.window, n)
    b = ctx.batch([(lid, qid, w.n_samples, imp) for (w, lat, lid, qid, spins, imp, Q) in mem],
                  m0.settings.dtm, n, m0.stride, m0.precision, m0.fix_every)
    tuning = b.info()
    d_in = [torch.from_numpy(x[4]).to(dev) for x in mem]
    d_win = torch.from_numpy(win).to(dev)
    d_spec = [torch.zeros((3, x[6], n), dtype=torch.float64, device=dev) for x in mem]
    d_qss = [torch.zeros(n, dtype=torch.float64, device=dev) for x in mem]
    k = len(mem)
    VP = C.c_void_p
    ins = (VP * k)(*[t.data_ptr() for t in d_in])
    so = (VP * k)(*[t.data_ptr() for t in d_spec])
    qo = (VP * k)(*[t.data_ptr() for t in d_qss])

    def step():
        rep = _lib.Report()
        rc = lib.smd_batch_run_device(ctx.h, b.id, ins, VP(d_win.data_ptr()), so, qo, C.byref(rep))
        if rc:
            raise _lib.SMDError(rc, lib.smd_last_error(ctx.h).decode())
        return rep

    first = step()   # eager, with per-launch timing of the batch RK kernel
    for _ in range(max(0, args.warmup - 1)):
        step()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    reps = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            reps.append(step())
        torch.cuda.synchronize()
    ms_dev = sum(r.ms_device for r in reps)
    t = torch.tensor([ms_dev], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    site_steps_rank = sum(float(w.settings.N) * w.n_samples * w.steps for w, *_ in mem)
    value = site_steps_rank * world * args.steps / (ms_max / 1e3)
    n_samples = sum(w.n_samples for w, *_ in mem)
    spec32 = [x.cpu().numpy().copy() for x in d_spec]

    # e2e: host buffers through smd_batch_run
    pins = [torch.from_numpy(x[4]).pin_memory() for x in mem]
    pwin = torch.from_numpy(win).pin_memory()
    pspec = [torch.zeros((3, x[6], n), dtype=torch.float64).pin_memory() for x in mem]
    pqss = [torch.zeros(n, dtype=torch.float64).pin_memory() for x in mem]
    P = C.POINTER(C.c_double)
    cp = lambda tt: C.cast(C.c_void_p(tt.data_ptr()), P)
    hin = (P * k)(*[cp(x) for x in pins])
    hso = (P * k)(*[cp(x) for x in pspec])
    hqo = (P * k)(*[cp(x) for x in pqss])

    def e2e():
        rep = _lib.Report()
        t0 = time.perf_counter()
        rc = lib.smd_batch_run(ctx.h, b.id, hin, cp(pwin), hso, hqo, C.byref(rep))
        t1 = time.perf_counter()
        if rc:
            raise _lib.SMDError(rc, lib.smd_last_error(ctx.h).decode())
        return t1 - t0

    e2e()
    e2e_k = max(1, args.steps)
    e2e_t = sum(e2e() for _ in range(e2e_k)) / e2e_k   # mean step time over K steps
    e2e_value = site_steps_rank * world / e2e_t

    # FP64 plain form: every member alone through smd_run_device, FP64,
    # correction every step (no batching): the denominator of the 4x target
    fp64, dssf = None, None
    if not args.no_fp64:
        ms64, rels, rk64, ff64 = 0.0, [], 0.0, 0.0
        for mi, ((w, lat, lid, qid, spins, imp, Q), dsp, s32) in enumerate(zip(mem, d_spec, spec32)):
            dsp.zero_()
            dq = torch.zeros(n, dtype=torch.float64, device=dev)
            imp_arr = None if imp is None else np.ascontiguousarray(imp, np.int32)
            j = ctx.job(lid, qid, w.n_samples, w.settings.dtm, n, w.stride, _lib.SMD_FP64, 1, imp_arr)
            rep = _lib.Report()
            torch.cuda.synchronize()
            rc = lib.smd_run_device(ctx.h, C.byref(j), VP(d_in[mi].data_ptr()),
                                    VP(d_win.data_ptr()), VP(dsp.data_ptr()), VP(dq.data_ptr()), None,
                                    C.byref(rep))
            if rc:
                raise _lib.SMDError(rc, lib.smd_last_error(ctx.h).decode())
            ms64 += rep.ms_device
            rk64 += rep.ms_rk
            ff64 += flops_per_site_step(z_active(w, lat)) * float(w.settings.N) * w.n_samples * w.steps
            rels.append(rel_l2(s32, dsp.cpu().numpy()))
        fp64 = {"value": site_steps_rank / (ms64 / 1e3), "unit": UNIT, "ms_per_step": ms64,
                "ms_rk_per_step": rk64, "rk_achieved_tflops": ff64 / (rk64 / 1e3) / 1e12,
                "form": "each lattice alone through smd_run, FP64, correction every step"}
        dssf = {"max": float(max(rels)), "per_member": [float(x) for x in rels],
                "reference": "FP64 plain form of each lattice on the same samples"}

    # roofline of the batch RK kernel (eager first run: CUDA events around
    # every launch on the RK stream)
    flops = sum(flops_per_site_step(z_active(w, lat)) * float(w.settings.N) * w.n_samples * w.steps
                for (w, lat, *_rest) in mem)
    achieved = flops / (first.ms_rk / 1e3) / 1e12
    peak = C.c_double()
    okp = lib.smd_measure_fma_peak(local, m0.precision, C.byref(peak)) == 0
    traffic, traffic_src = profile_traffic("rk_batch_kernel_c3.md")
    roof = {"kernel": "rk_batch_kernel", "bound": "fp32" if m0.precision == _lib.SMD_FP32 else "fp64",
            "achieved": achieved, "peak": peak.value if okp else None, "unit": "TFLOP/s",
            "frac": achieved / peak.value if okp and peak.value > 0 else None,
            "peak_source": "smd_measure_fma_peak (FMA chains on every SM)",
            "algorithmic_flops_per_site_step": "42 z + 150 per member",
            "avg_launch_ms": first.ms_rk / max(1, first.rk_launches),
            "traffic": traffic, "traffic_unit": "bytes per launch (DRAM read + write)",
            "traffic_source": traffic_src}
    b.free()
    if dist is not None:
        dist.destroy_process_group()
    ctx.close()
    if rank != 0:
        return None
    h2d = sum(x[4].nbytes for x in mem) + win.nbytes
    d2h = sum(3 * x[6] * n * 8 + n * 8 for x in mem)
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 stages / f64 master+energy",
        "data": f"synthetic ({DATA['relaxed']}, sigma {m0.sigma} rad)",
        "config": {"workload": bw.describe(), "samples_per_gpu": n_samples, "rk_steps": m0.steps,
                   "records": n, "q_per_lattice": bw.n_q,
                   "l2": "inputs larger than L2 (time series %.1f GB per GPU)" %
                         (sum(w.n_samples * 3 * n * Q * 8 for (w, *_r, Q) in mem) / 1e9),
                   "parallelism": f"samples sharded over {world} GPU(s)",
                   "graph": "one CUDA graph launch per job step (the first, eager run is warm-up)"},
        "dssf_samples_per_s": n_samples * world * args.steps / (ms_max / 1e3),
        "autotuner": tuning,
        "energy_drift_per_site": {"max": max(r.drift_max for r in reps),
                                  "final": max(r.drift_final for r in reps)},
        "dssf_rel_l2": dssf, "fp64_plain": fp64,
        "speedup_vs_fp64_plain": value / fp64["value"] if fp64 else None,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_t * 1e3},
        "roofline": roof, "gpu_launches": sum(r.kernel_launches for r in reps),
        "clocks": clk.summary(),
    }


def run_mc(args, rank, world):
    """The Monte Carlo stage that produces the sample file (smd_mc_run):
    square L = 64 (N = 4096), J1 = 1, J2 = 0.3, 32 temperatures in
    [0.2, 1.0] x 4 chains = 128 replicas with parallel tempering, 200
    thermalization + 800 measurement MC steps of 5 overrelaxation + 5
    heat-bath sweeps, a record every 100 steps.  One bench step = one such
    run; the metric is site updates per second (replicas x N x sweeps x
    steps).  Replicas are independent across ranks (weak scaling)."""
    import torch
    from classical_mc_and_smd_for_2d_heisenberg_models_b200 import _lib, smd
    from classical_mc_and_smd_for_2d_heisenberg_models_b200.settings import SMDSettings
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    s = SMDSettings(geom="square", L=64, J1=1.0, J2=0.3)
    temps = np.linspace(0.2, 1.0, 32)
    chains, therm, meas, skip = 4, 200, 800, 100
    ctx = smd.Context(local)
    lat = smd.build_lattice(s.geom, s.L)
    lid = ctx.lattice(s, lat)
    run = lambda seed: ctx.mc_run(lid, temps, therm, meas, cr_skip=skip, chains=chains, pt=True,
                                  seed=seed + 7919 * rank)
    for k in range(args.warmup):
        run(k + 1)
    reps, walls = [], []
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            t0 = time.perf_counter()
            out = run(100 + k)
            walls.append(time.perf_counter() - t0)
            reps.append(out["report"])
    ms_dev = sum(r["ms_device"] for r in reps)
    updates = sum(r["site_steps"] for r in reps)
    t = torch.tensor([ms_dev], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.destroy_process_group()
    value = updates * world / (float(t.item()) / 1e3)
    e_site = out["energy"][:, :, therm:].mean(axis=(0, 2)) / lat.N
    peak64 = fp64_fma_peak(ctx, local)
    # one site update: the field (6 z flops) and the move (reflection 16,
    # heat bath about 60 incl. the rotation), averaged over the 5 + 5 sweeps
    fpu = 6 * 8 + 38
    ach = fpu * updates / (ms_dev / 1e3) / 1e12
    ctx.close()
    R = len(temps) * chains
    return {
        "metric": "MC site-updates/s", "value": value, "unit": "site-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_dev / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "seeded random start (IState high_T)",
        "config": {"workload": f"mc: square L=64 N=4096, J2=0.3, {len(temps)} temperatures in "
                               f"[0.2, 1.0] x {chains} chains = {R} replicas, parallel tempering, "
                               f"{therm} + {meas} MC steps of 5 + 5 sweeps, a record every {skip}",
                   "l2": "replica spins in shared memory (98 KB each)"},
        "energy_per_site_by_T": [float(x) for x in e_site],
        "pt_acceptance": float(out["pt_counts"][:, :, 1].sum() / max(1, out["pt_counts"][:, :, 0].sum())),
        "e2e": {"value": updates * world / sum(walls), "unit": "site-updates/s",
                "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(out["samples"].nbytes + out["energy"].nbytes)},
        "roofline": {"kernel": "mc_step_kernel", "bound": "fp64", "achieved": ach, "unit": "TFLOP/s",
                     "peak": peak64, "frac": ach / peak64 if peak64 else None,
                     "peak_source": "smd_measure_fma_peak (FP64 FMA chains on every SM)",
                     "algorithmic_flops_per_site_update": fpu},
        "gpu_launches": int(sum(r["kernel_launches"] for r in reps)),
        "clocks": clk.summary(),
    }


def fp64_fma_peak(ctx, device):
    """Measured FP64 FMA peak of the device (TFLOP/s), or None."""
    import ctypes as C
    from classical_mc_and_smd_for_2d_heisenberg_models_b200 import _lib
    v = C.c_double()
    return v.value if ctx.lib.smd_measure_fma_peak(device, _lib.SMD_FP64, C.byref(v)) == 0 else None


def mc_cpu_baseline(args):
    """The reference's own MC sweeps (smd_ref_run --mc) on the same lattice
    at one temperature, one single-rank process per host core, 100 MC steps
    each."""
    if not reference_available():
        return {"value": None, "unavailable": "oracle/_ref/smd_ref_run not built"}
    from classical_mc_and_smd_for_2d_heisenberg_models_b200.settings import SMDSettings
    procs = ref_procs()
    s = SMDSettings(geom="square", L=64, J1=1.0, J2=0.3, T1=0.5, T2=0.5, ntm=16)
    wd = tempfile.mkdtemp(prefix="smd_mc_ref_")
    s.write(wd)
    runner = os.path.join(ROOT, "oracle", "_ref", "smd_ref_run")
    jobs = [subprocess.Popen([runner, wd, "none", str(p + 1), "0", "--no-dwf-guard", "--mc", "0",
                              "100"], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
            for p in range(procs)]
    ms = []
    for j in jobs:
        out, err = j.communicate()
        if j.returncode != 0:
            raise RuntimeError(f"reference MC failed: {err.strip()[-300:]}")
        ms.append(json.loads(out.strip().splitlines()[-1])["mc_ms"])
    updates = procs * s.N * 100 * 10
    return {"value": updates / (max(ms) / 1e3), "unit": "site-updates/s", "cores": procs,
            "kind": "reference",
            "sample": f"{procs} processes x 100 MC steps (5 + 5 sweeps) of square L=64 at T=0.5"}


def cpu_baseline(w, args):
    """Bounded sample of the reference's own CPU code, all host cores."""
    if not reference_available():
        return {"value": None, "unavailable": "oracle/_ref/smd_ref_run not built"}
    procs = ref_procs()
    ntm = args.ref_ntm
    wd = prepare_reference(w, procs, ntm)
    site_steps, ms = reference_runner_step(w, procs, ntm, wd)
    return {"value": site_steps / (ms / 1e3), "unit": UNIT, "cores": procs, "kind": "reference",
            "sample": f"{procs} processes x 1 sample x {ntm - 1} RK steps of {w.name} "
                      f"(N={w.settings.N}), every step recorded; reference code, "
                      f"non-MKL DFT (MKL not available on this box)"}


def run_reference_arm(args, w, rank, world):
    if rank != 0:
        return None
    if not reference_available():
        return {"impl": "reference", "unavailable": "reference runner not built on this box"}
    procs = ref_procs()
    ntm = args.ref_ntm
    wd = prepare_reference(w, procs, ntm)
    for _ in range(args.warmup):
        reference_runner_step(w, procs, ntm, wd)
    tot, tmax = 0.0, 0.0
    for _ in range(args.steps):
        ss, ms = reference_runner_step(w, procs, ntm, wd)
        tot += ss
        tmax += ms
    value = tot / (tmax / 1e3)
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tmax / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded 120-degree states with 0.15 rad Gaussian tilts)",
        "config": {"workload": w.describe(), "samples_per_step": procs, "rk_steps": ntm - 1},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
                         "sample": f"{procs} processes x 1 sample x {ntm - 1} RK steps per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5", "mc"])
    ap.add_argument("--ref-ntm", type=int, default=1025)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serving-jobs", type=int, default=12)
    ap.add_argument("--records", type=int, default=0,
                    help="override the record count (small profiling cases only)")
    ap.add_argument("--samples", type=int, default=0,
                    help="override the samples per GPU (small profiling cases only)")
    ap.add_argument("--lattice", default="",
                    help="GEOM:L, override the lattice (profiling a lattice shape only; "
                         "ordered state ferro except triangular 120-degree and square stripe)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    from classical_mc_and_smd_for_2d_heisenberg_models_b200 import workloads
    import dataclasses
    if args.workload == "c5":
        # the served form alone: the C5-shaped job stream through the engine
        line = None
        if rank == 0:
            import torch
            local = int(os.environ.get("LOCAL_RANK", "0"))
            torch.cuda.set_device(local)
            if args.impl == "reference":
                line = {"impl": "reference", "unavailable": "the serving stream has no counterpart "
                        "in the reference (one job per process); its CPU code is timed by the "
                        "c1-c4 workloads"}
            else:
                with ClockSampler(local) as clk:
                    sv = serving_leg(local, args.serving_jobs, 0x5eed05, fp64=not args.no_fp64)
                line = {"metric": METRIC + " (served)", "value": sv["served_site_steps_per_s"],
                        "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": 1,
                        "ms_per_step": sv["burst_makespan_s"] * 1e3, "higher_is_better": True,
                        "scaling": "weak", "vs_baseline": None,
                        "dtype": "f32 stages / f64 master+energy", "data": "synthetic (C5 job mix)",
                        "config": {"workload": "c5: " + sv["sample"]},
                        "serving": sv, "clocks": clk.summary()}
        if line is not None:
            print(json.dumps(line))
        return
    if args.workload == "mc":
        if args.impl == "reference":
            line = mc_cpu_baseline(args) if rank == 0 else None
            if line is not None:
                line = dict(line, impl="reference", metric="MC site-updates/s",
                            e2e={"value": line["value"], "unit": "site-updates/s",
                                 "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        else:
            line = run_mc(args, rank, world)
            if rank == 0 and world == 1 and not args.no_cpu_baseline:
                line["cpu_baseline"] = mc_cpu_baseline(args)
        if rank == 0 and line is not None:
            print(json.dumps(line))
        return
    if args.workload == "c3":
        bw = workloads.c3(args.samples or 256)
        # the reference arm and the CPU baseline run the batch's largest lattice
        w = max(bw.members, key=lambda m: m.settings.N)
    else:
        bw = None
        w = workloads.WORKLOADS[args.workload]()
        if args.workload == "c4" and not args.samples:
            w = dataclasses.replace(w, n_samples=C4_SAMPLES)
        if args.records:
            w = dataclasses.replace(w, n_rec=args.records)
        if args.samples:
            w = dataclasses.replace(w, n_samples=args.samples)
        if args.lattice:
            geom, L = args.lattice.split(":")
            w = dataclasses.replace(w, settings=dataclasses.replace(w.settings, geom=geom, L=int(L)),
                                    state={"triang": "q120", "square": "stripe"}.get(geom, "ferro"))
    if args.impl == "reference":
        line = run_reference_arm(args, w, rank, world)
    else:
        line = run_batch(args, bw, rank, world) if bw is not None else run_ours(args, w, rank, world)
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(w, args)
    if rank == 0 and line is not None:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
