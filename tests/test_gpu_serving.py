"""Serving with continuous batching (smd_submit / smd_poll / smd_wait /
smd_cancel) on the GPU: jobs of different lattices, sizes and lengths share
persistent RK launches; each job's result equals the job run alone (through
the engine, bit for bit; through smd_run, within the form's tolerance), and
the failure paths (unknown objects, admission by HBM budget, cancellation)
report per job while the other jobs complete."""
import numpy as np
import pytest

from classical_mc_and_smd_for_2d_heisenberg_models_b200 import _lib, smd
from classical_mc_and_smd_for_2d_heisenberg_models_b200 import samples as smp
from classical_mc_and_smd_for_2d_heisenberg_models_b200.settings import SMDSettings

pytestmark = pytest.mark.gpu


def _jobs(ctx):
    """Six jobs: five geometries (Lieb without the d-wave term), uneven N,
    different sample counts, XXZ-free J1-J2-J3 with a field."""
    out = []
    for k, (geom, L, J2, n) in enumerate([("square", 16, 0.6, 4), ("triang", 12, 0.12, 3),
                                          ("kagome", 6, 0.3, 5), ("hexagn", 6, 0.2, 2),
                                          ("square", 24, 0.55, 6), ("lieb", 6, 0.4, 3)]):
        s = SMDSettings(geom=geom, L=L, J2=J2, JX=0.05, h=0.1, dtm=0.01, ntm=32, window="hann1")
        lat = smd.build_lattice(geom, L)
        lid = ctx.lattice(s, lat)
        qid = ctx.qset(lid)
        kind = "stripe" if geom == "square" else ("q120" if geom == "triang" else "ferro")
        spins, _ = smp.make_samples(s, n, kind, 0.3, 40 + k)
        out.append((s, lid, qid, spins, smd.window("hann1", 32)))
    return out


def _kw(precision):
    return dict(precision=precision, fix_every=16 if precision == _lib.SMD_FP32 else 1)


@pytest.mark.parametrize("precision", [_lib.SMD_FP64, _lib.SMD_FP32], ids=["fp64", "fp32"])
def test_served_jobs_equal_jobs_run_alone(precision):
    """Every job submitted at once (they share launches) gives the result of
    the same job served alone, bit for bit, and of smd_run of the job within
    1e-10 (FP64) / 1e-6 rel-L2 (FP32, rounding of the energy sums)."""
    kw = _kw(precision)
    with smd.Context(0) as ctx:
        jobs = _jobs(ctx)
        ids = [ctx.submit(lid, qid, sp, s.dtm, 32, stride=2, win=w, **kw) for s, lid, qid, sp, w in jobs]
        mixed = [ctx.wait(j) for j in ids]
        for (s, lid, qid, sp, w), (spec, qss, lat_ms) in zip(jobs, mixed):
            alone = ctx.wait(ctx.submit(lid, qid, sp, s.dtm, 32, stride=2, win=w, **kw))
            assert lat_ms > 0.0
            assert np.array_equal(spec, alone[0]) and np.array_equal(qss, alone[1])
            ref = ctx.run(lid, qid, sp, s.dtm, 32, stride=2, win=w, **kw)
            if precision == _lib.SMD_FP64:
                assert np.max(np.abs(spec - ref.spec)) <= 1e-10 * np.max(np.abs(ref.spec))
                assert np.max(np.abs(qss - ref.qss)) <= 1e-10
            else:
                assert np.linalg.norm(spec - ref.spec) / np.linalg.norm(ref.spec) <= 1e-6


def test_jobs_of_different_lengths_overlap():
    """A long job submitted first and short jobs arriving behind it: the short
    ones finish before the long one (they join its launches instead of
    queueing behind it), and all equal their lone runs."""
    kw = _kw(_lib.SMD_FP32)
    with smd.Context(0) as ctx:
        jobs = _jobs(ctx)
        s, lid, qid, sp, _ = jobs[4]
        long_w = smd.window("hann1", 4096)
        # 262 080 steps: long enough that the short jobs' first kernel loads
        # and admissions cannot outlast it
        long_id = ctx.submit(lid, qid, sp, s.dtm, 4096, stride=64, win=long_w, **kw)
        short = [ctx.submit(l2, q2, sp2, s2.dtm, 32, stride=2, win=w2, **kw)
                 for s2, l2, q2, sp2, w2 in jobs[:4]]
        short_res = [ctx.wait(j) for j in short]
        assert ctx.poll(long_id) == _lib.SMD_EBUSY
        long_res = ctx.wait(long_id)
        alone = ctx.wait(ctx.submit(lid, qid, sp, s.dtm, 4096, stride=64, win=long_w, **kw))
        assert np.array_equal(long_res[0], alone[0])
        for (s2, l2, q2, sp2, w2), r in zip(jobs[:4], short_res):
            a2 = ctx.wait(ctx.submit(l2, q2, sp2, s2.dtm, 32, stride=2, win=w2, **kw))
            assert np.array_equal(r[0], a2[0])


def test_unknown_objects_are_refused_at_submit(ctx):
    s, lid, qid, sp, w = _jobs(ctx)[0]
    with pytest.raises(_lib.SMDError):
        ctx.submit(lid + 999, qid, sp, s.dtm, 32, win=w)
    with pytest.raises(_lib.SMDError):
        ctx.submit(lid, qid + 999, sp, s.dtm, 32, win=w)


def test_admission_failure_is_per_job():
    """A job whose single sample exceeds the HBM budget fails with
    SMD_ENOMEM_ADMIT; a small job queued beside it completes."""
    with smd.Context(0, hbm_budget=1 << 30) as c:
        big = SMDSettings(geom="square", L=96, J2=0.5, dtm=0.01, ntm=4096)
        small = SMDSettings(geom="square", L=8, J2=0.5, dtm=0.01, ntm=32)
        ids = []
        for s, n_rec in ((big, 4096), (small, 32)):
            lat = smd.build_lattice(s.geom, s.L)
            lid = c.lattice(s, lat)
            qid = c.qset(lid)
            sp, _ = smp.make_samples(s, 2, "stripe", 0.2, 3)
            ids.append(c.submit(lid, qid, sp, s.dtm, n_rec, win=smd.window("hann1", n_rec)))
        with pytest.raises(_lib.SMDError) as e:
            c.wait(ids[0])
        assert e.value.code == _lib.SMD_ENOMEM_ADMIT
        spec, qss, _ = c.wait(ids[1])
        assert np.isfinite(spec).all() and qss[0] == 1.0


def test_cancelled_job_reports_cancelled(ctx):
    """Jobs queued behind running ones can be cancelled; a cancelled job
    reports SMD_ECANCELLED, the others complete."""
    s = SMDSettings(geom="triang", L=48, J2=0.12, dtm=0.02, ntm=1024)
    lat = smd.build_lattice(s.geom, s.L)
    lid = ctx.lattice(s, lat)
    qid = ctx.qset(lid)
    sp, _ = smp.make_samples(s, 8, "q120", 0.15, 5)
    w = smd.window("hann1", 1024)
    ids = [ctx.submit(lid, qid, sp, s.dtm, 1024, stride=4, win=w, precision=_lib.SMD_FP32,
                      fix_every=16) for _ in range(12)]
    rc = ctx.cancel(ids[-1])
    cancelled = rc == 0
    for j in ids[:-1]:
        spec, qss, _ = ctx.wait(j)
        assert np.isfinite(spec).all()
    if cancelled:
        with pytest.raises(_lib.SMDError) as e:
            ctx.wait(ids[-1])
        assert e.value.code == _lib.SMD_ECANCELLED
    else:
        ctx.wait(ids[-1])
