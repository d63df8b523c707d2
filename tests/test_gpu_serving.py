"""The job queue (smd_submit / smd_poll / smd_wait / smd_cancel) on the GPU:
concurrent lanes give each job the result of running it alone, and the
failure paths (unknown objects, admission by HBM budget, cancellation)
report per job while the other jobs complete."""
import numpy as np
import pytest

from classical_mc_and_smd_for_2d_heisenberg_models_b200 import _lib, smd
from classical_mc_and_smd_for_2d_heisenberg_models_b200 import samples as smp
from classical_mc_and_smd_for_2d_heisenberg_models_b200.settings import SMDSettings

pytestmark = pytest.mark.gpu


def _jobs(ctx):
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


@pytest.mark.parametrize("lanes", [1, 4])
@pytest.mark.parametrize("precision", [_lib.SMD_FP64, _lib.SMD_FP32])
def test_queued_jobs_equal_jobs_run_alone(monkeypatch, precision, lanes):
    """Jobs through the queue (one lane, or four running at once on lane
    contexts that share the lattices) give each job the result of smd_run of
    the job alone."""
    monkeypatch.setenv("SMD_SERVE_LANES", str(lanes))
    with smd.Context(0) as ctx:
        jobs = _jobs(ctx)
        kw = dict(precision=precision, fix_every=16 if precision == _lib.SMD_FP32 else 1)
        ids = [ctx.submit(lid, qid, sp, s.dtm, 32, stride=2, win=w, **kw)
               for s, lid, qid, sp, w in jobs]
        got = [ctx.wait(j) for j in ids]
        for (s, lid, qid, sp, w), (spec, qss, lat_ms) in zip(jobs, got):
            ref = ctx.run(lid, qid, sp, s.dtm, 32, stride=2, win=w, **kw)
            assert lat_ms > 0.0
            assert np.max(np.abs(spec - ref.spec)) <= 1e-12 * np.max(np.abs(ref.spec))
            assert np.max(np.abs(qss - ref.qss)) <= 1e-12


def test_unknown_objects_are_refused_at_submit(ctx):
    s, lid, qid, sp, w = _jobs(ctx)[0]
    with pytest.raises(_lib.SMDError):
        ctx.submit(lid + 999, qid, sp, s.dtm, 32, win=w)
    with pytest.raises(_lib.SMDError):
        ctx.submit(lid, qid + 999, sp, s.dtm, 32, win=w)


def test_admission_failure_is_per_job():
    """A job whose single sample exceeds a lane's share of the HBM budget
    fails with SMD_ENOMEM_ADMIT; a small job queued beside it completes."""
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
