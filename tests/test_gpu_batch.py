"""Batched form (smd_batch_*): several lattices of uneven N in one persistent
RK launch per chunk, the job step replayed as a CUDA graph (B200 only).

Each member's result in the batch must equal the same job run alone through
smd_run, which is pinned to the reference per spin:
  * FP64 plain form: spectra within 1e-10 of max |alone| (the batch kernel
    differs only in the order of its compensated energy sums);
  * FP32 form: rel-L2 within 1e-6 on short runs (same stage arithmetic;
    rounding of the sums can differ).
Replays of the captured graph must reproduce the eager first run bit for
bit.
"""
import numpy as np
import pytest

from classical_mc_and_smd_for_2d_heisenberg_models_b200 import _lib, smd
from classical_mc_and_smd_for_2d_heisenberg_models_b200 import samples as smp
from classical_mc_and_smd_for_2d_heisenberg_models_b200.settings import SMDSettings

pytestmark = pytest.mark.gpu


def _members(ctx, precision, with_list):
    """Square J1-J2 (N=256), triangular XXZ with field (N=144), kagome with
    5 % vacancies (N=108), honeycomb J1-J2 (N=72): four geometries, uneven N."""
    cases = [
        (SMDSettings(geom="square", L=16, J2=0.6, dtm=0.01), "stripe", 5, None),
        (SMDSettings(geom="triang", L=12, J2=0.12, zlamb1=0.9, zlamb2=0.9, h=0.2, dtm=0.02), "q120", 3, None),
        (SMDSettings(geom="kagome", L=6, J2=0.2, imp_ratio=0.05, dtm=0.02, NMeas=4000), "ferro", 4, "imp"),
        (SMDSettings(geom="hexagn", L=6, J2=0.3, dtm=0.02), "ferro", 2, None),
    ]
    out = []
    rng = np.random.default_rng(17)
    for k, (s, state, ns, want_imp) in enumerate(cases):
        lat = smd.build_lattice(s.geom, s.L)
        lid = ctx.lattice(s, lat)
        ql = rng.uniform(-np.pi, np.pi, size=(40, 2)) if with_list and k % 2 == 0 else None
        qid = ctx.qset(lid, use_grid=True, qlist=ql)
        spins, imp = smp.make_samples(s, ns, state, 0.25, 40 + k)
        impr = None
        if want_imp and imp is not None:
            impr = np.stack([imp[j // s.pack_size] for j in range(ns)]).astype(np.int32)
        out.append((s, lid, qid, spins, impr))
    return out


def _alone(ctx, mem, dt, n_rec, stride, precision, fix_every, win):
    s, lid, qid, spins, impr = mem
    return ctx.run(lid, qid, spins, dt, n_rec, stride=stride, precision=precision,
                   fix_every=fix_every, win=win, imp=impr, want_final=False)


@pytest.mark.parametrize("precision", [_lib.SMD_FP64, _lib.SMD_FP32], ids=["fp64", "fp32"])
def test_batch_members_equal_their_standalone_runs(ctx, precision):
    n_rec, stride, dt = 32, 2, 0.01
    fix = 1 if precision == _lib.SMD_FP64 else 16
    mems = _members(ctx, precision, with_list=True)
    win = smd.window("hann1", n_rec)
    b = ctx.batch([(m[1], m[2], len(m[3]), m[4]) for m in mems], dt, n_rec, stride, precision, fix)
    info = b.info()
    assert info["items"] >= 1 and info["clusters"] >= 1
    first = b.run([m[3] for m in mems], win)          # eager run with timing
    again = b.run([m[3] for m in mems], win)          # captured graph
    third = b.run([m[3] for m in mems], win)          # graph replay
    assert first[0].report["rk_kind"] == 3
    for k, m in enumerate(mems):
        ref = _alone(ctx, m, dt, n_rec, stride, precision, fix, win)
        got = first[k]
        if precision == _lib.SMD_FP64:
            assert np.max(np.abs(got.spec - ref.spec)) <= 1e-10 * np.max(np.abs(ref.spec)), k
            assert np.max(np.abs(got.qss - ref.qss)) <= 1e-10, k
        else:
            rel = np.linalg.norm(got.spec - ref.spec) / np.linalg.norm(ref.spec)
            assert rel <= 1e-6, (k, rel)
        assert np.array_equal(again[k].spec, got.spec), k
        assert np.array_equal(third[k].spec, got.spec), k
        assert np.array_equal(third[k].qss, got.qss), k
    assert first[0].report["drift_max"] <= (1e-12 if precision == _lib.SMD_FP64 else 1e-8)
    b.free()


def test_batch_of_one_equals_member_in_a_mix(ctx, monkeypatch):
    """A lattice alone in a batch and the same lattice inside a mixed batch
    (same configuration forced) give bit-identical spectra: a member's work
    does not depend on what it shares the launch with."""
    monkeypatch.setenv("SMD_BATCH_SPT", "2")
    monkeypatch.setenv("SMD_BATCH_CLUSTER", "4")
    mems = _members(ctx, _lib.SMD_FP32, with_list=False)
    n_rec, stride, dt = 32, 2, 0.01
    win = smd.window("hann1", n_rec)
    mix = ctx.batch([(m[1], m[2], len(m[3]), m[4]) for m in mems], dt, n_rec, stride, _lib.SMD_FP32, 16)
    rm = mix.run([m[3] for m in mems], win)
    for k in (0, 2):
        m = mems[k]
        one = ctx.batch([(m[1], m[2], len(m[3]), m[4])], dt, n_rec, stride, _lib.SMD_FP32, 16)
        assert one.info()["member_ctas"][0] == mix.info()["member_ctas"][k]
        r1 = one.run([m[3]], win)
        assert np.array_equal(r1[0].spec, rm[k].spec), k
        one.free()
    mix.free()


def test_batch_rejects_lattices_outside_the_cluster_kernel(ctx):
    s = SMDSettings(geom="lieb", L=4, J2=0.3, J2_delta=0.1, dtm=0.01)
    lat = smd.build_lattice(s.geom, s.L)
    lid = ctx.lattice(s, lat)
    qid = ctx.qset(lid)
    with pytest.raises(_lib.SMDError) as e:
        ctx.batch([(lid, qid, 2, None)], 0.01, 16, 1, _lib.SMD_FP64, 1)
    assert e.value.code == _lib.SMD_EINVAL
