"""GPU Monte Carlo sampler (smd_mc_run) against the reference's own MC stage.

The sampler visits sites by colour class with a counter-based generator, the
reference in shuffled order with dSFMT: the two agree in distribution, not
draw by draw.  The fixtures mc_*.npz hold the mean energy per site of
independent runs of the reference's MC sweeps (oracle/_ref/smd_ref_run --mc,
tests/golden/make_golden.py --mc); the GPU's mean over its chains must lie
within 5 combined standard errors of it.
"""
import numpy as np
import pytest

from conftest import load_golden
from classical_mc_and_smd_for_2d_heisenberg_models_b200 import samples as smp, smd
from classical_mc_and_smd_for_2d_heisenberg_models_b200.settings import SMDSettings

pytestmark = pytest.mark.gpu

MC_CASES = ["mc_square_j1j2", "mc_triang_h_vac", "mc_kagome_xxz", "mc_qct239"]


def _lattice(ctx, s, d):
    if s.qcrystal:
        lat = smd.Lattice(s.geom, s.G, s.N, s.G, 1, list(s.zn), np.asarray(d["rvec"]), None,
                          [np.asarray(d[k]) for k in ("nb1", "nb2", "nbx")])
    else:
        lat = smd.build_lattice(s.geom, s.L)
    return lat, ctx.lattice(s, lat)


@pytest.mark.parametrize("geom,L,J2,JX", [("square", 8, 0.3, 0.0), ("triang", 12, 0.2, 0.1),
                                          ("kagome", 6, 0.3, 0.1), ("hexagn", 6, 0.2, 0.05),
                                          ("lieb", 8, 0.0, 0.0)])
def test_colour_classes_partition_the_sites_without_shared_bonds(ctx, geom, L, J2, JX):
    s = SMDSettings(geom=geom, L=L, J2=J2, JX=JX)
    lat = smd.build_lattice(geom, L)
    lid = ctx.lattice(s, lat)
    order, cst = ctx.mc_colouring(lid)
    assert sorted(order.tolist()) == list(range(lat.N))
    col = np.empty(lat.N, int)
    for c in range(len(cst) - 1):
        col[order[cst[c]:cst[c + 1]]] = c
    on = [True, s.j2_on, s.jx_on]
    for k in range(3):
        if not on[k]:
            continue
        nb = lat.nbrs[k]
        ok = nb >= 0
        i = np.repeat(np.arange(lat.N)[:, None], nb.shape[1], axis=1)
        assert not np.any(col[i[ok]] == col[nb[ok]]), (geom, k)


def _chain_means(e, s, therm):
    """Mean energy per site of every chain over the measurement steps."""
    return e[:, :, therm:].mean(axis=2) / s.N        # [chains][T]


@pytest.mark.parametrize("name", MC_CASES)
def test_energy_matches_the_reference_mc(ctx, name):
    s, d = load_golden(name)
    lat, lid = _lattice(ctx, s, d)
    temps = np.asarray(d["temps"])
    therm, meas, runs = int(d["therm"]), int(d["meas"]), int(d["runs"])
    ref = np.asarray(d["e_site"])                       # [T][runs]
    for ti, T in enumerate(temps):
        chains = 2 * runs
        imp = None
        if "imp" in d:
            # the reference's impurity maps, each on two chains
            maps = np.asarray(d["imp"])[ti].astype(np.int32)       # [runs][N]
            imp = np.repeat(maps, 2, axis=0)[:, None, :]
        out = ctx.mc_run(lid, [T], therm, meas, cr_skip=meas, chains=chains, seed=101 + ti,
                         imp=imp, want_samples=False)
        m = _chain_means(out["energy"], s, therm)[:, 0]
        gpu, gpu_se = m.mean(), m.std(ddof=1) / np.sqrt(len(m))
        r, r_se = ref[ti].mean(), ref[ti].std(ddof=1) / np.sqrt(runs)
        tol = 5.0 * np.hypot(gpu_se, r_se)
        assert abs(gpu - r) <= tol, (name, T, gpu, r, tol)


def test_tempering_keeps_each_temperature_at_its_reference_energy(ctx):
    """Parallel tempering over T = 0.3, 0.45, 0.6, 0.8 on the square J1-J2
    case: exchanges are attempted and accepted, and the energies at 0.3 and
    0.8 still match the reference's single-temperature runs (exchanges leave
    every temperature's distribution unchanged)."""
    s, d = load_golden("mc_square_j1j2")
    lat, lid = _lattice(ctx, s, d)
    therm, meas, runs = int(d["therm"]), int(d["meas"]), int(d["runs"])
    temps = [0.3, 0.45, 0.6, 0.8]
    out = ctx.mc_run(lid, temps, therm, meas, cr_skip=meas, chains=16, pt=True, seed=7,
                     want_samples=False)
    cnt = out["pt_counts"]
    assert cnt[:, :, 0].sum() > 0 and cnt[:, :, 1].sum() > 0
    assert np.all(cnt[:, :, 1] <= cnt[:, :, 0])
    m = _chain_means(out["energy"], s, therm)
    ref = np.asarray(d["e_site"])
    for ti, tg in ((0, 0), (3, 1)):
        gpu, gpu_se = m[:, ti].mean(), m[:, ti].std(ddof=1) / np.sqrt(m.shape[0])
        r, r_se = ref[tg].mean(), ref[tg].std(ddof=1) / np.sqrt(runs)
        assert abs(gpu - r) <= 5.0 * np.hypot(gpu_se, r_se), (temps[ti], gpu, r)
    # energy decreases with temperature
    assert np.all(np.diff(m.mean(axis=0)) > 0)


def test_records_are_unit_spin_fields_that_feed_the_smd_path(ctx, tmp_path):
    """Records every cr_skip measurement steps, unit spins, reproducible for a
    seed; written in the reference's sample-file format and read back, they
    run through smd_run."""
    s = SMDSettings(geom="triang", L=6, J2=0.12, T1=0.4, T2=0.4, NMeas=4000, crSkip=1000, ntm=32,
                    dtm=0.02)
    lat = smd.build_lattice(s.geom, s.L)
    lid = ctx.lattice(s, lat)
    a = ctx.mc_run(lid, [0.4], 200, 4000, cr_skip=1000, chains=1, seed=3)
    b = ctx.mc_run(lid, [0.4], 200, 4000, cr_skip=1000, chains=1, seed=3)
    rec = a["samples"][0, 0]
    assert rec.shape == (4, lat.N, 3)
    assert np.allclose(np.linalg.norm(rec, axis=2), 1.0, atol=1e-12)
    assert np.array_equal(a["energy"], b["energy"]) and np.array_equal(a["samples"], b["samples"])
    path = str(tmp_path / smp.sample_file_name(s))
    smp.write_sample_file(path, s, rec, None)
    spins, _ = smp.read_sample_file(path, s)
    assert np.array_equal(spins, rec)
    qid = ctx.qset(lid)
    r = ctx.run(lid, qid, spins, s.dtm, s.ntm, want_final=False)
    assert np.all(np.isfinite(r.spec)) and r.qss[0] == 1.0


def test_large_lattice_runs_with_the_block_size_its_registers_allow(ctx):
    """Square L = 64 with J2: 4 colour classes of 1024 sites each, more than
    the kernel's register budget allows threads for; the sampler strides over
    the class with the largest block it can launch."""
    s = SMDSettings(geom="square", L=64, J2=0.3)
    lat = smd.build_lattice(s.geom, s.L)
    lid = ctx.lattice(s, lat)
    out = ctx.mc_run(lid, [0.4, 0.8], 5, 10, cr_skip=5, chains=2, pt=True, seed=9)
    assert np.all(np.isfinite(out["energy"])) and out["samples"].shape == (2, 2, 2, lat.N, 3)
    assert np.allclose(np.linalg.norm(out["samples"], axis=-1), 1.0, atol=1e-12)
