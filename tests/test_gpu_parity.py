"""CUDA path against the oracle and the reference's own outputs (B200 only).

Tolerances (FP64 plain form), as the path's contract states them:
  * per spin, within 1e-10 of the reference over the first 200 steps;
  * spectra and autocorrelation of short runs: max |diff| <= 1e-10 of max |ref|.
The GPU correction step updates all sites from one set of fields (Jacobi)
where the reference updates in site order; the difference is O(scale^2) per
step, far below these bounds.
"""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from classical_mc_and_smd_for_2d_heisenberg_models_b200 import _lib, smd
from classical_mc_and_smd_for_2d_heisenberg_models_b200 import samples as smp
from classical_mc_and_smd_for_2d_heisenberg_models_b200.settings import SMDSettings

pytestmark = pytest.mark.gpu

SPIN_TOL = 1e-10
SPEC_TOL = 1e-10


def _upload(ctx, s, d=None):
    """Build and upload a lattice: from the geometry for a crystal, from the
    fixture's reference tables (sitesList / nborsList) for a quasi-crystal."""
    if s.qcrystal:
        lat = smd.Lattice(s.geom, s.G, s.N, s.G, 1, list(s.zn), np.asarray(d["rvec"]), None,
                          [np.asarray(d[k]) for k in ("nb1", "nb2", "nbx")])
    else:
        lat = smd.build_lattice(s.geom, s.L)
    return lat, ctx.lattice(s, lat)


def _golden_qset(ctx, s, lat, lid):
    """The fixture's q set: the DFT grid of a crystal; for a quasi-crystal
    the direct-sum Lsz x Lsz set of get_qct_SqData."""
    if s.qcrystal:
        q, sc = smd.qcrystal_qpoints(lat)
        return ctx.qset(lid, use_grid=False, qlist=q, list_scale=sc)
    return ctx.qset(lid, use_grid=True)


@pytest.mark.parametrize("name", golden_names("traj_"))
def test_fp64_200_steps_per_spin(ctx, name):
    s, d = load_golden(name)
    lat, lid = _upload(ctx, s, d)
    n = int(d["n"])
    imp = None if "imp" not in d else np.tile(d["imp"], (n, 1))
    fin = ctx.evolve(lid, d["spins0"][:n], s.dtm, s.ntm - 1, imp=imp)
    err = np.max(np.abs(fin - d["final"]))
    assert err <= SPIN_TOL, err


@pytest.mark.parametrize("name", golden_names("spec_"))
def test_fp64_spectrum_equals_reference(ctx, name):
    s, d = load_golden(name)
    lat, lid = _upload(ctx, s, d)
    qid = _golden_qset(ctx, s, lat, lid)
    n = int(d["n"])
    imp = None if "imp" not in d else np.tile(d["imp"], (n, 1))
    r = ctx.run(lid, qid, d["spins0"][:n], s.dtm, s.ntm, win=d["window"], imp=imp)
    ref = d["spec_sum"] / n
    assert np.max(np.abs(r.spec - ref)) <= SPEC_TOL * np.max(np.abs(ref))
    assert np.max(np.abs(r.qss - d["qss_sum"] / n)) <= SPEC_TOL
    assert np.max(np.abs(r.final - d["final"])) <= SPIN_TOL


def test_reference_entry_point(ctx):
    """smd_dyn_spectrum_ref: the data of get_dynSpectrum with flat arrays."""
    s, d = load_golden("spec_triang")
    lat, lid = _upload(ctx, s)
    qid = ctx.qset(lid, use_grid=True)
    sf = d["spins0"][0].copy()
    x, y, z, q = ctx.get_dyn_spectrum(lid, qid, s.dtm, s.ntm, d["window"], sf)
    assert np.max(np.abs(sf - d["final"][0])) <= SPIN_TOL
    assert x.shape == (s.G * s.G, s.ntm)
    assert q[0] == 1.0


@pytest.mark.parametrize("geom,L,J2,JX,stride,n_rec", [
    ("square", 16, 0.6, 0.0, 4, 64),
    ("triang", 12, 0.12, 0.0, 2, 48),
    ("kagome", 6, 0.3, 0.1, 3, 40),
    ("hexagn", 6, 0.2, 0.05, 2, 30),
])
def test_fp64_strided_grid_and_list_vs_oracle(ctx, oracle_mod, geom, L, J2, JX, stride, n_rec):
    s = SMDSettings(geom=geom, L=L, J2=J2, JX=JX, dtm=0.01, ntm=n_rec, window="hann1",
                    NMeas=4000)
    lat, lid = _upload(ctx, s)
    rng = np.random.default_rng(3)
    ql = rng.uniform(-np.pi, np.pi, size=(7, 2))
    qid = ctx.qset(lid, use_grid=True, qlist=ql)
    kind = "q120" if geom == "triang" else ("stripe" if geom == "square" else "ferro")
    spins, _ = smp.make_samples(s, 3, kind, 0.4, 9)
    win = smd.window("hann1", n_rec)
    r = ctx.run(lid, qid, spins, s.dtm, n_rec, stride=stride, win=win)
    olat = oracle_mod.make_lattice(geom, L)
    m = oracle_mod.Model(s, olat)
    acc, accq = 0.0, 0.0
    for k in range(3):
        o = oracle_mod.dyn_spectrum(m, spins[k], s.dtm, n_rec, stride=stride, win=win,
                                    qlist=ql, pos=lat.grid_positions(), list_scale=1.0 / lat.G)
        acc = acc + o["spec"]
        accq = accq + o["qss"]
        assert np.max(np.abs(r.final[k] - o["final"])) <= SPIN_TOL
    acc /= 3
    accq /= 3
    assert np.max(np.abs(r.spec - acc)) <= SPEC_TOL * np.max(np.abs(acc))
    assert np.max(np.abs(r.qss - accq)) <= SPEC_TOL


@pytest.mark.parametrize("precision", [_lib.SMD_FP64, _lib.SMD_FP32])
@pytest.mark.parametrize("n_rec", [16, 32, 128, 512, 2048, 4096, 96, 1000])
def test_time_transform_lengths_vs_oracle(ctx, oracle_mod, precision, n_rec):
    """Every class of record count: powers of two 16 .. 4096 (register
    radix-16 passes closing with radix 2, 4 or 8) and mixed radices (shared-
    memory stages); an odd q count leaves the last q block half used."""
    s = SMDSettings(geom="square", L=4, J2=0.6, dtm=0.002, ntm=n_rec, window="hann2")
    lat, lid = _upload(ctx, s)
    ql = np.random.default_rng(5).uniform(-np.pi, np.pi, size=(5, 2))
    qid = ctx.qset(lid, use_grid=True, qlist=ql)
    spins, _ = smp.make_samples(s, 2, "stripe", 0.4, 3)
    win = smd.window("hann2", n_rec)
    kw = dict(precision=precision, fix_every=16) if precision == _lib.SMD_FP32 else {}
    r = ctx.run(lid, qid, spins, s.dtm, n_rec, win=win, **kw)
    m = oracle_mod.Model(s, oracle_mod.make_lattice("square", 4))
    acc = 0.0
    for k in range(2):
        acc = acc + oracle_mod.dyn_spectrum(m, spins[k], s.dtm, n_rec, win=win, qlist=ql,
                                            pos=lat.grid_positions(),
                                            list_scale=1.0 / lat.G)["spec"]
    acc /= 2
    if precision == _lib.SMD_FP64:
        assert np.max(np.abs(r.spec - acc)) <= SPEC_TOL * np.max(np.abs(acc))
    else:
        G2 = lat.G * lat.G
        for part in (slice(0, G2), slice(G2, None)):
            a, b = r.spec[:, part], acc[:, part]
            assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-3


@pytest.mark.parametrize("geom,L", [("kagome", 12), ("hexagn", 6), ("square", 16)])
def test_two_pass_grid_transform_vs_oracle(ctx, oracle_mod, monkeypatch, geom, L):
    """The two-pass grid transform (rows, then columns through a global
    scratch) against the oracle, FP64, on grids that also fit one block."""
    monkeypatch.setenv("SMD_GRID_TWO_PASS", "1")
    s = SMDSettings(geom=geom, L=L, J2=0.3, JX=0.05, dtm=0.01, ntm=24, window="hann1")
    lat, lid = _upload(ctx, s)
    qid = ctx.qset(lid, use_grid=True)
    kind = "stripe" if geom == "square" else "ferro"
    spins, _ = smp.make_samples(s, 3, kind, 0.4, 12)
    win = smd.window("hann1", 24)
    r = ctx.run(lid, qid, spins, s.dtm, 24, stride=2, win=win)
    m = oracle_mod.Model(s, oracle_mod.make_lattice(geom, L))
    acc = 0.0
    for k in range(3):
        acc = acc + oracle_mod.dyn_spectrum(m, spins[k], s.dtm, 24, stride=2, win=win)["spec"]
    acc /= 3
    assert np.max(np.abs(r.spec - acc)) <= SPEC_TOL * np.max(np.abs(acc))


@pytest.mark.parametrize("precision", [_lib.SMD_FP64, _lib.SMD_FP32])
def test_grid_larger_than_one_block(ctx, oracle_mod, precision):
    """Honeycomb L = 48 (N = 4608, a 144 x 144 grid): the FP64 form takes the
    two-pass transform (beyond one block's shared memory), the FP32 form one
    block per component with its rows and columns in three batches each;
    against the oracle (FP64 within 1e-10, FP32 form within 1e-3 rel-L2)."""
    s = SMDSettings(geom="hexagn", L=48, J2=0.2, dtm=0.01, ntm=16, window="hann1")
    lat, lid = _upload(ctx, s)
    qid = ctx.qset(lid, use_grid=True)
    spins, _ = smp.make_samples(s, 2, "ferro", 0.3, 21)
    win = smd.window("hann1", 16)
    kw = dict(precision=precision, fix_every=16) if precision == _lib.SMD_FP32 else {}
    r = ctx.run(lid, qid, spins, s.dtm, 16, win=win, **kw)
    m = oracle_mod.Model(s, oracle_mod.make_lattice("hexagn", 48))
    acc = 0.0
    for k in range(2):
        acc = acc + oracle_mod.dyn_spectrum(m, spins[k], s.dtm, 16, win=win)["spec"]
    acc /= 2
    if precision == _lib.SMD_FP64:
        assert np.max(np.abs(r.spec - acc)) <= SPEC_TOL * np.max(np.abs(acc))
    else:
        assert np.linalg.norm(r.spec - acc) / np.linalg.norm(acc) <= 1e-3


@pytest.mark.parametrize("two_pass", [False, True])
@pytest.mark.parametrize("precision", [_lib.SMD_FP64, _lib.SMD_FP32])
def test_radix5_grid_and_time_transforms_vs_oracle(ctx, oracle_mod, monkeypatch, precision, two_pass):
    """Honeycomb L = 30: a 90 x 90 grid (radices 2, 3, 3, 5) in one block and
    through the two-pass transform, and 50 records (radices 2, 5, 5): the
    inline radix-5 stages against the oracle (FP64 within 1e-10, FP32 form
    within 1e-3 rel-L2)."""
    if two_pass:
        monkeypatch.setenv("SMD_GRID_TWO_PASS", "1")
    s = SMDSettings(geom="hexagn", L=30, J2=0.2, JX=0.05, dtm=0.01, ntm=50, window="hann1")
    lat, lid = _upload(ctx, s)
    assert lat.G == 90
    qid = ctx.qset(lid, use_grid=True)
    spins, _ = smp.make_samples(s, 2, "ferro", 0.4, 17)
    win = smd.window("hann1", 50)
    kw = dict(precision=precision, fix_every=16) if precision == _lib.SMD_FP32 else {}
    r = ctx.run(lid, qid, spins, s.dtm, 50, win=win, **kw)
    m = oracle_mod.Model(s, oracle_mod.make_lattice("hexagn", 30))
    acc = 0.0
    for k in range(2):
        acc = acc + oracle_mod.dyn_spectrum(m, spins[k], s.dtm, 50, win=win)["spec"]
    acc /= 2
    if precision == _lib.SMD_FP64:
        assert np.max(np.abs(r.spec - acc)) <= SPEC_TOL * np.max(np.abs(acc))
    else:
        assert np.linalg.norm(r.spec - acc) / np.linalg.norm(acc) <= 1e-3


def test_list_points_on_the_grid_equal_grid_values(ctx):
    s = SMDSettings(geom="kagome", L=6, J2=0.3, dtm=0.01, ntm=16)
    lat, lid = _upload(ctx, s)
    gq = lat.grid_qvectors()
    pick = np.array([0, 5, 17, 40, 143])
    qid = ctx.qset(lid, use_grid=True, qlist=gq[pick])
    spins, _ = smp.make_samples(s, 2, "ferro", 0.5, 4)
    r = ctx.run(lid, qid, spins, s.dtm, 16)
    G2 = lat.G * lat.G
    a = r.spec[:, pick, :]
    b = r.spec[:, G2:, :]
    assert np.max(np.abs(a - b)) <= 1e-11 * np.max(np.abs(a))


def test_runs_are_deterministic(ctx):
    s = SMDSettings(geom="square", L=16, J2=0.6, dtm=0.01, ntm=32)
    lat, lid = _upload(ctx, s)
    qid = ctx.qset(lid)
    spins, _ = smp.make_samples(s, 4, "stripe", 0.2, 1)
    a = ctx.run(lid, qid, spins, s.dtm, 32, stride=2)
    b = ctx.run(lid, qid, spins, s.dtm, 32, stride=2)
    assert np.array_equal(a.spec, b.spec) and np.array_equal(a.final, b.final)


def test_fp32_form_energy_and_spectrum_error(ctx):
    """Precision form: FP32 stages, FP64 correction every 16 steps, grid by
    FP32 FFT and a Gamma-K-M path by split-BF16 tensor-core GEMM."""
    from classical_mc_and_smd_for_2d_heisenberg_models_b200 import workloads
    s = SMDSettings(geom="triang", L=48, J2=0.12, dtm=0.02, ntm=256, window="hann1")
    lat, lid = _upload(ctx, s)
    qid = ctx.qset(lid, qlist=workloads.path_points("triang", 512))
    spins, _ = smp.make_samples(s, 8, "q120", 0.15, 2)
    win = smd.window("hann1", 256)
    r64 = ctx.run(lid, qid, spins, s.dtm, 256, stride=4, win=win)
    r32 = ctx.run(lid, qid, spins, s.dtm, 256, stride=4, win=win, precision=_lib.SMD_FP32,
                  fix_every=16)
    G2 = lat.G * lat.G
    for part in (slice(0, G2), slice(G2, None)):
        a, b = r32.spec[:, part], r64.spec[:, part]
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert rel <= 1e-3, rel
    assert r32.report["drift_final"] <= 1e-8, r32.report
    assert r32.report["drift_max"] <= 1e-8, r32.report


@pytest.mark.parametrize("N_L", [(16, 300), (30, 700)])
def test_tensor_core_projection_matches_grid_fft(ctx, N_L):
    """List points placed on grid q: the split-BF16 tensor-core values equal
    the FP32 FFT values (same FP32 trajectory) to the split-BF16 accuracy."""
    L, nl = N_L
    s = SMDSettings(geom="square", L=L, J2=0.6, dtm=0.01, ntm=32)
    lat, lid = _upload(ctx, s)
    gq = lat.grid_qvectors()
    pick = np.random.default_rng(1).choice(len(gq), size=min(nl, len(gq)), replace=False)
    qid = ctx.qset(lid, use_grid=True, qlist=gq[pick])
    spins, _ = smp.make_samples(s, 3, "stripe", 0.3, 6)
    r = ctx.run(lid, qid, spins, s.dtm, 32, stride=2, precision=_lib.SMD_FP32, fix_every=16)
    G2 = lat.G * lat.G
    a = r.spec[:, pick, :]
    b = r.spec[:, G2:, :]
    assert np.linalg.norm(a - b) / np.linalg.norm(a) <= 2e-4


@pytest.fixture
def cluster_size(monkeypatch):
    """Force the number of CTAs the cluster kernel spreads a sample over
    (SMD_CLUSTER_CTAS)."""
    def set_(cs):
        monkeypatch.setenv("SMD_CLUSTER_CTAS", str(cs))
    return set_


@pytest.mark.parametrize("cs", [1, 2, 4])
def test_cluster_fp32_form_tracks_fp64(ctx, cluster_size, cs):
    """FP32 precision form on the cluster kernel (XXZ, field, three shells,
    vacancies): spectrum within 1e-3 (rel-L2) of the FP64 form, energy drift
    within 1e-8 per site."""
    cluster_size(cs)
    s = SMDSettings(geom="square", L=24, J2=0.55, JX=0.1, zlamb1=0.9, zlamb2=0.9, h=0.3,
                    imp_ratio=0.05, dtm=0.01, ntm=128, NMeas=4000)
    lat, lid = _upload(ctx, s)
    qid = ctx.qset(lid)
    spins, imp = smp.make_samples(s, 4, "stripe", 0.1, 5)
    impr = np.tile(imp[0], (4, 1))
    win = smd.window("hann1", 128)
    r64 = ctx.run(lid, qid, spins, s.dtm, 128, stride=4, win=win, imp=impr)
    r32 = ctx.run(lid, qid, spins, s.dtm, 128, stride=4, win=win, imp=impr,
                  precision=_lib.SMD_FP32, fix_every=16)
    assert r32.report["rk_kind"] == 1 and r64.report["rk_kind"] == 1
    assert r32.report["rk_ctas"] == cs and r64.report["rk_ctas"] == cs
    rel = np.linalg.norm(r32.spec - r64.spec) / np.linalg.norm(r64.spec)
    assert rel <= 1e-3, rel
    assert r32.report["drift_max"] <= 1e-8 and r32.report["drift_final"] <= 1e-8


@pytest.mark.parametrize("cs", [1, 2, 4, 8])
@pytest.mark.parametrize("name", ["traj_square_xxz_h_vac", "traj_triang_j1j2", "traj_kagome",
                                  "traj_hexagn"])
def test_cluster_kernel_200_steps_per_spin(ctx, cluster_size, cs, name):
    """The cluster kernel (sample split over cs CTAs, halo exchange through
    distributed shared memory) keeps the reference's per-spin parity."""
    cluster_size(cs)
    s, d = load_golden(name)
    lat, lid = _upload(ctx, s)
    n = int(d["n"])
    imp = None if "imp" not in d else np.tile(d["imp"], (n, 1))
    fin = ctx.evolve(lid, d["spins0"][:n], s.dtm, s.ntm - 1, imp=imp)
    assert np.max(np.abs(fin - d["final"])) <= SPIN_TOL


@pytest.mark.parametrize("cs", [2, 4])
def test_cluster_kernel_spectrum(ctx, cluster_size, cs):
    cluster_size(cs)
    s, d = load_golden("spec_kagome")
    lat, lid = _upload(ctx, s)
    qid = ctx.qset(lid, use_grid=True)
    n = int(d["n"])
    r = ctx.run(lid, qid, d["spins0"][:n], s.dtm, s.ntm, win=d["window"])
    ref = d["spec_sum"] / n
    assert np.max(np.abs(r.spec - ref)) <= SPEC_TOL * np.max(np.abs(ref))
    assert np.max(np.abs(r.final - d["final"])) <= SPIN_TOL


@pytest.mark.parametrize("cs", [1, 2, 4])
def test_cluster_fp32_form_tracks_fp64(ctx, cluster_size, cs):
    """FP32 precision form on a cluster: spectrum within 1e-3 (rel-L2) of the
    FP64 form, energy drift within 1e-8 per site."""
    cluster_size(cs)
    s = SMDSettings(geom="square", L=32, J2=0.55, JX=0.1, zlamb1=0.9, zlamb2=0.9, h=0.3,
                    imp_ratio=0.05, dtm=0.01, ntm=128, NMeas=4000)
    lat, lid = _upload(ctx, s)
    qid = ctx.qset(lid)
    spins, imp = smp.make_samples(s, 4, "stripe", 0.1, 5)
    impr = np.tile(imp[0], (4, 1))
    win = smd.window("hann1", 128)
    r64 = ctx.run(lid, qid, spins, s.dtm, 128, stride=4, win=win, imp=impr)
    r32 = ctx.run(lid, qid, spins, s.dtm, 128, stride=4, win=win, imp=impr,
                  precision=_lib.SMD_FP32, fix_every=16)
    rel = np.linalg.norm(r32.spec - r64.spec) / np.linalg.norm(r64.spec)
    assert rel <= 1e-3, rel
    assert r32.report["drift_max"] <= 1e-8 and r32.report["drift_final"] <= 1e-8


def test_cluster_vacancies_match_oracle(ctx, oracle_mod, cluster_size):
    """Vacancy disorder through the masked cluster kernel against the oracle."""
    cluster_size(2)
    s = SMDSettings(geom="square", L=16, J2=0.55, JX=0.1, zlamb1=0.9, zlamb2=0.9, h=0.3,
                    imp_ratio=0.05, dtm=0.01, ntm=24, NMeas=2000)
    lat, lid = _upload(ctx, s)
    qid = ctx.qset(lid)
    spins, imp = smp.make_samples(s, 2, "stripe", 0.2, 8)
    impr = np.tile(imp[0], (2, 1))
    r = ctx.run(lid, qid, spins, s.dtm, 24, stride=3, imp=impr)
    m = oracle_mod.Model(s, oracle_mod.make_lattice(s.geom, s.L), imp[0])
    acc = 0.0
    for k in range(2):
        o = oracle_mod.dyn_spectrum(m, spins[k], s.dtm, 24, stride=3)
        acc = acc + o["spec"]
        assert np.max(np.abs(r.final[k] - o["final"])) <= SPIN_TOL
    acc /= 2
    assert np.max(np.abs(r.spec - acc)) <= SPEC_TOL * np.max(np.abs(acc))


@pytest.mark.parametrize("geom,L,cs", [("triang", 48, 2), ("triang", 48, 16), ("hexagn", 24, 4),
                                        ("square", 32, 8)])
@pytest.mark.parametrize("precision", [_lib.SMD_FP64, _lib.SMD_FP32])
def test_async_halo_equals_cluster_barrier_halo(ctx, cluster_size, monkeypatch, geom, L, cs, precision):
    """Halo publishes through st.async stores completing on the receiver's
    mbarriers (the default) and through cluster barriers (SMD_RK_HALO=barrier)
    move the same values: identical trajectories and spectra over several
    record chunks, energy corrections included."""
    cluster_size(cs)
    s = SMDSettings(geom=geom, L=L, J2=0.12, JX=0.05, h=0.1, imp_ratio=0.05 if geom == "square" else 0.0,
                    dtm=0.02, ntm=150, NMeas=2000)
    lat, lid = _upload(ctx, s)
    qid = ctx.qset(lid)
    kind = {"triang": "q120", "square": "stripe"}.get(geom, "ferro")
    spins, imp = smp.make_samples(s, 3, kind, 0.15, 11)
    impr = None if imp is None else np.tile(imp[0], (3, 1))
    kw = dict(stride=4, precision=precision, fix_every=16 if precision == _lib.SMD_FP32 else 1, imp=impr)
    a = ctx.run(lid, qid, spins, s.dtm, 150, **kw)
    monkeypatch.setenv("SMD_RK_HALO", "barrier")
    b = ctx.run(lid, qid, spins, s.dtm, 150, **kw)
    assert a.report["rk_kind"] == 1 and a.report["rk_ctas"] == cs
    assert np.array_equal(a.final, b.final)
    assert np.array_equal(a.spec, b.spec) and np.array_equal(a.qss, b.qss)


def test_invalid_jobs_fail_loudly(ctx):
    s = SMDSettings(geom="square", L=8, J2=0.6, dtm=0.01, ntm=16)
    lat, lid = _upload(ctx, s)
    qid = ctx.qset(lid)
    spins, _ = smp.make_samples(s, 1, "stripe", 0.2, 1)
    with pytest.raises(_lib.SMDError):
        ctx.run(lid, qid, spins, -0.01, 16)
    with pytest.raises(_lib.SMDError):
        ctx.run(lid, qid + 1000, spins, 0.01, 16)
    with pytest.raises(_lib.SMDError):
        ctx.run(lid, qid, spins, 0.01, 1)


def _c2_forms(ctx, n_samples, n_rec):
    """FP64, FP32 and FP32-roundoff-perturbed FP64 runs of the benched
    workload's lattice (triangular L = 48, stride 4, dt = 0.02, 48 x 48 grid
    plus the 512-point path) over n_rec records."""
    from classical_mc_and_smd_for_2d_heisenberg_models_b200 import workloads
    w = workloads.c2(n_samples)
    s = w.settings
    lat, lid = _upload(ctx, s)
    ql = workloads.path_points(s.geom, w.qpath_points)
    qid = ctx.qset(lid, use_grid=True, qlist=ql)
    spins, _ = workloads.make_inputs(w)
    win = smd.window(w.window, n_rec)
    kw = dict(stride=w.stride, win=win, want_final=False)
    r64 = ctx.run(lid, qid, spins, s.dtm, n_rec, **kw)
    r32 = ctx.run(lid, qid, spins, s.dtm, n_rec, precision=_lib.SMD_FP32, fix_every=w.fix_every, **kw)
    pert = workloads.tangent_perturb(spins, workloads.FP32_ROUNDOFF, 11)
    r64p = ctx.run(lid, qid, pert, s.dtm, n_rec, **kw)
    G2 = lat.G * lat.G
    parts = {"grid": slice(0, G2), "path": slice(G2, None)}

    def rel(a, b, part):
        return np.linalg.norm(a.spec[:, part] - b.spec[:, part]) / np.linalg.norm(b.spec[:, part])

    return r64, r32, r64p, parts, rel


def test_fp32_form_within_1e3_before_the_chaotic_horizon(ctx):
    """1024 records (4092 RK steps) of the benched workload on 4 samples,
    a length over which an FP32-sized input perturbation has not yet grown
    (the FP64 form's own sensitivity stays far below 1e-3): the FP32 form's
    spectrum is within 1e-3 rel-L2 of the FP64 form's, grid and path
    separately, with energy drift at most 1e-8 per site."""
    r64, r32, r64p, parts, rel = _c2_forms(ctx, 4, 1024)
    for name, part in parts.items():
        assert rel(r64p, r64, part) <= 1e-4, (name, "the run is already chaotic")
        assert rel(r32, r64, part) <= 1e-3, (name, rel(r32, r64, part))
    assert r32.report["drift_max"] <= 1e-8 and r32.report["drift_final"] <= 1e-8, r32.report


def test_fp32_form_at_c2_length_within_the_chaos_floor(ctx):
    """The benched length -- 4096 records at stride 4, 16 380 RK steps -- on 8
    samples.  Over this length the trajectories are chaotic: the FP64 form run
    from inputs moved by one FP32 rounding (2^-24) ends with spins
    decorrelated from the unperturbed run, and its spectrum differs by a few
    1e-2.  No arithmetic that rounds at FP32 can get closer than that floor, so
    the FP32 form's DSSF rel-L2 against the FP64 form must be of the floor's
    order: at most 2 x the floor (grid and path separately; the FP32 form
    rounds at every stage, not once at the start).  Its energy drift is at
    most 1e-8 per site.  The FP64 form is the one pinned to the reference per
    spin."""
    r64, r32, r64p, parts, rel = _c2_forms(ctx, 8, 4096)
    for name, part in parts.items():
        floor = rel(r64p, r64, part)
        assert rel(r32, r64, part) <= max(1e-3, 2.0 * floor), (name, rel(r32, r64, part), floor)
    assert r32.report["drift_max"] <= 1e-8 and r32.report["drift_final"] <= 1e-8, r32.report
