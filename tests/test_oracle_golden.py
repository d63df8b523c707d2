"""The oracle (C restatement) against fixtures produced by the reference's own code."""
import numpy as np
import pytest

from conftest import golden_lattice, golden_names, load_golden


@pytest.mark.parametrize("name", golden_names())
def test_lattice_tables_match_reference(oracle_mod, name):
    s, d = load_golden(name)
    lat = golden_lattice(oracle_mod, s, d)
    assert np.array_equal(lat["rvec"], d["rvec"])
    assert np.array_equal(lat["grid_map"], d["grid_map"])
    for a, b in zip(lat["nbrs"], (d["nb1"], d["nb2"], d["nbx"])):
        assert np.array_equal(a, b)
    bonds, nb = oracle_mod.make_bonds(lat, s.j2_on, s.jx_on)
    assert list(nb) == list(d["nbonds"])
    assert np.array_equal(bonds, d["bonds"])


@pytest.mark.parametrize("name", golden_names("traj_"))
def test_trajectory_matches_reference(oracle_mod, name):
    s, d = load_golden(name)
    lat = golden_lattice(oracle_mod, s, d)
    for k in range(int(d["n"])):
        m = oracle_mod.Model(s, lat, d.get("imp"))
        fin, _ = oracle_mod.evolve(m, d["spins0"][k], s.dtm, s.ntm - 1)
        # same arithmetic as the reference: equal to the last bit
        assert np.max(np.abs(fin - d["final"][k])) <= 1e-15


@pytest.mark.parametrize("name", golden_names("spec_"))
def test_spectrum_matches_reference(oracle_mod, name):
    s, d = load_golden(name)
    lat = golden_lattice(oracle_mod, s, d)
    kw = {}
    if s.qcrystal:
        # the direct-sum transform of get_qct_SqData over the Lsz x Lsz q set
        q, sc = oracle_mod.qct_qpoints(s.G, s.N)
        kw = dict(grid=False, qlist=q, pos=d["rvec"], list_scale=sc)
    acc = 0.0
    accq = 0.0
    for k in range(int(d["n"])):
        m = oracle_mod.Model(s, lat, d.get("imp"))
        out = oracle_mod.dyn_spectrum(m, d["spins0"][k], s.dtm, s.ntm, win=d["window"], **kw)
        acc = acc + out["spec"]
        accq = accq + out["qss"]
        assert np.max(np.abs(out["final"] - d["final"][k])) <= 1e-15
    ref = d["spec_sum"]
    assert np.max(np.abs(acc - ref)) <= 1e-13 * np.max(np.abs(ref))
    assert np.max(np.abs(accq - d["qss_sum"])) <= 1e-14


@pytest.mark.parametrize("name", ["gauss", "ntall", "black", "flatw", "lancz", "sincw",
                                  "hann1", "hann2", "hann3", "nowin"])
def test_windows_are_finite_and_peak_at_centre(oracle_mod, name):
    w = oracle_mod.window(name, 64)
    assert np.all(np.isfinite(w))
    assert w.shape == (64,)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 12, 16, 48, 90, 97, 128, 210])
def test_oracle_fft_matches_naive_dft(oracle_mod, n):
    rng = np.random.default_rng(n)
    x = rng.normal(size=n) + 1j * rng.normal(size=n)
    a = oracle_mod.fft1d(x)
    b = oracle_mod.dft1d_naive(x)
    assert np.max(np.abs(a - b)) <= 1e-12 * max(1.0, np.max(np.abs(b)))
    assert np.max(np.abs(a - np.fft.fft(x))) <= 1e-12 * max(1.0, np.max(np.abs(b)))


def test_stride_one_equals_reference_semantics(oracle_mod):
    """stride s records every s-th state of the stride-1 trajectory."""
    s, d = load_golden("traj_square_j1j2")
    lat = oracle_mod.make_lattice(s.geom, s.L)
    m = oracle_mod.Model(s, lat)
    a = oracle_mod.dyn_spectrum(m, d["spins0"][0], s.dtm, 9, stride=1, want_series=True)
    b = oracle_mod.dyn_spectrum(m, d["spins0"][0], s.dtm, 5, stride=2, want_series=True)
    assert np.max(np.abs(a["series"][:, :, ::2] - b["series"])) == 0.0
