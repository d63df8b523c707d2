"""Host-side product code (no GPU): lattice builder, bonds, windows, settings,
sample files, and the exported C ABI."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_names, load_golden
from classical_mc_and_smd_for_2d_heisenberg_models_b200 import _lib, samples as smp, smd
from classical_mc_and_smd_for_2d_heisenberg_models_b200.settings import SMDSettings, SettingsError

HEADER = os.path.join(ROOT, "include", "smd_b200.h")


def header_symbols():
    txt = open(HEADER).read()
    return re.findall(r"^SMD_API\s+[\w\s\*]*?\b(smd_\w+)\s*\(", txt, flags=re.M)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    syms = header_symbols()
    assert syms == _lib.EXPORTS
    for s in syms:
        assert hasattr(lib, s), s
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (smd_\w+)", out))
    assert exported == set(syms)


def test_version_string():
    assert b"sm_100a" in _lib.load().smd_version()


@pytest.mark.parametrize("name", golden_names())
def test_product_lattice_equals_reference_tables(name, tmp_path):
    """Crystals: the product's lattice builder against the reference's
    make_rvecList / make_nborsTable / make_bondList.  Quasi-crystals: the
    product's table loader on the approximant's files (written back in the
    reference's binary layouts) and its bond list with ghost neighbours."""
    s, d = load_golden(name)
    if s.qcrystal:
        tag = s.size_tag
        np.asarray(d["rvec"], np.float64).tofile(str(tmp_path / f"sitesList{tag}.bin"))
        np.concatenate([d["nb1"], d["nb2"], d["nbx"]], axis=1).astype(np.int32).tofile(
            str(tmp_path / f"nborsList{tag}.bin"))
        lat = smd.load_qcrystal(str(tmp_path), s.N, s.geom)
        assert lat.G == s.G and lat.grid_map is None
    else:
        lat = smd.build_lattice(s.geom, s.L)
        assert np.array_equal(lat.grid_map, d["grid_map"])
    assert np.array_equal(lat.rvec, d["rvec"])
    for a, b in zip(lat.nbrs, (d["nb1"], d["nb2"], d["nbx"])):
        assert np.array_equal(a, b)
    bonds, nb = smd.build_bonds(lat, s.j2_on, s.jx_on)
    assert nb == list(d["nbonds"])
    assert np.array_equal(bonds, d["bonds"])


@pytest.mark.parametrize("geom,L", [("square", 4), ("square", 10), ("square", 24),
                                    ("triang", 12), ("triang", 18), ("hexagn", 12),
                                    ("kagome", 12), ("lieb", 10), ("lieb", 16)])
def test_product_lattice_equals_oracle(oracle_mod, geom, L):
    a = smd.build_lattice(geom, L)
    b = oracle_mod.make_lattice(geom, L)
    assert np.array_equal(a.rvec, b["rvec"])
    assert np.array_equal(a.grid_map, b["grid_map"])
    for x, y in zip(a.nbrs, b["nbrs"]):
        assert np.array_equal(x, y)


def test_lattice_rejects_sizes_the_reference_rejects(oracle_mod):
    for geom, L in [("square", 3), ("triang", 8), ("kagome", 4), ("hexagn", 10)]:
        with pytest.raises(_lib.SMDError):
            smd.build_lattice(geom, L)
    # square L=2 passes the size rule but has no third-neighbour shell
    with pytest.raises(_lib.SMDError):
        smd.build_lattice("square", 2)
    with pytest.raises(RuntimeError):
        oracle_mod.make_lattice("square", 2)


@pytest.mark.parametrize("name", ["gauss", "ntall", "black", "flatw", "lancz", "sincw",
                                  "hann1", "hann2", "hann3", "nowin"])
@pytest.mark.parametrize("n", [16, 1000, 4096])
def test_product_windows_equal_oracle(oracle_mod, name, n):
    assert np.array_equal(smd.window(name, n), oracle_mod.window(name, n))


def test_unknown_window_rejected():
    with pytest.raises(_lib.SMDError):
        smd.window("kaiser", 16)


def test_settings_roundtrip(tmp_path):
    s = SMDSettings(L=12, J2=0.12, JX=0.05, geom="triang", zlamb1=0.9, h=0.25, ntm=4096,
                    dtm=0.02, window="hann2", imp_ratio=0.05, NMeas=64000)
    s.write(str(tmp_path))
    r = SMDSettings.read(str(tmp_path))
    assert r == s
    assert s.j2_on and s.jx_on and s.disorder
    assert s.t_tag == "_T(0.10000)_J2(0.120)"


def test_settings_validation():
    with pytest.raises(SettingsError):
        SMDSettings(L=8, geom="triang").validate()
    with pytest.raises(SettingsError):
        SMDSettings(L=7).validate()
    with pytest.raises(SettingsError):
        SMDSettings(L=8, ntm=1024, dtm=0.01).validate()          # dwf = 0.61 > 0.1
    SMDSettings(L=8, ntm=1024, dtm=0.01).validate(check_dwf=False)
    with pytest.raises(SettingsError):
        SMDSettings(L=8, J2_delta=0.1).validate(check_dwf=False)


@pytest.mark.parametrize("N,ratio", [(64, 0.05), (2304, 0.05), (16384, 0.05), (100, 0.01),
                                     (50, 0.3)])
def test_impurity_count_follows_reference_loop(N, ratio):
    # explicit restatement of Codes_Folder/subrouts.cpp:3336-3350
    iNs = 1.0 / N
    mark, cnt = 1, 0
    for i in range(N):
        cnt += mark
        if (i + 2) * iNs > ratio:
            mark = 0
    assert smp.impurity_count(N, ratio) == cnt


@pytest.mark.parametrize("disorder", [False, True])
def test_sample_file_roundtrip(tmp_path, disorder):
    s = SMDSettings(L=8, J2=0.6, NMeas=3000, crSkip=1000,
                    imp_ratio=0.05 if disorder else 0.0)
    spins, imp = smp.make_samples(s, 6, "stripe", 0.2, 5)
    p = str(tmp_path / smp.sample_file_name(s))
    smp.write_sample_file(p, s, spins, imp)
    sp2, imp2 = smp.read_sample_file(p, s)
    assert np.array_equal(sp2, spins)
    for k in range(6):
        assert smp.field_norm(spins[k]) <= 1.0
    if disorder:
        assert imp2.shape == (6, s.N)
        assert np.array_equal(imp2[0], imp[0]) and np.array_equal(imp2[3], imp[1])
        assert int(imp[0].sum()) == smp.impurity_count(s.N, 0.05)
    else:
        assert imp2 is None


def test_qcrystal_qpoints_follow_the_direct_sum_order(oracle_mod):
    """The direct-sum q set of get_qct_SqData: index j Lsz + i, FFT order
    along both axes, dq = 8 pi / Lsz, scale 1 / sqrt(N)."""
    lat = smd.Lattice("Aamman", 14, 239, 14, 1, [8, 3, 8], np.zeros((239, 2)), None,
                      [np.zeros((239, z), np.int32) for z in (8, 3, 8)])
    q, sc = smd.qcrystal_qpoints(lat)
    qo, sco = oracle_mod.qct_qpoints(14, 239)
    assert np.array_equal(q, qo) and sc == sco
    dq = 8.0 * np.pi / 14
    assert np.allclose(q[1], (dq, 0.0)) and np.allclose(q[14], (0.0, dq))
    assert np.allclose(q[13], (-dq, 0.0)) and np.allclose(q[7], (-7 * dq, 0.0))


def test_qcrystal_settings_follow_the_reference_checks():
    """latSize is the site count, Lsz the even integer below its square root,
    and a quasi-crystal run needs PBC_OFF = 1 and qct_RemovePBC = 0
    (Codes_Folder/subrouts.cpp:1105-1114, smd_code.cpp:365-372)."""
    from classical_mc_and_smd_for_2d_heisenberg_models_b200.settings import SettingsError
    s = SMDSettings(geom="Aamman", L=1393, NMeas=2000)
    s.flags["qcrystal"] = 1
    s.flags["PBC_OFF"] = 1
    s.validate(check_dwf=False)
    assert (s.N, s.Lsz, s.G, s.zn) == (1393, 36, 36, (8, 3, 8))
    assert s.size_tag == "_AppxtSz(1393)"
    s.flags["qct_RemovePBC"] = 1
    with pytest.raises(SettingsError):
        s.validate(check_dwf=False)
    s.flags["qct_RemovePBC"] = 0
    s.flags["PBC_OFF"] = 0
    with pytest.raises(SettingsError):
        s.validate(check_dwf=False)
