"""The C++ process-level drop-in (xsmd, built on the library's C ABI) against
the reference's own output stage.

The fixtures text_<case>.npz hold what the reference's code wrote for a
spectrum case (oracle/_ref/smd_ref_run --outputs, generated by
tests/golden/make_golden.py): MC_Bin_SpecData, the window files, the
autocorrelation file and every zz text file (centred slices every
ceil(npw / 10) bins, the KGMYG / YGMXG path and its cut).  With RecVd1 = 2
(the reference's getEvoData) xsmd reads that MC_Bin_SpecData instead of
integrating, so these checks need no GPU: its zz outputs, the
autocorrelation and the window form must equal the reference's byte for
byte.  The reference's xy, yz and tt text outputs are undefined (its quantum
correction never assigns yVal, Codes_Folder/smd_code.cpp:3662-3664); xsmd's
are checked for their defining relations instead.  The GPU test runs the
whole program, evolution included.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, golden_names, load_golden
from classical_mc_and_smd_for_2d_heisenberg_models_b200 import samples as smp
from classical_mc_and_smd_for_2d_heisenberg_models_b200.settings import SMDSettings

PKG = os.path.join(ROOT, "classical_mc_and_smd_for_2d_heisenberg_models_b200")
XSMD = os.path.join(PKG, "xsmd")


@pytest.fixture(scope="module")
def xsmd_bin():
    if not os.path.exists(XSMD):
        subprocess.run(["make", "-s", "-C", os.path.join(PKG, "csrc"), "../xsmd"], check=True)
    return XSMD


def _fixture(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    import json
    s = SMDSettings(**json.loads(str(z["settings"])))
    files = {str(n): z[f"f{i}"].tobytes() for i, n in enumerate(z["names"])}
    return s, files


def _resume_dir(tmp_path, s, files):
    import dataclasses
    s = dataclasses.replace(s, RecVd1=2)
    wd = str(tmp_path)
    s.write(wd)
    os.makedirs(os.path.join(wd, "outBin"), exist_ok=True)
    for k, v in files.items():
        if k.startswith("outBin/"):
            with open(os.path.join(wd, k), "wb") as f:
                f.write(v)
    return wd


def _prepass_file(k):
    return "MCSamples_DFT_" in k or "locFieldHist" in k


def _floats(text):
    return np.array([float(x) for x in text.split()])


@pytest.mark.parametrize("name", golden_names("text_"))
def test_resumed_outputs_equal_the_reference(tmp_path, xsmd_bin, name):
    s, files = _fixture(name)
    wd = _resume_dir(tmp_path, s, files)
    r = subprocess.run([xsmd_bin, wd, "--no-dwf-guard"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    compared = 0
    for k, ref in files.items():
        if not k.startswith("outData/") or _prepass_file(k):
            continue   # the pre-pass reads the sample file, which a resumed run has not
        got = open(os.path.join(wd, k), "rb").read()
        if "0WinSpec_" in k:
            # log10 of the window's power spectrum: round-off decides the
            # digits of the near-zero bins, so compare where it is resolved
            a, b = _floats(got.decode()).reshape(-1, 2), _floats(ref.decode()).reshape(-1, 2)
            assert np.array_equal(a[:, 0], b[:, 0])
            ok = b[:, 1] > -10.0
            assert np.allclose(a[ok, 1], b[ok, 1], atol=1e-5), k
        else:
            assert got == ref, k
        compared += 1
    assert compared >= 10


@pytest.mark.parametrize("name", ["text_spec_triang", "text_spec_square"])
def test_undefined_reference_components_follow_their_definitions(tmp_path, xsmd_bin, name):
    """xy = (x + y) / 2, yz = (y + z) / 2, tt = (x + y + z) / 3 of the
    corrected spectra: on the path, tt = (2 xy + zz) / 3 exactly when
    x = y, and every file has the zz file's rows and wavevectors."""
    s, files = _fixture(name)
    wd = _resume_dir(tmp_path, s, files)
    assert subprocess.run([xsmd_bin, wd, "--no-dwf-guard"], capture_output=True).returncode == 0
    res = os.path.join(wd, "outData", "RK_Results")
    zz = [f for f in os.listdir(res) if "wDepn_DFT_zzSpec" in f and "Cut" not in f][0]
    cols = {}
    for c in ("xy", "yz", "zz", "tt"):
        cols[c] = _floats(open(os.path.join(res, zz.replace("zz", c))).read()).reshape(-1, 3)
        assert np.array_equal(cols[c][:, :2], cols["xy"][:, :2])
        assert np.isfinite(cols[c]).all()
    x_plus_y = 2.0 * cols["xy"][:, 2]
    z = cols["zz"][:, 2]
    y = 2.0 * cols["yz"][:, 2] - z
    x = x_plus_y - y
    assert np.allclose(cols["tt"][:, 2], (x + y + z) / 3.0, rtol=1e-9, atol=1e-12)


def test_resume_refuses_a_missing_or_wrong_size_spectrum(tmp_path, xsmd_bin):
    s, files = _fixture("text_spec_square")
    wd = _resume_dir(tmp_path, s, files)
    for k in files:
        if k.startswith("outBin/"):
            p = os.path.join(wd, k)
            open(p, "ab").write(b"\0" * 8)
    r = subprocess.run([xsmd_bin, wd, "--no-dwf-guard"], capture_output=True, text=True)
    assert r.returncode == 1 and "no valid data" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["spec_square", "spec_triang", "spec_lieb_disorder"])
def test_full_run_reproduces_reference_outputs(tmp_path, xsmd_bin, name):
    """Settings and sample files in, pre-pass and evolution on the GPU:
    MC_Bin_SpecData within 1e-10 of the reference's, the zz path file within
    1e-9 (relative) of the reference's output stage, the local-field
    histogram identical and the static structure factor within 1e-9."""
    s, d = load_golden(name)
    st, files = _fixture("text_" + name)
    wd = str(tmp_path)
    st.write(wd)
    n = int(d["n"])
    spins = d["spins0"][:n]
    imp = None
    if "imp" in d:
        imp = np.tile(d["imp"], (max(1, n // st.pack_size), 1))
    smp.write_sample_file(os.path.join(wd, "outBin", smp.sample_file_name(st)), st, spins, imp)
    r = subprocess.run([xsmd_bin, wd, "--no-dwf-guard"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for k, ref in files.items():
        got = open(os.path.join(wd, k), "rb").read()
        if k.startswith("outBin/"):
            a, b = np.frombuffer(got, np.float64), np.frombuffer(ref, np.float64)
            assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(b)), k
        elif "wDepn_DFT_zzSpec" in k:
            a, b = _floats(got.decode()), _floats(ref.decode())
            assert np.allclose(a, b, rtol=1e-9, atol=1e-12 * np.abs(b).max()), k
        elif "locFieldHist" in k:
            assert got == ref, k
        elif "MCSamples_DFT_" in k:
            # printed with 6 digits: equal up to the last digit's rounding
            ga = [x for x in got.decode().split() if x != "NaN"]
            ra = [x for x in ref.decode().split() if x != "NaN"]
            assert got.decode().count("NaN") == ref.decode().count("NaN"), k
            assert np.allclose(np.array(ga, float), np.array(ra, float), rtol=2e-5, atol=1e-14), k


@pytest.mark.gpu
def test_quasicrystal_run_reproduces_the_reference_spectrum(tmp_path, xsmd_bin):
    """qcrystal = 1: the 239-site approximant's tables in outBin/ (the
    reference's binary layouts), the direct-sum q set of get_qct_SqData:
    MC_Bin_SpecData within 1e-10 of the reference's sample average (the read
    window rescaled by its maximum, as the reference does) and the
    autocorrelation file written."""
    s, d = load_golden("spec_qct239_open")
    import dataclasses
    n = int(d["n"])
    s = dataclasses.replace(s, window="wread", NMeas=1000 * max(2, n), crSkip=1000)
    wd = str(tmp_path)
    s.write(wd)
    ob = os.path.join(wd, "outBin")
    os.makedirs(ob, exist_ok=True)
    smp.write_sample_file(os.path.join(ob, smp.sample_file_name(s)), s, np.asarray(d["spins0"][:n]), None)
    np.asarray(d["window"], np.float64).tofile(os.path.join(ob, "winvec.bin"))
    tag = s.size_tag
    np.asarray(d["rvec"], np.float64).tofile(os.path.join(ob, f"sitesList{tag}.bin"))
    np.concatenate([d["nb1"], d["nb2"], d["nbx"]], axis=1).astype(np.int32).tofile(
        os.path.join(ob, f"nborsList{tag}.bin"))
    r = subprocess.run([xsmd_bin, wd, "--no-dwf-guard"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    Q, ntm = s.G * s.G, s.ntm
    raw = np.fromfile(os.path.join(ob, "MC_Bin_SpecData" + s.t_tag + ".bin"))
    spec = raw[: 3 * Q * ntm].reshape(Q, 3, ntm).transpose(1, 0, 2)
    wmax = float(np.max(d["window"]))
    ref = d["spec_sum"] / n / (wmax * wmax)
    assert np.max(np.abs(spec - ref)) <= 1e-10 * np.max(np.abs(ref))
    assert np.max(np.abs(raw[3 * Q * ntm:] - d["qss_sum"] / n)) <= 1e-10
    corr = os.path.join(wd, "outData", "MC_Results", "SpinSpin_Temporal_Corr" + s.t_tag + ".dat")
    assert len(open(corr).read().splitlines()) == ntm


def test_quasicrystal_settings_are_checked_as_the_reference_does(tmp_path, xsmd_bin):
    """A quasi-crystal directory with PBC_OFF = 0 is refused (smd_code.cpp:
    365-372), before any device work."""
    s = SMDSettings(geom="Aamman", L=239, NMeas=2000, ntm=16)
    s.flags["qcrystal"] = 1
    s.write(str(tmp_path))
    r = subprocess.run([xsmd_bin, str(tmp_path), "--no-dwf-guard"], capture_output=True, text=True)
    assert r.returncode == 1 and "PBC_OFF" in r.stderr
