"""Process-level drop-in (xsmd): the reference's settings and sample files
in, its binary spectrum dump and autocorrelation file out."""
import os

import numpy as np
import pytest

from conftest import load_golden
from classical_mc_and_smd_for_2d_heisenberg_models_b200 import samples as smp, xsmd


def test_scientific_format_matches_the_reference_writer():
    # fmtDbleSci (Codes_Folder/aux_code.cpp:545-554): scientific, showpos,
    # setprecision(dg), setw(wd)
    assert xsmd._fmt_sci(0.01, 8, 15) == "+1.00000000e-02"
    assert xsmd._fmt_sci(0.0, 8, 15) == "+0.00000000e+00"
    assert xsmd._fmt_sci(1.0, 12, 22) == "   +1.000000000000e+00"
    assert xsmd._fmt_sci(-2.5e-7, 12, 22) == "   -2.500000000000e-07"


def test_spec_binary_layout_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    spec, qss = rng.random((3, 5, 7)), rng.random(7)
    p = str(tmp_path / "s.bin")
    xsmd.write_spec_bin(p, spec, qss)
    raw = np.fromfile(p)
    # per q: x, y, z rows of ntm, then the autocorrelation
    assert np.array_equal(raw[:7], spec[0, 0]) and np.array_equal(raw[7:14], spec[1, 0])
    assert np.array_equal(raw[14:21], spec[2, 0]) and np.array_equal(raw[-7:], qss)
    s2, q2 = xsmd.read_spec_bin(p, 5, 7)
    assert np.array_equal(s2, spec) and np.array_equal(q2, qss)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["spec_square", "spec_triang", "spec_lieb_disorder",
                                  "spec_qct239_open"])
def test_driver_reproduces_reference_outputs(tmp_path, name):
    """Settings and sample files written in the reference's formats, the
    window as outBin/winvec.bin: the driver's MC_Bin_SpecData equals the
    reference's sample average.  The reference rescales a read window by
    its maximum (Codes_Folder/smd_code.cpp:2828-2848), so the fixture's
    spectrum, computed with the raw window, scales by 1 / max^2."""
    s, d = load_golden(name)
    n = int(d["n"])
    import dataclasses
    s = dataclasses.replace(s, window="wread", NMeas=1000 * n, crSkip=1000)
    wd = str(tmp_path)
    s.write(wd)
    os.makedirs(os.path.join(wd, "outBin"), exist_ok=True)
    imp = None
    if "imp" in d:
        imp = np.asarray(d["imp"])[None]
    smp.write_sample_file(os.path.join(wd, "outBin", smp.sample_file_name(s)), s,
                          np.asarray(d["spins0"][:n]), imp)
    np.asarray(d["window"], np.float64).tofile(os.path.join(wd, "outBin", "winvec.bin"))
    if s.qcrystal:
        # the approximant's tables in the reference's binary layouts
        tag = s.size_tag
        np.asarray(d["rvec"], np.float64).tofile(os.path.join(wd, "outBin", f"sitesList{tag}.bin"))
        tab = np.concatenate([d["nb1"], d["nb2"], d["nbx"]], axis=1).astype(np.int32)
        tab.tofile(os.path.join(wd, "outBin", f"nborsList{tag}.bin"))
    rep = xsmd.run(wd, dwf_guard=False)
    Q = rep["Q"]
    spec, qss = xsmd.read_spec_bin(rep["spec_file"], Q, s.ntm)
    wmax = float(np.max(d["window"]))
    ref = d["spec_sum"] / n / (wmax * wmax)
    assert np.max(np.abs(spec - ref)) <= 1e-10 * np.max(np.abs(ref))
    assert np.max(np.abs(qss - d["qss_sum"] / n)) <= 1e-10
    lines = open(rep["corr_file"]).read().splitlines()
    assert len(lines) == s.ntm and lines[0].split()[1] == "+1.000000000000e+00"
