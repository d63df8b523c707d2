"""Process-level drop-in for the SMD part of the reference's xSMD_run (Python
mirror of the C++ program csrc/xsmd.cpp, which also writes the text
spectra).

    python -m classical_mc_and_smd_for_2d_heisenberg_models_b200.xsmd WORKDIR
        [--device D] [--precision fp64|fp32] [--stride S] [--fix-every F]
        [--no-dwf-guard]

Reads what the reference's main program reads from WORKDIR: the five
settings files (Settings_CodeExec / MODEL / MC_SIM / SMD_SIM / Disorder,
Codes_Folder/subrouts.cpp:105-123, smd_code.cpp:497-539) and the MC sample
file outBin/MC_Bin_SpinField<tag>.bin (smd_code.cpp:997-1180; the temporal
window from outBin/winvec.bin when the window is "wread").  It runs every
sample through the CUDA path and writes, with the reference's names and
layouts:

  outBin/MC_Bin_SpecData<tag>.bin   the sample-averaged spectra, per q the
                                    ntm doubles of x, y, z, then the ntm
                                    doubles of the autocorrelation
                                    (smd_code.cpp:3613-3631; the reference's
                                    checkpoint format)
  outData/MC_Results/SpinSpin_Temporal_Corr<tag>.dat
                                    time and autocorrelation per record
                                    (smd_code.cpp:4019-4033)

Defaults are the reference's semantics: FP64, every step recorded (stride
1), energy correction every step.  Settings_B200.txt (optional: precision
stride fix_every, e.g. "fp32 4 16") or the flags select the precision form.
The dwf guard of smd_code.cpp:2120 applies unless --no-dwf-guard.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

from . import _lib, samples as smp, smd
from .settings import SMDSettings, SettingsError


def _fmt_sci(x: float, digits: int, width: int) -> str:
    """C++ `scientific << showpos << setprecision(digits) << setw(width)`."""
    return f"{x:+.{digits}e}".rjust(width)


def write_spec_bin(path: str, spec: np.ndarray, qss: np.ndarray) -> None:
    """spec [3][Q][ntm], qss [ntm] in the layout of smd_code.cpp:3613-3631."""
    if os.path.exists(path):
        os.remove(path)
    Q, ntm = spec.shape[1], spec.shape[2]
    body = np.ascontiguousarray(np.transpose(spec, (1, 0, 2))).reshape(Q * 3 * ntm)
    with open(path, "wb") as f:
        f.write(np.ascontiguousarray(body, np.float64).tobytes())
        f.write(np.ascontiguousarray(qss, np.float64).tobytes())


def read_spec_bin(path: str, Q: int, ntm: int):
    """Inverse of write_spec_bin: (spec [3][Q][ntm], qss [ntm])."""
    raw = np.fromfile(path, dtype=np.float64)
    if raw.size != (3 * Q + 1) * ntm:
        raise ValueError(f"{path}: {raw.size} doubles, expected {(3 * Q + 1) * ntm}")
    spec = raw[:3 * Q * ntm].reshape(Q, 3, ntm).transpose(1, 0, 2).copy()
    return spec, raw[3 * Q * ntm:].copy()


def write_corr_dat(path: str, dtm: float, qss: np.ndarray) -> None:
    """Time and autocorrelation per record, smd_code.cpp:4019-4033."""
    with open(path, "w") as f:
        for n, v in enumerate(qss):
            f.write(_fmt_sci(n * dtm, 8, 15) + "    " + _fmt_sci(float(v), 12, 22) + "\n")


def _window(s: SMDSettings, workdir: str) -> np.ndarray:
    if s.window == "wread":
        # the file's values rescaled by their maximum (smd_code.cpp:2828-2848)
        w = np.fromfile(os.path.join(workdir, "outBin", "winvec.bin"), dtype=np.float64)
        if w.size < s.ntm:
            raise SettingsError(f"winvec.bin holds {w.size} values, ntm = {s.ntm}")
        w = w[:s.ntm]
        return (1.0 / w.max()) * w
    return smd.window(s.window, s.ntm)


def _options(workdir: str, args) -> dict:
    o = {"precision": "fp64", "stride": 1, "fix_every": 1}
    p = os.path.join(workdir, "Settings_B200.txt")
    if os.path.exists(p):
        tok = open(p).read().split()
        o.update(precision=tok[0], stride=int(tok[1]), fix_every=int(tok[2]))
    for k in ("precision", "stride", "fix_every"):
        if getattr(args, k) is not None:
            o[k] = getattr(args, k)
    if o["precision"] not in ("fp64", "fp32"):
        raise SettingsError(f"precision {o['precision']!r}: fp64 or fp32")
    return o


def run(workdir: str, device: int = 0, precision=None, stride=None, fix_every=None,
        dwf_guard: bool = True) -> dict:
    ns = argparse.Namespace(precision=precision, stride=stride, fix_every=fix_every)
    s = SMDSettings.read(workdir)
    s.validate(check_dwf=dwf_guard)
    o = _options(workdir, ns)
    tag = s.t_tag
    spins, imp = smp.read_sample_file(os.path.join(workdir, "outBin", smp.sample_file_name(s)), s)
    win = _window(s, workdir)
    if s.qcrystal:
        # tables from outBin/ and the direct-sum q set of get_qct_SqData
        lat = smd.load_qcrystal(os.path.join(workdir, "outBin"), s.N, s.geom)
    else:
        lat = smd.build_lattice(s.geom, s.L)
    t0 = time.perf_counter()
    with smd.Context(device) as ctx:
        lid = ctx.lattice(s, lat)
        if s.qcrystal:
            q, sc = smd.qcrystal_qpoints(lat)
            qid = ctx.qset(lid, use_grid=False, qlist=q, list_scale=sc)
        else:
            qid = ctx.qset(lid, use_grid=True)
        prec = _lib.SMD_FP64 if o["precision"] == "fp64" else _lib.SMD_FP32
        # ntm records: ntm - 1 steps at stride 1, as the reference records
        # every step (subrouts.cpp:11734)
        n_rec = s.ntm if o["stride"] == 1 else (s.ntm - 1) // o["stride"] + 1
        r = ctx.run(lid, qid, spins, s.dtm, n_rec, stride=o["stride"], precision=prec,
                    fix_every=o["fix_every"], win=win[:n_rec],
                    imp=None if imp is None else np.ascontiguousarray(imp, np.int32),
                    want_final=False)
    wall = time.perf_counter() - t0
    bin_dir = os.path.join(workdir, "outBin")
    dat_dir = os.path.join(workdir, "outData", "MC_Results")
    os.makedirs(dat_dir, exist_ok=True)
    spec_path = os.path.join(bin_dir, "MC_Bin_SpecData" + tag + ".bin")
    corr_path = os.path.join(dat_dir, "SpinSpin_Temporal_Corr" + tag + ".dat")
    write_spec_bin(spec_path, r.spec, r.qss)
    write_corr_dat(corr_path, s.dtm * o["stride"], r.qss)
    return {"samples": int(spins.shape[0]), "N": s.N, "Q": int(r.spec.shape[1]), "records": n_rec,
            "precision": o["precision"], "stride": o["stride"], "fix_every": o["fix_every"],
            "site_steps": r.report["site_steps"], "wall_s": wall,
            "spec_file": spec_path, "corr_file": corr_path,
            "drift_max_per_site": r.report["drift_max"]}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="xsmd", description=__doc__.split("\n\n")[0])
    ap.add_argument("workdir")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--precision", choices=["fp64", "fp32"])
    ap.add_argument("--stride", type=int)
    ap.add_argument("--fix-every", dest="fix_every", type=int)
    ap.add_argument("--no-dwf-guard", action="store_true")
    a = ap.parse_args(argv)
    try:
        rep = run(a.workdir, a.device, a.precision, a.stride, a.fix_every, not a.no_dwf_guard)
    except (SettingsError, ValueError, OSError, _lib.SMDError) as e:
        print(f"xsmd: {e}", file=sys.stderr)
        return 1
    print(json.dumps(rep))
    return 0


if __name__ == "__main__":
    sys.exit(main())
