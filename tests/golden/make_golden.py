"""Generate the golden fixtures of tests/golden/ from the reference itself.

The reference ships no test vectors for its SMD path, so the fixtures are
produced by running the reference's own code: oracle/_ref/smd_ref_run is
Codes_Folder/subrouts.cpp compiled from its sources (see oracle/Makefile),
driven through the same calls its main program makes.  Inputs are seeded
synthetic samples in the reference's sample-file format.

Every case stores: the settings, the reference's lattice tables (positions,
grid map, neighbour tables, bond list), the input samples and impurity map,
the reference's final spins after ntm - 1 RK steps, and the reference's sums
over samples of |S(q,w)|^2 and of the autocorrelation.

Spectrum cases also get text_<name>.npz: the reference's output stage
(sample averages, window files, quantum-corrected zz slices, path and cut
files, autocorrelation) through smd_ref_run --outputs.

Run from the repository root (needs the reference sources at build time):
    make -C oracle ref && python tests/golden/make_golden.py [--text | --qct | --mc]
"""
from __future__ import annotations

import dataclasses
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from classical_mc_and_smd_for_2d_heisenberg_models_b200 import samples as smp  # noqa: E402
from classical_mc_and_smd_for_2d_heisenberg_models_b200.settings import SMDSettings  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# (name, settings overrides, ntm, samples, ordered state, tilt sigma, seed)
CASES = [
    # 200-step per-spin trajectories, the north-star parity window
    ("traj_square_j1j2", dict(geom="square", L=8, J2=0.6, dtm=0.01), 201, 2, "stripe", 0.2, 11),
    ("traj_triang_j1j2", dict(geom="triang", L=6, J2=0.12, dtm=0.02), 201, 2, "q120", 0.15, 12),
    ("traj_square_xxz_h_vac", dict(geom="square", L=8, J2=0.55, JX=0.1, zlamb1=0.9, zlamb2=0.9,
                                   h=0.3, imp_ratio=0.05, dtm=0.01), 201, 2, "stripe", 0.1, 13),
    ("traj_kagome", dict(geom="kagome", L=6, J2=0.3, JX=0.1, dtm=0.01), 201, 1, "ferro", 0.6, 14),
    ("traj_hexagn", dict(geom="hexagn", L=6, J2=0.2, JX=0.05, dtm=0.01), 201, 1, "ferro", 0.6, 15),
    ("traj_lieb_delta", dict(geom="lieb", L=6, J2=0.4, J2_delta=0.15, JX=0.05, dtm=0.01), 201, 1,
     "ferro", 0.6, 16),
    # short spectra over the full grid with a window
    ("spec_square", dict(geom="square", L=4, J2=0.6, dtm=0.02, window="hann1"), 16, 2, "stripe",
     0.3, 21),
    ("spec_triang", dict(geom="triang", L=6, J2=0.12, h=0.2, dtm=0.02, window="black"), 16, 2,
     "q120", 0.3, 22),
    ("spec_hexagn", dict(geom="hexagn", L=6, J2=0.2, dtm=0.02, window="gauss"), 16, 2, "ferro",
     0.7, 23),
    ("spec_kagome", dict(geom="kagome", L=6, J2=0.3, JX=0.1, dtm=0.02, window="flatw"), 16, 2,
     "ferro", 0.7, 24),
    ("spec_lieb_disorder", dict(geom="lieb", L=4, J2=0.4, imp_ratio=0.1, J1ic=0.5, J2ic=0.2,
                                J1ii=0.3, dtm=0.02, window="ntall"), 16, 2, "ferro", 0.7, 25),
]


# Quasi-crystal cases (qcrystal = 1): the reference's Ammann-Beenker
# approximant tables from QCrystal_Data/ copied into the work directory's
# outBin/, samples tilted from one of the approximant's ordered states.
# (name, table folder, N, settings overrides, ntm, samples, state, sigma, seed)
QCT_DIR = "/root/reference/QCrystal_Data"
QCT_CASES = [
    ("traj_qct239_pbc", "with_PBC/239", 239, dict(J2=0.3, dtm=0.01), 201, 2, "stateNeel0", 0.2, 31),
    ("traj_qct239_open_xxz_h", "no_PBC/239", 239, dict(J2=0.25, JX=0.1, zlamb1=0.9, zlamb2=0.9,
                                                        h=0.2, dtm=0.01), 201, 1, "stateStrp2", 0.2, 33),
    ("spec_qct239_open", "no_PBC/239", 239, dict(J2=0.2, JX=0.1, dtm=0.02, window="hann1"), 16, 2,
     "stateStrp1", 0.3, 32),
    # more sites than one CTA holds: the lattice is split over a cluster
    ("traj_qct1393_pbc_jx", "with_PBC/1393", 1393, dict(J2=0.3, JX=0.1, dtm=0.01), 101, 1,
     "stateStrp3", 0.2, 34),
]


def run_qct_case(name, folder, N, over, ntm, n, state, sigma, seed, workroot):
    import shutil
    s = SMDSettings(geom="Aamman", L=N, ntm=ntm, NMeas=1000 * max(n, 2), crSkip=1000, **over)
    s.flags["qcrystal"] = 1
    s.flags["PBC_OFF"] = 1
    s.validate(check_dwf=False)
    wd = os.path.join(workroot, name)
    s.write(wd)
    os.makedirs(os.path.join(wd, "outBin"), exist_ok=True)
    src = os.path.join(QCT_DIR, folder)
    tag = s.size_tag
    for f in (f"sitesList{tag}.bin", f"nborsList{tag}.bin"):
        shutil.copy(os.path.join(src, f), os.path.join(wd, "outBin", f))
    base = np.fromfile(os.path.join(src, f"{state}{tag}.bin")).reshape(N, 3)
    total = max(n, 2)
    spins, _ = smp.make_samples(s, total, "ferro", sigma, seed, base=base)
    path = os.path.join(wd, "samples.bin")
    smp.write_sample_file(path, s, spins, None)
    info = O.run_reference(wd, path, 0, n, dump_final=True, dwf_guard=False)
    lat = O.read_ref_lattice(wd)
    spec, qss = O.read_ref_spec(wd, s.G * s.G, ntm)
    final = O.read_ref_final(wd, n, s.N)
    win = O.window(s.window, ntm) if s.window != "nowin" else np.ones(ntm)
    out = dict(
        settings=json.dumps(dataclasses.asdict(s)),
        spins0=spins[:n], final=final, spec_sum=spec, qss_sum=qss,
        rvec=lat["rvec"], grid_map=lat["grid_map"], nb1=lat["nbrs"][0], nb2=lat["nbrs"][1],
        nbx=lat["nbrs"][2], bonds=lat["bonds"], nbonds=np.array(lat["nbonds"], np.int32),
        window=win, n=np.int32(n), qct_table=np.array(folder),
    )
    if name.startswith("traj_"):
        out.pop("spec_sum")
        out.pop("qss_sum")
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    return info


# Monte Carlo cases: the reference's MC stage (overrelaxation + heat-bath
# sweeps, one rank, no tempering) through smd_ref_run --mc, RUNS independent
# runs per temperature (dSFMT and rand() seeded per run) of THERM + MEAS MC
# steps; a fixture keeps every run's mean energy per site and, on disordered
# lattices, every run's impurity map.
# (name, settings overrides, temperatures, runs, therm, meas, qct table)
MC_CASES = [
    ("mc_square_j1j2", dict(geom="square", L=8, J2=0.3), (0.3, 0.8), 8, 1000, 8000, None),
    ("mc_triang_h_vac", dict(geom="triang", L=6, J2=0.1, h=0.3, imp_ratio=0.1, J1ic=0.5, J2ic=0.2),
     (0.4,), 8, 1000, 8000, None),
    ("mc_kagome_xxz", dict(geom="kagome", L=6, J2=0.2, zlamb1=0.8, zlamb2=0.8), (0.25,), 8, 1000, 8000,
     None),
    ("mc_qct239", dict(geom="Aamman", L=239, J2=0.3), (0.5,), 8, 1000, 8000, "with_PBC/239"),
]


def run_mc_case(name, over, temps, runs, therm, meas, table, workroot):
    import shutil
    import subprocess
    out = dict(temps=np.array(temps), runs=np.int32(runs), therm=np.int32(therm),
               meas=np.int32(meas))
    e_site, imps = [], []
    for ti, T in enumerate(temps):
        s = SMDSettings(ntm=16, NMeas=2000, crSkip=1000, T1=T, T2=T, **over)
        if table:
            s.flags["qcrystal"] = 1
            s.flags["PBC_OFF"] = 1
        wd = os.path.join(workroot, f"{name}_{ti}")
        s.write(wd)
        if table:
            os.makedirs(os.path.join(wd, "outBin"), exist_ok=True)
            for f in (f"sitesList{s.size_tag}.bin", f"nborsList{s.size_tag}.bin"):
                shutil.copy(os.path.join(QCT_DIR, table, f), os.path.join(wd, "outBin", f))
        row, irow = [], []
        for run in range(runs):
            r = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "smd_ref_run"), wd, "none",
                                str(1000 * ti + run + 1), "0", "--no-dwf-guard", "--mc", str(therm),
                                str(meas)], capture_output=True, text=True)
            if r.returncode:
                raise RuntimeError(r.stderr)
            row.append(json.loads(r.stdout.strip().splitlines()[-1])["e_site"])
            if s.disorder:
                irow.append(np.fromfile(os.path.join(wd, "ref_imp.bin"), dtype=np.int32))
        e_site.append(row)
        if irow:
            imps.append(np.stack(irow))
        if ti == 0:
            out["settings"] = json.dumps(dataclasses.asdict(s))
            if table:
                lat = O.read_ref_lattice(wd)
                out.update(rvec=lat["rvec"], nb1=lat["nbrs"][0], nb2=lat["nbrs"][1],
                           nbx=lat["nbrs"][2])
    out["e_site"] = np.array(e_site)
    if imps:
        out["imp"] = np.stack(imps).astype(np.int8)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    e = out["e_site"]
    return [(float(m), float(sd)) for m, sd in zip(e.mean(1), e.std(1, ddof=1) / np.sqrt(runs))]


def run_case(name, over, ntm, n, kind, sigma, seed, workroot):
    s = SMDSettings(ntm=ntm, NMeas=1000 * max(n, 2), crSkip=1000, **over)
    s.validate(check_dwf=False)
    wd = os.path.join(workroot, name)
    s.write(wd)
    pack = s.pack_size
    total = n if not s.disorder else pack * ((n + pack - 1) // pack)
    if not s.disorder and total not in (1,) and total % pack:
        total = pack * ((total + pack - 1) // pack)
    spins, imp = smp.make_samples(s, total, kind, sigma, seed)
    path = os.path.join(wd, "samples.bin")
    smp.write_sample_file(path, s, spins, imp)
    info = O.run_reference(wd, path, 0, n, dump_final=True, dwf_guard=False)
    lat = O.read_ref_lattice(wd)
    spec, qss = O.read_ref_spec(wd, s.G * s.G, ntm)
    final = O.read_ref_final(wd, n, s.N)
    win = O.window(s.window, ntm) if s.window != "nowin" else np.ones(ntm)
    out = dict(
        settings=json.dumps(dataclasses.asdict(s)),
        spins0=spins[:n], final=final, spec_sum=spec, qss_sum=qss,
        rvec=lat["rvec"], grid_map=lat["grid_map"], nb1=lat["nbrs"][0], nb2=lat["nbrs"][1],
        nbx=lat["nbrs"][2], bonds=lat["bonds"], nbonds=np.array(lat["nbonds"], np.int32),
        window=win, n=np.int32(n),
    )
    if imp is not None:
        out["imp"] = imp[0]
    if name.startswith("traj_"):
        # trajectories keep only the final spins; the spectrum is not needed
        out.pop("spec_sum")
        out.pop("qss_sum")
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    return info


def run_text_case(name, over, ntm, n, kind, sigma, seed, workroot):
    """The reference's output stage on a spectrum case (smd_ref_run
    --outputs --prepass): its static pre-pass records (MCSamples_DFT_*,
    locFieldHist), MC_Bin_SpecData, window files, autocorrelation and every
    zz text file (slices, path, cut), stored as text_<name>.npz."""
    import subprocess
    s = SMDSettings(ntm=ntm, NMeas=1000 * max(n, 2), crSkip=1000, **over)
    wd = os.path.join(workroot, "text_" + name)
    s.write(wd)
    pack = s.pack_size
    total = n if not s.disorder else pack * ((n + pack - 1) // pack)
    if not s.disorder and total not in (1,) and total % pack:
        total = pack * ((total + pack - 1) // pack)
    spins, imp = smp.make_samples(s, total, kind, sigma, seed)
    path = os.path.join(wd, "samples.bin")
    smp.write_sample_file(path, s, spins, imp)
    r = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "smd_ref_run"), wd, path, "0", str(n),
                        "--no-dwf-guard", "--outputs", "--prepass"], capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(r.stderr)
    files = {}
    for sub in ("outData", "outBin"):
        for root, _, names in os.walk(os.path.join(wd, sub)):
            for f in names:
                if f == "nborsList.bin":
                    continue
                rel = os.path.relpath(os.path.join(root, f), wd)
                files[rel] = open(os.path.join(root, f), "rb").read()
    np.savez_compressed(os.path.join(HERE, f"text_{name}.npz"),
                        settings=json.dumps(dataclasses.asdict(s)),
                        names=np.array(sorted(files)),
                        **{f"f{i}": np.frombuffer(files[k], np.uint8) for i, k in enumerate(sorted(files))})
    return len(files)


def main():
    if not O.reference_available():
        raise SystemExit("oracle/_ref/smd_ref_run is missing: run `make -C oracle ref` first")
    text_only = "--text" in sys.argv
    qct_only = "--qct" in sys.argv
    if "--mc" in sys.argv:
        with tempfile.TemporaryDirectory() as tmp:
            for c in MC_CASES:
                print(c[0], run_mc_case(*c, tmp))
        return
    with tempfile.TemporaryDirectory() as tmp:
        if not text_only:
            for c in QCT_CASES:
                print(c[0], run_qct_case(*c, tmp))
        if qct_only:
            return
        for c in CASES:
            if not text_only:
                info = run_case(*c, tmp)
                print(c[0], info)
            if c[0].startswith("spec_"):
                print("text", c[0], run_text_case(*c, tmp), "files")


if __name__ == "__main__":
    main()
