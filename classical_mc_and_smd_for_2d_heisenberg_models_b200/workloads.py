"""Synthetic SMD workloads with the shapes of the benchmark configurations.

There is no public data set for this path: seeded synthetic samples in the
reference's sample-file format stand in for MC output (ordered states with
Gaussian tangent tilts).  Every workload is a settings object, a sample
count, the ordered state and tilt, the record stride and length, the
precision form, and the q points.

  c1  square L=16 (N=256), J1=1 J2=0.6, 8 samples, stripe +x with 0.2 rad
      tilts, FP64 plain, dt=0.01, stride 4, 1024 records (512 positive
      frequencies), full 16 x 16 grid
  c2  triangular L=48 (N=2304), J2=0.12, 64 samples, 120-degree state with
      0.15 rad tilts, FP32 precision form, dt=0.02, stride 4, 4096 records
      (2048 positive frequencies), FP64 correction every 16 steps,
      48 x 48 grid + 512-point Gamma-K-M-Gamma path
  c3  batch of seven lattices of uneven N (square L=24..64, kagome 24,
      honeycomb 30, Lieb 32), 5% vacancies, 256 samples, relaxed random
      states, FP32, 8192 steps, 4096 random first-BZ q per lattice
  c4  square L=128 (N=16384), J2=0.55 J3=0.1 lambda=0.9 h=0.3, 5% vacancies,
      512 samples, stripe with 0.1 rad tilts, FP32, dt=0.01, stride 8,
      4096 records, 128 x 128 grid + 1024-point path
  c5  serving stream (c5_stream): five geometries, N log-uniform in
      [256, 16384], 16-256 samples, 2^12-2^15 steps
The number of RK steps of a job is (records - 1) * stride.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

from ._lib import SMD_FP32, SMD_FP64
from .settings import SMDSettings


@dataclasses.dataclass
class Workload:
    name: str
    settings: SMDSettings
    n_samples: int
    state: str
    sigma: float
    stride: int
    n_rec: int
    precision: int
    fix_every: int
    qpath_points: int
    seed: int
    window: str = "hann1"

    @property
    def steps(self) -> int:
        return (self.n_rec - 1) * self.stride

    def describe(self) -> str:
        s = self.settings
        return (f"{self.name}: {s.geom} L={s.L} N={s.N}, J2={s.J2} JX={s.JX} h={s.h} "
                f"vac={s.imp_ratio}, {self.n_samples} samples, {self.steps} RK4 steps "
                f"(stride {self.stride}, {self.n_rec} records), "
                f"{'FP64 plain' if self.precision == SMD_FP64 else 'FP32 precision form'}, "
                f"{s.G}x{s.G} grid + {self.qpath_points}-point path")


def path_points(geom: str, n: int) -> np.ndarray:
    """n points along a closed high-symmetry path, uniform in arc length.

    C3 lattices: Gamma -> K -> M -> Gamma with K = (4 pi / 3, 0) (the
    reference's Qvec0, Codes_Folder/subrouts.cpp:523-530) and M = (pi, pi/sqrt3);
    square-like lattices: Gamma -> X -> M -> Gamma with X = (pi, 0), M = (pi, pi).
    """
    if geom in ("square", "lieb"):
        corners = [(0.0, 0.0), (math.pi, 0.0), (math.pi, math.pi), (0.0, 0.0)]
    else:
        corners = [(0.0, 0.0), (4.0 * math.pi / 3.0, 0.0),
                   (math.pi, math.pi / math.sqrt(3.0)), (0.0, 0.0)]
    c = np.array(corners)
    seg = np.linalg.norm(np.diff(c, axis=0), axis=1)
    total = seg.sum()
    t = np.arange(n) * total / n
    out = np.zeros((n, 2))
    start = np.concatenate([[0.0], np.cumsum(seg)])
    for k in range(n):
        s = min(np.searchsorted(start, t[k], side="right") - 1, len(seg) - 1)
        f = (t[k] - start[s]) / seg[s]
        out[k] = c[s] + f * (c[s + 1] - c[s])
    return out


def c1() -> Workload:
    s = SMDSettings(geom="square", L=16, J1=1.0, J2=0.6, dtm=0.01, ntm=1024, NMeas=8000)
    return Workload("c1", s, 8, "stripe", 0.2, 4, 1024, SMD_FP64, 1, 0, 0x5eed01)


def c2(n_samples: int = 64) -> Workload:
    s = SMDSettings(geom="triang", L=48, J1=1.0, J2=0.12, dtm=0.02, ntm=4096,
                    NMeas=1000 * max(2, n_samples))
    return Workload("c2", s, n_samples, "q120", 0.15, 4, 4096, SMD_FP32, 16, 512, 0x5eed02)


def c4(n_samples: int = 512) -> Workload:
    s = SMDSettings(geom="square", L=128, J1=1.0, J2=0.55, JX=0.1, zlamb1=0.9, zlamb2=0.9,
                    h=0.3, imp_ratio=0.05, dtm=0.01, ntm=4096, NMeas=1000 * n_samples,
                    outTag="Htag")
    return Workload("c4", s, n_samples, "stripe", 0.1, 8, 4096, SMD_FP32, 16, 1024, 0x5eed04)


@dataclasses.dataclass
class BatchWorkload:
    """Several lattices run as one batch (smd_batch_*): one Workload per
    member, all with the same dt, records, stride and precision form."""
    name: str
    members: list
    n_q: int

    @property
    def steps(self) -> int:
        return self.members[0].steps

    def describe(self) -> str:
        parts = [f"{w.settings.geom} L={w.settings.L} (N={w.settings.N}, J2={w.settings.J2:.3f}, "
                 f"{w.n_samples} samples)" for w in self.members]
        m0 = self.members[0]
        return (f"{self.name}: batch of {len(self.members)} lattices [" + "; ".join(parts) +
                f"], 5% vacancies each, {sum(w.n_samples for w in self.members)} samples, "
                f"{m0.steps} RK4 steps (stride {m0.stride}, {m0.n_rec} records), "
                f"{'FP64 plain' if m0.precision == SMD_FP64 else 'FP32 precision form'}, "
                f"{self.n_q} random first-BZ q per lattice")


def bz_points(lat, n: int, seed: int) -> np.ndarray:
    """n points drawn uniformly in the first Brillouin zone of the lattice's
    Bravais lattice (the Wigner-Seitz cell of its reciprocal lattice), in
    the frame of the lattice's grid positions."""
    g1, g2 = lat.grid_basis()
    b1, b2 = g1 * lat.G / lat.grid_fac, g2 * lat.G / lat.grid_fac   # reciprocal of the Bravais cell
    rng = np.random.default_rng(seed)
    u = rng.uniform(0.0, 1.0, size=(n, 2))
    q = u[:, :1] * b1 + u[:, 1:] * b2
    best = q.copy()
    for n1 in (-2, -1, 0, 1, 2):
        for n2 in (-2, -1, 0, 1, 2):
            c = q - (n1 * b1 + n2 * b2)
            better = np.linalg.norm(c, axis=1) < np.linalg.norm(best, axis=1)
            best[better] = c[better]
    return best


def relaxed_samples(s: SMDSettings, lat, n_samples: int, sweeps: int, sigma: float, seed: int):
    """Random unit vectors relaxed toward a ground state by `sweeps` damped
    local-field alignment steps S_i <- normalise(S_i - eta h_i) (vectorised
    over sites and samples, FP64), then tilted by Gaussian tangent vectors of
    width sigma.  Vacancies feel no exchange field and keep their random
    spin.  Returns (spins [n][N][3], imp [n][N] or None)."""
    from . import samples as smp
    rng = np.random.default_rng(seed)
    N = lat.N
    S = rng.normal(size=(n_samples, N, 3))
    S /= np.linalg.norm(S, axis=2, keepdims=True)
    imp = None
    if s.disorder:
        imp = np.stack([smp.impurity_map(N, s.imp_ratio, rng) for _ in range(n_samples)])
    J = [s.J1, s.J2, s.JX]
    on = [True, s.j2_on, s.jx_on]
    lam = np.array(s.lambdas())
    mask = None if imp is None else (1.0 - imp)[:, :, None]
    eta = 0.5 / max(1e-12, sum(abs(J[k]) * lat.zn[k] for k in range(3) if on[k]))
    for _ in range(sweeps):
        Sm = S if mask is None else S * mask
        h = np.zeros_like(S)
        for k in range(3):
            if not on[k] or lat.zn[k] == 0:
                continue
            nb = lat.nbrs[k]
            for e in range(lat.zn[k]):
                j = nb[:, e]
                ok = (j >= 0)[None, :, None]
                h += J[k] * lam[k][None, None, :] * np.where(ok, Sm[:, np.clip(j, 0, None), :], 0.0)
        if mask is not None:
            h *= mask
        h[:, :, 2] -= s.h
        S = S - eta * h
        S /= np.linalg.norm(S, axis=2, keepdims=True)
    out = np.stack([smp.tilt(S[k], sigma, rng) for k in range(n_samples)])
    return out, imp


def c3(n_samples: int = 256) -> BatchWorkload:
    """Batched uneven mix: square L in {24, 32, 48, 64}, kagome L=24
    (N=1728), honeycomb L=30 (N=1800; the reference's honeycomb needs L a
    multiple of 6, so L=32 is not buildable) and Lieb L=32 (N=2048: the
    reference's Lieb cell has 2 sites, not 3), 5% vacancies each, J1=1, J2
    drawn in [0, 0.8] per lattice, lambda=1; the samples split evenly over
    the seven lattices; 8192 RK steps (2048 records at stride 4) in the FP32
    form with FP64 correction every 16 steps; 4096 random first-BZ q per
    lattice."""
    rng = np.random.default_rng(0x5eed03)
    lats = [("square", 24), ("square", 32), ("square", 48), ("square", 64), ("kagome", 24),
            ("hexagn", 30), ("lieb", 32)]
    per = [n_samples // len(lats) + (1 if k < n_samples % len(lats) else 0) for k in range(len(lats))]
    members = []
    for k, ((geom, L), ns) in enumerate(zip(lats, per)):
        J2 = float(rng.uniform(0.0, 0.8))
        s = SMDSettings(geom=geom, L=L, J1=1.0, J2=J2, imp_ratio=0.05, dtm=0.01, ntm=2048,
                        NMeas=1000 * ns)
        members.append(Workload(f"c3_{geom}{L}", s, ns, "relaxed", 0.1, 4, 2048, SMD_FP32, 16, 0,
                                0x5eed03 + 17 * k))
    return BatchWorkload("c3", members, 4096)


WORKLOADS = {"c1": c1, "c2": c2, "c4": c4}

C5_GEOMS = ("square", "triang", "hexagn", "kagome", "lieb")


def _valid_L(geom: str, n_target: float, n_max: int) -> Optional[int]:
    """The L whose site count is nearest n_target (log scale) among the sizes
    the reference's lattice builders accept, N <= n_max."""
    from .smd import geometry_info
    from ._lib import SMDError
    best, best_d = None, None
    for L in range(2, 200):
        try:
            N = geometry_info(geom, L)[0]
        except SMDError:
            continue
        if N > n_max:
            break
        d = abs(math.log(N / n_target))
        if best_d is None or d < best_d:
            best, best_d = L, d
    return best


def c5_stream(n_jobs: int, seed: int, n_min: int = 256, n_max: int = 16384,
              samples=(16, 256), log2_steps=(12, 15), n_rec: int = 1024):
    """Jobs of the serving workload: lattice drawn uniformly from the five
    crystal types, N log-uniform in [n_min, n_max] snapped to a valid L,
    J1 = 1, J2 in [0, 0.8], JX in [0, 0.2], lambda in [0.8, 1.0], h in
    [0, 0.5], 0-10 % vacancies, 16-256 samples, 2^12-2^15 RK steps
    (log-uniform) recorded at the stride that gives n_rec records, seeded
    ordered states with Gaussian tilts, grid q, FP32 form."""
    rng = np.random.default_rng(seed)
    jobs = []
    states = {"square": "stripe", "triang": "q120"}
    while len(jobs) < n_jobs:
        geom = C5_GEOMS[rng.integers(len(C5_GEOMS))]
        L = _valid_L(geom, math.exp(rng.uniform(math.log(n_min), math.log(n_max))), n_max)
        if L is None:
            continue
        lam = float(rng.uniform(0.8, 1.0))
        steps = int(round(2.0 ** rng.uniform(log2_steps[0], log2_steps[1])))
        stride = max(1, steps // n_rec)
        s = SMDSettings(geom=geom, L=L, J1=1.0, J2=float(rng.uniform(0.0, 0.8)),
                        JX=float(rng.uniform(0.0, 0.2)), zlamb1=lam, zlamb2=lam,
                        h=float(rng.uniform(0.0, 0.5)), imp_ratio=float(rng.uniform(0.0, 0.1)),
                        dtm=0.01, ntm=n_rec)
        n = int(rng.integers(samples[0], samples[1] + 1))
        s = dataclasses.replace(s, NMeas=1000 * n)
        w = Workload(f"c5_{len(jobs)}", s, n, states.get(geom, "ferro"), 0.1, stride,
                     n_rec, SMD_FP32, 16, 0, seed + 101 * len(jobs))
        jobs.append(w)
    return jobs


def make_inputs(w: Workload, rank: int = 0, lat=None):
    """Samples (and per-sample impurity maps) for one rank."""
    from . import samples as smp
    if w.state == "relaxed":
        if lat is None:
            from .smd import build_lattice
            lat = build_lattice(w.settings.geom, w.settings.L)
        spins, imp = relaxed_samples(w.settings, lat, w.n_samples, 200, w.sigma, w.seed + 7919 * rank)
        return spins, (None if imp is None else imp.astype(np.int32))
    spins, imp = smp.make_samples(w.settings, w.n_samples, w.state, w.sigma, w.seed + 7919 * rank)
    imp_per_sample = None
    if imp is not None:
        P = w.settings.pack_size
        imp_per_sample = np.stack([imp[k // P] for k in range(w.n_samples)])
    return spins, imp_per_sample


# FP32 unit roundoff: the size of the rounding the FP32 form makes in every
# stage, used as the input perturbation of the chaos-floor comparison
FP32_ROUNDOFF = 2.0 ** -24


def tangent_perturb(spins: np.ndarray, eps: float, seed: int) -> np.ndarray:
    """Every spin moved by a seeded Gaussian tangent vector of rms size eps
    and renormalised to |S| = 1.  Long SMD trajectories are chaotic: the
    spectrum of an FP64 run from these inputs differs from the unperturbed
    FP64 run by the least DSSF difference that any arithmetic making errors
    of size eps can reach on that run (the chaos floor)."""
    rng = np.random.default_rng(seed)
    g = rng.normal(size=spins.shape) * eps
    g -= (g * spins).sum(-1, keepdims=True) * spins
    out = spins + g
    return out / np.linalg.norm(out, axis=-1, keepdims=True)
