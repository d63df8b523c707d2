"""Synthetic spin samples in the reference's MC sample-file format.

The SMD program reads ``outBin/MC_Bin_SpinField_T(%.5f)<label>.bin``
(Codes_Folder/smd_code.cpp:913-928).  The MC program writes it pack by pack
(Codes_Folder/mc_hm_code.cpp:4111-4125, 5167-5178):

* with disorder, one int32 impurity map of Ns entries opens every pack;
* then PackSize = NMeas / crSkip spin fields of Ns x 3 float64 (x, y, z per
  site, sites in lattice order).

There is no public data set for this path, so seeded synthetic states stand in
for MC output: an ordered state of the lattice with every spin tilted by an
isotropic Gaussian tangent vector and renormalised.
"""
from __future__ import annotations

import math
import os
from typing import Optional

import numpy as np

from .settings import SMDSettings

QVAL = 4.0 * math.pi / 3.0            # Codes_Folder/subrouts.cpp:526
C60 = math.cos(math.pi / 3.0)


def impurity_count(N: int, ratio: float) -> int:
    """Number of impurity sites ``make_impurityField`` marks.

    Follows the marking loop of Codes_Folder/subrouts.cpp:3336-3350: site
    positions 0, 1, ... of a shuffled list are marked until
    (i + 2) / Ns exceeds the ratio.
    """
    iNs = 1.0 / N
    mark, count = 1, 0
    for i in range(N):
        count += mark
        if (i + 2) * iNs > ratio:
            mark = 0
        if not mark:
            break
    return count


def impurity_map(N: int, ratio: float, rng: np.random.Generator) -> np.ndarray:
    imp = np.zeros(N, dtype=np.int32)
    if ratio > 0.0:
        imp[rng.permutation(N)[: impurity_count(N, ratio)]] = 1
    return imp


def field_norm(S: np.ndarray) -> float:
    """``fieldNorm`` (Codes_Folder/subrouts.cpp:4913-4925): sequential sum of |S_i|^2 / Ns."""
    d = (S[:, 0] * S[:, 0] + S[:, 1] * S[:, 1]) + S[:, 2] * S[:, 2]
    return abs(float(np.cumsum(d)[-1])) * (1.0 / S.shape[0])


def _normalise(v: np.ndarray) -> np.ndarray:
    n = np.sqrt((v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2])
    return v / n[:, None]


def ordered_state(s: SMDSettings, kind: str) -> np.ndarray:
    """Ordered reference states on Bravais lattices.

    ``stripe``: S = cos(j pi) x  (HStpPhase, Codes_Folder/subrouts.cpp:4360-4372);
    ``q120``:   S = (cos t, sin t, 0), t = Q (i + j c60)
                (Q120Phase, Codes_Folder/subrouts.cpp:4318-4328);
    ``ferro``:  S = z.
    Sites are numbered k = i * L + j (Codes_Folder/subrouts.cpp:2700-2708).
    """
    if s.qcrystal:
        # a quasi-crystal has no Bravais cell: only the uniform state here
        # (its ordered states come as table files, see smd.load_qcrystal)
        if kind != "ferro":
            raise ValueError(f"{kind}: pass the approximant's state file as base")
        S = np.zeros((s.N, 3))
        S[:, 2] = 1.0
        return S
    L = s.L
    i, j = np.meshgrid(np.arange(L), np.arange(L), indexing="ij")
    i = i.ravel().astype(np.float64)
    j = j.ravel().astype(np.float64)
    S = np.zeros((L * L, 3))
    if kind == "stripe":
        S[:, 0] = np.cos(j * math.pi)
    elif kind == "q120":
        t = QVAL * (i + j * C60)
        S[:, 0] = np.cos(t)
        S[:, 1] = np.sin(t)
    elif kind == "ferro":
        S[:, 2] = 1.0
    else:
        raise ValueError(kind)
    if s.nsubs > 1:
        S = np.repeat(S, s.nsubs, axis=0)
    return S


def tilt(S: np.ndarray, sigma: float, rng: np.random.Generator) -> np.ndarray:
    """Add an isotropic Gaussian tangent vector of width sigma and renormalise."""
    g = rng.normal(0.0, sigma, size=S.shape)
    g -= np.sum(g * S, axis=1, keepdims=True) * S
    out = _normalise(S + g)
    # The reference rejects a sample whose fieldNorm exceeds 1
    # (Codes_Folder/smd_code.cpp:3124-3126); pull rounding-level excess back.
    while field_norm(out) > 1.0:
        out *= 1.0 - 2.0 ** -52
    return out


def make_samples(s: SMDSettings, n_samples: int, kind: str, sigma: float,
                 seed: int, base: Optional[np.ndarray] = None):
    """Return (spins[n, N, 3], imp[n_packs, N] or None) for n_samples samples."""
    rng = np.random.default_rng(seed)
    S0 = ordered_state(s, kind) if base is None else np.asarray(base, np.float64)
    spins = np.stack([tilt(S0, sigma, rng) for _ in range(n_samples)])
    imp = None
    if s.disorder:
        n_packs = -(-n_samples // s.pack_size)
        imp = np.stack([impurity_map(s.N, s.imp_ratio, rng) for _ in range(n_packs)])
    return spins, imp


def sample_file_name(s: SMDSettings) -> str:
    return f"MC_Bin_SpinField{s.t_tag}.bin"


def write_sample_file(path: str, s: SMDSettings, spins: np.ndarray,
                      imp: Optional[np.ndarray]) -> None:
    n = spins.shape[0]
    P = s.pack_size
    if s.disorder:
        if n % P:
            raise ValueError("with disorder the sample count must fill whole packs")
    elif n != 1 and n % P:
        raise ValueError("sample count must be 1 or a multiple of PackSize")
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "wb") as f:
        for p in range(max(1, -(-n // P))):
            if s.disorder:
                f.write(np.ascontiguousarray(imp[p], dtype="<i4").tobytes())
            f.write(np.ascontiguousarray(spins[p * P:(p + 1) * P], dtype="<f8").tobytes())


def read_sample_file(path: str, s: SMDSettings):
    """Read a sample file; returns (spins[n, N, 3], imp_per_sample[n, N] or None).

    Follows the size checks of Codes_Folder/smd_code.cpp:997-1066.
    """
    N, P = s.N, s.pack_size
    size = os.path.getsize(path)
    conf = N * 3 * 8
    pack = (N * 4 if s.disorder else 0) + P * conf
    ref = pack if s.disorder else conf
    if size == ref:
        n_packs = 1
    elif size % ref:
        raise ValueError(f"{path}: size {size} is not a multiple of {ref}")
    else:
        n_packs = size // pack
        if n_packs * P != (size - (n_packs * N * 4 if s.disorder else 0)) // conf:
            raise ValueError(f"{path}: inconsistent pack layout")
    raw = np.fromfile(path, dtype=np.uint8)
    spins, imps = [], []
    off = 0
    n_in_first = 1 if (size == conf and not s.disorder) else P
    for p in range(n_packs):
        imp = None
        if s.disorder:
            imp = raw[off:off + 4 * N].view("<i4").copy()
            off += 4 * N
        cnt = n_in_first if p == 0 else P
        block = raw[off:off + cnt * conf].view("<f8").reshape(cnt, N, 3)
        off += cnt * conf
        spins.append(block)
        if imp is not None:
            imps.extend([imp] * cnt)
    spins = np.concatenate(spins).copy()
    return spins, (np.stack(imps) if s.disorder else None)
