"""Python access to the oracle (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` import this module, and only as the
checker or the timed CPU baseline.  The product path never does.

Two things live here:

* ``liboracle.so`` -- the plain-C restatement of the reference's SMD path
  (``oracle/smd_oracle.c``);
* ``_ref/smd_ref_run`` -- the reference's own ``Codes_Folder/subrouts.cpp``
  compiled from its sources against stand-in headers (``oracle/Makefile``),
  used to pin the restatement and as the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
from typing import Dict, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_RUN = os.path.join(HERE, "_ref", "smd_ref_run")

GEOMS = {"square": 0, "triang": 1, "hexagn": 2, "kagome": 3, "lieb": 4}

_lib = None


def build(force: bool = False) -> None:
    """Compile liboracle.so (and the reference runner where its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE] + (["-B"] if force else []),
                   check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.orc_geometry.argtypes = [C.c_int, C.c_int, ip, ip, ip, ip]
        L.orc_make_lattice.argtypes = [C.c_int, C.c_int, dp, ip, ip, ip, ip]
        L.orc_make_bonds.argtypes = [C.c_int, ip, ip, ip, ip, C.c_int, C.c_int,
                                     ip, C.c_int, ip]
        L.orc_local_field.argtypes = [C.c_void_p, C.c_int, dp, dp]
        L.orc_energy.argtypes = [C.c_void_p, dp]
        L.orc_energy.restype = C.c_double
        L.orc_window.argtypes = [C.c_char_p, C.c_int, dp]
        L.orc_dyn_spectrum.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int,
                                       C.c_int, dp, dp, C.c_int, ip, C.c_int, dp, dp,
                                       C.c_double, dp, dp, dp, dp]
        L.orc_evolve.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, dp,
                                 C.c_int, dp]
        L.orc_fft1d.argtypes = [dp, C.c_long, C.c_int]
        L.orc_dft1d_naive.argtypes = [dp, dp, C.c_long, C.c_int]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int)) if a is not None else None


class _Model(C.Structure):
    _fields_ = [("N", C.c_int), ("zn", C.c_int * 3), ("nbr", C.c_void_p * 3),
                ("shell_on", C.c_int * 3), ("disorder", C.c_int),
                ("imp", C.c_void_p), ("J", C.c_double * 12),
                ("lam", C.c_double * 9), ("lieb_delta_on", C.c_int),
                ("j2_delta", C.c_double), ("h", C.c_double),
                ("nbonds", C.c_int * 3), ("bonds", C.c_void_p)]


def make_lattice(geom: str, L: int) -> Dict:
    lb = lib()
    N, G, ns = C.c_int(), C.c_int(), C.c_int()
    zn = (C.c_int * 3)()
    if lb.orc_geometry(GEOMS[geom], L, C.byref(N), C.byref(G), C.byref(ns), zn):
        raise ValueError(geom)
    N, G, zn = N.value, G.value, list(zn)
    rvec = np.zeros((N, 2))
    gmap = np.zeros(G * G, np.int32)
    nb = [np.zeros((N, z), np.int32) for z in zn]
    flag = lb.orc_make_lattice(GEOMS[geom], L, _dp(rvec), _ip(gmap), _ip(nb[0]),
                               _ip(nb[1]), _ip(nb[2]))
    if flag:
        raise RuntimeError(f"orc_make_lattice flag {flag}")
    return dict(geom=geom, L=L, N=N, G=G, nsubs=ns.value, zn=zn, rvec=rvec,
                grid_map=gmap, nbrs=nb)


def tables_lattice(rvec: np.ndarray, nbrs, G: int) -> Dict:
    """A lattice given by its tables (a quasi-crystal approximant read from
    the reference's sitesList / nborsList files, smd_code.cpp:1248-1300 and
    1575-1660): positions, three neighbour tables with -1 ghosts, no DFT
    grid (grid_map all -1), G the side of the direct-sum q set."""
    nb = [np.ascontiguousarray(a, np.int32) for a in nbrs]
    N = len(rvec)
    return dict(geom="table", L=G, N=N, G=G, nsubs=1, zn=[a.shape[1] for a in nb],
                rvec=np.ascontiguousarray(rvec, np.float64),
                grid_map=np.full(G * G, -1, np.int32), nbrs=nb)


def qct_qpoints(G: int, N: int):
    """q set of get_qct_SqData (Codes_Folder/subrouts.cpp:8460-8525): for
    output index j G + i, q = dq (nx(i), ny(j)) with n(i) = i for i < G/2,
    else i - G, and dq = 4 pi2 / G (smd_code.cpp:1774); scale 1/sqrt(N)."""
    dq = 4.0 * (2.0 * np.pi) / G
    q = np.zeros((G * G, 2))
    for j in range(G):
        ny = j if j < G // 2 else j - G
        for i in range(G):
            nx = i if i < G // 2 else i - G
            q[j * G + i] = (nx * dq, ny * dq)
    return q, 1.0 / np.sqrt(N)


def make_bonds(lat: Dict, j2_on: bool, jx_on: bool):
    N, zn = lat["N"], lat["zn"]
    maxb = N * sum(zn)
    bonds = np.zeros((maxb, 2), np.int32)
    nb = (C.c_int * 4)()
    zarr = np.array(zn, np.int32)
    rc = lib().orc_make_bonds(N, _ip(zarr), _ip(lat["nbrs"][0]), _ip(lat["nbrs"][1]),
                              _ip(lat["nbrs"][2]), int(j2_on), int(jx_on),
                              _ip(bonds), maxb, nb)
    if rc:
        raise RuntimeError("bond buffer too small")
    return bonds[: nb[0]].copy(), list(nb)[1:]


class Model:
    """orc_model built from settings, a lattice and an impurity map."""

    def __init__(self, settings, lat: Dict, imp: Optional[np.ndarray] = None):
        s = settings
        self.lat = lat
        self.N = lat["N"]
        self.bonds, self.nbonds = make_bonds(lat, s.j2_on, s.jx_on)
        self.imp = (np.ascontiguousarray(imp, np.int32) if s.disorder
                    else np.zeros(self.N, np.int32))
        self._keep = [np.ascontiguousarray(a, np.int32) for a in lat["nbrs"]]
        m = _Model()
        m.N = self.N
        for k in range(3):
            m.zn[k] = lat["zn"][k]
            m.nbr[k] = self._keep[k].ctypes.data
        m.shell_on[0], m.shell_on[1], m.shell_on[2] = 1, int(s.j2_on), int(s.jx_on)
        m.disorder = int(s.disorder)
        m.imp = self.imp.ctypes.data
        J = s.jmat()
        for a in range(3):
            for b in range(2):
                for c in range(2):
                    m.J[a * 4 + b * 2 + c] = J[a][b][c]
        lam = s.lambdas()
        for a in range(3):
            for c in range(3):
                m.lam[a * 3 + c] = lam[a][c]
        m.lieb_delta_on = int(abs(s.J2_delta) > 1e-12)
        m.j2_delta = s.J2_delta
        m.h = s.h
        for k in range(3):
            m.nbonds[k] = self.nbonds[k]
        m.bonds = self.bonds.ctypes.data
        self.struct = m

    def ptr(self):
        return C.byref(self.struct)

    def local_field(self, i: int, S: np.ndarray) -> np.ndarray:
        out = np.zeros(3)
        S = np.ascontiguousarray(S, np.float64)
        lib().orc_local_field(self.ptr(), i, _dp(S), _dp(out))
        return out

    def energy(self, S: np.ndarray) -> float:
        S = np.ascontiguousarray(S, np.float64)
        return lib().orc_energy(self.ptr(), _dp(S))


def window(name: str, n: int) -> np.ndarray:
    w = np.zeros(n)
    if lib().orc_window(name.encode(), n, _dp(w)):
        raise ValueError(name)
    return w


def dyn_spectrum(model: Model, S: np.ndarray, dt: float, n_rec: int, stride: int = 1,
                 fix_every: int = 1, win: Optional[np.ndarray] = None,
                 grid: bool = True, qlist: Optional[np.ndarray] = None,
                 pos: Optional[np.ndarray] = None, list_scale: Optional[float] = None,
                 want_series: bool = False, want_energy: bool = False):
    """One sample; returns dict(spec[3][Q][n_rec], qss, final, series?, energy?)."""
    lat = model.lat
    G = lat["G"] if grid else 0
    S = np.array(S, np.float64, order="C", copy=True)
    nl = 0 if qlist is None else len(qlist)
    Q = G * G + nl
    win = np.ones(n_rec) if win is None else np.ascontiguousarray(win, np.float64)
    ql = np.ascontiguousarray(qlist, np.float64) if nl else np.zeros((1, 2))
    ps = np.ascontiguousarray(pos if pos is not None else lat["rvec"], np.float64)
    sc = (1.0 / lat["G"]) if list_scale is None else list_scale
    spec = np.zeros((3, Q, n_rec))
    qss = np.zeros(n_rec)
    ser = np.zeros((3, Q, n_rec, 2)) if want_series else None
    en = np.zeros(n_rec) if want_energy else None
    rc = lib().orc_dyn_spectrum(model.ptr(), dt, n_rec, stride, fix_every, _dp(win),
                                _dp(S), G, _ip(lat["grid_map"]), nl, _dp(ql),
                                _dp(ps), sc, _dp(spec), _dp(qss), _dp(ser), _dp(en))
    if rc:
        raise RuntimeError(f"orc_dyn_spectrum rc={rc}")
    out = dict(spec=spec, qss=qss, final=S)
    if want_series:
        out["series"] = ser[..., 0] + 1j * ser[..., 1]
    if want_energy:
        out["energy"] = en
    return out


def evolve(model: Model, S: np.ndarray, dt: float, nsteps: int, fix_every: int = 1,
           every: int = 0):
    S = np.array(S, np.float64, order="C", copy=True)
    traj = None
    if every > 0:
        traj = np.zeros((nsteps // every + 1, model.N, 3))
    lib().orc_evolve(model.ptr(), dt, nsteps, fix_every, _dp(S), every, _dp(traj))
    return S, traj


def fft1d(x: np.ndarray, sign: int = -1) -> np.ndarray:
    a = np.zeros((len(x), 2))
    a[:, 0], a[:, 1] = x.real, x.imag
    lib().orc_fft1d(_dp(a), len(x), sign)
    return a[:, 0] + 1j * a[:, 1]


def dft1d_naive(x: np.ndarray, sign: int = -1) -> np.ndarray:
    a = np.zeros((len(x), 2))
    a[:, 0], a[:, 1] = x.real, x.imag
    o = np.zeros_like(a)
    lib().orc_dft1d_naive(_dp(a), _dp(o), len(x), sign)
    return o[:, 0] + 1j * o[:, 1]


# ------------------------------------------------------ reference runner

def reference_available() -> bool:
    return os.path.exists(REF_RUN)


def run_reference(workdir: str, samples: str, first: int, count: int,
                  dump_final: bool = True, dwf_guard: bool = False,
                  timeout: Optional[float] = None) -> Dict:
    """Run the reference's own get_dynSpectrum loop on samples [first, first+count)."""
    args = [REF_RUN, workdir, samples, str(first), str(count)]
    if dump_final:
        args.append("--dump-final")
    if not dwf_guard:
        args.append("--no-dwf-guard")
    r = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"smd_ref_run rc={r.returncode}: {r.stderr.strip()[-500:]}")
    info = json.loads(r.stdout.strip().splitlines()[-1])
    return info


def read_ref_lattice(workdir: str) -> Dict:
    raw = np.fromfile(os.path.join(workdir, "ref_lattice.bin"), dtype=np.uint8)
    hdr = raw[:32].view(np.int32)
    N, z1, z2, zx, G, nb1, nb2, nbx = (int(v) for v in hdr)
    off = 32
    rvec = raw[off:off + 16 * N].view(np.float64).reshape(N, 2)
    off += 16 * N
    tabs = []
    for z in (z1, z2, zx):
        tabs.append(raw[off:off + 4 * N * z].view(np.int32).reshape(N, z).copy())
        off += 4 * N * z
    gmap = raw[off:off + 4 * G * G].view(np.int32).copy()
    off += 4 * G * G
    nb = nb1 + nb2 + nbx
    bonds = raw[off:off + 8 * nb].view(np.int32).reshape(nb, 2).copy()
    return dict(N=N, zn=[z1, z2, zx], G=G, rvec=rvec.copy(), nbrs=tabs,
                grid_map=gmap, bonds=bonds, nbonds=[nb1, nb2, nbx])


def read_ref_spec(workdir: str, Nq: int, ntm: int):
    """ref_spec.bin -> (spec[3][Nq][ntm] sums, qss sum)."""
    a = np.fromfile(os.path.join(workdir, "ref_spec.bin"), dtype=np.float64)
    body = a[: 3 * Nq * ntm].reshape(Nq, 3, ntm).transpose(1, 0, 2).copy()
    return body, a[3 * Nq * ntm:].copy()


def read_ref_final(workdir: str, count: int, N: int) -> np.ndarray:
    return np.fromfile(os.path.join(workdir, "ref_final.bin"),
                       dtype=np.float64).reshape(count, N, 3)
