"""Host-side mirror of the reference's SMD interface over the C ABI.

The reference computes one sample's dynamical spectrum with

    get_dynSpectrum(procNum, tWinVec, spinField, SqxWVec, SqyWVec, SqzWVec, qSStVec)
    (Codes_Folder/subrouts.cpp:11547-12149)

reading the lattice, couplings and time grid from process globals, and its
main program loops over samples and averages (Codes_Folder/smd_code.cpp:
3079-3291, 3596-3611).  Here the same data are explicit: a ``Context`` holds
device state, ``Context.lattice`` uploads the tables and couplings that
``convert_inputs2data`` and the lattice builders would have set, and
``Context.run`` / ``get_dyn_spectrum`` run the CUDA path.  Every array uses
the reference's layouts: spins [N][3] per sample, spectra [Q][ntm] per
component with grid q first in k = i * Gsz + j order.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import SMDError, SMD_FP32, SMD_FP64
from .settings import GEOMETRY, SMDSettings

_dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None
_ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int)) if a is not None else None


# ------------------------------------------------------------- lattices

@dataclasses.dataclass
class Lattice:
    geom: str
    L: int
    N: int
    G: int
    nsubs: int
    zn: List[int]
    rvec: np.ndarray          # [N][2]
    grid_map: np.ndarray      # [G*G]
    nbrs: List[np.ndarray]    # 3 x [N][zn[s]]

    @property
    def grid_fac(self) -> int:
        return self.G // self.L

    @property
    def qcrystal(self) -> bool:
        return self.grid_map is None

    def grid_positions(self) -> np.ndarray:
        """Site positions in the frame of the DFT grid.

        The grid transform of get_SqData_iMKL (Codes_Folder/subrouts.cpp:
        8330-8432) uses phases exp(-2 pi i (a i + b j) / G) of the grid
        indices (a, b); the grid is the lattice shifted by i0 cells along x
        for lieb and kagome (Codes_Folder/subrouts.cpp:2905-2936).  Positions
        R = a fc e1 + b fc e2 make exp(-i q . R) equal those phases at grid
        q, so list points reproduce grid values exactly.  A quasi-crystal's
        positions are its table's (rvecList).
        """
        if self.qcrystal:
            return self.rvec.copy()
        sz = {"square": 1.0, "triang": 1.0, "hexagn": math.sqrt(3.0), "kagome": 2.0,
              "lieb": math.sqrt(2.0)}[self.geom]
        fc = sz / self.grid_fac
        i0 = 1 if self.geom in ("lieb", "kagome") else 0
        R = self.rvec.copy()
        R[:, 0] += i0 * fc
        return R

    def grid_basis(self) -> Tuple[np.ndarray, np.ndarray]:
        """Reciprocal vectors g1, g2 with q(i, j) = i g1 + j g2 for grid index (i, j)."""
        sz = {"square": 1.0, "triang": 1.0, "hexagn": math.sqrt(3.0), "kagome": 2.0,
              "lieb": math.sqrt(2.0)}[self.geom]
        fc = sz / self.grid_fac
        if self.geom in ("square", "lieb"):
            e1, e2 = np.array([1.0, 0.0]), np.array([0.0, 1.0])
        else:
            e1, e2 = np.array([1.0, 0.0]), np.array([0.5, math.sqrt(3.0) / 2.0])
        A = np.stack([e1, e2]) * fc                    # rows: grid basis vectors
        B = 2.0 * math.pi * np.linalg.inv(A).T / self.G  # rows: g1, g2
        return B[0], B[1]

    def grid_qvectors(self) -> np.ndarray:
        g1, g2 = self.grid_basis()
        i, j = np.meshgrid(np.arange(self.G), np.arange(self.G), indexing="ij")
        return (i.ravel()[:, None] * g1 + j.ravel()[:, None] * g2)


def geometry_info(geom: str, L: int):
    lib = _lib.load()
    N, G, ns = C.c_int(), C.c_int(), C.c_int()
    zn = (C.c_int * 3)()
    rc = lib.smd_geometry_info(_lib.GEOMS[geom], L, C.byref(N), C.byref(G), C.byref(ns), zn)
    if rc:
        raise SMDError(rc, f"geometry {geom} with L={L}")
    return N.value, G.value, ns.value, list(zn)


def build_lattice(geom: str, L: int) -> Lattice:
    """Positions, grid map and neighbour tables (the reference's make_rvecList /
    make_nborsTable, built in O(N))."""
    lib = _lib.load()
    N, G, ns, zn = geometry_info(geom, L)
    rvec = np.zeros((N, 2))
    gmap = np.zeros(G * G, np.int32)
    nb = [np.zeros((N, z), np.int32) for z in zn]
    rc = lib.smd_build_lattice(_lib.GEOMS[geom], L, _dp(rvec), _ip(gmap), _ip(nb[0]),
                               _ip(nb[1]), _ip(nb[2]))
    if rc:
        raise SMDError(rc, f"smd_build_lattice({geom}, {L})")
    return Lattice(geom, L, N, G, ns, zn, rvec, gmap, nb)


def load_qcrystal(table_dir: str, N: int, geom: str = "Aamman") -> Lattice:
    """A quasi-crystal approximant from the reference's table files in
    ``table_dir`` (the outBin/ folder of a qcrystal run):

      sitesList_AppxtSz(N).bin  N x 2 doubles, the site positions (rvecList)
      nborsList_AppxtSz(N).bin  per site Zn1, Zn2 then ZnX int32 neighbour
                                indices, -1 where a site has fewer (ghosts)

    as Codes_Folder/smd_code.cpp:1248-1300 and 1575-1660 read them, with
    the same checks: exact file sizes and a unit nearest-neighbour spacing
    (check_latticeSpc, Codes_Folder/subrouts.cpp:5803-5832).  The returned
    lattice has no DFT grid (G = the side of its direct-sum q set)."""
    import os
    from .settings import QCT_GEOMETRY, SettingsError
    if geom not in QCT_GEOMETRY:
        raise SettingsError(f"unknown quasi-geometry {geom!r}")
    zn = list(QCT_GEOMETRY[geom][2])
    tag = f"_AppxtSz({N})"
    sites = os.path.join(table_dir, f"sitesList{tag}.bin")
    nbors = os.path.join(table_dir, f"nborsList{tag}.bin")
    if not os.path.exists(sites) or os.path.getsize(sites) != N * 16:
        raise SettingsError(f"invalid or missing {sites}")
    if not os.path.exists(nbors) or os.path.getsize(nbors) != N * sum(zn) * 4:
        raise SettingsError(f"invalid or missing {nbors}")
    rvec = np.fromfile(sites, dtype=np.float64).reshape(N, 2)
    tab = np.fromfile(nbors, dtype=np.int32).reshape(N, sum(zn))
    if tab.max() >= N:
        raise SettingsError(f"{nbors}: neighbour index out of range")
    nb = [np.ascontiguousarray(tab[:, :zn[0]]),
          np.ascontiguousarray(tab[:, zn[0]:zn[0] + zn[1]]),
          np.ascontiguousarray(tab[:, zn[0] + zn[1]:])]
    # check_latticeSpc: shortest first-shell distance from site 0 (entries
    # > 0, as the reference tests them) within 5 % of one
    d = [float(np.hypot(*(rvec[j] - rvec[0]))) for j in nb[0][0] if j > 0]
    if not d or not (0.95 <= min(d) <= 1.05):
        raise SettingsError("lattice spacing is not unit")
    Lsz = (int(math.sqrt(N)) // 2) * 2
    return Lattice(geom, Lsz, N, Lsz, 1, zn, rvec, None, nb)


def qcrystal_qpoints(lat: Lattice) -> Tuple[np.ndarray, float]:
    """The q set and scale of get_qct_SqData (Codes_Folder/subrouts.cpp:
    8460-8525) for a quasi-crystal: Lsz x Lsz points q = dq (nx, ny), nx
    and ny in FFT order (0 .. Lsz/2 - 1, then -Lsz/2 .. -1), output index
    j Lsz + i for (nx(i), ny(j)), dq = 4 (2 pi) / Lsz
    (Codes_Folder/smd_code.cpp:1774), scale 1 / sqrt(N)."""
    L = lat.G
    dq = 4.0 * (2.0 * math.pi) / L
    n = np.where(np.arange(L) < L // 2, np.arange(L), np.arange(L) - L)
    ny, nx = np.meshgrid(n, n, indexing="ij")     # row j (ny), column i (nx)
    q = np.stack([nx.ravel() * dq, ny.ravel() * dq], axis=1)
    return q, 1.0 / math.sqrt(lat.N)


def build_bonds(lat: Lattice, j2_on: bool, jx_on: bool):
    lib = _lib.load()
    maxb = lat.N * sum(lat.zn)
    bonds = np.zeros((maxb, 2), np.int32)
    nb = (C.c_int * 4)()
    z = np.array(lat.zn, np.int32)
    rc = lib.smd_build_bonds(lat.N, _ip(z), _ip(lat.nbrs[0]), _ip(lat.nbrs[1]),
                             _ip(lat.nbrs[2]), int(j2_on), int(jx_on), _ip(bonds), maxb, nb)
    if rc:
        raise SMDError(rc, "smd_build_bonds")
    return bonds[: nb[0]].copy(), [nb[1], nb[2], nb[3]]


def window(name: str, n: int) -> np.ndarray:
    w = np.zeros(n)
    rc = _lib.load().smd_window(name.encode(), n, _dp(w))
    if rc:
        raise SMDError(rc, f"window {name!r}")
    return w


# --------------------------------------------------------------- context

@dataclasses.dataclass
class RunResult:
    spec: np.ndarray          # [3][Q][n_rec] sample average of |S(q,w)|^2
    qss: np.ndarray           # [n_rec]
    final: Optional[np.ndarray]
    report: dict


class Context:
    """One device context (smd_ctx)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self.lib = _lib.load()
        opts = _lib.DeviceOpts(device, hbm_budget)
        h = C.c_void_p()
        rc = self.lib.smd_ctx_create(C.byref(opts), C.byref(h))
        if rc:
            raise SMDError(rc, "smd_ctx_create (needs an sm_100 GPU)")
        self.h = h
        self._keep = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.smd_serve_shutdown(self.h)
            self.lib.smd_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int, what: str):
        if rc:
            raise SMDError(rc, f"{what}: {self.lib.smd_last_error(self.h).decode()}")

    # -- objects
    def lattice(self, s: SMDSettings, lat: Lattice) -> int:
        """Upload a lattice with the couplings of settings ``s``."""
        bonds, nbonds = build_bonds(lat, s.j2_on, s.jx_on)
        nb = [np.ascontiguousarray(a, np.int32) for a in lat.nbrs]
        gmap = None if lat.qcrystal else np.ascontiguousarray(lat.grid_map, np.int32)
        pos = np.ascontiguousarray(lat.grid_positions(), np.float64)
        d = _lib.LatticeDesc()
        d.N = lat.N
        for k in range(3):
            d.zn[k] = lat.zn[k]
            d.nbr[k] = nb[k].ctypes.data
        d.shell_on[0], d.shell_on[1], d.shell_on[2] = 1, int(s.j2_on), int(s.jx_on)
        J = s.jmat()
        for a in range(3):
            for b in range(2):
                for c in range(2):
                    d.J[a * 4 + b * 2 + c] = J[a][b][c]
        lam = s.lambdas()
        for a in range(3):
            for c in range(3):
                d.lambda_[a * 3 + c] = lam[a][c]
        d.lieb_delta_on = int(abs(s.J2_delta) > 1e-12)
        d.j2_delta = s.J2_delta
        d.h = s.h
        for k in range(3):
            d.nbonds[k] = nbonds[k]
        d.bonds = bonds.ctypes.data
        # a quasi-crystal has no DFT grid: its q set is a direct-sum list
        d.G = 0 if lat.qcrystal else lat.G
        d.grid_map = None if gmap is None else gmap.ctypes.data
        d.pos = pos.ctypes.data
        lid = C.c_int()
        self._check(self.lib.smd_lattice_upload(self.h, C.byref(d), C.byref(lid)), "lattice upload")
        self._keep[("lat", lid.value)] = (lat, s)
        return lid.value

    def qset(self, lattice_id: int, use_grid: bool = True,
             qlist: Optional[np.ndarray] = None, list_scale: Optional[float] = None) -> int:
        lat, _ = self._keep[("lat", lattice_id)]
        nl = 0 if qlist is None else len(qlist)
        ql = np.ascontiguousarray(qlist if nl else np.zeros((1, 2)), np.float64)
        sc = (1.0 / lat.G) if list_scale is None else list_scale
        qid = C.c_int()
        self._check(self.lib.smd_qset_upload(self.h, lattice_id, int(use_grid), nl, _dp(ql), sc,
                                             C.byref(qid)), "qset upload")
        return qid.value

    def qset_size(self, qset_id: int) -> int:
        Q = C.c_int()
        self._check(self.lib.smd_qset_size(self.h, qset_id, C.byref(Q)), "qset size")
        return Q.value

    # -- jobs
    def job(self, lattice_id, qset_id, n_samples, dt, n_rec, stride=1, precision=SMD_FP64,
            fix_every=1, imp: Optional[np.ndarray] = None):
        j = _lib.JobDesc()
        j.lattice, j.qset, j.n_samples = lattice_id, qset_id, n_samples
        j.dt, j.n_rec, j.stride = dt, n_rec, stride
        j.precision, j.fix_every = precision, fix_every
        self._imp = None
        if imp is not None:
            self._imp = np.ascontiguousarray(imp, np.int32)
            j.imp = self._imp.ctypes.data
        return j

    def run(self, lattice_id: int, qset_id: int, spins: np.ndarray, dt: float, n_rec: int,
            stride: int = 1, precision: int = SMD_FP64, fix_every: int = 1,
            win: Optional[np.ndarray] = None, imp: Optional[np.ndarray] = None,
            want_final: bool = True) -> RunResult:
        spins = np.ascontiguousarray(spins, np.float64)
        if spins.ndim == 2:
            spins = spins[None]
        S = spins.shape[0]
        Q = self.qset_size(qset_id)
        win = np.ones(n_rec) if win is None else np.ascontiguousarray(win, np.float64)
        j = self.job(lattice_id, qset_id, S, dt, n_rec, stride, precision, fix_every, imp)
        spec = np.zeros((3, Q, n_rec))
        qss = np.zeros(n_rec)
        fin = np.zeros_like(spins) if want_final else None
        rep = _lib.Report()
        self._check(self.lib.smd_run(self.h, C.byref(j), _dp(spins), _dp(win), _dp(spec),
                                     _dp(qss), _dp(fin), C.byref(rep)), "smd_run")
        report = {k: getattr(rep, k) for k, _ in _lib.Report._fields_}
        return RunResult(spec, qss, fin, report)

    def evolve(self, lattice_id: int, spins: np.ndarray, dt: float, nsteps: int,
               precision: int = SMD_FP64, fix_every: int = 1,
               imp: Optional[np.ndarray] = None) -> np.ndarray:
        sp = np.array(spins, np.float64, order="C", copy=True)
        if sp.ndim == 2:
            sp = sp[None]
        ia = None if imp is None else np.ascontiguousarray(imp, np.int32)
        rep = _lib.Report()
        self._check(self.lib.smd_evolve(self.h, lattice_id, precision, sp.shape[0], dt, nsteps,
                                        fix_every, _ip(ia), _dp(sp), C.byref(rep)), "smd_evolve")
        return sp

    def get_dyn_spectrum(self, lattice_id: int, qset_id: int, dtm: float, ntm: int,
                         tWinVec: np.ndarray, spinField: np.ndarray,
                         imp: Optional[np.ndarray] = None):
        """The reference's get_dynSpectrum for one sample.

        Returns (SqxWVec, SqyWVec, SqzWVec, qSStVec), each spectrum [Q][ntm];
        spinField ([N][3]) is updated in place to the final state, as the
        reference leaves it.
        """
        Q = self.qset_size(qset_id)
        sf = np.ascontiguousarray(spinField, np.float64)
        x, y, z = (np.zeros((Q, ntm)) for _ in range(3))
        q = np.zeros(ntm)
        ia = None if imp is None else np.ascontiguousarray(imp, np.int32)
        self._check(self.lib.smd_dyn_spectrum_ref(self.h, lattice_id, qset_id, dtm, ntm,
                                                  _dp(np.ascontiguousarray(tWinVec, np.float64)),
                                                  _dp(sf), _ip(ia), _dp(x), _dp(y), _dp(z),
                                                  _dp(q)), "smd_dyn_spectrum_ref")
        if sf is not spinField:
            spinField[...] = sf
        return x, y, z, q

    # -- batches
    def batch(self, members, dt: float, n_rec: int, stride: int = 1, precision: int = SMD_FP32,
              fix_every: int = 16) -> "Batch":
        """A batched job over several lattices.  members: [(lattice_id,
        qset_id, n_samples, imp or None)]."""
        return Batch(self, members, dt, n_rec, stride, precision, fix_every)

    # -- Monte Carlo
    def mc_run(self, lattice_id: int, temps, n_therm: int, n_meas: int, cr_skip: int = 1000,
               chains: int = 1, pt: bool = False, seed: int = 1, spins0=None, imp=None,
               sweeps=(5, 5, 2, 8), want_samples: bool = True) -> dict:
        """The MC stage that writes the SMD sample file (smd_mc_run; the
        reference's Codes_Folder/mc_hm_code.cpp).  temps: the temperature
        ladder; chains: independent replicas per temperature; sweeps:
        (nmicro, ncanon, nmicro2, ncanon2).  Returns samples
        [chains][T][n_rec][N][3], energy [chains][T][n_therm + n_meas] and
        pt_counts [chains][T][2] (attempts, acceptances)."""
        lat, _ = self._keep[("lat", lattice_id)]
        N = lat.N
        temps = np.ascontiguousarray(temps, np.float64)
        T = len(temps)
        d = _lib.MCDesc()
        d.lattice, d.n_temps = lattice_id, T
        d.temps = temps.ctypes.data_as(C.POINTER(C.c_double))
        d.chains, d.n_therm, d.n_meas, d.cr_skip, d.pt = chains, n_therm, n_meas, cr_skip, int(pt)
        d.n_micro, d.n_canon, d.n_micro2, d.n_canon2 = sweeps
        d.seed = seed
        imp_a = None
        if imp is not None:
            imp_a = np.ascontiguousarray(np.broadcast_to(imp, (chains, T, N)), np.int32)
            d.imp = imp_a.ctypes.data_as(C.POINTER(C.c_int))
        sp = None if spins0 is None else np.ascontiguousarray(spins0, np.float64).reshape(chains, T, N, 3)
        n_rec = -(-n_meas // cr_skip)
        samples = np.zeros((chains, T, n_rec, N, 3)) if want_samples and n_rec else None
        energy = np.zeros((chains, T, n_therm + n_meas))
        counts = np.zeros((chains, T, 2), np.int32)
        rep = _lib.Report()
        self._check(self.lib.smd_mc_run(self.h, C.byref(d), _dp(sp), _dp(samples), _dp(energy),
                                        _ip(counts), C.byref(rep)), "smd_mc_run")
        return dict(samples=samples, energy=energy, pt_counts=counts,
                    report={k: getattr(rep, k) for k, _ in _lib.Report._fields_})

    def mc_colouring(self, lattice_id: int):
        """The MC sweeps' colour classes: (order [N], class offsets)."""
        lat, _ = self._keep[("lat", lattice_id)]
        order = np.zeros(lat.N, np.int32)
        cst = np.zeros(65, np.int32)
        n = C.c_int(64)
        self._check(self.lib.smd_mc_colouring(self.h, lattice_id, _ip(order), _ip(cst), C.byref(n)),
                    "smd_mc_colouring")
        return order, cst[: n.value + 1].copy()

    # -- serving
    def submit(self, lattice_id, qset_id, spins, dt, n_rec, stride=1, precision=SMD_FP64,
               fix_every=1, win=None, imp=None):
        spins = np.ascontiguousarray(spins, np.float64)
        if spins.ndim == 2:
            spins = spins[None]
        Q = self.qset_size(qset_id)
        win = np.ones(n_rec) if win is None else np.ascontiguousarray(win, np.float64)
        j = self.job(lattice_id, qset_id, spins.shape[0], dt, n_rec, stride, precision,
                     fix_every, imp)
        spec = np.zeros((3, Q, n_rec))
        qss = np.zeros(n_rec)
        jid = C.c_longlong()
        self._check(self.lib.smd_submit(self.h, C.byref(j), _dp(spins), _dp(win), _dp(spec),
                                        _dp(qss), C.byref(jid)), "smd_submit")
        self._keep[("job", jid.value)] = (spec, qss)
        return jid.value

    def wait(self, job_id: int, timeout_ms: float = -1.0):
        lat = C.c_double()
        rc = self.lib.smd_wait(self.h, job_id, timeout_ms, C.byref(lat))
        if rc:
            raise SMDError(rc, f"job {job_id} ({self.lib.smd_last_error(self.h).decode()})")
        spec, qss = self._keep.pop(("job", job_id))
        return spec, qss, lat.value

    def job_info(self, job_id: int) -> dict:
        """Latency, site-steps and energy drift of a finished job."""
        rep = _lib.Report()
        rc = self.lib.smd_job_info(self.h, job_id, C.byref(rep))
        if rc:
            raise SMDError(rc, f"job {job_id}")
        return {k: getattr(rep, k) for k, _ in _lib.Report._fields_}

    def poll(self, job_id: int) -> int:
        lat = C.c_double()
        return self.lib.smd_poll(self.h, job_id, C.byref(lat))

    def cancel(self, job_id: int) -> int:
        return self.lib.smd_cancel(self.h, job_id)


class Batch:
    """Several jobs on different lattices run as one batch (smd_batch_*):
    one persistent RK launch per chunk of records for every member, the job
    step replayed as one CUDA graph.  ``run`` returns each member's sample
    averages as a RunResult (final spins are not kept)."""

    def __init__(self, ctx: Context, members, dt, n_rec, stride, precision, fix_every):
        self.ctx = ctx
        self.n_rec = n_rec
        self._imps = []
        arr = (_lib.BatchMember * len(members))()
        self.sizes = []
        for k, (lid, qid, ns, imp) in enumerate(members):
            arr[k].lattice, arr[k].qset, arr[k].n_samples = lid, qid, ns
            if imp is not None:
                ia = np.ascontiguousarray(imp, np.int32)
                self._imps.append(ia)
                arr[k].imp = ia.ctypes.data
            lat, _ = ctx._keep[("lat", lid)]
            self.sizes.append((ns, lat.N, ctx.qset_size(qid)))
        d = _lib.BatchDesc()
        d.n_members = len(members)
        d.members = arr
        d.dt, d.n_rec, d.stride, d.precision, d.fix_every = dt, n_rec, stride, precision, fix_every
        bid = C.c_int()
        ctx._check(ctx.lib.smd_batch_create(ctx.h, C.byref(d), C.byref(bid)), "smd_batch_create")
        self.id = bid.value

    def info(self) -> dict:
        t = _lib.BatchTuning()
        self.ctx._check(self.ctx.lib.smd_batch_info(self.ctx.h, self.id, C.byref(t)), "smd_batch_info")
        out = {k: getattr(t, k) for k, _ in _lib.BatchTuning._fields_ if k != "member_ctas"}
        out["member_ctas"] = [t.member_ctas[i] for i in range(len(self.sizes))]
        return out

    def run(self, spins, win=None):
        """spins: one [S][N][3] array per member; returns [RunResult]."""
        n = self.n_rec
        win = np.ones(n) if win is None else np.ascontiguousarray(win, np.float64)
        sp = [np.ascontiguousarray(x, np.float64) for x in spins]
        spec = [np.zeros((3, Q, n)) for (_, _, Q) in self.sizes]
        qss = [np.zeros(n) for _ in self.sizes]
        k = len(sp)
        P = C.POINTER(C.c_double)
        ins = (P * k)(*[_dp(x) for x in sp])
        so = (P * k)(*[_dp(x) for x in spec])
        qo = (P * k)(*[_dp(x) for x in qss])
        rep = _lib.Report()
        self.ctx._check(self.ctx.lib.smd_batch_run(self.ctx.h, self.id, ins, _dp(win), so, qo,
                                                   C.byref(rep)), "smd_batch_run")
        report = {f: getattr(rep, f) for f, _ in _lib.Report._fields_}
        return [RunResult(spec[i], qss[i], None, report) for i in range(k)]

    def free(self):
        if self.id is not None:
            self.ctx.lib.smd_batch_free(self.ctx.h, self.id)
            self.id = None
