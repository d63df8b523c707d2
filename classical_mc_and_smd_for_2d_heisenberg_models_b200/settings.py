"""The reference's five plain-text settings files plus the code-execution flags.

The SMD program reads, in order (Codes_Folder/smd_code.cpp:219-277, 472-539):

* ``Settings_CodeExec.txt``  16 ``<name> <0|1>`` pairs in the fixed order of
  ``Code_Settings`` (Codes_Folder/subrouts.cpp:105-123);
* ``Settings_MODEL.txt``     11 tokens: L J1 J2 JX J2_delta zLamb1 zLamb2 h T1 T2 geometry;
* ``Settings_MC_SIM.txt``    8 tokens: NTerm NMeas IState TpGrid outTag crSkip vrSkip MClive;
* ``Settings_SMD_SIM.txt``   7 tokens: ntm tpLstSz tpIndex dtm window RecVd1 RecVd2;
* ``Settings_Disorder.txt``  7 tokens: ratio J1ic J2ic JXic J1ii J2ii JXii.

Only the first N whitespace-separated tokens of each file are read; anything
after them is a comment (Set_Params.py:287-295).  This module writes and reads
those files and applies the validation rules of ``convert_inputs2data``
(Codes_Folder/subrouts.cpp:955-2186) that matter to the SMD path.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, List

CODE_SETTINGS: List[str] = [
    "ptON", "ptAdapt", "ptTrack", "ANNL_ON", "FFTW_ON", "RKCheck", "PBC_OFF",
    "IsiModel", "qcrystal", "with_recField", "with_DFTcodes", "force_Stripes",
    "refState_Zero", "qct_NeelPhase", "qct_RemovePBC", "rec_orderMaps",
]

WINDOWS = ("wread", "gauss", "ntall", "black", "flatw", "hann1", "sincw",
           "hann2", "lancz", "hann3", "nowin")

# geometry -> (nSubs, gridFac, (Zn1, Zn2, ZnX)); Codes_Folder/subrouts.cpp:1028-1067
GEOMETRY = {
    "square": (1, 1, (4, 4, 4)),
    "triang": (1, 1, (6, 6, 6)),
    "hexagn": (2, 3, (3, 6, 3)),
    "kagome": (3, 2, (4, 4, 6)),
    "lieb": (2, 2, (4, 4, 4)),
}

# quasi-crystal approximants read from table files (qcrystal = 1):
# Ammann-Beenker tilings, Codes_Folder/subrouts.cpp:1006-1012
QCT_GEOMETRY = {
    "Aamman": (1, 1, (8, 3, 8)),
}

BIN_SZ = 1000          # Codes_Folder/subrouts.cpp:309
TEMP_MAX = 2.0         # Codes_Folder/subrouts.cpp:389
DWF_MIN = 0.10         # Codes_Folder/subrouts.cpp:391


class SettingsError(ValueError):
    """Raised where the reference's input check would stop the run."""


def _is_not_zero(x: float) -> bool:
    return abs(x) > 1.0e-12   # isNotZero, Codes_Folder/subrouts.cpp:773-778


@dataclasses.dataclass
class SMDSettings:
    # Settings_MODEL.txt
    L: int = 16
    J1: float = 1.0
    J2: float = 0.0
    JX: float = 0.0
    J2_delta: float = 0.0
    zlamb1: float = 1.0
    zlamb2: float = 1.0
    h: float = 0.0
    T1: float = 0.1
    T2: float = 0.1
    geom: str = "square"
    # Settings_MC_SIM.txt (only NMeas, crSkip and outTag matter to SMD)
    NTerm: int = 1000
    NMeas: int = 2000
    IState: str = "high_T"
    TpGrid: str = "linear"
    outTag: str = "J2tag"
    crSkip: int = 1000
    vrSkip: int = 0
    MClive: int = 0
    # Settings_SMD_SIM.txt
    ntm: int = 1024
    tpLstSz: int = 1
    tpIndex: int = 0
    dtm: float = 0.01
    window: str = "nowin"
    RecVd1: int = 0
    RecVd2: int = 0
    # Settings_Disorder.txt
    imp_ratio: float = 0.0
    J1ic: float = 0.0
    J2ic: float = 0.0
    JXic: float = 0.0
    J1ii: float = 0.0
    J2ii: float = 0.0
    JXii: float = 0.0
    # Settings_CodeExec.txt
    flags: Dict[str, int] = dataclasses.field(
        default_factory=lambda: {k: (1 if k == "with_DFTcodes" else 0)
                                 for k in CODE_SETTINGS})

    # ------------------------------------------------------------ derived
    @property
    def qcrystal(self) -> bool:
        """A lattice read from table files; L then holds the site count
        (the reference's latSize, Codes_Folder/subrouts.cpp:1105-1114)."""
        return bool(self.flags.get("qcrystal", 0))

    def _geo(self):
        table = QCT_GEOMETRY if self.qcrystal else GEOMETRY
        if self.geom not in table:
            raise SettingsError(f"unknown geometry {self.geom!r}")
        return table[self.geom]

    @property
    def nsubs(self) -> int:
        return self._geo()[0]

    @property
    def grid_fac(self) -> int:
        return self._geo()[1]

    @property
    def zn(self):
        return self._geo()[2]

    @property
    def N(self) -> int:
        if self.qcrystal:
            return self.L
        return self.nsubs * self.L * self.L

    @property
    def Lsz(self) -> int:
        """Lattice length; for a quasi-crystal the even integer below
        sqrt(N), the side of its square q set (subrouts.cpp:1111)."""
        if self.qcrystal:
            return (int(math.sqrt(self.L)) // 2) * 2
        return self.L

    @property
    def G(self) -> int:
        return self.grid_fac * self.Lsz

    @property
    def size_tag(self) -> str:
        """SzTag of the table and sample file names (subrouts.cpp:1109)."""
        return f"_AppxtSz({self.L})" if self.qcrystal else ""

    @property
    def disorder(self) -> bool:
        return self.imp_ratio > 0.0

    @property
    def j2_on(self) -> bool:
        on = _is_not_zero(self.J2) or _is_not_zero(self.J2_delta)
        if self.disorder:
            on = on or _is_not_zero(self.J2ic) or _is_not_zero(self.J2ii)
        return on

    @property
    def jx_on(self) -> bool:
        on = _is_not_zero(self.JX)
        if self.disorder:
            on = on or _is_not_zero(self.JXic) or _is_not_zero(self.JXii)
        return on

    @property
    def pack_size(self) -> int:
        return self.NMeas // self.crSkip      # Codes_Folder/smd_code.cpp:978

    @property
    def temperature(self) -> float:
        if self.tpLstSz > 1:
            return self.T1 + self.tpIndex * (self.T2 - self.T1) / (self.tpLstSz - 1)
        return self.T1

    @property
    def out_label(self) -> str:
        """Output label, Codes_Folder/subrouts.cpp:2158-2185."""
        tag, val = {"Htag": ("_extH(", self.h), "J2tag": ("_J2(", self.J2),
                    "J1tag": ("_J1(", self.J1)}[self.outTag]
        return f"{tag}{val:.3f})"

    @property
    def t_tag(self) -> str:
        """``_T(%.5f)<label>``, Codes_Folder/smd_code.cpp:913-928."""
        return f"_T({self.temperature:.5f}){self.out_label}"

    def jmat(self):
        """3 x 2 x 2 couplings J[shell][a_i][a_j], Codes_Folder/subrouts.cpp:2093-2099."""
        if self.disorder:
            ic = (self.J1ic, self.J2ic, self.JXic)
            ii = (self.J1ii, self.J2ii, self.JXii)
        else:
            ic = ii = (0.0, 0.0, 0.0)
        cc = (self.J1, self.J2, self.JX)
        return [[[cc[s], ic[s]], [ic[s], ii[s]]] for s in range(3)]

    def lambdas(self):
        """lambdaVec1..3, Codes_Folder/subrouts.cpp:2112-2133."""
        if self.zlamb1 != 1.0 or self.zlamb2 != 1.0:
            l1 = (1.0, 1.0, self.zlamb1)
            l2 = (1.0, 1.0, self.zlamb2)
            return [l1, l2, l2]
        return [(1.0, 1.0, 1.0)] * 3

    # ----------------------------------------------------------- checks
    def validate(self, check_dwf: bool = True) -> None:
        """The input checks of convert_inputs2data and main that apply to SMD."""
        self._geo()
        if self.qcrystal:
            # smd_code.cpp:365-372: a quasi-crystal run needs PBC_OFF = 1 and
            # qct_RemovePBC = 0
            if self.flags.get("qct_RemovePBC", 0) or not self.flags.get("PBC_OFF", 0):
                raise SettingsError("qcrystal needs PBC_OFF = 1 and qct_RemovePBC = 0")
            if self.L < 4:
                raise SettingsError("quasi-crystal size too small")
        else:
            if self.L % 2:
                raise SettingsError("lattice length must be a multiple of 2")
            if self.geom not in ("square", "lieb") and self.L % 3:
                raise SettingsError("lattice length must be a multiple of 3")
        if _is_not_zero(self.J2_delta) and self.geom != "lieb":
            raise SettingsError("J2_delta requires the lieb geometry")
        if self.NMeas % BIN_SZ or self.NMeas // BIN_SZ == 1:
            raise SettingsError("NMeas must be a multiple of BinSz with more than one bin")
        if self.crSkip <= 0 or BIN_SZ % self.crSkip or self.crSkip > BIN_SZ:
            raise SettingsError("crSkip must divide BinSz")
        if self.ntm < 10:
            raise SettingsError("ntm too small")
        if self.dtm > 0.05:
            raise SettingsError("dtm too large")
        if self.window not in WINDOWS:
            raise SettingsError(f"invalid window {self.window!r}")
        if not (0.0 <= self.imp_ratio < 1.0):
            raise SettingsError("impurity ratio must lie in [0, 1)")
        if not (0 <= self.tpIndex < self.tpLstSz):
            raise SettingsError("tpIndex outside the temperature list")
        if self.temperature > TEMP_MAX:
            raise SettingsError("temperature exceeds TempMax")
        if check_dwf:
            dwf = 2.0 * math.pi / (self.ntm * self.dtm)
            if dwf > DWF_MIN:
                raise SettingsError(f"dwf = {dwf:.4f} exceeds dwf_min = {DWF_MIN}")

    # ------------------------------------------------------------- files
    def write(self, workdir: str) -> None:
        os.makedirs(workdir, exist_ok=True)

        def w(name, toks):
            with open(os.path.join(workdir, name), "w") as f:
                f.write("\n".join(str(t) for t in toks) + "\n")

        with open(os.path.join(workdir, "Settings_CodeExec.txt"), "w") as f:
            for k in CODE_SETTINGS:
                f.write(f"{k} {int(self.flags.get(k, 0))}\n")
        w("Settings_MODEL.txt", [self.L, repr(self.J1), repr(self.J2), repr(self.JX),
                                 repr(self.J2_delta), repr(self.zlamb1),
                                 repr(self.zlamb2), repr(self.h), repr(self.T1),
                                 repr(self.T2), self.geom])
        w("Settings_MC_SIM.txt", [self.NTerm, self.NMeas, self.IState, self.TpGrid,
                                  self.outTag, self.crSkip, self.vrSkip, self.MClive])
        w("Settings_SMD_SIM.txt", [self.ntm, self.tpLstSz, self.tpIndex,
                                   repr(self.dtm), self.window, self.RecVd1,
                                   self.RecVd2])
        w("Settings_Disorder.txt", [repr(self.imp_ratio), repr(self.J1ic),
                                    repr(self.J2ic), repr(self.JXic), repr(self.J1ii),
                                    repr(self.J2ii), repr(self.JXii)])

    @classmethod
    def read(cls, workdir: str) -> "SMDSettings":
        def toks(name, n):
            with open(os.path.join(workdir, name)) as f:
                t = f.read().split()
            if len(t) < n:
                raise SettingsError(f"{name}: expected {n} tokens")
            return t[:n]

        s = cls()
        flags = {}
        with open(os.path.join(workdir, "Settings_CodeExec.txt")) as f:
            t = f.read().split()
        if len(t) < 32:
            raise SettingsError("Settings_CodeExec.txt: expected 16 pairs")
        for i, k in enumerate(CODE_SETTINGS):
            v = int(t[2 * i + 1])
            if v not in (0, 1):
                raise SettingsError(f"invalid code-exec setting {t[2 * i]}")
            flags[k] = v
        s.flags = flags
        m = toks("Settings_MODEL.txt", 11)
        s.L = int(m[0])
        s.J1, s.J2, s.JX, s.J2_delta = map(float, m[1:5])
        s.zlamb1, s.zlamb2, s.h, s.T1, s.T2 = map(float, m[5:10])
        s.geom = m[10]
        c = toks("Settings_MC_SIM.txt", 8)
        s.NTerm, s.NMeas = int(c[0]), int(c[1])
        s.IState, s.TpGrid, s.outTag = c[2], c[3], c[4]
        s.crSkip, s.vrSkip, s.MClive = int(c[5]), int(c[6]), int(c[7])
        d = toks("Settings_SMD_SIM.txt", 7)
        s.ntm, s.tpLstSz, s.tpIndex = int(d[0]), int(d[1]), int(d[2])
        s.dtm, s.window = float(d[3]), d[4]
        s.RecVd1, s.RecVd2 = int(d[5]), int(d[6])
        r = toks("Settings_Disorder.txt", 7)
        (s.imp_ratio, s.J1ic, s.J2ic, s.JXic, s.J1ii, s.J2ii,
         s.JXii) = map(float, r)
        return s
