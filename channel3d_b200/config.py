"""Run configuration: the reference's .prm namelists, read unchanged.

The reference reads &BasicParam and &LesOptions in ReadAndInitParameters
(src/CFD_2nd/m_Parameters.f90:267-308), &ubulk_Param in InitTimeScheme
(src/CFD_2nd/m_TScheme.f90:40-57) and &MeshSection/&MeshOptions in
InitMeshAndMetries (src/CFD_2nd/m_MeshAndMetries.f90:122-143).  One optional
namelist, &GpuOptions (precision, device), is read here and ignored by the
reference.
"""
import dataclasses
import re
from dataclasses import dataclass, field
from typing import List

import numpy as np

from . import _lib


@dataclass
class ChannelConfig:
    order: int = 2
    FlowType: int = 1
    xlx: float = 2 * np.pi
    yly: float = 2.0
    zlz: float = np.pi
    nxc: int = 64
    nyc: int = 64
    nzc: int = 64
    xnu: float = 2.0 / 5600.0
    dtMax: float = 0.002
    iCFL: int = 2
    CFLc: float = 1.0
    ifirst: int = 1
    ilast: int = 200
    ischeme: int = 3
    IsImplicit: int = 1
    FFTW_plan_type: int = 2
    BcOption: List[int] = field(default_factory=lambda: [0, 0, -1, -1, 0, 0])
    uxBcValue: List[float] = field(default_factory=lambda: [0.0] * 6)
    uyBcValue: List[float] = field(default_factory=lambda: [0.0] * 6)
    uzBcValue: List[float] = field(default_factory=lambda: [0.0] * 6)
    gravity: List[float] = field(default_factory=lambda: [0.0] * 3)
    ivstats: int = 20
    SaveStat: int = 2500
    SaveVisu: int = 5000
    BackupFreq: int = 10000
    RestartFlag: bool = True
    RunName: str = "channel"
    ResultsDir: str = "./CFD/Results/"
    RestartDir: str = "./CFD/Restart/"
    vel_limit: float = 2.0
    div_limit: float = 0.2
    # &ubulk_Param
    IsUxConst: bool = True
    IsUbulkGlobal: bool = True
    ubulk: float = 1.0
    ybulk1: float = 0.0
    ybulk2: float = 2.0
    # &LesOptions
    LES_type: int = 0
    FilterType: int = 1
    Cs: float = 0.1
    # &MeshSection / &MeshOptions
    nSection: int = 2
    SectionLength: List[float] = field(default_factory=lambda: [1.0, 1.0])
    nycSection: List[int] = field(default_factory=lambda: [32, 32])
    StretType: List[int] = field(default_factory=lambda: [1, 1])
    StretOption: List[int] = field(default_factory=lambda: [0, 1])
    SectioncStret: List[float] = field(default_factory=lambda: [2.0, 2.0])
    # &GpuOptions
    precision: str = "fp64"
    device: int = 0

    def copy(self, **kw):
        return dataclasses.replace(self, **kw)

    @property
    def shape(self):
        """(nzc, nyc, nxc): numpy C-order shape of a Fortran (nxc,nyc,nzc) array."""
        return (self.nzc, self.nyc, self.nxc)

    @property
    def npoints(self):
        return self.nxc * self.nyc * self.nzc

    def effective_ybulk(self):
        # InitTimeScheme: IsUbulkGlobal overrides ybulk1/2 (src/CFD_2nd/m_TScheme.f90:53-55)
        if self.IsUbulkGlobal:
            return 0.0, self.yly
        return self.ybulk1, self.ybulk2

    def to_c(self):
        c = _lib.Ch3dConfig()
        c.order = self.order
        c.nxc, c.nyc, c.nzc = self.nxc, self.nyc, self.nzc
        c.xlx, c.yly, c.zlz = self.xlx, self.yly, self.zlz
        c.xnu = self.xnu
        c.dtMax = self.dtMax
        c.iCFL = self.iCFL
        c.CFLc = self.CFLc
        c.ischeme = self.ischeme
        c.IsImplicit = self.IsImplicit
        c.FlowType = self.FlowType
        for q in range(6):
            c.BcOption[q] = int(self.BcOption[q])
            c.uxBcValue[q] = float(self.uxBcValue[q])
            c.uyBcValue[q] = float(self.uyBcValue[q])
            c.uzBcValue[q] = float(self.uzBcValue[q])
        for q in range(3):
            c.gravity[q] = float(self.gravity[q])
        c.IsUxConst = int(bool(self.IsUxConst))
        c.ubulk = self.ubulk
        c.ybulk1, c.ybulk2 = self.effective_ybulk()
        c.LES_type = self.LES_type
        c.FilterType = self.FilterType
        c.Cs = self.Cs
        c.vel_limit = self.vel_limit
        c.div_limit = self.div_limit
        c.precision = _lib.PREC_MIXED if self.precision == "mixed" else _lib.PREC_FP64
        c.device = self.device
        return c

    @classmethod
    def from_prm(cls, path, **overrides):
        nml = parse_namelists(open(path).read())
        cfg = cls()
        names = {f.name: f for f in dataclasses.fields(cls)}
        for group in ("basicparam", "ubulk_param", "lesoptions", "meshsection", "meshoptions", "gpuoptions"):
            for key, val in nml.get(group, {}).items():
                for n in names:
                    if n.lower() == key:
                        setattr(cfg, n, _coerce(val, getattr(cfg, n)))
        for k, v in overrides.items():
            setattr(cfg, k, v)
        return cfg


def _coerce(val, like):
    if isinstance(like, list):
        vals = val if isinstance(val, list) else [val]
        elem = like[0] if like else 0.0
        return [type(elem)(v) if not isinstance(elem, bool) else bool(v) for v in vals]
    v = val[0] if isinstance(val, list) else val
    if isinstance(like, bool):
        return bool(v)
    if isinstance(like, int):
        return int(v)
    if isinstance(like, float):
        return float(v)
    return str(v)


_TOKEN = re.compile(r"""'[^']*'|"[^"]*"|[^\s,]+""")


def _parse_value(tok):
    t = tok.strip()
    if (t.startswith("'") and t.endswith("'")) or (t.startswith('"') and t.endswith('"')):
        return t[1:-1]
    tl = t.lower()
    if tl in ("t", ".true.", "true", ".t."):
        return True
    if tl in ("f", ".false.", "false", ".f."):
        return False
    try:
        if re.fullmatch(r"[+-]?\d+", t):
            return int(t)
        return float(tl.replace("d", "e"))
    except ValueError:
        return t


def parse_namelists(text):
    """Minimal Fortran namelist reader: groups -> {lowercase key: value or list}."""
    out = {}
    lines = []
    for raw in text.splitlines():
        s = raw
        # strip comments outside quotes
        q = None
        for idx, ch in enumerate(s):
            if ch in "'\"":
                q = None if q == ch else (ch if q is None else q)
            elif ch == "!" and q is None:
                s = s[:idx]
                break
        if s.strip().startswith("/"):
            s = "/"  # namelist terminator; the rest of the line is free text
        lines.append(s)
    text = "\n".join(lines)
    for m in re.finditer(r"&(\w+)(.*?)(?:^|\s)/", text, flags=re.S | re.M):
        group = m.group(1).lower()
        body = m.group(2)
        items = {}
        for km in re.finditer(r"(\w+)\s*=\s*(.*?)(?=(?:\b\w+\s*=)|\Z)", body, flags=re.S):
            key = km.group(1).lower()
            toks = _TOKEN.findall(km.group(2))
            vals = []
            for t in toks:
                rep = re.fullmatch(r"(\d+)\*(.+)", t)
                if rep:
                    vals.extend([_parse_value(rep.group(2))] * int(rep.group(1)))
                else:
                    vals.append(_parse_value(t))
            items[key] = vals[0] if len(vals) == 1 else vals
        out[group] = items
    return out


def mesh_y(cfg, lib=None):
    """yp(1:nyp) from the mesh sections, computed by the library (clcCoord)."""
    lib = lib or _lib.load_library()
    n = cfg.nSection
    yp = np.zeros(cfg.nyc + 1)
    SL = np.asarray(cfg.SectionLength[:n], dtype=np.float64)
    SC = np.asarray(cfg.SectioncStret[:n], dtype=np.float64)
    NY = np.asarray(cfg.nycSection[:n], dtype=np.int32)
    ST = np.asarray(cfg.StretType[:n], dtype=np.int32)
    SO = np.asarray(cfg.StretOption[:n], dtype=np.int32)
    ip = lambda a: a.ctypes.data_as(_lib._IP)
    _lib.check(lib.ch3d_mesh_y(cfg.nyc, cfg.yly, n, _lib.dptr(SL), ip(NY), ip(ST), ip(SO), _lib.dptr(SC),
                               _lib.dptr(yp)), lib)
    return yp
