"""ctypes wrapper of the CPU oracle (oracle/ch3d_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker and by bench.py's CPU-baseline leg.  Parity against reference
runs is UNPINNED (no Fortran compiler here; the reference ships no tests or
golden vectors); known-answer tests in tests/ pin the restatement instead.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libch3d_oracle.so")

_D6 = ctypes.c_double * 6
_I6 = ctypes.c_int * 6
_D3 = ctypes.c_double * 3
_D8 = ctypes.c_double * 8
_I8 = ctypes.c_int * 8
_DP = ctypes.POINTER(ctypes.c_double)


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("order", ctypes.c_int), ("nxc", ctypes.c_int), ("nyc", ctypes.c_int), ("nzc", ctypes.c_int),
        ("xlx", ctypes.c_double), ("yly", ctypes.c_double), ("zlz", ctypes.c_double),
        ("xnu", ctypes.c_double), ("dtMax", ctypes.c_double), ("iCFL", ctypes.c_int), ("CFLc", ctypes.c_double),
        ("ischeme", ctypes.c_int), ("IsImplicit", ctypes.c_int), ("FlowType", ctypes.c_int),
        ("BcOption", _I6), ("uxBcValue", _D6), ("uyBcValue", _D6), ("uzBcValue", _D6), ("gravity", _D3),
        ("IsUxConst", ctypes.c_int), ("ubulk", ctypes.c_double), ("ybulk1", ctypes.c_double),
        ("ybulk2", ctypes.c_double), ("LES_type", ctypes.c_int), ("FilterType", ctypes.c_int),
        ("Cs", ctypes.c_double), ("vel_limit", ctypes.c_double), ("div_limit", ctypes.c_double),
        ("nSection", ctypes.c_int), ("SectionLength", _D8), ("SectioncStret", _D8), ("nycSection", _I8),
        ("StretType", _I8), ("StretOption", _I8),
    ]


class OrcInfo(ctypes.Structure):
    _fields_ = [
        ("SimTime", ctypes.c_double), ("dt", ctypes.c_double), ("cflmp", ctypes.c_double),
        ("divmax1", ctypes.c_double), ("divmax2", ctypes.c_double), ("vmax", _D3), ("uxm", ctypes.c_double),
        ("PrGradAver", ctypes.c_double), ("itime", ctypes.c_int), ("status", ctypes.c_int),
    ]

    def as_dict(self):
        return {"SimTime": self.SimTime, "dt": self.dt, "cflmp": self.cflmp, "divmax1": self.divmax1,
                "divmax2": self.divmax2, "vmax": list(self.vmax), "uxm": self.uxm,
                "PrGradAver": self.PrGradAver, "itime": self.itime, "status": self.status}


_lib = None


def build():
    """Compiles the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.POINTER(OrcParams)]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_state.argtypes = [ctypes.c_void_p, _DP, _DP, _DP, _DP, _DP]
        L.orc_get_state.argtypes = [ctypes.c_void_p, _DP, _DP, _DP, _DP, _DP]
        L.orc_get_array.restype = ctypes.c_longlong
        L.orc_get_array.argtypes = [ctypes.c_void_p, ctypes.c_int, _DP]
        L.orc_set_array.restype = ctypes.c_longlong
        L.orc_set_array.argtypes = [ctypes.c_void_p, ctypes.c_int, _DP]
        L.orc_stage.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_step.restype = ctypes.c_int
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(OrcInfo)]
        L.orc_poisson.argtypes = [ctypes.c_void_p, _DP, _DP]
        L.orc_r2hc.argtypes = [ctypes.c_int, _DP]
        L.orc_redft10.argtypes = [ctypes.c_int, _DP]
        L.orc_redft01.argtypes = [ctypes.c_int, _DP]
        L.orc_hc2r.argtypes = [ctypes.c_int, _DP]
        L.orc_get_mesh.argtypes = [ctypes.c_void_p, _DP, _DP, _DP, _DP]
        L.orc_set_dt.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.orc_stats_accumulate.argtypes = [ctypes.c_void_p]
        L.orc_stats_get.restype = ctypes.c_int
        L.orc_stats_get.argtypes = [ctypes.c_void_p, _DP, _DP]
        L.orc_stats_get_grad.restype = ctypes.c_int
        L.orc_stats_get_grad.argtypes = [ctypes.c_void_p, _DP]
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_sgs.restype = ctypes.c_double
        L.orc_sgs.argtypes = [ctypes.c_void_p]
        L.orc_set_sgs_tau.argtypes = [ctypes.c_void_p, _DP]
        L.orc_set_num_threads.argtypes = [ctypes.c_int]
        L.orc_interp.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_spectra_accumulate.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_spectra_get.restype = ctypes.c_int
        L.orc_spectra_get.argtypes = [ctypes.c_void_p, _DP, _DP]
        L.orc_spectra_get2d.restype = ctypes.c_int
        L.orc_spectra_get2d.argtypes = [ctypes.c_void_p, _DP]
        L.orc_dissipation.argtypes = [ctypes.c_void_p]
        L.orc_dissipation.restype = ctypes.c_double
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_DP)


def params_from(cfg):
    """OrcParams from any object with the ChannelConfig attribute names."""
    P = OrcParams()
    P.order = cfg.order
    P.nxc, P.nyc, P.nzc = cfg.nxc, cfg.nyc, cfg.nzc
    P.xlx, P.yly, P.zlz = cfg.xlx, cfg.yly, cfg.zlz
    P.xnu, P.dtMax, P.iCFL, P.CFLc = cfg.xnu, cfg.dtMax, cfg.iCFL, cfg.CFLc
    P.ischeme, P.IsImplicit, P.FlowType = cfg.ischeme, cfg.IsImplicit, cfg.FlowType
    for q in range(6):
        P.BcOption[q] = int(cfg.BcOption[q])
        P.uxBcValue[q], P.uyBcValue[q], P.uzBcValue[q] = cfg.uxBcValue[q], cfg.uyBcValue[q], cfg.uzBcValue[q]
    for q in range(3):
        P.gravity[q] = cfg.gravity[q]
    P.IsUxConst = int(bool(cfg.IsUxConst))
    P.ubulk = cfg.ubulk
    if getattr(cfg, "IsUbulkGlobal", True):
        P.ybulk1, P.ybulk2 = 0.0, cfg.yly
    else:
        P.ybulk1, P.ybulk2 = cfg.ybulk1, cfg.ybulk2
    P.LES_type, P.FilterType, P.Cs = cfg.LES_type, cfg.FilterType, cfg.Cs
    P.vel_limit, P.div_limit = cfg.vel_limit, cfg.div_limit
    P.nSection = cfg.nSection
    for q in range(cfg.nSection):
        P.SectionLength[q] = cfg.SectionLength[q]
        P.SectioncStret[q] = cfg.SectioncStret[q]
        P.nycSection[q] = cfg.nycSection[q]
        P.StretType[q] = cfg.StretType[q]
        P.StretOption[q] = cfg.StretOption[q]
    return P


class Oracle:
    # orc_get_array ids
    UX, UY, UZ, P, HISTX, HISTY, HISTZ, ARR1, ARR2, HALO, NUT = range(11)

    def __init__(self, cfg):
        self.L = lib()
        self.cfg = cfg
        self.params = params_from(cfg)
        self.h = self.L.orc_create(ctypes.byref(self.params))
        if not self.h:
            raise ValueError("oracle rejected the configuration")
        self.shape = (cfg.nzc, cfg.nyc, cfg.nxc)

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def mesh(self):
        n = self.cfg.nyc + 1
        yp, yc, dyp, dyc = (np.zeros(n) for _ in range(4))
        self.L.orc_get_mesh(self.h, _p(yp), _p(yc), _p(dyp), _p(dyc))
        return yp, yc, dyp, dyc

    def set_state(self, ux, uy, uz, p, hist=None):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (ux, uy, uz, p)]
        h = None if hist is None else np.ascontiguousarray(np.stack(hist), dtype=np.float64)
        self.L.orc_set_state(self.h, *(_p(x) for x in a), _p(h))

    def get_state(self, hist=False):
        out = [np.empty(self.shape) for _ in range(4)]
        h = np.empty((3,) + self.shape) if hist else None
        self.L.orc_get_state(self.h, *(_p(x) for x in out), _p(h))
        d = dict(zip(("ux", "uy", "uz", "p"), out))
        if hist:
            d["hist"] = h
        return d

    def get_ghosted(self, which):
        n = self.L.orc_get_array(self.h, which, None)
        out = np.empty(n)
        self.L.orc_get_array(self.h, which, _p(out))
        return out

    def get_interior(self, which):
        """Interior block of an oracle array as (nzc, nyc, nxc)."""
        a = self.get_ghosted(which)
        nx, ny, nz = self.cfg.nxc, self.cfg.nyc, self.cfg.nzc
        if a.size == nx * ny * nz:
            return a.reshape(nz, ny, nx)
        if self.cfg.order == 4:  # (-1:nxc+2, 0:nyc+1, -1:nzc+2)
            g = a.reshape(nz + 4, ny + 2, nx + 4)
            return np.ascontiguousarray(g[2:nz + 2, 1:ny + 1, 2:nx + 2])
        g = a.reshape(nz + 3, ny + 3, nx + 3)   # (0:nxc+2, 0:nyc+2, 0:nzc+2)
        return np.ascontiguousarray(g[1:nz + 1, 1:ny + 1, 1:nx + 1])

    def interp_from(self, src):
        """Resamples src's state onto this grid (the interpolateField tool's
        Interp_uvwp); it becomes this oracle's state."""
        self.L.orc_interp(self.h, src.h)

    def stage(self, st, ns):
        self.L.orc_stage(self.h, st, ns)

    def step(self, n=1):
        info = OrcInfo()
        st = self.L.orc_step(self.h, n, ctypes.byref(info))
        d = info.as_dict()
        d["rc"] = st
        return d

    def poisson(self, src):
        src = np.ascontiguousarray(src, dtype=np.float64)
        phi = np.empty(self.shape)
        self.L.orc_poisson(self.h, _p(src), _p(phi))
        return phi

    def sgs(self):
        """Clc_SGS_Vis on the current state: nut (interior) and u_tau."""
        ut = self.L.orc_sgs(self.h)
        return self.get_interior(self.NUT), ut

    def set_sgs_tau(self, tau):
        """Learned closure: cell-centred SGS stresses (6, nzc, nyc, nxc) whose divergence the LES RHS adds."""
        if tau is None:
            self.L.orc_set_sgs_tau(self.h, None)
            return
        t = np.ascontiguousarray(tau, dtype=np.float64)
        assert t.size == 6 * self.cfg.nxc * self.cfg.nyc * self.cfg.nzc
        self.L.orc_set_sgs_tau(self.h, _p(t))

    def stats_accumulate(self):
        self.L.orc_stats_accumulate(self.h)

    def stats_get(self):
        s = np.empty(35 * (self.cfg.nyc + 1))
        pg = ctypes.c_double()
        n = self.L.orc_stats_get(self.h, _p(s), ctypes.byref(pg))
        return s.reshape(self.cfg.nyc + 1, 35), n, pg.value

    def spectra_accumulate(self, jfor=(1, 1)):
        """4th order: one sample of the 1-D spectra (clcSpectra1D) with the
        linear coherence spectra against rows jForLCS(1:2) (1-based)."""
        self.L.orc_spectra_accumulate(self.h, int(jfor[0]), int(jfor[1]))

    def spectra_get(self):
        """(EnergySpecX as (18, nyc, nxc/2+1), EnergySpecZ as (18, nyc, nzc/2+1), nSpectime)."""
        c = self.cfg
        sx = np.empty((18, c.nyc, c.nxc // 2 + 1))
        sz = np.empty((18, c.nyc, c.nzc // 2 + 1))
        n = self.L.orc_spectra_get(self.h, _p(sx), _p(sz))
        return sx, sz, n

    def spectra_get2d(self):
        """EnergySpec2D as (9, nzc/2+1, nyc/2, nxc/2+1), and nSpectime."""
        c = self.cfg
        s2 = np.empty((9, c.nzc // 2 + 1, c.nyc // 2, c.nxc // 2 + 1))
        n = self.L.orc_spectra_get2d(self.h, _p(s2))
        return s2, n

    def dissipation(self):
        """clcStat_TG's value: xnu * mean over the cells of CalcDissipationRate."""
        return float(lib().orc_dissipation(self.h))

    def stats_get_grad(self):
        """4th order: SumGrad(98, nyp) as (nyp, 98), and nfstime."""
        g = np.empty(98 * (self.cfg.nyc + 1))
        n = self.L.orc_stats_get_grad(self.h, _p(g))
        return g.reshape(self.cfg.nyc + 1, 98), n


def r2hc(x):
    y = np.array(x, dtype=np.float64)
    lib().orc_r2hc(y.size, _p(y))
    return y


def hc2r(x):
    y = np.array(x, dtype=np.float64)
    lib().orc_hc2r(y.size, _p(y))
    return y


def redft10(x):
    y = np.array(x, dtype=np.float64)
    lib().orc_redft10(y.size, _p(y))
    return y


def redft01(x):
    y = np.array(x, dtype=np.float64)
    lib().orc_redft01(y.size, _p(y))
    return y


def set_threads(n):
    lib().orc_set_num_threads(int(n))


def num_threads():
    return lib().orc_num_threads()
