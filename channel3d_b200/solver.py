"""Host-side mirror of the reference's ChannelInitialize / ChannelIterate
(src/CFD_2nd/m_ChannelSystem.f90:28-154) over the C ABI of libch3d.so.

Arrays are numpy float64, C-order shape (nzc, nyc, nxc), which is the
memory order of the reference's Fortran (nxc, nyc, nzc) arrays.
"""
import ctypes

import numpy as np

from . import _lib
from .config import mesh_y


class ChannelSolver:
    # ch3d_get_array ids (include/ch3d.h)
    UX, UY, UZ, P, HISTX, HISTY, HISTZ, RHSX, RHSY, PRPHI, NUT, RHSZ = 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11

    def __init__(self, cfg, yp=None):
        self.lib = _lib.load_library()
        self.cfg = cfg
        self.yp = np.ascontiguousarray(mesh_y(cfg, self.lib) if yp is None else yp, dtype=np.float64)
        self._c = cfg.to_c()
        h = ctypes.c_void_p()
        _lib.check(self.lib.ch3d_create(ctypes.byref(self._c), _lib.dptr(self.yp), ctypes.byref(h)), self.lib)
        self.ctx = h

    def close(self):
        if self.ctx:
            self.lib.ch3d_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _arr(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.size == self.cfg.npoints, "array size does not match the grid"
        return a

    def layout_shape(self, layout):
        """C-order shape of a host array of the given layout: interior
        (nzc, nyc, nxc); GHOST2 the 2nd-order bounds (0:nxc+2, 0:nyc+2,
        0:nzc+2); GHOST4 the 4th-order bounds (-1:nxc+2, 0:nyc+1, -1:nzc+2)."""
        nx, ny, nz = self.cfg.nxc, self.cfg.nyc, self.cfg.nzc
        if layout == _lib.LAYOUT_GHOST2:
            return (nz + 3, ny + 3, nx + 3)
        if layout == _lib.LAYOUT_GHOST4:
            return (nz + 4, ny + 2, nx + 4)
        return (nz, ny, nx)

    def upload(self, ux, uy, uz, p, hist=None, layout=_lib.LAYOUT_INTERIOR):
        n = int(np.prod(self.layout_shape(layout)))
        fields = [np.ascontiguousarray(a, dtype=np.float64) for a in (ux, uy, uz, p)]
        assert all(a.size == n for a in fields), "array size does not match the layout"
        h = None
        if hist is not None:
            h = np.ascontiguousarray(np.stack([self._arr(a) for a in hist]))
        _lib.check(self.lib.ch3d_upload_state(self.ctx, int(layout), *(_lib.dptr(a) for a in fields), _lib.dptr(h)),
                   self.lib)

    def download(self, hist=False, layout=_lib.LAYOUT_INTERIOR, out=None):
        """Current state as {"ux", "uy", "uz", "p"[, "hist"]}.  With a ghosted
        layout the ghost cells follow the reference's boundary and halo rules;
        `out` may give the host arrays (their cells outside the rules keep
        their values), else they start at zero."""
        shp = self.layout_shape(layout)
        if out is None:
            out = {k: np.zeros(shp) for k in ("ux", "uy", "uz", "p")}
        for k in ("ux", "uy", "uz", "p"):
            a = out[k]
            assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"] and a.size == int(np.prod(shp))
        h = np.empty((3,) + self.cfg.shape) if hist else None
        _lib.check(self.lib.ch3d_download_state(self.ctx, int(layout), *(_lib.dptr(out[k]) for k in ("ux", "uy", "uz",
                                                                                                      "p")),
                                                _lib.dptr(h)), self.lib)
        if hist:
            out["hist"] = h
        return out

    def step(self, n=1, raise_on_diverge=True):
        info = _lib.Ch3dStepInfo()
        rc = self.lib.ch3d_step(self.ctx, int(n), ctypes.byref(info))
        if rc == _lib.CH3D_ERR_DIVERGED and not raise_on_diverge:
            return info.as_dict()
        _lib.check(rc, self.lib)
        return info.as_dict()

    def stage(self, st, ns):
        _lib.check(self.lib.ch3d_stage(self.ctx, int(st), int(ns)), self.lib)

    def get_array(self, which):
        out = np.empty(self.cfg.shape)
        _lib.check(self.lib.ch3d_get_array(self.ctx, int(which), _lib.dptr(out)), self.lib)
        return out

    def set_array(self, which, a):
        a = self._arr(a)
        _lib.check(self.lib.ch3d_set_array(self.ctx, int(which), _lib.dptr(a)), self.lib)

    def poisson(self, src):
        src = self._arr(src)
        phi = np.empty(self.cfg.shape)
        _lib.check(self.lib.ch3d_poisson(self.ctx, _lib.dptr(src), _lib.dptr(phi)), self.lib)
        return phi

    def project(self):
        b, a = ctypes.c_double(), ctypes.c_double()
        _lib.check(self.lib.ch3d_project(self.ctx, ctypes.byref(b), ctypes.byref(a)), self.lib)
        return b.value, a.value

    def memory_bytes(self):
        v = ctypes.c_longlong()
        _lib.check(self.lib.ch3d_memory_bytes(self.ctx, ctypes.byref(v)), self.lib)
        return v.value

    def sgs_viscosity(self):
        """LES: nut from the current velocity (Clc_SGS_Vis); returns it (interior)."""
        _lib.check(self.lib.ch3d_sgs_viscosity(self.ctx))
        return self.get_array(self.NUT)

    def sgs_mlp_set(self, params, norm):
        """Learned closure: network parameters (9414 FP32) and standardisation (52 FP32)."""
        p = np.ascontiguousarray(params, dtype=np.float32)
        n = np.ascontiguousarray(norm, dtype=np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        _lib.check(self.lib.ch3d_sgs_mlp_set(self.ctx, p.ctypes.data_as(fp), n.ctypes.data_as(fp)), self.lib)

    def sgs_training_samples(self, fx, fy, fz):
        """Box-filtered training samples of the current field: (X [n x 10], T [n x 6]) device tensors."""
        import torch
        nb = (self.cfg.nxc // fx) * (self.cfg.nyc // fy) * (self.cfg.nzc // fz)
        dev = torch.device("cuda", self.cfg.device)
        X = torch.empty((nb, 10), dtype=torch.float32, device=dev)
        T = torch.empty((nb, 6), dtype=torch.float32, device=dev)
        n = ctypes.c_longlong()
        _lib.check(self.lib.ch3d_sgs_training_samples(self.ctx, fx, fy, fz, X.data_ptr(), T.data_ptr(),
                                                      ctypes.byref(n)), self.lib)
        return X[:n.value], T[:n.value]

    def stats_accumulate(self):
        _lib.check(self.lib.ch3d_stats_accumulate(self.ctx), self.lib)

    def stats_fetch(self, reset=False):
        """(SumStat as (nyp, 35), nfstime, PrGradsum)."""
        s = np.empty((self.cfg.nyc + 1) * 35)
        n = ctypes.c_int()
        pg = ctypes.c_double()
        _lib.check(self.lib.ch3d_stats_fetch(self.ctx, _lib.dptr(s), ctypes.byref(n), ctypes.byref(pg), int(reset)),
                   self.lib)
        return s.reshape(self.cfg.nyc + 1, 35), n.value, pg.value

    def interp_from(self, src):
        """Resamples another solver's state onto this grid (the reference's
        interpolateField tool, Interp_uvwp) and makes it this solver's state."""
        _lib.check(self.lib.ch3d_interp_state(self.ctx, src.ctx), self.lib)

    def spectra_accumulate(self, jfor=(1, 1)):
        """4th order: one sample of the 1-D spectra (clcSpectra1D) with the
        coherence spectra against rows jForLCS(1:2) (1-based)."""
        _lib.check(self.lib.ch3d_spectra_accumulate(self.ctx, int(jfor[0]), int(jfor[1])), self.lib)

    def spectra_fetch(self, reset=False, two_d=False):
        """(EnergySpecX as (18, nyc, nxc/2+1), EnergySpecZ as (18, nyc, nzc/2+1), nSpectime),
        with two_d also EnergySpec2D as (9, nzc/2+1, nyc/2, nxc/2+1) before nSpectime."""
        c = self.cfg
        sx = np.empty((18, c.nyc, c.nxc // 2 + 1))
        sz = np.empty((18, c.nyc, c.nzc // 2 + 1))
        s2 = np.empty((9, c.nzc // 2 + 1, c.nyc // 2, c.nxc // 2 + 1)) if two_d else None
        n = ctypes.c_int()
        _lib.check(self.lib.ch3d_spectra_fetch(self.ctx, _lib.dptr(sx), _lib.dptr(sz), _lib.dptr(s2), ctypes.byref(n),
                                               int(reset)), self.lib)
        return (sx, sz, s2, n.value) if two_d else (sx, sz, n.value)

    def stats_fetch_grad(self):
        """4th order: SumGrad(98, nyp) as (nyp, 98) (the vGrad moment sums)."""
        g = np.empty((self.cfg.nyc + 1) * 98)
        _lib.check(self.lib.ch3d_stats_fetch_grad(self.ctx, _lib.dptr(g)), self.lib)
        return g.reshape(self.cfg.nyc + 1, 98)

    def dissipation(self):
        """clcStat_TG (src/CFD_2nd/m_FlowType_TGVortex.f90:87-113): xnu times the
        mean over the cells of CalcDissipationRate, 2 S_ij S_ij, of the current field."""
        v = np.zeros(1)
        _lib.check(self.lib.ch3d_dissipation(self.ctx, _lib.dptr(v)), self.lib)
        return float(v[0])

    def kernel_times(self, nsteps=1):
        out = np.zeros(7)
        _lib.check(self.lib.ch3d_kernel_times(self.ctx, int(nsteps), _lib.dptr(out), 7), self.lib)
        return out

    def last_step_ms(self):
        v = ctypes.c_double()
        _lib.check(self.lib.ch3d_last_step_ms(self.ctx, ctypes.byref(v)), self.lib)
        return v.value

    def path_flags(self):
        """Kernel layout of the step: a set of "march", "twisted", "gsub"
        (CH3D_PATH_* of include/ch3d.h)."""
        v = ctypes.c_int()
        _lib.check(self.lib.ch3d_path_flags(self.ctx, ctypes.byref(v)), self.lib)
        return {n for bit, n in ((1, "march"), (2, "twisted"), (4, "gsub")) if v.value & bit}
