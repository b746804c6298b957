"""Known-answer tests that pin the CPU oracle (no reference runs exist)."""
import numpy as np
import pytest

from helpers import rel_l2, small_channel


def test_r2hc_matches_dft(built):
    from oracle import oracle as O
    rng = np.random.default_rng(0)
    for n in (2, 3, 4, 6, 8, 9, 12, 16, 24, 36, 48, 64, 96, 5, 7, 10, 15, 384, 576):
        x = rng.standard_normal(n)
        k = np.arange(n)
        X = np.exp(-2j * np.pi * np.outer(k, k) / n) @ x  # naive DFT
        hc = O.r2hc(x)
        ref = np.zeros(n)
        ref[: n // 2 + 1] = X.real[: n // 2 + 1]
        for q in range(1, (n + 1) // 2):
            ref[n - q] = X.imag[q]
        assert np.abs(hc - ref).max() < 1e-12 * max(1.0, np.abs(X).max()), n
        assert np.abs(O.hc2r(hc) / n - x).max() < 1e-13, n


def _laplacian(cfg, o, phi):
    """Discrete operator of the Poisson solve (src/CFD_2nd/m_Poisson.f90): 3-point
    second differences in x and z (periodic) and [am2Pr, ac2Pr, ap2Pr] in y."""
    yp, yc, dyp, dyc = o.mesh()
    ny = cfg.nyc
    dyp_ = yp[1:] - yp[:-1]
    yc_ = 0.5 * (yp[1:] + yp[:-1])
    dyc_ = np.empty(ny + 1)
    dyc_[1:ny] = yc_[1:] - yc_[:-1]
    dyc_[0] = dyp_[0]
    dyc_[ny] = dyp_[-1]
    am = 1 / dyp_ / dyc_[:ny]
    ap = 1 / dyp_ / dyc_[1:]
    am[0] = 0.0
    ap[-1] = 0.0
    ac = -(am + ap)
    rdx2 = (cfg.nxc / cfg.xlx) ** 2
    rdz2 = (cfg.nzc / cfg.zlz) ** 2
    L = (np.roll(phi, 1, 2) - 2 * phi + np.roll(phi, -1, 2)) * rdx2
    L += (np.roll(phi, 1, 0) - 2 * phi + np.roll(phi, -1, 0)) * rdz2
    pm = np.concatenate([phi[:, :1], phi[:, :-1]], axis=1)
    pp = np.concatenate([phi[:, 1:], phi[:, -1:]], axis=1)
    L += am[None, :, None] * pm + ac[None, :, None] * phi + ap[None, :, None] * pp
    return L


def test_poisson_residual(built):
    from oracle import oracle as O
    cfg = small_channel(24, 20, 12)
    o = O.Oracle(cfg)
    src = np.random.default_rng(3).standard_normal(cfg.shape)
    phi = o.poisson(src)
    r = _laplacian(cfg, o, phi) - src
    # the (kx,kz)=(0,0) system has its first row replaced by phi_hat = 0
    # (m_Poisson.f90:1136-1140): the residual is a plane constant at j=1 only
    rm = r.mean(axis=(0, 2))
    assert np.abs(r - rm[None, :, None]).max() < 1e-9 * np.abs(src).max()
    assert np.abs(rm[1:]).max() < 1e-9 * np.abs(src).max()
    assert abs(phi[:, 0, :].mean()) < 1e-12 * np.abs(phi).max()


def test_step_is_divergence_free_and_deterministic(built):
    from channel3d_b200 import initfield
    from oracle import oracle as O
    cfg = small_channel(32, 24, 16)
    o = O.Oracle(cfg)
    yp = o.mesh()[0]
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp)
    O.set_threads(1)
    o.set_state(ux, uy, uz, p)
    d = o.step(3)
    a = o.get_state()
    assert d["divmax2"] < 1e-13 and d["rc"] == 0
    O.set_threads(4)
    o.set_state(ux, uy, uz, p)
    o.step(3)
    b = o.get_state()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_laminar_stays_laminar(built):
    """A parabolic profile with v = w = 0 keeps v = w = 0 and stays uniform in x, z."""
    from channel3d_b200 import initfield
    from oracle import oracle as O
    cfg = small_channel(16, 24, 8)
    o = O.Oracle(cfg)
    yp = o.mesh()[0]
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp, amplitude=0.0)
    o.set_state(ux, uy, uz, p)
    d = o.step(5)
    s = o.get_state()
    assert np.abs(s["uy"]).max() < 1e-13 and np.abs(s["uz"]).max() < 1e-13
    assert np.abs(s["ux"] - s["ux"][:1, :, :1]).max() < 1e-13
    assert abs(d["uxm"] - 1.0) < 1e-3


def test_nan_field_is_skipped_by_the_reference_limit_checks(built):
    """The reference's maxima (`if(udiv>divmax1)`, m_Tools.f90:70; CalcVmax :93-98)
    skip NaN, so a NaN field does not trip div_limit/vel_limit there; the GPU
    path deliberately propagates NaN and trips (tests/test_gpu_failures.py)."""
    from channel3d_b200 import initfield
    from oracle import oracle as O
    cfg = small_channel(16, 12, 8)
    o = O.Oracle(cfg)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=o.mesh()[0])
    ux[3, 4, 5] = np.nan
    o.set_state(ux, uy, uz, p)
    d = o.step(1)
    assert np.isnan(o.get_state()["ux"]).any()
    assert d["rc"] == 0


def test_golden_fixtures_reproduce(built):
    import json
    import os
    from oracle import oracle as O
    here = os.path.join(os.path.dirname(__file__), "golden")
    g = np.load(os.path.join(here, "channel16x12x8.npz"))
    meta = json.load(open(os.path.join(here, "channel16x12x8.json")))
    import importlib.util
    spec = importlib.util.spec_from_file_location("mk", os.path.join(here, "make_golden.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    cfg = mk.case()
    o = O.Oracle(cfg)
    assert np.array_equal(o.mesh()[0], g["yp"])
    o.set_state(g["ux0"], g["uy0"], g["uz0"], g["p0"])
    d = o.step(1)
    s = o.get_state()
    for k in ("ux", "uy", "uz", "p"):
        assert rel_l2(s[k], g[k + "1"]) < 1e-14, k
    assert abs(d["divmax2"] - meta["info"]["1"]["divmax2"]) < 1e-14
