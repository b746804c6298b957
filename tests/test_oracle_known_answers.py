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
    path folds NaN into +inf and trips (tests/test_gpu_failures.py)."""
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


def _cfg4(nx, ny, nz):
    from channel3d_b200 import workloads
    cfg, _ = workloads.get("channel128_re5600_4th")
    return cfg.copy(nxc=nx, nyc=ny, nzc=nz, nycSection=[ny // 2, ny - ny // 2])


def _d4(a, axis, rd, shift):
    """Staggered 4th-order first difference (1/24, -9/8, 9/8, -1/24) * rd over
    the points shift-1 .. shift+2 relative to each cell (periodic axis)."""
    c = (1.0 / 24.0, -1.125, 1.125, -1.0 / 24.0)
    return sum(cq * np.roll(a, -(shift + q - 1), axis) for q, cq in enumerate(c)) * rd


def test_poisson_residual_4th(built):
    """The 4th-order pressure operator is div4(grad4 phi) in x and z: the
    modified wavenumber rdx2/288 (cos 3t - 54 cos 2t + 783 cos t - 730)
    (src/CFD_4th/m_Poisson.f90:40-47) is the symbol of the composition of the
    staggered 4th-order difference with itself."""
    from oracle import oracle as O
    cfg = _cfg4(24, 20, 12)
    o = O.Oracle(cfg)
    src = np.random.default_rng(5).standard_normal(cfg.shape)
    phi = o.poisson(src)
    rdx, rdz = cfg.nxc / cfg.xlx, cfg.nzc / cfg.zlz
    # gradient at the face below the cell (shift -1: points i-2..i+1), divergence
    # over the faces i..i+1 with the wide neighbours (points i-1..i+2)
    L = _d4(_d4(phi, 2, rdx, -1), 2, rdx, 0) + _d4(_d4(phi, 0, rdz, -1), 0, rdz, 0)
    yL = _laplacian(cfg, o, phi) - (
        (np.roll(phi, 1, 2) - 2 * phi + np.roll(phi, -1, 2)) * rdx ** 2
        + (np.roll(phi, 1, 0) - 2 * phi + np.roll(phi, -1, 0)) * rdz ** 2)
    r = L + yL - src
    rm = r.mean(axis=(0, 2))
    assert np.abs(r - rm[None, :, None]).max() < 1e-9 * np.abs(src).max()
    assert np.abs(rm[1:]).max() < 1e-9 * np.abs(src).max()


def test_step_4th_is_divergence_free_and_deterministic(built):
    from channel3d_b200 import initfield
    from oracle import oracle as O
    cfg = _cfg4(32, 24, 16)
    o = O.Oracle(cfg)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=o.mesh()[0])
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


def test_laminar_4th_keeps_flux_balance(built):
    """Without noise the 4th-order step keeps v = w = 0 and an x,z-uniform
    ux; the forcing (mean viscous stress, src/CFD_4th/m_TScheme.f90:364-377)
    balances the wall friction, so the bulk velocity is unchanged."""
    from channel3d_b200 import initfield
    from oracle import oracle as O
    cfg = _cfg4(16, 24, 8)
    o = O.Oracle(cfg)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=o.mesh()[0], amplitude=0.0)
    o.set_state(ux, uy, uz, p)
    d0 = o.step(1)
    d = o.step(9)
    s = o.get_state()
    assert np.abs(s["uy"]).max() < 1e-14 and np.abs(s["uz"]).max() < 1e-14
    assert np.abs(s["ux"] - s["ux"][:1, :, :1]).max() < 1e-13
    assert abs(d["uxm"] - d0["uxm"]) < 1e-12


def _cfg_fimp(nx, ny, nz):
    from channel3d_b200 import workloads
    cfg, _ = workloads.get("channel128_re5600_fimp")
    return cfg.copy(nxc=nx, nyc=ny, nzc=nz, nycSection=[ny // 2, ny - ny // 2])


def test_fimp_adi_factorisation(built):
    """clcU1Hat_FIMP_010 (src/CFD_2nd/m_TSchemeFIMP_inc.f90:263-347): the
    increment du = u* - u satisfies (I - b Lx)(I - b Lz)(I - b Ly) du = RhsX
    with the periodic 3-point Lx, Lz and the Crank-Nicolson Ly whose wall
    coefficient is doubled (am2cForCN(1), ap2cForCN(nyc))."""
    from oracle import oracle as O
    cfg = _cfg_fimp(16, 12, 10)
    o = O.Oracle(cfg)
    from channel3d_b200 import initfield
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=o.mesh()[0])
    o.set_state(ux, uy, uz, p)
    o.stage(0, 1)
    o.stage(1, 1)
    rhs = o.get_interior(o.ARR1)
    u0 = o.get_state()["ux"]
    o.stage(2, 1)
    du = o.get_state()["ux"] - u0
    beta = 0.5 * (8.0 / 15.0) * cfg.xnu * cfg.dtMax
    rdx2, rdz2 = (cfg.nxc / cfg.xlx) ** 2, (cfg.nzc / cfg.zlz) ** 2
    yp = o.mesh()[0]
    ny = cfg.nyc
    dyp = yp[1:] - yp[:-1]
    yc = 0.5 * (yp[1:] + yp[:-1])
    dyc = np.ones(ny + 2)
    dyc[2:ny + 1] = yc[1:] - yc[:-1]
    dyc[1] = dyp[0]
    dyc[ny + 1] = dyp[-1]
    rdyc = 1.0 / dyc
    am = np.array([rdyc[j] / dyp[j - 1] for j in range(1, ny + 1)])
    ap = np.array([rdyc[j + 1] / dyp[j - 1] for j in range(1, ny + 1)])
    am[0] = 4 * rdyc[1] / (dyc[1] + 2 * dyc[2])
    ap[0] = 4 * rdyc[2] / (dyc[1] + 2 * dyc[2])
    am[-1] = 4 * rdyc[ny] / (dyc[ny + 1] + 2 * dyc[ny])
    ap[-1] = 4 * rdyc[ny + 1] / (dyc[ny + 1] + 2 * dyc[ny])
    am[0] *= 2.0
    ap[-1] *= 2.0
    tp, tm = -beta * ap, -beta * am
    tc = 1.0 - tp - tm
    w = tc[None, :, None] * du
    w[:, :-1, :] += tp[None, :-1, None] * du[:, 1:, :]
    w[:, 1:, :] += tm[None, 1:, None] * du[:, :-1, :]
    w = (1 + 2 * beta * rdz2) * w - beta * rdz2 * (np.roll(w, 1, 0) + np.roll(w, -1, 0))
    w = (1 + 2 * beta * rdx2) * w - beta * rdx2 * (np.roll(w, 1, 2) + np.roll(w, -1, 2))
    assert np.abs(w - rhs).max() < 1e-12 * np.abs(rhs).max()


def test_fimp_step_is_divergence_free_and_laminar_steady(built):
    from channel3d_b200 import initfield
    from oracle import oracle as O
    cfg = _cfg_fimp(32, 24, 16)
    o = O.Oracle(cfg)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=o.mesh()[0])
    o.set_state(ux, uy, uz, p)
    d = o.step(3)
    assert d["divmax2"] < 1e-13 and d["rc"] == 0
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=o.mesh()[0], amplitude=0.0)
    o.set_state(ux, uy, uz, p)
    d0 = o.step(1)
    d = o.step(5)
    s = o.get_state()
    assert np.abs(s["uy"]).max() < 1e-14 and np.abs(s["uz"]).max() < 1e-14
    assert np.abs(s["ux"] - s["ux"][:1, :, :1]).max() < 1e-13
    # the bulk controller drives <u> to ubulk = 1 from the discretised profile
    assert abs(d["uxm"] - 1.0) < 0.01 * abs(d0["uxm"] - 1.0)


def test_fexp_step_is_divergence_free_and_laminar_steady(built):
    """The explicit scheme (clcRhsX/Y/Z_FEXP, clcU1/2/3Hat_FEXP,
    PressureUpdate_FEXP): divergence-free steps from a noisy field; a laminar
    profile stays a function of y alone with uy = uz = 0, and the bulk
    controller drives <u> to ubulk."""
    from channel3d_b200 import initfield
    from oracle import oracle as O
    cfg = _cfg_fimp(32, 24, 16).copy(IsImplicit=0, dtMax=2e-4)
    o = O.Oracle(cfg)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=o.mesh()[0])
    o.set_state(ux, uy, uz, p)
    d = o.step(3)
    assert d["divmax2"] < 1e-13 and d["rc"] == 0
    assert np.all(o.get_state()["uy"][:, 0, :] == 0.0)  # the wall row keeps uy_ym
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=o.mesh()[0], amplitude=0.0)
    o.set_state(ux, uy, uz, p)
    d0 = o.step(1)
    d = o.step(5)
    s = o.get_state()
    assert np.abs(s["uy"]).max() < 1e-14 and np.abs(s["uz"]).max() < 1e-14
    assert np.abs(s["ux"] - s["ux"][:1, :, :1]).max() < 1e-13
    assert abs(d["uxm"] - 1.0) < 0.01 * abs(d0["uxm"] - 1.0)


def _cfg_les(model, nx=24, ny=16, nz=12):
    from channel3d_b200 import workloads
    cfg, _ = workloads.get("channel48_les")
    return cfg.copy(nxc=nx, nyc=ny, nzc=nz, nycSection=[ny // 2, ny - ny // 2], LES_type=model, Cs=0.1)


def test_sgs_models_on_laminar_shear(built):
    """Properties of the eddy-viscosity models on a laminar profile u(y):
    WALE (Nicoud & Ducros 1999) vanishes in pure shear, the mixed-time-scale
    model's test-filtered energy is zero for an x,z-uniform field, and the
    Smagorinsky / van Driest model equals xnu + (Cs D Delta)^2 |du/dy| with
    the staggered |S| of ClcVelStrainRate."""
    from channel3d_b200 import initfield
    from oracle import oracle as O
    for model in (2, 3):
        cfg = _cfg_les(model)
        o = O.Oracle(cfg)
        ux, uy, uz, p = initfield.laminar_noise(cfg, yp=o.mesh()[0], amplitude=0.0)
        o.set_state(ux, uy, uz, p)
        nut, _ = o.sgs()
        assert np.abs(nut - cfg.xnu).max() < 1e-15, model
    cfg = _cfg_les(10)
    o = O.Oracle(cfg)
    yp = o.mesh()[0]
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp, amplitude=0.0)
    o.set_state(ux, uy, uz, p)
    nut, utau = o.sgs()
    ny = cfg.nyc
    u = ux[0, :, 0]
    yc = 0.5 * (yp[1:] + yp[:-1])
    dyp = yp[1:] - yp[:-1]
    ug = np.concatenate([[-u[0]], u, [-u[-1]]])          # no-slip ghosts 2*0 - u
    ycg = np.concatenate([[2 * yp[0] - yc[0]], yc, [2 * yp[-1] - yc[-1]]])
    rdyc = 1.0 / np.diff(ycg)                               # rdyc(jc), jc = 1..nyp
    rdyc[0] = 1.0 / dyp[0]
    rdyc[-1] = 1.0 / dyp[-1]
    st4 = 0.125 * (2 * ug[2:] * rdyc[1:] + 2 * ug[1:-1] * (rdyc[:-1] - rdyc[1:]) - 2 * ug[:-2] * rdyc[:-1])
    S = np.abs(2 * st4)
    tw = cfg.xnu * 0.5 * (abs(u[0]) / (yc[0] - yp[0]) + abs(u[-1]) / (yp[-1] - yc[-1]))
    assert abs(utau - np.sqrt(tw)) < 1e-14
    dw = np.minimum(yc - yp[0], yp[-1] - yc)
    D = 1 - np.exp(-(dw * utau / cfg.xnu) / 26.0)
    delta = (dyp * (cfg.xlx / cfg.nxc) * (cfg.zlz / cfg.nzc)) ** (1.0 / 3.0)
    ref = cfg.xnu + (cfg.Cs * D * delta) ** 2 * S
    assert np.abs(nut[0, :, 0] - ref).max() < 1e-12 * ref.max()
    assert np.abs(nut - nut[:1, :, :1]).max() < 1e-18


def test_les_step_is_divergence_free(built):
    from channel3d_b200 import initfield
    from oracle import oracle as O
    for model in (2, 3, 10):
        cfg = _cfg_les(model)
        o = O.Oracle(cfg)
        ux, uy, uz, p = initfield.laminar_noise(cfg, yp=o.mesh()[0])
        o.set_state(ux, uy, uz, p)
        d = o.step(3)
        assert d["divmax2"] < 1e-13 and d["rc"] == 0, model


def test_oracle_interp_known_answers():
    """The oracle's restatement of the interpolateField tool
    (Tool/interpolateField/src/m_Interp.f90:20-361): onto the same grid it
    returns the field unchanged; a field linear in y is reproduced exactly at
    the cell centres of another stretching away from the walls; ux is held at
    ubulk when the flow rate is constant."""
    from channel3d_b200 import initfield, mesh_y
    from oracle import oracle as O
    cfg = small_channel(32, 24, 16)
    st = initfield.laminar_noise(cfg, yp=mesh_y(cfg))
    a = O.Oracle(cfg)
    a.set_state(*st)
    b = O.Oracle(cfg.copy(IsUxConst=False))
    b.interp_from(a)
    g, r = b.get_state(), a.get_state()
    for k in ("ux", "uy", "uz", "p"):
        assert np.array_equal(g[k], r[k]), k
    new = small_channel(32, 20, 16, StretType=[2, 2], SectioncStret=[1.0, 1.0])
    yc = 0.5 * (mesh_y(cfg)[1:] + mesh_y(cfg)[:-1])
    f = np.broadcast_to((0.3 * yc + 0.1)[None, :, None], cfg.shape).copy()
    a.set_state(f, np.zeros(cfg.shape), f, f)
    c = O.Oracle(new.copy(IsUxConst=False))
    c.interp_from(a)
    ycn = 0.5 * (mesh_y(new)[1:] + mesh_y(new)[:-1])
    got = c.get_state()
    for k in ("uz", "p"):
        assert np.abs(got[k][:, 2:-2, :] - (0.3 * ycn[2:-2] + 0.1)[None, :, None]).max() < 1e-14, k
    d = O.Oracle(new.copy(ubulk=0.8))
    d.interp_from(a)
    ux = d.get_state()["ux"]
    dy = np.diff(mesh_y(new))
    assert abs((ux * dy[None, :, None]).sum() / (new.nxc * new.nzc * new.yly) - 0.8) < 1e-12


def test_oracle_tg_dissipation_known_answer():
    """CalcDissipationRate of the Taylor-Green field (clcStat_TG) on a uniform
    mesh of spacing h: xnu (s^2/2 + c^2/4), s = sin(h/2)/(h/2),
    c = sin(h) cos(h/2)/h, for two resolutions."""
    from channel3d_b200 import initfield, workloads
    from oracle import oracle as O
    for n in (16, 32):
        cfg = workloads.taylor_green(n)
        h = cfg.xlx / n
        s, c = np.sin(h / 2) / (h / 2), np.sin(h) * np.cos(h / 2) / h
        o = O.Oracle(cfg)
        o.set_state(*initfield.taylor_green(cfg, yp=o.mesh()[0]))
        eps = o.dissipation()
        assert abs(eps / (cfg.xnu * (s * s / 2 + c * c / 4)) - 1.0) < 1e-13, (n, eps)



def test_poisson_residual_periodic_y():
    """clcPPE_z1_periodic (src/CFD_2nd/m_Poisson.f90:954-1073): with y periodic
    the operator is the 3-point Laplacian in all three directions; for a source
    of zero mean the pinned (0,0) system also satisfies its first row, so the
    residual vanishes everywhere."""
    from channel3d_b200 import workloads
    from oracle import oracle as O
    cfg = workloads.taylor_green_periodic(16).copy(nxc=24, nyc=20, nzc=12, nycSection=[20])
    o = O.Oracle(cfg)
    src = np.random.default_rng(4).standard_normal(cfg.shape)
    src -= src.mean()
    phi = o.poisson(src)
    r2 = [(cfg.nxc / cfg.xlx) ** 2, (cfg.nyc / cfg.yly) ** 2, (cfg.nzc / cfg.zlz) ** 2]
    L = sum((np.roll(phi, 1, a) - 2 * phi + np.roll(phi, -1, a)) * r2[2 - a] for a in range(3))
    assert np.abs(L - src).max() < 1e-10 * np.abs(src).max()
    assert abs(phi[:, 0, :].mean()) < 1e-12 * np.abs(phi).max()


@pytest.mark.parametrize("implicit", [1, 2])
def test_oracle_periodic_box_mirrors_free_slip_half_box(implicit):
    """The Taylor-Green field is mirror-symmetric about y = 0 and pi, the planes
    where the free-slip walls of the half-period box sit: 20 steps of the
    triply periodic box (clcU*Hat_PIMP_0 or clcU*Hat_FIMP_000,
    clcPPE_z1_periodic) equal, on its lower half, those of the 2pi x pi x 2pi
    box with free-slip walls (clcU*Hat_PIMP or clcU*Hat_FIMP_010), to rounding."""
    from channel3d_b200 import initfield, workloads
    from oracle import oracle as O
    n = 16
    out = []
    for cfg in (workloads.taylor_green_periodic(n, dt=0.02).copy(IsImplicit=implicit),
                workloads.taylor_green(n, dt=0.02).copy(IsImplicit=implicit)):
        o = O.Oracle(cfg)
        o.set_state(*initfield.taylor_green(cfg, yp=o.mesh()[0]))
        info = o.step(20)
        assert info["divmax2"] < 1e-13
        out.append((o.get_state(), o.dissipation()))
    (a, ea), (b, eb) = out
    for k in ("ux", "uy", "uz", "p"):
        assert np.abs(a[k][:, :n // 2, :] - b[k]).max() < 1e-13 * max(1.0, np.abs(b[k]).max()), k
    assert abs(ea / eb - 1.0) < 1e-12


def test_redft_matches_definition():
    """FFTW's REDFT10 / REDFT01 (the z transforms between walls,
    src/CFD_2nd/m_Poisson.f90:267-307) against their definitions:
    Y_k = 2 sum_j X_j cos(pi (j + 1/2) k / n) and
    Y_k = X_0 + 2 sum_{j>=1} X_j cos(pi j (k + 1/2) / n); the pair is 2n times
    the identity."""
    from oracle import oracle as O
    for n in (6, 8, 12, 18):
        x = np.random.default_rng(n).standard_normal(n)
        j = np.arange(n)
        y10 = np.array([2 * np.sum(x * np.cos(np.pi * (j + 0.5) * k / n)) for k in range(n)])
        y01 = np.array([x[0] + 2 * np.sum(x[1:] * np.cos(np.pi * j[1:] * (k + 0.5) / n)) for k in range(n)])
        assert np.abs(O.redft10(x) - y10).max() < 1e-12 * np.abs(y10).max()
        assert np.abs(O.redft01(x) - y01).max() < 1e-12 * np.abs(y01).max()
        assert np.abs(O.redft01(O.redft10(x)) / (2 * n) - x).max() < 1e-13


def _z_walls(cfg, bc):
    return cfg.copy(BcOption=[0, 0, cfg.BcOption[2], cfg.BcOption[3], bc, bc])


def test_poisson_residual_z_walls():
    """clcPPE with walls in z: the operator is the periodic 3-point Laplacian in
    x, [am2Pr, ac2Pr, ap2Pr] in y and the 3-point Laplacian with Neumann ghosts
    (phi_0 = phi_1, phi_nzc+1 = phi_nzc) in z; the residual is a plane constant
    at j = 1 only (the (0,0)-mode pin)."""
    from oracle import oracle as O
    cfg = _z_walls(small_channel(24, 20, 12), -1)
    o = O.Oracle(cfg)
    src = np.random.default_rng(5).standard_normal(cfg.shape)
    phi = o.poisson(src)
    L = _laplacian(cfg, o, phi)
    rdz2 = (cfg.nzc / cfg.zlz) ** 2
    # replace the periodic z second difference of _laplacian by the Neumann one
    L -= (np.roll(phi, 1, 0) - 2 * phi + np.roll(phi, -1, 0)) * rdz2
    zm = np.concatenate([phi[:1], phi[:-1]], axis=0)
    zp = np.concatenate([phi[1:], phi[-1:]], axis=0)
    L += (zm - 2 * phi + zp) * rdz2
    r = L - src
    rm = r.mean(axis=(0, 2))
    assert np.abs(r - rm[None, :, None]).max() < 1e-9 * np.abs(src).max()
    assert np.abs(rm[1:]).max() < 1e-9 * np.abs(src).max()


@pytest.mark.parametrize("implicit", [0, 1, 2])
def test_oracle_z_walls_box_mirrors_z_periodic_box(implicit):
    """The Taylor-Green field is also mirror-symmetric about z = 0 and pi (ux and
    uy even, uz odd): 20 steps of the 2pi x pi x pi box with free-slip walls in
    y and z (the z walls of m_BC_and_Halo.f90:313-338, REDFT10/01 in the Poisson
    solve, FIMP's clcU*Hat_FIMP_011 sweeps) equal, on its lower z half, those of
    the 2pi x pi x 2pi box with periodic z, to rounding, for the explicit,
    partially and fully implicit schemes."""
    from channel3d_b200 import initfield, workloads
    from oracle import oracle as O
    n = 16
    full = workloads.taylor_green(n, dt=0.02).copy(IsImplicit=implicit, **({"dtMax": 0.005} if implicit == 0 else {}))
    half = _z_walls(full.copy(nzc=n // 2, zlz=np.pi), -2)
    out = []
    for cfg in (full, half):
        o = O.Oracle(cfg)
        o.set_state(*initfield.taylor_green(cfg, yp=o.mesh()[0]))
        d = o.step(20)
        assert d["divmax2"] < 1e-13
        out.append(o.get_state())
    a, b = out
    assert np.abs(b["uz"]).max() > 1e-2  # the flow has left the plane initial field
    for k in ("ux", "uy", "uz", "p"):
        assert np.abs(a[k][: n // 2] - b[k]).max() < 1e-13 * max(1.0, np.abs(b[k]).max()), k


@pytest.mark.parametrize("implicit", [0, 1, 2])
def test_oracle_duct_laminar_invariants(implicit):
    """A duct (no-slip walls in y and z, periodic x): a streamwise field ux(y, z)
    keeps uy = uz = 0 and stays independent of x under every scheme, and steps
    from a noisy field are divergence-free."""
    from channel3d_b200 import initfield
    from oracle import oracle as O
    cfg = _z_walls(small_channel(16, 12, 10, IsImplicit=implicit, dtMax=2e-4), -1)
    o = O.Oracle(cfg)
    yp = o.mesh()[0]
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp)
    o.set_state(ux, uy, uz, p)
    assert o.step(3)["divmax2"] < 1e-13
    zc = (np.arange(cfg.nzc) + 0.5) / cfg.nzc
    ux0 = initfield.laminar_noise(cfg, yp=yp, amplitude=0.0)[0] * (4 * zc * (1 - zc))[:, None, None]
    o.set_state(ux0, np.zeros(cfg.shape), np.zeros(cfg.shape), np.zeros(cfg.shape))
    o.step(5)
    s = o.get_state()
    assert np.abs(s["uy"]).max() < 1e-14 and np.abs(s["uz"]).max() < 1e-14
    assert np.abs(s["ux"] - s["ux"][:, :, :1]).max() < 1e-13


@pytest.mark.parametrize("implicit", [0, 1, 2])
def test_oracle_walled_box_mirrors_periodic_box(implicit):
    """Walls in x as well (clcU*Hat_FIMP_111's x sweep, the x-wall ghost rules of
    m_BC_and_Halo.f90:285-311, REDFT10/01 in x): the Taylor-Green field is
    mirror-symmetric about x = 0 and pi too (ux odd, uy and uz even), so 20 steps
    of the pi x pi x pi box with free-slip walls on all six faces equal, on the
    corner x, z in [0, pi], those of the 2pi x pi x 2pi box periodic in x and z."""
    from channel3d_b200 import initfield, workloads
    from oracle import oracle as O
    n = 16
    full = workloads.taylor_green(n, dt=0.02).copy(IsImplicit=implicit, **({"dtMax": 0.005} if implicit == 0 else {}))
    box = full.copy(nxc=n // 2, nzc=n // 2, xlx=np.pi, zlz=np.pi, BcOption=[-2, -2, -2, -2, -2, -2])
    out = []
    for cfg in (full, box):
        o = O.Oracle(cfg)
        o.set_state(*initfield.taylor_green(cfg, yp=o.mesh()[0]))
        assert o.step(20)["divmax2"] < 1e-13
        out.append(o.get_state())
    a, b = out
    for k in ("ux", "uy", "uz", "p"):
        assert np.abs(a[k][: n // 2, :, : n // 2] - b[k]).max() < 1e-13 * max(1.0, np.abs(b[k]).max()), k


def test_poisson_residual_x_and_z_walls():
    """clcPPE with walls in x and z: Neumann 3-point Laplacians in x and z, the
    walls' operator in y; the residual is a plane constant at j = 1 only."""
    from oracle import oracle as O
    cfg = small_channel(16, 20, 12).copy(BcOption=[-1, -1, -1, -1, -1, -1])
    o = O.Oracle(cfg)
    src = np.random.default_rng(6).standard_normal(cfg.shape)
    phi = o.poisson(src)
    L = _laplacian(cfg, o, phi)
    r2 = {2: (cfg.nxc / cfg.xlx) ** 2, 0: (cfg.nzc / cfg.zlz) ** 2}
    for ax, rr in r2.items():
        n = phi.shape[ax]
        L -= (np.roll(phi, 1, ax) - 2 * phi + np.roll(phi, -1, ax)) * rr
        lo = np.take(phi, [0] + list(range(n - 1)), axis=ax)
        hi = np.take(phi, list(range(1, n)) + [n - 1], axis=ax)
        L += (lo - 2 * phi + hi) * rr
    r = L - src
    rm = r.mean(axis=(0, 2))
    assert np.abs(r - rm[None, :, None]).max() < 1e-9 * np.abs(src).max()
    assert np.abs(rm[1:]).max() < 1e-9 * np.abs(src).max()


def test_oracle_lid_driven_cavity_symmetry():
    """The lid-driven cavity of Input/LidDrivenCavity.prm (FlowType 5, no-slip
    walls on all faces, the top wall moving with ux = 1, fully implicit,
    xnu 1e-2) at 16^3: started from rest the flow is divergence-free and stays
    mirror-symmetric about the mid-plane z = 1/2 (ux, uy, p even, uz odd)."""
    from channel3d_b200 import ChannelConfig
    from oracle import oracle as O
    n = 16
    cfg = ChannelConfig(FlowType=5, nxc=n, nyc=n, nzc=n, xlx=1.0, yly=1.0, zlz=1.0, xnu=1e-2, dtMax=1e-2, iCFL=2,
                        IsImplicit=2, BcOption=[-1, -1, -1, -1, -1, -1], uxBcValue=[0, 0, 0, 1.0, 0, 0],
                        IsUxConst=False, ubulk=0.0, ybulk1=0.0, ybulk2=1.0, nSection=1, SectionLength=[1.0],
                        nycSection=[n], StretType=[0], StretOption=[0], SectioncStret=[0.0], RunName="LidCavity")
    o = O.Oracle(cfg)
    z = np.zeros(cfg.shape)
    o.set_state(z, z, z, z)
    d = o.step(20)
    assert d["rc"] == 0 and d["divmax2"] < 1e-13
    s = o.get_state()
    assert np.abs(s["ux"]).max() > 0.1  # the lid has set the fluid moving
    for k in ("ux", "uy", "p"):
        assert np.abs(s[k] - s[k][::-1]).max() < 1e-13, k
    # uz lives on the z faces k = 0..n-1 (face 0 the wall): face k mirrors face n - k
    uz = s["uz"]
    assert np.abs(uz[1:] + uz[:0:-1]).max() < 1e-13 and np.abs(uz[0]).max() == 0.0


@pytest.mark.parametrize("bc", ["periodic_y", "walls_xz"])
def test_boundary_variants_are_thread_count_independent(bc):
    """The oracle is also the timed CPU baseline on all host threads: the
    periodic-y (cyclic Poisson solve, FIMP_000) and walled (cosine transforms,
    FIMP_111) variants give bit-identical states on 1 and 4 threads."""
    from channel3d_b200 import initfield, workloads
    from oracle import oracle as O
    if bc == "periodic_y":
        cfg = workloads.taylor_green_periodic(16).copy(nxc=16, nyc=12, nzc=8, nycSection=[12])
    else:
        cfg = small_channel(16, 12, 8, IsImplicit=2).copy(BcOption=[-1, -1, -1, -1, -1, -1], IsUxConst=False,
                                                          uxBcValue=[0, 0, 0, 1.0, 0, 0])
    o = O.Oracle(cfg)
    st = initfield.laminar_noise(cfg, yp=o.mesh()[0])
    out = []
    nthr = O.num_threads()
    try:
        for n in (1, 4):
            O.set_threads(n)
            o.set_state(*st)
            assert o.step(3)["divmax2"] < 1e-13
            out.append(o.get_state())
    finally:
        O.set_threads(nthr)
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k
