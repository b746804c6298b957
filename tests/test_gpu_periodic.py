"""The triply periodic steps (BcOption 0 0 0 0 0 0) on the device against the
CPU oracle, FP64, through the C ABI: explicit (IsImplicit 0, the scheme of
Input/TaylorGreenVortex.prm: clcRhsX/Y/Z_FEXP and clcU1/2/3Hat_FEXP,
src/CFD_2nd/m_TSchemeFEXP_inc.f90), fully implicit (IsImplicit 2)
clcU1/2/3Hat_FIMP_000 (src/CFD_2nd/m_TSchemeFIMP_inc.f90:187-258, 559-631,
950-1030: periodic x, z and y sweeps with constant coefficients,
InversePTriFixedCoe), partially implicit (IsImplicit 1) clcU1/2/3Hat_PIMP_0
(src/CFD_2nd/m_TSchemePIMP_inc.f90:435-461, 594-621, 745-771: the periodic y
sweep alone), and clcPPE_z1_periodic (src/CFD_2nd/m_Poisson.f90:954-1073:
cyclic y systems, InversePeriodicTridiagonal), with the periodic y halos of
SetBC_and_UpdateHalo (src/CFD_2nd/m_BC_and_Halo.f90:20-29); and the
Taylor-Green vortex of Input/TaylorGreenVortex.prm in its own 2pi^3 box.

Size-independent property: the vortex is mirror-symmetric about y = 0 and pi,
where the free-slip walls of the 2pi x pi x 2pi box sit, so the lower half of
the periodic box evolves as that box does (FEXP, PIMP or FIMP_010 with
free-slip ghosts).

Tolerances as the fully implicit parity tests: per stage 5e-12 (RHS),
1e-12 (u*), 5e-11 (phi, L2), 1e-11 (end of the substep); whole steps 1e-10;
the mirrored half box within 1e-12 relative (max norm; the two runs differ in
the rounding of their y and Poisson solves only); the dissipation 1e-12."""
import numpy as np
import pytest

from helpers import rel_l2, rel_max

pytestmark = pytest.mark.gpu


IMPLICIT = [0, 1, 2]


def _periodic(nx, ny, nz, **kw):
    from channel3d_b200 import workloads
    return workloads.taylor_green_periodic(16).copy(nxc=nx, nyc=ny, nzc=nz, nycSection=[ny], **kw)


def _noisy_tg(cfg, yp, seed=0x5EED):
    """The Taylor-Green field with noise on every component and the pressure,
    so that every mode of every solve is exercised."""
    from channel3d_b200 import initfield
    rng = np.random.default_rng(seed)
    ux, uy, uz, p = initfield.taylor_green(cfg, yp=yp)
    return tuple(a + 0.05 * rng.standard_normal(cfg.shape) for a in (ux, uy, uz, p))


def _pair(cfg, st):
    from channel3d_b200 import ChannelSolver, mesh_y
    from oracle import oracle as O
    o = O.Oracle(cfg)
    o.set_state(*st)
    s = ChannelSolver(cfg, yp=mesh_y(cfg))
    s.upload(*st)
    return o, s


@pytest.mark.parametrize("implicit", IMPLICIT)
@pytest.mark.parametrize("shape", [(32, 24, 16), (48, 36, 32)])
def test_stage_parity_periodic(built, shape, implicit):
    from channel3d_b200 import mesh_y
    cfg = _periodic(*shape, IsImplicit=implicit)
    o, s = _pair(cfg, _noisy_tg(cfg, mesh_y(cfg)))
    for ns in (1, 2, 3):
        o.stage(0, ns); s.stage(0, ns)
        o.stage(1, ns); s.stage(1, ns)
        for wo, wg in ((o.ARR1, s.RHSX), (o.ARR2, s.RHSY), (o.HALO, s.RHSZ), (o.HISTX, s.HISTX),
                       (o.HISTY, s.HISTY), (o.HISTZ, s.HISTZ)):
            a, b = s.get_array(wg), o.get_interior(wo)
            assert rel_max(a, b) < 5e-12, (ns, wg, rel_max(a, b))
        o.stage(2, ns); s.stage(2, ns)
        go = o.get_state()
        for k, w in (("ux", 12), ("uy", 13), ("uz", 14)):
            ustar = s.get_array(w)
            assert rel_max(ustar, go[k]) < 1e-12, (ns, "uhat", k, rel_max(ustar, go[k]))
        o.stage(3, ns); s.stage(3, ns)
        o.stage(4, ns); s.stage(4, ns)
        phi_o, phi_g = o.get_interior(o.HALO), s.get_array(s.PRPHI)
        assert rel_l2(phi_g, phi_o) < 5e-11, (ns, "phi", rel_l2(phi_g, phi_o))
        o.stage(5, ns); s.stage(5, ns)
        o.stage(6, ns); s.stage(6, ns)
        go, gs = o.get_state(), s.download()
        for k in ("ux", "uy", "uz", "p"):
            assert rel_max(gs[k], go[k]) < 1e-11, (ns, "final", k, rel_max(gs[k], go[k]))
    s.close()


@pytest.mark.parametrize("implicit", IMPLICIT)
def test_step_parity_periodic(built, implicit):
    """50 whole steps (graph-captured) of a noisy vortex at 48 x 40 x 32, with the
    step diagnostics (CheckDivergence, CalcVmax, CalcMaxCFL over periodic y)."""
    from channel3d_b200 import mesh_y
    cfg = _periodic(48, 40, 32, IsImplicit=implicit)
    o, s = _pair(cfg, _noisy_tg(cfg, mesh_y(cfg)))
    di = s.step(50)
    do = o.step(50)
    go, gs = o.get_state(), s.download()
    s.close()
    for k in ("ux", "uy", "uz", "p"):
        e = rel_l2(gs[k], go[k])
        assert e < 1e-10, (k, e)
    assert di["divmax2"] < 1e-12 and do["divmax2"] < 1e-12
    for q in range(3):
        assert abs(di["vmax"][q] / do["vmax"][q] - 1.0) < 1e-10, q
    assert abs(di["cflmp"] / do["cflmp"] - 1.0) < 1e-10


@pytest.mark.parametrize("implicit", IMPLICIT)
def test_periodic_tg_mirrors_free_slip_half_box(built, implicit):
    """64 x 64 x 64 periodic box against 64 x 32 x 64 with free-slip walls, both
    on the device, 50 steps: the lower half, the dissipation and the step
    diagnostics agree."""
    from channel3d_b200 import ChannelSolver, initfield, mesh_y, workloads
    n = 64
    runs = []
    for cfg in (workloads.taylor_green_periodic(n).copy(IsImplicit=implicit),
                workloads.taylor_green(n).copy(IsImplicit=implicit)):
        yp = mesh_y(cfg)
        with ChannelSolver(cfg, yp=yp) as s:
            s.upload(*initfield.taylor_green(cfg, yp=yp))
            info = s.step(50)
            runs.append((s.download(), s.dissipation(), info))
    (a, ea, ia), (b, eb, ib) = runs
    for k in ("ux", "uy", "uz", "p"):
        e = np.abs(a[k][:, :n // 2, :] - b[k]).max() / max(1.0, np.abs(b[k]).max())
        assert e < 1e-12, (k, e)
    assert abs(ea / eb - 1.0) < 1e-12
    assert ia["divmax2"] < 1e-12 and ib["divmax2"] < 1e-12
    assert abs(ia["cflmp"] / ib["cflmp"] - 1.0) < 1e-12


def test_periodic_tg_dissipation(built):
    """clcStat_TG in the periodic box: the closed form at t = 0 (the box holds
    whole periods, so the mean is that of the half box) and the oracle after
    20 steps, with the energy decaying."""
    from channel3d_b200 import ChannelSolver, initfield, mesh_y, workloads
    from oracle import oracle as O
    cfg = workloads.taylor_green_periodic(32)
    yp = mesh_y(cfg)
    st = initfield.taylor_green(cfg, yp=yp)
    h = cfg.xlx / cfg.nxc
    sf, cf = np.sin(h / 2) / (h / 2), np.sin(h) * np.cos(h / 2) / h
    o = O.Oracle(cfg)
    o.set_state(*st)
    with ChannelSolver(cfg, yp=yp) as s:
        s.upload(*st)
        assert abs(s.dissipation() / (cfg.xnu * (sf * sf / 2 + cf * cf / 4)) - 1.0) < 1e-12
        s.step(20)
        o.step(20)
        assert abs(s.dissipation() / o.dissipation() - 1.0) < 1e-12
        g = s.download()
    e0 = sum(float((a ** 2).sum()) for a in st[:3])
    e1 = sum(float((g[k] ** 2).sum()) for k in ("ux", "uy", "uz"))
    assert e1 < e0


@pytest.mark.parametrize("implicit", IMPLICIT)
def test_periodic_ghost2_layout_matches_oracle_arrays(built, implicit):
    """The GHOST2 host layout with periodic y: the halo rows j = 0 and nyp are
    copies of rows nyc and 1 (then the x and z halos), as in the oracle's arrays."""
    from channel3d_b200 import ChannelSolver, _lib, mesh_y
    from oracle import oracle as O
    cfg = _periodic(32, 24, 16, IsImplicit=implicit)
    yp = mesh_y(cfg)
    st = _noisy_tg(cfg, yp)
    o = O.Oracle(cfg)
    o.set_state(*st)
    ids = {"ux": O.Oracle.UX, "uy": O.Oracle.UY, "uz": O.Oracle.UZ, "p": O.Oracle.P}
    layout = _lib.LAYOUT_GHOST2
    with ChannelSolver(cfg, yp=yp) as s:
        shp = s.layout_shape(layout)
        g0 = {k: o.get_ghosted(w).reshape(shp) for k, w in ids.items()}
        s.upload(g0["ux"], g0["uy"], g0["uz"], g0["p"], layout=layout)
        s.step(5)
        got = s.download(layout=layout)
    o.step(5)
    for k, w in ids.items():
        ref = o.get_ghosted(w).reshape(shp)
        e = rel_max(got[k], ref)
        assert e < 1e-10, (k, e, np.unravel_index(np.argmax(np.abs(got[k] - ref)), shp))
