"""The explicit 2nd-order step (IsImplicit 0: clcRhsX/Y/Z_FEXP with the whole
viscous term explicit, clcU1/2/3Hat_FEXP u* = u + Rhs, clcPrSrcOther and
PressureUpdate_FEXP p += phi; src/CFD_2nd/m_TSchemeFEXP_inc.f90) in the channel
between no-slip walls, in the half channel with a free-slip top and with the
LES eddy viscosities (the _FEXP_LES right-hand sides), on the
device against the CPU oracle, FP64, through the C ABI; and the reference's
own Taylor-Green input (Input/TaylorGreenVortex.prm: explicit, triply
periodic, xnu 6.25e-4, dt 0.01) at 64^3.

The explicit viscous term limits dt by dy_min^2 / xnu: the channel cases use
dt = 2e-4 at Re_b 5600.  Tolerances as the fully implicit parity tests: per
stage 5e-12 (RHS), 1e-12 (u*), 5e-11 (phi, L2), 1e-11 (velocity at the end of
the substep); whole steps 1e-10.  The pressure at the end of a substep is
within 5e-11: the explicit update adds phi alone (p += phi), so p carries
phi's error, relative to a pressure of the size of phi."""
import numpy as np
import pytest

from helpers import rel_l2, rel_max, small_channel

pytestmark = pytest.mark.gpu


def _pair(cfg, seed=0x5EED):
    from channel3d_b200 import ChannelSolver, initfield, mesh_y
    from oracle import oracle as O
    yp = mesh_y(cfg)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp, seed=seed)
    p = 0.01 * np.random.default_rng(seed).standard_normal(cfg.shape)
    o = O.Oracle(cfg)
    o.set_state(ux, uy, uz, p)
    s = ChannelSolver(cfg, yp=yp)
    s.upload(ux, uy, uz, p)
    return o, s


def _channel(nx, ny, nz, **kw):
    return small_channel(nx, ny, nz, IsImplicit=0, dtMax=2e-4, **kw)


def _half_channel(nx, ny, nz):
    return _channel(nx, ny, nz).copy(FlowType=2, yly=1.0, nSection=1, SectionLength=[1.0], nycSection=[ny],
                                     StretType=[1], StretOption=[0], SectioncStret=[2.0],
                                     BcOption=[0, 0, -1, -2, 0, 0])


@pytest.mark.parametrize("shape", [(32, 24, 16), (48, 32, 36)])
def test_stage_parity_fexp(built, shape):
    o, s = _pair(_channel(*shape))
    for ns in (1, 2, 3):
        o.stage(0, ns); s.stage(0, ns)
        o.stage(1, ns); s.stage(1, ns)
        for wo, wg in ((o.ARR1, s.RHSX), (o.ARR2, s.RHSY), (o.HALO, s.RHSZ), (o.HISTX, s.HISTX),
                       (o.HISTY, s.HISTY), (o.HISTZ, s.HISTZ)):
            a, b = s.get_array(wg), o.get_interior(wo)
            assert rel_max(a, b) < 5e-12, (ns, wg, rel_max(a, b))
        o.stage(2, ns); s.stage(2, ns)
        o.stage(3, ns); s.stage(3, ns)  # the oracle sets the wall row of uy here
        go = o.get_state()
        for k, w in (("ux", 12), ("uy", 13), ("uz", 14)):
            ustar = s.get_array(w)
            assert rel_max(ustar, go[k]) < 1e-12, (ns, "uhat", k, rel_max(ustar, go[k]))
        o.stage(4, ns); s.stage(4, ns)
        phi_o, phi_g = o.get_interior(o.HALO), s.get_array(s.PRPHI)
        assert rel_l2(phi_g, phi_o) < 5e-11, (ns, "phi", rel_l2(phi_g, phi_o))
        o.stage(5, ns); s.stage(5, ns)
        o.stage(6, ns); s.stage(6, ns)
        go, gs = o.get_state(), s.download()
        for k in ("ux", "uy", "uz", "p"):
            tol = 5e-11 if k == "p" else 1e-11
            assert rel_max(gs[k], go[k]) < tol, (ns, "final", k, rel_max(gs[k], go[k]))
    s.close()


@pytest.mark.parametrize("case", ["channel", "half_channel_free_slip"])
def test_step_parity_fexp(built, case):
    cfg = _channel(48, 40, 32) if case == "channel" else _half_channel(48, 32, 24)
    o, s = _pair(cfg)
    di = s.step(50)
    do = o.step(50)
    go, gs = o.get_state(), s.download()
    s.close()
    for k in ("ux", "uy", "uz", "p"):
        e = rel_l2(gs[k], go[k])
        assert e < 1e-10, (k, e)
    assert di["divmax2"] < 1e-12 and do["divmax2"] < 1e-12
    assert abs(di["PrGradAver"] - do["PrGradAver"]) <= 1e-10 * max(1.0, abs(do["PrGradAver"]))
    assert np.all(gs["uy"][:, 0, :] == cfg.uyBcValue[2])  # the wall row keeps uy_ym


def test_reference_tg_input_fexp(built):
    """Input/TaylorGreenVortex.prm as it stands (explicit, triply periodic,
    xnu 6.25e-4, dt 0.01; 64^3 instead of 512^3), 20 steps against the oracle
    and the dissipation against the oracle's."""
    from channel3d_b200 import ChannelSolver, initfield, mesh_y, workloads
    from oracle import oracle as O
    cfg = workloads.taylor_green_periodic(64).copy(IsImplicit=0)
    yp = mesh_y(cfg)
    st = initfield.taylor_green(cfg, yp=yp)
    o = O.Oracle(cfg)
    o.set_state(*st)
    with ChannelSolver(cfg, yp=yp) as s:
        s.upload(*st)
        s.step(20)
        gs, eps = s.download(), s.dissipation()
    o.step(20)
    go = o.get_state()
    for k in ("ux", "uy", "uz", "p"):
        assert rel_l2(gs[k], go[k]) < 1e-10, (k, rel_l2(gs[k], go[k]))
    assert abs(eps / o.dissipation() - 1.0) < 1e-12


def _les(model, nx=32, ny=24, nz=16):
    from channel3d_b200 import workloads
    cfg, _ = workloads.get("channel48_les")
    return cfg.copy(nxc=nx, nyc=ny, nzc=nz, nycSection=[ny // 2, ny - ny // 2], LES_type=model, Cs=0.1,
                    IsImplicit=0, dtMax=2e-4)


@pytest.mark.parametrize("model", (2, 3, 10))
def test_les_fexp_parity(built, model):
    """clcRhsX/Y/Z_FEXP_LES (src/CFD_2nd/m_TSchemeFEXP_inc.f90:80-386) with the
    WALE, mixed-time-scale and Smagorinsky / van Driest eddy viscosities: stage
    by stage at 32 x 24 x 16, then 20 whole steps, against the oracle."""
    o, s = _pair(_les(model))
    s.sgs_viscosity()
    o.sgs()
    for ns in (1, 2, 3):
        o.stage(0, ns); s.stage(0, ns)
        o.stage(1, ns); s.stage(1, ns)
        for wo, wg in ((o.ARR1, s.RHSX), (o.ARR2, s.RHSY), (o.HALO, s.RHSZ), (o.HISTX, s.HISTX),
                       (o.HISTY, s.HISTY), (o.HISTZ, s.HISTZ)):
            a, b = s.get_array(wg), o.get_interior(wo)
            assert rel_max(a, b) < 5e-12, (ns, wg, rel_max(a, b))
        o.stage(2, ns); s.stage(2, ns)
        o.stage(3, ns); s.stage(3, ns)
        go = o.get_state()
        for k, w in (("ux", 12), ("uy", 13), ("uz", 14)):
            assert rel_max(s.get_array(w), go[k]) < 1e-12, (ns, "uhat", k)
        o.stage(4, ns); s.stage(4, ns)
        assert rel_l2(s.get_array(s.PRPHI), o.get_interior(o.HALO)) < 5e-11, (ns, "phi")
        o.stage(5, ns); s.stage(5, ns)
        o.stage(6, ns); s.stage(6, ns)
        go, gs = o.get_state(), s.download()
        for k in ("ux", "uy", "uz", "p"):
            tol = 5e-11 if k == "p" else 1e-11
            assert rel_max(gs[k], go[k]) < tol, (ns, "final", k, rel_max(gs[k], go[k]))
    s.close()
    o, s = _pair(_les(model))
    di = s.step(20)
    o.step(20)
    go, gs = o.get_state(), s.download()
    s.close()
    for k in ("ux", "uy", "uz", "p"):
        assert rel_l2(gs[k], go[k]) < 1e-10, (k, rel_l2(gs[k], go[k]))
    assert di["divmax2"] < 1e-12


@pytest.mark.parametrize("les", [0, 2])
def test_fexp_mixed_precision(built, les):
    """The explicit scheme with FP32 fields (and the FP64 low-mode Poisson
    solves of the mixed path), without LES and with WALE: 20 steps stay within
    1e-4 of the FP64 oracle, the bound of the other mixed-path tests."""
    from channel3d_b200 import ChannelSolver, initfield, mesh_y
    from oracle import oracle as O
    cfg = _channel(48, 40, 32) if les == 0 else _les(les, 48, 40, 32)
    yp = mesh_y(cfg)
    st = initfield.laminar_noise(cfg, yp=yp)
    o = O.Oracle(cfg)
    o.set_state(*st)
    with ChannelSolver(cfg.copy(precision="mixed"), yp=yp) as s:
        s.upload(*st)
        di = s.step(20)
        gs = s.download()
    o.step(20)
    go = o.get_state()
    for k in ("ux", "uy", "uz"):
        assert rel_l2(gs[k], go[k]) < 1e-4, (k, rel_l2(gs[k], go[k]))
    assert di["divmax2"] < 1e-4
