"""Parity of the 4th-order solver (src/CFD_4th) on the device with the CPU
oracle, FP64, through the C ABI.

Tolerances: per-stage results within 1e-12 relative (max norm; the RHS
arrays within 5e-12: by the third substep the device's fused multiply-adds
and the oracle's separately rounded products differ by a few ulp, which the
near-wall 1/dy^2 coefficients of the y viscous term amplify), the pressure
correction within 5e-11 (L2: its source, the divergence of u*, is a small
difference of O(1) velocities, which amplifies their relative differences), whole steps within the 1e-10 relative bound."""
import numpy as np
import pytest

from helpers import rel_l2, rel_max

pytestmark = pytest.mark.gpu


def cfg4(nx, ny, nz, **kw):
    from channel3d_b200 import workloads
    cfg, _ = workloads.get("channel128_re5600_4th", **kw)
    return cfg.copy(nxc=nx, nyc=ny, nzc=nz, nycSection=[ny // 2, ny - ny // 2])


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


@pytest.mark.parametrize("shape", [(32, 24, 16), (48, 32, 36)])
def test_stage_parity_4th(built, shape):
    o, s = _pair(cfg4(*shape))
    for ns in (1, 2, 3):
        o.stage(0, ns); s.stage(0, ns)
        o.stage(1, ns); s.stage(1, ns)
        # RhsX carries -pmAlpha*dpmdxns on both sides (src/CFD_4th/m_TScheme.f90:364-377)
        for wo, wg in ((o.ARR1, s.RHSX), (o.ARR2, s.RHSY), (o.HALO, s.RHSZ), (o.HISTX, s.HISTX),
                       (o.HISTY, s.HISTY), (o.HISTZ, s.HISTZ)):
            a, b = s.get_array(wg), o.get_interior(wo)
            if wg == s.RHSY:  # row jc=1 is replaced by the wall condition in clcU2Hat
                a, b = a[:, 1:, :], b[:, 1:, :]
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


def test_step_parity_4th_64cubed_200_steps(built):
    o, s = _pair(cfg4(64, 64, 64))
    di = s.step(200)
    do = o.step(200)
    go, gs = o.get_state(), s.download()
    for k in ("ux", "uy", "uz", "p"):
        e = rel_l2(gs[k], go[k])
        assert e < 1e-10, (k, e)
    assert di["divmax2"] < 1e-12 and do["divmax2"] < 1e-12
    assert abs(di["PrGradAver"] - do["PrGradAver"]) <= 1e-10 * max(1.0, abs(do["PrGradAver"]))
    assert abs(di["uxm"] - do["uxm"]) <= 1e-10


def test_step_parity_4th_128cubed(built):
    """The 4th-order 128^3 workload itself, 20 steps against the oracle."""
    from channel3d_b200 import workloads
    cfg, _ = workloads.get("channel128_re5600_4th")
    o, s = _pair(cfg)
    di = s.step(20)
    do = o.step(20)
    go, gs = o.get_state(), s.download()
    for k in ("ux", "uy", "uz", "p"):
        e = rel_l2(gs[k], go[k])
        assert e < 1e-10, (k, e)
    assert di["divmax2"] < 1e-12


def test_fused_4th_matches_stages(built):
    from channel3d_b200 import ChannelSolver, initfield, mesh_y
    cfg = cfg4(48, 40, 24)
    yp = mesh_y(cfg)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp)
    a = ChannelSolver(cfg, yp=yp); a.upload(ux, uy, uz, p)
    b = ChannelSolver(cfg, yp=yp); b.upload(ux, uy, uz, p)
    for ns in (1, 2, 3):
        for st in range(7):
            a.stage(st, ns)
    b.step(1)
    ga, gb = a.download(hist=True), b.download(hist=True)
    for k in ("ux", "uy", "uz", "p", "hist"):
        assert rel_max(ga[k], gb[k]) < 1e-11, (k, rel_max(ga[k], gb[k]))


def test_poisson_parity_4th(built):
    """Poisson solve with the 4th-order modified wavenumbers."""
    from channel3d_b200 import ChannelSolver, mesh_y
    from oracle import oracle as O
    cfg = cfg4(48, 40, 24)
    src = np.random.default_rng(1).standard_normal(cfg.shape)
    o = O.Oracle(cfg)
    s = ChannelSolver(cfg, yp=mesh_y(cfg))
    a, b = s.poisson(src), o.poisson(src)
    assert rel_l2(a, b) < 1e-12, rel_l2(a, b)
