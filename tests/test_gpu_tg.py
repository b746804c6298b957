"""The Taylor-Green vortex (FlowType 3, Input/TaylorGreenVortex.prm) in a
2pi x pi x 2pi box with free-slip walls at y = 0 and pi: half a period of the
triply periodic vortex, whose mirror symmetry (uy odd, ux and uz even about
both planes) the walls keep.  Initial field InitVelocity_TG
(src/CFD_2nd/m_FlowType_TGVortex.f90:20-47), statistic clcStat_TG (:87-113):
xnu times the mean of CalcDissipationRate (src/CFD_2nd/m_Tools.f90:497-540).

Known answer: on a uniform mesh of spacing h the reference's stencils give
the initial field 2 S_ij S_ij with mean s^2/2 + c^2/4, s = sin(h/2)/(h/2),
c = sin(h) cos(h/2)/h (3/4 in the continuum: the diagonal strains carry the
factor s, the xz and yz shear strains c, the xy shear strain vanishes).

Tolerances: the dissipation within 1e-12 relative of the closed form and of
the oracle (FP64; 1e-6 with FP32 fields), steps within 1e-10 of the oracle,
the kinetic-energy budget dE/dt = -eps within 2% over the first time unit."""
import numpy as np
import pytest

from helpers import rel_max

pytestmark = pytest.mark.gpu


def closed_form(cfg):
    h = cfg.xlx / cfg.nxc
    s = np.sin(h / 2) / (h / 2)
    c = np.sin(h) * np.cos(h / 2) / h
    return cfg.xnu * (s * s / 2 + c * c / 4)


def _solver(cfg):
    from channel3d_b200 import ChannelSolver, initfield, mesh_y
    yp = mesh_y(cfg)
    st = initfield.taylor_green(cfg, yp=yp)
    s = ChannelSolver(cfg, yp=yp)
    s.upload(*st)
    return s, st


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_tg_initial_dissipation_known_answer(built, precision, tol):
    from channel3d_b200 import workloads
    cfg = workloads.taylor_green(32, precision=precision)
    s, _ = _solver(cfg)
    eps = s.dissipation()
    s.close()
    assert abs(eps / closed_form(cfg) - 1.0) < tol, (eps, closed_form(cfg))


def test_tg_steps_match_oracle(built):
    from channel3d_b200 import workloads
    from oracle import oracle as O
    cfg = workloads.taylor_green(32)
    s, st = _solver(cfg)
    o = O.Oracle(cfg)
    o.set_state(*st)
    assert abs(s.dissipation() / o.dissipation() - 1.0) < 1e-12
    for _ in range(2):
        s.step(10)
        o.step(10)
        gs, go = s.download(), o.get_state()
        for k in ("ux", "uy", "uz", "p"):
            assert rel_max(gs[k], go[k]) < 1e-10, (k, rel_max(gs[k], go[k]))
        assert abs(s.dissipation() / o.dissipation() - 1.0) < 1e-11
    # the mirror symmetry the free-slip walls stand for: uy vanishes on both walls' planes
    assert np.abs(s.download()["uy"][:, 0, :]).max() < 1e-14
    s.close()


def test_tg_energy_budget(built):
    """Over the first time unit (100 steps of 0.01) the kinetic energy falls by
    the time integral of the dissipation; vortex stretching raises the
    dissipation, so the energy falls faster than the initial mode's viscous
    decay E0 exp(-eps0 t / E0) (dE/dt = -eps, eps = 2 xnu k^2 E for a single mode)."""
    from channel3d_b200 import workloads, mesh_y
    cfg = workloads.taylor_green(32)
    s, _ = _solver(cfg)
    dy = np.diff(mesh_y(cfg))

    def energy():
        f = s.download()
        w = dy[None, :, None] / cfg.yly
        return 0.5 * ((f["ux"] ** 2 + f["uy"] ** 2 + f["uz"] ** 2) * w).sum() / (cfg.nxc * cfg.nzc)

    E, eps = [energy()], [s.dissipation()]
    for _ in range(10):
        s.step(10)
        E.append(energy())
        eps.append(s.dissipation())
    s.close()
    dt = 10 * cfg.dtMax
    loss = E[0] - E[-1]
    integral = dt * (0.5 * eps[0] + sum(eps[1:-1]) + 0.5 * eps[-1])
    assert abs(loss / integral - 1.0) < 0.02, (loss, integral)
    assert all(a > b for a, b in zip(E, E[1:]))
    assert all(a < b for a, b in zip(eps, eps[1:]))
    assert E[-1] < E[0] * np.exp(-eps[0] / E[0])
