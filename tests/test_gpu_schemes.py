"""The reference's other time schemes (ischeme, src/CFD_2nd/m_Parameters.f90:
135-150 and src/CFD_4th/m_Parameters.f90:158-173): AB2 (one substep, gamma 3/2,
theta -1/2) and RK2 (two substeps, gamma 1/2, 1; theta 0, -1/2), through the
same kernels as RK3 with their PMcoeUpdate constants.  Whole steps on the
device against the CPU oracle, FP64, through the C ABI, with a nonzero old
history uploaded, which the first AB2 substep reads (theta != 0).

Tolerance: 1e-10 relative (L2), the whole-step bound of the FP64 path."""
import numpy as np
import pytest

from helpers import rel_l2, small_channel

pytestmark = pytest.mark.gpu

CASES = {
    # name: (config factory, steps)
    "pimp_march": (lambda: small_channel(48, 40, 32), 20),
    "pimp_substituting_march": (lambda: small_channel(256, 16, 162), 4),  # the layout of large grids
    "fimp": (lambda: small_channel(32, 24, 16, IsImplicit=2), 20),
    "fexp": (lambda: small_channel(32, 24, 16, IsImplicit=0, dtMax=2e-4), 20),
    "order4": (lambda: small_channel(32, 24, 16, order=4), 20),
}


@pytest.mark.parametrize("ischeme", [1, 2])
@pytest.mark.parametrize("name", sorted(CASES))
def test_time_scheme_step_parity(built, name, ischeme):
    from channel3d_b200 import ChannelSolver, initfield, mesh_y
    from oracle import oracle as O
    factory, nsteps = CASES[name]
    cfg = factory().copy(ischeme=ischeme)
    yp = mesh_y(cfg)
    rng = np.random.default_rng(0x5EED + ischeme)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp)
    hist = [0.1 * rng.standard_normal(cfg.shape) for _ in range(3)]
    o = O.Oracle(cfg)
    o.set_state(ux, uy, uz, p, hist=hist)
    with ChannelSolver(cfg, yp=yp) as s:
        s.upload(ux, uy, uz, p, hist=np.stack(hist))
        di = s.step(nsteps)
        gs = s.download(hist=True)
    do = o.step(nsteps)
    go = o.get_state(hist=True)
    for k in ("ux", "uy", "uz", "p", "hist"):
        e = rel_l2(gs[k], go[k])
        assert e < 1e-10, (name, ischeme, k, e)
    assert abs(di["SimTime"] - do["SimTime"]) < 1e-12
    assert abs(di["PrGradAver"] - do["PrGradAver"]) <= 1e-10 * max(1.0, abs(do["PrGradAver"]))
