"""The register-resident FFT kernels (channel3d_b200/csrc/rfft.cuh) against
the CPU oracle, for every line length that has a plan: x half-lengths 384,
256, 128, 64 and z lengths 576, 384, 256, 128.  Other lengths run the generic
shared-memory FFT, which the remaining parity tests cover.

Tolerances: FP64 Poisson solves within 1e-12 relative (L2), as the generic
path; the mixed path (FP32 transforms, FP64 low-mode y solves) within 2e-5;
whole FP64 steps within the 1e-10 relative bound of the specification."""
import numpy as np
import pytest

from helpers import rel_l2, small_channel

pytestmark = pytest.mark.gpu

SHAPES = [(768, 8, 576), (512, 8, 384), (256, 8, 256), (128, 8, 128)]


def _poisson_pair(cfg, seed=1):
    from channel3d_b200 import ChannelSolver, mesh_y
    from oracle import oracle as O
    src = np.random.default_rng(seed).standard_normal(cfg.shape)
    o = O.Oracle(cfg.copy(precision="fp64"))
    s = ChannelSolver(cfg, yp=mesh_y(cfg))
    a, b = s.poisson(src), o.poisson(src)
    s.close()
    return a, b


@pytest.mark.parametrize("shape", SHAPES)
def test_poisson_plans_fp64(built, shape):
    a, b = _poisson_pair(small_channel(*shape))
    assert rel_l2(a, b) < 1e-12, (shape, rel_l2(a, b))


@pytest.mark.parametrize("shape", SHAPES)
def test_poisson_plans_mixed(built, shape):
    a, b = _poisson_pair(small_channel(*shape, precision="mixed"))
    assert rel_l2(a, b) < 2e-5, (shape, rel_l2(a, b))


@pytest.mark.parametrize("shape,nsteps", [((256, 32, 128), 10), ((768, 16, 576), 2)])
def test_step_parity_plans(built, shape, nsteps):
    """Whole steps (projection, divergence source, both transforms in each
    substep) at sizes whose x and z lengths have plans."""
    from channel3d_b200 import ChannelSolver, initfield, mesh_y
    from oracle import oracle as O
    cfg = small_channel(*shape)
    yp = mesh_y(cfg)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp, seed=7)
    o = O.Oracle(cfg)
    o.set_state(ux, uy, uz, p)
    s = ChannelSolver(cfg, yp=yp)
    s.upload(ux, uy, uz, p)
    di = s.step(nsteps)
    o.step(nsteps)
    go, gs = o.get_state(), s.download()
    for k in ("ux", "uy", "uz", "p"):
        e = rel_l2(gs[k], go[k])
        assert e < 1e-10, (shape, k, e)
    assert di["divmax2"] < 1e-12
    s.close()


# the largest x length with every z plan, odd and smallest-odd ny
ODD_NY_SHAPES = [(768, 9, 576), (768, 8, 384), (768, 5, 256)]


@pytest.mark.parametrize("shape", ODD_NY_SHAPES)
def test_poisson_plans_odd_ny_fp64(built, shape):
    a, b = _poisson_pair(small_channel(*shape))
    assert rel_l2(a, b) < 1e-12, (shape, rel_l2(a, b))


@pytest.mark.parametrize("shape", ODD_NY_SHAPES)
def test_poisson_plans_odd_ny_mixed(built, shape):
    a, b = _poisson_pair(small_channel(*shape, precision="mixed"))
    assert rel_l2(a, b) < 2e-5, (shape, rel_l2(a, b))


def test_step_parity_plans_odd_ny(built):
    from channel3d_b200 import ChannelSolver, initfield, mesh_y
    from oracle import oracle as O
    cfg = small_channel(768, 17, 576)
    yp = mesh_y(cfg)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp, seed=9)
    o = O.Oracle(cfg)
    o.set_state(ux, uy, uz, p)
    s = ChannelSolver(cfg, yp=yp)
    s.upload(ux, uy, uz, p)
    di = s.step(2)
    o.step(2)
    go, gs = o.get_state(), s.download()
    for k in ("ux", "uy", "uz", "p"):
        e = rel_l2(gs[k], go[k])
        assert e < 1e-10, (k, e)
    assert di["divmax2"] < 1e-12
    s.close()


def test_step_parity_persistent_march(built):
    """More column tiles (8 x 81 = 648) than resident march blocks (4 FP64,
    5 FP32 per SM on 148 SMs: 592 / 740), so the persistent FP64 blocks overlap
    each tile's back substitution with the next tile's forward march; 3 steps
    against the oracle."""
    from channel3d_b200 import ChannelSolver, initfield, mesh_y
    from oracle import oracle as O
    cfg = small_channel(256, 24, 324)
    yp = mesh_y(cfg)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp, seed=5)
    o = O.Oracle(cfg)
    o.set_state(ux, uy, uz, p)
    s = ChannelSolver(cfg, yp=yp)
    s.upload(ux, uy, uz, p)
    s.step(3)
    o.step(3)
    go, gs = o.get_state(), s.download(hist=True)
    for k in ("ux", "uy", "uz", "p"):
        e = rel_l2(gs[k], go[k])
        assert e < 1e-10, (k, e)
    s.close()
