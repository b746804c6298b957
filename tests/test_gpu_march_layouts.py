"""The column march (right-hand sides fused with the y Crank-Nicolson solves,
channel3d_b200/csrc/ch3d_march.cu) in each of its launch layouts, whole steps
against the oracle within the 1e-10 relative bound:

- twisted blocks (few column tiles: two thread groups per tile, the lower
  eliminating upwards and the upper downwards, meeting in the middle), with
  odd ny so the groups march different numbers of rows, ragged tiles in x and
  z, and the smallest ny the layout takes;
- one tile per plain block (more tiles than twisted blocks fit on the GPU, fewer
  than the resident persistent blocks), with a ragged last z tile;
- the 4th-order march both ways (128 column tiles twisted, 384 plain);
- the march that stops at g on grids with more tiles than twisted blocks fit
  (2nd order): the divergence and projection marches substitute u* from g
  themselves, and the last projection carries the step diagnostics."""
import numpy as np
import pytest

from helpers import rel_l2, small_channel

pytestmark = pytest.mark.gpu


def _run(cfg, nsteps, seed=11):
    from channel3d_b200 import ChannelSolver, initfield, mesh_y
    from oracle import oracle as O
    yp = mesh_y(cfg)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp, seed=seed)
    p = 0.01 * np.random.default_rng(seed).standard_normal(cfg.shape)
    o = O.Oracle(cfg)
    o.set_state(ux, uy, uz, p)
    s = ChannelSolver(cfg, yp=yp)
    s.upload(ux, uy, uz, p)
    di = s.step(nsteps)
    o.step(nsteps)
    go, gs = o.get_state(), s.download(hist=True)
    s.close()
    return go, gs, di


def _check(go, gs, tol=1e-10):
    for k in ("ux", "uy", "uz", "p"):
        e = rel_l2(gs[k], go[k])
        assert e < tol, (k, e)


@pytest.mark.parametrize("shape", [(48, 25, 18), (32, 5, 16), (64, 24, 48)])
def test_twisted_march(built, shape):
    go, gs, di = _run(small_channel(*shape), 4)
    _check(go, gs)
    assert di["divmax2"] < 1e-12


def test_plain_blocks_one_tile_each(built):
    # 8 x 41 = 328 tiles: above the 296 twisted FP64 blocks that fit, below the 592 persistent ones
    go, gs, _ = _run(small_channel(256, 16, 162), 3)
    _check(go, gs)


def test_twisted_march_mixed(built):
    """FP32 twisted march (mixed path) within the mixed path's 1e-4 bound."""
    go, gs, _ = _run(small_channel(48, 25, 18, precision="mixed"), 4)
    for k in ("ux", "uy", "uz"):
        assert rel_l2(gs[k], go[k]) < 1e-4, (k, rel_l2(gs[k], go[k]))


@pytest.mark.parametrize("shape", [(128, 33, 128), (256, 16, 192)])
def test_march_4th(built, shape):
    from channel3d_b200 import workloads
    cfg, _ = workloads.get("channel128_re5600_4th")
    nx, ny, nz = shape
    cfg = cfg.copy(nxc=nx, nyc=ny, nzc=nz, nycSection=[ny // 2, ny - ny // 2])
    go, gs, di = _run(cfg, 3)
    _check(go, gs)
    assert di["divmax2"] < 1e-12


def test_gsub_step_info(built):
    """The diagnostics the last projection computes from g (divergence, velocity
    maxima, CFL, bulk mean) and the divergence before it, against the oracle's
    step, on a grid above the twisted threshold (8 x 41 = 328 tiles)."""
    go, gs, di = _run(small_channel(256, 16, 162), 3)
    _check(go, gs)
    from oracle import oracle as O
    from channel3d_b200 import initfield, mesh_y
    cfg = small_channel(256, 16, 162)
    yp = mesh_y(cfg)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp, seed=11)
    p = 0.01 * np.random.default_rng(11).standard_normal(cfg.shape)
    o = O.Oracle(cfg)
    o.set_state(ux, uy, uz, p)
    do = o.step(3)
    for k in ("divmax1", "cflmp", "uxm", "PrGradAver"):
        assert abs(di[k] - do[k]) <= 1e-9 * max(1.0, abs(do[k])), (k, di[k], do[k])
    for q in range(3):
        assert abs(di["vmax"][q] - do["vmax"][q]) <= 1e-10 * abs(do["vmax"][q]), (q, di["vmax"], do["vmax"])
    assert di["divmax2"] < 1e-12


def test_gsub_mixed(built):
    """Mixed path with the march stopping at g (8 x 81 = 648 tiles)."""
    go, gs, di = _run(small_channel(256, 24, 324, precision="mixed"), 3)
    for k in ("ux", "uy", "uz"):
        assert rel_l2(gs[k], go[k]) < 1e-4, (k, rel_l2(gs[k], go[k]))
    assert di["divmax2"] < 1e-4
