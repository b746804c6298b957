"""The named channel configurations at their own sizes and lengths, against
the CPU oracle.

- 128^3, 4pi x 2 x 4pi/3, Re_b 5600, dt 0.001: the 4th-order solver
  (src/CFD_4th/m_ChannelSystem.f90:83-190) and the 2nd-order fully implicit
  (ADI) step, each for the configuration's full 1000 steps.
- 256x192x256, Re_b 13750, dt 0.0005, FP64: 10 steps.
- 768x384x64, Re_b 21900, dt 0.0003: the layout the 768x384x576 benchmark
  runs (ny = 384, more column tiles than resident march blocks, so the march
  stops at g and the divergence and projection marches substitute u*), FP64
  and mixed precision, 3 steps, with the step diagnostics.
- 256x192x256 mixed against FP64 over the configuration's 2000 steps: the
  mean profile and rms velocities of the statistics.

Tolerances: FP64 fields within 1e-10 relative (L2), the specification's
bound; mixed precision within 1e-4 relative of FP64 in the velocity after 3
steps and in the mean-profile and rms statistics after 2000 steps.
"""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu


def _start(cfg, seed=0x5EED):
    from channel3d_b200 import initfield, mesh_y
    yp = mesh_y(cfg)
    return yp, initfield.laminar_noise(cfg, yp=yp, seed=seed)


def _oracle_run(cfg, state, nsteps):
    from oracle import oracle as O
    o = O.Oracle(cfg)
    o.set_state(*state)
    info = o.step(nsteps)
    st = o.get_state()
    o.close()
    return st, info


def _gpu_run(cfg, yp, state, nsteps):
    from channel3d_b200 import ChannelSolver
    with ChannelSolver(cfg, yp=yp) as s:
        s.upload(*state)
        info = s.step(nsteps)
        return s.download(), info, s.path_flags()


def _check_fp64(gs, go, di, do, tol=1e-10):
    for k in ("ux", "uy", "uz", "p"):
        e = rel_l2(gs[k], go[k])
        assert e < tol, (k, e)
    assert di["divmax2"] < 1e-12 and do["divmax2"] < 1e-12, (di["divmax2"], do["divmax2"])
    assert abs(di["PrGradAver"] - do["PrGradAver"]) <= tol * max(1.0, abs(do["PrGradAver"]))
    assert abs(di["uxm"] - do["uxm"]) <= tol


def test_channel768x384x64_benchmark_layout(built):
    """The 768x384x576 benchmark's kernel layout (ny = 384, march stopping at
    g) on a 64-plane slab of it: FP64 to 1e-10 and the mixed path to 1e-4,
    3 steps, including the step diagnostics fused into the last projection."""
    from channel3d_b200 import workloads
    cfg, _ = workloads.get("channel768x384x576_re21900")
    cfg = cfg.copy(nzc=64, zlz=cfg.zlz * 64 / 576)
    yp, st = _start(cfg)
    go, do = _oracle_run(cfg, st, 3)
    gs, di, path = _gpu_run(cfg, yp, st, 3)
    assert "gsub" in path and "twisted" not in path, path
    _check_fp64(gs, go, di, do)
    for k in ("cflmp", "divmax1"):
        assert abs(di[k] - do[k]) <= 1e-9 * abs(do[k]), (k, di[k], do[k])
    for q in range(3):
        assert abs(di["vmax"][q] - do["vmax"][q]) <= 1e-10 * do["vmax"][q]
    gm, dm, path = _gpu_run(cfg.copy(precision="mixed"), yp, st, 3)
    assert "gsub" in path, path
    for k in ("ux", "uy", "uz"):
        assert rel_l2(gm[k], go[k]) < 1e-4, (k, rel_l2(gm[k], go[k]))
    assert dm["divmax2"] < 1e-4


def test_channel256x192x256_fp64_10_steps(built):
    from channel3d_b200 import workloads
    cfg, _ = workloads.get("channel256x192x256_re13750")
    yp, st = _start(cfg)
    go, do = _oracle_run(cfg, st, 10)
    gs, di, _ = _gpu_run(cfg, yp, st, 10)
    _check_fp64(gs, go, di, do)


def test_channel256x192x256_mixed_vs_fp64_2000_steps(built):
    """The precision comparison of the 256x192x256 configuration over its 2000
    steps: statistics (FP64 moment sums in both runs) every 20 steps from a
    projected seeded start; mean U(y) and u', v', w' rms within 1e-4
    relative (L2 over y), Re_tau within 1e-3, divergence at FP32 round-off."""
    from channel3d_b200 import compare_precision
    r = compare_precision.compare("channel256x192x256_re13750", steps=2000, ivstats=20)
    for k in ("rel_err_U", "rel_err_urms", "rel_err_vrms", "rel_err_wrms"):
        assert r[k] < 1e-4, (k, r)
    assert r["rel_err_Re_tau"] < 1e-3, r
    assert r["divmax_fp64"] < 1e-12 and r["divmax_mixed"] < 1e-4, r


@pytest.mark.parametrize("name", ["channel128_re5600_4th", "channel128_re5600_fimp"])
def test_channel128_full_run(built, name):
    """The 128^3 configuration for its full 1000 steps (dt 0.001, t = 1)."""
    from channel3d_b200 import workloads
    cfg, nsteps = workloads.get(name)
    assert nsteps == 1000
    yp, st = _start(cfg)
    go, do = _oracle_run(cfg, st, nsteps)
    gs, di, _ = _gpu_run(cfg, yp, st, nsteps)
    assert di["itime"] == do["itime"] == nsteps
    _check_fp64(gs, go, di, do)
