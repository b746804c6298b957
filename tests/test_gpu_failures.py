"""Failure detection of the device step without any GPU fault: the limit
checks of ChannelIterate (src/CFD_2nd/m_ChannelSystem.f90:127-130) run on the
device and set a status that the host reads after the step.  Unlike the
reference, whose maxima skip NaN (m_Tools.f90:70, :93-98), the device folds
NaN into +inf, so a NaN field trips the divergence limit.  The tensor-core
kernels' bounded mbarrier waits give up with a status the host reads; a wait
on a barrier that nothing completes shows it, and the context stays usable."""
import numpy as np
import pytest

from helpers import small_channel

pytestmark = pytest.mark.gpu


def _solver(cfg):
    from channel3d_b200 import ChannelSolver, initfield, mesh_y
    yp = mesh_y(cfg)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp)
    s = ChannelSolver(cfg, yp=yp)
    return s, (ux, uy, uz, p)


def test_nan_field_trips_the_divergence_limit(built):
    from channel3d_b200 import _lib
    cfg = small_channel(32, 24, 16)
    s, (ux, uy, uz, p) = _solver(cfg)
    ux = ux.copy()
    ux[3, 4, 5] = np.nan
    s.upload(ux, uy, uz, p)
    info = s.step(2, raise_on_diverge=False)
    assert info["status"] == 1 and info["itime"] == 1
    with pytest.raises(_lib.Ch3dError) as e:
        s.step(1)
    assert e.value.code == _lib.CH3D_ERR_DIVERGED


def test_velocity_limit_trips_and_state_stays_finite(built):
    cfg = small_channel(32, 24, 16, vel_limit=0.01)  # all three maxima exceed it
    s, st = _solver(cfg)
    s.upload(*st)
    info = s.step(3, raise_on_diverge=False)
    assert info["status"] == 2 and info["itime"] == 1
    # the steps after the trip returned early: the state is that of step 1
    assert all(np.isfinite(v).all() for v in s.download().values())


def test_healthy_run_has_status_zero(built):
    cfg = small_channel(32, 24, 16)
    s, st = _solver(cfg)
    s.upload(*st)
    info = s.step(5)
    assert info["status"] == 0 and info["itime"] == 5


def test_tensor_core_wait_expiry_sets_status(built):
    import ctypes
    import torch
    from channel3d_b200 import _lib
    from channel3d_b200.mlp import MLPClosure
    lib = _lib.load_library()
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.ch3d_mlp_wait_check(1024, ctypes.c_void_p(st.data_ptr()), None) == 0
    torch.cuda.synchronize()
    assert st.item() == 1
    # the context is intact: a forward pass afterwards completes with its own status 0
    net = MLPClosure(seed=1)
    y = net.forward(torch.randn(300, 10, device="cuda"))
    torch.cuda.synchronize()
    assert torch.isfinite(y).all() and int(net.status.item()) == 0

