"""The allocation-free Poisson entry point (ch3d_poisson_noalloc).

Some hosts cannot make device allocations of their own (their device memory
is owned by another runtime, or every allocation must go through the
application's allocator).  ch3d_poisson_noalloc serves them: the caller
passes device inputs and outputs, and the solve works in one static device
array of the library.  This test calls it through the C ABI twice in a row and
checks both results against the context-based ch3d_poisson and against the
CPU oracle's clcPPE (src/CFD_2nd/m_Poisson.f90:1078-1201), with no-slip and
free-slip walls.  The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from helpers import rel_l2, small_channel

pytestmark = pytest.mark.gpu


def test_noalloc_poisson_matches_context_solve(built):
    import torch
    from channel3d_b200 import ChannelSolver, _lib, mesh_y
    lib = _lib.load_library()
    cfg = small_channel(48, 40, 24)
    yp = np.ascontiguousarray(mesh_y(cfg))
    rng = np.random.default_rng(11)
    srcs = [rng.standard_normal(cfg.shape), rng.standard_normal(cfg.shape)]
    with ChannelSolver(cfg, yp=yp) as s:
        refs = [s.poisson(a) for a in srcs]
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    for src, ref in zip(srcs, refs):
        d_src = torch.from_numpy(src.copy()).cuda()
        d_phi = torch.full_like(d_src, float("nan"))
        rc = lib.ch3d_poisson_noalloc(cfg.nxc, cfg.nyc, cfg.nzc, cfg.xlx, cfg.zlz, _lib.dptr(yp),
                                      cfg.BcOption[2], cfg.BcOption[3], ctypes.c_void_p(d_src.data_ptr()),
                                      ctypes.c_void_p(d_phi.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.ch3d_last_error()
        torch.cuda.synchronize()
        phi = d_phi.cpu().numpy()
        assert np.isfinite(phi).all()
        assert rel_l2(phi, ref) < 1e-12, rel_l2(phi, ref)


def test_noalloc_rejects_oversized_grids(built):
    import torch
    from channel3d_b200 import _lib
    lib = _lib.load_library()
    nx, ny, nz = 512, 256, 512
    yp = np.linspace(0.0, 2.0, ny + 1)
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = lib.ch3d_poisson_noalloc(nx, ny, nz, 6.28, 3.14, _lib.dptr(yp), -1, -1, ctypes.c_void_p(d.data_ptr()),
                                  ctypes.c_void_p(d.data_ptr()), None)
    assert rc == _lib.CH3D_ERR_INVALID
    assert b"CH3D_NOALLOC_SCRATCH_BYTES" in lib.ch3d_last_error()


def _noalloc(lib, cfg, yp, src, bc=(-1, -1), device=0):
    import torch
    from channel3d_b200 import _lib
    with torch.cuda.device(device):
        stream = torch.cuda.current_stream()
        d_src = torch.from_numpy(np.ascontiguousarray(src)).to(f"cuda:{device}")
        d_phi = torch.full_like(d_src, float("nan"))
        rc = lib.ch3d_poisson_noalloc(cfg.nxc, cfg.nyc, cfg.nzc, cfg.xlx, cfg.zlz, _lib.dptr(yp), bc[0], bc[1],
                                      ctypes.c_void_p(d_src.data_ptr()), ctypes.c_void_p(d_phi.data_ptr()),
                                      ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.ch3d_last_error()
        torch.cuda.synchronize()
        return d_phi.cpu().numpy()


@pytest.mark.parametrize("bc", [(-1, -1), (-1, -2)])
def test_noalloc_poisson_matches_oracle(built, bc):
    """Two calls in a row against the oracle's Poisson solve (1e-12), with a
    free-slip top wall in the second case (the pressure equation's y metrics
    are the same for both wall types, m_MeshAndMetries.f90:227-238)."""
    from channel3d_b200 import _lib, mesh_y
    from oracle import oracle as O
    lib = _lib.load_library()
    cfg = small_channel(48, 40, 24).copy(BcOption=[0, 0, bc[0], bc[1], 0, 0])
    yp = np.ascontiguousarray(mesh_y(cfg))
    o = O.Oracle(cfg)
    rng = np.random.default_rng(12)
    for _ in range(2):
        src = rng.standard_normal(cfg.shape)
        phi = _noalloc(lib, cfg, yp, src, bc)
        ref = o.poisson(src)
        assert rel_l2(phi, ref) < 1e-12, rel_l2(phi, ref)


def test_noalloc_on_a_second_device(built):
    """The set-up is per device: a call on device 1 after device 0 succeeds and
    agrees with device 0 (needs two visible GPUs)."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("one visible GPU")
    from channel3d_b200 import _lib, mesh_y
    lib = _lib.load_library()
    cfg = small_channel(48, 40, 24)
    yp = np.ascontiguousarray(mesh_y(cfg))
    src = np.random.default_rng(13).standard_normal(cfg.shape)
    a = _noalloc(lib, cfg, yp, src, device=0)
    b = _noalloc(lib, cfg, yp, src, device=1)
    assert rel_l2(b, a) < 1e-14

