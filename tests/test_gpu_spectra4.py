"""Spectra of the 4th-order statistics on the device
(ch3d_spectra_accumulate: clcStat's clcSpectra1D branch,
src/CFD_4th/m_FlowCase.f90:642-880, with clcEnergySpectraX/Z,
clcCospectraX/Z and clcLTS_x/z, and its clcSpectra2D branch with
clcSpecAndLCSR2DFrom1D and clcCosSpectra2D, :1896-2298) against the oracle,
which transforms every x and z line with R2HC as the reference does; the
device reaches the z and 2-D spectra through the 2-D spectrum and Parseval's
theorem along x.

Tolerance: each of the 2 x 18 one-dimensional and 9 two-dimensional spectra
within 1e-10 of its largest magnitude (FP64), 1e-4 for the mixed path's
energy spectra."""
import numpy as np
import pytest

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


# register transforms in both directions (128, 128) and the generic ones (48, 36)
@pytest.mark.parametrize("shape", [(48, 40, 36), (128, 32, 128)])
def test_spectra_parity_4th(built, shape):
    o, s = _pair(cfg4(*shape))
    jfor = (3, 7)
    for _ in range(2):
        s.step(2)
        o.step(2)
        s.spectra_accumulate(jfor)
        o.spectra_accumulate(jfor)
    ax, az, a2, na = s.spectra_fetch(two_d=True)
    bx, bz, nb = o.spectra_get()
    b2, _ = o.spectra_get2d()
    assert na == nb == 2
    for m in range(18):
        for a, b, d in ((ax, bx, "x"), (az, bz, "z")):
            e = np.abs(a[m] - b[m]).max() / max(np.abs(b[m]).max(), 1e-300)
            assert e < 1e-10, (d, m, e)
    for m in range(9):  # the 2-D spectra (clcSpectra2D)
        e = np.abs(a2[m] - b2[m]).max() / max(np.abs(b2[m]).max(), 1e-300)
        assert e < 1e-10, ("2d", m, e)
    s.spectra_fetch(reset=True)
    ax, az, n = s.spectra_fetch()
    assert n == 0 and not ax.any() and not az.any()
    # one sample: the energy spectra of uz sum to the plane mean squares (Parseval)
    s.spectra_accumulate(jfor)
    ax, az, n = s.spectra_fetch()
    ms = (s.download()["uz"] ** 2).mean(axis=(0, 2))
    assert n == 1
    assert np.allclose(ax[2].sum(axis=1), ms, rtol=1e-12) and np.allclose(az[2].sum(axis=1), ms, rtol=1e-12)
    s.close()


def test_spectra_mixed_precision(built):
    cfg = cfg4(48, 40, 36)
    o, _ = _pair(cfg)
    _, s = _pair(cfg.copy(precision="mixed"))
    s.spectra_accumulate((3, 7))
    o.spectra_accumulate((3, 7))
    ax, az, _ = s.spectra_fetch()
    bx, bz, _ = o.spectra_get()
    for m in range(4):
        for a, b in ((ax, bx), (az, bz)):
            assert np.abs(a[m] - b[m]).max() < 1e-4 * np.abs(b[m]).max(), m
    s.close()


def test_spectra_argument_checks(built):
    from channel3d_b200 import ChannelSolver, _lib
    from helpers import small_channel
    s = ChannelSolver(cfg4(48, 40, 36))
    assert s.lib.ch3d_spectra_accumulate(s.ctx, 0, 1) == _lib.CH3D_ERR_INVALID
    assert s.lib.ch3d_spectra_accumulate(s.ctx, 1, 21) == _lib.CH3D_ERR_INVALID
    s.close()
    s = ChannelSolver(small_channel(32, 24, 16))
    assert s.lib.ch3d_spectra_accumulate(s.ctx, 1, 1) == _lib.CH3D_ERR_UNSUPPORTED
    s.close()
