"""Statistics of the 4th-order solver on the device against the oracle: the
35 moments of clcStat (src/CFD_4th/m_FlowCase.f90:330-640) and the 98
gradient moments of its HighOrderGradStat block (:485-589), accumulated in
FP64 every other step.

Tolerances: SumStat within 1e-11 relative (max norm over the array, as the
2nd-order statistics); SumGrad moment <a^m> within 1e-10 of a_rms^m, the
quantity's rms over the plane to the same power (largest over y): the odd
moments of x and z derivatives telescope to round-off over the periodic
directions, so a moment's own size is no scale for them."""
import numpy as np
import pytest

from helpers import rel_max

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


@pytest.mark.parametrize("shape", [(32, 24, 16), (48, 40, 36)])
def test_statistics_parity_4th(built, shape):
    o, s = _pair(cfg4(*shape))
    for _ in range(3):
        s.step(2)
        o.step(2)
        s.stats_accumulate()
        o.stats_accumulate()
    a, na, pa = s.stats_fetch()
    b, nb, pb = o.stats_get()
    assert na == nb == 3
    assert rel_max(a, b) < 1e-11, rel_max(a, b)
    assert abs(pa - pb) <= 1e-10 * max(1.0, abs(pb))
    ga = s.stats_fetch_grad()
    gb, _ = o.stats_get_grad()
    scale = np.empty(98)
    prms = np.sqrt(np.maximum(b[:, 7] / nb, 0.0)).max()  # <p^2> of SumStat (sums of nb samples)
    scale[0], scale[1] = prms ** 3, prms ** 4
    for t in range(24):  # SumVec2(3 + 4t .. 6 + 4t): the powers 1..4 of gradient t
        rms = np.sqrt(np.maximum(gb[:, 3 + 4 * t] / nb, 0.0)).max()
        scale[2 + 4 * t: 6 + 4 * t] = [rms, rms ** 2, rms ** 3, rms ** 4]
    err = np.abs(ga - gb).max(axis=0) / nb / np.maximum(scale, 1e-300)
    assert err.max() < 1e-10, (int(err.argmax()) + 1, err.max())
    # the moments the nyp row carries (SumVec2 7..10 and 31..34) are non-zero there
    assert np.all(gb[-1, 6:10] != 0) and np.all(gb[-1, 30:34] != 0)
    s.stats_fetch(reset=True)
    assert not s.stats_fetch_grad().any()
    s.close()


def test_statistics_4th_mixed_precision(built):
    """The mixed path's statistics (FP32 fields, FP64 sums) stay within 1e-4
    of the FP64 oracle's mean-velocity and rms moments after 10 steps."""
    cfg = cfg4(32, 24, 16)
    o, _ = _pair(cfg)
    _, s = _pair(cfg.copy(precision="mixed"))
    s.step(10)
    o.step(10)
    s.stats_accumulate()
    o.stats_accumulate()
    a, _, _ = s.stats_fetch()
    b, _, _ = o.stats_get()
    for q in (0, 4, 5, 6):  # <u>, <u^2>, <v^2>, <w^2>
        assert rel_max(a[:, q], b[:, q]) < 1e-4, (q, rel_max(a[:, q], b[:, q]))
    s.close()
