"""Resampling a channel state onto another grid (ch3d_interp_state), the
reference's interpolateField tool (Tool/interpolateField/src/m_Interp.f90:
Interp_init :20-179, Interp_uvwp :184-361), against the oracle's restatement
of the same tool: coarsening (a DNS field onto a coarser LES-like grid) and
refining, with other stretchings of y, and a free-slip top.  The resampled
field then serves as a restart: a few steps from it agree with the oracle's.

Tolerances: FP64 resampled fields within 1e-12 relative (max norm; the
device forms the same eight-term sums with fused multiply-adds), 1e-6 in
mixed precision (FP32 fields); steps after it within 1e-10."""
import numpy as np
import pytest

from helpers import rel_l2, rel_max, small_channel

pytestmark = pytest.mark.gpu


def _state(cfg, seed=0x5EED):
    from channel3d_b200 import initfield, mesh_y
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=mesh_y(cfg), seed=seed)
    p = 0.01 * np.random.default_rng(seed).standard_normal(cfg.shape)
    return ux, uy, uz, p


GRIDS = {
    # name: (old grid, new grid)
    "coarsen": (dict(nx=48, ny=32, nz=24), dict(nx=32, ny=24, nz=16, StretType=[2, 2], SectioncStret=[1.0, 1.0])),
    "refine": (dict(nx=32, ny=24, nz=16), dict(nx=64, ny=40, nz=36)),
    "halfchannel": (dict(nx=32, ny=24, nz=16, half=True), dict(nx=48, ny=32, nz=24, half=True)),
}


def _cfg(d, **kw):
    d = dict(d)
    half = d.pop("half", False)
    nx, ny, nz = d.pop("nx"), d.pop("ny"), d.pop("nz")
    cfg = small_channel(nx, ny, nz, **d, **kw)
    if half:
        cfg = cfg.copy(FlowType=2, yly=1.0, nSection=1, SectionLength=[1.0], nycSection=[ny], StretType=[1],
                       StretOption=[0], SectioncStret=[2.0], BcOption=[0, 0, -1, -2, 0, 0])
    return cfg


@pytest.mark.parametrize("name", sorted(GRIDS))
def test_interp_matches_oracle(built, name):
    from channel3d_b200 import ChannelSolver
    from oracle import oracle as O
    old, new = (_cfg(g) for g in GRIDS[name])
    st = _state(old)
    os_, on = O.Oracle(old), O.Oracle(new)
    os_.set_state(*st)
    on.interp_from(os_)
    go = on.get_state(hist=True)
    with ChannelSolver(old) as s_old, ChannelSolver(new) as s_new:
        s_old.upload(*st)
        s_new.interp_from(s_old)
        gs = s_new.download(hist=True)
        for k in ("ux", "uy", "uz", "p"):
            assert rel_max(gs[k], go[k]) < 1e-12, (name, k, rel_max(gs[k], go[k]))
        assert not gs["hist"].any()
        # the resampled field as a restart
        di = s_new.step(5)
        do = on.step(5)
        gs = s_new.download()
        go = on.get_state()
        for k in ("ux", "uy", "uz", "p"):
            assert rel_l2(gs[k], go[k]) < 1e-10, (name, "after steps", k, rel_l2(gs[k], go[k]))
        assert abs(di["uxm"] - do["uxm"]) < 1e-10


def test_interp_holds_the_flow_rate(built):
    """With IsUxConst the resampled ux carries the bulk velocity ubulk
    (Interp_uvwp :225-236): the y-weighted mean over the new grid is ubulk."""
    from channel3d_b200 import ChannelSolver
    old, new = _cfg(GRIDS["coarsen"][0]), _cfg(GRIDS["coarsen"][1], ubulk=0.9)
    with ChannelSolver(old) as s_old, ChannelSolver(new) as s_new:
        s_old.upload(*_state(old))
        s_new.interp_from(s_old)
        ux = s_new.download()["ux"]
        dy = np.diff(s_new.yp)
        mean = (ux * dy[None, :, None]).sum() / (new.nxc * new.nzc * new.yly)
        assert abs(mean - 0.9) < 1e-12, mean


def test_interp_mixed_precision(built):
    from channel3d_b200 import ChannelSolver
    from oracle import oracle as O
    old, new = (_cfg(g) for g in GRIDS["refine"])
    st = _state(old)
    os_, on = O.Oracle(old), O.Oracle(new)
    os_.set_state(*st)
    on.interp_from(os_)
    go = on.get_state()
    with ChannelSolver(old.copy(precision="mixed")) as s_old, ChannelSolver(new.copy(precision="mixed")) as s_new:
        s_old.upload(*st)
        s_new.interp_from(s_old)
        gs = s_new.download()
    for k in ("ux", "uy", "uz", "p"):
        assert rel_max(gs[k], go[k]) < 1e-6, (k, rel_max(gs[k], go[k]))


def test_interp_rejects_mismatched_contexts(built):
    from channel3d_b200 import ChannelSolver, _lib
    a = ChannelSolver(small_channel(32, 24, 16))
    b = ChannelSolver(small_channel(32, 24, 16, yly=3.0))
    c = ChannelSolver(small_channel(32, 24, 16, precision="mixed"))
    for dst, src in ((b, a), (c, a), (a, a)):
        assert a.lib.ch3d_interp_state(dst.ctx, src.ctx) == _lib.CH3D_ERR_INVALID
    for s in (a, b, c):
        s.close()
