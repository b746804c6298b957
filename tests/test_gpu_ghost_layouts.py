"""The ghosted array layouts of the C ABI, which a Fortran host of the
reference passes straight from its own arrays, and the free-slip walls.

Upload takes the interior of a ghosted array; download writes the interior
and rebuilds the ghost cells with the reference's boundary and halo rules
(SetBC_and_UpdateHalo and SetBC_and_UpdateHalo_pr: src/CFD_2nd/m_BC_and_Halo.f90:
232-344, 410-456 with one halo plane per side; src/CFD_4th/m_BC_and_Halo.f90:
51-96, 136-150 with two, and one above for the pressure).  The oracle keeps
the reference's ghosted arrays and applies those routines after every
substep, so each whole array, ghosts included, is compared with the oracle's
after a few steps.  Cells the reference never writes hold zero in both (the
oracle allocates zeros; the download leaves them as the host array had them).

Tolerance: 1e-10 relative (max norm over the whole array), the whole-step
bound of the FP64 path.
"""
import numpy as np
import pytest

from helpers import rel_l2, rel_max, small_channel

pytestmark = pytest.mark.gpu


def _half_channel(nx, ny, nz, bc_lo=-1, **kw):
    """Half channel of the 2nd-order tree (FlowType 2): no-slip (or free-slip)
    bottom, free-slip top, one tanh-stretched section of height 1."""
    cfg = small_channel(nx, ny, nz)
    return cfg.copy(FlowType=2, yly=1.0, nSection=1, SectionLength=[1.0], nycSection=[ny], StretType=[1],
                    StretOption=[0], SectioncStret=[2.0], BcOption=[0, 0, bc_lo, -2, 0, 0], **kw)


def _start(cfg, seed=0x5EED):
    from channel3d_b200 import initfield, mesh_y
    yp = mesh_y(cfg)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp, seed=seed)
    p = 0.01 * np.random.default_rng(seed).standard_normal(cfg.shape)
    return yp, (ux, uy, uz, p)


CASES = {
    # name: (config factory, layout, steps)
    "pimp_ghost2": (lambda: small_channel(32, 24, 16), "GHOST2", 5),
    "fimp_ghost2": (lambda: small_channel(32, 24, 16, IsImplicit=2), "GHOST2", 5),
    "order4_ghost4": (lambda: small_channel(32, 24, 16, order=4), "GHOST4", 5),
    "halfchannel_freeslip_ghost2": (lambda: _half_channel(32, 24, 16), "GHOST2", 5),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_ghosted_layout_matches_oracle_arrays(built, name):
    from channel3d_b200 import ChannelSolver, _lib
    from oracle import oracle as O
    factory, lay, nsteps = CASES[name]
    cfg = factory()
    layout = getattr(_lib, "LAYOUT_" + lay)
    yp, st = _start(cfg)
    o = O.Oracle(cfg)
    o.set_state(*st)
    ids = {"ux": O.Oracle.UX, "uy": O.Oracle.UY, "uz": O.Oracle.UZ, "p": O.Oracle.P}  # array ids of orc_get_array
    with ChannelSolver(cfg, yp=yp) as s:
        shp = s.layout_shape(layout)
        # the host passes its ghosted arrays as they are (the oracle's, here)
        g0 = {k: o.get_ghosted(w).reshape(shp) for k, w in ids.items()}
        s.upload(g0["ux"], g0["uy"], g0["uz"], g0["p"], layout=layout)
        s.step(nsteps)
        got = s.download(layout=layout)
    o.step(nsteps)
    for k, w in ids.items():
        ref = o.get_ghosted(w).reshape(shp)
        e = rel_max(got[k], ref)
        assert e < 1e-10, (name, k, e, np.unravel_index(np.argmax(np.abs(got[k] - ref)), shp))


def test_ghosted_download_keeps_cells_outside_the_rules(built):
    """Cells the reference's routines never write keep the host's values."""
    from channel3d_b200 import ChannelSolver, _lib
    cfg = small_channel(32, 24, 16)
    yp, st = _start(cfg)
    with ChannelSolver(cfg, yp=yp) as s:
        s.upload(*st)
        shp = s.layout_shape(_lib.LAYOUT_GHOST2)
        out = {k: np.full(shp, 7.0) for k in ("ux", "uy", "uz", "p")}
        s.download(layout=_lib.LAYOUT_GHOST2, out=out)
    nx, ny, nz = cfg.nxc, cfg.nyc, cfg.nzc
    for k in ("ux", "uy", "uz", "p"):
        a = out[k]  # C order (k, j, i) over (0:nzc+2, 0:nyc+2, 0:nxc+2)
        assert np.all(a[1:nz + 1, 1:ny + 1, nx + 2] == 7.0), k  # x = nxc+2 never written
    assert np.all(out["ux"][1:nz + 1, ny + 2, 1:nx + 1] == 7.0)  # ux(:,nyp+1,:) never written
    assert not np.any(out["uy"][1:nz + 1, ny + 2, 1:nx + 1] == 7.0)  # uy(:,nyp+1,:) is


@pytest.mark.parametrize("bc_lo", [-1, -2])
def test_free_slip_step_parity(built, bc_lo):
    """Free-slip walls (BcOption -2, src/CFD_2nd/m_BC_and_Halo.f90:247-282 and
    the Crank-Nicolson wall coefficients of src/CFD_2nd/m_TScheme.f90:73-85):
    20 steps of a half channel against the oracle, FP64 within 1e-10."""
    from channel3d_b200 import ChannelSolver
    from oracle import oracle as O
    cfg = _half_channel(48, 32, 24, bc_lo=bc_lo)
    yp, st = _start(cfg)
    o = O.Oracle(cfg)
    o.set_state(*st)
    with ChannelSolver(cfg, yp=yp) as s:
        s.upload(*st)
        di = s.step(20)
        gs = s.download()
    do = o.step(20)
    go = o.get_state()
    for k in ("ux", "uy", "uz", "p"):
        assert rel_l2(gs[k], go[k]) < 1e-10, (k, rel_l2(gs[k], go[k]))
    assert abs(di["PrGradAver"] - do["PrGradAver"]) <= 1e-10 * max(1.0, abs(do["PrGradAver"]))
    assert di["divmax2"] < 1e-12


def test_free_slip_mixed_precision(built):
    """The mixed path with a free-slip top stays within 1e-4 of the FP64 oracle."""
    from channel3d_b200 import ChannelSolver
    from oracle import oracle as O
    cfg = _half_channel(48, 32, 24)
    yp, st = _start(cfg)
    o = O.Oracle(cfg)
    o.set_state(*st)
    with ChannelSolver(cfg.copy(precision="mixed"), yp=yp) as s:
        s.upload(*st)
        s.step(20)
        gs = s.download()
    o.step(20)
    go = o.get_state()
    for k in ("ux", "uy", "uz"):
        assert rel_l2(gs[k], go[k]) < 1e-4, (k, rel_l2(gs[k], go[k]))
