"""Parity of the LES step (2nd order, partially implicit, FP64) on the device
with the CPU oracle through the C ABI: the eddy viscosity of the WALE,
mixed-time-scale and Smagorinsky / van Driest models, the variable-viscosity
right-hand sides and y solves, and whole steps of the 48^3 LES channel.

Tolerances: nut within 1e-12 relative (max norm), stage results within
5e-12, whole steps within 1e-10 (L2)."""
import numpy as np
import pytest

from helpers import rel_l2, rel_max

pytestmark = pytest.mark.gpu

MODELS = (2, 3, 10)


def cfgl(model, nx=48, ny=48, nz=48):
    from channel3d_b200 import workloads
    cfg, _ = workloads.get("channel48_les")
    return cfg.copy(nxc=nx, nyc=ny, nzc=nz, nycSection=[ny // 2, ny - ny // 2], LES_type=model, Cs=0.1)


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


@pytest.mark.parametrize("model", MODELS)
def test_sgs_viscosity_parity(built, model):
    o, s = _pair(cfgl(model, 32, 24, 16))
    a = s.sgs_viscosity()
    b, _ = o.sgs()
    assert rel_max(a, b) < 1e-12, rel_max(a, b)


@pytest.mark.parametrize("model", MODELS)
def test_stage_parity_les(built, model):
    o, s = _pair(cfgl(model, 32, 24, 16))
    s.sgs_viscosity()
    o.sgs()
    for ns in (1, 2, 3):
        o.stage(0, ns); s.stage(0, ns)
        o.stage(1, ns); s.stage(1, ns)
        for wo, wg in ((o.ARR1, s.RHSX), (o.ARR2, s.RHSY), (o.HALO, s.RHSZ), (o.HISTX, s.HISTX),
                       (o.HISTY, s.HISTY), (o.HISTZ, s.HISTZ)):
            a, b = s.get_array(wg), o.get_interior(wo)
            if wg == s.RHSY:  # row jc=1 is replaced by the wall condition in clcU2Hat
                a, b = a[:, 1:, :], b[:, 1:, :]
            assert rel_max(a, b) < 5e-12, (ns, wg, rel_max(a, b))
        o.stage(2, ns); s.stage(2, ns)
        go = o.get_state()
        for k, w in (("ux", 12), ("uy", 13), ("uz", 14)):
            ustar = s.get_array(w)
            assert rel_max(ustar, go[k]) < 1e-12, (ns, "uhat", k, rel_max(ustar, go[k]))
        for st in (3, 4, 5, 6):
            o.stage(st, ns); s.stage(st, ns)
        go, gs = o.get_state(), s.download()
        for k in ("ux", "uy", "uz", "p"):
            assert rel_max(gs[k], go[k]) < 1e-11, (ns, "final", k, rel_max(gs[k], go[k]))


@pytest.mark.parametrize("model", MODELS)
def test_step_parity_les_48cubed(built, model):
    o, s = _pair(cfgl(model))
    di = s.step(100)
    do = o.step(100)
    go, gs = o.get_state(), s.download()
    for k in ("ux", "uy", "uz", "p"):
        e = rel_l2(gs[k], go[k])
        assert e < 1e-10, (model, k, e)
    assert di["divmax2"] < 1e-12
    assert rel_max(s.get_array(s.NUT), o.get_interior(o.NUT)) < 1e-10


@pytest.mark.parametrize("model", MODELS)
def test_les_mixed_precision(built, model):
    """The LES step in the mixed path (FP32 fields; the eddy viscosity and the
    variable-viscosity solves computed in FP64 from them): 50 steps of the
    48^3 LES channel within 1e-4 (L2) of the FP64 oracle, nut within 1e-4."""
    o, _ = _pair(cfgl(model))
    _, s = _pair(cfgl(model).copy(precision="mixed"))
    di = s.step(50)
    o.step(50)
    go, gs = o.get_state(), s.download()
    for k in ("ux", "uy", "uz"):
        e = rel_l2(gs[k], go[k])
        assert e < 1e-4, (model, k, e)
    assert di["status"] == 0 and di["divmax2"] < 1e-4
    assert rel_l2(s.get_array(s.NUT), o.get_interior(o.NUT)) < 1e-4
    s.close()
