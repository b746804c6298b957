"""The synthetic channel workloads the benchmarks and parity tests run.

All are turbulent-channel set-ups of the 2nd/4th-order solvers: periodic x,z,
no-slip walls (BcOption 0 0 -1 -1 0 0), tanh-stretched y in two sections
(StretType 1 1, StretOption 0 1, SectioncStret 2.0 2.0), constant flow rate
U_b = 1 with h = 1 (yly = 2), xnu = 2 U_b h / Re_b, RK3 with fixed dt.
"""
import numpy as np

from .config import ChannelConfig


def channel(nxc, nyc, nzc, xlx, zlz, re_b, dt, order=2, implicit=1, precision="fp64", stret=2.0, **kw):
    half = nyc // 2
    return ChannelConfig(order=order, nxc=nxc, nyc=nyc, nzc=nzc, xlx=xlx, yly=2.0, zlz=zlz, xnu=2.0 / re_b,
                         dtMax=dt, iCFL=2, IsImplicit=implicit, nSection=2, SectionLength=[1.0, 1.0],
                         nycSection=[half, nyc - half], StretType=[1, 1], StretOption=[0, 1],
                         SectioncStret=[stret, stret], precision=precision, **kw)


# name -> (factory, timed steps); the factories return a fresh ChannelConfig
WORKLOADS = {
    # 2nd-order partially implicit, 64^3, Re_b 5600, dt 0.002, 200 steps
    "channel64_re5600": (lambda **kw: channel(64, 64, 64, 2 * np.pi, np.pi, 5600.0, 0.002, **kw), 200),
    # 4th-order solver, 128^3, 4pi x 2 x 4pi/3, Re_b 5600, dt 0.001, 1000 steps
    "channel128_re5600_4th": (lambda **kw: channel(128, 128, 128, 4 * np.pi, 4 * np.pi / 3, 5600.0, 0.001, order=4, **kw), 1000),
    # 2nd-order fully implicit (ADI: periodic x, periodic z, then y Crank-Nicolson), 128^3, same box
    "channel128_re5600_fimp": (lambda **kw: channel(128, 128, 128, 4 * np.pi, 4 * np.pi / 3, 5600.0, 0.001, implicit=2, **kw), 1000),
    # 2nd-order, 256x192x256, Re_b 13750, dt 0.0005, 2000 steps (FP64 vs mixed)
    "channel256x192x256_re13750": (lambda **kw: channel(256, 192, 256, 2 * np.pi, np.pi, 13750.0, 0.0005, **kw), 2000),
    # LES grid, 48^3, 2pi x 2 x pi, dt 0.002
    "channel48_les": (lambda **kw: channel(48, 48, 48, 2 * np.pi, np.pi, 13750.0, 0.002, **kw), 20000),
    # 2nd-order, 768x384x576 (~170M cells), Re_b 21900, dt 0.0003, 200 timed steps
    "channel768x384x576_re21900": (lambda **kw: channel(768, 384, 576, 2 * np.pi, np.pi, 21900.0, 0.0003, **kw), 200),
}


def taylor_green(n=64, xnu=6.25e-4, dt=0.01, **kw):
    """The Taylor-Green vortex of Input/TaylorGreenVortex.prm (FlowType 3, V = L = 1,
    xnu 6.25e-4, dt 0.01 fixed) in a 2pi x pi x 2pi box with free-slip walls at
    y = 0 and pi (half a period of the triply periodic vortex, whose symmetry
    the walls keep), n x n/2 x n uniform cells (dy = dx, so the staggered
    initial field is discretely divergence-free); no forcing."""
    return ChannelConfig(FlowType=3, nxc=n, nyc=n // 2, nzc=n, xlx=2 * np.pi, yly=np.pi, zlz=2 * np.pi, xnu=xnu,
                         dtMax=dt, iCFL=2, IsImplicit=1, BcOption=[0, 0, -2, -2, 0, 0], IsUxConst=False, ubulk=0.0,
                         ybulk1=0.0, ybulk2=np.pi, nSection=1, SectionLength=[1.0], nycSection=[n // 2],
                         StretType=[0], StretOption=[0], SectioncStret=[0.0], RunName="TGVortex", **kw)


def taylor_green_periodic(n=64, xnu=6.25e-4, dt=0.01, **kw):
    """The Taylor-Green vortex of Input/TaylorGreenVortex.prm (FlowType 3, V = L = 1,
    xnu 6.25e-4, dt 0.01 fixed) in its triply periodic 2pi x 2pi x 2pi box
    (BcOption 0 0 0 0 0 0), n^3 uniform cells, with the fully implicit step
    (IsImplicit 2: clcU*Hat_FIMP_000 and clcPPE_z1_periodic; the reference's
    input runs the explicit scheme, IsImplicit 0, which is not built); no forcing."""
    return ChannelConfig(FlowType=3, nxc=n, nyc=n, nzc=n, xlx=2 * np.pi, yly=2 * np.pi, zlz=2 * np.pi, xnu=xnu,
                         dtMax=dt, iCFL=2, IsImplicit=2, BcOption=[0, 0, 0, 0, 0, 0], IsUxConst=False, ubulk=0.0,
                         ybulk1=0.0, ybulk2=2 * np.pi, nSection=1, SectionLength=[1.0], nycSection=[n],
                         StretType=[0], StretOption=[0], SectioncStret=[0.0], RunName="TGVortex", **kw)


def get(name, **kw):
    factory, steps = WORKLOADS[name]
    return factory(**kw), steps
