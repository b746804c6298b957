"""Seeded initial channel field (replaces the clock-seeded InitVelocity_CH,
src/CFD_2nd/m_FlowType_Channel.f90:37-115, whose random seed comes from
system_clock and so cannot be reproduced).

u = 1.5 U_b (1 - (y-1)^2) + a r,  v = a r,  w = a r,  p = 0,
with r ~ U(-1,1) drawn from numpy's Philox generator with a fixed key, one
component after the other in Fortran order, a = 0.1 U_b, y = yc (cell
centres), and uy = 0 on the bottom wall (uy(:,1,:) is the wall value).
The field can then be made discretely divergence-free with
ChannelSolver.project().
"""
import numpy as np

from .config import mesh_y

SEED = 0x5EED


def cell_centres(yp):
    yp = np.asarray(yp)
    return 0.5 * (yp[:-1] + yp[1:])


def laminar_noise(cfg, amplitude=0.1, seed=SEED, yp=None, ubulk=1.0):
    if yp is None:
        yp = mesh_y(cfg)
    yc = cell_centres(yp)
    rng = np.random.Generator(np.random.Philox(key=seed))
    shape = cfg.shape  # (nz, ny, nx)
    prof = 1.5 * ubulk * (1.0 - (yc / (0.5 * cfg.yly) - 1.0) ** 2)
    ux = rng.uniform(-1.0, 1.0, size=shape)
    ux *= amplitude * ubulk
    ux += prof[None, :, None]
    uy = rng.uniform(-1.0, 1.0, size=shape)
    uy *= amplitude * ubulk
    uy[:, 0, :] = 0.0
    uz = rng.uniform(-1.0, 1.0, size=shape)
    uz *= amplitude * ubulk
    p = np.zeros(shape)
    return ux, uy, uz, p
