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


def large_scale(cfg, amplitude=0.3, seed=SEED, yp=None, ubulk=1.0, kmax=4):
    """Laminar profile plus large-scale perturbations that trigger transition:
    a sum of Fourier modes |kx|, |kz| <= kmax (random phases and amplitudes
    from the seeded generator) shaped by (1 - (y-1)^2) so that they vanish at
    the walls, scaled to `amplitude` * U_b in max norm per component.  The
    field is not divergence-free; ChannelSolver.project() makes it so.  (The
    white-noise start of laminar_noise decays on fine grids.)"""
    if yp is None:
        yp = mesh_y(cfg)
    yc = cell_centres(yp)
    rng = np.random.Generator(np.random.Philox(key=seed + 1))
    nz, ny, nx = cfg.shape
    x = (np.arange(nx) + 0.5) * cfg.xlx / nx
    z = (np.arange(nz) + 0.5) * cfg.zlz / nz
    eta = yc / (0.5 * cfg.yly) - 1.0
    env = (1.0 - eta ** 2)
    prof = 1.5 * ubulk * env
    out = []
    for comp in range(3):
        f = np.zeros((nz, ny, nx))
        for kx in range(0, kmax + 1):
            for kz in range(-kmax, kmax + 1):
                if kx == 0 and kz == 0:
                    continue
                a, ph, ny_mode = rng.uniform(0.5, 1.0), rng.uniform(0, 2 * np.pi), rng.integers(1, 4)
                wave = np.cos(2 * np.pi * (kx * x[None, :] / cfg.xlx + kz * z[:, None] / cfg.zlz) + ph)
                yshape = env * np.sin(ny_mode * np.pi * (eta + 1.0) / 2.0 + rng.uniform(0, np.pi))
                f += a * wave[:, None, :] * yshape[None, :, None]
        f *= amplitude * ubulk / max(np.abs(f).max(), 1e-30)
        out.append(f)
    ux = out[0] + prof[None, :, None]
    uy = out[1]
    uy[:, 0, :] = 0.0
    uz = out[2]
    return ux, uy, uz, np.zeros((nz, ny, nx))


def taylor_green(cfg, yp=None, vel=1.0, length=1.0):
    """InitVelocity_TG (src/CFD_2nd/m_FlowType_TGVortex.f90:20-47) on the
    staggered mesh: ux(i,j,k) = V sin(x_i / L) cos(yc_j / L) cos(zc_k / L),
    uy = -V cos(xc_i / L) sin(yp_j / L) cos(zc_k / L), uz = 0, p = 0, with
    x_i = (i - 1) dx, xc = x + dx / 2 (the same in z), yp the y nodes and yc
    the cell centres.  The field is mirror-symmetric about y = 0 and y = pi L
    (uy odd, ux and uz even), so a box of height pi L with free-slip walls
    holds half a period of the triply periodic vortex; a box of height 2 pi L
    with periodic y holds the whole period."""
    if yp is None:
        yp = mesh_y(cfg)
    yp = np.asarray(yp)
    yc = cell_centres(yp)
    nx, nz = cfg.nxc, cfg.nzc
    dx, dz = cfg.xlx / nx, cfg.zlz / nz
    xp = np.arange(nx) * dx
    zp = np.arange(nz) * dz
    xc, zc = xp + 0.5 * dx, zp + 0.5 * dz
    ux = vel * np.sin(xp / length)[None, None, :] * np.cos(yc / length)[None, :, None] * np.cos(zc / length)[:, None, None]
    uy = -vel * np.cos(xc / length)[None, None, :] * np.sin(yp[:-1] / length)[None, :, None] * np.cos(zc / length)[:, None, None]
    uz = np.zeros(cfg.shape)
    p = np.zeros(cfg.shape)
    return np.ascontiguousarray(ux), np.ascontiguousarray(uy), uz, p

