"""Numpy restatement of the learned closure's per-point quantities (test
checker for channel3d_b200/csrc/ch3d_les.cu k_sgs_mlp (its inputs) and
k_sgs_train_samples): cell-centre velocity gradients with the WALE stencils
of src/CFD_2nd/m_LESModels.f90:98-111, the Smagorinsky / van Driest
fallback stress, y+ and the box-filtered training samples."""
import numpy as np


def mesh(cfg, yp):
    ny = cfg.nyc
    dyp = yp[1:] - yp[:-1]
    yc = 0.5 * (yp[1:] + yp[:-1])
    dyc = np.empty(ny + 1)          # jc = 1..nyp
    dyc[0] = dyp[0]
    dyc[1:ny] = yc[1:] - yc[:-1]
    dyc[ny] = dyp[-1]
    return dyp, yc, 1.0 / dyc


def ghost_view(G):
    """G: oracle ghosted array (nz+3, ny+3, nx+3), Fortran bounds 0..n+2."""
    nz, ny, nx = G.shape[0] - 3, G.shape[1] - 3, G.shape[2] - 3
    return lambda di, dj, dk: G[1 + dk:1 + dk + nz, 1 + dj:1 + dj + ny, 1 + di:1 + di + nx]


def fields(o, cfg):
    shp = (cfg.nzc + 3, cfg.nyc + 3, cfg.nxc + 3)
    return [ghost_view(o.get_ghosted(w).reshape(shp)) for w in (o.UX, o.UY, o.UZ)]


def gradients(o, cfg, yp):
    U, V, W = fields(o, cfg)
    dyp, yc, rdyc = mesh(cfg, yp)
    rdx, rdz = cfg.nxc / cfg.xlx, cfg.nzc / cfg.zlz
    caj = (1.0 / dyp)[None, :, None]
    cac1 = rdyc[:-1][None, :, None]
    cac2 = rdyc[1:][None, :, None]
    cac12 = cac1 - cac2
    g = np.empty((9,) + cfg.shape)
    g[0] = (U(1, 0, 0) - U(0, 0, 0)) * rdx
    g[1] = ((U(1, 1, 0) + U(0, 1, 0)) * cac2 + (U(1, 0, 0) + U(0, 0, 0)) * cac12 - (U(1, -1, 0) + U(0, -1, 0)) * cac1) * 0.25
    g[2] = (U(1, 0, 1) + U(0, 0, 1) - U(1, 0, -1) - U(0, 0, -1)) * rdz * 0.25
    g[3] = (V(1, 1, 0) - V(-1, 1, 0) + V(1, 0, 0) - V(-1, 0, 0)) * rdx * 0.25
    g[4] = (V(0, 1, 0) - V(0, 0, 0)) * caj
    g[5] = (V(0, 1, 1) + V(0, 0, 1) - V(0, 1, -1) - V(0, 0, -1)) * rdz * 0.25
    g[6] = (W(1, 0, 1) - W(-1, 0, 1) + W(1, 0, 0) - W(-1, 0, 0)) * rdx * 0.25
    g[7] = ((W(0, 1, 1) + W(0, 1, 0)) * cac2 + (W(0, 0, 1) + W(0, 0, 0)) * cac12 - (W(0, -1, 1) + W(0, -1, 0)) * cac1) * 0.25
    g[8] = (W(0, 0, 1) - W(0, 0, 0)) * rdz
    return g


def utau(ux, cfg, yp):
    yc = 0.5 * (yp[1:] + yp[:-1])
    m1, mN = ux[:, 0, :].mean(), ux[:, -1, :].mean()
    tw = cfg.xnu * 0.5 * (abs(m1) / (yc[0] - yp[0]) + abs(mN) / (yp[-1] - yc[-1]))
    return np.sqrt(tw)


def smag_tau(g, cfg, yp, ut):
    dyp, yc, _ = mesh(cfg, yp)
    S11, S22, S33 = g[0], g[4], g[8]
    S12, S13, S23 = 0.5 * (g[1] + g[3]), 0.5 * (g[2] + g[6]), 0.5 * (g[5] + g[7])
    Sm = np.sqrt(2.0 * (S11 ** 2 + S22 ** 2 + S33 ** 2 + 2.0 * (S12 ** 2 + S13 ** 2 + S23 ** 2)))
    dw = np.minimum(yc - yp[0], yp[-1] - yc)
    D = 1.0 - np.exp(-(dw * ut / cfg.xnu) / 26.0)
    delta = (dyp * (cfg.xlx / cfg.nxc) * (cfg.zlz / cfg.nzc)) ** (1.0 / 3.0)
    l = (cfg.Cs * D * delta)[None, :, None]
    nt = l * l * Sm
    return np.stack([-2 * nt * S11, -2 * nt * S12, -2 * nt * S13, -2 * nt * S22, -2 * nt * S23, -2 * nt * S33])


def features(g, cfg, yp, ut):
    """Network inputs (unstandardised): gradients in wall units and y+, shape (N, 10)."""
    _, yc, _ = mesh(cfg, yp)
    dw = np.minimum(yc - yp[0], yp[-1] - yc)
    yplus = np.broadcast_to((dw * ut / cfg.xnu)[None, :, None], cfg.shape)
    return np.concatenate([g.reshape(9, -1) * (cfg.xnu / ut ** 2), yplus.reshape(1, -1)]).T
