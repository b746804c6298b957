"""Training and evaluation pipeline of the learned subgrid-stress closure.

1. A DNS of the channel (the library's own FP64 step) produces snapshots;
   each is box filtered on the device (ch3d_sgs_training_samples: boxes of
   fx x fy x fz cells) into samples of the nine filtered velocity gradients
   and y+ (inputs, wall units) and the six SGS stresses tau_ij / u_tau^2
   (targets).
2. The inputs and targets are standardised; the network
   (include/ch3d_mlp.h, 10 -> 64 -> 64 -> 64 -> 6, GELU, BF16 tensor-core
   forward and backward) is trained with Adam on mini-batches.
3. The LES (LES_type = CH3D_LES_MLP) evaluates it every step; inputs outside
   the training range fall back to the Smagorinsky / van Driest stress.

torch holds the sample tensors and does the mini-batch bookkeeping; the
solver, the sampling, the network and the optimiser are the library's CUDA
kernels.  The model has no counterpart in the reference.
"""
import numpy as np

from . import initfield
from .mlp import MLPClosure
from .solver import ChannelSolver


def box_width(cfg, box):
    """Effective filter width (cube root of the box volume) at each box row, length nyc // fy."""
    from .config import mesh_y
    yp = mesh_y(cfg)
    fx, fy, fz = box
    dy = (yp[fy::fy] - yp[:-fy:fy])[: cfg.nyc // fy]
    return (fx * cfg.xlx / cfg.nxc * dy * fz * cfg.zlz / cfg.nzc) ** (1.0 / 3.0)


def collect_samples(cfg, steps, n_snapshots, per_snapshot, box=(4, 2, 4), seed=0, solver=None, state=None):
    """Runs the DNS `steps` steps and takes `n_snapshots` evenly spaced box-filtered
    snapshots, keeping `per_snapshot` random samples of each.  Returns the device
    tensors X [n x 10], T [n x 6], the filter width in wall units of every sample
    (for the Smagorinsky comparison) and the solver (for continuing the run)."""
    import torch
    from .config import mesh_y
    yp = mesh_y(cfg)
    wb = box_width(cfg, box)                                   # width of each box row
    yb = np.array([0.5 * (yp[j * box[1]] + yp[(j + 1) * box[1]]) for j in range(len(wb))])
    dwb = np.minimum(yb - yp[0], yp[-1] - yb)                  # wall distance of each box row
    s = solver or ChannelSolver(cfg)
    if solver is None:
        if state is None:
            state = initfield.laminar_noise(cfg, yp=s.yp)
        s.upload(*state)
        s.project()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    every = max(1, steps // n_snapshots)
    Xs, Ts, Ds = [], [], []
    nb = (cfg.nxc // box[0], cfg.nyc // box[1], cfg.nzc // box[2])
    row = np.broadcast_to(np.arange(nb[1])[None, :, None], (nb[2], nb[1], nb[0])).ravel()
    while len(Xs) < n_snapshots:
        s.step(every)
        X, T = s.sgs_training_samples(*box)
        # u_tau / xnu of this snapshot: y+ of any box over its wall distance
        ratio = float(X[0, 9].item()) / dwb[0]
        D = torch.as_tensor(wb[row] * ratio, device=X.device)
        if per_snapshot < X.shape[0]:
            idx = torch.randperm(X.shape[0], device=X.device, generator=gen)[:per_snapshot]
            X, T, D = X.index_select(0, idx), T.index_select(0, idx), D.index_select(0, idx)
        Xs.append(X.clone())
        Ts.append(T.clone())
        Ds.append(D.clone())
    return torch.cat(Xs), torch.cat(Ts), torch.cat(Ds), s


def fit_norm(X, T, margin=0.05):
    """Standardisation (52 floats: in_mean, in_std, in_lo, in_hi, out_mean, out_std);
    the accepted input range is the training range of the standardised inputs,
    widened by `margin` of its extent."""
    x = X.double()
    t = T.double()
    mu, sd = x.mean(0), x.std(0).clamp_min(1e-12)
    xs = (x - mu) / sd
    lo, hi = xs.min(0).values, xs.max(0).values
    w = hi - lo
    n = np.zeros(52, dtype=np.float32)
    n[0:10] = mu.cpu().numpy()
    n[10:20] = sd.cpu().numpy()
    n[20:30] = (lo - margin * w).cpu().numpy()
    n[30:40] = (hi + margin * w).cpu().numpy()
    n[40:46] = t.mean(0).cpu().numpy()
    n[46:52] = t.std(0).clamp_min(1e-12).cpu().numpy()
    return n


def standardise(X, T, norm):
    import torch
    n = torch.as_tensor(norm, device=X.device)
    Xs = ((X - n[0:10]) / n[10:20]).float().contiguous()
    Ts = None if T is None else ((T - n[40:46]) / n[46:52]).float().contiguous()
    return Xs, Ts


def train(X, T, norm, iters=2000, batch=65536, lr=1e-3, seed=0, log_every=100):
    """Adam on standardised mini-batches with the tensor-core gradient; returns the network and loss history."""
    Xs, Ts = standardise(X, T, norm)
    net = MLPClosure(seed=seed)
    hist = net.train(Xs, Ts, iters=iters, batch=min(batch, Xs.shape[0]), lr=lr, seed=seed, log_every=log_every)
    return net, hist


def predict(net, X, norm):
    """Network stresses tau / u_tau^2 for raw inputs X."""
    import torch
    Xs, _ = standardise(X, None, norm)
    n = torch.as_tensor(norm, device=X.device)
    return net.forward(Xs) * n[46:52] + n[40:46]


def smagorinsky(X, delta_plus, Cs=0.1):
    """Smagorinsky / van Driest stress tau / u_tau^2 from wall-unit gradients X[:, :9],
    y+ = X[:, 9] and the filter width in wall units delta_plus (per sample)."""
    import torch
    g = X[:, :9].double()
    S11, S22, S33 = g[:, 0], g[:, 4], g[:, 8]
    S12, S13, S23 = 0.5 * (g[:, 1] + g[:, 3]), 0.5 * (g[:, 2] + g[:, 6]), 0.5 * (g[:, 5] + g[:, 7])
    Sm = torch.sqrt(2.0 * (S11 ** 2 + S22 ** 2 + S33 ** 2 + 2.0 * (S12 ** 2 + S13 ** 2 + S23 ** 2)))
    D = 1.0 - torch.exp(-X[:, 9].double() / 26.0)
    nt = (Cs * D * delta_plus) ** 2 * Sm
    return torch.stack([-2 * nt * S11, -2 * nt * S12, -2 * nt * S13, -2 * nt * S22, -2 * nt * S23, -2 * nt * S33], 1)


def stress_error(pred, T):
    """Relative L2 error of predicted SGS stresses over all components."""
    d = (pred.double() - T.double())
    return float(d.norm() / T.double().norm())


def profiles(fields, cfg):
    """Mean streamwise velocity and rms of u, v, w at the cell centres (x-z averages)."""
    ux, uy, uz = fields["ux"], fields["uy"], fields["uz"]
    uc = 0.5 * (ux + np.roll(ux, -1, axis=2))
    vn = np.concatenate([uy, np.zeros_like(uy[:, :1, :])], axis=1)   # wall value above the top row
    vc = 0.5 * (vn[:, :-1, :] + vn[:, 1:, :])
    wc = 0.5 * (uz + np.roll(uz, -1, axis=0))
    U = uc.mean(axis=(0, 2))
    rms = [np.sqrt(((a - a.mean(axis=(0, 2), keepdims=True)) ** 2).mean(axis=(0, 2))) for a in (uc, vc, wc)]
    return {"U": U, "urms": rms[0], "vrms": rms[1], "wrms": rms[2]}


def profile_errors(p, ref, yp, yref):
    """Relative L2 errors of the profiles p (on centres of yp) against ref (on centres of yref),
    compared on the coarser set of centres by linear interpolation."""
    yc = 0.5 * (yp[1:] + yp[:-1])
    yr = 0.5 * (yref[1:] + yref[:-1])
    out = {}
    for k in ("U", "urms", "vrms", "wrms"):
        r = np.interp(yc, yr, ref[k])
        out[k] = float(np.linalg.norm(p[k] - r) / max(np.linalg.norm(r), 1e-30))
    return out
