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


def box_filtered_profiles(fields, cfg, box):
    """Mean and rms profiles of the box-filtered cell-centre velocities
    (the filtered-DNS reference of the LES), on the box-row centres."""
    fx, fy, fz = box
    from .config import mesh_y
    yp = mesh_y(cfg)
    dyp = np.diff(yp)
    ux, uy, uz = fields["ux"], fields["uy"], fields["uz"]
    uc = 0.5 * (ux + np.roll(ux, -1, axis=2))
    vn = np.concatenate([uy, np.zeros_like(uy[:, :1, :])], axis=1)
    vc = 0.5 * (vn[:, :-1, :] + vn[:, 1:, :])
    wc = 0.5 * (uz + np.roll(uz, -1, axis=0))
    w = np.broadcast_to(dyp[None, :, None], uc.shape)
    sh = (cfg.nzc // fz, fz, cfg.nyc // fy, fy, cfg.nxc // fx, fx)
    ws = w.reshape(sh).sum(axis=(1, 3, 5))
    out = {}
    for name, a in (("u", uc), ("v", vc), ("w", wc)):
        b = (a * w).reshape(sh).sum(axis=(1, 3, 5)) / ws       # box means
        m = b.mean(axis=(0, 2))
        out[name + "mean"] = m
        out[name + "rms"] = np.sqrt(((b - m[None, :, None]) ** 2).mean(axis=(0, 2)))
    yb = np.array([0.5 * (yp[j * fy] + yp[(j + 1) * fy]) for j in range(cfg.nyc // fy)])
    return {"y": yb, "U": out["umean"], "urms": out["urms"], "vrms": out["vrms"], "wrms": out["wrms"]}


def evaluate(dns_cfg, les_cfg, dns_warm, dns_steps, n_snapshots, per_snapshot, les_steps, les_avg_from,
             box=(4, 2, 4), train_iters=3000, batch=65536, lr=1e-3, n_profile_snapshots=10, seed=0, log=print,
             turbulent_start=0.0, warm_dt=None, les_start="seeded"):
    """The learned-closure experiment end to end on one GPU: DNS with
    box-filtered snapshots, training, and LES runs with the learned closure
    and with the Smagorinsky / van Driest model from the same start: the
    seeded start, or (les_start="dns") the last DNS field resampled onto the
    LES grid (ch3d_interp_state, the reference's interpolateField).
    Returns a report dict (profiles, errors against the filtered DNS,
    a-priori stress errors, LES cost per step)."""
    import time
    import torch
    from .config import mesh_y
    rep = {"box": list(box)}
    t0 = time.time()
    if turbulent_start > 0:
        # large-scale start, warm-up in the mixed path with a larger time step,
        # then the state continues in FP64 with the sampling time step
        wcfg = dns_cfg.copy(precision="mixed", dtMax=warm_dt or dns_cfg.dtMax)
        w = ChannelSolver(wcfg)
        w.upload(*initfield.large_scale(wcfg, amplitude=turbulent_start, yp=w.yp, seed=seed))
        w.project()
        for _ in range(max(1, dns_warm // 1000)):
            info = w.step(min(1000, dns_warm))
        st = w.download()
        log("dns warm-up (mixed, dt %g) %d steps: u' max %.3f, %.1f s"
            % (wcfg.dtMax, info["itime"], float(np.abs(st["uy"]).max()), time.time() - t0))
        w.close()
        s = ChannelSolver(dns_cfg)
        s.upload(st["ux"], st["uy"], st["uz"], st["p"])
        s.project()
    else:
        s = ChannelSolver(dns_cfg)
        s.upload(*initfield.laminar_noise(dns_cfg, yp=s.yp, seed=seed))
        s.project()
        s.step(dns_warm)
    log("dns warm-up %d steps: %.1f s" % (dns_warm, time.time() - t0))
    X, T, D, s = collect_samples(dns_cfg, dns_steps, n_snapshots, per_snapshot, box=box, seed=seed, solver=s)
    log("dns sampling %d snapshots: %d samples, %.1f s" % (n_snapshots, X.shape[0], time.time() - t0))
    # filtered-DNS reference profiles: a few more snapshots after the sampling window
    prof = []
    every = max(1, dns_steps // n_snapshots)
    for _ in range(n_profile_snapshots):
        s.step(every)
        prof.append(box_filtered_profiles(s.download(), dns_cfg, box))
    ref = {k: np.mean([p[k] for p in prof], axis=0) for k in prof[0]}
    dns_start = None
    if les_start == "dns":  # the DNS field on the LES grid
        r = ChannelSolver(les_cfg.copy(LES_type=10))
        r.interp_from(s)
        st = r.download()
        dns_start = (st["ux"], st["uy"], st["uz"], st["p"])
        r.close()
    s.close()
    # train / hold-out split by snapshot
    nho = max(1, n_snapshots // 10) * per_snapshot
    Xtr, Ttr, Xte, Tte, Dte = X[:-nho], T[:-nho], X[-nho:], T[-nho:], D[-nho:]
    norm = fit_norm(Xtr, Ttr)
    net, hist = train(Xtr, Ttr, norm, iters=train_iters, batch=batch, lr=lr, seed=seed, log_every=max(1, train_iters // 20))
    rep["train_loss"] = hist
    rep["a_priori"] = {"mlp": stress_error(predict(net, Xte, norm), Tte),
                       "smagorinsky_vd": stress_error(smagorinsky(Xte, Dte, les_cfg.Cs), Tte)}
    log("a priori stress errors: %s (%.1f s)" % (rep["a_priori"], time.time() - t0))
    params = net.params().astype(np.float32)
    del X, T, D, Xtr, Ttr
    torch.cuda.empty_cache()
    # LES runs from the same seeded start
    yl = mesh_y(les_cfg)
    rep["les"] = {}
    for name, lt in (("mlp", 11), ("smagorinsky_vd", 10)):
        cfg = les_cfg.copy(LES_type=lt)
        ls = ChannelSolver(cfg)
        if dns_start is not None:
            start = dns_start
        elif turbulent_start > 0:
            start = initfield.large_scale(cfg, amplitude=turbulent_start, yp=ls.yp, seed=seed)
        else:
            start = initfield.laminar_noise(cfg, yp=ls.yp, seed=seed)
        ls.upload(*start)
        ls.project()
        if lt == 11:
            ls.sgs_mlp_set(params, norm)
        info = ls.step(les_avg_from, raise_on_diverge=False)
        acc, n, ms = None, 0, 0.0
        while info["status"] == 0 and info["itime"] < les_steps:
            info = ls.step(min(100, les_steps - info["itime"]), raise_on_diverge=False)
            ms += ls.last_step_ms()
            p = profiles(ls.download(), cfg)
            acc = p if acc is None else {k: acc[k] + p[k] for k in acc}
            n += 1
        r = {"status": info["status"], "steps": info["itime"], "ms_per_step": ms / max(1, info["itime"] - les_avg_from)}
        if acc is not None:
            pm = {k: v / n for k, v in acc.items()}
            yc = 0.5 * (yl[1:] + yl[:-1])
            errs = {}
            for k in ("U", "urms", "vrms", "wrms"):
                rr = np.interp(yc, ref["y"], ref[k])
                errs[k] = float(np.linalg.norm(pm[k] - rr) / max(np.linalg.norm(rr), 1e-30))
            r["profile_errors"] = errs
            r["profiles"] = {k: v.tolist() for k, v in pm.items()}
        rep["les"][name] = r
        ls.close()
        log("les %s: %s (%.1f s)" % (name, {k: v for k, v in r.items() if k != "profiles"}, time.time() - t0))
    rep["reference_profiles"] = {k: v.tolist() for k, v in ref.items()}
    return rep


def main():
    import argparse
    import json
    from . import workloads
    ap = argparse.ArgumentParser(description="learned SGS closure: DNS sampling, training, LES comparison")
    ap.add_argument("--out", default="les_closure_report.json")
    ap.add_argument("--dns-warm", type=int, default=16000)
    ap.add_argument("--dns-steps", type=int, default=4000)
    ap.add_argument("--snapshots", type=int, default=400)
    ap.add_argument("--per-snapshot", type=int, default=16384)
    ap.add_argument("--les-steps", type=int, default=20000)
    ap.add_argument("--les-avg-from", type=int, default=4000)
    ap.add_argument("--train-iters", type=int, default=3000)
    ap.add_argument("--turbulent-start", type=float, default=0.0,
                    help="amplitude of a large-scale start (0: the seeded white-noise start)")
    ap.add_argument("--warm-dt", type=float, default=None, help="time step of the mixed-precision warm-up")
    ap.add_argument("--dns-grid", default="256x192x256",
                    help="DNS cells nx x ny x nz of the 2pi x 2 x pi Re_b 13750 channel; 192x192x192 with --box 4,4,4 "
                         "gives filter boxes that are exactly the cells of the 48^3 LES grid")
    ap.add_argument("--box", default="4,2,4", help="filter box fx,fy,fz in DNS cells")
    ap.add_argument("--les-start", default="seeded", choices=["seeded", "dns"],
                    help="start of the LES runs: the seeded field, or the last DNS field resampled onto the LES grid")
    args = ap.parse_args()
    nx, ny, nz = (int(v) for v in args.dns_grid.lower().split("x"))
    dns, _ = workloads.get("channel256x192x256_re13750")
    dns = dns.copy(nxc=nx, nyc=ny, nzc=nz, nycSection=[ny // 2, ny - ny // 2])
    les, _ = workloads.get("channel48_les", LES_type=10, Cs=0.1)
    box = tuple(int(v) for v in args.box.split(","))
    rep = evaluate(dns, les, args.dns_warm, args.dns_steps, args.snapshots, args.per_snapshot, args.les_steps,
                   args.les_avg_from, box=box, train_iters=args.train_iters, turbulent_start=args.turbulent_start,
                   warm_dt=args.warm_dt, les_start=args.les_start)
    rep["dns_grid"] = [nx, ny, nz]
    rep["les_start"] = args.les_start
    json.dump(rep, open(args.out, "w"))


if __name__ == "__main__":
    main()
