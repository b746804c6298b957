"""The learned closure inside the LES step (LES_type = CH3D_LES_MLP): the
network inputs and the Smagorinsky fallback stress against a numpy
restatement, the tensor-core network's stresses against the CPU network
oracle, the stress divergence and the whole LES step against the CPU oracle
given the same stresses, and the box-filtered training samples against a
numpy box filter.  Tolerances: FP64 quantities 1e-12 (max norm), network
outputs 1e-3 (L2, BF16 operands), one step 1e-11, FP32 samples 1e-5."""
import numpy as np
import pytest

from helpers import rel_l2, rel_max

pytestmark = pytest.mark.gpu


def _cfg(nx=32, ny=24, nz=16, les=11):
    from channel3d_b200 import workloads
    cfg, _ = workloads.get("channel48_les")
    return cfg.copy(nxc=nx, nyc=ny, nzc=nz, nycSection=[ny // 2, ny - ny // 2], LES_type=les, Cs=0.1)


def _pair(cfg, seed=0x5EED):
    from channel3d_b200 import ChannelSolver, initfield, mesh_y
    from oracle import oracle as O
    yp = mesh_y(cfg)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp, seed=seed)
    o = O.Oracle(cfg)
    o.set_state(ux, uy, uz, p)
    s = ChannelSolver(cfg, yp=yp)
    s.upload(ux, uy, uz, p)
    return o, s, yp, ux


def _norm(lo, hi, in_mean=None, in_std=None):
    n = np.zeros(52, dtype=np.float32)
    n[0:10] = 0.0 if in_mean is None else in_mean
    n[10:20] = 1.0 if in_std is None else in_std
    n[20:30] = lo
    n[30:40] = hi
    n[40:46] = 0.0
    n[46:52] = 1.0
    return n


def _tau(s):
    return np.stack([s.get_array(15 + q) for q in range(6)])


def test_fallback_stress_matches_numpy(built):
    import sgs_numpy as SN
    from oracle import mlp_oracle as M
    cfg = _cfg()
    o, s, yp, ux = _pair(cfg)
    s.sgs_mlp_set(M.init_params(1), _norm(1e30, -1e30))   # every input out of range
    s.sgs_viscosity()
    ref = SN.smag_tau(SN.gradients(o, cfg, yp), cfg, yp, SN.utau(ux, cfg, yp))
    assert rel_max(_tau(s), ref) < 1e-12, rel_max(_tau(s), ref)


def test_network_stress_matches_oracle(built):
    import sgs_numpy as SN
    from oracle import mlp_oracle as M
    cfg = _cfg()
    o, s, yp, ux = _pair(cfg)
    P = M.init_params(5) * 0.5
    ut = SN.utau(ux, cfg, yp)
    X = SN.features(SN.gradients(o, cfg, yp), cfg, yp, ut)
    mean, std = X.mean(axis=0), X.std(axis=0) + 1e-3
    s.sgs_mlp_set(P, _norm(-1e30, 1e30, mean, std))         # every input in range
    s.sgs_viscosity()
    Xs = ((X - mean.astype(np.float32)) / std.astype(np.float32)).astype(np.float32)
    Y, _, _ = M.forward(P.astype(np.float64), Xs.astype(np.float64))
    ref = (Y * ut ** 2).T.reshape((6,) + cfg.shape)
    assert rel_l2(_tau(s), ref) < 1e-3, rel_l2(_tau(s), ref)


def test_les_step_with_stress_matches_oracle(built):
    from oracle import mlp_oracle as M
    cfg = _cfg()
    o, s, yp, ux = _pair(cfg)
    s.sgs_mlp_set(M.init_params(1), _norm(1e30, -1e30))
    s.sgs_viscosity()
    tau = _tau(s)
    o.sgs()
    o.set_sgs_tau(tau)
    for ns in (1, 2, 3):
        for st in range(7):
            o.stage(st, ns)
            s.stage(st, ns)
    go, gs = o.get_state(), s.download()
    for k in ("ux", "uy", "uz", "p"):
        assert rel_max(gs[k], go[k]) < 1e-11, (k, rel_max(gs[k], go[k]))


def test_learned_closure_steps(built):
    """Whole graph-captured steps with the network in the loop stay finite and divergence-free."""
    import sgs_numpy as SN
    from oracle import mlp_oracle as M
    cfg = _cfg()
    o, s, yp, ux = _pair(cfg)
    X = SN.features(SN.gradients(o, cfg, yp), cfg, yp, SN.utau(ux, cfg, yp))
    s.sgs_mlp_set(M.init_params(3) * 0.01, _norm(-8, 8, X.mean(axis=0), X.std(axis=0) + 1e-3))
    info = s.step(20)
    assert info["status"] == 0 and info["divmax2"] < 1e-12


def test_training_samples_match_numpy_box_filter(built):
    import sgs_numpy as SN
    cfg = _cfg(les=0)
    o, s, yp, ux = _pair(cfg)
    X, T = s.sgs_training_samples(4, 2, 4)
    X, T = X.cpu().numpy(), T.cpu().numpy()
    g = SN.gradients(o, cfg, yp)
    U, V, W = SN.fields(o, cfg)
    uc = [0.5 * (U(0, 0, 0) + U(1, 0, 0)), 0.5 * (V(0, 0, 0) + V(0, 1, 0)), 0.5 * (W(0, 0, 0) + W(0, 0, 1))]
    dyp, yc, _ = SN.mesh(cfg, yp)
    ut = SN.utau(ux, cfg, yp)
    w = np.broadcast_to(dyp[None, :, None], cfg.shape)

    def box(a):  # (nz, ny, nx) -> (nz/4, ny/2, nx/4) volume-weighted means
        sh = (cfg.nzc // 4, 4, cfg.nyc // 2, 2, cfg.nxc // 4, 4)
        return (a * w).reshape(sh).sum(axis=(1, 3, 5)) / w.reshape(sh).sum(axis=(1, 3, 5))
    mu = [box(u) for u in uc]
    pairs = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    Tref = np.stack([(box(uc[a] * uc[b]) - mu[a] * mu[b]).ravel() for a, b in pairs], axis=1) / ut ** 2
    yb = box(np.broadcast_to(yc[None, :, None], cfg.shape))
    dw = np.minimum(yb - yp[0], yp[-1] - yb)
    Xref = np.concatenate([np.stack([box(g[q]).ravel() for q in range(9)], axis=1) * cfg.xnu / ut ** 2,
                           (dw * ut / cfg.xnu).reshape(-1, 1)], axis=1)
    assert rel_max(X, Xref) < 1e-5, rel_max(X, Xref)
    assert rel_max(T, Tref) < 1e-4, rel_max(T, Tref)


def test_learned_closure_mixed_precision(built):
    """The learned closure in the mixed path: its stresses from the FP32 fields
    within 1e-3 (L2) of those of the FP64 path on the same state, and 20 steps
    stay finite and divergence-free to FP32 round-off."""
    import sgs_numpy as SN
    from channel3d_b200 import ChannelSolver
    from oracle import mlp_oracle as M
    cfg = _cfg()
    o, s, yp, ux = _pair(cfg)
    X = SN.features(SN.gradients(o, cfg, yp), cfg, yp, SN.utau(ux, cfg, yp))
    P, norm = M.init_params(3) * 0.5, _norm(-8, 8, X.mean(axis=0), X.std(axis=0) + 1e-3)
    s.sgs_mlp_set(P, norm)
    s.sgs_viscosity()
    t64 = _tau(s)
    st = s.download()
    m = ChannelSolver(cfg.copy(precision="mixed"), yp=yp)
    m.upload(st["ux"], st["uy"], st["uz"], st["p"])
    m.sgs_mlp_set(P, norm)
    m.sgs_viscosity()
    assert rel_l2(_tau(m), t64) < 1e-3, rel_l2(_tau(m), t64)
    info = m.step(20)
    assert info["status"] == 0 and info["divmax2"] < 1e-4
    m.close()
