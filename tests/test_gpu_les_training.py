"""The learned closure trained on the device end to end: DNS snapshots of
the channel are box filtered into (filtered gradients, y+) -> SGS stress
samples, the network is trained with the tensor-core gradient and Adam, and
on held-out snapshots it predicts the stresses better than the Smagorinsky /
van Driest model that it replaces (an a-priori test: relative L2 error of
tau_ij over all components)."""
import pytest

pytestmark = pytest.mark.gpu


def test_trained_network_beats_smagorinsky_a_priori(built):
    from channel3d_b200 import les_closure as LC, workloads
    cfg, _ = workloads.get("channel48_les")
    cfg = cfg.copy(nxc=64, nyc=48, nzc=64, nycSection=[24, 24], dtMax=0.002)
    X, T, D, s = LC.collect_samples(cfg, steps=600, n_snapshots=24, per_snapshot=4096, box=(4, 2, 4), seed=1)
    ntr = 20 * 4096
    norm = LC.fit_norm(X[:ntr], T[:ntr])
    net, hist = LC.train(X[:ntr], T[:ntr], norm, iters=600, batch=16384, lr=2e-3, seed=2, log_every=100)
    assert hist[-1][1] < hist[0][1]
    e_mlp = LC.stress_error(LC.predict(net, X[ntr:], norm), T[ntr:])
    e_smag = LC.stress_error(LC.smagorinsky(X[ntr:], D[ntr:]), T[ntr:])
    assert e_mlp < e_smag, (e_mlp, e_smag)
    assert e_mlp < 0.9, e_mlp
