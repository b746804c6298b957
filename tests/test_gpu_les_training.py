"""The learned closure trained on the device end to end: DNS snapshots of
the channel are box filtered into (filtered gradients, y+) -> SGS stress
samples, the network is trained with the tensor-core gradient and Adam, and
on held-out snapshots it predicts the stresses better than the Smagorinsky /
van Driest model that it replaces (an a-priori test: relative L2 error of
tau_ij over all components)."""
import numpy as np
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


def test_short_a_posteriori_run(built):
    """The whole closure experiment at reduced size: a 96^3 DNS of the 2pi x 2 x
    pi Re_b 13750 channel (warmed from a large-scale start), 2 x 2 x 2 box
    filter (the cells of the 48^3 LES grid, whose tanh mesh the DNS mesh
    nests), training, and 48^3 LES runs with the learned closure and with the
    Smagorinsky / van Driest model from the DNS field resampled onto the LES
    grid, both compared with the box-filtered DNS profiles.  Asserted: the
    network beats Smagorinsky a priori on held-out snapshots, both LES runs
    stay finite and keep the mean profile within 10% of the filtered DNS, and
    the learned closure's cost per step is reported."""
    from channel3d_b200 import les_closure as LC, workloads
    dns, _ = workloads.get("channel256x192x256_re13750")
    dns = dns.copy(nxc=96, nyc=96, nzc=96, nycSection=[48, 48])
    les, _ = workloads.get("channel48_les", LES_type=10, Cs=0.1)
    rep = LC.evaluate(dns, les, dns_warm=6000, dns_steps=800, n_snapshots=40, per_snapshot=8192, les_steps=3000,
                      les_avg_from=1000, box=(2, 2, 2), train_iters=600, turbulent_start=0.3, warm_dt=0.002,
                      les_start="dns", log=lambda *a: None)
    assert rep["a_priori"]["mlp"] < rep["a_priori"]["smagorinsky_vd"], rep["a_priori"]
    for name in ("mlp", "smagorinsky_vd"):
        r = rep["les"][name]
        assert r["status"] == 0 and r["steps"] == 3000, (name, r)
        assert r["profile_errors"]["U"] < 0.1, (name, r["profile_errors"])
        assert all(np.isfinite(v) for v in r["profile_errors"].values())
    assert rep["les"]["mlp"]["ms_per_step"] > 0
