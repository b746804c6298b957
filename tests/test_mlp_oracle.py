"""Pins the CPU restatement of the learned closure's network: its backward
pass against central finite differences of its own forward pass (without the
BF16 and FP32 rounding, which finite differences cannot follow)."""
import numpy as np


def test_mlp_oracle_gradient_matches_finite_differences():
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(3)
    P = M.init_params(1).astype(np.float64)
    P[M.NPARAM - 6:] = rng.standard_normal(6) * 0.1          # non-zero output bias
    X = rng.standard_normal((40, M.NIN))
    T = rng.standard_normal((40, M.NOUT))
    ident = lambda x: np.asarray(x, dtype=np.float64)
    saved = (M.bf16, M.f32)
    M.bf16 = ident
    M.f32 = ident
    try:
        f = lambda p: M.loss_and_grad(p, X, T)[0] / (X.shape[0] * M.NOUT)
        _, g = M.loss_and_grad(P, X, T)
        idx = rng.choice(M.NPARAM, 60, replace=False)
        for q in idx:
            h = 1e-6
            Pp, Pm = P.copy(), P.copy()
            Pp[q] += h
            Pm[q] -= h
            fd = (f(Pp) - f(Pm)) / (2 * h)
            assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (q, fd, g[q])
    finally:
        M.bf16, M.f32 = saved


def test_bf16_rounding_is_nearest_even():
    from oracle import mlp_oracle as M
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.14159265], dtype=np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == 1.0 and r[4] == -2.5
    assert abs(r[5] - 3.140625) < 1e-12
