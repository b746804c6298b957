"""The learned closure's tensor-core kernels (tcgen05, BF16 operands, FP32
accumulation) against the CPU oracle (oracle/mlp_oracle.py, which rounds the
same operands to BF16 and accumulates in FP64).

Tolerances: forward outputs and the gradient within 1e-3 relative (L2): the
residual differences come from FP32 accumulation order and from the rare
activation whose FP32 value falls on the other side of a BF16 rounding
boundary; the summed squared error within 1e-5 relative."""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu


def _data(B, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((B, 10)).astype(np.float32)
    T = (0.5 * rng.standard_normal((B, 6))).astype(np.float32)
    return X, T


def test_mlp_forward_matches_oracle(built):
    import torch
    from channel3d_b200.mlp import MLPClosure
    from oracle import mlp_oracle as M
    P = M.init_params(7)
    P[M.NPARAM - 6:] = 0.1
    net = MLPClosure(params=P)
    for B in (128, 1000, 4096):
        X, _ = _data(B, B)
        Y = net.forward(torch.as_tensor(X, device="cuda")).cpu().numpy()
        Yo, _, _ = M.forward(P.astype(np.float64), X.astype(np.float64))
        assert rel_l2(Y, Yo) < 1e-3, (B, rel_l2(Y, Yo))
    net._check_status()


def test_mlp_gradient_matches_oracle(built):
    import torch
    from channel3d_b200.mlp import MLPClosure
    from oracle import mlp_oracle as M
    P = M.init_params(11)
    X, T = _data(3000, 5)
    net = MLPClosure(params=P)
    loss = float(net.grad(torch.as_tensor(X, device="cuda"), torch.as_tensor(T, device="cuda")).item())
    g = net.g.cpu().numpy().astype(np.float64)
    lo, go = M.loss_and_grad(P.astype(np.float64), X.astype(np.float64), T.astype(np.float64))
    net._check_status()
    assert abs(loss - lo) <= 1e-5 * lo
    o = 0
    for name, s in M.SHAPES:
        n = int(np.prod(s))
        assert rel_l2(g[o:o + n], go[o:o + n]) < 1e-3, (name, rel_l2(g[o:o + n], go[o:o + n]))
        o += n


def test_mlp_training_fits_a_teacher(built):
    """Adam with the tensor-core gradient fits a random teacher network."""
    import torch
    from channel3d_b200.mlp import MLPClosure
    from oracle import mlp_oracle as M
    teacher = M.init_params(21)
    X, _ = _data(65536, 9)
    T, _, _ = M.forward(teacher.astype(np.float64), X.astype(np.float64))
    Xd = torch.as_tensor(X, device="cuda")
    Td = torch.as_tensor(T.astype(np.float32), device="cuda")
    net = MLPClosure(seed=3)
    hist = net.train(Xd, Td, iters=300, batch=8192, lr=2e-3, log_every=50)
    assert hist[-1][1] < 0.1 * hist[0][1], hist
