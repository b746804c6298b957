"""CPU restatement of the learned SGS closure's network (channel3d_b200/csrc/mlp_tc.cu).

TEST INFRASTRUCTURE ONLY: the checker of the tensor-core forward and
backward kernels.  A 10 -> 64 -> 64 -> 64 -> 6 MLP with the tanh form of
GELU (Hendrycks & Gimpel 2016);
every GEMM operand is rounded to BF16 (round to nearest even) where the
device rounds it, products are accumulated in FP64, biases, pre-activations
and the loss stay unrounded.  The model has no counterpart in the reference,
so this restatement is pinned by finite differences (tests/test_mlp_oracle.py).
"""
import numpy as np

NIN, NH, NOUT = 10, 64, 6
SHAPES = [("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NH, NH)), ("b3", (NH,)),
          ("W4", (NOUT, NH)), ("b4", (NOUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def f32(x):
    """Round to float32 (returned as float64): the device's FP32 values."""
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def unpack(P):
    out, o = {}, 0
    for name, s in SHAPES:
        n = int(np.prod(s))
        out[name] = np.asarray(P[o:o + n], dtype=np.float64).reshape(s)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SHAPES])


def init_params(seed=0):
    """He-style initialisation (uniform, fan-in scaled), zero biases."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, s in SHAPES:
        if name[0] == "W":
            lim = np.sqrt(6.0 / s[1])
            d[name] = rng.uniform(-lim, lim, size=s)
        else:
            d[name] = np.zeros(s)
    return pack(d).astype(np.float32)


C_GELU = np.sqrt(2.0 / np.pi)


def gelu(z):
    """0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))."""
    return 0.5 * z * (1.0 + np.tanh(C_GELU * (z + 0.044715 * z ** 3)))


def gelu_d(z):
    t = np.tanh(C_GELU * (z + 0.044715 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * C_GELU * (1.0 + 3.0 * 0.044715 * z * z)


def forward(P, X):
    """Y [B x 6] and the saved pre-activations / BF16 activations."""
    w = unpack(P)
    Wb = {k: bf16(v) for k, v in w.items() if k[0] == "W"}
    h = bf16(X)
    Z, H = [], [h]
    for l in (1, 2, 3):
        z = f32(h @ Wb["W%d" % l].T + f32(w["b%d" % l]))
        Z.append(z)
        h = bf16(gelu(z))
        H.append(h)
    Y = h @ Wb["W4"].T + f32(w["b4"])
    return Y, Z, H


def loss_and_grad(P, X, T):
    """Sum of squared errors and the gradient of sum((Y-T)^2)/(6B)."""
    B = X.shape[0]
    w = unpack(P)
    Wb = {k: bf16(v) for k, v in w.items() if k[0] == "W"}
    Y, Z, H = forward(P, X)
    E = Y - T
    loss = float(np.sum(E * E))
    d = f32(2.0 * E / (B * NOUT))
    g = {}
    for l in (4, 3, 2, 1):
        g["b%d" % l] = d.sum(axis=0)
        db = bf16(d)
        g["W%d" % l] = db.T @ H[l - 1]
        if l > 1:
            dh = db @ Wb["W%d" % l]
            d = dh * gelu_d(Z[l - 2])
    return loss, pack(g)
