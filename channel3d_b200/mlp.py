"""Host side of the learned subgrid-stress closure (include/ch3d_mlp.h).

The network, its tensor-core forward/backward kernels and the Adam update
live in libch3d.so (csrc/mlp_tc.cu); torch only holds the device buffers and
the stream.  There is no CPU path: a missing library raises.
"""
import numpy as np

from . import _lib

NIN, NOUT = 10, 6
NPARAM = 9414


def _ptr(t):
    return None if t is None else t.data_ptr()


class MLPClosure:
    """FP32 master parameters on the GPU with Adam state; BF16 tensor-core math."""

    def __init__(self, params=None, seed=0, device=0):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.lib = _lib.load_library()
        if params is None:
            from_oracle = _init_params(seed)
            params = from_oracle
        self.P = torch.as_tensor(np.asarray(params, dtype=np.float32), device=self.dev).contiguous()
        assert self.P.numel() == NPARAM
        self.m = torch.zeros_like(self.P)
        self.v = torch.zeros_like(self.P)
        self.g = torch.zeros_like(self.P)
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.step_count = 0
        self.work = None
        self.work_batch = 0

    def _stream(self):
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    def _check_status(self):
        if int(self.status.item()) != 0:
            raise RuntimeError("tensor-core MLP kernel timed out waiting for its MMAs (status %d)"
                               % int(self.status.item()))

    def forward(self, X):
        """Y [B x 6] for X [B x 10] (device float32)."""
        X = X.contiguous()
        B = X.shape[0]
        Y = self.torch.empty((B, NOUT), dtype=self.torch.float32, device=self.dev)
        rc = self.lib.ch3d_mlp_forward(_ptr(X), B, _ptr(self.P), _ptr(Y), _ptr(self.status), self._stream())
        if rc != 0:
            raise RuntimeError("ch3d_mlp_forward failed (%d)" % rc)
        return Y

    def grad(self, X, T):
        """Gradient of sum((Y-T)^2)/(6B) into self.g; returns the summed squared error (device tensor)."""
        X, T = X.contiguous(), T.contiguous()
        B = X.shape[0]
        if self.work is None or self.work_batch < B:
            nb = int(self.lib.ch3d_mlp_workspace_bytes(B))
            self.work = self.torch.empty(nb, dtype=self.torch.uint8, device=self.dev)
            self.work_batch = B
        rc = self.lib.ch3d_mlp_grad(_ptr(X), _ptr(T), B, _ptr(self.P), _ptr(self.work), _ptr(self.g),
                                    _ptr(self.loss), _ptr(self.status), self._stream())
        if rc != 0:
            raise RuntimeError("ch3d_mlp_grad failed (%d)" % rc)
        return self.loss

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        rc = self.lib.ch3d_mlp_adam(_ptr(self.P), _ptr(self.g), _ptr(self.m), _ptr(self.v), lr, beta1, beta2, eps,
                                    self.step_count, self._stream())
        if rc != 0:
            raise RuntimeError("ch3d_mlp_adam failed (%d)" % rc)

    def train(self, X, T, iters, batch=65536, lr=1e-3, seed=0, log_every=0):
        """Adam on random mini-batches of (X, T) (device tensors); returns the loss history."""
        torch = self.torch
        gen = torch.Generator(device=self.dev)
        gen.manual_seed(seed)
        n = X.shape[0]
        hist = []
        for it in range(iters):
            if batch < n:
                idx = torch.randint(0, n, (batch,), device=self.dev, generator=gen)
                xb, tb = X.index_select(0, idx), T.index_select(0, idx)
            else:
                xb, tb = X, T
            loss = self.grad(xb, tb)
            self.adam(lr)
            if log_every and (it % log_every == 0 or it == iters - 1):
                hist.append((it, float(loss.item()) / (xb.shape[0] * NOUT)))
        self._check_status()
        return hist

    def params(self):
        return self.P.detach().cpu().numpy().astype(np.float64)


def _init_params(seed):
    """He-style uniform initialisation, zero biases (same rule as the test oracle)."""
    rng = np.random.default_rng(seed)
    shapes = [(64, 10), (64,), (64, 64), (64,), (64, 64), (64,), (6, 64), (6,)]
    out = []
    for s in shapes:
        if len(s) == 2:
            lim = np.sqrt(6.0 / s[1])
            out.append(rng.uniform(-lim, lim, size=s).ravel())
        else:
            out.append(np.zeros(s))
    return np.concatenate(out).astype(np.float32)
