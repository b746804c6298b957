"""Shared helpers of the parity tests."""
import numpy as np


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0)


def rel_max(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max()
    return np.abs(a - b).max() / (den if den > 0 else 1.0)


def small_channel(nx=32, ny=24, nz=16, **kw):
    from channel3d_b200 import workloads
    cfg, _ = workloads.get("channel64_re5600")
    return cfg.copy(nxc=nx, nyc=ny, nzc=nz, nycSection=[ny // 2, ny - ny // 2], **kw)
