"""B200 implementation of Channel3d's RK3 channel-flow time step.

The compute path is libch3d.so (hand-written sm_100a CUDA behind the C ABI
of include/ch3d.h); this package is the host-side mirror of the reference's
start-up and time-loop call sites.
"""
from .config import ChannelConfig, mesh_y, parse_namelists  # noqa: F401
from .solver import ChannelSolver  # noqa: F401
from . import workloads  # noqa: F401
from ._lib import load_library, Ch3dError  # noqa: F401
