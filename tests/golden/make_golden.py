"""Generates the golden fixtures of tests/golden/ with the CPU oracle.

    python tests/golden/make_golden.py

Case: 2nd-order partially implicit channel, 16 x 12 x 8 cells, 2pi x 2 x pi,
tanh-stretched y (2 sections, stretch 2.0), Re_b 5600, dt 0.002, RK3, seeded
laminar + 10% noise start (channel3d_b200.initfield with the default seed).
Stored: the initial state and the state after 1 and after 5 steps, with the
step diagnostics.  The fixtures pin the oracle against regressions and give
the GPU path a fixed target.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from channel3d_b200 import initfield, workloads  # noqa: E402
from oracle import oracle as O  # noqa: E402


def case():
    cfg, _ = workloads.get("channel64_re5600")
    return cfg.copy(nxc=16, nyc=12, nzc=8, nycSection=[6, 6])


def main():
    cfg = case()
    o = O.Oracle(cfg)
    yp = o.mesh()[0]
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp)
    o.set_state(ux, uy, uz, p)
    out = {"yp": yp, "ux0": ux, "uy0": uy, "uz0": uz, "p0": p}
    infos = {}
    done = 0
    for n in (1, 5):
        d = o.step(n - done)
        done = n
        st = o.get_state(hist=True)
        for k in ("ux", "uy", "uz", "p"):
            out["%s%d" % (k, n)] = st[k]
        out["hist%d" % n] = st["hist"]
        infos[str(n)] = d
    np.savez_compressed(os.path.join(HERE, "channel16x12x8.npz"), **out)
    with open(os.path.join(HERE, "channel16x12x8.json"), "w") as f:
        json.dump({"case": "16x12x8 channel, Re_b 5600, dt 0.002, RK3 PIMP", "info": infos}, f, indent=1)


if __name__ == "__main__":
    main()
