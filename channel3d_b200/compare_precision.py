"""Mixed FP32/FP64 against FP64 on the same seeded channel run.

    python -m channel3d_b200.compare_precision --workload channel256x192x256_re13750 --steps 2000

Both runs start from the same divergence-free seeded field, accumulate the
clcStat_CH moments every --ivstats steps (FP64 reductions in both modes) and
report the relative L2 error (over y) of the mean profile U(y) and of the
u', v', w' rms profiles, the relative error of Re_tau (from the time-averaged
mean pressure gradient), the final max |div u| of each run, and the step times.
"""
import argparse
import json

import numpy as np

from . import ChannelSolver, initfield, workloads
from .stats import profiles


def run(cfg, state, steps, ivstats, stat_from):
    s = ChannelSolver(cfg)
    s.upload(*state)
    ms = 0.0
    info = None
    done = 0
    while done < steps:
        n = min(ivstats, steps - done)
        info = s.step(n)
        ms += s.last_step_ms()
        done += n
        if done >= stat_from and done % ivstats == 0:
            s.stats_accumulate()
    sumstat, nf, pg = s.stats_fetch()
    s.close()
    return profiles(sumstat, nf, pg, cfg.xnu), info, ms / steps


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def compare(workload="channel256x192x256_re13750", steps=0, ivstats=20, stat_from=0, device=0):
    """Runs the workload in FP64 and in mixed precision from the same projected
    seeded start and returns the comparison (a dict, see the module text)."""
    cfg64, nsteps = workloads.get(workload, precision="fp64")
    cfg64 = cfg64.copy(device=device)
    steps = steps or nsteps
    s = ChannelSolver(cfg64)
    s.upload(*initfield.laminar_noise(cfg64, yp=s.yp))
    s.project()
    st = s.download()
    s.close()
    state = (st["ux"], st["uy"], st["uz"], st["p"])
    p64, i64, ms64 = run(cfg64, state, steps, ivstats, stat_from)
    p32, i32, ms32 = run(cfg64.copy(precision="mixed"), state, steps, ivstats, stat_from)
    return {
        "workload": workload, "steps": steps, "ivstats": ivstats, "stat_from": stat_from,
        "rel_err_U": rel(p32["U"], p64["U"]), "rel_err_urms": rel(p32["urms"], p64["urms"]),
        "rel_err_vrms": rel(p32["vrms"], p64["vrms"]), "rel_err_wrms": rel(p32["wrms"], p64["wrms"]),
        "Re_tau_fp64": p64["Re_tau"], "Re_tau_mixed": p32["Re_tau"],
        "rel_err_Re_tau": abs(p32["Re_tau"] - p64["Re_tau"]) / max(abs(p64["Re_tau"]), 1e-300),
        "divmax_fp64": i64["divmax2"], "divmax_mixed": i32["divmax2"],
        "ms_per_step_fp64": ms64, "ms_per_step_mixed": ms32, "speedup": ms64 / ms32,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="channel256x192x256_re13750")
    ap.add_argument("--steps", type=int, default=0)
    ap.add_argument("--ivstats", type=int, default=20)
    ap.add_argument("--stat-from", type=int, default=0)
    a = ap.parse_args()
    out = compare(a.workload, a.steps, a.ivstats, a.stat_from)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
