"""Throughput benchmark of the B200 channel-flow RK3 step.

Default workload: the 2nd-order, partially implicit (y Crank-Nicolson) FP64
channel at 768 x 384 x 576 cells (~170M), Re_b 21900, dt 3e-4: the large
throughput configuration.  Metric: grid-point-steps per second (Gpt-steps/s
= cells * steps / s / 1e9), whole job over all ranks.

One process per GPU (torchrun for N > 1).  The path has no data-path
exchange on one GPU per field, so N GPUs run N independent replicas ("replicas
only", weak scaling); the only collectives are the timing barrier and the
max-over-ranks reduction.

An FP64 run also times the same workload in mixed precision in the same
process and reports it in the line's "mixed" object (the metric compares the
two precisions), with its own clocks and the speed-up at equal clock.

--impl reference times the reference algorithm's CPU implementation (the C++
restatement in oracle/, all host threads) on a z-slab of the workload (the
same slab as the CPU-baseline leg of the GPU line, --cpu-nz planes) and prints
the same JSON line with "impl": "reference" and the slab's own time per step.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic HBM traffic: full-field arrays that must cross HBM once per
# substep (reads + writes) under the minimal-fusion plan of the data
# dependencies, x 3 substeps x word size.  2nd-order partially implicit and
# 4th order: 32 arrays per substep; fully implicit (ADI): 47.
ALG_ARRAYS_PER_SUBSTEP = {"pimp": 32, "order4": 32, "fimp": 47, "les": 32}
# per-launch algorithmic arrays of each kernel group of ch3d_kernel_times
# (0: RHS + y Helmholtz solve, fused: read u v w p Hist x3, write Hist x3 u* x3;
#  2: divergence + forward x FFT: read u* x3, write the half spectrum;
#  3: z FFT, y Poisson solve, inverse z FFT: 3 x (read + write) of the spectrum;
#  4: inverse x FFT: read spectrum, write phi;
#  5: projection + pressure update: read phi u* x3 p, write u x3 p)
GROUP_ARRAYS = {0: 13, 2: 4, 3: 6, 4: 2, 5: 9}
GROUP_NAMES = {0: "rhs", 1: "y_solves", 2: "k_prsrc_xfft", 3: "k_zfft+k_ysolve2+k_zfft", 4: "k_xifft",
               5: "k_proj", 6: "scalar_kernels_per_step"}
# the group-0 kernel of each scheme (RHS, fused with the y solves for pimp and order4)
GROUP0_KERNEL = {"pimp": "k_rhs_march", "order4": "k_rhs_march", "fimp": "k_rhs_fimp", "les": "k_rhs_les"}
# CUDA kernels launched per step by the step graph (ch3d_api.cu record_step):
# step_begin 1 + per substep (reduce_partials + substep_setup 2, march table (pimp) or
# helm_factors 1, rhs+uhat 1, prsrc_xfft 1, zfft + ysolve2 + zfft 3 (the mixed path's FP64
# low modes inside the same y-solve kernel), xifft 1, proj 1) + diag_reset + diag 2
# (the diag kernel only where the last projection does not carry the diagnostics)
# + reduce_partials + step_end 2
LAUNCHES_PER_SUBSTEP = {"fp64": 10, "mixed": 10}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="channel768x384x576_re21900")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-threads", type=int, default=0)
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision timing of an FP64 run")
    ap.add_argument("--les-type", type=int, default=0,
                    help="LES closure of an LES workload: 2 WALE, 3 MTS, 10 Smagorinsky / van Driest, 11 the learned "
                         "closure (the network's seeded initial weights, inputs never out of range)")
    ap.add_argument("--cpu-nz", type=int, default=48,
                    help="z planes of the CPU sample (the CPU-baseline leg and --impl reference)")
    ap.add_argument("--cpu-steps", type=int, default=3, help="timed steps of the CPU-baseline leg")
    return ap.parse_args()


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) >= 9:
                for n, v in zip(names, r[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl"
        try:
            import torch
            if not torch.cuda.is_available():
                backend = "gloo"
            else:
                torch.cuda.set_device(local)
        except Exception:
            backend = "gloo"
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(ws, v):
    if ws <= 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_sample_cfg(cfg, nz_sample):
    """A bounded sample of a workload for the CPU timing: the same x-y grid,
    metrics and parameters on a z-slab of nz_sample planes (the step's cost
    per grid point does not depend on nz beyond the z FFT's log factor)."""
    if nz_sample >= cfg.nzc:
        return cfg
    return cfg.copy(nzc=nz_sample, zlz=cfg.zlz * nz_sample / cfg.nzc)


def cpu_reference(cfg, args, steps=3, warmup=1):
    """Times the CPU restatement (oracle/, OpenMP over all host threads) on
    `steps` RK3 steps of cfg after `warmup` untimed ones (page-in,
    first-touch).  Returns (Gpt-steps/s, threads, seconds, steps)."""
    from oracle import oracle as O
    from channel3d_b200 import initfield
    if args.cpu_threads:
        O.set_threads(args.cpu_threads)
    threads = O.num_threads()
    o = O.Oracle(cfg)
    yp = o.mesh()[0]
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=yp)
    o.set_state(ux, uy, uz, p)
    del ux, uy, uz, p
    o.step(max(1, warmup))
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    o.close()
    return cfg.npoints * steps / dt / 1e9, threads, dt, steps


def solver_name(cfg):
    if cfg.LES_type:
        return "2nd-order PIMP RK3 LES (LES_type %d)" % cfg.LES_type
    if cfg.order == 4:
        return "4th-order RK3 (y Crank-Nicolson)"
    return "2nd-order %s RK3" % ("FIMP (ADI)" if cfg.IsImplicit == 2 else "PIMP")


def scheme_key(cfg):
    if cfg.LES_type:
        return "les"
    if cfg.order == 4:
        return "order4"
    return "fimp" if cfg.IsImplicit == 2 else "pimp"


def run_reference(args, ws, rank):
    """The reference's algorithm on the host cores: the C++ restatement of the
    step (oracle/, OpenMP over all host threads), each timed step one RK3 step
    of the same z-slab sample of the workload the CPU-baseline leg of the GPU
    line uses; ms_per_step is the slab's own time per step."""
    from channel3d_b200 import workloads
    cfg, _ = workloads.get(args.workload, precision="fp64")
    if rank != 0:
        return
    sample = cpu_sample_cfg(cfg, args.cpu_nz)
    v, thr, dt, nst = cpu_reference(sample, args, steps=args.steps, warmup=args.warmup)
    slab = "%s (%dx%dx%d z-slab)" % (args.workload, sample.nxc, sample.nyc, sample.nzc)
    line = {
        "impl": "reference", "metric": "Gpt-steps/s", "value": v, "unit": "Gpt-steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / nst * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded laminar + 10% uniform noise)",
        "config": {"workload": slab, "grid": [sample.nxc, sample.nyc, sample.nzc], "solver": solver_name(cfg),
                   "precision": "fp64", "full_grid": [cfg.nxc, cfg.nyc, cfg.nzc]},
        "cpu_baseline": {"value": v, "unit": "Gpt-steps/s", "cores": thr, "kind": "port",
                         "sample": "%d RK3 steps (after %d untimed) of a %dx%dx%d z-slab of the %s workload "
                                   "(%.1f s); C++ restatement of the reference step (oracle/), OpenMP, %d threads"
                                   % (nst, max(1, args.warmup), sample.nxc, sample.nyc, sample.nzc,
                                      args.workload, dt, thr)},
        "e2e": {"value": v, "unit": "Gpt-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def profile_traffic(kernel, precision):
    """DRAM bytes per grid point per launch of `kernel`, from the committed ncu
    summaries (a line 'bench-traffic: <kernel> <precision> <bytes per point>')."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None, None
    for fn in sorted(os.listdir(d)):
        if not fn.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(d, fn)):
            t = line.strip().split()
            if len(t) == 4 and t[0] == "bench-traffic:" and t[1] == kernel and t[2] == precision:
                return float(t[3]), fn
    return None, None


def launches_per_step(cfg, key, precision, gsub):
    """Kernel launches of one graph-replayed step (ch3d_api.cu record_step)."""
    launches = 1 + 3 * LAUNCHES_PER_SUBSTEP[precision] + 4
    if key == "pimp" and cfg.nxc % 32 == 0 and cfg.nzc % 4 == 0:
        launches -= 1  # the last projection carries the step diagnostics (no diag kernel)
    if gsub:
        launches += 3  # divergence march + x FFT in place of the fused divergence/x FFT kernel
    if key == "order4":
        launches += 3 * 2        # mean viscous stress partials, interpolated velocities
    elif key == "fimp":
        launches += 3 * 4        # RHS and y solve unfused, x/z periodic sweeps + their factors
    elif key == "les":
        launches += 3 * 1 + 1 + (1 if cfg.LES_type == 10 else 0)  # RHS/y solve unfused, eddy viscosity (+ wall shear)
    return launches


def measure(args, ws, rank, local, precision, want_e2e):
    """One precision of the workload: device-timed steps (CUDA events on the
    context's stream, max over ranks), kernel-group times, the roofline of the
    dominant group and, optionally, the end-to-end time through the C ABI."""
    import torch
    from channel3d_b200 import ChannelSolver, initfield, workloads
    cfg, _ = workloads.get(args.workload, precision=precision)
    cfg = cfg.copy(device=local)
    if args.les_type:
        cfg = cfg.copy(LES_type=args.les_type, Cs=0.1)
    torch.cuda.set_device(local)
    s = ChannelSolver(cfg)
    if args.les_type == 11:  # the learned closure: seeded weights, a standardisation that accepts every input
        from channel3d_b200.mlp import MLPClosure
        norm = np.zeros(52, dtype=np.float32)
        norm[10:20], norm[20:30], norm[30:40], norm[46:52] = 1.0, -1e30, 1e30, 1.0
        s.sgs_mlp_set(MLPClosure(seed=0, device=local).params(), norm)
    ux, uy, uz, p = initfield.laminar_noise(cfg, yp=s.yp)
    s.upload(ux, uy, uz, p)
    s.project()
    s.step(max(args.warmup, 3))

    clk = ClockSampler(local)
    barrier(ws)
    torch.cuda.synchronize()
    clk.start()
    t0 = time.perf_counter()
    info = s.step(args.steps)
    ms_dev = s.last_step_ms()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    barrier(ws)
    clocks = clk.stop()
    ms_max = allmax(ws, ms_dev)
    ms_per_step = ms_max / args.steps
    value = ws * cfg.npoints * args.steps / (ms_max * 1e-3) / 1e9

    # per-kernel-group device times: CUDA events around each group on the
    # context's stream over two more (ungraphed) steps; groups 0-5 per substep
    # launch, the scalar kernels per step
    kt = s.kernel_times(2)
    word = 4 if precision == "mixed" else 8
    key = scheme_key(cfg)
    names = dict(GROUP_NAMES)
    names[0] = GROUP0_KERNEL[key]
    if key == "pimp":
        names[5] = "k_proj_march"
    path = sorted(s.path_flags())
    gsub = "gsub" in path
    if gsub:  # the march stops at g; the divergence and projection marches substitute u*
        names[2] = "k_div_bsub+k_prsrc_xfft"
        names[5] = "k_proj_bsub"
    per_group = {}
    for g, arrs in GROUP_ARRAYS.items():
        b = arrs * cfg.npoints * word
        per_group[names[g]] = {"ms": kt[g], "alg_bytes": b, "GBps": b / (kt[g] * 1e-3) / 1e9 if kt[g] > 0 else None}
    if kt[1] > 0:
        per_group[names[1]] = {"ms": kt[1]}
    per_group[names[6]] = {"ms": kt[6]}
    dom = max(GROUP_ARRAYS, key=lambda g: kt[g])
    peak, peak_kind = load_peaks()
    dom_b = GROUP_ARRAYS[dom] * cfg.npoints * word
    achieved = dom_b / (kt[dom] * 1e-3) / 1e9
    # the march that stops at g moves less than the one that substitutes: its own profile line
    tpp, tsrc = profile_traffic(names[dom] + ("/g" if gsub and dom == 0 else ""), precision)
    traffic = tpp * cfg.npoints if tpp is not None else None
    step_alg = ALG_ARRAYS_PER_SUBSTEP[key] * 3 * word * cfg.npoints
    step_achieved = step_alg / (ms_per_step * 1e-3) / 1e9
    launches = launches_per_step(cfg, key, precision, gsub)

    # end-to-end through the public API: pinned host arrays -> upload -> K steps -> download
    e2e = None
    if want_e2e:
        pin = [torch.empty(cfg.npoints, dtype=torch.float64).pin_memory().numpy().reshape(cfg.shape)
               for _ in range(4)]
        for dst, src in zip(pin, (ux, uy, uz, p)):
            dst[...] = src
        outs = [torch.empty(cfg.npoints, dtype=torch.float64).pin_memory().numpy().reshape(cfg.shape)
                for _ in range(4)]
        barrier(ws)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.upload(*pin)
        s.step(args.steps)
        from channel3d_b200 import _lib
        _lib.check(s.lib.ch3d_download_state(s.ctx, _lib.LAYOUT_INTERIOR, *(_lib.dptr(o) for o in outs), None))
        torch.cuda.synchronize()
        te = time.perf_counter() - t0
        te = allmax(ws, te)
        bytes_io = 4 * cfg.npoints * 8
        e2e = {"value": ws * cfg.npoints * args.steps / te / 1e9, "unit": "Gpt-steps/s",
               "h2d_bytes_per_step": bytes_io / args.steps, "d2h_bytes_per_step": bytes_io / args.steps,
               "what": "ch3d_upload_state (4 FP64 arrays from pinned host memory) + ch3d_step(K) + "
                       "ch3d_download_state (4 arrays), wall clock, max over ranks"}
    r = {
        "cfg": cfg, "value": value, "ms_per_step": ms_per_step, "info": info, "wall_s": wall, "clocks": clocks,
        "path": path, "launches": launches, "kernels": per_group, "memory_bytes": s.memory_bytes(), "e2e": e2e,
        "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": peak_kind + " (hbm_gbs, burst copy)",
                     "alg_bytes_per_launch": dom_b,
                     "traffic_source": ("profiles/%s: ncu dram__bytes_read.sum + dram__bytes_write.sum per grid "
                                        "point of a smaller capture, scaled to this launch" % tsrc) if tsrc else None},
        "step_roofline": {"alg_bytes_per_cell_step": ALG_ARRAYS_PER_SUBSTEP[key] * 3 * word,
                          "achieved": step_achieved, "peak": peak, "frac": step_achieved / peak},
    }
    s.close()
    return r


def run_ours(args, ws, rank, local):
    main = measure(args, ws, rank, local, args.precision, not args.no_e2e)
    cfg = main["cfg"]
    # the other precision of the same workload, in the same process (FP64 against mixed)
    other = None
    if not args.no_mixed and args.precision == "fp64" and scheme_key(cfg) in ("pimp", "order4", "fimp") \
            and not args.les_type:
        other = measure(args, ws, rank, local, "mixed", not args.no_e2e)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            sample = cpu_sample_cfg(cfg.copy(precision="fp64", device=0), args.cpu_nz)
            v, thr, dt, nst = cpu_reference(sample, args, steps=args.cpu_steps)
            cpu = {"value": v, "unit": "Gpt-steps/s", "cores": thr, "kind": "port",
                   "sample": "%d RK3 steps (after 1 untimed) of a %dx%dx%d z-slab of %s (%.1f s); C++ restatement "
                             "of the reference step (oracle/), OpenMP, %d threads"
                             % (nst, sample.nxc, sample.nyc, sample.nzc, args.workload, dt, thr)}
        except Exception as ex:  # keep the GPU line even if host memory is short
            cpu = {"value": None, "unit": "Gpt-steps/s", "cores": None, "kind": "port", "sample": "failed: %s" % ex}

    if rank == 0:
        line = {
            "metric": "Gpt-steps/s", "value": main["value"], "unit": "Gpt-steps/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": main["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic (seeded laminar + 10% uniform noise, projected divergence-free)",
            "config": {"workload": args.workload, "grid": [cfg.nxc, cfg.nyc, cfg.nzc], "solver": solver_name(cfg),
                       "precision": args.precision, "parallelism": "replicas" if ws > 1 else "single",
                       "l2": "inputs larger than L2 (%.1f GB of fields)" % (main["memory_bytes"] / 1e9),
                       "kernel_path": main["path"]},
            "steps_per_s": 1e3 / main["ms_per_step"],
            "gpu_launches": int(args.steps * main["launches"]),
            "roofline": main["roofline"],
            "step_roofline": main["step_roofline"],
            "kernels": main["kernels"],
            "memory_bytes": main["memory_bytes"],
            "clocks": main["clocks"],
            "e2e": main["e2e"],
            "cpu_baseline": cpu,
            "last_info": main["info"],
            "wall_s": main["wall_s"],
        }
        if other is not None:
            c64, c32 = main["clocks"].get("sm_mhz"), other["clocks"].get("sm_mhz")
            line["mixed"] = {
                "value": other["value"], "unit": "Gpt-steps/s", "ms_per_step": other["ms_per_step"],
                "steps": args.steps, "dtype": "f32+f64", "steps_per_s": 1e3 / other["ms_per_step"],
                "gpu_launches": int(args.steps * other["launches"]), "kernel_path": other["path"],
                "roofline": other["roofline"], "step_roofline": other["step_roofline"],
                "kernels": other["kernels"], "memory_bytes": other["memory_bytes"], "clocks": other["clocks"],
                "e2e": other["e2e"], "last_info": other["info"],
                "speedup_vs_fp64": main["ms_per_step"] / other["ms_per_step"],
                "speedup_vs_fp64_at_equal_clock": (main["ms_per_step"] * c64) / (other["ms_per_step"] * c32)
                if c64 and c32 else None,
                "what": "the same workload in mixed precision (FP32 fields, stencils, ADI and FFTs; FP64 low-mode "
                        "Poisson y solves, bulk constraint and reductions), timed like the FP64 line in the same "
                        "process; speedup_vs_fp64_at_equal_clock compares time x median sampled SM clock",
            }
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_init()
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
