#!/usr/bin/env python
"""Benchmark of the SuperConga self-consistency hot path on B200.

Metric: in-grain Riccati site-updates per second (one site-update = one
midpoint step of gamma or gammaTilde at one lattice site with domain label > 0,
for one Fermi angle and one Ozaki energy), mixed precision (FP32 Riccati
stepping, FP64 accumulation) next to plain FP64, plus the time to converge to a
self-consistency residual of 1e-6.  A step is one self-consistency iteration
(Context::compute) of the workload.

Workload: the d_{x2-y2} square of side 30 xi0 with crystal axes at 45 degrees
at 20 points/xi0 (N0 = 606, N1 = 858), 256 Fermi angles, T = 0.1 Tc (14 Ozaki
poles), self-consistent vector potential with kappa = 2, seeded initial order
parameter Delta_bulk (1 + 0.1 (N + iN)).  Synthetic, generated from a seed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Under torchrun every rank runs an independent replica of the workload (the
path does not shard across GPUs here); the value is the sum over ranks and the
time the maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "c2"
# Algorithmic work per site-update: 32 B (FP64) or 16 B (FP32 storage) of
# coherence function written once and read once; ~135 flops (midpoint step plus
# the shared Green / free-energy evaluation).
BYTES_PER_SU = {"fp64": 32.0, "mixed": 16.0}
FLOPS_PER_SU = 135.0
FALLBACK_HBM_GBS = 6650.0


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def _traffic(mode: str):
    """DRAM bytes per sweep launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "sweep_traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith(f"{mode} "):
                    return float(line.split()[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"scb_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_reference(steps: int, warmup: int, angles_per_step: int = 16, workload: str = WORKLOAD):
    """Times the CPU oracle (the restated OpenMP reference path) on a bounded
    sample of the workload: whole Fermi angles of the Riccati sweep and Green
    accumulation, all host threads."""
    from oracle import oracle as O
    from superconga_b200 import workloads
    import numpy as np

    cfg = workloads.WORKLOADS[workload]()
    o = O.Oracle(cfg)
    s = o.setup
    d, a = workloads.initial_state(workload, cfg, s.n0)
    o.set_state(d, a)
    o.set_boundary_initial()
    na = s.n_angles
    inside = [int(np.count_nonzero(o.geometry(k)[0] > 0)) for k in range(na)]
    order = [(k * 37) % na for k in range(na)]
    times, sus = [], []
    idx = 0
    for step in range(warmup + steps):
        su = 0
        t0 = time.perf_counter()
        for _ in range(angles_per_step):
            ang = order[idx % na]
            idx += 1
            o.angle_greens(ang)
            su += 2 * s.n_energies * inside[ang]
        dt = time.perf_counter() - t0
        if step >= warmup:
            times.append(dt)
            sus.append(su)
    value = sum(sus) / sum(times)
    threads = os.cpu_count()
    try:
        threads = int(os.environ.get("OMP_NUM_THREADS", threads))
    except ValueError:
        pass
    return value, sum(times) / len(times), threads, f"{angles_per_step} Fermi angle(s) of {na} per step"


def run_reference(args):
    world, rank, _ = _dist()
    if rank != 0:
        return
    value, sec, threads, sample = cpu_reference(args.steps, args.warmup, workload=args.workload)
    line = {
        "impl": "reference", "metric": "riccati_site_updates_per_s", "value": value,
        "unit": "site-updates/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": "c2: d-wave square 30 xi0 @20/xi0, 256 angles, T=0.1, 14 Ozaki poles, kappa=2",
                   "sample": sample},
        "cpu_baseline": {"value": value, "unit": "site-updates/s", "cores": threads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "site-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_engine(args):
    import numpy as np
    import torch

    world, rank, local = _dist()
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    from superconga_b200 import build
    if rank == 0:
        build.build()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    import superconga_b200 as sb
    from superconga_b200 import workloads
    from superconga_b200.engine import fma_peak

    cfg = workloads.WORKLOADS[args.workload]()
    hbm, hbm_kind = _peaks()
    results = {}
    modes = args.modes.split(",")
    for mode in modes:
        ctx = sb.Context(cfg, mode=mode)
        stream = torch.cuda.Stream()
        ctx.set_stream(stream.cuda_stream)
        n0, nc = ctx.dims.n0, ctx.dims.n_comp
        su = ctx.site_updates()
        d0, a0 = workloads.initial_state(args.workload, cfg, n0)
        ctx.set_state(d0, a0)
        for _ in range(args.warmup):
            ctx.compute(1)
        # device-timed region: K iterations, inputs resident in HBM
        ctx.profile(True)
        launches0 = ctx.launch_count()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            ev0.record(stream)
            ctx.compute(args.steps)
            ev1.record(stream)
            torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        launches = ctx.launch_count() - launches0
        sweep_ms, sweep_n = ctx.profile_read(0)
        rb_ms, _ = ctx.profile_read(1)
        pois_ms, _ = ctx.profile_read(2)
        bc_ms, _ = ctx.profile_read(3)
        ctx.profile(False)
        clocks = clk.summary()
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms = float(t.item())
        per_step = ms / args.steps
        value = world * su * args.steps / (ms * 1e-3)
        # end to end through the public API with host buffers: every step the
        # host sends x (pinned) and reads x back.
        nd = nc * 2 * n0 * n0
        host_d = torch.empty((nc, 2, n0, n0), dtype=torch.float64, pin_memory=True).numpy()
        host_a = torch.empty((2, n0, n0), dtype=torch.float64, pin_memory=True).numpy()
        xd, xa = ctx.state()
        host_d[...] = xd
        host_a[...] = xa
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ctx.set_state(host_d, host_a)
            ctx.compute(1)
            xd, xa = ctx.state()
            host_d[...] = xd
            host_a[...] = xa
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        if world > 1:
            t = torch.tensor([e2e_s], device="cuda")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = world * su * args.steps / e2e_s
        bytes_io = (nd + 2 * n0 * n0) * 8
        # roofline of the dominant kernel, the sweep
        sweep_avg_s = (sweep_ms / max(sweep_n, 1)) * 1e-3
        sweeps_per_step = max(sweep_n, 1) / args.steps
        su_per_launch = su / sweeps_per_step
        achieved_gbs = su_per_launch * BYTES_PER_SU[mode] / sweep_avg_s / 1e9
        pipe_peak = fma_peak(64 if mode == "fp64" else 32)
        achieved_flops = su_per_launch * FLOPS_PER_SU / sweep_avg_s
        traffic = _traffic(mode)
        results[mode] = {
            "value": value, "ms_per_step": per_step, "site_updates_per_step": su,
            "gpu_launches": launches, "clocks": clocks,
            "e2e": {"value": e2e, "unit": "site-updates/s", "h2d_bytes_per_step": bytes_io,
                    "d2h_bytes_per_step": bytes_io},
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm, "unit": "GB/s",
                         "frac": achieved_gbs / hbm, "traffic": traffic,
                         "peak_kind": hbm_kind,
                         "kernel": "k_sweep", "kernel_ms_per_launch": sweep_avg_s * 1e3,
                         "pipe": {"precision": "fp64" if mode == "fp64" else "fp32",
                                  "achieved_tflops": achieved_flops / 1e12,
                                  "peak_tflops": pipe_peak / 1e12,
                                  "frac": achieved_flops / pipe_peak,
                                  "peak_kind": "measured FMA loop"}},
            "kernel_ms_per_step": {"sweep": sweep_ms / args.steps, "rotate_back": rb_ms / args.steps,
                                   "poisson": pois_ms / args.steps, "boundary": bc_ms / args.steps},
        }
        # time to converge (residual 1e-6) from the seeded start, bounded
        conv = None
        if not args.no_converge:
            ctx2 = sb.Context(cfg, mode=mode)
            ctx2.set_stream(stream.cuda_stream)
            ctx2.set_state(d0, a0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            it, ok, res = 0, False, None
            while it < args.converge_max_it and time.perf_counter() - t0 < args.converge_max_s:
                res, ok = ctx2.compute(1)
                it += 1
                if ok:
                    break
            conv = {"seconds": time.perf_counter() - t0, "iterations": it, "converged": bool(ok),
                    "final_residual": res, "criterion": 1e-6}
            ctx2.close()
        results[mode]["time_to_converge"] = conv
        ctx.close()
        del stream

    m = results[modes[0]]
    line = {
        "metric": "riccati_site_updates_per_s", "value": m["value"], "unit": "site-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 stepping / f64 accumulation", "data": "synthetic (seeded)",
        "config": {"workload": "c2: d_x2-y2 square 30 xi0 @20/xi0 (N0=606, N1=858), axes 45 deg, "
                               "256 angles, T=0.1 (14 Ozaki poles), kappa=2, zero field",
                   "global_batch": 1, "seq_len": None, "parallelism": "replicas" if world > 1 else "single",
                   "mode": modes[0], "l2": "inputs larger than L2 (multi-GB sweep scratch per step)"},
        "e2e": m["e2e"], "gpu_launches": m["gpu_launches"], "roofline": m["roofline"],
        "clocks": m["clocks"], "kernel_ms_per_step": m["kernel_ms_per_step"],
        "time_to_converge": m["time_to_converge"],
    }
    if "fp64" in results and modes[0] != "fp64":
        line["fp64"] = results["fp64"]
        line["mixed_over_fp64"] = m["value"] / results["fp64"]["value"]
    if args.workload != WORKLOAD:
        line["config"]["workload"] = args.workload + " (profiling case, not the benchmark workload)"
    if rank == 0 and world == 1 and not args.no_cpu:
        v, sec, threads, sample = cpu_reference(2, 1, workload=args.workload)
        line["cpu_baseline"] = {"value": v, "unit": "site-updates/s", "cores": threads,
                                "kind": "port", "sample": sample + ", oracle (FP64)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--workload", default=WORKLOAD, choices=["c1", "c2", "c2p", "c4", "c5"])
    ap.add_argument("--modes", default="mixed,fp64")
    ap.add_argument("--no-converge", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--converge-max-it", type=int, default=400)
    ap.add_argument("--converge-max-s", type=float, default=60.0)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
