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


def _cpu_model() -> str:
    """The host CPU's model name (lscpu), for the CPU baseline's record."""
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for line in out.splitlines():
            if line.startswith("Model name:"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def _config(workload: str, world: int) -> dict:
    """The workload description both arms report (same dict in both lines)."""
    return {"workload": WORKLOAD_DESC.get(workload, workload + " (profiling case, not the benchmark workload)"),
            "global_batch": 1, "seq_len": None, "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2 (multi-GB sweep scratch per step)"}


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
    sample = (f"{angles_per_step} Fermi angle(s) of {na} per step: the Riccati sweep and Green "
              f"accumulation of those angles (no boundary condition, Poisson solve, accelerator or "
              f"rotation back), oracle port in FP64 on {threads} threads of {_cpu_model()}")
    return value, sum(times) / len(times), threads, sample


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
        "config": _config(args.workload, world),
        "cpu_baseline": {"value": value, "unit": "site-updates/s", "cores": threads,
                         "kind": "port", "sample": sample, "cpu_model": _cpu_model(),
                         "host_threads": os.cpu_count()},
        "e2e": {"value": value, "unit": "site-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


WORKLOAD_DESC = {
    "c2": "c2: d_x2-y2 square 30 xi0 @20/xi0 (N0=606, N1=858), axes 45 deg, 256 angles, "
          "T=0.1 (14 Ozaki poles), kappa=2, zero field",
}


def max_over_ranks(value: float, world: int, device: str = "cuda") -> float:
    """The largest value over all ranks (the replicas' timing rule); the
    identity for one process."""
    if world <= 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def _time_context(ctx, stream, steps, warmup, world):
    """Device-timed self-consistency iterations of one context (inputs resident)."""
    import torch
    for _ in range(warmup):
        ctx.compute(1)
    ctx.profile(True)
    launches0 = ctx.launch_count()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    ctx.compute(steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = ctx.launch_count() - launches0
    prof = {k: ctx.profile_read(i)
            for i, k in enumerate(("sweep", "rotate_back", "poisson", "boundary", "frame_fields"))}
    ctx.profile(False)
    ms = max_over_ranks(ms, world)
    return ms, launches, prof


def _e2e(ctx, steps, world):
    """Same metric through the public API with host buffers: every step the
    host sends x from pinned memory and reads x back into it."""
    import torch
    n0, nc = ctx.dims.n0, ctx.dims.n_comp
    host_d = torch.empty((nc, 2, n0, n0), dtype=torch.float64, pin_memory=True).numpy()
    host_a = torch.empty((2, n0, n0), dtype=torch.float64, pin_memory=True).numpy()
    xd, xa = ctx.state()
    host_d[...] = xd
    host_a[...] = xa
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.set_state(host_d, host_a)
        ctx.compute(1)
        ctx.state(host_d, host_a)
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    sec = max_over_ranks(sec, world)
    return sec, (nc * 2 * n0 * n0 + 2 * n0 * n0) * 8


def _curl(a, h):
    """B = curl A on the reference grid (curl_kernel, GridFunctions_GPU.h:326-352)."""
    import numpy as np
    n = a.shape[-1]
    idx = np.arange(n)
    xn, xp = np.minimum(idx + 1, n - 1), np.maximum(idx - 1, 0)
    day = (a[1][:, xn] - a[1][:, xp]) / (xn - xp)[None, :]
    dax = (a[0][xn, :] - a[0][xp, :]) / (xn - xp)[:, None]
    return (day - dax) / h


def converge_c1(max_it: int, max_s: float, extra_it: int = 400):
    """Time to converge (residual 1e-6) of the C1 disc in both precisions from
    the same seeded start, and the distance of the mixed solution from the FP64
    one in Delta, j, B and Omega: where both runs stop at the criterion, and
    after both continue for extra_it more iterations towards their fixed
    points (with the FP64 run's own distance between the two for scale)."""
    import numpy as np
    import superconga_b200 as sb
    from superconga_b200 import workloads
    cfg = workloads.c1()
    out, sol = {}, {}
    for mode in ("fp64", "mixed"):
        ctx = sb.Context(cfg, mode=mode)
        d0, a0 = workloads.initial_state("c1", cfg, ctx.dims.n0)
        ctx.set_state(d0, a0)
        import torch
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it, ok, res = 0, False, None
        while it < max_it and time.perf_counter() - t0 < max_s:
            res, ok = ctx.compute(1)
            it += 1
            if ok:
                break
        sec = time.perf_counter() - t0
        out[mode] = {"seconds": sec, "iterations": it, "converged": bool(ok), "final_residual": res,
                     "criterion": 1e-6}
        d, j, _ = ctx.results()
        _, a = ctx.state()
        sol[mode] = (d, j, a, ctx.scalars()["free_energy"])
        # Then on towards the fixed point itself: the difference of the two
        # runs at the criterion is mostly where each stopped.
        res2, _ = ctx.compute(extra_it)
        d, j, _ = ctx.results()
        _, a = ctx.state()
        sol[mode + "_fp"] = (d, j, a, ctx.scalars()["free_energy"])
        out[mode]["residual_after_more"] = res2
        ctx.close()
    out["mixed_vs_fp64"] = _field_errors(cfg, "s", sol["fp64"], sol["mixed"])
    out["continued_iterations"] = extra_it
    out["mixed_vs_fp64_continued"] = _field_errors(cfg, "s", sol["fp64_fp"], sol["mixed_fp"])
    out["fp64_at_criterion_vs_continued"] = _field_errors(cfg, "s", sol["fp64_fp"], sol["fp64"])
    out["speedup_mixed_over_fp64"] = out["fp64"]["seconds"] / out["mixed"]["seconds"]
    out["workload"] = "c1: s-wave disc R=10 xi0 @10/xi0, 64 angles, T=0.5, b=0.02 B0, kappa=2"
    return out


def _field_errors(cfg, sym, ref, other):
    """Max differences of (Delta, j, A, Omega) `other` from `ref`: Delta relative
    to the bulk gap, j and B = curl A to their largest FP64 magnitude, Omega
    relative."""
    import numpy as np
    from superconga_b200 import workloads
    lam2 = cfg["physics"]["penetration_depth"] ** 2
    h = 1.0 / cfg["numerics"]["points_per_coherence_length"]
    db = workloads.delta_bulk(cfg["physics"]["temperature"], sym)
    (d64, j64, a64, f64), (d32, j32, a32, f32) = ref, other
    b64, b32 = _curl(a64 / lam2, h), _curl(a32 / lam2, h)
    return {
        "delta_max_abs_over_delta_bulk": float(np.max(np.abs(d32 - d64)) / db),
        "j_max_abs_over_max_j": float(np.max(np.abs(j32 - j64)) / max(np.max(np.abs(j64)), 1e-300)),
        "b_max_abs_over_max_b": float(np.max(np.abs(b32 - b64)) / max(np.max(np.abs(b64)), 1e-300)),
        "omega_rel": float(abs(f32 - f64) / abs(f64)),
    }


def precision_c2(checkpoints=(1, 5, 20, 60)):
    """C2 from the seeded start in FP64 (the reference run), in mixed precision
    with mirror pairing (the default), in mixed precision without it, and in
    FP64 again from a start perturbed by 1e-7 relative (FP32 rounding level):
    the max error of Delta, j, B and Omega of each against the FP64 run after
    1, 5, 20 and 60 iterations.  C2 does not converge with the default
    accelerator (its residual wanders near 1e-3), so the comparison is at fixed
    iteration counts.  FP64 runs from starts perturbed by 1e-7, 1e-6 and 1e-5
    relative measure how much the iteration itself amplifies a difference of
    the size the mixed form makes in one iteration (the accelerator's adaptive
    steps and inertia switches are discrete decisions), against which the
    mixed errors are read."""
    import numpy as np
    import superconga_b200 as sb
    from superconga_b200 import workloads
    cfg = workloads.c2()
    runs = (("fp64", "fp64", False, 0.0), ("mixed", "mixed", False, 0.0),
            ("mixed_unpaired", "mixed", True, 0.0), ("fp64_perturbed_1e-7", "fp64", False, 1e-7),
            ("fp64_perturbed_1e-6", "fp64", False, 1e-6), ("fp64_perturbed_1e-5", "fp64", False, 1e-5))
    sol = {}
    for key, mode, unpaired, perturb in runs:
        if unpaired:
            os.environ["SCB_NO_PAIRING"] = "1"
        try:
            ctx = sb.Context(cfg, mode=mode)
        finally:
            os.environ.pop("SCB_NO_PAIRING", None)
        d0, a0 = workloads.initial_state("c2", cfg, ctx.dims.n0)
        if perturb:
            d0 = d0 * (1.0 + perturb * np.random.default_rng(22).standard_normal(d0.shape))
        ctx.set_state(d0, a0)
        done, snaps = 0, {}
        for cp in checkpoints:
            res, _ = ctx.compute(cp - done)
            done = cp
            d, j, _ = ctx.results()
            _, a = ctx.state()
            snaps[cp] = ((d, j, a, ctx.scalars()["free_energy"]), res)
        sol[key] = (snaps, ctx.sweep_plan()[1])
        ctx.close()
    out = {"workload": "c2", "checkpoints": list(checkpoints),
           "fp64_residual": {cp: sol["fp64"][0][cp][1] for cp in checkpoints}}
    for key, _, _, _ in runs[1:]:
        out[key] = {"mirror_pairing": sol[key][1]}
        for cp in checkpoints:
            e = _field_errors(cfg, "dx2-y2", sol["fp64"][0][cp][0], sol[key][0][cp][0])
            e["residual"] = sol[key][0][cp][1]
            out[key][f"after_{cp}"] = e
    return out


def c5_solve_and_ldos(max_it: int, max_s: float, blocks: int, ldos_max_it: int):
    """C5: the nine-vortex square (N0 = 1606, 128 angles, kappa = 5, b = 0.3)
    solved self-consistently in mixed precision (iterations until the 1e-6
    residual, at most max_it or max_s seconds, residual reported), then the
    LDOS postprocess on the result: 512 real energies in [-2 Delta0, 2 Delta0],
    broadening 0.02 Delta0, blocks of 32, each block run as runPostprocess runs
    it (burn-in until the boundary converges, then iterations until the LDOS
    converges, criterion 1e-4 as in the reference's examples).  By default all
    16 blocks run (`blocks` < 16 runs the first ones and estimates the rest
    from their mean time)."""
    import numpy as np
    import torch
    import superconga_b200 as sb
    from superconga_b200 import workloads
    cfg = workloads.c5()
    out = {"workload": "c5: s square 100 xi0 @16/xi0 (N0=1606, N1=2272), 128 angles, T=0.5 (7 Ozaki poles), "
                       "kappa=5, b=0.3 B0, nine seeded vortices, mixed precision"}
    ta = time.perf_counter()
    ctx = sb.Context(cfg, mode="mixed")
    out["setup_s"] = time.perf_counter() - ta
    d0, a0 = workloads.initial_state("c5", cfg, ctx.dims.n0)
    ctx.set_state(d0, a0)
    su = ctx.site_updates()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    it, ok, res, hist = 0, False, None, []
    while it < max_it and time.perf_counter() - t0 < max_s:
        res, ok = ctx.compute(1)
        it += 1
        if it % 25 == 0:
            hist.append([it, res])
        if ok:
            break
    sec = time.perf_counter() - t0
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    ctx.compute(5)
    ev1.record()
    torch.cuda.synchronize()
    ms_it = ev0.elapsed_time(ev1) / 5
    out["solve"] = {"iterations": it, "converged": bool(ok), "final_residual": res, "criterion": 1e-6,
                    "seconds": sec, "residual_every_25": hist, "ms_per_iteration": ms_it,
                    "site_updates_per_iteration": su, "site_updates_per_s": su / (ms_it * 1e-3)}
    d, a = ctx.state()
    ctx.close()
    d0 = workloads.S_WAVE_BULK
    pp = {"spectroscopy": {"energy_min": -2 * d0, "energy_max": 2 * d0, "num_energies": 512,
                           "energy_broadening": 0.02 * d0},
          "numerics": {"convergence_criterion": 1e-4, "norm": "l2", "num_energies_per_block": 32,
                       "num_fermi_momenta": 128}}
    e = sb.LdosContext(cfg, pp, mode="mixed")
    e.set_state(d, a)
    su_l = e.site_updates()
    per_block = []
    for blk in range(min(blocks, e.n_blocks)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e.begin_block(blk)
        nb = 0
        for nb in range(1, 1001):
            _, bconv = e.burn_in(1)
            if bconv:
                break
        ni, conv, r = 0, False, None
        while ni < ldos_max_it:
            r, conv = e.iterate(1)
            ni += 1
            if conv:
                break
        torch.cuda.synchronize()
        per_block.append({"block": blk, "burn_in_iterations": nb, "iterations": ni, "converged": bool(conv),
                          "residual": r, "seconds": time.perf_counter() - t0})
    ev0.record()
    e.iterate(2)
    ev1.record()
    torch.cuda.synchronize()
    ms_l = ev0.elapsed_time(ev1) / 2
    mean_s = float(np.mean([b["seconds"] for b in per_block]))
    all_run = len(per_block) == e.n_blocks
    out["ldos"] = {"energies": 512, "per_block": 32, "blocks_total": e.n_blocks, "blocks_run": len(per_block),
                   "blocks": per_block, "mean_s_per_block": mean_s,
                   "s_all_blocks": float(sum(b["seconds"] for b in per_block)) if all_run else None,
                   "estimated_s_all_blocks": None if all_run else mean_s * e.n_blocks,
                   "all_blocks_converged": all(b["converged"] for b in per_block),
                   "ms_per_ldos_iteration": ms_l, "site_updates_per_ldos_iteration": su_l,
                   "site_updates_per_s": su_l / (ms_l * 1e-3), "criterion": 1e-4}
    e.close()
    return out


def _run_batch_to_end(b, max_s: float):
    """Iterates a batch until every grain has finished (converged, at its
    iteration cap or diverged) or max_s seconds have passed; returns the
    seconds, synchronised with the device."""
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    while b.compute(10) > 0 and time.perf_counter() - t0 < max_s:
        pass
    torch.cuda.synchronize()
    return time.perf_counter() - t0


def _grain_summary(b):
    import numpy as np
    st = b.grain_states()
    _, it, r = b.status()
    return {"grains": len(st), "converged": st.count("converged"), "at_iteration_cap": st.count("at_cap"),
            "diverged": st.count("diverged"), "still_running": st.count("running"),
            "median_iterations": float(np.median(it)), "max_iterations": int(np.max(it)),
            "unconverged_final_residuals": [float(x) for x, s_ in zip(r, st) if s_ != "converged"]}


def batched_c3(n_grains: int, iters: int, subset: int, cap: int, max_s: float, full: bool):
    """The C3 batch: n seeded grains (discs and squares of uneven size, s/d,
    T ~ U(0.1, 0.9), fields up to 0.1 B0), each to residual 1e-6 or its
    iteration cap (num_iterations_max = cap).
    1. Throughput of the whole batch in both precisions: device-timed
       iterations with every grain active (CUDA-graph replays, after
       autotuning, which is set-up and timed apart).
    2. Convergence, measured end to end on a seeded subset of `subset` grains:
       the mixed batch, the FP64 batch, and the plain FP64 form one grain at a
       time (each grain its own context run until converged or capped, as the
       reference runs one grain per process).
    3. With `full`, every grain of the whole batch to its end in both
       precisions (minutes)."""
    import numpy as np
    import torch
    import superconga_b200 as sb
    from superconga_b200 import workloads
    cfgs, states = workloads.c3_grains(n_grains)
    for c in cfgs:
        c["numerics"]["num_iterations_max"] = cap
    res = {"workload": f"c3: {n_grains} seeded grains (discs R~U(4,20), squares w~U(8,40) xi0 @10/xi0, "
                       "s/d, T~U(0.1,0.9), b~U(0,0.1), kappa=2)", "criterion": 1e-6, "iteration_cap": cap}
    for mode in ("mixed", "fp64"):
        b = sb.Batch(cfgs, mode=mode)
        for g, c, st in zip(b.grains, cfgs, states):
            d, a = workloads.c3_initial_state(c, st, g.dims.n0)
            g.set_state(d, a)
        su = int(b.site_updates().sum())
        b.compute(1)  # first iteration (initial boundary values)
        ta = time.perf_counter()
        lg, mb, _ = b.autotune()
        t_tune = time.perf_counter() - ta
        b.compute(1)  # graph capture
        torch.cuda.synchronize()
        l0 = b.launch_count()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record()
        b.compute(iters)
        ev1.record()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / iters
        act, _, _ = b.status()
        full_active = bool(act.all())
        res[mode] = {"site_updates_per_s": su / (ms * 1e-3) if full_active else None,
                     "ms_per_iteration": ms, "site_updates_per_iteration": su,
                     "all_grains_active_while_timed": full_active,
                     "kernel_launches_per_iteration": (b.launch_count() - l0) / iters,
                     "sweep_mapping": {"max_energies_per_thread": lg, "min_blocks_per_sm": mb},
                     "autotune_seconds": t_tune}
        if full:
            sec = _run_batch_to_end(b, max_s)
            res[mode]["all_grains"] = dict(_grain_summary(b), seconds_after_tuning=sec)
        b.close()
    # Convergence on a seeded subset, end to end in all three forms.
    sub = sorted(np.random.default_rng(33).choice(n_grains, size=min(subset, n_grains), replace=False).tolist())
    scfg = [cfgs[i] for i in sub]
    conv = {"grains": sub}
    for mode in ("mixed", "fp64"):
        b = sb.Batch(scfg, mode=mode)
        for g, i in zip(b.grains, sub):
            g.set_state(*workloads.c3_initial_state(cfgs[i], states[i], g.dims.n0))
        sec = _run_batch_to_end(b, max_s)
        conv[f"{mode}_batch"] = dict(_grain_summary(b), seconds=sec)
        b.close()
    torch.cuda.synchronize()
    t_wall = time.perf_counter()
    n_conv, its, plain_s = 0, [], 0.0
    for i in sub:
        ctx = sb.Context(cfgs[i], mode="fp64")
        d0, a0 = workloads.c3_initial_state(cfgs[i], states[i], ctx.dims.n0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.set_state(d0, a0)
        k, ok = ctx.run(0, cap)
        torch.cuda.synchronize()
        plain_s += time.perf_counter() - t0
        n_conv += int(ok)
        its.append(k)
        ctx.close()
    conv["plain_fp64_one_grain_at_a_time"] = {
        "seconds": plain_s, "converged": n_conv, "median_iterations": float(np.median(its)),
        "seconds_with_setup": time.perf_counter() - t_wall,
        "note": "sum over the grains of set_state + iterations to the end (as the batch runs are timed, "
                "contexts created beforehand); seconds_with_setup adds each grain's context creation"}
    conv["mixed_batch_over_plain_fp64"] = plain_s / conv["mixed_batch"]["seconds"]
    conv["mixed_batch_over_fp64_batch"] = conv["fp64_batch"]["seconds"] / conv["mixed_batch"]["seconds"]
    res["convergence_subset"] = conv
    return res


def ldos_c5(iters: int, ppxi: float = 16.0, modes=("mixed", "fp64")):
    """LDOS postprocess throughput on the C5 grain: one block of 32 real
    energies in [-2 Delta0, 2 Delta0], broadening 0.02 Delta0, on the seeded
    nine-vortex state (LDOS iterations after one burn-in and one iteration),
    with the device time of the sweep and of the rotation back per iteration.
    ppxi < 16 runs the same grain at a coarser lattice (a small case for
    profiling)."""
    import torch
    import superconga_b200 as sb
    from superconga_b200 import workloads
    cfg = workloads.c5()
    cfg["numerics"]["points_per_coherence_length"] = ppxi
    d0 = workloads.S_WAVE_BULK
    pp = {"spectroscopy": {"energy_min": -2 * d0, "energy_max": 2 * d0, "num_energies": 512,
                           "energy_broadening": 0.02 * d0},
          "numerics": {"convergence_criterion": 1e-6, "norm": "l2", "num_energies_per_block": 32,
                       "num_fermi_momenta": 128}}
    out = {"workload": f"c5 LDOS: s square 100 xi0 @{ppxi:g}/xi0, 128 angles, 32 energies per block"}
    for mode in modes:
        e = sb.LdosContext(cfg, pp, mode=mode)
        d, a = workloads.initial_state("c5", cfg, e.dims.n0)
        e.set_state(d, a)
        e.begin_block(0)
        e.burn_in(1)
        e.iterate(1)
        su = e.site_updates()
        torch.cuda.synchronize()
        e.profile(True)
        t0 = time.perf_counter()
        e.iterate(iters)
        torch.cuda.synchronize()
        sec = (time.perf_counter() - t0) / iters
        split = {k: e.profile_read(i)[0] / iters for i, k in enumerate(("sweep", "rotate_back"))}
        e.profile(False)
        out[mode] = {"n0": e.dims.n0, "n1": e.dims.n1, "angle_chunks": e.sweep_plan()[0],
                     "site_updates_per_s": su / sec, "s_per_iteration": sec,
                     "site_updates_per_iteration": su, "kernel_ms_per_iteration": split}
        e.close()
    return out


def adjoint_c4(n_dirs: int = 64, eps: float = 1e-4):
    """The adjoint on C4 (chiral d + i d_xy disc R = 15 xi0 @15/xi0, 128 angles,
    T = 0.3, b = 0.05, kappa = 2), FP64, frozen boundary after 5 burn-in
    iterations: the median time (host clock around the call, synchronised)
    of a frozen-boundary evaluation and of five adjoints, and the largest
    relative difference between the adjoint's
    directional derivatives and central differences (step eps) along n_dirs
    seeded random directions, for the free energy and for the total azimuthal
    current in a 2 xi0 ring at the edge."""
    import numpy as np
    import torch
    import superconga_b200 as sb
    from superconga_b200 import workloads
    from superconga_b200.autograd import edge_current_weights
    cfg = workloads.c4()
    e = sb.Context(cfg, mode="fp64")
    n0 = e.dims.n0
    d, a = workloads.initial_state("c4", cfg, n0)
    a = 0.05 * np.random.default_rng(44).standard_normal((2, n0, n0))
    e.set_state(d, a)
    e.burn_in(5)
    dom = e.domain() > 0
    d = d * dom
    h = 1.0 / cfg["numerics"]["points_per_coherence_length"]
    beta = edge_current_weights(e.domain(), h, 2.0)
    b0 = e.external_field()
    db = workloads.delta_bulk(0.3, "dx2-y2")

    def f(dd, aa, bb, loss):
        e.set_state(dd, aa)
        e.set_external_field(bb)
        fe = e.evaluate()
        return fe if loss == "omega" else float(np.sum(beta * e.results()[1]))

    out = {"workload": "c4: chiral d+id disc R=15 xi0 @15/xi0 (N0=%d), 128 angles, T=0.3, b=0.05, kappa=2" % n0,
           "directions": n_dirs, "fd_step": eps}
    for loss in ("omega", "edge_current"):
        t_adj = []
        for _ in range(5):
            f(d, a, b0, loss)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            gd, ga, gb = e.adjoint(1.0, None) if loss == "omega" else e.adjoint(0.0, beta)
            torch.cuda.synchronize()
            t_adj.append(time.perf_counter() - t0)
        rng = np.random.default_rng(4)
        worst = 0.0
        t_eval = []
        for _ in range(n_dirs):
            vd = rng.standard_normal(d.shape) * db * dom
            va = rng.standard_normal(a.shape) * 0.05
            vb = float(rng.standard_normal()) * 0.01
            t0 = time.perf_counter()
            fp = f(d + eps * vd, a + eps * va, b0 + eps * vb, loss)
            t_eval.append(time.perf_counter() - t0)
            fm = f(d - eps * vd, a - eps * va, b0 - eps * vb, loss)
            fd = (fp - fm) / (2 * eps)
            ad = float(np.sum(gd * vd) + np.sum(ga * va) + gb * vb)
            worst = max(worst, abs(fd - ad) / max(abs(fd), abs(ad), 1e-300))
        out[loss] = {"adjoint_s": float(np.median(t_adj)), "evaluation_s": float(np.median(t_eval)),
                     "max_rel_diff_vs_fd": worst}
    e.close()
    return out


def run_engine(args):
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
        torch.distributed.barrier()
    import superconga_b200 as sb
    from superconga_b200 import workloads
    from superconga_b200.engine import fma_peak

    if args.ldos_only:
        if rank == 0:
            print(json.dumps({"ldos": ldos_c5(2, args.ldos_ppxi, args.modes.split(","))}), flush=True)
        return
    cfg = workloads.WORKLOADS[args.workload]()
    hbm, hbm_kind = _peaks()
    results = {}
    modes = args.modes.split(",")
    sampler = ClockSampler(local)
    sampler.__enter__()
    for mode in modes:
        unpaired = mode == "mixed_unpaired"
        if unpaired:  # mixed precision with the mirror pairing turned off
            os.environ["SCB_NO_PAIRING"] = "1"
        try:
            ctx = sb.Context(cfg, mode="mixed" if unpaired else mode)
        finally:
            os.environ.pop("SCB_NO_PAIRING", None)
        n_chunks, paired = ctx.sweep_plan()
        stream = torch.cuda.Stream()
        ctx.set_stream(stream.cuda_stream)
        su = ctx.site_updates()
        d0, a0 = workloads.initial_state(args.workload, cfg, ctx.dims.n0)
        ctx.set_state(d0, a0)
        ms, launches, prof = _time_context(ctx, stream, args.steps, args.warmup, world)
        value = world * su * args.steps / (ms * 1e-3)
        e2e_s, bytes_io = _e2e(ctx, args.steps, world)
        sweep_ms, sweep_n = prof["sweep"]
        sweep_avg_s = (sweep_ms / max(sweep_n, 1)) * 1e-3
        su_per_launch = su / (max(sweep_n, 1) / args.steps)
        bpsu = BYTES_PER_SU["fp64" if mode == "fp64" else "mixed"]
        # A paired sweep steps only the primary angle of each mirror pair: the
        # Riccati steps it executes are half the site-updates it delivers, and
        # only their coherence functions are stored and read back.  The
        # roofline counts the executed steps (the delivered count is reported
        # beside it as the notional figure).
        executed = su / 2 if paired else su
        exec_per_launch = su_per_launch / 2 if paired else su_per_launch
        achieved_gbs = exec_per_launch * bpsu / sweep_avg_s / 1e9
        pipe_peak = fma_peak(64 if mode == "fp64" else 32)
        achieved_flops = exec_per_launch * FLOPS_PER_SU / sweep_avg_s
        tr = _traffic(mode)
        traffic = None if tr is None else tr * su_per_launch
        results[mode] = {
            "value": value, "ms_per_step": ms / args.steps, "site_updates_per_step": su,
            "executed_riccati_steps_per_s": world * executed * args.steps / (ms * 1e-3),
            "mirror_pairing": paired, "angle_chunks": n_chunks,
            "gpu_launches": launches,
            "e2e": {"value": world * su * args.steps / e2e_s, "unit": "site-updates/s",
                    "h2d_bytes_per_step": bytes_io, "d2h_bytes_per_step": bytes_io},
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm, "unit": "GB/s",
                         "frac": achieved_gbs / hbm,
                         "traffic": traffic,
                         "peak_kind": hbm_kind, "kernel": "k_sweep",
                         "kernel_ms_per_launch": sweep_avg_s * 1e3,
                         "algorithmic_bytes_per_launch": exec_per_launch * bpsu,
                         "executed_site_updates_per_launch": exec_per_launch,
                         "delivered_site_updates_per_launch": su_per_launch,
                         "notional_frac_delivered": su_per_launch * bpsu / sweep_avg_s / 1e9 / hbm,
                         "dram_gbs": None if traffic is None else traffic / sweep_avg_s / 1e9,
                         "dram_frac": None if traffic is None else traffic / sweep_avg_s / 1e9 / hbm,
                         "traffic_over_algorithmic": None if traffic is None else traffic / (exec_per_launch * bpsu),
                         "note": ("achieved counts the algorithmic bytes (16 B FP32 / 32 B FP64 of "
                                  "coherence function written and read) of the executed Riccati steps; with "
                                  "mirror pairing the partner angle's half of the delivered site-updates is "
                                  "derived, not stepped (notional_frac_delivered counts those too). "
                                  "dram_frac is the measured DRAM traffic (ncu) over the launch time: the "
                                  "sweep is issue/latency-bound, not DRAM-bound; pipe counts ~135 flops "
                                  "per executed step against the library's FMA-loop peak."),
                         "pipe": {"precision": "fp64" if mode == "fp64" else "fp32",
                                  "achieved_tflops": achieved_flops / 1e12,
                                  "peak_tflops": pipe_peak / 1e12,
                                  "frac": achieved_flops / pipe_peak,
                                  "peak_kind": "measured FMA loop"}},
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in prof.items()},
        }
        ctx.close()
        del stream
    extra = {}
    if rank == 0 and world == 1 and not args.no_precision:
        extra["precision_c2"] = precision_c2()
    if rank == 0 and world == 1 and not args.no_converge:
        extra["time_to_converge"] = converge_c1(args.converge_max_it, args.converge_max_s)
    if rank == 0 and world == 1 and not args.no_batch:
        extra["batched"] = batched_c3(args.batch_grains, args.batch_iters, args.batch_subset, args.batch_cap,
                                      args.batch_max_s, args.c3_full)
    if rank == 0 and world == 1 and args.ldos:
        extra["ldos"] = ldos_c5(2, args.ldos_ppxi)
    if rank == 0 and world == 1 and not args.no_c5:
        extra["c5"] = c5_solve_and_ldos(args.c5_max_it, args.c5_max_s, args.c5_blocks, args.c5_ldos_max_it)
    if rank == 0 and world == 1 and not args.no_adjoint:
        extra["adjoint"] = adjoint_c4()
    sampler.__exit__(None, None, None)
    clocks = sampler.summary()

    m = results[modes[0]]
    line = {
        "metric": "riccati_site_updates_per_s", "value": m["value"], "unit": "site-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 stepping / f64 accumulation" if modes[0] == "mixed" else "f64",
        "data": "synthetic (seeded)",
        "config": _config(args.workload, world), "mode": modes[0],
        "e2e": m["e2e"], "gpu_launches": m["gpu_launches"], "roofline": m["roofline"],
        "clocks": clocks, "kernel_ms_per_step": m["kernel_ms_per_step"],
    }
    line["executed_riccati_steps_per_s"] = m["executed_riccati_steps_per_s"]
    line["mirror_pairing"] = m["mirror_pairing"]
    if "fp64" in results and modes[0] != "fp64":
        line["fp64"] = results["fp64"]
        line["mixed_over_fp64"] = m["value"] / results["fp64"]["value"]
    if "mixed_unpaired" in results:
        line["mixed_unpaired"] = results["mixed_unpaired"]
    if "fp64" in results and "mixed_unpaired" in results and modes[0] == "mixed":
        # The mixed/FP64 ratio split into its two factors: FP32 stepping alone
        # (both sweep every angle) and the mirror pairing of mixed mode.
        prec = results["mixed_unpaired"]["value"] / results["fp64"]["value"]
        line["precision_split"] = {
            "mixed_over_fp64": m["value"] / results["fp64"]["value"],
            "mixed_unpaired_over_fp64": prec,
            "pairing_gain": m["value"] / results["mixed_unpaired"]["value"],
            "sweep_ms": {k: results[k]["kernel_ms_per_step"]["sweep"] for k in ("mixed", "mixed_unpaired", "fp64")},
        }
    line.update(extra)
    if rank == 0 and world == 1 and not args.no_cpu:
        v, sec, threads, sample = cpu_reference(2, 1, workload=args.workload)
        line["cpu_baseline"] = {"value": v, "unit": "site-updates/s", "cores": threads,
                                "kind": "port", "sample": sample, "cpu_model": _cpu_model(),
                                "host_threads": os.cpu_count()}
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
    ap.add_argument("--modes", default="mixed,fp64,mixed_unpaired")
    ap.add_argument("--no-precision", action="store_true")
    ap.add_argument("--no-c5", action="store_true")
    ap.add_argument("--c5-max-it", type=int, default=1500)
    ap.add_argument("--c5-max-s", type=float, default=60.0)
    ap.add_argument("--c5-blocks", type=int, default=16)
    ap.add_argument("--c5-ldos-max-it", type=int, default=200)
    ap.add_argument("--no-converge", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--converge-max-it", type=int, default=400)
    ap.add_argument("--converge-max-s", type=float, default=60.0)
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--batch-grains", type=int, default=128)
    ap.add_argument("--batch-iters", type=int, default=5)
    ap.add_argument("--ldos", action="store_true", help="also time the C5 LDOS postprocess")
    ap.add_argument("--ldos-only", action="store_true",
                    help="only the C5 LDOS iteration timing (modes from --modes), one JSON line")
    ap.add_argument("--ldos-ppxi", type=float, default=16.0, help="lattice points per xi0 of that run")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--batch-max-s", type=float, default=300.0)
    ap.add_argument("--batch-subset", type=int, default=16)
    ap.add_argument("--batch-cap", type=int, default=3000)
    ap.add_argument("--c3-full", action="store_true", help="every grain of the C3 batch to its end (minutes)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
