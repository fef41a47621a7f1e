"""Benchmark: MGPCG pressure-projection solves/s on one B200 (and N replicas).

Workload (one "step" = one projection): the 128x96x128 dam break with 16
falling spheres, consecutive steps at dt = 1/60 s, each with its own seeded
velocity field, solved to relative residual 1e-6 with the mixed-precision
solver (float16 V-cycle levels, float32 CG vectors, float64 dots/scalars).
Inputs are resident in HBM before timing; L2 is flushed (a 256 MB write)
between timed steps; every step is timed with CUDA events on the launching
stream.  The same steps are also timed with the plain float32 solver, through
the public API with host buffers (e2e), and with per-stage kernel events for
the roofline.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) every rank runs its own replica (the path does not
shard within a solve): value = all solves / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MGPCG solves/s @rel-res 1e-6: mixed/batched vs plain FP32 on 1 B200; p50/p99 ms"
WORKLOAD = "dam break + 16 falling spheres, 128x96x128 uniform MAC grid, dt=1/60, rel-res 1e-6"
L2_FLUSH_BYTES = 256 << 20

# Algorithmic bytes per finest cell of one launch, by kernel stage (s = bytes of
# the V-cycle storage type): every array a launch touches counts once at its
# storage width, stencil neighbours are assumed cached.
def stage_bytes_per_cell(stage: str, s: int) -> float:
    return {
        "smooth0": 4 + 4 + s + 1 + 2,          # z, r, diag(s), label in; half of z out
        "residual0": 4 + 4 + s + 1 + s,        # z, r, diag, label in; residual out
        "restrict0": 4 + 4 + s + 1 + (s + 1) / 8.0,   # z, r, diag, label in; coarse label in, coarse rhs out
        "prolong0": 4 + 4 + 1 + s / 8.0,       # z in/out, label, coarse z
        "spmv": 4 + 4 + 1 + 4,                 # d, diag, label in; q out
        "update": 4 * 5 + 1 + 4 * 3,           # x, xlo, d, q, r, label in; x, xlo, r out
        "dot": 4 + 4 + 1,
        "dir": 4 + 4 + 1 + 4,
        "true": 4 * 4 + 1 + 4,
        "down0": 4 + s + 1 + 4 + (1 + s) / 8.0,     # r, diag, label in; z out; coarse label in, coarse rhs out
        "up0": 4 + 4 + s + 1 + 4 + s / 8.0,         # z, r, diag, label, coarse z in; z out
        "dirspmv": 4 + 4 + 1 + 4 + 4 + 4,           # z, d, label, diag in; d', q out
    }.get(stage, 0.0)


# DRAM bytes per launch of the dominant kernel from the committed ncu capture
# (profiles/); None until a capture of the current kernel exists.
NCU_TRAFFIC_BYTES = {}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index: int, out_path: str | None = None):
        self.index = index
        self.proc = None
        self.path = out_path or os.path.join("/tmp", f"fluid_clocks_{os.getpid()}.csv")

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self) -> dict:
        try:
            rows = [l.strip().split(", ") for l in open(self.path) if l.strip()]
        except Exception:
            rows = []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reference_arm(args):
    """The reference's CPU path (float64 Jacobi-PCG of the atlas oracle), all host threads."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    from fluid_b200 import configs
    from oracle.oracle import Oracle
    threads = os.cpu_count() or 1
    times = []
    iters = []
    total = args.warmup + args.steps
    o = None
    for k in range(total):
        s = configs.dam_spheres(step=k % 50)
        if o is None:
            o = Oracle(s.nx, s.ny, s.nz, s.h, s.rho)
            o.set_threads(threads)
        o.set_state(s.vof, s.u, s.v, s.w, s.dt)
        t0 = time.perf_counter()
        _, info = o.solve_jacobi(1e-6, 0.0)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(dt)
            iters.append(info["iterations"])
    tot = sum(times)
    value = len(times) / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells": 128 * 96 * 128, "solver": "Jacobi-PCG float64 (atlas oracle)"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"{len(times)} full solves of consecutive steps, rel-res 1e-6, "
                                   f"mean {statistics.mean(iters):.0f} PCG iterations"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "p50_ms": 1000 * statistics.median(times), "p99_ms": 1000 * float(np.percentile(times, 99)),
    }
    print(json.dumps(line))
    return 0


def cpu_baseline_sample():
    from fluid_b200 import configs
    from oracle.oracle import Oracle
    threads = os.cpu_count() or 1
    s = configs.dam_spheres(step=0)
    o = Oracle(s.nx, s.ny, s.nz, s.h, s.rho)
    o.set_threads(threads)
    o.set_state(s.vof, s.u, s.v, s.w, s.dt)
    t0 = time.perf_counter()
    _, info = o.solve_jacobi(1e-6, 0.0)
    dt = time.perf_counter() - t0
    return {"value": 1.0 / dt, "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": f"1 full solve of step 0 (float64 Jacobi-PCG, {int(info['iterations'])} iterations, "
                      f"rel-res 1e-6) on the host, OpenMP"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp16", choices=["fp32", "fp16", "bf16"])
    ap.add_argument("--sweeps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)

    import torch

    from fluid_b200 import PressureProjector, configs
    from fluid_b200.projector import kernel_launches

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.current_stream()
    total = args.warmup + args.steps
    # 50 consecutive simulation steps; timed steps cycle through them
    states = [configs.dam_spheres(step=k) for k in range(min(total, 50))]
    nst = len(states)
    s0 = states[0]
    dev = [tuple(torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (s.vof, s.u, s.v, s.w)) for s in states]
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    opts = dict(rel_tol=1e-6, pre_sweeps=args.sweeps, post_sweeps=args.sweeps)

    def run(precision, profile=False):
        pp = PressureProjector((s0.nx, s0.ny, s0.nz), s0.h, s0.rho, precision=precision, device=local)
        pp.set_stream(stream.cuda_stream)
        pp.set_profiling(profile)
        times, recs = [], []
        for k in range(total):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            pp.upload_state_device(*(t.data_ptr() for t in dev[k % nst]))
            rec = pp.project(states[k % nst].dt, **opts)
            b.record(stream)
            b.synchronize()
            if k >= args.warmup:
                times.append(a.elapsed_time(b))
                recs.append(rec)
            if k == args.warmup - 1 and profile:
                pp.profile(reset=True)
        prof = pp.profile(reset=True) if profile else None
        pp.destroy()
        return times, recs, prof

    # timed region: mixed precision (headline)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    l0 = kernel_launches()
    with ClockSampler(local) as clk:
        times, recs, _ = run(args.precision)
    torch.cuda.synchronize()
    launches = kernel_launches() - l0
    tot_ms = sum(times)
    if world > 1:
        t = torch.tensor([tot_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        tot_ms = float(t.item())
    value = world * args.steps / (tot_ms / 1000.0)
    bad = [r for r in recs if r["status_name"] != "OK" or r["true_rel_residual"] > 1e-6]

    # plain float32 on the same steps
    times32, recs32, _ = run("fp32")
    plain = args.steps / (sum(times32) / 1000.0)

    # per-stage kernel events on the same steps (roofline)
    _, _, prof = run(args.precision, profile=True)
    sbytes = 4 if args.precision == "fp32" else 2
    ncell = s0.cells
    stages = {k: v for k, v in prof.items() if stage_bytes_per_cell(k, sbytes) > 0}
    dom = max(stages, key=lambda k: stages[k]["ms"])
    per_launch_ms = prof[dom]["ms"] / prof[dom]["launches"]
    alg = stage_bytes_per_cell(dom, sbytes) * ncell
    hbm, peak_kind = peaks()
    achieved = alg / (per_launch_ms / 1000.0) / 1e9
    tot_prof = sum(v["ms"] for v in prof.values())
    traffic = NCU_TRAFFIC_BYTES.get(dom)

    # end to end through the public API with pinned host buffers
    pp = PressureProjector((s0.nx, s0.ny, s0.nz), s0.h, s0.rho, precision=args.precision, device=local)
    pp.set_stream(stream.cuda_stream)
    host_in = [tuple(torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (s.vof, s.u, s.v, s.w))
               for s in states]
    host_out = tuple(torch.empty(sh, dtype=torch.float32).pin_memory()
                     for sh in ((s0.nz, s0.ny, s0.nx), (s0.nz, s0.ny, s0.nx + 1), (s0.nz, s0.ny + 1, s0.nx),
                                (s0.nz + 1, s0.ny, s0.nx)))
    h2d = sum(t.numel() * 4 for t in host_in[0])
    d2h = sum(t.numel() * 4 for t in host_out)
    from fluid_b200 import _abi
    L = _abi.load()
    e2e_ms = []
    for k in range(total):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        pp.upload_state(*(t.numpy() for t in host_in[k % nst]))
        pp.project(states[k % nst].dt, **opts)
        L.fluid_pp_download(pp.handle, *(_abi.ptr(t.numpy()) for t in host_out))
        b.record(stream)
        b.synchronize()
        if k >= args.warmup:
            e2e_ms.append(a.elapsed_time(b))
    pp.destroy()
    e2e_tot = sum(e2e_ms)
    if world > 1:
        t = torch.tensor([e2e_tot], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_tot = float(t.item())
    e2e_value = world * args.steps / (e2e_tot / 1000.0)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample()

    its = [r["iterations"] for r in recs]
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells": ncell, "precision": f"{args.precision} V-cycle levels, f32 CG "
                   "vectors, f64 dots/scalars/coarsest", "sweeps": args.sweeps, "l2": "flushed between steps (256 MB write)",
                   "parallelism": f"{world} replicas" if world > 1 else "single GPU"},
        "p50_ms": statistics.median(times), "p99_ms": float(np.percentile(times, 99)),
        "iterations_mean": statistics.mean(its),
        "cell_iterations_per_s": ncell * statistics.mean(its) * value,
        "plain_fp32_solves_per_s": plain, "plain_fp32_p50_ms": statistics.median(times32),
        "mixed_vs_plain": value / (world * plain),
        "failed_solves": len(bad),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_kind": peak_kind, "traffic": traffic,
                     "alg_bytes_per_launch": alg, "launch_ms": per_launch_ms,
                     "share_of_step": prof[dom]["ms"] / tot_prof},
        "stage_ms_per_step": {k: round(v["ms"] / args.steps, 4) for k, v in sorted(prof.items())},
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
