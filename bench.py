"""Benchmark: MGPCG solves/s on one B200 (and N replicas): mixed/batched vs plain FP32.

Headline workload (one "step" = one batched projection): 64 independent
uniform MAC grids of uneven size (edges log-uniform in 24-128 per axis, liquid
= seeded unions of 1-6 boxes and spheres filling 20-70%, Gaussian velocities
sigma 0.2 m/s), all projected to relative residual 1e-6 by one batched solve
(one launch per stage for every instance, CUDA graphs with a device-side
loop) with float16 V-cycle levels, float32 CG vectors and float64 dots.  The
comparator is plain float32 single-solve MGPCG over the same 64 instances, one
handle after the other.  Secondary: the 128x96x128 dam break with 16 spheres
(consecutive steps), mixed vs plain, single solve.

Inputs are resident in HBM before timing (the timed step re-uploads each
instance's state device-to-device, as a simulation step hands over its
advected state); L2 is flushed (256 MB write) before every timed step; every
step is timed with CUDA events on the launching stream.  `e2e` repeats the
headline through the public API from pinned host buffers with the results read
back to the host: PipelinedBatchProjector keeps three ticks in flight on three
streams, so one tick's copies overlap the others' solves; `serial_solves_per_s`
is the same ticks one after another.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) every rank runs its own replica (a solve does not
shard): value = all solves / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import faulthandler
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
WORKLOAD = ("64 independent uniform MAC grids in one batched projection per step: edges log-uniform 24-128 "
            "per axis, liquid = 1-6 seeded boxes/spheres filling 20-70%, Gaussian velocities sigma 0.2 m/s, "
            "rel-res 1e-6 per instance")
WORKLOAD2 = "dam break + 16 falling spheres, 128x96x128 uniform MAC grid, 50 consecutive steps, dt=1/60, rel-res 1e-6"
L2_FLUSH_BYTES = 256 << 20
BATCH = 64


# Algorithmic bytes per finest cell of one launch, by kernel stage (s = bytes of
# the V-cycle storage type): every array a launch touches counts once at its
# storage width, stencil neighbours are assumed cached.
def stage_bytes_per_cell(stage: str, s: int) -> float:
    return {
        "smooth0": 4 + 4 + s + 1 + 2,          # z, r, diag(s), label in; half of z out
        "restrict0": 4 + 4 + s + 1 + (s + 1) / 8.0,   # z, r, diag, label in; coarse label in, coarse rhs out
        "prolong0": 4 + 4 + 1 + s / 8.0,       # z in/out, label, coarse z
        "spmv": 4 + 4 + 1 + 4,                 # d, diag, label in; q out
        "update": 4 * 5 + 1 + 4 * 3,           # x, xlo, d, q, r, label in; x, xlo, r out
        "dot": 4 + 4 + 1,
        "dir": 4 + 4 + 1 + 4,
        "true": 4 * 4 + 1 + 4,
        "down0": 4 + 4 + 4 + (1 + s) / 8.0,         # r, diag (f32) in; z out; coarse label in, coarse rhs out
        "up0": 4 + 4 + 4 + 4 + s / 8.0,             # pre-smoothed z, r, diag (f32), coarse z in; z out
        "dirspmv": 4 + 4 + 4 + 4 + 4,               # z, d, diag in; d', q out (liquid = diag > 0)
    }.get(stage, 0.0)


# DRAM bytes (read + write) of one launch of a stage's kernel on the headline
# batch when every one of the 64 instances iterates (the first CG iteration),
# from the committed ncu capture of that launch (profiles/column_kernels_batch64_fp16.md,
# cold cache).  The roofline scales it to the average launch of a solve by the
# cells that launch processes (later launches skip finished instances).
CYCLE_STEPS = 8
SOLID_DIMS = (128, 96, 128)   # the 128x96x128 lattice with a ramp and a moving ball as embedded solids
SOLID_STEPS = 8
TRANSPORT_DIMS = (128, 96, 128)   # the density-transport lattice (dam block + ball, swirling extrapolated faces)
TRANSPORT_STEPS = 20
ATLAS_DIMS = (256, 192, 256)   # the sparse-atlas domain (a pool and 40 drops: 8508 of 24576 bricks)
ATLAS_STEPS = 10
SERVE_CELLS = 8e6     # resident uniform cells: the batched step stays near 8 ms
SERVE_TALL = 2        # resident tall-cell simulations (they share the tall slices)
NCU_FIRST_LAUNCH_BYTES = {"down0": 149.1e6, "up0": 214.4e6, "dirspmv": 250.8e6}


def tall_bytes_per_iteration(level_samples, level_storage, sweeps=1) -> float:
    """Algorithmic bytes of one tall-cell CG iteration: the CG vector kernels on
    the finest samples (SpMV s + 16 + s, update 6x4, direction 3x4 at float32
    vectors) plus, on every level l at its storage width s_l (coefficients 3
    floats and a flag: 16 B, or 8 B at 2-byte storage), (pre + post) RBGS sweeps
    of 2(s + s + coeff) + s, residual + restriction s + s + coeff + s/8 and
    prolongation s/8 + 2s per sample."""
    n0 = level_samples[0]
    total = n0 * ((4 + 16 + 4) + 6 * 4 + 3 * 4)
    for n, s in zip(level_samples, level_storage):
        coeff = 16 if s == 4 else 8
        per = 2 * sweeps * (2 * (s + s + coeff) + s) + (s + s + coeff + s / 8.0) + (s / 8.0 + 2 * s)
        total += n * per
    return total


def transport_bytes_per_cell(diffusion_iterations: int = 1) -> float:
    """Algorithmic bytes of one density-transport step per cell (float32
    fields, int32 deposits, each array once per kernel): deposit clears 12 + 4,
    trace and beta (u, v, w, gamma, gamma~, beta, trace offsets) 36, deficit
    scatter (beta, rho, gamma, two deposits) 20, gather (gamma~, beta, rho, two
    deposits, trace offsets, rho', gamma') 40, 16 per diffusion pass (3 per
    repetition) and 8 for the gamma copy after an odd pass count, sharpening
    12, its scatter 4 and resolve 12, the two mass receipts 8."""
    passes = 3 * diffusion_iterations
    return 16 + 36 + 20 + 40 + 16 * passes + (8 if passes % 2 else 0) + 12 + 4 + 12 + 8


def atlas_bytes_per_cell_iteration(sweeps: int = 2) -> float:
    """Algorithmic bytes of one V-cycle PCG iteration of the sparse atlas per
    level-0 cell (float32 level arrays, float64 CG vectors, byte labels; each
    array once per launch): the level-0 V-cycle (first colour from zero 13,
    each tiled smoother colour 15 (4 sweeps - 1 launches), residual 17,
    restriction 5, prolongation 9, input 13) and the CG kernels (z 13, r.z 17,
    direction 25, SpMV 21, update 49), times 8/7 for the coarser levels."""
    return (13 + (4 * sweeps - 1) * 15 + 17 + 5 + 9 + 13 + 13 + 17 + 25 + 21 + 49) * 8.0 / 7.0


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
    """The reference's CPU path (float64 Jacobi-PCG of the atlas oracle) on the headline
    workload, all host threads.  Each step solves a bounded sample of the 64 instances
    (step k solves instances 4k .. 4k+3 mod 64) and the metric counts solves."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    from fluid_b200 import configs
    from oracle.oracle import Oracle
    threads = os.cpu_count() or 1
    insts = configs.batch_instances(BATCH)
    per_step = 4
    times, iters = [], []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        for j in range(per_step):
            s = insts[(k * per_step + j) % BATCH]
            o = Oracle(s.nx, s.ny, s.nz, s.h, s.rho)
            o.set_threads(threads)
            o.set_state(s.vof, s.u, s.v, s.w, s.dt)
            _, info = o.solve_jacobi(1e-6, 0.0)
            iters.append(info["iterations"])
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(dt)
    tot = sum(times)
    value = per_step * len(times) / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "instances": BATCH, "cells": int(sum(s.cells for s in insts)),
                   "solver": "Jacobi-PCG float64 (atlas oracle), one instance after another"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port", "cpu_model": cpu_model(),
                         "sample": f"{per_step} of the 64 instances per step (rotating), full solves to rel-res "
                                   f"1e-6, mean {statistics.mean(iters):.0f} PCG iterations, OpenMP"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "p50_ms": 1000 * statistics.median(times) / per_step,
        "p99_ms": 1000 * float(np.percentile(times, 99)) / per_step,
    }
    print(json.dumps(line))
    return 0


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline_sample(insts):
    """The oracle's float64 Jacobi-PCG (the reference's CPU algorithm) on 4 of the 64
    headline instances: on all host threads (OpenMP, the reported value) and on one
    thread (the reference's own CPU path is single-threaded JavaScript)."""
    from oracle.oracle import Oracle
    threads = os.cpu_count() or 1

    def run(nthreads):
        t0 = time.perf_counter()
        its = []
        for s in insts[:4]:
            o = Oracle(s.nx, s.ny, s.nz, s.h, s.rho)
            o.set_threads(nthreads)
            o.set_state(s.vof, s.u, s.v, s.w, s.dt)
            _, info = o.solve_jacobi(1e-6, 0.0)
            its.append(int(info["iterations"]))
        return time.perf_counter() - t0, its
    dt, its = run(threads)
    dt1, _ = run(1)
    return {"value": 4 / dt, "unit": "solves/s", "cores": threads, "kind": "port", "cpu_model": cpu_model(),
            "sample": f"instances 0-3 of the 64 ({sum(s.cells for s in insts[:4])} cells), float64 Jacobi-PCG "
                      f"to rel-res 1e-6 ({its} iterations), OpenMP on the host",
            "single_thread": {"value": 4 / dt1, "unit": "solves/s", "cores": 1,
                              "sample": "the same 4 solves on one thread"}}


SEQ_STEPS = 50


def fp64_errors(states, steps, results: dict) -> dict:
    """Relative L2 error of each run's pressure (finest-cell units) against the
    float64 oracle's MGPCG solved to rel-res 1e-12 on the same input, per step."""
    from oracle.oracle import Oracle
    errs = {k: [] for k in results}
    for j in steps:
        st = states[j]
        o = Oracle(st.nx, st.ny, st.nz, st.h, st.rho, st.open_top)
        o.set_threads(os.cpu_count() or 1)
        o.set_state(st.vof, st.u, st.v, st.w, st.dt)
        p_ref, _ = o.solve_mgpcg(1e-12, 0.0, 300, 2, 2)
        nrm = float(np.linalg.norm(p_ref))
        for k, ps in results.items():
            errs[k].append(float(np.linalg.norm(ps[j] - p_ref)) / nrm)
    out = {"steps": list(steps), "oracle": "float64 MGPCG of the CPU oracle to rel-res 1e-12, same inputs"}
    for k, e in errs.items():
        out[k] = {"rel_l2_max": max(e), "rel_l2_median": statistics.median(e), "rel_l2": e}
    return out


def tall_fp64_error(tp, ts, pressures: dict) -> dict:
    """Relative L2 error of each timed tall-cell pressure against the float64
    solution of the oracle's independently assembled system (iterative
    refinement: float64 residuals with the oracle's operator, corrections from
    the device solver `tp`); outside the timed region."""
    from oracle import tall as toracle
    A, b = toracle.assemble_fp64(ts.nx, ts.fine_ny, ts.nz, ts.band, ts.bases, ts.vof, ts.u, ts.v, ts.w)
    tp.upload_state(ts.vof, ts.u, ts.v, ts.w)
    x = np.zeros_like(b)
    rel, steps = 1.0, 0
    for steps in range(12):
        r = b - A @ x
        rel = float(np.linalg.norm(r) / np.linalg.norm(b))
        if rel <= 1e-12:
            break
        e, _ = tp.solve_rhs(ts.dt, r.astype(np.float32), rel_tol=1e-6)
        x += e.ravel().astype(np.float64)
    out = {k: float(np.linalg.norm(p.ravel().astype(np.float64) - x) / np.linalg.norm(x))
           for k, p in pressures.items()}
    return {"rel_l2": out["plain_fp32"], "rel_l2_by_precision": out, "oracle_rel_residual": rel,
            "refinement_steps": steps,
            "oracle": "float64 tall-cell operator and rhs assembled by the CPU oracle from the dense faces; "
                      "solution by iterative refinement with device corrections"}


def note(msg: str):
    """Progress on stderr (stdout carries only the JSON line)."""
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def main():
    faulthandler.enable()
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp16", choices=["fp32", "fp16", "bf16"])
    ap.add_argument("--sweeps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=120.0,
                    help="length of the serving stream (single GPU only; 0 skips it)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)

    import torch

    from fluid_b200 import BatchProjector, PipelinedBatchProjector, PressureProjector, _abi, configs
    from fluid_b200.autotune import autotune_batch
    from fluid_b200.projector import kernel_launches

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    opts = dict(rel_tol=1e-6, pre_sweeps=args.sweeps, post_sweeps=args.sweeps)
    total = args.warmup + args.steps

    def max_over_ranks(ms):
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            return float(t.item())
        return ms

    def timed(fn):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        out = fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b), out

    # ------------------------------------------------------------ headline: batched
    note("generating the 64 instances")
    insts = configs.batch_instances(BATCH)
    cells = int(sum(s.cells for s in insts))
    dev = [tuple(torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (s.vof, s.u, s.v, s.w)) for s in insts]
    dts = [s.dt for s in insts]

    def make(precision):
        pps = [PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho, precision=precision, device=local) for s in insts]
        for p in pps:
            p.set_stream(stream.cuda_stream)
        return pps

    def upload_dev(pps):
        for p, d in zip(pps, dev):
            p.upload_state_device(*(t.data_ptr() for t in d))

    def run_batched(precision, steps, profile=False, tuning=None, o=None):
        o = opts if o is None else o
        pps = make(precision)
        B = BatchProjector(pps, tuning=tuning)
        B.set_profiling(profile)
        times, recs = [], None

        def step():
            upload_dev(pps)
            return B.project(dts, **o)
        for k in range(args.warmup + steps):
            ms, recs = timed(step)
            if k >= args.warmup:
                times.append(ms)
            if profile and k == args.warmup - 1:
                B.profile(reset=True)
        prof = B.profile(reset=True) if profile else None
        B.destroy()
        for p in pps:
            p.destroy()
        return times, recs, prof

    def run_single_sequence(precision, steps):
        pps = make(precision)
        times, recs = [], None

        def step():
            out = []
            for p, d, s in zip(pps, dev, insts):
                p.upload_state_device(*(t.data_ptr() for t in d))
                out.append(p.project(s.dt, **opts))
            return out
        for k in range(args.warmup + steps):
            ms, recs = timed(step)
            if k >= args.warmup:
                times.append(ms)
        for p in pps:
            p.destroy()
        return times, recs

    # the batch's layout and sweep schedule, measured on this batch before timing
    # (layouts never change results; fluid_b200.autotune)
    note("autotune")
    pps_t = make(args.precision)
    tune_failed = None
    try:
        tune = autotune_batch(pps_t, dts, lambda: upload_dev(pps_t), rel_tol=1e-6, repeats=2)
    except (RuntimeError, ValueError, MemoryError) as exc:
        # the library's default layout if tuning itself fails; a CUDA error that
        # left the context unusable surfaces here, not later in the timed region
        torch.cuda.synchronize()
        tune_failed = f"{type(exc).__name__}: {exc}"
        note(f"autotune failed ({tune_failed}); default layout")
        from fluid_b200.autotune import TuneResult
        from fluid_b200.projector import batch_tuning
        tune = TuneResult(batch_tuning().as_dict(), (args.sweeps, args.sweeps), None, None, [])
    for p in pps_t:
        p.destroy()
    tuned = dict(opts, pre_sweeps=tune.sweeps[0], post_sweeps=tune.sweeps[1])

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    l0 = kernel_launches()
    note("headline: batched mixed")
    with ClockSampler(local) as clk:
        times, recs, _ = run_batched(args.precision, args.steps, tuning=tune.tuning, o=tuned)
    torch.cuda.synchronize()
    launches = kernel_launches() - l0
    tot_ms = max_over_ranks(sum(times))
    value = world * BATCH * args.steps / (tot_ms / 1000.0)
    bad = [r for r in recs if r["status_name"] != "OK" or r["true_rel_residual"] > 1e-6]

    plain_steps = max(3, args.steps // 5)
    note("plain fp32 single-solve sequence")
    times_plain, _ = run_single_sequence("fp32", plain_steps)
    note("batched fp32")
    plain = BATCH * len(times_plain) / (sum(times_plain) / 1000.0)
    times_b32, _, _ = run_batched("fp32", plain_steps)
    batched32 = BATCH * len(times_b32) / (sum(times_b32) / 1000.0)

    # ------------------------------------------------ secondary: 128x96x128 single
    # 50 consecutive steps, whatever --steps is: each step's input is the
    # previous step's plain-FP32 projected velocity plus this step's gravity
    # (configs.dam_spheres_sequence); mixed and plain time the same 50 inputs,
    # and both are scored against the float64 oracle on every fifth step.
    steps2 = SEQ_STEPS
    note("128x96x128 consecutive inputs")
    s0 = configs.dam_spheres()
    seq_pp = PressureProjector((s0.nx, s0.ny, s0.nz), s0.h, s0.rho, precision="fp32", device=local)

    def carry(st):
        seq_pp.upload_state(st.vof, st.u, st.v, st.w)
        seq_pp.project(st.dt, **opts)
        _, u_, v_, w_ = seq_pp.download()
        return u_, v_, w_
    states = configs.dam_spheres_sequence(steps2, carry)
    seq_pp.destroy()
    nst = len(states)
    dev2 = [tuple(torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (s.vof, s.u, s.v, s.w)) for s in states]
    fp64_steps = list(range(0, nst, 5))

    def run_single(precision, profile=False, keep=(), o=None, nsteps=None):
        o = opts if o is None else o
        nsteps = steps2 if nsteps is None else nsteps
        pp = PressureProjector((s0.nx, s0.ny, s0.nz), s0.h, s0.rho, precision=precision, device=local)
        pp.set_stream(stream.cuda_stream)
        pp.set_profiling(profile)
        tt, rr, kept = [], [], {}
        for k in range(args.warmup + nsteps):
            j = (k - args.warmup) % nst   # warm-up steps replay the last inputs
            st, d2 = states[j], dev2[j]

            def step():
                pp.upload_state_device(*(t.data_ptr() for t in d2))
                return pp.project(st.dt, **o)
            ms, rec = timed(step)
            if k >= args.warmup:
                tt.append(ms)
                rr.append(rec)
                if j in keep:
                    kept[j] = pp.pressure_cells().astype(np.float64)
            if profile and k == args.warmup - 1:
                pp.profile(reset=True)
        prof = pp.profile(reset=True) if profile else None
        pp.destroy()
        return tt, rr, prof, kept

    t2_mixed, r2_mixed, _, p2_mixed = run_single(args.precision, keep=fp64_steps)
    t2_plain, r2_plain, _, p2_plain = run_single("fp32", keep=fp64_steps)
    # per-stage kernel events of the 128x96x128 solves (direct launches), reported per solve
    _, _, prof, _ = run_single(args.precision, profile=True)
    note("128x96x128 float64 oracle on every fifth step")
    fp64 = fp64_errors(states, fp64_steps, {"mixed": p2_mixed, "plain_fp32": p2_plain})

    # preconditioner choice: one V-cycle under PCG (the default) against one
    # full cycle under flexible CG, on the first CYCLE_STEPS inputs of the
    # 128x96x128 sequence and on the headline batch
    note("V-cycle vs full cycle")
    cycles = {}
    for cyc in ("v", "f"):
        tt, rr, _, _ = run_single(args.precision, o=dict(opts, cycle=cyc), nsteps=CYCLE_STEPS)
        tb, rb, _ = run_batched(args.precision, CYCLE_STEPS, tuning=tune.tuning, o=dict(tuned, cycle=cyc))
        cycles[cyc] = {
            "dam_spheres_128x96x128": {"solves_per_s": len(tt) / (sum(tt) / 1000.0),
                                       "iterations_mean": statistics.mean(r["iterations"] for r in rr),
                                       "failed_solves": sum(r["status_name"] != "OK" for r in rr)},
            "batch64": {"solves_per_s": BATCH * len(tb) / (sum(tb) / 1000.0),
                        "iterations_mean": statistics.mean(r["iterations"] for r in rb),
                        "failed_solves": sum(r["status_name"] != "OK" for r in rb)}}

    # roofline of the headline: per-stage kernel events of the batched solve
    # (direct launches of the same 64 solves).  A launch of a level-0 stage
    # touches every cell of every instance still iterating, so the stage's
    # algorithmic bytes over the solve are bytes/cell x sum(cells_i x iterations_i).
    note("headline per-stage events")
    prof_steps = 2
    _, brecs, bprof = run_batched(args.precision, prof_steps, profile=True, tuning=tune.tuning, o=tuned)
    sbytes = 4 if args.precision == "fp32" else 2
    cell_iters = prof_steps * sum(s_.cells * r["iterations"] for s_, r in zip(insts, brecs))
    stages = {k: v for k, v in bprof.items() if stage_bytes_per_cell(k, sbytes) > 0 and v["launches"] > 0}
    dom = max(stages, key=lambda k: stages[k]["ms"])
    per_launch_ms = bprof[dom]["ms"] / bprof[dom]["launches"]
    alg = stage_bytes_per_cell(dom, sbytes) * cell_iters / bprof[dom]["launches"]
    hbm, peak_kind = peaks()
    achieved = alg / (per_launch_ms / 1000.0) / 1e9
    tot_prof = sum(v["ms"] for v in bprof.values())
    # traffic of the average launch: the first-iteration capture times the share
    # of the batch's cells an average launch of the stage processes
    first = NCU_FIRST_LAUNCH_BYTES.get(dom)
    avg_cells = cell_iters / bprof[dom]["launches"]
    traffic = first * avg_cells / (cells * 1.0) if first else None
    stage_gbs = {k: round(stage_bytes_per_cell(k, sbytes) * cell_iters / (v["ms"] / 1000.0) / 1e9, 1)
                 for k, v in stages.items()}

    # The per-feature workloads (embedded solids, LCP, extrapolation, transport,
    # sparse atlas, tall cells) run at N = 1 only: under torchrun every rank
    # would repeat the same single-GPU measurement and its CPU oracle.
    def secondary_lines():
        # ------------------------------------ secondary: embedded solids (cut cells)
        note("embedded solids")
        sc = configs.solid_scene(*SOLID_DIMS)
        ss = sc.state
        dev4 = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (ss.vof, ss.u, ss.v, ss.w)]

        def run_solid(precision):
            pp_ = PressureProjector((ss.nx, ss.ny, ss.nz), ss.h, ss.rho, ss.open_top, precision, device=local)
            pp_.set_stream(stream.cuda_stream)
            pp_.upload_solids(*sc.solids())
            tt, rec_ = [], None

            def step():
                pp_.upload_state_device(*(t.data_ptr() for t in dev4))
                return pp_.project(ss.dt, **opts)
            for k in range(args.warmup + SOLID_STEPS):
                ms, rec_ = timed(step)
                if k >= args.warmup:
                    tt.append(ms)
            p_ = pp_.pressure_cells().astype(np.float64)
            pp_.destroy()
            return tt, rec_, p_
        t5, r5, p5 = run_solid("fp32")
        t5m, r5m, p5m = run_solid(args.precision)
        from oracle.oracle import Oracle
        o5 = Oracle(ss.nx, ss.ny, ss.nz, ss.h, ss.rho, ss.open_top)
        o5.set_threads(os.cpu_count() or 1)
        o5.set_state(ss.vof, ss.u, ss.v, ss.w, ss.dt)
        o5.set_solids(*sc.solids())
        p5_ref, _ = o5.solve_mgpcg(1e-12, 0.0, 400, 2, 2)
        nref = float(np.linalg.norm(p5_ref))
        solids_line = {
            "workload": sc.state.meta["workload"] + " (cell and dual-face open fractions by 8 samples, "
                        "the ball's velocity on its faces)",
            "cells": ss.cells, "steps": SOLID_STEPS,
            "plain_fp32_solves_per_s": len(t5) / (sum(t5) / 1000.0), "plain_p50_ms": statistics.median(t5),
            "mixed_solves_per_s": len(t5m) / (sum(t5m) / 1000.0), "mixed_p50_ms": statistics.median(t5m),
            "iterations": r5["iterations"], "mixed_iterations": r5m["iterations"],
            "status": [r5["status_name"], r5m["status_name"]],
            "max_div_ratio": r5["max_div_after"] / max(r5["max_div_before"], 1e-30),
            "fp64_error": {"plain_fp32": float(np.linalg.norm(p5 - p5_ref)) / nref,
                           "mixed": float(np.linalg.norm(p5m - p5_ref)) / nref,
                           "oracle": "float64 MGPCG of the CPU oracle with the same solids, rel-res 1e-12"},
            "kernels": "face-weighted per-pass V-cycle and CG kernels (the fused column kernels assume uniform weights)",
        }

        # ------------------------------------ secondary: the CM11a LCP variant
        note("LCP variant")
        lc = configs.solid_scene(*SOLID_DIMS, sphere_velocity=(0.0, -2.0, 0.0), ball=(0.25, 0.35, 0.5))
        ls = lc.state
        dev6 = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (ls.vof, ls.u, ls.v, ls.w)]
        lp = PressureProjector((ls.nx, ls.ny, ls.nz), ls.h, ls.rho, ls.open_top, args.precision, device=local)
        lp.set_stream(stream.cuda_stream)
        lp.upload_solids(*lc.solids())
        t6, r6 = [], None

        def lcp_step():
            lp.upload_state_device(*(t.data_ptr() for t in dev6))
            return lp.project_lcp(ls.dt)
        for k in range(args.warmup + SOLID_STEPS):
            ms, r6 = timed(lcp_step)
            if k >= args.warmup:
                t6.append(ms)
        x6 = lp.pressure_cells().astype(np.float64)
        lp.destroy()
        o6 = Oracle(ls.nx, ls.ny, ls.nz, ls.h, ls.rho, ls.open_top)
        o6.set_threads(os.cpu_count() or 1)
        o6.set_state(ls.vof, ls.u, ls.v, ls.w, ls.dt)
        o6.set_solids(*lc.solids())
        p6, i6 = o6.solve_lcp(3, 4)
        lab6 = o6.level(0)[0].astype(bool)
        solid6 = lab6 & (np.clip(lc.open, 0, 1) <= 1e-5)
        lcp_line = {
            "workload": ls.meta["workload"] + " with the ball inside the liquid moving down at 2 m/s (the bound active "
                        "on the solid cells the linear solve would pull)",
            "schedule": "3 full cycles + 4 V-cycles (the reference's), projected red-black smoother, 3 constrained levels",
            "solves_per_s": len(t6) / (sum(t6) / 1000.0), "p50_ms": statistics.median(t6),
            "projected_rel_residual": r6["true_rel_residual"], "rows_at_bound_oracle": i6["at_bound"],
            "min_pressure_on_solid_unknowns": float(x6[solid6].min()) if solid6.any() else None,
            "vs_fp64_oracle_schedule": float(np.linalg.norm(x6 - p6) / np.linalg.norm(p6)),
            "precision": f"{args.precision} coarse levels, f32 level 0, f64 coarsest sweeps",
        }

        # ------------------------------------ secondary: velocity extrapolation
        note("velocity extrapolation")
        from oracle import oracle as orc
        xs = configs.dam_spheres()
        xpp = PressureProjector((xs.nx, xs.ny, xs.nz), xs.h, xs.rho, xs.open_top, args.precision, device=local)
        xpp.set_stream(stream.cuda_stream)
        devx = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (xs.vof, xs.u, xs.v, xs.w)]
        xpp.upload_state_device(*(t.data_ptr() for t in devx))
        xpp.project(xs.dt, **opts)
        _, xu, xv, xw = xpp.download()   # the projected faces, the extrapolation's input
        devxp = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (xs.vof, xu, xv, xw)]
        t8 = []
        for k in range(args.warmup + TRANSPORT_STEPS):
            xpp.upload_state_device(*(t.data_ptr() for t in devxp))
            ms, filled8 = timed(lambda: xpp.extrapolate_velocity())
            if k >= args.warmup:
                t8.append(ms)
        _, eu, ev, ew = xpp.download()
        xpp.destroy()
        t_cpu8 = time.perf_counter()
        (ou, ov, ow), filled_o, _ = orc.extrapolate_velocity(xs.nx, xs.ny, xs.nz, xs.h, xs.open_top, xs.vof, xu, xv, xw)
        t_cpu8 = time.perf_counter() - t_cpu8
        extrap_line = {
            "workload": "the dam break + 16 spheres 128x96x128 step after its projection: FIM band of 2 cells, then "
                        "the known-value hierarchy fill",
            "cells": xs.cells, "steps": TRANSPORT_STEPS,
            "extrapolations_per_s": len(t8) / (sum(t8) / 1000.0), "p50_ms": statistics.median(t8),
            "filled_faces": int(filled8),
            "bit_exact_vs_oracle": bool(int(filled8) == int(filled_o)
                                        and all(np.array_equal(a.view(np.uint32), b.view(np.uint32))
                                                for a, b in ((eu, ou), (ev, ov), (ew, ow)))),
            "cpu_baseline": {"value": 1.0 / t_cpu8, "unit": "extrapolations/s", "cores": 1, "kind": "port",
                             "sample": "one extrapolation of the same faces by the oracle's float32 restatement"},
        }

        # ------------------------------------ secondary: CM12 density transport
        note("density transport")
        tsc = configs.transport_scene(*TRANSPORT_DIMS, seed=21, cells_per_step=2.5)
        devt = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (tsc.vof, tsc.u, tsc.v, tsc.w)]
        tpp = PressureProjector((tsc.nx, tsc.ny, tsc.nz), tsc.h, tsc.rho, tsc.open_top, device=local)
        tpp.set_stream(stream.cuda_stream)
        tpp.upload_state_device(*(t.data_ptr() for t in devt))
        tpp.set_gamma(None)
        tpp.transport_density(tsc.dt)
        rho_dev, g_dev = tpp.vof(), tpp.gamma()
        t_cpu = time.perf_counter()
        rho_orc, g_orc = orc.transport_density(tsc.nx, tsc.ny, tsc.nz, tsc.h, tsc.dt, tsc.open_top, tsc.vof, tsc.u, tsc.v,
                                               tsc.w)
        t_cpu = time.perf_counter() - t_cpu
        tr_exact = bool(np.array_equal(rho_dev.view(np.uint32), rho_orc.view(np.uint32))
                        and np.array_equal(g_dev.view(np.uint32), g_orc.view(np.uint32)))
        tpp.upload_state_device(*(t.data_ptr() for t in devt))
        tpp.set_gamma(None)
        t7, r7s = [], []
        for k in range(args.warmup + TRANSPORT_STEPS):
            ms, r7 = timed(lambda: tpp.transport_density(tsc.dt))
            if k >= args.warmup:
                t7.append(ms)
                r7s.append(r7)
        tpp.destroy()
        hbm7, kind7 = peaks()
        tr_bytes = transport_bytes_per_cell(1) * tsc.cells
        tr_gbs = tr_bytes / (statistics.mean(t7) / 1000.0) / 1e9
        transport_line = {
            "workload": tsc.meta["workload"] + ": dam block + ball, swirling face velocities on every open face "
                        "(an extrapolated field), fastest face 2.5 cells per step, dt 1/60, consecutive steps with "
                        "the persistent gamma carried",
            "cells": tsc.cells, "steps": TRANSPORT_STEPS,
            "steps_per_s": len(t7) / (sum(t7) / 1000.0), "p50_ms": statistics.median(t7),
            "p99_ms": float(np.percentile(t7, 99)),
            "cells_per_s": tsc.cells * len(t7) / (sum(t7) / 1000.0),
            "passes": "trace + beta, deficit scatter, gather, 3 gamma-diffusion passes, sharpening + mass return",
            "bit_exact_vs_oracle": tr_exact,
            "mass_drift_rel_over_steps": (r7s[-1]["mass_after"] - r7s[0]["mass_before"]) / r7s[0]["mass_before"],
            "roofline": {"bound": "hbm (formula); the traces are issue-bound", "alg_bytes_per_cell": transport_bytes_per_cell(1),
                         "achieved": round(tr_gbs, 1), "peak": hbm7, "unit": "GB/s", "frac": round(tr_gbs / hbm7, 4),
                         "peak_kind": kind7},
            "cpu_baseline": {"value": 1.0 / t_cpu, "unit": "steps/s", "cores": 1, "kind": "port",
                             "sample": "one step of the same lattice by the oracle's float32 restatement"},
        }

        # ------------------------------------ secondary: sparse brick atlas
        note("sparse brick atlas")
        from fluid_b200.atlas import AtlasProjector, bricks_from_dense
        asc = configs.atlas_scene(*ATLAS_DIMS, seed=11, drops=40)
        acoords = configs.atlas_bricks(asc.vof)
        adens, afaces = bricks_from_dense(asc.vof, asc.u, asc.v, asc.w, acoords)
        ap = AtlasProjector(ATLAS_DIMS, asc.h, asc.rho, device=local)
        ap.set_stream(stream.cuda_stream)
        atlas_runs = {}
        for cyc in ("v", "jacobi"):
            ta, ra = [], None
            for k in range(args.warmup + ATLAS_STEPS):
                ap.upload(acoords, adens, afaces)   # host planning and copies, outside the timed region
                ms, ra = timed(lambda: ap.project(asc.dt, cycle=cyc, rel_tol=1e-6, max_iters=4000))
                if k >= args.warmup:
                    ta.append(ms)
            atlas_runs[cyc] = {"solves_per_s": len(ta) / (sum(ta) / 1000.0), "p50_ms": statistics.median(ta),
                               "mean_ms": statistics.mean(ta),
                               "iterations": ra["iterations"], "status": ra["status_name"],
                               "true_rel_residual": ra["true_rel_residual"],
                               "max_div_ratio": ra["max_div_after"] / max(ra["max_div_before"], 1e-30)}
        ap.destroy()
        # float64 parity and the CPU baseline on the 128x96x128 atlas (the dense oracle on the embedding)
        asm = configs.atlas_scene(128, 96, 128, seed=11, drops=12)
        scoords = configs.atlas_bricks(asm.vof)
        sdens, sfaces = bricks_from_dense(asm.vof, asm.u, asm.v, asm.w, scoords)
        ap = AtlasProjector((128, 96, 128), asm.h, asm.rho, device=local)
        ap.set_stream(stream.cuda_stream)
        ap.upload(scoords, sdens, sfaces)
        ap.project(asm.dt, rel_tol=1e-6)
        ps, _ = ap.download()
        ap.destroy()
        from oracle.oracle import Oracle as _Oracle
        oa = _Oracle(128, 96, 128, asm.h, asm.rho)
        oa.set_threads(os.cpu_count() or 1)
        oa.set_state(asm.vof, asm.u, asm.v, asm.w, asm.dt)
        pa_ref, _ = oa.solve_mgpcg(1e-12, 0.0, 400, 2, 2)
        pa = np.zeros_like(pa_ref)
        for k, (bx, by, bz) in enumerate(scoords):
            pa[bz * 8:bz * 8 + 8, by * 8:by * 8 + 8, bx * 8:bx * 8 + 8] = ps[k] / (asm.rho * asm.h / asm.dt)
        t_cpu_a = time.perf_counter()
        _, ja = oa.solve_jacobi(1e-6, 0.0)
        t_cpu_a = time.perf_counter() - t_cpu_a
        hbm_a, kind_a = peaks()
        a_alg = atlas_bytes_per_cell_iteration() * len(acoords) * 512 * atlas_runs["v"]["iterations"]
        a_gbs = a_alg / (atlas_runs["v"]["mean_ms"] / 1000.0) / 1e9
        atlas_line = {
            "workload": asc.meta["workload"] + f": {len(acoords)} of {(ATLAS_DIMS[0] // 8) * (ATLAS_DIMS[1] // 8) * (ATLAS_DIMS[2] // 8)} "
                        "bricks (8^3 cells) present, Gaussian velocities sigma 0.2 on faces with a liquid side, rel-res 1e-6",
            "cells": len(acoords) * 512, "dense_equivalent_cells": int(np.prod(ATLAS_DIMS)), "steps": ATLAS_STEPS,
            "v_cycle": atlas_runs["v"], "jacobi": atlas_runs["jacobi"],
            "fp64_error_128x96x128": float(np.linalg.norm(pa - pa_ref) / np.linalg.norm(pa_ref)),
            "roofline": {"bound": "hbm", "scope": "whole V-cycle PCG solve (setup, receipts and projection included)",
                         "alg_bytes_per_cell_iteration": round(atlas_bytes_per_cell_iteration(), 1),
                         "achieved": round(a_gbs, 1), "peak": hbm_a, "unit": "GB/s", "frac": round(a_gbs / hbm_a, 4),
                         "peak_kind": kind_a},
            "cpu_baseline": {"value": 1.0 / t_cpu_a, "unit": "solves/s", "cores": os.cpu_count() or 1, "kind": "port",
                             "sample": f"the 128x96x128 atlas ({len(scoords)} bricks) as its dense embedding: the oracle's "
                                       f"float64 Jacobi-PCG (the reference's CPU algorithm) to rel-res 1e-6, "
                                       f"{int(ja['iterations'])} iterations, OpenMP"},
        }

        # ------------------------------------ secondary: tall-cell 256^2 columns x 1024 rows
        note("tall-cell waves")
        from fluid_b200.tall import TallProjector
        ts = configs.tall_waves()
        dev3 = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (ts.vof, ts.u, ts.v, ts.w)]
        steps3 = max(3, min(args.steps, 20))

        def run_tall(precision):
            tp_ = TallProjector(ts.nx, ts.nz, ts.fine_ny, ts.band, ts.bases, ts.h, ts.rho, precision=precision,
                                device=local)
            tp_.set_stream(stream.cuda_stream)
            tt, rec_ = [], None

            def tall_step():
                tp_.upload_state_device(*(t.data_ptr() for t in dev3))
                return tp_.project(ts.dt, rel_tol=1e-6)
            for k in range(args.warmup + steps3):
                ms, rec_ = timed(tall_step)
                if k >= args.warmup:
                    tt.append(ms)
            return tp_, tt, rec_
        tp, t3, r3 = run_tall("fp32")
        tpm, t3m, r3m = run_tall(args.precision)
        # solve-level roofline of the tall path: the formula's bytes of every CG
        # iteration over the whole solve time (setup and receipt included)
        from fluid_b200.tall import plan_tall_hierarchy
        tshapes = plan_tall_hierarchy(ts.nx, ts.nz, ts.fine_ny, ts.band, ts.bases)
        tsamples = [lx * lz * (lb + 2) for lx, _, lz, lb in tshapes]
        hbm3, kind3 = peaks()

        def tall_roofline(times, rec, storage):
            alg = tall_bytes_per_iteration(tsamples, storage, sweeps=2) * rec["iterations"]   # the default two sweeps
            gbs = alg / (statistics.mean(times) / 1000.0) / 1e9
            return {"bound": "hbm", "scope": "whole solve (all kernels, setup and receipt included)",
                    "algorithmic_bytes_per_solve": alg, "achieved": round(gbs, 1), "peak": hbm3,
                    "unit": "GB/s", "frac": round(gbs / hbm3, 4), "peak_kind": kind3}
        half = 4 if args.precision == "fp32" else 2
        roof3 = tall_roofline(t3, r3, [4] * len(tsamples))
        roof3m = tall_roofline(t3m, r3m, [4] + [half, half] + [4] * max(0, len(tsamples) - 3))
        p3m = tpm.pressure()
        tpm.destroy()
        note("tall-cell float64 oracle")
        tall_fp64 = tall_fp64_error(tp, ts, {"plain_fp32": tp.pressure(), "mixed": p3m})
        tp.destroy()
        tall_line = {
            "workload": ts.meta["workload"] + ", surface 600 + 8 seeded sinusoids (amplitude <= 12, wavelength 16-256)",
            "samples": ts.samples, "dense_equivalent_cells": ts.dense_cells, "steps": steps3,
            "solves_per_s": len(t3) / (sum(t3) / 1000.0), "p50_ms": statistics.median(t3),
            "p99_ms": float(np.percentile(t3, 99)), "iterations": r3["iterations"], "levels": r3["levels"],
            "status": r3["status_name"], "true_rel_residual": r3["true_rel_residual"],
            "sample_iterations_per_s": ts.samples * r3["iterations"] * len(t3) / (sum(t3) / 1000.0),
            "precision": "f32 levels, f32 CG vectors, f64 dots/scalars/coarsest",
            "mixed": {"precision": f"{args.precision} grid levels 1-2, f32 level 0 and block levels",
                      "solves_per_s": len(t3m) / (sum(t3m) / 1000.0), "p50_ms": statistics.median(t3m),
                      "iterations": r3m["iterations"], "status": r3m["status_name"],
                      "true_rel_residual": r3m["true_rel_residual"], "roofline": roof3m},
            "roofline": roof3,
            "level_samples": tsamples,
            "fp64_error": tall_fp64,
        }
        return {"embedded_solids_128x96x128": solids_line, "lcp_cm11a_128x96x128": lcp_line,
                "velocity_extrapolation_128x96x128": extrap_line, "density_transport_128x96x128": transport_line,
                "sparse_atlas_256x192x256": atlas_line, "tall_cell_256x256x1024": tall_line}

    if world == 1:
        sec = secondary_lines()
    else:
        sec = {k: {"skipped": "measured at N = 1 only (each rank would repeat the single-GPU workload)"}
               for k in ("embedded_solids_128x96x128", "lcp_cm11a_128x96x128", "velocity_extrapolation_128x96x128",
                         "density_transport_128x96x128", "sparse_atlas_256x192x256", "tall_cell_256x256x1024")}

    # ------------------------- serving: Poisson stream with continuous batching
    serving = None
    if world == 1 and args.serve_seconds > 0:
        note(f"serving stream ({args.serve_seconds:.0f} s)")
        from fluid_b200.serving import Server, serving_requests
        serve_s = float(args.serve_seconds)
        reqs = serving_requests(rate=40.0, duration_s=serve_s, seed=5)
        srv = Server(budget_bytes=150e9, precision=args.precision, device=local, max_resident_cells=SERVE_CELLS,
                     max_tall=SERVE_TALL)
        serving = srv.run(reqs, duration_s=serve_s)
        srv.shutdown()
        serving.update({
            "workload": f"Poisson arrivals at 40/s for {serve_s:.0f} s: 50/50 uniform grids (edges log-uniform "
                        "32-160 per axis, drawn per request) and tall-cell grids (64^2-256^2 columns, 24-40 band, "
                        "256 rows, drawn per request), 30-300 steps each, each from its own seeded initial state",
            "budget_bytes": 150e9, "max_resident_uniform_cells": SERVE_CELLS, "max_resident_tall": SERVE_TALL,
            "note": "admission: HBM budget (hard) and the step-latency budget (resident uniform cells, resident "
                    "tall simulations); the offered load (about 6600 step-solves/s, half of them tall) exceeds one "
                    "GPU, so requests queue: queue delay is reported beside step latency"})

    # ------------------------------------------- e2e: public API from host buffers
    note("e2e from host buffers")
    pps = make(args.precision)
    B = BatchProjector(pps, tuning=tune.tuning)
    host_in = [tuple(torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (s.vof, s.u, s.v, s.w))
               for s in insts]
    host_out = [tuple(torch.empty(sh, dtype=torch.float32).pin_memory()
                      for sh in ((s.nz, s.ny, s.nx), (s.nz, s.ny, s.nx + 1), (s.nz, s.ny + 1, s.nx),
                                 (s.nz + 1, s.ny, s.nx))) for s in insts]
    h2d = sum(t.numel() * 4 for tup in host_in for t in tup)
    d2h = sum(t.numel() * 4 for tup in host_out for t in tup)
    L = _abi.load()

    def e2e_step():
        for p, hi in zip(pps, host_in):
            p.upload_state(*(t.numpy() for t in hi))
        out = B.project(dts, **tuned)
        for p, ho in zip(pps, host_out):
            L.fluid_pp_download(p.handle, *(_abi.ptr(t.numpy()) for t in ho))
        return out
    e2e_ms = []
    for k in range(total):
        ms, _ = timed(e2e_step)
        if k >= args.warmup:
            e2e_ms.append(ms)
    B.destroy()
    for p in pps:
        p.destroy()
    e2e_serial = world * BATCH * len(e2e_ms) / (max_over_ranks(sum(e2e_ms)) / 1000.0)

    # the same ticks with three batches in flight on three streams: one batch's
    # uploads and read-back overlap the others' solves (PipelinedBatchProjector)
    note("e2e pipelined")
    depth = 3   # ticks in flight (4 measured slower: 4436 vs 5433 solves/s with 4-part batches)
    side = [torch.cuda.Stream() for _ in range(depth)]
    sets = []
    for st in side:
        ps_ = make(args.precision)
        for p in ps_:
            p.set_stream(st.cuda_stream)
        sets.append(ps_)
    outs = [host_out] + [[tuple(torch.empty_like(t).pin_memory() for t in tup) for tup in host_out]
                         for _ in range(depth - 1)]
    ins_np = [tuple(t.numpy() for t in tup) for tup in host_in]
    outs_np = [[tuple(t.numpy() for t in tup) for tup in o] for o in outs]
    pipe_bad = 0

    def pipe_ticks(n):
        nonlocal pipe_bad
        tickets = []
        for k in range(n):
            slot = k % depth
            if k >= depth:
                pipe_bad += sum(r["status"] != 0 for r in pipe.result(tickets[k - depth]))
            with torch.cuda.stream(side[slot]):
                flush.zero_()   # L2 flushed before every tick, on the tick's own stream
            tickets.append(pipe.submit(ins_np, outs_np[slot], dts, **tuned))
        for t in tickets[-depth:]:
            pipe_bad += sum(r["status"] != 0 for r in pipe.result(t))

    # parts per batch for the pipeline, measured here before timing: ticks in
    # flight already overlap one another's solves, so fewer parts than a lone
    # batch wants can be faster
    pipe_rates = {}
    for np_ in sorted({1, 2, int(tune.tuning["parts"])}):
        pipe = PipelinedBatchProjector(sets, tuning=dict(tune.tuning, parts=np_))
        pipe_ticks(depth)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pipe_ticks(3 * depth)
        torch.cuda.synchronize()
        pipe_rates[np_] = round(3 * depth * BATCH / (time.perf_counter() - t0), 1)
        pipe.destroy()
    pipe_parts = max(pipe_rates, key=lambda k: (pipe_rates[k], -k))
    pipe = PipelinedBatchProjector(sets, tuning=dict(tune.tuning, parts=pipe_parts))
    pipe_bad = 0
    pipe_ticks(args.warmup)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev0.record(side[0])
    for st in side[1:]:
        st.wait_event(ev0)
    pipe_ticks(args.steps)
    ends = [torch.cuda.Event(enable_timing=True) for _ in side]
    for e, st in zip(ends, side):
        e.record(st)
    torch.cuda.synchronize()
    pipe_ms = max(ev0.elapsed_time(e) for e in ends)
    pipe.destroy()
    for ps_ in sets:
        for p in ps_:
            p.destroy()
    e2e_value = world * BATCH * args.steps / (max_over_ranks(pipe_ms) / 1000.0)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        note("cpu baseline sample")
        cpu = cpu_baseline_sample(insts)

    its = [r["iterations"] for r in recs]
    cell_its = sum(s.cells * r["iterations"] for s, r in zip(insts, recs))
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "instances": BATCH, "cells": cells, "seed": 4,
                   "precision": f"{args.precision} V-cycle levels, f32 CG vectors, f64 dots/scalars/coarsest",
                   "sweeps": list(tune.sweeps), "tuning": tune.tuning,
                   "l2": "flushed before every timed step (256 MB write)",
                   "parallelism": f"{world} replicas" if world > 1 else "single GPU"},
        "p50_ms": statistics.median(times), "p99_ms": float(np.percentile(times, 99)),
        "iterations_min_max": [min(its), max(its)],
        "cell_iterations_per_s": world * cell_its * args.steps / (tot_ms / 1000.0),
        "plain_fp32_single_solves_per_s": plain,
        "plain_fp32_single_p50_ms_per_64": statistics.median(times_plain),
        "batched_fp32_solves_per_s": batched32,
        "mixed_batched_vs_plain_single": value / (world * plain),
        "failed_solves": len(bad),
        "autotune": {"failed": tune_failed, "candidates": len(tune.table), "chosen_ms": tune.ms,
                     "default_layout_ms": tune.default_ms,
                     "table": [[r["tuning"]["fill_tiles"], r["tuning"]["chunk_planes"], r["tuning"]["box_shape"],
                                r["tuning"]["parts"], list(r["sweeps"]), round(r["ms"], 3)] for r in tune.table],
                     "table_columns": ["fill_tiles", "chunk_planes", "box_shape", "parts", "sweeps", "median_ms"],
                     "note": "median solve of each candidate layout / sweep schedule on this batch before timing"},
        "dam_spheres_128x96x128": {
            "workload": WORKLOAD2, "steps": steps2,
            "sequence": "consecutive: each input is the previous step's projected velocity (plain FP32) plus "
                        "this step's gravity, spheres moved a quarter cell per step; mixed and plain time the "
                        "same inputs",
            "mixed_solves_per_s": len(t2_mixed) / (sum(t2_mixed) / 1000.0),
            "plain_fp32_solves_per_s": len(t2_plain) / (sum(t2_plain) / 1000.0),
            "mixed_p50_ms": statistics.median(t2_mixed), "mixed_p99_ms": float(np.percentile(t2_mixed, 99)),
            "plain_p50_ms": statistics.median(t2_plain), "plain_p99_ms": float(np.percentile(t2_plain, 99)),
            "iterations_mean": statistics.mean(r["iterations"] for r in r2_mixed),
            "plain_iterations_mean": statistics.mean(r["iterations"] for r in r2_plain),
            "failed_solves": sum(r["status_name"] != "OK" for r in r2_mixed + r2_plain),
            "fp64_error": fp64,
            "stage_ms_per_solve": {k: round(v["ms"] / steps2, 4) for k, v in sorted(prof.items())},
        },
        "preconditioner_cycles": {"steps": CYCLE_STEPS, "default": "v",
                                  "v": cycles["v"], "f": cycles["f"],
                                  "note": "v: one V-cycle under PCG (fused column kernels); f: one full cycle "
                                          "under flexible CG (per-pass kernels); same inputs, same tolerance"},
        **sec,
        "serving": serving,
        "roofline": {"bound": "hbm", "kernel": dom, "workload": "the headline batch (64 instances per launch)",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": peak_kind, "traffic": traffic, "alg_bytes_per_launch": alg,
                     "traffic_note": "ncu DRAM bytes of the first-iteration launch (all 64 instances) scaled by "
                                     "the cells of the average launch; alg_bytes_per_launch is that average launch",
                     "first_launch_traffic": first, "first_launch_alg_bytes": stage_bytes_per_cell(dom, sbytes) * cells,
                     "launch_ms": per_launch_ms, "share_of_step": bprof[dom]["ms"] / tot_prof,
                     "stage_gbs": stage_gbs,
                     "stage_ms_per_step": {k: round(v["ms"] / prof_steps, 4) for k, v in sorted(bprof.items())
                                           if v["launches"] > 0}},
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "PipelinedBatchProjector: each tick uploads the 64 inputs from pinned host memory, projects "
                        "and reads back p,u,v,w; three ticks in flight on three streams; timed over all ticks",
                "failed_solves": int(pipe_bad), "serial_solves_per_s": e2e_serial, "ticks_in_flight": depth,
                "parts_per_batch": pipe_parts, "parts_measured_solves_per_s": pipe_rates},
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
