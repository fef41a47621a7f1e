"""Continuous-batching projection server: many resident simulations on one GPU.

Stands where the reference's per-simulation advance loop stands
(``GPUSolverInstance.advanceTo``, lib/core/method-contract.ts:355, driven per
simulation from the render worker): every admitted simulation keeps its
state, hierarchy and CG workspace resident on the device and advances one
projection step after another.

One host thread drives the device and interleaves two kinds of work: a
batched step of every resident uniform simulation (one launch per kernel
stage across all of them, ``fluid_pp_batch_project``), then a slice of at
most ``tall_slice_iterations`` CG iterations of the current tall-cell solve
(``fluid_pp_tall_project_begin/continue/end``; the tall-cell simulations take
their steps in round-robin order), or, in a round that admits a request, the
admission instead; then the next batched uniform step, and so on.  A uniform
step therefore waits for at most one slice or one admission, however many
tall-cell simulations are resident, and every resident simulation keeps
advancing.  Between steps, finished
simulations leave (their device blocks go to the library's allocation cache,
``fluid_pp_set_allocation_cache``, since cudaFree of a large arena can take
longer than many steps) and queued requests are admitted FIFO by an HBM budget
(``fluid_pp_required_bytes`` / ``fluid_pp_tall_required_bytes`` plus the
resident state) and a slot limit, at most ``admit_per_step`` at a time.

Step latency is wall time from the moment a step is ready (the simulation's
previous step finished, or its admission) to the moment its projection has
finished, as a client of the server would see it.
"""
from __future__ import annotations

import ctypes
import math
import statistics
import threading
import time
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

from . import _abi, configs
from ._abi import Config, TallConfig, load
from .projector import BatchProjector, PressureProjector
from .tall import TallProjector


@dataclass
class Request:
    rid: int
    kind: str                  # "uniform" | "tall"
    states: Optional[list]     # states the steps cycle through (configs.GridState / TallState), or None until made
    steps: int
    arrival: float             # seconds after the start of the run
    meta: dict = field(default_factory=dict)
    make: Optional[Callable[[], list]] = None   # builds `states` (the request's own seeded initial state)

    def materialize(self):
        if self.states is None:
            self.states = self.make()
        return self.states

    @property
    def ready(self) -> bool:
        return self.states is not None

    @property
    def cells(self) -> int:
        if self.states is None:
            return int(self.meta.get("cells", 0))
        s = self.states[0]
        return s.cells if self.kind == "uniform" else s.samples


def required_bytes(req: Request, precision: str) -> int:
    """Device bytes the request holds while resident (handle + its state copies)."""
    s = req.states[0]
    out = ctypes.c_ulonglong()
    L = load()
    if req.kind == "uniform":
        cfg = Config(s.nx, s.ny, s.nz, float(s.h), float(s.rho), int(s.open_top), _abi.PRECISIONS[precision], 0)
        rc = L.fluid_pp_required_bytes(ctypes.byref(cfg), ctypes.byref(out))
        state = 4 * (s.cells + (s.nx + 1) * s.ny * s.nz + s.nx * (s.ny + 1) * s.nz + s.nx * s.ny * (s.nz + 1))
    else:
        cfg = TallConfig(s.nx, s.nz, s.fine_ny, s.band, float(s.h), float(s.rho), _abi.PRECISIONS[precision], 0)
        b = np.ascontiguousarray(s.bases.ravel(), np.int32)
        rc = L.fluid_pp_tall_required_bytes(ctypes.byref(cfg), _abi.ptr(b), ctypes.byref(out))
        state = 4 * 4 * s.samples
    if rc != _abi.OK:
        raise ValueError(L.fluid_pp_last_error(None).decode())
    return int(out.value) + state * len(req.states)


class _Sim:
    def __init__(self, req: Request, precision: str, device: int, stream, copy_stream, torch):
        self.req = req
        self.kind = req.kind
        s = req.states[0]
        if req.kind == "uniform":
            self.h = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho, s.open_top, precision, device)
        else:
            self.h = TallProjector(s.nx, s.nz, s.fine_ny, s.band, s.bases, s.h, s.rho, precision, device)
        self.h.set_stream(stream.cuda_stream)
        with torch.cuda.stream(copy_stream):
            self.dev = [tuple(torch.from_numpy(np.ascontiguousarray(a)).to(f"cuda:{device}", non_blocking=False)
                              for a in (st.vof, st.u, st.v, st.w)) for st in req.states]
        copy_stream.synchronize()   # the states are complete before another stream reads them
        self.step = 0
        self.ready = 0.0
        self.bytes = 0
        self.latencies: list[float] = []
        self.receipts: list[dict] = []
        self.pressures: list[np.ndarray] = []

    def upload(self):
        d = self.dev[self.step % len(self.dev)]
        self.h.upload_state_device(*(t.data_ptr() for t in d))

    @property
    def dt(self) -> float:
        return self.req.states[self.step % len(self.req.states)].dt

    def destroy(self):
        self.h.destroy()
        self.dev = None


class Server:
    """Admits requests by HBM budget and advances every resident simulation,
    interleaving batched uniform steps with single tall-cell steps (continuous
    batching).

    Admission: a request is admitted when its device bytes fit the HBM budget
    (``budget_bytes``, the hard limit) and the resident work stays inside the
    step-latency budget: at most ``max_resident_cells`` uniform cells in the
    batched step (its duration grows with the cells it solves) and at most
    ``max_tall`` tall-cell simulations (they share the tall slices round-robin,
    so each one's step waits for the others').  Requests of each kind are
    admitted in arrival order; a kind whose latency budget is full does not
    hold back the other.  Each request's initial state is built from its seed
    by a background thread a few requests ahead of admission."""

    def __init__(self, budget_bytes: float = 150e9, max_slots: int = 256, precision: str = "fp16", device: int = 0,
                 rel_tol: float = 1e-6, record: bool = False, admit_per_step: int = 1,
                 cache_bytes: float = 16e9, reserve_bytes: float = 4e9, tall_slice_iterations: int = 3,
                 max_resident_cells: float = float("inf"), max_tall: int = 1 << 30, prefetch: int = 6):
        import torch
        self.torch = torch
        self.budget = float(budget_bytes)
        self.max_slots = int(max_slots)
        self.precision = precision
        self.device = int(device)
        self.rel_tol = float(rel_tol)
        self.record = record
        self.admit_per_step = int(admit_per_step)
        torch.cuda.set_device(self.device)
        self.stream = torch.cuda.Stream(device=self.device)
        # handles come and go every few steps: keep their blocks for reuse
        # instead of cudaFree / cudaFreeHost, which take up to ~1 s for large arenas
        self.L = load()
        self.cache_bytes = int(cache_bytes)
        self.L.fluid_pp_set_allocation_cache(self.device, ctypes.c_ulonglong(self.cache_bytes))
        self.L.fluid_pp_set_allocation_cache(-1, ctypes.c_ulonglong(min(self.cache_bytes, 256 << 20)))
        # memory mapped before the first admission: handles are carved from a
        # reserved slab, and torch's pool (the state copies) is warmed the same way
        have = ctypes.c_ulonglong()
        self.L.fluid_pp_allocation_cache_bytes(self.device, ctypes.byref(have))
        if reserve_bytes > have.value:   # top up what the cache already holds free
            self.L.fluid_pp_reserve_allocation(self.device, ctypes.c_ulonglong(int(reserve_bytes) - have.value))
            warm = torch.empty(int(reserve_bytes) // 4, dtype=torch.uint8, device=f"cuda:{self.device}")
            del warm
        self.pending: list[tuple[Request, int]] = []
        self.active: list[_Sim] = []
        self.done: list[_Sim] = []
        self.used = 0.0
        self.peak_used = 0.0
        self.batch_sizes: list[int] = []
        self.uniform_steps = 0
        self.tall_steps = 0
        self._batch = None
        self._members: list[_Sim] = []
        self._next_tall = 0
        self._tall_cur = None            # the tall-cell simulation whose solve is in progress
        self.tall_slice = int(tall_slice_iterations)
        self.max_cells = float(max_resident_cells)
        self.max_tall = int(max_tall)
        self.queue_delays: list[float] = []
        self.peak_uniform_cells = 0
        self.peak_tall = 0
        # background construction of the queued requests' initial states
        self.prefetch = int(prefetch)
        self._lock = threading.Lock()
        self._stop = threading.Event()
        self._gen_error: Optional[BaseException] = None
        self._gen = threading.Thread(target=self._generate, name="serving-states", daemon=True)
        self._gen.start()

    # -- request states (background thread) ------------------------------------------
    def _generate(self):
        """Builds the states of the first `prefetch` queued requests of each kind
        that have none yet, oldest first."""
        while not self._stop.is_set():
            with self._lock:
                todo = []
                for kind in ("uniform", "tall"):
                    todo += [r for r, _ in [p for p in self.pending if p[0].kind == kind][:self.prefetch]
                             if not r.ready]
            if not todo:
                self._stop.wait(0.002)
                continue
            try:
                min(todo, key=lambda r: r.arrival).materialize()
            except BaseException as exc:   # surfaced by the serving loop
                self._gen_error = exc
                return

    # -- admission and retirement (between steps) ----------------------------------
    def submit(self, req: Request):
        with self._lock:
            self.pending.append([req, None])

    def _fits(self, req: Request) -> bool:
        """Latency budget of the request's kind (an empty server always admits)."""
        kind = [s for s in self.active if s.kind == req.kind]
        if not kind:
            return True
        if req.kind == "tall":
            return len(kind) < self.max_tall
        return sum(s.req.cells for s in kind) + req.cells <= self.max_cells

    def _admit(self, now: float) -> int:
        if self._gen_error is not None:
            raise RuntimeError("building a request's state failed") from self._gen_error
        admitted = 0
        blocked = set()   # kinds whose oldest queued request cannot be admitted now
        while len(self.active) < self.max_slots and admitted < self.admit_per_step:
            with self._lock:
                heads = {}
                for p in self.pending:
                    if p[0].kind not in heads and p[0].kind not in blocked:
                        heads[p[0].kind] = p
                if not heads:
                    break
                entry = min(heads.values(), key=lambda p: p[0].arrival)
            req = entry[0]
            if not req.ready or not self._fits(req):
                blocked.add(req.kind)
                continue
            if entry[1] is None:
                entry[1] = required_bytes(req, self.precision)
            need = entry[1]
            if self.used + need > self.budget:
                if not self.active and need > self.budget:
                    raise MemoryError(f"request {req.rid} needs {need} bytes, over the whole budget")
                blocked.add(req.kind)
                continue
            with self._lock:
                self.pending = [p for p in self.pending if p is not entry]
            sim = _Sim(req, self.precision, self.device, self.stream, self.stream, self.torch)
            sim.bytes = need
            sim.ready = now
            self.queue_delays.append(max(0.0, now - req.arrival))
            self.used += need
            self.peak_used = max(self.peak_used, self.used)
            self.active.append(sim)
            self.peak_uniform_cells = max(self.peak_uniform_cells,
                                          sum(s.req.cells for s in self.active if s.kind == "uniform"))
            self.peak_tall = max(self.peak_tall, sum(1 for s in self.active if s.kind == "tall"))
            admitted += 1
        return admitted

    def _retire(self):
        leaving = [s for s in self.active if s.step >= s.req.steps]
        if not leaving:
            return
        if self._batch is not None and any(s in self._members for s in leaving):
            self._batch.destroy()
            self._batch, self._members = None, []
        for s in leaving:
            self.active.remove(s)
            self.used -= s.bytes
            s.destroy()
            s.req.states = None   # the host copies of a finished request are no longer needed
            self.done.append(s)

    def _record(self, sim: _Sim, receipt: dict, t: float):
        sim.receipts.append(receipt)
        sim.latencies.append(t - sim.ready)
        if self.record:
            sim.pressures.append(sim.h.pressure_cells() if sim.kind == "uniform" else sim.h.pressure())
        sim.ready = t
        sim.step += 1

    # -- steps ----------------------------------------------------------------------
    def _uniform_step(self, members: list[_Sim], clock):
        if [id(s) for s in members] != [id(s) for s in self._members]:
            if self._batch is not None:
                self._batch.destroy()
            self._batch = BatchProjector([s.h for s in members])
            self._batch.set_graphs(False)   # membership changes every few steps: direct launches
            self._members = list(members)
        for s in members:
            s.upload()
        recs = self._batch.project([s.dt for s in members], rel_tol=self.rel_tol)
        t = clock()
        for s, r in zip(members, recs):
            self._record(s, r, t)
        self.batch_sizes.append(len(members))
        self.uniform_steps += 1

    def _tall_slice(self, clock):
        """At most tall_slice iterations of the current tall-cell solve; a new
        solve (upload, assembly, CG start) begins with the next simulation in
        round-robin order when none is in progress."""
        sim = self._tall_cur
        if sim is None:
            tall = [s for s in self.active if s.kind == "tall"]
            self._next_tall %= len(tall)
            sim = tall[self._next_tall]
            self._next_tall += 1
            sim.upload()
            sim.h.project_begin(sim.dt, rel_tol=self.rel_tol)
            self._tall_cur = sim
        if sim.h.project_continue(self.tall_slice):
            r = sim.h.project_end()
            self._record(sim, r, clock())
            self.tall_steps += 1
            self._tall_cur = None

    def _round(self, clock, admitted: bool):
        """One batched uniform step (if any uniform simulation is resident), then
        one slice of a tall-cell solve unless this round admitted a request: an
        admission takes the slice's place between two uniform steps instead of
        adding to the gap."""
        uni = [s for s in self.active if s.kind == "uniform"]
        if uni:
            self._uniform_step(uni, clock)
        if any(s.kind == "tall" for s in self.active) and not (admitted and uni):
            self._tall_slice(clock)

    # -- the loop -------------------------------------------------------------------
    def run(self, requests: list[Request], duration_s: float | None = None) -> dict:
        """Feeds requests at their arrival times (wall clock) and runs rounds until
        every request finished, or until duration_s (then the run stops after the round)."""
        queue = sorted(requests, key=lambda r: r.arrival)
        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0
        i = 0
        while True:
            now = clock()
            while i < len(queue) and queue[i].arrival <= now:
                self.submit(queue[i])
                i += 1
            admitted = self._admit(now)
            if self.active:
                self._round(clock, admitted > 0)
                self._retire()
            elif i < len(queue):
                time.sleep(max(0.0, min(0.005, queue[i].arrival - clock())))
            elif not self.pending:
                break
            else:
                time.sleep(0.001)   # queued requests whose states are still being built
            if duration_s is not None and clock() >= duration_s:
                break
        if self._batch is not None:
            self._batch.destroy()
            self._batch, self._members = None, []
        elapsed = clock()
        sims = self.done + self.active
        lat = [x for s in sims for x in s.latencies]
        big = [x for s in sims if s.req.cells >= 1_200_000 for x in s.latencies]
        big_u = [x for s in sims if s.kind == "uniform" and s.req.cells >= 1_200_000 for x in s.latencies]
        lat_u = [x for s in sims if s.kind == "uniform" for x in s.latencies]
        lat_t = [x for s in sims if s.kind == "tall" for x in s.latencies]
        pct = lambda xs, q: 1000 * float(np.percentile(xs, q)) if xs else None
        cell_steps = sum(s.req.cells * len(s.latencies) for s in sims)
        out = {
            "elapsed_s": elapsed, "requests_submitted": i, "requests_finished": len(self.done),
            "requests_resident_at_end": len(self.active), "requests_waiting_at_end": len(self.pending),
            "step_solves": len(lat), "solves_per_s": len(lat) / elapsed if elapsed > 0 else 0.0,
            "p50_step_ms": pct(lat, 50), "p99_step_ms": pct(lat, 99),
            "p50_step_ms_ge_1p2M_cells": pct(big, 50), "p99_step_ms_ge_1p2M_cells": pct(big, 99),
            "steps_ge_1p2M_cells": len(big),
            "p99_uniform_step_ms_ge_1p2M_cells": pct(big_u, 99),
            "p50_uniform_step_ms": pct(lat_u, 50), "p99_uniform_step_ms": pct(lat_u, 99),
            "p50_tall_step_ms": pct(lat_t, 50), "p99_tall_step_ms": pct(lat_t, 99),
            "requests_admitted": len(self.queue_delays),
            "p50_queue_delay_ms": pct(self.queue_delays, 50), "p99_queue_delay_ms": pct(self.queue_delays, 99),
            "cell_steps_per_s": cell_steps / elapsed if elapsed > 0 else 0.0,
            "uniform_batched_steps": self.uniform_steps, "tall_steps": self.tall_steps,
            "mean_uniform_batch": statistics.mean(self.batch_sizes) if self.batch_sizes else 0.0,
            "peak_resident_bytes": self.peak_used,
            "peak_resident_uniform_cells": self.peak_uniform_cells, "peak_resident_tall": self.peak_tall,
            "failed_steps": sum(1 for s in sims for r in s.receipts if r["status_name"] != "OK"),
        }
        return out

    def shutdown(self):
        """Destroys the resident simulations and frees the allocation cache."""
        self._stop.set()
        self._gen.join()
        if self._batch is not None:
            self._batch.destroy()
            self._batch, self._members = None, []
        for s in self.active:
            s.destroy()
        self.active = []
        self.L.fluid_pp_set_allocation_cache(self.device, ctypes.c_ulonglong(0))
        self.L.fluid_pp_set_allocation_cache(-1, ctypes.c_ulonglong(0))


def _uniform_states(nx, ny, nz, seed) -> list:
    """A uniform request's two states: seeded liquid boxes/spheres and two
    draws of Gaussian velocities (the steps alternate between them)."""
    vof = configs.random_liquid(nx, ny, nz, np.random.default_rng(seed))
    out = []
    for step in range(2):
        u, v, w = configs.velocities(vof, np.random.default_rng(seed + 17 * (step + 1)), 1 / 60, "gauss", 0.2)
        out.append(configs.GridState(nx, ny, nz, 1.0 / max(nx, ny, nz), 1 / 60, vof, u, v, w))
    return out


def _tall_states(side, band, rows, seed) -> list:
    """A tall-cell request's two states: a seeded wave tank and the same layout
    (bases are fixed per handle) with redrawn velocities."""
    s0 = configs.tall_waves(side, side, rows, band, seed=seed, mean=0.6 * rows, amp_max=8)
    vrng = np.random.default_rng(seed + 17)
    redraw = lambda a: np.where(a != 0, vrng.normal(0.0, 0.1, a.shape), 0.0).astype(np.float32)
    s1 = configs.TallState(s0.nx, s0.nz, s0.fine_ny, s0.band, s0.bases, s0.h, s0.dt, s0.vof, redraw(s0.u),
                           redraw(s0.v), redraw(s0.w), meta=dict(s0.meta))
    return [s0, s1]


def serving_requests(rate: float = 40.0, duration_s: float = 120.0, seed: int = 5, templates: int = 0,
                     steps=(30, 300), uniform_edge=(32, 160), tall_side=(64, 256), tall_band=(24, 40),
                     tall_rows: int = 256, pin_1p2m: bool = False) -> list[Request]:
    """Poisson arrivals (rate per second) over duration_s: 50/50 a uniform grid
    (edges log-uniform in uniform_edge per axis) or a tall-cell grid (columns
    log-uniform side in tall_side, band uniform in tall_band), each for a seeded
    number of steps from its own seeded initial state (dam-break-like liquid
    boxes and spheres, or a wave tank), built when the request nears admission.
    With templates > 0 the requests share that many seeded shapes of each kind
    instead (states built up front); with pin_1p2m the first uniform template is
    a 1.2M-cell grid."""
    rng = np.random.default_rng(seed)
    uni_t, tall_t = [], []
    for k in range(templates):
        nx, ny, nz = (configs.log_uniform_edge(rng, *uniform_edge) for _ in range(3))
        if k == 0 and pin_1p2m:
            nx, ny, nz = 112, 96, 112   # 1,204,224 cells: the size the latency target names
        uni_t.append(_uniform_states(nx, ny, nz, seed * 1000 + k))
        side = int(round(math.exp(rng.uniform(math.log(tall_side[0]), math.log(tall_side[1])))))
        band = int(rng.integers(tall_band[0], tall_band[1] + 1))
        tall_t.append(_tall_states(side, band, tall_rows, seed * 1000 + k))
    out, t, rid = [], 0.0, 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration_s:
            break
        kind = "uniform" if rng.random() < 0.5 else "tall"
        nsteps = int(rng.integers(steps[0], steps[1] + 1))
        if templates:
            tpl = (uni_t if kind == "uniform" else tall_t)[int(rng.integers(0, templates))]
            out.append(Request(rid, kind, tpl, nsteps, t))
        elif kind == "uniform":
            nx, ny, nz = (configs.log_uniform_edge(rng, *uniform_edge) for _ in range(3))
            rs = seed * 100003 + rid
            out.append(Request(rid, kind, None, nsteps, t, meta={"dims": (nx, ny, nz), "cells": nx * ny * nz},
                               make=lambda nx=nx, ny=ny, nz=nz, rs=rs: _uniform_states(nx, ny, nz, rs)))
        else:
            side = int(round(math.exp(rng.uniform(math.log(tall_side[0]), math.log(tall_side[1])))))
            band = int(rng.integers(tall_band[0], tall_band[1] + 1))
            rs = seed * 100003 + rid
            out.append(Request(rid, kind, None, nsteps, t,
                               meta={"side": side, "band": band, "cells": side * side * (band + 2)},
                               make=lambda side=side, band=band, rs=rs: _tall_states(side, band, tall_rows, rs)))
        rid += 1
    return out
