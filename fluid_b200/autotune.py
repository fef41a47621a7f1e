"""Measured choice of a batch's work layout and smoothing schedule.

A batch of uneven lattices can lay its V-cycle work out several ways: the box
kernels' tile shape, the z chunk of the column kernels' tiles, the tile count
a launch must reach before a larger shape or a longer chunk is used, and how
many concurrent parts (sub-batches on their own streams) the handles are split
into (``fluid_pp_batch_tuning``).  The library's default rule picks
from tile counts alone, with one part.  ``autotune_batch`` instead times the
candidates on the caller's own batch: the layouts with one part, then the best
of those split into 2-8 parts, then the other smoothing schedules (sweeps
down and up per V-cycle) with the fastest layout.

Layouts never change results: every layout applies the same arithmetic per
cell and folds the CG scalars over the same fixed tiles, so they give the same
bits.  A smoothing schedule changes the preconditioner, and hence iteration
counts and rounding; a schedule is kept only if every solve still converges.

The choice is cached per batch signature (lattice sizes, precision) in the
process, and in a JSON file when ``cache_path`` is given.
"""
from __future__ import annotations

import json
import os
import statistics
import time
from dataclasses import asdict, dataclass, field

from .projector import BatchProjector, batch_tuning

# fill_tiles: one (the default), two or four tiles per SM; chunk_planes: the
# default rule (0) or forced z chunks of the column kernels
LAYOUTS = tuple(dict(fill_tiles=f, chunk_planes=0, box_shape=-1, parts=1) for f in (148, 296, 592)) + tuple(
    dict(fill_tiles=148, chunk_planes=c, box_shape=-1, parts=1) for c in (16, 32, 64))
PARTS = (2, 3, 4, 6, 8)
SWEEPS = ((1, 1), (2, 2))


@dataclass
class TuneResult:
    tuning: dict                 # fields of fluid_pp_batch_tuning
    sweeps: tuple                # (pre, post) sweeps per V-cycle level
    ms: float                    # median solve time of the choice
    default_ms: float            # the library's default layout with 1 + 1 sweeps
    table: list = field(default_factory=list)   # every candidate measured: dict(tuning, sweeps, ms)


_cache: dict[str, TuneResult] = {}


def signature(projectors) -> str:
    """Key of a batch for the cache: its lattice sizes (in order) and precision."""
    dims = ",".join("x".join(str(v) for v in p.dims) for p in projectors)
    return f"{projectors[0].precision}:{dims}"


def pick(table) -> dict:
    """The fastest measured candidate (ties: the earliest); inf marks a failed one."""
    best = min(range(len(table)), key=lambda k: (table[k]["ms"], k))
    if table[best]["ms"] == float("inf"):
        raise RuntimeError("no candidate converged")
    return table[best]


def _load(cache_path):
    if not cache_path or not os.path.exists(cache_path):
        return {}
    with open(cache_path) as f:
        return json.load(f)


def autotune_batch(projectors, dts, restore, *, rel_tol=1e-6, layouts=LAYOUTS, parts=PARTS, sweeps=SWEEPS,
                   repeats=3, cache_path=None) -> TuneResult:
    """Time ``repeats`` solves (after one untimed) of each candidate on this batch.

    ``restore()`` must put every projector's step input back on the device (a
    solve projects the velocities in place); it runs before each solve, outside
    the timed span.  Returns the fastest layout and schedule.
    """
    key = signature(projectors)
    if key in _cache:
        return _cache[key]
    stored = _load(cache_path).get(key)
    if stored:
        res = TuneResult(stored["tuning"], tuple(stored["sweeps"]), stored["ms"], stored["default_ms"],
                         stored.get("table", []))
        _cache[key] = res
        return res

    def solve_ms(batch, pre, post):
        times = []
        for k in range(repeats + 1):
            restore()
            for p in projectors:
                p.synchronize()
            t0 = time.perf_counter()
            recs = batch.project(dts, rel_tol=rel_tol, pre_sweeps=pre, post_sweeps=post)
            dt = (time.perf_counter() - t0) * 1e3
            if any(r["status"] != 0 for r in recs):
                return float("inf")
            if k:
                times.append(dt)
        return statistics.median(times)

    table = []
    default = batch_tuning().as_dict()
    for lay in layouts:
        b = BatchProjector(projectors, tuning=lay)
        try:
            table.append(dict(tuning=dict(lay), sweeps=(1, 1), ms=solve_ms(b, 1, 1)))
        finally:
            b.destroy()
    if not any(row["tuning"] == default for row in table):
        b = BatchProjector(projectors)
        try:
            table.append(dict(tuning=default, sweeps=(1, 1), ms=solve_ms(b, 1, 1)))
        finally:
            b.destroy()
    best_layout = pick(table)["tuning"]
    for np_ in parts:
        if np_ < 2 or np_ > len(projectors):
            continue
        lay = dict(best_layout, parts=np_)
        b = BatchProjector(projectors, tuning=lay)
        try:
            table.append(dict(tuning=lay, sweeps=(1, 1), ms=solve_ms(b, 1, 1)))
        finally:
            b.destroy()
    best_layout = pick(table)["tuning"]
    for sw in sweeps:
        if tuple(sw) == (1, 1):
            continue
        b = BatchProjector(projectors, tuning=best_layout)
        try:
            table.append(dict(tuning=dict(best_layout), sweeps=tuple(sw), ms=solve_ms(b, *sw)))
        finally:
            b.destroy()
    best = pick(table)
    default_ms = next(row["ms"] for row in table if row["tuning"] == default and row["sweeps"] == (1, 1))
    res = TuneResult(dict(best["tuning"]), tuple(best["sweeps"]), best["ms"], default_ms, table)
    _cache[key] = res
    if cache_path:
        data = _load(cache_path)
        data[key] = asdict(res)
        with open(cache_path, "w") as f:
            json.dump(data, f, indent=1)
    return res
