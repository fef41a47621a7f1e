"""Continuous-batching server: results alone and in the mix, admission by budget (GPU)."""
import numpy as np
import pytest

from fluid_b200 import configs
from fluid_b200.serving import Request, Server, required_bytes, serving_requests

pytestmark = pytest.mark.gpu


def _uniform(nx, ny, nz, seed):
    pair = []
    for step in range(2):
        vof = configs.random_liquid(nx, ny, nz, np.random.default_rng(seed))
        u, v, w = configs.velocities(vof, np.random.default_rng(seed + 17 * step), 1 / 60, "gauss", 0.2)
        pair.append(configs.GridState(nx, ny, nz, 1.0 / max(nx, ny, nz), 1 / 60, vof, u, v, w))
    return pair


def _tall(side, seed):
    s0 = configs.tall_waves(side, side, 96, 24, seed=seed, mean=50, amp_max=4, lam=(8, 32))
    s1 = configs.TallState(s0.nx, s0.nz, s0.fine_ny, s0.band, s0.bases, s0.h, s0.dt, s0.vof, -s0.u, -s0.v, -s0.w)
    return [s0, s1]


def _requests():
    return [Request(0, "uniform", _uniform(40, 28, 36, 1), 4, 0.0),
            Request(1, "tall", _tall(20, 2), 3, 0.0),
            Request(2, "uniform", _uniform(24, 50, 30, 3), 5, 0.0),
            Request(3, "uniform", _uniform(33, 33, 33, 4), 3, 0.0)]


def test_each_result_is_the_same_alone_and_in_the_mix():
    mix = Server(record=True)
    stats = mix.run(_requests())
    mix.shutdown()
    assert stats["requests_finished"] == 4 and stats["failed_steps"] == 0
    got = {s.req.rid: s.pressures for s in mix.done}
    for req in _requests():
        alone = Server(record=True)
        alone.run([req])
        alone.shutdown()
        (sim,) = alone.done
        assert len(sim.pressures) == req.steps == len(got[req.rid])
        for a, b in zip(sim.pressures, got[req.rid]):
            np.testing.assert_array_equal(a, b)


def test_admission_respects_the_budget():
    reqs = _requests()
    need = [required_bytes(r, "fp16") for r in reqs]
    budget = max(need) + min(need) // 2     # never two of the larger ones at once
    srv = Server(budget_bytes=budget)
    stats = srv.run(reqs)
    srv.shutdown()
    assert stats["requests_finished"] == 4
    assert srv.peak_used <= budget


def test_poisson_stream_short():
    reqs = serving_requests(rate=20.0, duration_s=1.5, seed=7, templates=2, steps=(3, 8), uniform_edge=(24, 64),
                            tall_side=(16, 32), tall_band=(24, 32), tall_rows=96)
    srv = Server(max_slots=16)
    stats = srv.run(reqs)
    srv.shutdown()
    assert stats["requests_finished"] == len(reqs)
    assert stats["failed_steps"] == 0
    assert stats["p99_step_ms"] is not None and stats["solves_per_s"] > 0


def test_per_request_shapes_and_latency_budgets():
    """Requests with their own seeded shapes, built by the background thread;
    admission keeps the resident uniform cells and tall simulations inside the
    latency budgets (one request alone may exceed the cell budget), and every
    admitted request reports its queue delay."""
    reqs = serving_requests(rate=30.0, duration_s=1.0, seed=9, steps=(3, 6), uniform_edge=(24, 56),
                            tall_side=(16, 40), tall_band=(24, 32), tall_rows=96)
    assert all(r.states is None for r in reqs)
    cap = 150_000
    srv = Server(max_resident_cells=cap, max_tall=1)
    stats = srv.run(reqs)
    srv.shutdown()
    assert stats["requests_finished"] == len(reqs) == stats["requests_admitted"]
    assert stats["failed_steps"] == 0
    biggest = max(r.meta["cells"] for r in reqs if r.kind == "uniform")
    assert stats["peak_resident_uniform_cells"] <= max(cap, biggest)
    assert stats["peak_resident_tall"] <= 1
    assert stats["p99_queue_delay_ms"] is not None and stats["p50_queue_delay_ms"] <= stats["p99_queue_delay_ms"]


def test_allocation_cache_carves_and_returns_reserved_memory():
    """Handles are carved from a reserved slab, give their ranges back on destroy,
    and a solve on reused memory is bit-identical to the first."""
    import ctypes
    from fluid_b200._abi import load
    from fluid_b200.projector import PressureProjector
    L = load()
    got = ctypes.c_ulonglong()
    assert L.fluid_pp_set_allocation_cache(0, ctypes.c_ulonglong(1 << 30)) == 0
    assert L.fluid_pp_reserve_allocation(0, ctypes.c_ulonglong(512 << 20)) == 0
    L.fluid_pp_allocation_cache_bytes(0, ctypes.byref(got))
    free0 = got.value
    assert free0 >= 512 << 20
    (s, _) = _uniform(40, 28, 36, 1)
    out = []
    for _ in range(2):
        p = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho, precision="fp16")
        L.fluid_pp_allocation_cache_bytes(0, ctypes.byref(got))
        assert got.value < free0          # the arena came from the slab
        p.upload_state(s.vof, s.u, s.v, s.w)
        assert p.project(s.dt, rel_tol=1e-6)["status_name"] == "OK"
        out.append(p.pressure_cells())
        p.destroy()
        L.fluid_pp_allocation_cache_bytes(0, ctypes.byref(got))
        assert got.value == free0         # every range coalesced back
    np.testing.assert_array_equal(out[0], out[1])
    assert L.fluid_pp_set_allocation_cache(0, ctypes.c_ulonglong(0)) == 0
    L.fluid_pp_allocation_cache_bytes(0, ctypes.byref(got))
    assert got.value == 0
