"""The serving stream's request generator (CPU): per-request seeded shapes."""
import numpy as np

from fluid_b200.serving import serving_requests


def test_requests_draw_their_own_shapes_and_build_states_on_demand():
    reqs = serving_requests(rate=40.0, duration_s=2.0, seed=5, tall_rows=96, tall_side=(16, 40))
    assert len(reqs) > 40
    kinds = {r.kind for r in reqs}
    assert kinds == {"uniform", "tall"}
    arrivals = [r.arrival for r in reqs]
    assert arrivals == sorted(arrivals) and arrivals[-1] < 2.0
    assert all(r.states is None and 30 <= r.steps <= 300 for r in reqs)
    dims = {r.meta["dims"] for r in reqs if r.kind == "uniform"}
    assert len(dims) > 10   # not a handful of templates
    assert all(32 <= e <= 160 for d in dims for e in d)
    u = next(r for r in reqs if r.kind == "uniform")
    t = next(r for r in reqs if r.kind == "tall")
    su, st = u.materialize(), t.materialize()
    assert (su[0].nx, su[0].ny, su[0].nz) == u.meta["dims"] and u.cells == np.prod(u.meta["dims"])
    assert st[0].nx == st[0].nz == t.meta["side"] and st[0].band == t.meta["band"]
    assert t.cells == st[0].samples == t.meta["cells"]
    # the same seed gives the same request and the same state
    again = serving_requests(rate=40.0, duration_s=2.0, seed=5, tall_rows=96, tall_side=(16, 40))
    u2 = next(r for r in again if r.rid == u.rid)
    np.testing.assert_array_equal(u2.materialize()[0].vof, su[0].vof)
