"""The CM11a LCP variant (projected multigrid, p >= 0 on solid unknowns) on the
device against the float64 oracle's restatement of the same schedule (GPU)."""
import numpy as np
import pytest

from fluid_b200 import PressureProjector, configs
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def _scene(velocity=(0.0, -2.0, 0.0), dims=(48, 40, 44)):
    """A ball moving inside the liquid: the linear solve wants negative
    pressure on some solid cells, so the bound is active there."""
    return configs.solid_scene(*dims, seed=3, sphere_velocity=velocity, ball=(0.25, 0.35, 0.5))


def _pair(sc, precision="fp32"):
    s = sc.state
    pp = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho, s.open_top, precision)
    pp.upload_solids(*sc.solids())
    pp.upload_state(s.vof, s.u, s.v, s.w)
    o = Oracle(s.nx, s.ny, s.nz, s.h, s.rho, s.open_top)
    o.set_state(s.vof, s.u, s.v, s.w, s.dt)
    o.set_solids(*sc.solids())
    return pp, o


def _solid_unknowns(sc, o):
    lab = o.level(0)[0].astype(bool)
    return lab & (np.clip(sc.open, 0, 1) <= 1e-5)


@pytest.mark.parametrize("velocity", [(0.0, -2.0, 0.0), (0.0, 3.0, 0.0)])
@pytest.mark.parametrize("cycles", [(3, 4), (3, 12)])
def test_lcp_matches_oracle_schedule(velocity, cycles):
    """The device runs the oracle's schedule: same pressure to rounding, the
    bound held exactly, the same projected residual."""
    sc = _scene(velocity)
    pp, o = _pair(sc)
    fc, vc = cycles
    rec = pp.project_lcp(sc.state.dt, full_cycles=fc, v_cycles=vc)
    assert rec["status_name"] == "OK" and rec["iterations"] == fc + vc
    p_o, info = o.solve_lcp(fc, vc)
    solid = _solid_unknowns(sc, o)
    x = pp.pressure_cells().astype(np.float64)
    assert info["at_bound"] > 0                       # the bound is active in this scene
    assert x[solid].min() >= 0.0                      # p >= p_min = 0 on every solid unknown
    assert np.linalg.norm(x - p_o) <= 1e-3 * np.linalg.norm(p_o)
    got = rec["true_rel_residual"] * rec["b_norm"]
    assert abs(got - info["l2_residual"]) <= 0.05 * info["l2_residual"] + 1e-6 * info["b_norm"]
    pp.destroy()


def test_lcp_more_cycles_reduce_the_projected_residual_and_half_levels_agree():
    sc = _scene()
    pp, _ = _pair(sc)
    r7 = pp.project_lcp(sc.state.dt)
    pp.upload_state(sc.state.vof, sc.state.u, sc.state.v, sc.state.w)
    r20 = pp.project_lcp(sc.state.dt, v_cycles=17)
    assert r20["true_rel_residual"] < r7["true_rel_residual"]
    x32 = pp.pressure_cells().astype(np.float64)
    pp.destroy()
    ph, _ = _pair(sc, "fp16")
    rh = ph.project_lcp(sc.state.dt, v_cycles=17)
    assert rh["status_name"] == "OK"
    xh = ph.pressure_cells().astype(np.float64)
    assert np.linalg.norm(xh - x32) <= 2e-2 * np.linalg.norm(x32)
    ph.destroy()


def test_lcp_without_an_active_bound_approaches_the_linear_solution():
    """With the ball outside the liquid no bound is active, and the projected
    multigrid converges to the linear system's solution."""
    sc = configs.solid_scene(40, 32, 36, seed=4)
    pp, o = _pair(sc)
    rec = pp.project_lcp(sc.state.dt, full_cycles=3, v_cycles=60)
    assert rec["status_name"] == "OK"
    p_ref, info = o.solve_mgpcg(1e-12, 0.0, 400, 2, 2)
    assert info["converged"] == 1.0
    x = pp.pressure_cells().astype(np.float64)
    assert np.linalg.norm(x - p_ref) <= 1e-3 * np.linalg.norm(p_ref)
    pp.destroy()


def test_lcp_needs_embedded_solids():
    s = configs.dam_break_32()
    pp = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho)
    pp.upload_state(s.vof, s.u, s.v, s.w)
    with pytest.raises(ValueError, match="embedded solids"):
        pp.project_lcp(s.dt)
    pp.destroy()
