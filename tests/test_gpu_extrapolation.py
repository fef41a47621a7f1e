"""Velocity extrapolation on the device against the oracle's float32
restatement, bit for bit (GPU)."""
import numpy as np
import pytest

from fluid_b200 import PressureProjector, configs
from oracle.oracle import extrapolate_velocity

pytestmark = pytest.mark.gpu

CASES = {
    "dam32": lambda: (configs.dam_break_32(), None),
    "odd37x50x29": lambda: (configs.random_small(37, 50, 29, seed=11), None),
    "open_top24": lambda: (configs.random_small(24, 24, 24, seed=13, open_top=True), None),
    "solids48x40x44": lambda: (lambda sc: (sc.state, sc))(configs.solid_scene(48, 40, 44, seed=3)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_extrapolation_matches_oracle_bit_for_bit(name):
    """After a projection (the call order of a step), the device's extrapolated
    faces equal the oracle's exactly, with the same count of filled faces."""
    s, sc = CASES[name]()
    pp = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho, s.open_top)
    if sc is not None:
        pp.upload_solids(*sc.solids())
    pp.upload_state(s.vof, s.u, s.v, s.w)
    assert pp.project(s.dt, rel_tol=1e-6)["status_name"] == "OK"
    _, u, v, w = pp.download()
    filled = pp.extrapolate_velocity()
    _, ue, ve, we = pp.download()
    extra = {} if sc is None else dict(open_frac=sc.open, fx=sc.fx, fy=sc.fy, fz=sc.fz)
    (uo, vo, wo), filled_o, ran = extrapolate_velocity(s.nx, s.ny, s.nz, s.h, s.open_top, s.vof, u, v, w, **extra)
    assert ran >= 1 and filled == filled_o
    for dev, ref in ((ue, uo), (ve, vo), (we, wo)):
        np.testing.assert_array_equal(dev.view(np.uint32), ref.view(np.uint32))
    pp.destroy()
