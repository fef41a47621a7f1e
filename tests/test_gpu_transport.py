"""CM12 density transport on the device against the oracle's float32
restatement: bit for bit (GPU)."""
import numpy as np
import pytest

from fluid_b200 import PressureProjector, configs
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

SCENES = {
    "closed_48x40x44": lambda: configs.transport_scene(48, 40, 44, seed=5, cells_per_step=2.5),
    "open_top_37x30x26": lambda: configs.transport_scene(37, 30, 26, seed=9, cells_per_step=4.0, open_top=True),
    "fast_33x20x41": lambda: configs.transport_scene(33, 20, 41, seed=11, cells_per_step=12.0),
}
OPTIONS = {
    "default": {},
    "no_sharpening": {"sharpening": False},
    "no_mass_return": {"mass_return": False},
    "diffusion_3_strength_2": {"gamma_diffusion_iterations": 3, "strength": 2.0, "distance": 3.1},
    "no_diffusion": {"gamma_diffusion_iterations": 0},
}


def _oracle(s, gamma, o):
    return orc.transport_density(s.nx, s.ny, s.nz, s.h, s.dt, s.open_top, s.vof, s.u, s.v, s.w, gamma=gamma,
                                 diffusion=o.get("gamma_diffusion_iterations", 1),
                                 sharpening=o.get("sharpening", True), mass_return=o.get("mass_return", True),
                                 strength=o.get("strength", 1.0), distance=o.get("distance", 2.1))


def _handle(s):
    pp = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho, s.open_top)
    pp.upload_state(s.vof, s.u, s.v, s.w)
    return pp


@pytest.mark.parametrize("opt", sorted(OPTIONS))
@pytest.mark.parametrize("name", sorted(SCENES))
def test_transport_matches_oracle_bit_for_bit(name, opt):
    s = SCENES[name]()
    o = OPTIONS[opt]
    pp = _handle(s)
    rec = pp.transport_density(s.dt, **o)
    rho_o, g_o = _oracle(s, None, o)
    rho = pp.vof()
    np.testing.assert_array_equal(rho.view(np.uint32), rho_o.view(np.uint32))
    np.testing.assert_array_equal(pp.gamma().view(np.uint32), g_o.view(np.uint32))
    assert rec["mass_before"] == pytest.approx(float(np.sum(s.vof, dtype=np.float64)), rel=1e-12)
    assert rec["mass_after"] == pytest.approx(float(np.sum(rho_o, dtype=np.float64)), rel=1e-12)
    assert rec["rho_min"] == rho_o.min() and rec["rho_max"] == rho_o.max()
    pp.destroy()


def test_five_steps_with_persistent_gamma_then_projection():
    """Five transport steps (gamma carried by the handle) stay bit-identical to
    the oracle's, and the projection then runs on the transported density."""
    s = configs.transport_scene(40, 32, 36, seed=13, cells_per_step=3.0)
    pp = _handle(s)
    rho, g = s.vof, None
    for _ in range(5):
        pp.transport_density(s.dt)
        st = configs.GridState(s.nx, s.ny, s.nz, s.h, s.dt, rho, s.u, s.v, s.w)
        rho, g = _oracle(st, g, {})
        np.testing.assert_array_equal(pp.vof().view(np.uint32), rho.view(np.uint32))
        np.testing.assert_array_equal(pp.gamma().view(np.uint32), g.view(np.uint32))
    rec = pp.project(s.dt, rel_tol=1e-6)
    assert rec["status_name"] == "OK"
    pp.destroy()


def test_gamma_set_get_and_reset():
    s = configs.transport_scene(20, 18, 16, seed=3)
    pp = _handle(s)
    np.testing.assert_array_equal(pp.gamma(), np.ones((s.nz, s.ny, s.nx), np.float32))
    g = np.random.default_rng(1).uniform(0.5, 2.0, size=(s.nz, s.ny, s.nx)).astype(np.float32)
    pp.set_gamma(g)
    np.testing.assert_array_equal(pp.gamma(), g)
    pp.transport_density(s.dt)
    rho_o, g_o = _oracle(s, g, {})
    np.testing.assert_array_equal(pp.vof().view(np.uint32), rho_o.view(np.uint32))
    np.testing.assert_array_equal(pp.gamma().view(np.uint32), g_o.view(np.uint32))
    pp.set_gamma(None)
    np.testing.assert_array_equal(pp.gamma(), np.ones_like(g))
    pp.destroy()


def test_transport_rejects_embedded_solids_and_bad_dt():
    sc = configs.solid_scene(24, 20, 22, seed=3)
    s = sc.state
    pp = PressureProjector((s.nx, s.ny, s.nz), s.h, s.rho, s.open_top)
    pp.upload_solids(*sc.solids())
    pp.upload_state(s.vof, s.u, s.v, s.w)
    with pytest.raises(Exception, match="embedded solids"):
        pp.transport_density(s.dt)
    pp.destroy()
    t = configs.transport_scene(16, 14, 12, seed=2)
    pp = _handle(t)
    with pytest.raises(ValueError):
        pp.transport_density(0.0)
    pp.destroy()
