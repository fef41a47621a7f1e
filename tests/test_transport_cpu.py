"""The CM12 density transport restatement of the oracle (float32): properties
the step must have, on the CPU."""
import numpy as np

from fluid_b200 import configs
from oracle import oracle as orc


def _run(s, **kw):
    return orc.transport_density(s.nx, s.ny, s.nz, s.h, s.dt, s.open_top, s.vof, s.u, s.v, s.w, **kw)


def _still(s):
    return configs.GridState(s.nx, s.ny, s.nz, s.h, s.dt, s.vof, np.zeros_like(s.u), np.zeros_like(s.v),
                             np.zeros_like(s.w), open_top=s.open_top)


def test_zero_velocity_without_sharpening_is_the_identity():
    """No motion: every cell is its own donor with weight 1 and beta = 1, so
    rho and gamma = 1 come back unchanged (and gamma diffusion has no gradient)."""
    s = _still(configs.transport_scene(20, 18, 16, seed=1))
    rho, g = _run(s, sharpening=False, diffusion=3)
    np.testing.assert_array_equal(rho, s.vof)
    np.testing.assert_array_equal(g, np.ones_like(g))


def test_whole_cell_translation_is_exact():
    """A uniform x velocity of exactly one cell per step moves an interior blob
    by one cell, bit for bit (the RK2 midpoint and the trace are exact)."""
    nx, ny, nz = 24, 12, 10
    s = configs.transport_scene(nx, ny, nz, seed=2)
    vof = np.zeros((nz, ny, nx), np.float32)
    vof[3:7, 3:8, 4:9] = np.linspace(0.2, 1.0, 5, dtype=np.float32)[None, None, :]
    u = np.full((nz, ny, nx + 1), np.float32(s.h / s.dt), np.float32)
    u[:, :, 0] = u[:, :, nx] = 0.0
    st = configs.GridState(nx, ny, nz, s.h, s.dt, vof, u, np.zeros((nz, ny + 1, nx), np.float32),
                           np.zeros((nz + 1, ny, nx), np.float32))
    rho, g = _run(st, sharpening=False, diffusion=0)
    want = np.zeros_like(vof)
    want[3:7, 3:8, 5:10] = vof[3:7, 3:8, 4:9]
    np.testing.assert_array_equal(rho, want)
    np.testing.assert_array_equal(g, np.ones_like(g))


def test_transport_conserves_mass_and_keeps_bounds():
    """The conservative operator with its deficit scatter keeps the total
    mass up to the 2^-20 fixed-point rounding of each deposit; gamma stays in
    [0, 2.5 + deposits]; density stays non-negative."""
    for seed, open_top in ((3, False), (4, True)):
        s = configs.transport_scene(32, 28, 24, seed=seed, cells_per_step=2.5, open_top=open_top)
        m0 = float(np.sum(s.vof, dtype=np.float64))
        rho, g, st = _run(s, sharpening=False, diffusion=0, stages=True)
        assert rho.min() >= 0.0 and np.isfinite(rho).all() and np.isfinite(g).all()
        m1 = float(np.sum(rho, dtype=np.float64))
        assert abs(m1 - m0) <= 1e-4 * m0 + 1e-6 * rho.size, (m0, m1)
        # gamma diffusion moves mass between face pairs with equal and opposite fluxes
        rho_d, _, st2 = _run(s, sharpening=False, diffusion=3, stages=True)
        md = float(np.sum(st2["rho_diffused"], dtype=np.float64))
        mg = float(np.sum(st2["rho_gather"], dtype=np.float64))
        assert abs(md - mg) <= 1e-5 * mg
        # sharpening with its mass return
        rho_s, _ = _run(s)
        ms = float(np.sum(rho_s, dtype=np.float64))
        assert abs(ms - md) <= 1e-4 * md + 1e-6 * rho.size, (md, ms)


def test_sharpening_only_moves_thin_density():
    """Sharpening changes only cells at or below the 0.5 contour; without the
    mass return it removes mass, with it the mass comes back near the contour."""
    s = configs.transport_scene(28, 24, 20, seed=6)
    _, _, st = _run(s, stages=True)
    delta = st["delta"]
    pre = st["rho_diffused"]
    assert (delta[pre > 0.5] == 0.0).all()
    assert (delta <= 0.0).all() and (delta < 0.0).any()
    rho_nm, _ = _run(s, mass_return=False)
    np.testing.assert_array_equal(rho_nm, pre + delta)
    rho_m, _ = _run(s)
    assert float(np.sum(rho_m, dtype=np.float64)) > float(np.sum(rho_nm, dtype=np.float64))


def test_options_clamp_as_the_reference():
    s = configs.transport_scene(16, 14, 12, seed=7)
    a, ga = _run(s, diffusion=9, strength=5.0, distance=9.0)
    b, gb = _run(s, diffusion=7, strength=2.0, distance=3.1)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(ga, gb)


def test_gamma_persists_across_steps():
    s = configs.transport_scene(20, 18, 16, seed=8, cells_per_step=3.0)
    r1, g1 = _run(s)
    st = configs.GridState(s.nx, s.ny, s.nz, s.h, s.dt, r1, s.u, s.v, s.w)
    r2, g2 = _run(st, gamma=g1)
    r2b, _ = _run(st)
    assert not np.array_equal(g1, np.ones_like(g1))
    assert not np.array_equal(r2, r2b)
