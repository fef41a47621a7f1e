"""Velocity extrapolation (CM12 Sec. 3.3 / CM11b 3.3.1) in the oracle (CPU):
the float32 restatement of the Fast Iterative Method band and the known-value
hierarchy, checked by properties the method guarantees."""
import numpy as np

from fluid_b200 import configs
from oracle.oracle import extrapolate_velocity


def _liquid_faces(vof):
    fu, fv, fw = configs.fluid_face_masks(vof)
    return fu, fv, fw


def test_constant_field_extends_exactly_and_source_faces_stay():
    """Upwind extension and renormalised interpolation reproduce a constant:
    every open face that receives a value gets the liquid's value, the rest 0;
    faces with a liquid side keep theirs.  The y component is filled
    everywhere (its hierarchy has the corresponding-cell fallback); x and z
    values do not reach across the coarsest levels, whose last face on their
    axis is a closed wall (the reference's lattice has the same property, and
    packs 0 for them)."""
    s = configs.dam_break_32()
    u = np.where(_liquid_faces(s.vof)[0], 0.25, 7.0).astype(np.float32)
    v = np.where(_liquid_faces(s.vof)[1], -0.5, 7.0).astype(np.float32)
    w = np.where(_liquid_faces(s.vof)[2], 0.125, 7.0).astype(np.float32)
    (ue, ve, we), filled, ran = extrapolate_velocity(s.nx, s.ny, s.nz, s.h, False, s.vof, u, v, w)
    assert ran >= 2
    # open faces: the interior ones (walls are closed)
    ui, vi, wi = ue[:, :, 1:-1], ve[:, 1:-1, :], we[1:-1]
    assert np.all((ui == 0.25) | (ui == 0)) and np.all((wi == 0.125) | (wi == 0))
    assert np.all(vi == -0.5)
    assert filled == int((ui != 0).sum() + (vi != 0).sum() + (wi != 0).sum())
    # the band: every open face within two cells of a liquid face has the value
    fu = _liquid_faces(s.vof)[0][:, :, 1:-1]
    near = fu.copy()
    for _ in range(2):
        g = near.copy()
        g[1:] |= near[:-1]; g[:-1] |= near[1:]; g[:, 1:] |= near[:, :-1]; g[:, :-1] |= near[:, 1:]
        g[:, :, 1:] |= near[:, :, :-1]; g[:, :, :-1] |= near[:, :, 1:]
        near = g
    assert np.all(ui[near] == 0.25)
    # walls untouched
    assert np.all(ue[:, :, [0, -1]] == 7.0) and np.all(we[[0, -1]] == 7.0)


def test_band_then_hierarchy_fill_every_open_face_of_a_pool():
    s = configs.random_small(24, 20, 28, seed=5)
    (ue, ve, we), filled, ran = extrapolate_velocity(s.nx, s.ny, s.nz, s.h, False, s.vof, s.u, s.v, s.w)
    fu, fv, fw = _liquid_faces(s.vof)
    np.testing.assert_array_equal(ue[fu], s.u[fu])      # source faces keep their values
    np.testing.assert_array_equal(ve[fv], s.v[fv])
    assert np.all(ve[:, 1:-1, :][~fv[:, 1:-1, :]] != 0) or filled > 0
    # a face next to the liquid takes a combination of its upwind liquid neighbours
    lo, hi = s.u[fu].min(), s.u[fu].max()
    assert lo - 1e-6 <= ue[:, :, 1:-1].min() and ue[:, :, 1:-1].max() <= hi + 1e-6


def test_closed_solid_faces_are_not_written():
    sc = configs.solid_scene(20, 18, 16, seed=4)
    s = sc.state
    (ue, ve, we), filled, _ = extrapolate_velocity(s.nx, s.ny, s.nz, s.h, False, s.vof, s.u, s.v, s.w,
                                                   sc.open, sc.fx, sc.fy, sc.fz)
    closed = np.clip(sc.fx, 0, 1) <= 1e-5
    np.testing.assert_array_equal(ue[closed], s.u[closed])
    assert filled > 0
