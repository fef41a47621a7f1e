"""Sparse brick atlas: host planner (block hierarchy, unanchored components)
and the scene helpers, on the CPU."""
import numpy as np
import pytest

from fluid_b200 import configs
from fluid_b200.atlas import bricks_from_dense, plan_atlas


def test_hierarchy_levels_halve_bricks_then_the_brick_grid():
    coords = [(x, y, z) for z in range(8) for y in range(4) for x in range(8)]   # 256 bricks
    cells = plan_atlas((64, 32, 64), coords)["level_cells"]
    # 8, 4, 2, 1 cells per brick edge, then the 8 x 4 x 8 brick grid halved to 4 x 2 x 4
    assert cells == [256 * 512, 256 * 64, 256 * 8, 256, 32]
    # a sparse atlas: a halved block exists where any child exists
    cells = plan_atlas((64, 32, 64), [(0, 0, 0), (1, 0, 0), (7, 3, 7), (6, 2, 6)] * 1)["level_cells"]
    assert cells == [4 * 512, 4 * 64, 4 * 8]


def test_single_brick_stops_at_the_coarse_limit():
    plan = plan_atlas((16, 16, 16), [(1, 0, 1)])
    assert plan["level_cells"] == [512, 64]


def test_components_without_air_are_found():
    ones = np.ones((8, 8, 8), np.float32)
    # two full bricks filling the domain: one pure Neumann component
    p = plan_atlas((16, 8, 8), [(0, 0, 0), (1, 0, 0)], np.stack([ones, ones]))
    assert p["unanchored_components"] == 1 and p["unanchored_cells"] == 1024
    # an absent neighbour brick inside the domain is air: anchored
    p = plan_atlas((24, 8, 8), [(0, 0, 0), (1, 0, 0)], np.stack([ones, ones]))
    assert p["unanchored_components"] == 0
    # a sealed liquid cube inside an air-filled brick is anchored by its air cells
    d = np.zeros((8, 8, 8), np.float32)
    d[2:6, 2:6, 2:6] = 1.0
    p = plan_atlas((8, 8, 8), [(0, 0, 0)], d[None])
    assert p["unanchored_components"] == 0


def test_planner_rejects_bad_bricks():
    with pytest.raises(ValueError):
        plan_atlas((16, 16, 16), [(2, 0, 0)])
    with pytest.raises(ValueError):
        plan_atlas((16, 16, 16), [(0, 0, 0), (0, 0, 0)])
    with pytest.raises(ValueError):
        plan_atlas((12, 16, 16), [(0, 0, 0)])


def test_atlas_scene_bricks_cover_the_liquid():
    s = configs.atlas_scene(48, 40, 32, seed=3)
    coords = configs.atlas_bricks(s.vof)
    gx, gy, gz = s.nx // 8, s.ny // 8, s.nz // 8
    assert 0 < len(coords) < gx * gy * gz
    mask = np.zeros((gz, gy, gx), bool)
    mask[coords[:, 2], coords[:, 1], coords[:, 0]] = True
    dense_mask = np.repeat(np.repeat(np.repeat(mask, 8, 0), 8, 1), 8, 2)
    assert (s.vof[~dense_mask] == 0).all()
    dens, faces = bricks_from_dense(s.vof, s.u, s.v, s.w, coords)
    bx, by, bz = coords[0]
    np.testing.assert_array_equal(dens[0], s.vof[bz * 8:bz * 8 + 8, by * 8:by * 8 + 8, bx * 8:bx * 8 + 8])
    assert faces.shape == (len(coords), 3, 576)
