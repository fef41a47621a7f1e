"""Sparse brick atlas on the device (GPU): against the row-form restatement of
the reference's atlas projection on the reference's own benchmark fixtures,
and against the float64 dense oracle on atlases embedded in a dense lattice
(the same system: absent bricks are air, domain faces walls)."""
import numpy as np
import pytest

from fluid_b200 import configs
from fluid_b200.atlas import RES, AtlasProjector, bricks_from_dense
from oracle import atlas_rows
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def dense_from_atlas(grid, velocity):
    nx, ny, nz = grid.dims
    vof = np.zeros((nz, ny, nx), np.float32)
    for (gx, gy, gz), d in zip(grid.cell_coord, grid.density):
        vof[gz, gy, gx] = d
    u = np.zeros((nz, ny, nx + 1), np.float32)
    v = np.zeros((nz, ny + 1, nx), np.float32)
    w = np.zeros((nz + 1, ny, nx), np.float32)
    for rid, row in enumerate(grid.rows):
        axis, (gx, gy, gz) = grid.row_face(row)
        (u, v, w)[axis][gz, gy, gx] = velocity[rid]
    return vof, u, v, w


def dense_faces(dims, coords, faces):
    """Dense MAC arrays from brick faces; both copies of every port must agree."""
    nx, ny, nz = dims
    out = [np.full((nz, ny, nx + 1), np.nan, np.float32), np.full((nz, ny + 1, nx), np.nan, np.float32),
           np.full((nz + 1, ny, nx), np.nan, np.float32)]
    shapes = [(RES, RES, RES + 1), (RES, RES + 1, RES), (RES + 1, RES, RES)]
    for k, (bx, by, bz) in enumerate(coords):
        x0, y0, z0 = bx * RES, by * RES, bz * RES
        for a in range(3):
            blk = faces[k, a].reshape(shapes[a])
            sl = (slice(z0, z0 + shapes[a][0]), slice(y0, y0 + shapes[a][1]), slice(x0, x0 + shapes[a][2]))
            prev = out[a][sl]
            both = ~np.isnan(prev)
            assert np.array_equal(prev[both], blk[both]), "the two copies of a port differ"
            out[a][sl] = blk
    return out


@pytest.mark.parametrize("cycle", ["v", "jacobi"])
@pytest.mark.parametrize("name", ["complete-regular-all-fine", "localized-liquid-island", "planar-free-surface"])
def test_atlas_matches_reference_rows_on_fixtures(name, cycle):
    dims, bricks = atlas_rows.reference_fixture(name)
    bricks = {c: d.astype(np.float32).astype(np.float64) for c, d in bricks.items()}
    grid = atlas_rows.AtlasGrid(dims, bricks)
    vel = atlas_rows.fixture_velocity(grid).astype(np.float32).astype(np.float64)
    ref = atlas_rows.project(grid, vel, rel_tol=1e-12, abs_tol=0.0)
    vof, u, v, w = dense_from_atlas(grid, vel)
    coords = np.array([c for c, _ in grid.bricks], np.int32)   # key order, as the rows' cells
    dens, faces = bricks_from_dense(vof, u, v, w, coords)
    A = AtlasProjector(dims, 1.0, 1.0)
    A.upload(coords, dens, faces)
    rec = A.project(1.0, cycle=cycle, rel_tol=1e-11, max_iters=2000)
    assert rec["status_name"] == "OK", rec
    p, f = A.download()
    p = p.reshape(-1).astype(np.float64)
    liq = ref["liquid"]
    scale = max(np.abs(ref["pressure"]).max(), 1e-30)
    assert np.abs(p[liq] - ref["pressure"][liq]).max() <= 1e-6 * scale
    assert (p[~liq] == 0).all()
    uo, vo, wo = dense_faces(dims, coords, f)
    for rid, row in enumerate(grid.rows):
        axis, (gx, gy, gz) = grid.row_face(row)
        got = float((uo, vo, wo)[axis][gz, gy, gx])
        assert abs(got - ref["projected"][rid]) <= 1e-6 * max(1.0, abs(ref["projected"][rid])), (rid, row)
    A.destroy()


SCENES = {
    "pool_drops_64x48x56": lambda: configs.atlas_scene(64, 48, 56, seed=7),
    "pool_drops_48x40x32": lambda: configs.atlas_scene(48, 40, 32, seed=3, drops=3),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_atlas_matches_fp64_dense_oracle(name):
    s = SCENES[name]()
    coords = configs.atlas_bricks(s.vof)
    dens, faces = bricks_from_dense(s.vof, s.u, s.v, s.w, coords)
    A = AtlasProjector((s.nx, s.ny, s.nz), s.h, s.rho)
    A.upload(coords, dens, faces)
    rec = A.project(s.dt, rel_tol=1e-7)
    assert rec["status_name"] == "OK" and rec["true_rel_residual"] <= 2e-7, rec
    assert rec["max_div_after"] <= 1e-5 * rec["max_div_before"], rec
    rec_j = A.project(s.dt, cycle="jacobi", rel_tol=1e-7, max_iters=3000)
    assert rec_j["status_name"] == "OK" and rec["iterations"] < rec_j["iterations"]
    A.upload(coords, dens, faces)
    A.project(s.dt, rel_tol=1e-7)
    p, f = A.download()
    o = Oracle(s.nx, s.ny, s.nz, s.h, s.rho)
    o.set_state(s.vof, s.u, s.v, s.w, s.dt)
    p_ref, info = o.solve_mgpcg(1e-12, 0.0, 400, 2, 2)
    assert info["converged"] == 1.0
    pscale = s.rho * s.h / s.dt
    got = np.zeros_like(p_ref)
    for k, (bx, by, bz) in enumerate(coords):
        got[bz * 8:bz * 8 + 8, by * 8:by * 8 + 8, bx * 8:bx * 8 + 8] = p[k] / pscale
    assert np.linalg.norm(got - p_ref) <= 1e-5 * np.linalg.norm(p_ref)
    (uo, vo, wo), _ = o.grad_subtract(p_ref)
    ud, vd, wd = dense_faces((s.nx, s.ny, s.nz), coords, f)
    top = max(np.abs(uo).max(), np.abs(vo).max(), np.abs(wo).max())
    for dev, ref in ((ud, uo), (vd, vo), (wd, wo)):
        m = ~np.isnan(dev)
        assert np.abs(dev[m] - ref[m]).max() <= 1e-4 * top
    A.destroy()


def test_atlas_rejects_bad_input():
    A = AtlasProjector((16, 16, 16), 0.1)
    with pytest.raises(ValueError):
        A.upload([(2, 0, 0)], np.zeros((1, 512)), np.zeros((1, 3, 576)))
    with pytest.raises(ValueError):
        A.project(1.0 / 60)
    A.upload([(0, 0, 0)], np.ones((1, 512)) * 0.2, np.zeros((1, 3, 576)))
    with pytest.raises(Exception):
        A.project(1.0 / 60, cycle="f")
    A.destroy()


def test_atlas_graph_and_direct_launches_give_the_same_bits():
    s = configs.atlas_scene(48, 40, 32, seed=5, drops=4)
    coords = configs.atlas_bricks(s.vof)
    dens, faces = bricks_from_dense(s.vof, s.u, s.v, s.w, coords)
    out = []
    for graphs in (True, False):
        A = AtlasProjector((s.nx, s.ny, s.nz), s.h, s.rho)
        A.set_graphs(graphs)
        A.upload(coords, dens, faces)
        rec = A.project(s.dt, rel_tol=1e-6)
        out.append((rec["iterations"], *A.download()))
        A.destroy()
    assert out[0][0] == out[1][0]
    np.testing.assert_array_equal(out[0][1], out[1][1])
    np.testing.assert_array_equal(out[0][2], out[1][2])


def test_a_port_takes_the_lower_bricks_copy():
    """A face shared by two present bricks is stored twice; the lower brick's
    copy is the canonical one.  An upper copy that disagrees on input changes
    nothing, and after the projection both copies hold the projected value."""
    s = configs.atlas_scene(48, 40, 32, seed=7, drops=4)
    coords = configs.atlas_bricks(s.vof)
    dens, faces = bricks_from_dense(s.vof, s.u, s.v, s.w, coords)
    present = {tuple(c): k for k, c in enumerate(coords)}
    noisy = faces.copy()
    shapes = [(RES, RES, RES + 1), (RES, RES + 1, RES), (RES + 1, RES, RES)]
    rng = np.random.default_rng(3)
    ports = 0
    for k, c in enumerate(coords):
        for a in range(3):
            low = list(c)
            low[a] -= 1
            if tuple(low) not in present:
                continue
            blk = noisy[k, a].reshape(shapes[a])
            sl = [slice(None)] * 3
            sl[2 - a] = 0   # the f = 0 layer of the axis (arrays are z, y, x)
            blk[tuple(sl)] = rng.normal(0.0, 5.0, blk[tuple(sl)].shape).astype(np.float32)
            noisy[k, a] = blk.reshape(-1)
            ports += 1
    assert ports > 0
    out = []
    for f in (faces, noisy):
        A = AtlasProjector((s.nx, s.ny, s.nz), s.h, s.rho)
        A.upload(coords, dens, f)
        rec = A.project(s.dt, rel_tol=1e-6)
        assert rec["status_name"] == "OK", rec
        out.append((rec["iterations"], rec["max_div_before"], *A.download()))
        A.destroy()
    assert out[0][:2] == out[1][:2]
    np.testing.assert_array_equal(out[0][2], out[1][2])
    np.testing.assert_array_equal(out[0][3], out[1][3])
    dense_faces((s.nx, s.ny, s.nz), coords, out[1][3])   # both copies of every port agree


@pytest.mark.parametrize("sweeps", [1, 3])
def test_atlas_sweep_counts_match_fp64_dense_oracle(sweeps):
    """One and three red-black sweeps per level (the tiled level 0-2 kernels,
    the fused residual-restriction and the one-CTA tail all run them) give the
    float64 dense oracle's pressure; more sweeps never take more iterations."""
    s = configs.atlas_scene(64, 48, 56, seed=7)
    coords = configs.atlas_bricks(s.vof)
    dens, faces = bricks_from_dense(s.vof, s.u, s.v, s.w, coords)
    A = AtlasProjector((s.nx, s.ny, s.nz), s.h, s.rho)
    its = {}
    for k in (sweeps, 2):
        A.upload(coords, dens, faces)
        rec = A.project(s.dt, rel_tol=1e-7, pre_sweeps=k, post_sweeps=k)
        assert rec["status_name"] == "OK" and rec["true_rel_residual"] <= 2e-7, rec
        its[k] = rec["iterations"]
        if k == sweeps:
            p, _ = A.download()
    A.destroy()
    assert (its[sweeps] >= its[2]) if sweeps < 2 else (its[sweeps] <= its[2])
    o = Oracle(s.nx, s.ny, s.nz, s.h, s.rho)
    o.set_state(s.vof, s.u, s.v, s.w, s.dt)
    p_ref, info = o.solve_mgpcg(1e-12, 0.0, 400, 2, 2)
    assert info["converged"] == 1.0
    pscale = s.rho * s.h / s.dt
    got = np.zeros_like(p_ref)
    for k, (bx, by, bz) in enumerate(coords):
        got[bz * 8:bz * 8 + 8, by * 8:by * 8 + 8, bx * 8:bx * 8 + 8] = p[k] / pscale
    assert np.linalg.norm(got - p_ref) <= 1e-5 * np.linalg.norm(p_ref)
