"""The dense-grid oracle against independent restatements (CPU).

* the row-form restatement of the atlas projection (oracle/atlas_rows.py) on the
  reference's own benchmark fixtures (tools/benchmark-sparse-cm12-pressure.ts);
* a scipy assembly of A = G^T W G / theta from labels and level sets, and a
  direct sparse solve;
* the V-cycle's symmetry and positivity, and the coarse level-set rule
  (mgDownsampleTopology, mg.wgsl.ts:169-195) restated in numpy float32.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from fluid_b200 import configs
from oracle import atlas_rows
from oracle.oracle import Oracle


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
        arr = (u, v, w)[axis]
        arr[gz, gy, gx] = velocity[rid]
    return vof, u, v, w


@pytest.mark.parametrize("name", ["complete-regular-all-fine", "localized-liquid-island", "planar-free-surface"])
def test_dense_oracle_matches_atlas_rows_on_reference_fixtures(name):
    dims, bricks = atlas_rows.reference_fixture(name)
    # the dense grid stores float32 volume fractions; give the rows the same values
    bricks = {c: d.astype(np.float32).astype(np.float64) for c, d in bricks.items()}
    grid = atlas_rows.AtlasGrid(dims, bricks)
    # both restatements see the same float32 face velocities
    vel = atlas_rows.fixture_velocity(grid).astype(np.float32).astype(np.float64)
    ref = atlas_rows.project(grid, vel, rel_tol=1e-12, abs_tol=0.0)
    vof, u, v, w = dense_from_atlas(grid, vel)
    nx, ny, nz = dims
    o = Oracle(nx, ny, nz, 1.0, 1.0)
    o.set_state(vof, u, v, w, 1.0)
    p, info = o.solve_jacobi(1e-12, 0.0)
    assert info["converged"] == 1.0
    # the two restatements give the same right-hand side and pressure on every liquid cell
    b, _ = o.rhs()
    idx = [(gz, gy, gx) for gx, gy, gz in grid.cell_coord]
    rows_b = np.array([b[i] for i in idx]) * ref["liquid"]
    if ref["anchored"] < ref["components"]:   # enclosed liquid: compare on the mean-zero quotient
        rows_b[ref["liquid"]] -= rows_b[ref["liquid"]].mean()
    np.testing.assert_allclose(rows_b, ref["rhs"] * ref["liquid"], rtol=0, atol=1e-12)
    # identical operators: A applied to the same vector agrees to round-off
    rng = np.random.default_rng(1)
    probe = rng.normal(size=len(idx)) * ref["liquid"]
    dense_probe = np.zeros((nz, ny, nx))
    for k, i in enumerate(idx):
        dense_probe[i] = probe[k]
    dense_ap = o.apply(dense_probe)
    rows_ap = ref["apply"](probe)
    np.testing.assert_allclose(np.array([dense_ap[i] for i in idx]), rows_ap, rtol=0,
                               atol=1e-12 * np.abs(rows_ap).max())
    # and both solves (rel-res 1e-12) agree well within the conditioning
    dense_p = np.array([p[i] for i in idx])
    scale = max(np.abs(ref["pressure"]).max(), 1e-30)
    assert np.abs(dense_p - ref["pressure"]).max() <= 1e-6 * scale
    # projected face velocities agree row by row
    (uo, vo, wo), rec = o.grad_subtract(p)
    for rid, row in enumerate(grid.rows):
        axis, (gx, gy, gz) = grid.row_face(row)
        got = float((uo, vo, wo)[axis][gz, gy, gx])
        assert abs(got - ref["projected"][rid]) <= 1e-6 * max(1.0, abs(ref["projected"][rid])), (rid, row)
    assert rec["max_div_after"] <= 1e-9 * max(rec["max_div_before"], 1e-30) + 1e-12


def scipy_operator(o):
    """Independent assembly from the oracle's labels and phi (atlas rules, Neumann walls)."""
    lab, phi, _ = o.level(0)
    nz, ny, nx = lab.shape
    idx = lambda x, y, z: x + nx * (y + ny * z)
    rows, cols, vals = [], [], []
    diag = np.zeros(lab.size)

    def theta(a, b):
        a = abs(float(a))
        return min(1.0, max(0.05, a / max(a + abs(float(b)), 1e-12)))

    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                for dx, dy, dz in ((1, 0, 0), (0, 1, 0), (0, 0, 1)):
                    X, Y, Z = x + dx, y + dy, z + dz
                    i = idx(x, y, z)
                    if X >= nx or Y >= ny or Z >= nz:
                        if o.open_top and dy == 1 and lab[z, y, x]:
                            diag[i] += 1.0 / theta(phi[z, y, x], 0.5)
                        continue
                    j = idx(X, Y, Z)
                    li, lj = lab[z, y, x], lab[Z, Y, X]
                    if li and lj:
                        diag[i] += 1
                        diag[j] += 1
                        rows += [i, j]
                        cols += [j, i]
                        vals += [-1.0, -1.0]
                    elif li:
                        diag[i] += 1.0 / theta(phi[z, y, x], phi[Z, Y, X])
                    elif lj:
                        diag[j] += 1.0 / theta(phi[Z, Y, X], phi[z, y, x])
    A = sp.coo_matrix((vals, (rows, cols)), shape=(lab.size, lab.size)).tocsr() + sp.diags(diag)
    return A, lab.ravel().astype(bool)


@pytest.mark.parametrize("case", ["dam32", "random24", "open_top20"])
def test_dense_oracle_matches_scipy_assembly_and_direct_solve(case):
    s = {"dam32": lambda: configs.dam_break_32(), "random24": lambda: configs.random_small(24, 20, 28, seed=5),
         "open_top20": lambda: configs.random_small(20, 20, 20, seed=6, open_top=True)}[case]()
    o = Oracle(s.nx, s.ny, s.nz, s.h, s.rho, s.open_top)
    o.set_state(s.vof, s.u, s.v, s.w, s.dt)
    A, liq = scipy_operator(o)
    rng = np.random.default_rng(0)
    p = rng.normal(size=liq.size) * liq
    np.testing.assert_allclose(o.apply(p).ravel(), A @ p, rtol=1e-12, atol=1e-12)
    b, _ = o.rhs()
    b = b.ravel()
    sub = A[liq][:, liq]
    x = np.zeros(liq.size)
    x[liq] = spla.spsolve(sub.tocsc(), b[liq])
    for solver in ("jacobi", "mgpcg"):
        if solver == "jacobi":
            p_o, info = o.solve_jacobi(1e-12, 0.0)
        else:
            p_o, info = o.solve_mgpcg(1e-12, 0.0, 300, 1, 1)
        assert info["converged"] == 1.0
        assert np.linalg.norm(p_o.ravel() - x) <= 1e-9 * np.linalg.norm(x)


@pytest.mark.parametrize("dims,seed", [((32, 32, 32), 1), ((37, 50, 29), 2), ((2, 64, 48), 3), ((40, 8, 24), 4)])
def test_vcycle_is_symmetric_and_positive(dims, seed):
    s = configs.random_small(*dims, seed=seed)
    o = Oracle(s.nx, s.ny, s.nz, s.h)
    o.set_state(s.vof, s.u, s.v, s.w, s.dt)
    lab, _, _ = o.level(0)
    rng = np.random.default_rng(seed)
    for pre in (1, 2):
        x = rng.normal(size=lab.shape) * lab
        y = rng.normal(size=lab.shape) * lab
        mx, my = o.vcycle(x, pre, pre), o.vcycle(y, pre, pre)
        assert abs((x * my).sum() - (mx * y).sum()) <= 1e-10 * np.sqrt((x * mx).sum() * (y * my).sum())
        assert (x * mx).sum() > 0


@pytest.mark.parametrize("case", ["dam32", "random24", "open_top20"])
def test_full_cycle_flexible_pcg_solves_the_system(case):
    """The float64 full cycle (fullCycle, webgpu-uniform-pressure-multigrid.ts:
    539-563) under flexible PCG reaches the direct solution in fewer iterations
    than the V-cycle PCG, for every first block level; a full cycle from a zero
    guess leaves a smaller A-norm error than one V-cycle."""
    s = {"dam32": lambda: configs.dam_break_32(), "random24": lambda: configs.random_small(24, 20, 28, seed=5),
         "open_top20": lambda: configs.random_small(20, 20, 20, seed=6, open_top=True)}[case]()
    o = Oracle(s.nx, s.ny, s.nz, s.h, s.rho, s.open_top)
    o.set_state(s.vof, s.u, s.v, s.w, s.dt)
    A, liq = scipy_operator(o)
    b, _ = o.rhs()
    b = b.ravel()
    x = np.zeros(liq.size)
    x[liq] = spla.spsolve(A[liq][:, liq].tocsc(), b[liq])
    _, iv = o.solve_mgpcg(1e-10, 0.0, 300, 1, 1)
    for fb in range(1, o.num_levels):
        p, info = o.solve_fcg(1e-10, 0.0, 300, 1, 1, fb)
        assert info["converged"] == 1.0
        assert info["iterations"] < iv["iterations"], (fb, info, iv)
        assert np.linalg.norm(p.ravel() - x) <= 1e-8 * np.linalg.norm(x)
        zf = o.fcycle(b.reshape(p.shape), 1, 1, fb).ravel()
        zv = o.vcycle(b.reshape(p.shape), 1, 1).ravel()
        ea = lambda z: float((z - x) @ (A @ (z - x)))
        assert ea(zf) < ea(zv), fb


def coarsen_numpy(F, stride, n_coarse, dest):
    """mgDownsampleTopology's phi rule in float32 with the mgD4Sum8 fold."""
    nz, ny, nx = n_coarse
    out = np.zeros((nz, ny, nx), np.float32)
    Fz, Fy, Fx = F.shape
    f32 = np.float32
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                vals = []
                for c in range(8):
                    o = (c & 1, (c >> 1) & 1, (c >> 2) & 1)
                    fx = min(stride[0] * x + o[0] * (stride[0] - 1), Fx - 1)
                    fy = min(stride[1] * y + o[1] * (stride[1] - 1), Fy - 1)
                    fz = min(stride[2] * z + o[2] * (stride[2] - 1), Fz - 1)
                    vals.append(F[fz, fy, fx])
                fold = lambda v: f32(f32(f32(v[0] + v[5]) + f32(v[1] + v[4])) + f32(f32(v[2] + v[7]) + f32(v[3] + v[6])))
                pos = [v if v >= 0 else f32(0) for v in vals]
                pf = [f32(1) if v >= 0 else f32(0) for v in vals]
                nf = [f32(0) if v >= 0 else f32(1) for v in vals]
                npos, nneg = fold(pf), fold(nf)
                if npos > 0 and nneg > 0 and dest <= 2:
                    out[z, y, x] = f32(fold(pos) / max(npos, f32(1)))
                else:
                    out[z, y, x] = f32(fold(vals) / f32(8))
    return out


@pytest.mark.parametrize("dims,seed", [((16, 16, 16), 1), ((19, 13, 22), 2), ((2, 24, 16), 3)])
def test_coarse_level_sets_follow_the_reference_rule_bit_exactly(dims, seed):
    from oracle.oracle import plan_hierarchy
    s = configs.random_small(*dims, seed=seed)
    o = Oracle(s.nx, s.ny, s.nz, s.h)
    o.set_state(s.vof, s.u, s.v, s.w, s.dt)
    plan = plan_hierarchy(*dims)
    for l in range(1, o.num_levels):
        _, phi_f, _ = o.level(l - 1)
        lab_c, phi_c, _ = o.level(l)
        nx, ny, nz = plan["levels"][l]
        expect = coarsen_numpy(phi_f, plan["strides"][l], (nz, ny, nx), l)
        np.testing.assert_array_equal(phi_c.view(np.uint32), expect.view(np.uint32))
        np.testing.assert_array_equal(lab_c, (expect < 0).astype(np.uint8))


def test_labels_follow_the_gpu_tie_rule():
    """liquid <=> rho' > 0.5 (ref.wgsl.ts:242); phi = 0.5 - rho' in cell units."""
    n = 8
    vof = np.full((n, n, n), 0.5, np.float32)
    vof[:, :2, :] = 0.75
    vof[:, 2, :] = np.nextafter(np.float32(0.5), np.float32(1))
    s = configs.GridState(n, n, n, 1.0 / n, 1 / 60, vof, *configs.velocities(vof, np.random.default_rng(0), 1 / 60,
                                                                              "uniform", 0.0))
    o = Oracle(n, n, n, s.h)
    o.set_state(s.vof, s.u, s.v, s.w, s.dt)
    lab, phi, _ = o.level(0)
    assert lab[:, :3, :].all() and not lab[:, 3:, :].any()
    np.testing.assert_array_equal(phi, np.float32(0.5) - vof)
