"""Embedded solids in the float64 oracle (CPU): an independent numpy/scipy
restatement of the cut-cell system (face weight = dual-cell open fraction,
rho' = vof / open with the open neighbours' maximum continued into solid cells,
CM11a's weighted divergence with solid face velocities) and the projection's
defining property: the weighted divergence vanishes after the projection."""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from fluid_b200 import configs
from oracle.oracle import Oracle


def _oracle(sc):
    s = sc.state
    o = Oracle(s.nx, s.ny, s.nz, s.h, s.rho, s.open_top)
    o.set_state(s.vof, s.u, s.v, s.w, s.dt)
    o.set_solids(*sc.solids())
    return o


def _theta(a, b):
    a = abs(float(a))
    return min(1.0, max(0.05, a / max(a + abs(float(b)), 1e-12)))


def restated_system(sc):
    """Labels, phi, A and b of the cut-cell system from the scene arrays alone."""
    s = sc.state
    nx, ny, nz = s.nx, s.ny, s.nz
    op = np.clip(np.nan_to_num(sc.open), 0, 1).astype(np.float32)
    vof = s.vof.astype(np.float32)
    rho = np.zeros_like(vof)
    openc = op > np.float32(1e-5)
    rho[openc] = vof[openc] / op[openc]
    pad = np.zeros((nz + 2, ny + 2, nx + 2), np.float32)
    pad[1:-1, 1:-1, 1:-1] = np.where(openc, rho, 0)
    padopen = np.zeros_like(pad, bool)
    padopen[1:-1, 1:-1, 1:-1] = openc
    cont = np.zeros_like(vof)
    for dz, dy, dx in ((0, 0, 1), (0, 0, -1), (0, 1, 0), (0, -1, 0), (1, 0, 0), (-1, 0, 0)):
        sl = (slice(1 + dz, nz + 1 + dz), slice(1 + dy, ny + 1 + dy), slice(1 + dx, nx + 1 + dx))
        cont = np.maximum(cont, np.where(padopen[sl], pad[sl], 0))
    rho = np.where(openc, rho, cont)
    phi = np.float32(0.5) - rho
    wts = [np.where(np.clip(f, 0, 1) > 1e-6, np.clip(f, 0, 1), 0.0).astype(np.float64) for f in (sc.fx, sc.fy, sc.fz)]
    # an unknown needs an open face (walls are closed; the open top counts)
    wx, wy, wz = (w.copy() for w in wts)
    wx[:, :, [0, -1]] = 0
    wz[[0, -1]] = 0
    wy[:, 0, :] = 0
    if not s.open_top:
        wy[:, -1, :] = 0
    any_open = ((wx[:, :, 1:] > 0) | (wx[:, :, :-1] > 0) | (wy[:, 1:, :] > 0) | (wy[:, :-1, :] > 0) |
                (wz[1:] > 0) | (wz[:-1] > 0))
    lab = (rho > np.float32(0.5)) & any_open
    idx = lambda x, y, z: x + nx * (y + ny * z)
    rows, cols, vals = [], [], []
    diag = np.zeros(nx * ny * nz)
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                for a, (dx, dy, dz) in enumerate(((1, 0, 0), (0, 1, 0), (0, 0, 1))):
                    X, Y, Z = x + dx, y + dy, z + dz
                    if X >= nx or Y >= ny or Z >= nz:
                        continue
                    w = wts[a][(z + dz, y, x) if a == 2 else ((z, y + dy, x) if a == 1 else (z, y, x + dx))]
                    if w == 0.0:
                        continue
                    i, j = idx(x, y, z), idx(X, Y, Z)
                    li, lj = lab[z, y, x], lab[Z, Y, X]
                    if li and lj:
                        diag[i] += w
                        diag[j] += w
                        rows += [i, j]
                        cols += [j, i]
                        vals += [-w, -w]
                    elif li:
                        diag[i] += w / _theta(phi[z, y, x], phi[Z, Y, X])
                    elif lj:
                        diag[j] += w / _theta(phi[Z, Y, X], phi[z, y, x])
    A = sp.coo_matrix((vals, (rows, cols)), shape=(lab.size, lab.size)).tocsr() + sp.diags(diag)
    # b = -(weighted divergence with the solids' terms - q(rho'))
    u, v, w = (a.astype(np.float64) for a in (s.u, s.v, s.w))
    us = [a.astype(np.float64) for a in (sc.usx, sc.usy, sc.usz)]
    vi = op.astype(np.float64)

    def axis_div(W, U, S, a):
        if a == 0:
            wp, wm, up, um, sp_, sm = W[:, :, 1:], W[:, :, :-1], U[:, :, 1:], U[:, :, :-1], S[:, :, 1:], S[:, :, :-1]
        elif a == 1:
            wp, wm, up, um, sp_, sm = W[:, 1:, :], W[:, :-1, :], U[:, 1:, :], U[:, :-1, :], S[:, 1:, :], S[:, :-1, :]
        else:
            wp, wm, up, um, sp_, sm = W[1:], W[:-1], U[1:], U[:-1], S[1:], S[:-1]
        return (wp * up - wm * um) + ((wp - vi) * sp_ - (wm - vi) * sm)

    walled = []
    for a, W in enumerate(wts):
        W = W.copy()
        if a == 0:
            W[:, :, 0] = W[:, :, -1] = 0
        elif a == 1:
            W[:, 0, :] = W[:, -1, :] = 0
        else:
            W[0] = W[-1] = 0
        walled.append(W)
    usw = [x.copy() for x in us]
    usw[0][:, :, [0, -1]] = 0
    usw[1][:, [0, -1], :] = 0
    usw[2][[0, -1]] = 0
    div = axis_div(walled[0], u, usw[0], 0) + axis_div(walled[2], w, usw[2], 2) + axis_div(walled[1], v, usw[1], 1)
    hdt = s.h / s.dt
    q = np.where(rho > 1, np.minimum(np.minimum(0.5 * (rho.astype(np.float64) - 1), 1.0), hdt), 0.0)
    b = np.where(lab, -(div - q), 0.0)
    return lab, phi, A, b


def test_all_open_solids_equal_no_solids():
    """Open fractions of 1 everywhere and no solid velocity give the system without solids."""
    s = configs.random_small(24, 20, 28, seed=5)
    o0 = Oracle(s.nx, s.ny, s.nz, s.h, s.rho)
    o0.set_state(s.vof, s.u, s.v, s.w, s.dt)
    o1 = Oracle(s.nx, s.ny, s.nz, s.h, s.rho)
    o1.set_state(s.vof, s.u, s.v, s.w, s.dt)
    ones = lambda a: np.ones_like(a, np.float32)
    o1.set_solids(np.ones_like(s.vof), ones(s.u), ones(s.v), ones(s.w))
    for l in range(o0.num_levels):
        a, b = o0.level(l), o1.level(l)
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])
        np.testing.assert_allclose(a[2], b[2], rtol=1e-15)
        assert np.all(o1.level_faces(l) == 1.0)
    np.testing.assert_allclose(o0.rhs()[0], o1.rhs()[0], rtol=0, atol=1e-12)
    p0, _ = o0.solve_mgpcg(1e-10, 0.0, 300, 1, 1)
    p1, _ = o1.solve_mgpcg(1e-10, 0.0, 300, 1, 1)
    np.testing.assert_allclose(p0, p1, rtol=0, atol=1e-12 * np.abs(p0).max())


def test_solid_system_matches_restatement_and_projects_divergence_free():
    sc = configs.solid_scene(20, 18, 16, seed=4)
    o = _oracle(sc)
    lab, phi, A, b = restated_system(sc)
    lab_o, phi_o, _ = o.level(0)
    np.testing.assert_array_equal(lab_o.astype(bool), lab)
    np.testing.assert_array_equal(phi_o.view(np.uint32), phi.view(np.uint32))
    b_o, _ = o.rhs()
    np.testing.assert_allclose(b_o.ravel(), b.ravel(), rtol=0, atol=1e-6 * np.abs(b).max())
    rng = np.random.default_rng(0)
    p = rng.normal(size=lab.shape) * lab
    np.testing.assert_allclose(o.apply(p).ravel(), (A @ p.ravel()) * lab.ravel(), rtol=0,
                               atol=1e-12 * np.abs(A @ p.ravel()).max())
    liq = lab.ravel()
    x = np.zeros(liq.size)
    x[liq] = spla.spsolve(A[liq][:, liq].tocsc(), b.ravel()[liq])
    p_o, info = o.solve_mgpcg(1e-12, 0.0, 300, 1, 1)
    assert info["converged"] == 1.0
    assert np.linalg.norm(p_o.ravel() - x) <= 1e-9 * np.linalg.norm(x)
    (uo, vo, wo), rec = o.grad_subtract(p_o)
    assert rec["max_div_after"] <= 1e-9 * rec["max_div_before"]
    # closed faces carry the solids' velocity
    closed = np.clip(sc.fy, 0, 1) <= 1e-6
    closed[:, [0, -1], :] = False
    np.testing.assert_array_equal(vo[closed], sc.usy[closed])


def test_coarse_face_fractions_are_child_means():
    sc = configs.solid_scene(20, 18, 16, seed=6)
    o = _oracle(sc)
    f0 = o.level_faces(0)
    assert f0.shape == (3, 16, 18, 20)
    np.testing.assert_array_equal(f0[0][:, :, :-1], np.clip(sc.fx[:, :, 1:-1], 0, 1))
    (cx, cy, cz), _, _ = o.level_dims(1)
    f1 = o.level_faces(1)
    for a in range(3):
        # every coarse cell halves each axis here: the mean of its 2 x 2 x 2 children
        ch = f0[a].reshape(cz, 2, cy, 2, cx, 2).astype(np.float64).mean(axis=(1, 3, 5))
        np.testing.assert_allclose(f1[a], ch, rtol=0, atol=1e-7)


def test_oracle_lcp_holds_the_bound_and_reduces_to_the_linear_solve_without_one():
    """The CM11a LCP restatement: p >= 0 on solid unknowns, rows at the bound
    where the linear solve would pull (negative pressure), and with no active
    bound the projected multigrid converges to the linear solution."""
    sc = configs.solid_scene(32, 28, 30, seed=3, sphere_velocity=(0.0, -2.0, 0.0), ball=(0.25, 0.35, 0.5))
    o = _oracle(sc)
    lab = o.level(0)[0].astype(bool)
    solid = lab & (np.clip(sc.open, 0, 1) <= 1e-5)
    p_lin, _ = o.solve_mgpcg(1e-10, 0.0, 400, 1, 1)
    assert (p_lin[solid] < 0).any()
    p, info = o.solve_lcp(3, 4)
    assert p[solid].min() >= 0.0 and info["at_bound"] > 0
    p2, info2 = o.solve_lcp(3, 20)
    assert info2["l2_residual"] < info["l2_residual"]
    quiet = configs.solid_scene(24, 20, 22, seed=4)   # the ball beside the liquid: no bound active
    oq = _oracle(quiet)
    pq, iq = oq.solve_lcp(3, 60)
    ref, _ = oq.solve_mgpcg(1e-12, 0.0, 400, 1, 1)
    assert np.linalg.norm(pq - ref) <= 1e-3 * np.linalg.norm(ref)
    assert iq["at_bound"] == 0
