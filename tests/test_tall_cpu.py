"""Tall-cell layout planner and the float64 tall-cell oracle (CPU only)."""
import numpy as np
import pytest
import scipy.sparse as sp

from fluid_b200 import configs
from fluid_b200 import tall as product
from oracle import tall as oracle


# Known answers worked by hand from lib/core/tall-cell-grid.ts:61-82
# (maximumBase = fineNy - B_y; lower = highest + 1 + air - B_y; upper = lowest + 1 - liquid;
# desired = Math.round((lower + upper) / 2) when lower <= upper, else lower).
@pytest.mark.parametrize("args,expected", [
    ((600, 601, 1024, 32, 16, 8), 582),     # lower 578, upper 585, round(581.5) = 582
    ((100, 140, 1024, 32, 16, 8), 117),     # lower 117 > upper 85: the air halo wins
    ((5, 6, 40, 32, 16, 8), 2),             # round(-13.5) = -13, clamped to 0, tall cell of 2 rows
    ((10, 30, 32, 32, 16, 8), 0),           # maximumBase 0 < 2: no restricted column
    ((40, 41, 60, 12, 8, 8), 36),           # lower 38, upper 33 -> 38, clamped to maximumBase 48 -> 38? see below
])
def test_choose_tall_base_known_answers(args, expected):
    lowest, highest, fine_ny, by, liq, air = args
    if args == (40, 41, 60, 12, 8, 8):
        # lower = 41 + 1 + 8 - 12 = 38 > upper = 40 + 1 - 8 = 33 -> desired 38 <= maximumBase 48
        expected = 38
    assert oracle.choose_tall_base(*args) == expected
    assert product.choose_tall_base(*args) == expected


def test_choose_tall_base_matches_oracle_sweep():
    rng = np.random.default_rng(0)
    for _ in range(3000):
        fine_ny = int(rng.integers(4, 300))
        by = int(rng.integers(1, fine_ny + 3))
        lo = int(rng.integers(-2, fine_ny + 2))
        hi = lo + int(rng.integers(0, 40))
        liq, air = int(rng.integers(0, 30)), int(rng.integers(0, 30))
        assert product.choose_tall_base(lo, hi, fine_ny, by, liq, air) == oracle.choose_tall_base(lo, hi, fine_ny, by, liq, air)


def test_limit_neighboring_bases_known_answer_and_sweep():
    # pass 1: [min(10, 0+4), 0, min(10, 0+4)] = [4, 0, 4]; pass 2 unchanged
    np.testing.assert_array_equal(product.limit_neighboring_bases([10, 0, 10], 3, 1, 4), [4, 0, 4])
    np.testing.assert_array_equal(oracle.limit_neighboring_bases([10, 0, 10], 3, 1, 4), [4, 0, 4])
    rng = np.random.default_rng(1)
    for nx, nz, d, passes in ((7, 5, 4, 2), (16, 9, 3, 25), (1, 12, 5, 3)):
        raw = rng.integers(2, 200, nx * nz).astype(np.float32)
        np.testing.assert_array_equal(product.limit_neighboring_bases(raw, nx, nz, d, passes),
                                      oracle.limit_neighboring_bases(raw, nx, nz, d, passes))


def test_generator_bases_are_limited_and_the_band_holds_the_surface():
    s = configs.tall_waves(64, 48, 256, 32, seed=9, mean=150, amp_max=12)
    b = s.bases.astype(int)
    assert b.min() >= 2 and (b + s.band).max() <= s.fine_ny
    assert np.abs(np.diff(b, axis=0)).max() <= 4 and np.abs(np.diff(b, axis=1)).max() <= 4
    # band samples hold the interface: each column has a partly wet band row
    band_vof = s.vof[:, 2:, :]
    assert ((band_vof > 0) & (band_vof < 1)).any(axis=1).mean() > 0.95


def test_hierarchy_plan_config3_shapes():
    s = configs.tall_waves()
    shapes = product.plan_tall_hierarchy(s.nx, s.nz, s.fine_ny, s.band, s.bases)
    assert shapes == [(256, 1024, 256, 32), (128, 512, 128, 16), (64, 256, 64, 8), (32, 128, 32, 4),
                      (16, 64, 16, 2), (8, 32, 8, 2), (4, 16, 4, 2)]


def _small():
    return configs.tall_waves(6, 5, 48, 16, seed=21, mean=24, amp_max=3, lam=(4, 12), quality="balanced")


def _dense_operator(g: oracle.TallGrid):
    """The dense MAC ghost-fluid operator over the equivalent dense grid and the
    interpolation T (dense cells x samples), both from the oracle's cell rules."""
    nd = g.nx * g.fine_ny * g.nz
    did = lambda x, y, z: x + g.nx * (y + g.fine_ny * z)
    rows, cols, vals = [], [], []
    for x, y, z, _, xn, yn, zn in g.faces():
        li, pi = g.cell(x, y, z)
        lj, pj = g.cell(xn, yn, zn)
        if not (li or lj):
            continue
        th = 1.0 if (li and lj) else (oracle.ghost_theta(pi, pj) if li else oracle.ghost_theta(pj, pi))
        e = {}
        if li:
            e[did(x, y, z)] = 1.0
        if lj:
            e[did(xn, yn, zn)] = -1.0
        for a, ca in e.items():
            for b, cb in e.items():
                rows.append(a); cols.append(b); vals.append(ca * cb / th)
    Ad = sp.csr_matrix((vals, (rows, cols)), shape=(nd, nd))
    tr, tc, tv = [], [], []
    for z in range(g.nz):
        for y in range(g.fine_ny):
            for x in range(g.nx):
                if not g.cell(x, y, z)[0]:
                    continue
                for k, wt in g.rep(x, y, z):
                    tr.append(did(x, y, z)); tc.append(k); tv.append(wt)
    T = sp.csr_matrix((tv, (tr, tc)), shape=(nd, g.n))
    return Ad, T


def test_tall_operator_is_galerkin_projection_and_spd():
    s = _small()
    g = oracle.TallGrid(s.nx, s.fine_ny, s.nz, s.band, s.bases)
    g.set_state(s.vof, s.u, s.v, s.w)
    A = g.operator()
    Ad, T = _dense_operator(g)
    G = (T.T @ Ad @ T).tocsr()
    assert abs(A - G).max() <= 1e-12 * abs(A).max()
    lab = g.liquid_samples().ravel()
    ids = np.nonzero(lab)[0]
    Al = A[ids][:, ids].toarray()
    np.testing.assert_allclose(Al, Al.T, rtol=0, atol=1e-12)
    assert np.linalg.eigvalsh(Al).min() > 1e-8
    # right-hand side is T^T b_dense
    b = g.rhs()
    bd = np.zeros(g.nx * g.fine_ny * g.nz)
    for z in range(g.nz):
        for y in range(g.fine_ny):
            for x in range(g.nx):
                if g.cell(x, y, z)[0]:
                    bd[x + g.nx * (y + g.fine_ny * z)] = -g.dense_divergence(x, y, z)
    np.testing.assert_allclose(b, T.T @ bd, rtol=0, atol=1e-12 * max(1.0, np.abs(b).max()))


def test_tall_projection_zeroes_divergence_on_represented_band_cells():
    """The packed faces carry the projected field exactly on band cells at rows inside
    the bands of their column and of its four neighbours (every face of such a cell
    is a sample's own face or a tall cell's top face); there the divergence after
    the projection vanishes.  Elsewhere the packed faces keep the layout's
    representation (the two-sample linear profile in tall cells, nothing above a
    band), which the projected field leaves."""
    for s in (_small(), configs.tall_waves(20, 14, 96, 24, seed=22, mean=50, amp_max=6, lam=(6, 30))):
        _check_represented_divergence(s)


def _check_represented_divergence(s):
    g = oracle.TallGrid(s.nx, s.fine_ny, s.nz, s.band, s.bases)
    g.set_state(s.vof, s.u, s.v, s.w)
    p, A, b = g.solve()
    u2, v2, w2 = g.grad_subtract(p)
    worst, before, count = 0.0, 0.0, 0
    for z in range(g.nz):
        for x in range(g.nx):
            cols = [int(s.bases[zz, xx]) for xx, zz in ((x, z), (x - 1, z), (x + 1, z), (x, z - 1), (x, z + 1))
                    if 0 <= xx < g.nx and 0 <= zz < g.nz]
            for y in range(max(cols), min(cols) + g.band):
                if g.cell(x, y, z)[0]:
                    worst = max(worst, abs(g.dense_divergence(x, y, z, u2, v2, w2)))
                    before = max(before, abs(g.dense_divergence(x, y, z)))
                    count += 1
    assert count > 50 and before > 1e-3
    assert worst <= 1e-10 * before


@pytest.mark.parametrize("seed", [21, 22])
def test_fp64_assembly_matches_face_loop_restatement(seed):
    """The C++ per-column float64 assembly (used at full size) gives the operator
    and right-hand side of the per-face Python restatement."""
    s = configs.tall_waves(12, 10, 64, 16, seed=seed, mean=30, amp_max=4, lam=(4, 16), quality="balanced")
    g = oracle.TallGrid(s.nx, s.fine_ny, s.nz, s.band, s.bases)
    g.set_state(s.vof, s.u, s.v, s.w)
    A_ref, b_ref = g.operator(), g.rhs()
    A, b = oracle.assemble_fp64(s.nx, s.fine_ny, s.nz, s.band, s.bases, s.vof, s.u, s.v, s.w)
    assert abs(A - A_ref).max() <= 1e-12 * abs(A_ref).max()
    np.testing.assert_allclose(b, b_ref, rtol=0, atol=1e-12 * np.abs(b_ref).max())
