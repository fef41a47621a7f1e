"""Float64 oracle of the restricted tall-cell pressure projection (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs may import
this module; the product never calls it.

Layout (lib/core/tall-cell-grid.ts):
  * ``choose_tall_base`` restates ``chooseTallCellBase`` (:61-82) and
    ``limit_neighboring_bases`` restates ``limitNeighboringTallCellBases`` (:84-106);
    JavaScript's ``Math.round`` is round-half-up (``js_round``).
  * Packed samples per x/z column, index ``x + nx * (j + P * z)`` with
    P = band + 2 (:171-190): j = 0 is the tall cell's bottom subcell (world row 0),
    j = 1 its top subcell (row base - 1), j >= 2 the cubic band row base + j - 2
    (active while below the domain top, :398-409).

Operator.  The paper's two-sample tall cell gives a non-symmetric system
(docs/papers/tallCells.txt:356-361).  This restatement instead keeps the repo's
own face-row idiom (sparse-atlas-composite-projection.ts:381-620, 978-1237):
every face of the equivalent dense MAC grid contributes (1/theta) g g^T with
g = T_i - T_j, where T maps the packed samples to a dense cell (a tall subcell
interpolates its column's two samples linearly, Eq. 5 of the paper, a band cell
is its sample, rows above the band are air).  A = T^T A_dense T is symmetric
positive definite by construction; the right-hand side is T^T b_dense.

Labels: a sample is liquid iff vof > 0.5 (phi = 0.5 - vof in cell units); a
tall segment is liquid iff its bottom sample is, and all its rows carry that
sample's phi; rows above the band are air with phi = 0.5.  theta is
cm12GhostFluidTheta (cm12-numerics.ts:37-45) with epsilon 1e-12.

Velocities are packed like the pressure: each sample owns the +x, +y and +z
faces of its dense cell; a tall subcell's faces interpolate the two samples'
faces; the -x/-y/-z faces of a cell are its neighbours' +faces (zero at walls).
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

# quality presets of lib/core/tall-cell-grid.ts:52-59
SETTINGS = {
    "balanced": dict(regular_layers=12, liquid_halo=8, air_halo=8, max_delta=4),
    "high": dict(regular_layers=32, liquid_halo=16, air_halo=8, max_delta=4),
    "ultra": dict(regular_layers=40, liquid_halo=24, air_halo=8, max_delta=5),
}


def js_round(v: float) -> int:
    """JavaScript Math.round: nearest integer, halves toward +infinity."""
    return int(math.floor(v + 0.5))


def choose_tall_base(lowest: int, highest: int, fine_ny: int, regular_layers: int, liquid_halo: int,
                     air_halo: int) -> int:
    """chooseTallCellBase (tall-cell-grid.ts:61-82)."""
    maximum_base = max(0, fine_ny - regular_layers)
    lower = highest + 1 + air_halo - regular_layers
    upper = lowest + 1 - liquid_halo
    desired = js_round((lower + upper) / 2) if lower <= upper else lower
    clamped = max(0, min(maximum_base, desired))
    return max(2, clamped) if maximum_base >= 2 else 0


def limit_neighboring_bases(source, nx: int, nz: int, max_delta: int, passes: int = 2) -> np.ndarray:
    """limitNeighboringTallCellBases (tall-cell-grid.ts:84-106): Jacobi passes of
    base <= neighbour + max_delta over the 4-neighbourhood, index x + nx*z."""
    cur = np.asarray(source, np.float32).copy()
    for _ in range(passes):
        nxt = cur.copy()
        for z in range(nz):
            for x in range(nx):
                i = x + nx * z
                upper = float(cur[i])
                if x > 0:
                    upper = min(upper, float(cur[i - 1]) + max_delta)
                if x + 1 < nx:
                    upper = min(upper, float(cur[i + 1]) + max_delta)
                if z > 0:
                    upper = min(upper, float(cur[i - nx]) + max_delta)
                if z + 1 < nz:
                    upper = min(upper, float(cur[i + nx]) + max_delta)
                nxt[i] = js_round(upper)
        cur = nxt
    return cur


def sample_row(j: int, base: int) -> int:
    """World row of packed sample j in a column of the given base."""
    return 0 if j == 0 else (base - 1 if j == 1 else base + j - 2)


def ghost_theta(liquid_phi: float, air_phi: float) -> float:
    a = abs(liquid_phi)
    return min(1.0, max(0.05, a / max(a + abs(air_phi), 1e-12)))


class TallGrid:
    """Packed tall-cell lattice: nx x nz columns, fine_ny world rows, a band of `band` rows."""

    def __init__(self, nx: int, fine_ny: int, nz: int, band: int, bases, h: float = 1.0, rho: float = 1000.0):
        self.nx, self.fine_ny, self.nz, self.band = int(nx), int(fine_ny), int(nz), int(band)
        self.P = self.band + 2
        self.bases = np.asarray(bases, np.int64).reshape(self.nz, self.nx)
        if self.bases.min() < 2:
            raise ValueError("every column needs a tall cell of at least two rows")
        if (self.bases + self.band).max() > self.fine_ny:
            raise ValueError("band above the domain top")
        self.h, self.rho = float(h), float(rho)
        self.n = self.nx * self.P * self.nz

    def idx(self, x, j, z):
        return x + self.nx * (j + self.P * z)

    # dense-cell representation ---------------------------------------------
    def rep(self, x, y, z):
        """[(sample index, weight)] of dense cell (x, y, z); [] above the band."""
        b = int(self.bases[z, x])
        if y < b:
            t = y / (b - 1)
            return [(self.idx(x, 0, z), 1.0 - t), (self.idx(x, 1, z), t)]
        if y < b + self.band:
            return [(self.idx(x, y - b + 2, z), 1.0)]
        return []

    def active(self, x, j, z):
        return j < 2 or int(self.bases[z, x]) + j - 2 < self.fine_ny

    def set_state(self, vof, u, v, w):
        """Packed (nz, P, nx) arrays."""
        sh = (self.nz, self.P, self.nx)
        self.vof = np.asarray(vof, np.float64).reshape(sh)
        self.u = np.asarray(u, np.float64).reshape(sh)
        self.v = np.asarray(v, np.float64).reshape(sh)
        self.w = np.asarray(w, np.float64).reshape(sh)

    def cell(self, x, y, z):
        """(liquid, phi) of dense cell (x, y, z)."""
        b = int(self.bases[z, x])
        if y < b:
            f = self.vof[z, 0, x]
        elif y < b + self.band:
            f = self.vof[z, y - b + 2, x]
        else:
            return False, 0.5
        return bool(f > 0.5), 0.5 - f

    def liquid_samples(self):
        lab = np.zeros((self.nz, self.P, self.nx), bool)
        for z in range(self.nz):
            for x in range(self.nx):
                tall = self.vof[z, 0, x] > 0.5
                lab[z, 0, x] = lab[z, 1, x] = tall
                for j in range(2, self.P):
                    lab[z, j, x] = self.active(x, j, z) and self.vof[z, j, x] > 0.5
        return lab

    # faces of the dense grid ---------------------------------------------------
    def faces(self):
        """Yields (x, y, z, axis, xn, yn, zn) for every interior face, positive side."""
        for z in range(self.nz):
            for x in range(self.nx):
                for y in range(self.fine_ny):
                    if x + 1 < self.nx:
                        yield x, y, z, 0, x + 1, y, z
                    if y + 1 < self.fine_ny:
                        yield x, y, z, 1, x, y + 1, z
                    if z + 1 < self.nz:
                        yield x, y, z, 2, x, y, z + 1

    def operator(self):
        """A = sum over faces of (1/theta) g g^T restricted to liquid samples (scipy CSR, n x n)."""
        rows, cols, vals = [], [], []
        for x, y, z, _, xn, yn, zn in self.faces():
            li, pi = self.cell(x, y, z)
            lj, pj = self.cell(xn, yn, zn)
            if not (li or lj):
                continue
            th = 1.0 if (li and lj) else (ghost_theta(pi, pj) if li else ghost_theta(pj, pi))
            g = {}
            if li:
                for k, wt in self.rep(x, y, z):
                    g[k] = g.get(k, 0.0) + wt
            if lj:
                for k, wt in self.rep(xn, yn, zn):
                    g[k] = g.get(k, 0.0) - wt
            items = [(k, c) for k, c in g.items() if c != 0.0]
            for ka, ca in items:
                for kb, cb in items:
                    rows.append(ka)
                    cols.append(kb)
                    vals.append(ca * cb / th)
        A = sp.csr_matrix((vals, (rows, cols)), shape=(self.n, self.n))
        A.sum_duplicates()
        return A

    # velocities ----------------------------------------------------------------
    def _face(self, arr, x, y, z):
        """Owner +face value of dense cell (x, y, z) from a packed face array."""
        return sum(wt * arr.flat[k] for k, wt in self.rep(x, y, z))

    def dense_divergence(self, x, y, z, u=None, v=None, w=None):
        u = self.u if u is None else u
        v = self.v if v is None else v
        w = self.w if w is None else w
        du = self._face(u, x, y, z) - (self._face(u, x - 1, y, z) if x > 0 else 0.0)
        dv = self._face(v, x, y, z) - (self._face(v, x, y - 1, z) if y > 0 else 0.0)
        dw = self._face(w, x, y, z) - (self._face(w, x, y, z - 1) if z > 0 else 0.0)
        return (du + dw) + dv

    def rhs(self):
        """b = T^T b_dense, b_dense = -(div u) on liquid dense cells (finest-cell units)."""
        b = np.zeros(self.n)
        for z in range(self.nz):
            for x in range(self.nx):
                for y in range(self.fine_ny):
                    liq, _ = self.cell(x, y, z)
                    if not liq:
                        continue
                    d = -self.dense_divergence(x, y, z)
                    for k, wt in self.rep(x, y, z):
                        b[k] += wt * d
        return b

    def solve(self, tol=1e-12):
        """Float64 pressure on the liquid samples (zero elsewhere)."""
        A = self.operator()
        b = self.rhs()
        lab = self.liquid_samples().ravel()
        ids = np.nonzero(lab)[0]
        p = np.zeros(self.n)
        if ids.size:
            Al = A[ids][:, ids].tocsc()
            p[ids] = spla.spsolve(Al, b[ids])
        return p, A, b

    def pressure_at(self, p, x, y, z):
        liq, _ = self.cell(x, y, z)
        return sum(wt * p[k] for k, wt in self.rep(x, y, z)) if liq else 0.0

    def grad_subtract(self, p):
        """Packed velocities after u_face -= (p_j - p_i) / theta at every sample's own faces;
        faces with no liquid side and wall faces become zero."""
        u2, v2, w2 = self.u.copy(), self.v.copy(), self.w.copy()
        for z in range(self.nz):
            for x in range(self.nx):
                b = int(self.bases[z, x])
                for j in range(self.P):
                    if not self.active(x, j, z):
                        u2[z, j, x] = v2[z, j, x] = w2[z, j, x] = 0.0
                        continue
                    y = sample_row(j, b)
                    for arr, (xn, yn, zn), inside in ((u2, (x + 1, y, z), x + 1 < self.nx),
                                                      (v2, (x, y + 1, z), y + 1 < self.fine_ny),
                                                      (w2, (x, y, z + 1), z + 1 < self.nz)):
                        if not inside:
                            arr[z, j, x] = 0.0
                            continue
                        li, pi_ = self.cell(x, y, z)
                        lj, pj_ = self.cell(xn, yn, zn)
                        if not (li or lj):
                            arr[z, j, x] = 0.0
                            continue
                        th = 1.0 if (li and lj) else (ghost_theta(pi_, pj_) if li else ghost_theta(pj_, pi_))
                        arr[z, j, x] -= (self.pressure_at(p, xn, yn, zn) - self.pressure_at(p, x, y, z)) / th
        return u2, v2, w2


# ---------------------------------------------------------------------------
# The same system at any size: oracle/tall_oracle.cpp assembles the operator and
# right-hand side from the dense faces in float64 (per column, in parallel).
def assemble_fp64(nx: int, fine_ny: int, nz: int, band: int, bases, vof, u, v, w):
    """(A as scipy CSR over the packed samples, b = T^T (-div u)) in float64;
    the arrays are packed (nz, band + 2, nx) as in TallGrid.set_state."""
    import ctypes

    from .oracle import lib
    L = lib()
    f = L.orc_tall_assemble
    vp, ci, cl = ctypes.c_void_p, ctypes.c_int, ctypes.c_long
    f.argtypes = [ci, ci, ci, ci, vp, vp, vp, vp, vp, vp, vp, vp, cl, ctypes.POINTER(cl), vp]
    f.restype = ci
    P = band + 2
    n = nx * P * nz
    arrs = [np.ascontiguousarray(np.asarray(a, np.float32).reshape(nz, P, nx)) for a in (vof, u, v, w)]
    bs = np.ascontiguousarray(np.asarray(bases, np.int32).reshape(nz, nx))
    ptr = lambda a: a.ctypes.data_as(vp) if a is not None else None
    indptr = np.zeros(n + 1, np.int64)
    nnz = cl(0)
    rc = f(nx, fine_ny, nz, band, ptr(bs), *(ptr(a) for a in arrs), ptr(indptr), None, None, 0, ctypes.byref(nnz),
           None)
    if rc:
        raise ValueError("tall oracle: band too wide")
    indices = np.zeros(nnz.value, np.int32)
    data = np.zeros(nnz.value, np.float64)
    b = np.zeros(n, np.float64)
    rc = f(nx, fine_ny, nz, band, ptr(bs), *(ptr(a) for a in arrs), ptr(indptr), ptr(indices), ptr(data), nnz.value,
           ctypes.byref(nnz), ptr(b))
    if rc:
        raise ValueError("tall oracle: assembly failed")
    return sp.csr_matrix((data, indices, indptr), shape=(n, n)), b
