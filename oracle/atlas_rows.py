"""Row-form restatement of the sparse-atlas ghost-fluid projection (test
infrastructure only: the oracle).

Follows lib/methods/adaptive-mass/sparse-atlas-composite-projection.ts for
atlases whose bricks all carry the finest resolution (8 cells per brick edge):
  * buildSparseAtlasCompositeGrid (:381-900): cells per brick in key order,
    intra-brick rows (:566-620), brick-interface ports (:655-760) and
    sparse-air rows for missing neighbour bricks (:762-790, exterior phi 0.5);
  * buildLiquidSystem (:978-1168), applyLiquidOperator (:1171-1192),
    projectNullspace (:1194-1213), assembleLiquidRhs (:1238-1262),
    pressureCorrection (:1263-1279);
  * projectSparseAtlasVelocity's Jacobi-PCG and projection (:1351-1566).
It is independent of oracle.cpp (rows, not stencils) and is used to check the
dense-grid oracle on the reference's own benchmark fixtures
(tools/benchmark-sparse-cm12-pressure.ts:76-120).
"""
from __future__ import annotations

import math

import numpy as np

RES = 8


def tangents(axis):
    return {0: (1, 2), 1: (0, 2), 2: (0, 1)}[axis]


class AtlasGrid:
    def __init__(self, dims, bricks):
        """bricks: {(bx,by,bz): density array [8][8][8] indexed [z][y][x]}."""
        self.dims = dims
        self.bdims = tuple(math.ceil(d / RES) for d in dims)
        bd = self.bdims
        key = lambda c: c[0] + bd[0] * (c[1] + bd[1] * c[2])
        self.bricks = sorted(bricks.items(), key=lambda kv: key(kv[0]))
        self.present = {c for c, _ in self.bricks}
        self.cell_coord, self.density = [], []
        self.cell_of = {}
        self.base = {}
        for c, dens in self.bricks:
            self.base[c] = len(self.cell_coord)
            for z in range(RES):
                for y in range(RES):
                    for x in range(RES):
                        g = (c[0] * RES + x, c[1] * RES + y, c[2] * RES + z)
                        self.cell_of[g] = len(self.cell_coord)
                        self.cell_coord.append(g)
                        self.density.append(float(dens[z][y][x]))
        self.rows = []   # (kind, axis, [(cell, coef)], negative fine coord of the face)
        for c, _ in self.bricks:
            b = self.base[c]
            for axis in range(3):
                for z in range(RES):
                    for y in range(RES):
                        for x in range(RES):
                            loc = (x, y, z)
                            if loc[axis] == 0:
                                continue
                            pos = b + x + RES * (y + RES * z)
                            neg = pos - (1 if axis == 0 else RES if axis == 1 else RES * RES)
                            self.rows.append(("intra-brick", axis, [(neg, -1.0), (pos, 1.0)]))
        for c, _ in self.bricks:
            for axis in range(3):
                t0, t1 = tangents(axis)
                if c[axis] + 1 < bd[axis]:
                    nb = list(c)
                    nb[axis] += 1
                    nb = tuple(nb)
                    if nb in self.present:
                        face = (c[axis] + 1) * RES
                        for v in range(c[t1] * RES, (c[t1] + 1) * RES):
                            for u in range(c[t0] * RES, (c[t0] + 1) * RES):
                                gn = [0, 0, 0]
                                gn[axis] = face - 1
                                gn[t0], gn[t1] = u, v
                                gp = list(gn)
                                gp[axis] = face
                                self.rows.append(("brick-face", axis, [(self.cell_of[tuple(gn)], -1.0),
                                                                       (self.cell_of[tuple(gp)], 1.0)]))
                    else:
                        self._sparse_air(c, axis, +1)
                if c[axis] > 0:
                    nb = list(c)
                    nb[axis] -= 1
                    if tuple(nb) not in self.present:
                        self._sparse_air(c, axis, -1)

    def _sparse_air(self, c, axis, side):
        b = self.base[c]
        coord = 0 if side < 0 else RES - 1
        for z in range(RES):
            for y in range(RES):
                for x in range(RES):
                    if (x, y, z)[axis] != coord:
                        continue
                    cell = b + x + RES * (y + RES * z)
                    self.rows.append(("sparse-air", axis, [(cell, 1.0 if side < 0 else -1.0)]))

    def row_face(self, row):
        """(axis, fine coordinate of the face's positive-side cell) of a row."""
        kind, axis, terms = row
        if kind == "sparse-air":
            cell, coef = terms[0]
            g = list(self.cell_coord[cell])
            if coef < 0:        # face on the cell's positive side
                g[axis] += 1
            return axis, tuple(g)
        return axis, self.cell_coord[terms[1][0]]


def theta(lphi, aphi, eps):
    a = abs(lphi)
    return min(1.0, max(0.05, a / max(a + abs(aphi), eps)))


def project(grid: AtlasGrid, velocity, rel_tol=1e-10, abs_tol=1e-12, eps=1e-12, max_iter=None, air_phi=0.5):
    n = len(grid.cell_coord)
    phi = np.array([0.5 - d for d in grid.density])
    liquid = phi <= 0
    active, th = [], {}
    diag = np.zeros(n)
    anchored = np.zeros(n, bool)
    for rid, (kind, axis, terms) in enumerate(grid.rows):
        lt = [(c, k) for c, k in terms if liquid[c]]
        at = [(c, k) for c, k in terms if not liquid[c]]
        if not lt:
            continue
        cut = bool(at) or kind == "sparse-air"
        t = 1.0
        if cut:
            lw = sum(abs(k) for _, k in lt)
            lp = sum(abs(k) * phi[c] for c, k in lt) / lw
            aw = sum(abs(k) for _, k in at)
            ap = sum(abs(k) * phi[c] for c, k in at)
            if kind == "sparse-air":
                ap += lw * air_phi
                aw += lw
            t = theta(lp, ap / aw, eps)
            for c, _ in lt:
                anchored[c] = True
        active.append(rid)
        th[rid] = t
        for c, k in lt:
            diag[c] += k * k / t
    # components (atlas :1074-1120)
    adj = [[] for _ in range(n)]
    for rid in active:
        terms = [c for c, _ in grid.rows[rid][2] if liquid[c]]
        for a in range(len(terms)):
            for b in range(a + 1, len(terms)):
                adj[terms[a]].append(terms[b])
                adj[terms[b]].append(terms[a])
    comp = -np.ones(n, int)
    comps = []
    for s in range(n):
        if not liquid[s] or comp[s] >= 0:
            continue
        stack, members, anch = [s], [], False
        comp[s] = len(comps)
        while stack:
            cur = stack.pop()
            members.append(cur)
            anch |= bool(anchored[cur])
            for nb in adj[cur]:
                if comp[nb] < 0:
                    comp[nb] = len(comps)
                    stack.append(nb)
        comps.append((members, anch))

    def proj(v):
        for members, anch in comps:
            if not anch:
                v[members] -= v[members].sum() / len(members)

    def apply(p):
        out = np.zeros(n)
        for rid in active:
            terms = grid.rows[rid][2]
            jump = sum(k * p[c] for c, k in terms if liquid[c])
            w = jump / th[rid]
            for c, k in terms:
                if liquid[c]:
                    out[c] += k * w
        return out

    rhs = np.zeros(n)
    for rid in active:
        for c, k in grid.rows[rid][2]:
            if liquid[c]:
                rhs[c] += k * velocity[rid]
    proj(rhs)
    bnorm = math.sqrt(float(rhs @ rhs))
    p = np.zeros(n)
    r = rhs.copy()
    z = np.where(diag > 0, r / np.where(diag > 0, diag, 1), 0.0)
    proj(z)
    d = z.copy()
    rz = float(r @ z)
    rnorm = math.sqrt(float(r @ r))
    target = max(abs_tol, rel_tol * bnorm)
    it, maxit = 0, max_iter or max(64, 4 * n)
    while it < maxit and rnorm > target:
        q = apply(d)
        proj(q)
        curv = float(d @ q)
        alpha = rz / curv
        p += alpha * d
        r -= alpha * q
        proj(p)
        proj(r)
        it += 1
        rnorm = math.sqrt(float(r @ r))
        if rnorm <= target:
            break
        z = np.where(diag > 0, r / np.where(diag > 0, diag, 1), 0.0)
        proj(z)
        rzn = float(r @ z)
        d = z + (rzn / rz) * d
        proj(d)
        rz = rzn
    projected = np.zeros(len(grid.rows))
    for rid in active:
        terms = grid.rows[rid][2]
        jump = sum(k * p[c] for c, k in terms if liquid[c])
        projected[rid] = velocity[rid] - jump / th[rid]
    return {"pressure": p, "liquid": liquid, "projected": projected, "iterations": it, "rhs": rhs,
            "components": len(comps), "anchored": sum(a for _, a in comps), "apply": apply}


def reference_fixture(name):
    """Fine-resolution fixtures of tools/benchmark-sparse-cm12-pressure.ts:76-120."""
    ones = np.ones((RES, RES, RES))
    if name == "complete-regular-all-fine":
        return (16, 8, 8), {(0, 0, 0): ones, (1, 0, 0): ones}
    if name == "localized-liquid-island":
        d = np.zeros((RES, RES, RES))
        d[2:6, 2:6, 2:6] = 1.0   # x, y, z in [2, 5]
        return (32, 16, 16), {(1, 0, 0): d}
    if name == "planar-free-surface":
        d = np.zeros((RES, RES, RES))
        d[:, :3, :] = 1.0
        d[:, 3, :] = 0.55
        return (16, 8, 8), {(0, 0, 0): d, (1, 0, 0): d.copy()}
    raise KeyError(name)


def fixture_velocity(grid: AtlasGrid, scale=0.01):
    """tools/benchmark-sparse-cm12-pressure.ts:293-295: scale * sin(0.173 (row + 1))."""
    return np.array([scale * math.sin(0.173 * (rid + 1)) for rid in range(len(grid.rows))])
