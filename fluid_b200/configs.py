"""Seeded synthetic inputs for the pressure-projection workloads.

The reference ships no dataset for this path; these generators stand in for
its scenes.  Every array is float32 with x fastest:

* ``vof``  [nz][ny][nx]    liquid volume fraction per cell
* ``u``    [nz][ny][nx+1]  x-face normal velocity (m/s), face x between cells x-1, x
* ``v``    [nz][ny+1][nx]  y-face normal velocity
* ``w``    [nz+1][ny][nx]  z-face normal velocity

A "fluid face" is an interior face with a liquid cell (vof > 0.5) on either
side; closed-wall faces are zero.  Gravity enters as ``v += dt * g`` on fluid
y-faces, the body-force update that precedes the projection in the reference
step (``lib/methods/uniform/webgpu-uniform-reference.ts:1180-1282``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

GRAVITY = -9.81


@dataclass
class GridState:
    nx: int
    ny: int
    nz: int
    h: float
    dt: float
    vof: np.ndarray
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    rho: float = 1000.0
    open_top: bool = False
    meta: dict = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz


def box_fraction(n: int, lo: float, hi: float) -> np.ndarray:
    """Per-cell coverage of [lo, hi) (in cell units) along one axis."""
    i = np.arange(n, dtype=np.float64)
    return np.clip(np.minimum(i + 1, hi) - np.maximum(i, lo), 0.0, 1.0)


def box_vof(nx, ny, nz, lo, hi) -> np.ndarray:
    fx = box_fraction(nx, lo[0], hi[0])
    fy = box_fraction(ny, lo[1], hi[1])
    fz = box_fraction(nz, lo[2], hi[2])
    return fz[:, None, None] * fy[None, :, None] * fx[None, None, :]


def sphere_vof(nx, ny, nz, centre, radius) -> np.ndarray:
    """Linear ramp of the signed distance over one cell (cell units)."""
    out = np.zeros((nz, ny, nx))
    lo = [max(0, int(math.floor(c - radius - 2))) for c in centre]
    hi = [min(n, int(math.ceil(c + radius + 2))) for c, n in zip(centre, (nx, ny, nz))]
    if any(h <= l for l, h in zip(lo, hi)):
        return out
    z, y, x = np.meshgrid(np.arange(lo[2], hi[2]) + 0.5, np.arange(lo[1], hi[1]) + 0.5,
                          np.arange(lo[0], hi[0]) + 0.5, indexing="ij")
    d = np.sqrt((x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2) - radius
    out[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] = np.clip(0.5 - d, 0.0, 1.0)
    return out


def fluid_face_masks(vof: np.ndarray):
    nz, ny, nx = vof.shape
    liq = vof > np.float32(0.5)
    fu = np.zeros((nz, ny, nx + 1), bool)
    fu[:, :, 1:nx] = liq[:, :, :-1] | liq[:, :, 1:]
    fv = np.zeros((nz, ny + 1, nx), bool)
    fv[:, 1:ny, :] = liq[:, :-1, :] | liq[:, 1:, :]
    fw = np.zeros((nz + 1, ny, nx), bool)
    fw[1:nz, :, :] = liq[:-1, :, :] | liq[1:, :, :]
    return fu, fv, fw


def velocities(vof: np.ndarray, rng: np.random.Generator, dt: float, kind: str, scale: float,
               gravity: float = GRAVITY):
    """MAC velocities on fluid faces: ``uniform`` in [-scale, scale] or ``gauss`` N(0, scale)."""
    fu, fv, fw = fluid_face_masks(vof)
    out = []
    for m in (fu, fv, fw):
        if kind == "uniform":
            a = rng.uniform(-scale, scale, size=m.shape)
        else:
            a = rng.normal(0.0, scale, size=m.shape)
        out.append(np.where(m, a, 0.0))
    out[1] = np.where(fv, out[1] + dt * gravity, 0.0)
    return tuple(np.ascontiguousarray(a, np.float32) for a in out)


def dam_break_32(seed: int = 1) -> GridState:
    """32^3, dx = 1/32 m, closed box, corner block x<0.4, y<0.6, z<0.4, U[-0.05,0.05], dt = 1/120."""
    n = 32
    rng = np.random.default_rng(seed)
    vof = box_vof(n, n, n, (0, 0, 0), (0.4 * n, 0.6 * n, 0.4 * n)).astype(np.float32)
    dt = 1.0 / 120.0
    u, v, w = velocities(vof, rng, dt, "uniform", 0.05)
    return GridState(n, n, n, 1.0 / n, dt, vof, u, v, w, meta={"workload": "dam-break 32^3", "seed": seed})


def transport_scene(nx: int = 48, ny: int = 40, nz: int = 44, seed: int = 5, cells_per_step: float = 2.5,
                    open_top: bool = False, noise: float = 0.15) -> GridState:
    """Density-transport input: a dam block (x < 0.45, y < 0.5) and a ball of
    radius 0.18 min(n) in the air (VOF ramps over one cell), and face
    velocities on every open face as an extrapolated field would have them: a
    smooth swirl in x-y plus a sinking drift in y, with seeded relative noise,
    scaled so the fastest face moves cells_per_step cells per step; wall faces
    are 0.  dt = 1/60 s, h = 1/max(n) m."""
    rng = np.random.default_rng(seed)
    n = max(nx, ny, nz)
    h = 1.0 / n
    dt = 1.0 / 60.0
    vof = box_vof(nx, ny, nz, (0, 0, 0), (0.45 * nx, 0.5 * ny, nz))
    r = 0.18 * min(nx, ny, nz)
    vof = np.maximum(vof, sphere_vof(nx, ny, nz, (0.7 * nx, 0.72 * ny, 0.5 * nz), r))

    def field(shape, c):
        z, y, x = np.meshgrid(*(np.arange(k, dtype=np.float64) for k in shape), indexing="ij")
        X = (x + (0.0 if c == 0 else 0.5)) / nx
        Y = (y + (0.0 if c == 1 else 0.5)) / ny
        Z = (z + (0.0 if c == 2 else 0.5)) / nz
        if c == 0:
            f = np.sin(np.pi * X) * np.cos(np.pi * Y) * (0.8 + 0.2 * np.cos(2 * np.pi * Z))
        elif c == 1:
            f = -np.cos(np.pi * X) * np.sin(np.pi * Y) - 0.4
        else:
            f = 0.3 * np.sin(2 * np.pi * X) * np.sin(np.pi * Z)
        return f * (1.0 + noise * rng.uniform(-1.0, 1.0, size=f.shape))

    u = field((nz, ny, nx + 1), 0)
    v = field((nz, ny + 1, nx), 1)
    w = field((nz + 1, ny, nx), 2)
    u[:, :, 0] = u[:, :, nx] = 0.0
    v[:, 0, :] = 0.0
    if not open_top:
        v[:, ny, :] = 0.0
    w[0] = w[nz] = 0.0
    top = max(np.abs(u).max(), np.abs(v).max(), np.abs(w).max())
    scale = cells_per_step * h / dt / top
    u, v, w = (np.ascontiguousarray(a * scale, np.float32) for a in (u, v, w))
    return GridState(nx, ny, nz, h, dt, vof.astype(np.float32), u, v, w, open_top=open_top,
                     meta={"workload": f"density transport {nx}x{ny}x{nz}", "seed": seed,
                           "cells_per_step": cells_per_step})


def atlas_bricks(vof: np.ndarray, dilate: int = 1) -> np.ndarray:
    """Brick coordinates (8-cell bricks) of an atlas over a dense VOF: every
    brick holding density, grown by ``dilate`` bricks in the 26-neighbourhood
    (the bricks a sparse method keeps around the liquid), in key order."""
    nz, ny, nx = vof.shape
    gz, gy, gx = nz // 8, ny // 8, nx // 8
    occ = vof.reshape(gz, 8, gy, 8, gx, 8).max(axis=(1, 3, 5)) > 1e-6
    grown = occ.copy()
    for _ in range(dilate):
        g = grown.copy()
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    sh = np.zeros_like(grown)
                    zs, ys, xs = (slice(max(0, d), n + min(0, d)) for d, n in ((dz, gz), (dy, gy), (dx, gx)))
                    zd, yd, xd = (slice(max(0, -d), n + min(0, -d)) for d, n in ((dz, gz), (dy, gy), (dx, gx)))
                    sh[zd, yd, xd] = grown[zs, ys, xs]
                    g |= sh
        grown = g
    z, y, x = np.nonzero(grown)
    return np.stack([x, y, z], axis=1).astype(np.int32)


def atlas_scene(nx: int = 64, ny: int = 48, nz: int = 56, seed: int = 7, drops: int = 5) -> GridState:
    """A sparse-atlas workload: a shallow pool (18 % of the height) and
    ``drops`` falling balls (radius 3-6 cells) in the air, Gaussian velocities
    (sigma 0.2 m/s) on the faces with a liquid side, dt 1/60.  Most of the
    domain is air, so the atlas holds a fraction of its bricks."""
    rng = np.random.default_rng(seed)
    vof = box_vof(nx, ny, nz, (0, 0, 0), (nx, 0.18 * ny, nz))
    for _ in range(drops):
        r = rng.uniform(3.0, 6.0)
        c = (rng.uniform(r + 2, nx - r - 2), rng.uniform(0.35 * ny + r, ny - r - 2), rng.uniform(r + 2, nz - r - 2))
        vof = np.maximum(vof, sphere_vof(nx, ny, nz, c, r))
    vof = vof.astype(np.float32)
    # no cell exactly at the 0.5 contour (the atlas and the dense labellers differ only there)
    vof[vof == np.float32(0.5)] = np.float32(0.5001)
    dt = 1.0 / 60.0
    u, v, w = velocities(vof, rng, dt, "gauss", 0.2)
    return GridState(nx, ny, nz, 1.0 / max(nx, ny, nz), dt, vof, u, v, w,
                     meta={"workload": f"sparse atlas {nx}x{ny}x{nz}: pool + {drops} drops", "seed": seed})


def dam_spheres(nx=128, ny=96, nz=128, seed: int = 2, step: int = 0, spheres: int = 16) -> GridState:
    """Dam block holding 40% of the volume plus falling spheres (r in [4,10] cells) in the air.

    ``step`` advances the sphere centres downward by a quarter cell per step and
    re-draws the Gaussian (sigma 0.2 m/s) face velocities; dt = 1/60 s.
    """
    rng = np.random.default_rng(seed)
    ax, az = rng.uniform(0.65, 0.85, size=2)
    ay = 0.4 / (ax * az)
    hi = (ax * nx, ay * ny, az * nz)
    vof = box_vof(nx, ny, nz, (0, 0, 0), hi)
    placed = []
    tries = 0
    while len(placed) < spheres and tries < 10000:
        tries += 1
        r = rng.uniform(4.0, 10.0)
        c = np.array([rng.uniform(r + 1, nx - r - 1), rng.uniform(r + 1, ny - r - 1), rng.uniform(r + 1, nz - r - 1)])
        # keep it in the air region, clear of the block and of other spheres
        if c[0] - r < hi[0] + 1 and c[1] - r < hi[1] + 1 + 0.25 * 60 and c[2] - r < hi[2] + 1:
            continue
        if any(np.linalg.norm(c - p[0]) < r + p[1] + 2 for p in placed):
            continue
        placed.append((c, r))
    for c, r in placed:
        cc = c.copy()
        cc[1] = max(r + 0.5, cc[1] - 0.25 * step)
        vof = np.maximum(vof, sphere_vof(nx, ny, nz, cc, r))
    vof = vof.astype(np.float32)
    srng = np.random.default_rng([seed, step])
    dt = 1.0 / 60.0
    u, v, w = velocities(vof, srng, dt, "gauss", 0.2)
    return GridState(nx, ny, nz, 1.0 / nx, dt, vof, u, v, w,
                     meta={"workload": f"dam+{len(placed)} spheres {nx}x{ny}x{nz}", "seed": seed, "step": step})


def dam_spheres_sequence(steps: int, project, nx=128, ny=96, nz=128, seed: int = 2) -> list[GridState]:
    """``steps`` consecutive inputs of the dam-break-with-spheres scene.

    Step 0 is ``dam_spheres(step=0)``.  The input of step k >= 1 is the previous
    step's projected velocity with the body-force update of this step: the
    spheres' VOF of ``dam_spheres(step=k)``, faces that have no liquid side under
    it set to zero, and ``v += dt * g`` on its fluid y-faces (the order of the
    reference step, ``webgpu-uniform-reference.ts:1180-1282``, without
    advection).  ``project(state) -> (u, v, w)`` is the projection that carries
    one step to the next; the caller passes it, so the sequence is defined by
    that solver's outputs.
    """
    out = [dam_spheres(nx, ny, nz, seed=seed, step=0)]
    for k in range(1, steps):
        prev = out[-1]
        u, v, w = project(prev)
        nxt = dam_spheres(nx, ny, nz, seed=seed, step=k)
        fu, fv, fw = fluid_face_masks(nxt.vof)
        v = np.where(fv, v + nxt.dt * GRAVITY, 0.0)
        out.append(GridState(nx, ny, nz, nxt.h, nxt.dt, nxt.vof,
                             np.ascontiguousarray(np.where(fu, u, 0.0), np.float32),
                             np.ascontiguousarray(v, np.float32),
                             np.ascontiguousarray(np.where(fw, w, 0.0), np.float32),
                             meta=dict(nxt.meta, sequence=True)))
    return out


def log_uniform_edge(rng, lo=24, hi=128) -> int:
    return int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))


def random_liquid(nx, ny, nz, rng, fill_lo=0.2, fill_hi=0.7, max_tries=200) -> np.ndarray:
    """Union of 1-6 seeded boxes and spheres whose liquid fraction lies in [fill_lo, fill_hi]."""
    best = None
    for _ in range(max_tries):
        k = int(rng.integers(1, 7))
        vof = np.zeros((nz, ny, nx))
        for _s in range(k):
            if rng.random() < 0.5:
                lo = [rng.uniform(0, 0.6) * n for n in (nx, ny, nz)]
                hi = [lo[a] + rng.uniform(0.25, 0.9) * n for a, n in enumerate((nx, ny, nz))]
                lo[1] = 0.0 if rng.random() < 0.5 else lo[1]   # pools rest on the floor half the time
                vof = np.maximum(vof, box_vof(nx, ny, nz, lo, hi))
            else:
                r = rng.uniform(0.15, 0.45) * min(nx, ny, nz)
                c = [rng.uniform(r, n - r) for n in (nx, ny, nz)]
                vof = np.maximum(vof, sphere_vof(nx, ny, nz, c, r))
        frac = float((vof > 0.5).mean())
        if fill_lo <= frac <= fill_hi:
            return vof.astype(np.float32)
        if best is None or abs(frac - 0.45) < abs(best[0] - 0.45):
            best = (frac, vof)
    return best[1].astype(np.float32)


def batch_instances(count: int = 64, seed: int = 4, lo: int = 24, hi: int = 128) -> list[GridState]:
    """Uneven batch: edges log-uniform in [lo, hi] per axis, 1-6 shapes filling 20-70%."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        nx, ny, nz = (log_uniform_edge(rng, lo, hi) for _ in range(3))
        vof = random_liquid(nx, ny, nz, rng)
        dt = 1.0 / 60.0
        u, v, w = velocities(vof, rng, dt, "gauss", 0.2)
        out.append(GridState(nx, ny, nz, 1.0 / 64.0, dt, vof, u, v, w,
                             meta={"workload": "batched uneven", "seed": seed, "index": k}))
    return out


def random_small(nx, ny, nz, seed: int, open_top: bool = False, fill=(0.2, 0.7)) -> GridState:
    rng = np.random.default_rng(seed)
    vof = random_liquid(nx, ny, nz, rng, *fill)
    dt = 1.0 / 60.0
    u, v, w = velocities(vof, rng, dt, "gauss", 0.2)
    if open_top:
        liq_top = vof[:, -1, :] > 0.5
        v[:, -1, :] = np.where(liq_top, rng.normal(0, 0.2, size=liq_top.shape), 0.0).astype(np.float32)
    return GridState(nx, ny, nz, 1.0 / max(nx, ny, nz), dt, vof, u, v, w, open_top=open_top,
                     meta={"workload": f"random {nx}x{ny}x{nz}", "seed": seed})


# ------------------------------------------------------------------ tall cells
@dataclass
class TallState:
    """Packed tall-cell state: arrays float32 [nz][P][nx], P = band + 2 (see fluid_b200.tall)."""
    nx: int
    nz: int
    fine_ny: int
    band: int
    bases: np.ndarray   # int32 [nz][nx]
    h: float
    dt: float
    vof: np.ndarray
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    rho: float = 1000.0
    meta: dict = field(default_factory=dict)

    @property
    def P(self) -> int:
        return self.band + 2

    @property
    def samples(self) -> int:
        return self.nx * self.P * self.nz

    @property
    def dense_cells(self) -> int:
        return self.nx * self.fine_ny * self.nz


def tall_sample_rows(bases: np.ndarray, band: int) -> np.ndarray:
    """World row of every packed sample, int64 [nz][P][nx]."""
    nz, nx = bases.shape
    j = np.arange(band + 2)[None, :, None]
    b = bases[:, None, :].astype(np.int64)
    return np.where(j == 0, 0, np.where(j == 1, b - 1, b + j - 2))


def tall_waves(nx: int = 256, nz: int = 256, fine_ny: int = 1024, band: int = 32, seed: int = 3,
               mean: float = 600.0, waves: int = 8, amp_max: float = 12.0, lam=(16.0, 256.0), sigma: float = 0.1,
               quality: str = "high") -> TallState:
    """Deep wave tank on a tall-cell grid: surface height (cells) = mean + sum of `waves`
    seeded sinusoids (amplitude <= amp_max, wavelength log-uniform in lam, random
    direction and phase).  Bases per column come from chooseTallCellBase with the
    band pinned to `band` and the quality preset's halos, then
    limitNeighboringTallCellBases with nx + nz passes (the reference's call);
    VOF is the covered fraction of each row (a tall sample holds its rows' mean);
    Gaussian velocities (sigma m/s) on faces with a liquid side, zero at walls."""
    from .tall import SETTINGS, choose_tall_base, limit_neighboring_bases
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.0, amp_max, waves)
    wl = np.exp(rng.uniform(math.log(lam[0]), math.log(lam[1]), waves))
    ang = rng.uniform(0.0, 2 * math.pi, waves)
    ph = rng.uniform(0.0, 2 * math.pi, waves)
    xs = np.arange(nx) + 0.5
    zs = np.arange(nz) + 0.5
    X, Z = np.meshgrid(xs, zs)   # [nz][nx]
    H = np.full((nz, nx), float(mean))
    for a, l, t, p in zip(amp, wl, ang, ph):
        H += a * np.sin(2 * math.pi / l * (math.cos(t) * X + math.sin(t) * Z) + p)
    H = np.clip(H, 1.0, fine_ny - 1.0)
    st = SETTINGS[quality]
    wet_rows = np.ceil(H - 0.5).astype(np.int64)   # rows y with y + 0.5 < H
    raw = np.empty(nx * nz, np.float32)
    for z in range(nz):
        for x in range(nx):
            top = int(wet_rows[z, x]) - 1
            raw[x + nx * z] = choose_tall_base(top, min(top + 1, fine_ny - 1), fine_ny, band, st["liquid_halo"],
                                               st["air_halo"])
    bases = limit_neighboring_bases(raw, nx, nz, st["max_delta"], nx + nz).astype(np.int32).reshape(nz, nx)
    P = band + 2
    rows = tall_sample_rows(bases, band)   # [nz][P][nx]
    frac_row = lambda y: np.clip(H[:, None, :] - y, 0.0, 1.0)
    vof = frac_row(rows).astype(np.float32)
    # a tall sample holds the mean covered fraction of its rows [0, base)
    bb = bases.astype(np.float64)
    covered = np.clip(H, 0.0, bb) / bb
    vof[:, 0, :] = covered
    vof[:, 1, :] = covered
    active = rows < fine_ny
    vof[~active] = 0.0
    liquid = vof > 0.5
    liquid[:, 1, :] = liquid[:, 0, :]

    def dense_liquid(xq, yq, zq):
        """Liquid flag of dense cells (arrays of equal shape); outside -> False."""
        inside = (xq >= 0) & (xq < nx) & (zq >= 0) & (zq < nz) & (yq >= 0) & (yq < fine_ny)
        xc, zc = np.clip(xq, 0, nx - 1), np.clip(zq, 0, nz - 1)
        b = bases[zc, xc].astype(np.int64)
        j = np.where(yq < b, 0, yq - b + 2)
        ok = inside & (j < P)
        jc = np.clip(j, 0, P - 1)
        return ok & liquid[zc, jc, xc]

    zi, ji, xi = np.meshgrid(np.arange(nz), np.arange(P), np.arange(nx), indexing="ij")
    own = liquid & active
    u = np.zeros((nz, P, nx), np.float32)
    v = np.zeros((nz, P, nx), np.float32)
    w = np.zeros((nz, P, nx), np.float32)
    for arr, (dx, dy, dz), wall in ((u, (1, 0, 0), xi + 1 >= nx), (v, (0, 1, 0), rows + 1 >= fine_ny),
                                    (w, (0, 0, 1), zi + 1 >= nz)):
        fluid = (own | dense_liquid(xi + dx, rows + dy, zi + dz)) & active & ~wall
        arr[fluid] = rng.normal(0.0, sigma, size=int(fluid.sum())).astype(np.float32)
    return TallState(nx, nz, fine_ny, band, bases, 1.0 / nx, 1.0 / 60.0, vof, u, v, w,
                     meta={"workload": f"tall waves {nx}x{nz} columns, {fine_ny} rows, band {band}", "seed": seed})


@dataclass
class SolidScene:
    """A uniform-grid state with embedded solids: cell open fractions and the
    MAC faces' dual-cell open fractions and solid normal velocities."""
    state: GridState
    open: np.ndarray
    fx: np.ndarray
    fy: np.ndarray
    fz: np.ndarray
    usx: np.ndarray
    usy: np.ndarray
    usz: np.ndarray

    def solids(self):
        return self.open, self.fx, self.fy, self.fz, self.usx, self.usy, self.usz


def _solid_samples(points, ramp, sphere):
    """(solid, sphere) flags of sample points [..., 3] (x, y, z in cell units):
    terrain below y = ramp[0] + ramp[1] * x, and a ball (centre, radius)."""
    x, y, z = points[..., 0], points[..., 1], points[..., 2]
    terrain = y < ramp[0] + ramp[1] * x
    c, r = sphere
    ball = (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 < r * r
    return terrain | ball, ball & ~terrain


def solid_scene(nx: int = 48, ny: int = 40, nz: int = 44, seed: int = 3, sphere_velocity=(0.0, -0.5, 0.0),
                open_top: bool = False, ball=(0.62, 0.42, 0.5)) -> SolidScene:
    """A dam break over a sloped terrain around a (moving) ball obstacle.

    Open fractions are measured the reference's way (pressureFaceData,
    webgpu-uniform-reference.wgsl.ts:530-556): a face's dual cell by 8 samples
    at +-0.4 cell around the face centre, a cell by 8 samples at +-0.25 cell.
    The liquid fills the open part of the dam block (vof = block fraction x open
    fraction); `ball` is the ball's centre as fractions of the lattice (the
    default sits beside the block, (0.25, 0.35, 0.5) inside it).  The solids' face velocity is the ball's velocity on faces whose
    solid samples are the ball's (weighted by their share), 0 for the terrain."""
    rng = np.random.default_rng(seed)
    ramp = (0.12 * ny, 0.25 * ny / nx)
    sphere = ((ball[0] * nx, ball[1] * ny, ball[2] * nz), 0.16 * min(nx, ny, nz))
    off8 = np.array([[(c & 1) * 2 - 1, ((c >> 1) & 1) * 2 - 1, ((c >> 2) & 1) * 2 - 1] for c in range(8)],
                    np.float64)

    def fraction(centres, half):
        pts = centres[..., None, :] + half * off8
        solid, ball = _solid_samples(pts, ramp, sphere)
        ns, nb = solid.sum(-1), ball.sum(-1)
        return 1.0 - ns / 8.0, np.where(ns > 0, nb / np.maximum(ns, 1), 0.0)

    zc, yc, xc = np.meshgrid(np.arange(nz) + 0.5, np.arange(ny) + 0.5, np.arange(nx) + 0.5, indexing="ij")
    open_frac, _ = fraction(np.stack([xc, yc, zc], -1), 0.25)
    faces, vel = [], []
    for a, shape in enumerate(((nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx))):
        idx = np.meshgrid(*(np.arange(s, dtype=np.float64) for s in shape), indexing="ij")   # z, y, x
        cen = [idx[2] + 0.5, idx[1] + 0.5, idx[0] + 0.5]
        cen[a] = idx[2 - a]   # the face sits on the cell boundary along its axis
        f, share = fraction(np.stack(cen, -1), 0.4)
        faces.append(np.ascontiguousarray(f, np.float32))
        vel.append(np.ascontiguousarray(share * sphere_velocity[a], np.float32))
    block = box_vof(nx, ny, nz, (0, 0, 0), (0.45 * nx, 0.7 * ny, nz))
    vof = np.ascontiguousarray(block * open_frac, np.float32)
    dt = 1.0 / 60.0
    u, v, w = velocities(vof, rng, dt, "gauss", 0.2)
    st = GridState(nx, ny, nz, 1.0 / max(nx, ny, nz), dt, vof, u, v, w, open_top=open_top,
                   meta={"workload": f"dam break over a ramp around a moving ball, {nx}x{ny}x{nz}", "seed": seed})
    return SolidScene(st, np.ascontiguousarray(open_frac, np.float32), *faces, *vel)
