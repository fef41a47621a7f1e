"""Host-side mirror of the restricted tall-cell layout and its pressure projection.

The planner functions mirror ``chooseTallCellBase`` and
``limitNeighboringTallCellBases`` (lib/core/tall-cell-grid.ts:61-106) and run in
the CUDA library's host code; ``TallProjector`` projects a packed tall-cell
state on the GPU (labels, SPD tall-column operator, MGPCG, gradient subtract).
Every packed array is float32 [nz][P][nx] with P = band + 2: sample 0 the tall
cell's bottom subcell (row 0), sample 1 its top subcell (row base - 1), sample
j >= 2 the band row base + j - 2; each sample owns the +x/+y/+z faces of its cell.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import Receipt, TallConfig, load, ptr
from .projector import FluidError, solve_opts

# quality presets of lib/core/tall-cell-grid.ts:52-59
SETTINGS = {
    "balanced": dict(regular_layers=12, liquid_halo=8, air_halo=8, max_delta=4),
    "high": dict(regular_layers=32, liquid_halo=16, air_halo=8, max_delta=4),
    "ultra": dict(regular_layers=40, liquid_halo=24, air_halo=8, max_delta=5),
}


def choose_tall_base(lowest: int, highest: int, fine_ny: int, regular_layers: int, liquid_halo: int,
                     air_halo: int) -> int:
    return int(load().fluid_pp_tall_choose_base(int(lowest), int(highest), int(fine_ny), int(regular_layers),
                                                int(liquid_halo), int(air_halo)))


def limit_neighboring_bases(bases, nx: int, nz: int, max_delta: int, passes: int = 2) -> np.ndarray:
    out = np.ascontiguousarray(np.asarray(bases, np.float32).ravel().copy())
    if out.size != nx * nz:
        raise ValueError(f"bases has {out.size} entries; expected {nx * nz}")
    rc = load().fluid_pp_tall_limit_bases(ptr(out), int(nx), int(nz), int(max_delta), int(passes))
    if rc != _abi.OK:
        raise ValueError("invalid arguments")
    return out


def plan_tall_hierarchy(nx: int, nz: int, fine_ny: int, band: int, bases) -> list[tuple[int, int, int, int]]:
    """Level shapes (nx, fine_ny, nz, band), finest first; ValueError when rejected."""
    b = np.ascontiguousarray(np.asarray(bases, np.int32).ravel())
    count = ctypes.c_int()
    shapes = np.zeros((_abi.MAX_LEVELS, 4), np.int32)
    L = load()
    rc = L.fluid_pp_tall_plan(int(nx), int(nz), int(fine_ny), int(band), ptr(b), ctypes.byref(count), ptr(shapes))
    if rc != _abi.OK:
        raise ValueError(L.fluid_pp_last_error(None).decode())
    return [tuple(int(v) for v in shapes[l]) for l in range(count.value)]


# Red-black block sweeps of the tall grid levels: two before and after the
# coarse correction take the 256^2 x 1024 waves from 20 to 13 iterations and
# 11.6 to 9.8 ms per solve (three: 11 iterations, 9.8 ms).
TALL_SWEEPS = {"pre_sweeps": 2, "post_sweeps": 2}


def _check(rc: int, handle, what: str):
    if rc == _abi.OK:
        return
    L = load()
    msg = (L.fluid_pp_tall_last_error(handle) if handle else L.fluid_pp_last_error(None)).decode()
    if rc == _abi.INVALID_ARG:
        raise ValueError(msg or what)
    if rc == _abi.OOM:
        raise MemoryError(msg or what)
    raise FluidError(f"{_abi.STATUS_NAMES.get(rc, rc)}: {msg or what}")


class TallProjector:
    """Pressure projection on a packed tall-cell grid (one handle per grid)."""

    def __init__(self, nx: int, nz: int, fine_ny: int, band: int, bases, spacing: float, rho: float = 1000.0,
                 precision: str = "fp32", device: int = 0):
        if precision not in _abi.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_abi.PRECISIONS)}")
        self.nx, self.nz, self.fine_ny, self.band = int(nx), int(nz), int(fine_ny), int(band)
        self.P = self.band + 2
        self.bases = np.ascontiguousarray(np.asarray(bases, np.int32).ravel())
        if self.bases.size != self.nx * self.nz:
            raise ValueError(f"bases has {self.bases.size} entries; expected {self.nx * self.nz}")
        cfg = TallConfig(self.nx, self.nz, self.fine_ny, self.band, float(spacing), float(rho),
                         _abi.PRECISIONS[precision], int(device))
        h = ctypes.c_void_p()
        _check(load().fluid_pp_tall_create(ctypes.byref(cfg), ptr(self.bases), ctypes.byref(h)), None, "create")
        self._h = h

    @property
    def shape(self):
        return (self.nz, self.P, self.nx)

    @property
    def samples(self) -> int:
        return self.nx * self.P * self.nz

    def destroy(self):
        if getattr(self, "_h", None):
            load().fluid_pp_tall_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def set_graphs(self, on: bool):
        """CUDA graphs of the CG iteration (default on); off for profilers."""
        _check(load().fluid_pp_tall_set_graphs(self._h, int(bool(on))), self._h, "set_graphs")

    def set_stream(self, stream: int):
        _check(load().fluid_pp_tall_set_stream(self._h, ctypes.c_void_p(int(stream))), self._h, "set_stream")

    def upload_state(self, vof, u, v, w):
        arrs = [np.ascontiguousarray(a, np.float32) for a in (vof, u, v, w)]
        for a, name in zip(arrs, ("vof", "u", "v", "w")):
            if a.size != self.samples:
                raise ValueError(f"{name} has {a.size} entries; expected {self.samples}")
        _check(load().fluid_pp_tall_upload_state(self._h, *(ptr(a) for a in arrs)), self._h, "upload")

    def upload_state_device(self, vof_ptr: int, u_ptr: int, v_ptr: int, w_ptr: int):
        _check(load().fluid_pp_tall_upload_state_device(self._h, *(ctypes.c_void_p(int(p)) for p in
                                                                  (vof_ptr, u_ptr, v_ptr, w_ptr))),
               self._h, "upload")

    def project(self, dt: float, **opts) -> dict:
        """One projection; the grid levels sweep twice before and after the
        coarse correction unless pre_sweeps / post_sweeps say otherwise."""
        o = solve_opts(**{**TALL_SWEEPS, **opts})
        r = Receipt()
        rc = load().fluid_pp_tall_project(self._h, float(dt), ctypes.byref(o), ctypes.byref(r))
        if rc not in (_abi.OK, _abi.NONCONVERGENCE, _abi.NONFINITE, _abi.UNSUPPORTED):
            _check(rc, self._h, "project")
        return r.as_dict()

    # -- the same projection in slices (a server interleaves other steps between them)
    def project_begin(self, dt: float, **opts):
        o = solve_opts(**{**TALL_SWEEPS, **opts})
        _check(load().fluid_pp_tall_project_begin(self._h, float(dt), ctypes.byref(o)), self._h, "project_begin")

    def project_continue(self, max_iterations: int) -> bool:
        """Runs at most max_iterations more CG iterations; True once the solve is finished."""
        done = ctypes.c_int()
        _check(load().fluid_pp_tall_project_continue(self._h, int(max_iterations), ctypes.byref(done)), self._h,
               "project_continue")
        return bool(done.value)

    def project_end(self) -> dict:
        r = Receipt()
        rc = load().fluid_pp_tall_project_end(self._h, ctypes.byref(r))
        if rc not in (_abi.OK, _abi.NONCONVERGENCE, _abi.NONFINITE, _abi.UNSUPPORTED):
            _check(rc, self._h, "project_end")
        return r.as_dict()

    def download(self):
        out = [np.empty(self.shape, np.float32) for _ in range(4)]
        _check(load().fluid_pp_tall_download(self._h, *(ptr(a) for a in out)), self._h, "download")
        return tuple(out)

    # -- diagnostics -----------------------------------------------------------
    def prepare(self, dt: float):
        _check(load().fluid_pp_tall_prepare(self._h, float(dt)), self._h, "prepare")

    def rhs(self):
        b = np.empty(self.shape, np.float32)
        _check(load().fluid_pp_tall_get_rhs(self._h, ptr(b)), self._h, "rhs")
        return b

    def labels(self, level: int = 0, count: int | None = None):
        n = self.samples if count is None else count
        lab = np.empty(n, np.uint8)
        _check(load().fluid_pp_tall_get_labels(self._h, int(level), ptr(lab)), self._h, "labels")
        return lab

    def apply_operator(self, p):
        p = np.ascontiguousarray(p, np.float32)
        out = np.empty_like(p)
        _check(load().fluid_pp_tall_apply_operator(self._h, ptr(p), ptr(out)), self._h, "apply")
        return out

    def pressure(self):
        p = np.empty(self.shape, np.float32)
        _check(load().fluid_pp_tall_get_pressure(self._h, ptr(p)), self._h, "pressure")
        return p

    def solve_rhs(self, dt: float, b, **opts):
        """Parity hook: solve A x = b (finest-cell units, packed) with the device
        MGPCG on the system built from the uploaded state; returns (x, receipt)."""
        b = np.ascontiguousarray(np.asarray(b, np.float32).reshape(self.shape))
        x = np.empty(self.shape, np.float32)
        o = solve_opts(**{**TALL_SWEEPS, **opts})
        r = Receipt()
        rc = load().fluid_pp_tall_solve_rhs(self._h, float(dt), ptr(b), ctypes.byref(o), ptr(x), ctypes.byref(r))
        if rc not in (_abi.OK, _abi.NONCONVERGENCE, _abi.NONFINITE, _abi.UNSUPPORTED):
            _check(rc, self._h, "solve_rhs")
        return x, r.as_dict()
