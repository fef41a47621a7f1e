"""Host-side mirror of the reference's uniform pressure-projection interface.

``PressureProjector`` stands where the reference's
``WebGPUUniformPressureMultigrid`` (lib/methods/uniform/
webgpu-uniform-pressure-multigrid.ts:228-607) plus the ``project`` dispatch
(lib/methods/uniform/webgpu-uniform-reference.ts:1280-1282) stand: the
constructor throws ``ValueError`` (the reference's ``RangeError``) for a lattice
without a hierarchy or a bad spacing; numerical failures on the device are
reported in the receipt's status, never raised.  All compute runs in the CUDA
library through the C ABI; nothing here computes the projection.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import BatchTuning, Config, Receipt, SolveOpts, load, ptr


class FluidError(RuntimeError):
    pass


def _check(rc: int, handle=None, what: str = ""):
    if rc == _abi.OK:
        return
    L = load()
    msg = L.fluid_pp_last_error(handle).decode() if handle is not None else L.fluid_pp_last_error(None).decode()
    if rc == _abi.INVALID_ARG:
        raise ValueError(msg or what)
    if rc == _abi.OOM:
        raise MemoryError(msg or what)
    raise FluidError(f"{_abi.STATUS_NAMES.get(rc, rc)}: {msg or what}")


def plan_uniform_cm11a_hierarchy(dimensions) -> dict:
    """Mirror of planUniformCM11aHierarchy (webgpu-uniform-pressure-multigrid.ts:149-169).

    Returns the reference's fields (levelCount, levelDimensions, coarsestCells,
    semiCoarsened, rejection) plus ``extended`` for ceil-halved lattices the
    reference rejects.
    """
    nx, ny, nz = (int(v) for v in dimensions)
    L = load()
    count, coarsest, semi, ext = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    dims = np.zeros((_abi.MAX_LEVELS, 3), np.int32)
    rc = L.fluid_pp_plan_hierarchy(nx, ny, nz, ctypes.byref(count), ptr(dims), ctypes.byref(coarsest),
                                   ctypes.byref(semi), ctypes.byref(ext))
    if rc != _abi.OK:
        return {"levelCount": 0, "levelDimensions": [], "coarsestCells": 0, "semiCoarsened": False,
                "extended": False, "rejection": L.fluid_pp_last_error(None).decode() or "rejected"}
    return {"levelCount": count.value, "levelDimensions": [tuple(int(v) for v in dims[l]) for l in range(count.value)],
            "coarsestCells": coarsest.value, "semiCoarsened": bool(semi.value), "extended": bool(ext.value),
            "rejection": None}


def kernel_launches() -> int:
    """Kernel launches issued by the CUDA library in this process."""
    return int(load().fluid_pp_kernel_launches())


def _read_profile(fn, handle, reset: bool) -> dict:
    n = len(_abi.STAGES)
    ms = np.zeros(n, np.float64)
    cnt = np.zeros(n, np.int64)
    _check(fn(handle, ptr(ms), ptr(cnt), int(reset)), handle)
    return {name: {"ms": float(ms[k]), "launches": int(cnt[k])} for k, name in enumerate(_abi.STAGES) if cnt[k]}


CYCLES = {"v": 0, "f": 1}


def solve_opts(rel_tol=1e-6, abs_tol=0.0, max_iters=200, pre_sweeps=1, post_sweeps=1, true_residual_every=4,
               warm_start=False, rel_tol_inf=0.0, cycle="v") -> SolveOpts:
    """``cycle``: "v" one V-cycle under PCG, "f" one full cycle under flexible CG."""
    if cycle not in CYCLES:
        raise ValueError(f"cycle must be one of {sorted(CYCLES)}")
    return SolveOpts(rel_tol, abs_tol, max_iters, pre_sweeps, post_sweeps, true_residual_every, int(warm_start),
                     rel_tol_inf, CYCLES[cycle])


class PressureProjector:
    """One uniform MAC grid resident on a B200: label -> divergence -> MGPCG -> gradient subtract."""

    def __init__(self, dimensions, spacing: float, rho: float = 1000.0, open_top: bool = False,
                 precision: str = "fp32", device: int = 0):
        nx, ny, nz = (int(v) for v in dimensions)
        if precision not in _abi.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_abi.PRECISIONS)}")
        L = load()
        self.dims = (nx, ny, nz)
        self.h = float(spacing)
        self.rho = float(rho)
        self.precision = precision
        cfg = Config(nx, ny, nz, self.h, self.rho, int(bool(open_top)), _abi.PRECISIONS[precision], int(device))
        handle = ctypes.c_void_p()
        _check(L.fluid_pp_create(ctypes.byref(cfg), ctypes.byref(handle)), None, "create")
        self._h = handle
        self._keep = []

    # -- lifecycle -----------------------------------------------------------
    def destroy(self):
        if getattr(self, "_h", None):
            load().fluid_pp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream: int):
        _check(load().fluid_pp_set_stream(self._h, ctypes.c_void_p(int(stream))), self._h)

    # -- state -----------------------------------------------------------------
    def upload_solids(self, open_frac, fx, fy, fz, usx=None, usy=None, usz=None):
        """Embedded solids: cell open fractions [nz][ny][nx], face open fractions
        and (optionally) solid normal face velocities in the layouts of u, v, w."""
        nx, ny, nz = self.dims
        sizes = (nx * ny * nz, (nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1))
        arrs = [np.ascontiguousarray(a, np.float32) for a in (open_frac, fx, fy, fz)]
        for a, s, name in zip(arrs, sizes, ("open", "fx", "fy", "fz")):
            if a.size != s:
                raise ValueError(f"{name} has {a.size} entries; expected {s}")
        vel = [None, None, None]
        if usx is not None:
            vel = [np.ascontiguousarray(a, np.float32) for a in (usx, usy, usz)]
            for a, s, name in zip(vel, sizes[1:], ("usx", "usy", "usz")):
                if a.size != s:
                    raise ValueError(f"{name} has {a.size} entries; expected {s}")
        self._solids = (arrs, vel)   # keep the host arrays alive until the copies are done
        _check(load().fluid_pp_upload_solids(self._h, *(ptr(a) for a in arrs),
                                             *(ptr(a) if a is not None else None for a in vel)), self._h, "solids")

    def level_faces(self, level: int) -> np.ndarray:
        """Face open fractions of a level, [3][nz][ny][nx] (+x, +y, +z face of each cell)."""
        nx, ny, nz = self.level_dims(level)
        out = np.empty((3, nz, ny, nx), np.float32)
        _check(load().fluid_pp_get_level_faces(self._h, int(level), ptr(out)), self._h)
        return out

    def upload_state(self, vof, u, v, w):
        nx, ny, nz = self.dims
        arrs = [np.ascontiguousarray(a, np.float32) for a in (vof, u, v, w)]
        sizes = (nx * ny * nz, (nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1))
        for a, s, name in zip(arrs, sizes, ("vof", "u", "v", "w")):
            if a.size != s:
                raise ValueError(f"{name} has {a.size} entries; expected {s}")
        _check(load().fluid_pp_upload_state(self._h, *(ptr(a) for a in arrs)), self._h, "upload")

    def upload_state_device(self, vof_ptr: int, u_ptr: int, v_ptr: int, w_ptr: int):
        _check(load().fluid_pp_upload_state_device(self._h, *(ctypes.c_void_p(int(p)) for p in
                                                             (vof_ptr, u_ptr, v_ptr, w_ptr))), self._h)

    def project(self, dt: float, **opts) -> dict:
        o = solve_opts(**opts)
        r = Receipt()
        rc = load().fluid_pp_project(self._h, float(dt), ctypes.byref(o), ctypes.byref(r))
        if rc not in (_abi.OK, _abi.NONCONVERGENCE, _abi.NONFINITE):
            _check(rc, self._h, "project")
        return r.as_dict()

    def project_lcp(self, dt: float, **opts) -> dict:
        """The CM11a LCP solve (p >= 0 on solid unknowns; needs embedded solids).
        opts: full_cycles, v_cycles, pre_sweeps, post_sweeps, constraint_levels,
        coarse_sweeps, coarse_tol, warm_start."""
        o = _abi.LcpOpts()
        load().fluid_pp_lcp_opts_default(ctypes.byref(o))
        for k, v in opts.items():
            if k not in dict(_abi.LcpOpts._fields_):
                raise TypeError(f"unknown LCP option {k}")
            setattr(o, k, type(getattr(o, k))(v))
        r = Receipt()
        rc = load().fluid_pp_project_lcp(self._h, float(dt), ctypes.byref(o), ctypes.byref(r))
        if rc not in (_abi.OK, _abi.NONCONVERGENCE, _abi.NONFINITE):
            _check(rc, self._h, "project_lcp")
        return r.as_dict()

    def extrapolate_velocity(self) -> int:
        """Extrapolates the handle's face velocities into the air (in place);
        returns the number of open faces holding a value."""
        filled = ctypes.c_longlong(0)
        _check(load().fluid_pp_extrapolate_velocity(self._h, ctypes.byref(filled)), self._h, "extrapolate")
        return int(filled.value)

    def transport_density(self, dt: float, gamma_diffusion_iterations: int = 1, sharpening: bool = True,
                          mass_return: bool = True, strength: float = 1.0, distance: float = 2.1) -> dict:
        """CM12 conservative density transport of the handle's VOF and gamma
        along its face velocities; returns the mass receipt."""
        o = _abi.TransportOpts()
        load().fluid_pp_transport_opts_default(ctypes.byref(o))
        o.gamma_diffusion_iterations = int(gamma_diffusion_iterations)
        o.sharpening = int(bool(sharpening))
        o.sharpening_mass_return = int(bool(mass_return))
        o.sharpening_strength = float(strength)
        o.sharpening_distance = float(distance)
        r = _abi.TransportReceipt()
        _check(load().fluid_pp_transport_density(self._h, float(dt), ctypes.byref(o), ctypes.byref(r)), self._h,
               "transport_density")
        return r.as_dict()

    def set_gamma(self, gamma=None):
        """Sets the persistent gamma ([nz][ny][nx]); None resets it to 1."""
        if gamma is None:
            _check(load().fluid_pp_set_gamma(self._h, None), self._h, "set_gamma")
            return
        nx, ny, nz = self.dims
        g = np.ascontiguousarray(gamma, np.float32)
        if g.size != nx * ny * nz:
            raise ValueError(f"gamma has {g.size} values; expected {nx * ny * nz}")
        _check(load().fluid_pp_set_gamma(self._h, ptr(g)), self._h, "set_gamma")

    def vof(self) -> np.ndarray:
        """The handle's VOF (surface density), [nz][ny][nx]."""
        nx, ny, nz = self.dims
        r = np.empty((nz, ny, nx), np.float32)
        _check(load().fluid_pp_get_vof(self._h, ptr(r)), self._h, "vof")
        return r

    def gamma(self) -> np.ndarray:
        nx, ny, nz = self.dims
        g = np.empty((nz, ny, nx), np.float32)
        _check(load().fluid_pp_get_gamma(self._h, ptr(g)), self._h, "gamma")
        return g

    def project_async(self, dt: float, **opts):
        o = solve_opts(**opts)
        _check(load().fluid_pp_project_async(self._h, float(dt), ctypes.byref(o)), self._h, "project_async")

    def receipt(self) -> dict:
        r = Receipt()
        rc = load().fluid_pp_receipt_read(self._h, ctypes.byref(r))
        if rc not in (_abi.OK, _abi.NONCONVERGENCE, _abi.NONFINITE):
            _check(rc, self._h, "receipt")
        return r.as_dict()

    def download(self):
        nx, ny, nz = self.dims
        p = np.empty((nz, ny, nx), np.float32)
        u = np.empty((nz, ny, nx + 1), np.float32)
        v = np.empty((nz, ny + 1, nx), np.float32)
        w = np.empty((nz + 1, ny, nx), np.float32)
        _check(load().fluid_pp_download(self._h, ptr(p), ptr(u), ptr(v), ptr(w)), self._h, "download")
        return p, u, v, w

    def download_async(self, p, u, v, w):
        """Enqueues the result copies into the caller's arrays (pinned memory, for
        overlap) on the handle's stream; they hold the results after
        ``synchronize()``.  Any array may be None."""
        nx, ny, nz = self.dims
        shapes = ((nz, ny, nx), (nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx))
        ptrs = []
        for a, shp, name in zip((p, u, v, w), shapes, ("p", "u", "v", "w")):
            if a is None:
                ptrs.append(None)
                continue
            if a.dtype != np.float32 or a.size != int(np.prod(shp)) or not a.flags.c_contiguous:
                raise ValueError(f"{name} must be a C-contiguous float32 array of {int(np.prod(shp))} entries")
            ptrs.append(ptr(a))
        _check(load().fluid_pp_download_async(self._h, *ptrs), self._h, "download_async")

    def synchronize(self):
        """Waits for everything enqueued on the handle's stream."""
        _check(load().fluid_pp_synchronize(self._h), self._h, "synchronize")

    def device_arrays(self) -> dict:
        ps = [ctypes.c_void_p() for _ in range(5)]
        _check(load().fluid_pp_device_arrays(self._h, *(ctypes.byref(p) for p in ps)), self._h)
        return dict(zip(("p", "u", "v", "w", "vof"), (p.value for p in ps)))

    # -- parity hooks ----------------------------------------------------------
    def prepare(self, dt: float):
        _check(load().fluid_pp_prepare(self._h, float(dt)), self._h, "prepare")

    def level_dims(self, level: int):
        d = np.zeros(3, np.int32)
        _check(load().fluid_pp_level_dims(self._h, level, ptr(d)), self._h)
        return tuple(int(v) for v in d)

    def level(self, level: int):
        nx, ny, nz = self.level_dims(level)
        lab = np.empty((nz, ny, nx), np.uint8)
        phi = np.empty((nz, ny, nx), np.float32)
        diag = np.empty((nz, ny, nx), np.float32)
        _check(load().fluid_pp_get_level(self._h, level, ptr(lab), ptr(phi), ptr(diag)), self._h)
        return lab, phi, diag

    def rhs(self):
        nx, ny, nz = self.dims
        b = np.empty((nz, ny, nx), np.float32)
        _check(load().fluid_pp_get_rhs(self._h, ptr(b)), self._h)
        return b

    def pressure_cells(self):
        nx, ny, nz = self.dims
        x = np.empty((nz, ny, nx), np.float32)
        _check(load().fluid_pp_get_pressure_cells(self._h, ptr(x)), self._h)
        return x

    def apply_operator(self, p):
        p = np.ascontiguousarray(p, np.float32)
        out = np.empty_like(p)
        _check(load().fluid_pp_apply_operator(self._h, ptr(p), ptr(out)), self._h)
        return out

    # -- diagnostics -----------------------------------------------------------
    def set_profiling(self, on: bool):
        _check(load().fluid_pp_set_profiling(self._h, int(bool(on))), self._h)

    def profile(self, reset: bool = True) -> dict:
        return _read_profile(load().fluid_pp_profile_read, self._h, reset)

    def apply_vcycle(self, r, pre: int = 1, post: int = 1):
        r = np.ascontiguousarray(r, np.float32)
        z = np.empty_like(r)
        _check(load().fluid_pp_apply_vcycle(self._h, ptr(r), ptr(z), int(pre), int(post)), self._h)
        return z

    def apply_fcycle(self, r, pre: int = 1, post: int = 1):
        """One full cycle z = F(r); returns (z, first block level)."""
        r = np.ascontiguousarray(r, np.float32)
        z = np.empty_like(r)
        fb = ctypes.c_int(0)
        _check(load().fluid_pp_apply_fcycle(self._h, ptr(r), ptr(z), int(pre), int(post), ctypes.byref(fb)), self._h)
        return z, int(fb.value)


def batch_tuning(fill_tiles=None, chunk_planes=None, box_shape=None, parts=None) -> BatchTuning:
    """The library's default batch layout with the given fields replaced
    (``fluid_pp_batch_tuning``; results never depend on it, only speed)."""
    t = BatchTuning()
    load().fluid_pp_batch_tuning_default(ctypes.byref(t))
    if fill_tiles is not None:
        t.fill_tiles = int(fill_tiles)
    if chunk_planes is not None:
        t.chunk_planes = int(chunk_planes)
    if box_shape is not None:
        t.box_shape = int(box_shape)
    if parts is not None:
        t.parts = int(parts)
    return t


class BatchProjector:
    """Projects several handles with one launch per stage (uneven grid sizes allowed).

    ``tuning`` (a dict of ``batch_tuning`` fields, a ``BatchTuning`` or None for
    the default) sets how the batch lays out its work; ``fluid_b200.autotune``
    picks it by measurement.
    """

    def __init__(self, projectors, tuning=None):
        self.projectors = list(projectors)
        arr = (ctypes.c_void_p * len(self.projectors))(*(p.handle for p in self.projectors))
        b = ctypes.c_void_p()
        if tuning is None:
            rc = load().fluid_pp_batch_create(arr, len(self.projectors), ctypes.byref(b))
        else:
            t = tuning if isinstance(tuning, BatchTuning) else batch_tuning(**tuning)
            rc = load().fluid_pp_batch_create_tuned(arr, len(self.projectors), ctypes.byref(t), ctypes.byref(b))
        _check(rc, None, "batch_create")
        self._b = b

    def destroy(self):
        if getattr(self, "_b", None):
            load().fluid_pp_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def set_profiling(self, on: bool):
        _check(load().fluid_pp_batch_set_profiling(self._b, int(bool(on))), None)

    def set_graphs(self, on: bool):
        """CUDA-graph replay (default) or direct launches; results are identical."""
        _check(load().fluid_pp_batch_set_graphs(self._b, int(bool(on))), None)

    def profile(self, reset: bool = True) -> dict:
        return _read_profile(load().fluid_pp_batch_profile_read, self._b, reset)

    def project(self, dts, **opts):
        o = solve_opts(**opts)
        n = len(self.projectors)
        dt = np.ascontiguousarray(np.broadcast_to(np.asarray(dts, np.float32), (n,)))
        rec = (Receipt * n)()
        rc = load().fluid_pp_batch_project(self._b, ptr(dt), ctypes.byref(o), rec)
        if rc not in (_abi.OK, _abi.NONCONVERGENCE, _abi.NONFINITE):
            _check(rc, None, "batch_project")
        return [r.as_dict() for r in rec]

    def project_async(self, dts, **opts):
        """Enqueues the batched projection on the batch's stream (the first
        projector's) and returns; ``receipts()`` waits and reads them."""
        o = solve_opts(**opts)
        n = len(self.projectors)
        dt = np.ascontiguousarray(np.broadcast_to(np.asarray(dts, np.float32), (n,)))
        _check(load().fluid_pp_batch_project_async(self._b, ptr(dt), ctypes.byref(o)), None, "batch_project_async")

    def receipts(self):
        n = len(self.projectors)
        rec = (Receipt * n)()
        rc = load().fluid_pp_batch_receipts_read(self._b, rec)
        if rc not in (_abi.OK, _abi.NONCONVERGENCE, _abi.NONFINITE):
            _check(rc, None, "batch_receipts")
        return [r.as_dict() for r in rec]


class PipelinedBatchProjector:
    """Batches of the same lattices used in turn, each on its own CUDA stream.

    A serving host that projects many independent simulations per tick submits
    a full set of host inputs per tick; while one batch solves, the next
    batch's inputs and the previous batch's results cross PCIe on the other
    stream's copy queue.  ``submit`` enqueues upload -> batched projection ->
    read-back on the next slot (first waiting for that slot's previous tick)
    and returns a ticket; ``result(ticket)`` waits for it and returns the
    receipts.  Inputs must stay untouched and outputs unread until the
    ticket's result is taken; both should be pinned host memory, or the copies
    run synchronously.  Results are those of ``BatchProjector.project``.
    """

    def __init__(self, projector_sets, tuning=None):
        self.sets = [list(s) for s in projector_sets]
        if len(self.sets) < 2 or any(len(s) != len(self.sets[0]) for s in self.sets):
            raise ValueError("need at least two projector sets of equal size")
        for s in self.sets[1:]:
            if [p.dims for p in s] != [p.dims for p in self.sets[0]]:
                raise ValueError("projector sets must hold the same lattices in the same order")
        self.batches = [BatchProjector(s, tuning=tuning) for s in self.sets]
        self._pending = [None] * len(self.sets)   # ticket in flight per slot
        self._done = {}
        self._next = 0

    def destroy(self):
        for t in list(self._pending):
            if t is not None:
                self.result(t)
        for b in self.batches:
            b.destroy()
        self.batches = []

    def _drain(self, slot):
        t = self._pending[slot]
        if t is not None:
            self._done[t] = self.batches[slot].receipts()
            self._pending[slot] = None

    def submit(self, inputs, outputs, dts, **opts) -> int:
        """inputs: per lattice (vof, u, v, w); outputs: per lattice (p, u, v, w)
        arrays (any may be None) that receive the results."""
        t = self._next
        slot = t % len(self.sets)
        self._drain(slot)
        projs = self.sets[slot]
        if len(inputs) != len(projs) or len(outputs) != len(projs):
            raise ValueError(f"need {len(projs)} inputs and outputs")
        n = len(projs)
        tabs = [(ctypes.c_void_p * n)() for _ in range(8)]   # vof u v w in, p u v w out
        for k, (p, ins, outs) in enumerate(zip(projs, inputs, outputs)):
            nx, ny, nz = p.dims
            sizes = (nx * ny * nz, (nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1))
            for j, (a, size) in enumerate(zip(list(ins) + list(outs), sizes + sizes)):
                if a is None and j >= 4:
                    continue
                if a is None or a.dtype != np.float32 or a.size != size or not a.flags.c_contiguous:
                    raise ValueError(f"lattice {k}: array {j} must be a C-contiguous float32 array of {size} entries")
                tabs[j][k] = a.ctypes.data
        b = self.batches[slot]
        L = load()
        _check(L.fluid_pp_batch_upload_state(b._b, *tabs[:4]), None, "batch_upload_state")
        b.project_async(dts, **opts)
        _check(L.fluid_pp_batch_download_async(b._b, *tabs[4:]), None, "batch_download_async")
        self._pending[slot] = t
        self._next = t + 1
        return t

    def result(self, ticket: int):
        for slot, t in enumerate(self._pending):
            if t == ticket:
                self._drain(slot)
        if ticket not in self._done:
            raise KeyError(f"ticket {ticket} was never submitted or its result was already taken")
        return self._done.pop(ticket)
