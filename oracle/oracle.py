"""ctypes front end of the CPU oracle (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline leg
and reference arm may import this module.  It wraps ``oracle/_build/liboracle.so``
(built from ``oracle/oracle.cpp`` by ``oracle/Makefile``), a float64 restatement
of the reference's dense MAC ghost-fluid pressure projection; see the header of
``oracle.cpp`` for the reference files and lines it follows.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        c_int, c_long, c_double, vp = ctypes.c_int, ctypes.c_long, ctypes.c_double, ctypes.c_void_p
        L.orc_plan_hierarchy.argtypes = [c_int, c_int, c_int, ctypes.POINTER(c_int), vp, vp,
                                         ctypes.POINTER(c_long), ctypes.POINTER(c_int), ctypes.POINTER(c_int)]
        L.orc_plan_hierarchy.restype = c_int
        L.orc_create.argtypes = [c_int, c_int, c_int, c_int, c_double, c_double]
        L.orc_create.restype = vp
        L.orc_destroy.argtypes = [vp]
        L.orc_set_threads.argtypes = [vp, c_int]
        L.orc_set_state.argtypes = [vp, vp, vp, vp, vp, c_double]
        L.orc_set_state.restype = c_int
        L.orc_num_levels.argtypes = [vp]
        L.orc_num_levels.restype = c_int
        L.orc_level_dims.argtypes = [vp, c_int, vp, vp, vp]
        L.orc_get_level.argtypes = [vp, c_int, vp, vp, vp]
        L.orc_get_rhs.argtypes = [vp, vp, vp]
        L.orc_apply_level.argtypes = [vp, c_int, vp, vp]
        L.orc_vcycle.argtypes = [vp, vp, vp, c_int, c_int]
        L.orc_set_solids.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
        L.orc_set_solids.restype = c_int
        L.orc_level_faces.argtypes = [vp, c_int, vp]
        L.orc_solve_lcp.argtypes = [vp, c_int, c_int, c_int, c_int, c_int, c_int, c_double, vp, vp]
        L.orc_solve_lcp.restype = c_int
        L.orc_extrapolate.argtypes = [c_int, c_int, c_int, c_double, c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.orc_extrapolate.restype = ctypes.c_long
        L.orc_transport.argtypes = [c_int, c_int, c_int, c_double, c_double, c_int, vp, vp, vp, vp, vp, c_int, c_int,
                                    c_int, c_double, c_double, vp]
        L.orc_transport.restype = None
        L.orc_fcycle.argtypes = [vp, vp, vp, c_int, c_int, c_int]
        L.orc_solve_fcg.argtypes = [vp, c_double, c_double, c_int, c_int, c_int, c_int, vp, vp]
        L.orc_solve_fcg.restype = c_int
        L.orc_solve_jacobi.argtypes = [vp, c_double, c_double, c_int, vp, vp]
        L.orc_solve_jacobi.restype = c_int
        L.orc_solve_mgpcg.argtypes = [vp, c_double, c_double, c_int, c_int, c_int, vp, vp]
        L.orc_solve_mgpcg.restype = c_int
        L.orc_grad_subtract.argtypes = [vp, vp, vp, vp, vp, vp]
        L.orc_pcg_dense.argtypes = [c_int, vp, vp, vp, vp, c_int, c_double, c_double, vp, vp]
        L.orc_pcg_dense.restype = c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def plan_hierarchy(nx: int, ny: int, nz: int) -> dict:
    """Planner restatement: reference lockstep/semi-coarsening, else ceil-halving."""
    L = lib()
    count = ctypes.c_int()
    dims = np.zeros((24, 3), np.int32)
    strides = np.zeros((24, 3), np.int32)
    coarsest = ctypes.c_long()
    semi = ctypes.c_int()
    ext = ctypes.c_int()
    rc = L.orc_plan_hierarchy(nx, ny, nz, ctypes.byref(count), _p(dims), _p(strides),
                              ctypes.byref(coarsest), ctypes.byref(semi), ctypes.byref(ext))
    return {"ok": rc == 0, "levels": [tuple(int(v) for v in dims[i]) for i in range(count.value)],
            "strides": [tuple(int(v) for v in strides[i]) for i in range(count.value)],
            "coarsest_cells": int(coarsest.value), "semi": bool(semi.value), "extended": bool(ext.value)}


INFO_KEYS = ("iterations", "converged", "recursive_rel_residual", "true_rel_residual", "b_norm",
             "reductions", "failure", "liquid_cells")
FAILURES = {0: None, 1: "non-positive-direction-curvature", 2: "maximum-iterations", 3: "true-residual-validation"}


def pcg_dense(A, b, minv=None, x0=None, max_iter=None, rel_tol=1e-10, abs_tol=0.0):
    """The C++ oracle's direct-curvature PCG on a dense system (known-answer checks)."""
    A = np.ascontiguousarray(A, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    n = b.size
    mv = None if minv is None else np.ascontiguousarray(minv, np.float64)
    g = None if x0 is None else np.ascontiguousarray(x0, np.float64)
    x = np.zeros(n, np.float64)
    info = np.zeros(8, np.float64)
    rc = lib().orc_pcg_dense(n, _p(A), _p(b), _p(mv), _p(g), int(n if max_iter is None else max_iter),
                             rel_tol, abs_tol, _p(x), _p(info))
    d = dict(zip(INFO_KEYS, info.tolist()))
    d["failure_name"] = FAILURES.get(rc, str(rc))
    return x, d


class Oracle:
    """One dense uniform grid; mirrors the device handle's lifecycle."""

    def __init__(self, nx: int, ny: int, nz: int, h: float, rho: float = 1000.0, open_top: bool = False):
        self.n = (nx, ny, nz)
        self.h, self.rho = h, rho
        self.open_top = bool(open_top)
        self._h = lib().orc_create(nx, ny, nz, int(open_top), h, rho)
        if not self._h:
            raise ValueError("CM11a coarsest grid must be integral and fit its 256-lane high-precision solve")
        self.dt = 1.0

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    def set_threads(self, threads: int):
        lib().orc_set_threads(self._h, int(threads))

    def set_state(self, vof, u, v, w, dt: float):
        nx, ny, nz = self.n
        self._vof = np.ascontiguousarray(vof, np.float32).reshape(nz, ny, nx)
        self._u = np.ascontiguousarray(u, np.float32).reshape(nz, ny, nx + 1)
        self._v = np.ascontiguousarray(v, np.float32).reshape(nz, ny + 1, nx)
        self._w = np.ascontiguousarray(w, np.float32).reshape(nz + 1, ny, nx)
        self.dt = dt
        lib().orc_set_state(self._h, _p(self._vof), _p(self._u), _p(self._v), _p(self._w), dt)

    @property
    def num_levels(self) -> int:
        return lib().orc_num_levels(self._h)

    def level_dims(self, l: int):
        d = np.zeros(3, np.int32)
        wgt = np.zeros(3, np.float64)
        anch = np.zeros(1, np.int32)
        lib().orc_level_dims(self._h, l, _p(d), _p(wgt), _p(anch))
        return tuple(int(x) for x in d), tuple(float(x) for x in wgt), bool(anch[0])

    def level(self, l: int):
        (nx, ny, nz), _, _ = self.level_dims(l)
        lab = np.zeros((nz, ny, nx), np.uint8)
        phi = np.zeros((nz, ny, nx), np.float32)
        diag = np.zeros((nz, ny, nx), np.float64)
        lib().orc_get_level(self._h, l, _p(lab), _p(phi), _p(diag))
        return lab, phi, diag

    def rhs(self):
        nx, ny, nz = self.n
        b = np.zeros((nz, ny, nx), np.float64)
        q = np.zeros((nz, ny, nx), np.float64)
        lib().orc_get_rhs(self._h, _p(b), _p(q))
        return b, q

    def apply(self, p, l: int = 0):
        (nx, ny, nz), _, _ = self.level_dims(l)
        p = np.ascontiguousarray(p, np.float64).reshape(nz, ny, nx)
        out = np.zeros_like(p)
        lib().orc_apply_level(self._h, l, _p(p), _p(out))
        return out

    def vcycle(self, r, pre: int = 1, post: int = 1):
        nx, ny, nz = self.n
        r = np.ascontiguousarray(r, np.float64).reshape(nz, ny, nx)
        z = np.zeros_like(r)
        lib().orc_vcycle(self._h, _p(r), _p(z), pre, post)
        return z

    def set_solids(self, open_frac, fx, fy, fz, usx=None, usy=None, usz=None):
        """Embedded solids (cell and face open fractions, optional solid face
        velocities); rebuilds the current state's system."""
        arrs = [np.ascontiguousarray(a, np.float32) for a in (open_frac, fx, fy, fz)]
        vel = [np.ascontiguousarray(a, np.float32) if a is not None else None for a in (usx, usy, usz)]
        lib().orc_set_solids(self._h, *(_p(a) for a in arrs), *(_p(a) if a is not None else None for a in vel))

    def solve_lcp(self, full_cycles=3, v_cycles=4, pre=1, post=1, constraint_levels=3, coarse_sweeps=4096,
                  coarse_tol=1e-6):
        """The CM11a LCP solve (p >= 0 on solid unknowns); returns p and
        {cycles, max/l2 projected residual, ||b||, rows at their bound}."""
        nx, ny, nz = self.n
        p = np.zeros((nz, ny, nx), np.float64)
        info = np.zeros(5, np.float64)
        rc = lib().orc_solve_lcp(self._h, full_cycles, v_cycles, pre, post, constraint_levels, coarse_sweeps,
                                 coarse_tol, _p(p), _p(info))
        if rc != 0:
            raise ValueError("the LCP solve needs embedded solids")
        return p, dict(zip(("cycles", "max_residual", "l2_residual", "b_norm", "at_bound"), info.tolist()))

    def level_faces(self, level: int) -> np.ndarray:
        (nx, ny, nz), _, _ = self.level_dims(level)
        out = np.empty((3, nz, ny, nx), np.float32)
        lib().orc_level_faces(self._h, int(level), _p(out))
        return out

    def fcycle(self, r, pre: int = 1, post: int = 1, first_block: int = 1):
        """One full cycle from a zero guess; levels from `first_block` on take one V-cycle."""
        nx, ny, nz = self.n
        r = np.ascontiguousarray(r, np.float64).reshape(nz, ny, nx)
        z = np.zeros_like(r)
        lib().orc_fcycle(self._h, _p(r), _p(z), pre, post, int(first_block))
        return z

    def solve_jacobi(self, rel_tol=1e-10, abs_tol=1e-12, max_iter=None):
        nx, ny, nz = self.n
        p = np.zeros((nz, ny, nx), np.float64)
        info = np.zeros(8, np.float64)
        if max_iter is None:
            max_iter = max(64, 4 * nx * ny * nz)
        lib().orc_solve_jacobi(self._h, rel_tol, abs_tol, int(max_iter), _p(p), _p(info))
        return p, dict(zip(INFO_KEYS, info.tolist()))

    def solve_mgpcg(self, rel_tol=1e-10, abs_tol=0.0, max_iter=200, pre=1, post=1):
        nx, ny, nz = self.n
        p = np.zeros((nz, ny, nx), np.float64)
        info = np.zeros(8, np.float64)
        lib().orc_solve_mgpcg(self._h, rel_tol, abs_tol, int(max_iter), pre, post, _p(p), _p(info))
        return p, dict(zip(INFO_KEYS, info.tolist()))

    def solve_fcg(self, rel_tol=1e-10, abs_tol=0.0, max_iter=200, pre=1, post=1, first_block=1):
        """Flexible PCG (Polak-Ribiere beta) with the full cycle as preconditioner."""
        nx, ny, nz = self.n
        p = np.zeros((nz, ny, nx), np.float64)
        info = np.zeros(8, np.float64)
        lib().orc_solve_fcg(self._h, rel_tol, abs_tol, int(max_iter), pre, post, int(first_block), _p(p), _p(info))
        return p, dict(zip(INFO_KEYS, info.tolist()))

    def grad_subtract(self, p):
        nx, ny, nz = self.n
        p = np.ascontiguousarray(p, np.float64).reshape(nz, ny, nx)
        uo = np.zeros((nz, ny, nx + 1), np.float32)
        vo = np.zeros((nz, ny + 1, nx), np.float32)
        wo = np.zeros((nz + 1, ny, nx), np.float32)
        out = np.zeros(4, np.float64)
        lib().orc_grad_subtract(self._h, _p(p), _p(uo), _p(vo), _p(wo), _p(out))
        return (uo, vo, wo), {"max_div_before": out[0], "max_div_after": out[1],
                              "l2_div_before": out[2], "l2_div_after": out[3]}

    def pressure_si(self, p_cells):
        """Dimensional pressure (Pa) from finest-cell-unit pressure."""
        return p_cells * self.rho * self.h / self.dt


def extrapolate_velocity(nx, ny, nz, h, open_top, vof, u, v, w, open_frac=None, fx=None, fy=None, fz=None):
    """The velocity extrapolation restatement (float32, in the device's
    operation order): returns (u, v, w) extrapolated copies, the open faces
    holding a value, and the band passes that changed the state."""
    f32 = lambda a: np.ascontiguousarray(a, np.float32) if a is not None else None
    vof, u, v, w = (f32(a) for a in (vof, u, v, w))
    u, v, w = u.copy(), v.copy(), w.copy()
    open_frac, fx, fy, fz = (f32(a) for a in (open_frac, fx, fy, fz))
    ran = ctypes.c_int(0)
    filled = lib().orc_extrapolate(nx, ny, nz, float(h), int(open_top), _p(vof), _p(open_frac), _p(fx), _p(fy),
                                   _p(fz), _p(u), _p(v), _p(w), ctypes.byref(ran))
    return (u, v, w), int(filled), int(ran.value)


def transport_density(nx, ny, nz, h, dt, open_top, vof, u, v, w, gamma=None, diffusion=1, sharpening=True,
                      mass_return=True, strength=1.0, distance=2.1, stages=False):
    """The CM12 density transport restatement (float32, in the device's
    operation order).  Returns (rho, gamma) after the step, and with stages a
    dict of the intermediate fields (rho and gamma after the gather, rho after
    the diffusion, the sharpening delta)."""
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    rho = f32(vof).copy().reshape(nz, ny, nx)
    g = np.ones((nz, ny, nx), np.float32) if gamma is None else f32(gamma).copy().reshape(nz, ny, nx)
    u, v, w = f32(u), f32(v), f32(w)
    st = np.empty((4, nz, ny, nx), np.float32) if stages else None
    # the reference's option clamps (webgpu-uniform-reference.ts:374-377)
    diffusion = int(min(7, max(0, diffusion)))
    strength = float(np.float32(min(2.0, max(0.25, strength))))
    distance = float(np.float32(min(3.1, max(0.1, distance))))
    lib().orc_transport(nx, ny, nz, float(np.float32(h)), float(np.float32(dt)), int(open_top), _p(u), _p(v), _p(w),
                        _p(rho), _p(g), diffusion, int(bool(sharpening)), int(bool(mass_return)), strength, distance,
                        _p(st))
    if stages:
        return rho, g, {"rho_gather": st[0], "gamma_gather": st[1], "rho_diffused": st[2], "delta": st[3]}
    return rho, g

