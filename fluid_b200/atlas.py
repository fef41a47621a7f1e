"""Sparse brick-atlas pressure projection (brick-compact storage, 8^3 bricks).

Python face of fluid_pp_atlas_* (include/fluid_pp.h), the default adaptive
method's projection (lib/methods/adaptive-mass/webgpu-sparse-cm12-resident.ts;
its CPU statement projectSparseAtlasVelocity in
sparse-atlas-composite-projection.ts:978-1566) for atlases whose bricks all
carry the finest resolution.  Bricks are given as coordinates on the 8-cell
brick grid with their density [z][y][x] and their faces (per brick the MAC
layout u [8][8][9], v [8][9][8], w [9][8][8]).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import AtlasConfig, Receipt, load, ptr
from .projector import FluidError, solve_opts

RES = 8
FACES = (RES + 1) * RES * RES


def _check(rc: int, handle, what: str):
    if rc == _abi.OK:
        return
    L = load()
    msg = L.fluid_pp_atlas_last_error(handle).decode()
    if rc == _abi.INVALID_ARG:
        raise ValueError(msg or what)
    if rc == _abi.OOM:
        raise MemoryError(msg or what)
    raise FluidError(f"{_abi.STATUS_NAMES.get(rc, rc)}: {msg or what}")


def plan_atlas(dims, coords, density=None) -> dict:
    """Host planner: cells per level of the block hierarchy and the liquid
    components without a face to air."""
    nx, ny, nz = (int(v) for v in dims)
    c = np.ascontiguousarray(np.asarray(coords, np.int32).reshape(-1, 3))
    count = ctypes.c_int()
    cells = np.zeros(16, np.int64)
    comps, comp_cells = ctypes.c_int(), ctypes.c_int()
    d = None if density is None else np.ascontiguousarray(np.asarray(density, np.float32).reshape(len(c), -1))
    rc = load().fluid_pp_atlas_plan(nx, ny, nz, len(c), ptr(c), ptr(d) if d is not None else None,
                                     ctypes.byref(count), ptr(cells), ctypes.byref(comps), ctypes.byref(comp_cells))
    _check(rc, None, "plan")
    out = {"level_cells": [int(v) for v in cells[:count.value]]}
    if d is not None:
        out["unanchored_components"] = comps.value
        out["unanchored_cells"] = comp_cells.value
    return out


class AtlasProjector:
    """One sparse brick atlas resident on the device."""

    def __init__(self, dims, spacing: float, rho: float = 1000.0, device: int = 0):
        self.dims = tuple(int(v) for v in dims)
        self.h = float(spacing)
        self.rho = float(rho)
        cfg = AtlasConfig(*self.dims, self.h, self.rho, int(device))
        h = ctypes.c_void_p()
        _check(load().fluid_pp_atlas_create(ctypes.byref(cfg), ctypes.byref(h)), None, "create")
        self._h = h
        self.nbricks = 0

    def set_stream(self, stream: int):
        _check(load().fluid_pp_atlas_set_stream(self._h, ctypes.c_void_p(stream)), self._h, "set_stream")

    def set_graphs(self, on: bool):
        """The PCG iteration as a CUDA graph (default on); off for profilers."""
        _check(load().fluid_pp_atlas_set_graphs(self._h, int(bool(on))), self._h, "set_graphs")

    def upload(self, coords, density, faces):
        """coords [nb][3] brick coordinates; density [nb][8][8][8]; faces [nb][3][576]."""
        c = np.ascontiguousarray(np.asarray(coords, np.int32).reshape(-1, 3))
        nb = len(c)
        d = np.ascontiguousarray(np.asarray(density, np.float32).reshape(nb, RES ** 3))
        f = np.ascontiguousarray(np.asarray(faces, np.float32).reshape(nb, 3 * FACES))
        _check(load().fluid_pp_atlas_upload(self._h, nb, ptr(c), ptr(d), ptr(f)), self._h, "upload")
        self.nbricks = nb

    def project(self, dt: float, cycle: str = "v", **opts) -> dict:
        """cycle "v": one V-cycle on the brick hierarchy per PCG iteration,
        two red-black sweeps before and after the coarse correction unless
        pre_sweeps / post_sweeps say otherwise; "jacobi": the reference's
        diagonal preconditioner."""
        o = solve_opts(**{"pre_sweeps": 2, "post_sweeps": 2, **opts})
        o.cycle = {"v": 0, "jacobi": 2}[cycle]
        r = Receipt()
        rc = load().fluid_pp_atlas_project(self._h, float(dt), ctypes.byref(o), ctypes.byref(r))
        if rc not in (_abi.OK, _abi.NONCONVERGENCE, _abi.NONFINITE):
            _check(rc, self._h, "project")
        return r.as_dict()

    def download(self):
        """(pressure [nb][8][8][8] in Pa, faces [nb][3][576])."""
        p = np.empty((self.nbricks, RES, RES, RES), np.float32)
        f = np.empty((self.nbricks, 3, FACES), np.float32)
        _check(load().fluid_pp_atlas_download(self._h, ptr(p), ptr(f)), self._h, "download")
        return p, f

    def destroy(self):
        if self._h:
            load().fluid_pp_atlas_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def bricks_from_dense(vof, u, v, w, coords):
    """Brick-compact arrays of a dense state: density [nb][8][8][8] and faces
    [nb][3][576] of the given bricks (the dense MAC layouts u [nz][ny][nx+1],
    v [nz][ny+1][nx], w [nz+1][ny][nx])."""
    c = np.asarray(coords, np.int64).reshape(-1, 3)
    nb = len(c)
    dens = np.empty((nb, RES, RES, RES), np.float32)
    faces = np.empty((nb, 3, FACES), np.float32)
    for k, (bx, by, bz) in enumerate(c):
        x0, y0, z0 = bx * RES, by * RES, bz * RES
        dens[k] = vof[z0:z0 + RES, y0:y0 + RES, x0:x0 + RES]
        faces[k, 0] = u[z0:z0 + RES, y0:y0 + RES, x0:x0 + RES + 1].ravel()
        faces[k, 1] = v[z0:z0 + RES, y0:y0 + RES + 1, x0:x0 + RES].ravel()
        faces[k, 2] = w[z0:z0 + RES + 1, y0:y0 + RES, x0:x0 + RES].ravel()
    return dens, faces
