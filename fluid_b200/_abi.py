"""ctypes binding of ``include/fluid_pp.h`` (``fluid_b200/_lib/libfluid_pp.so``).

There is no fallback: if the CUDA library is missing the import fails loudly.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libfluid_pp.so")

OK, INVALID_ARG, OOM, NONFINITE, NONCONVERGENCE, TIMEOUT, CUDA, UNSUPPORTED = range(8)
STATUS_NAMES = {OK: "OK", INVALID_ARG: "INVALID_ARG", OOM: "OOM", NONFINITE: "NONFINITE",
                NONCONVERGENCE: "NONCONVERGENCE", TIMEOUT: "TIMEOUT", CUDA: "CUDA", UNSUPPORTED: "UNSUPPORTED"}
PRECISIONS = {"fp32": 0, "fp16": 1, "bf16": 2}
MAX_LEVELS = 24

# Every symbol include/fluid_pp.h declares (checked by the CPU test suite).
EXPORTS = (
    "fluid_pp_plan_hierarchy", "fluid_pp_create", "fluid_pp_destroy", "fluid_pp_set_stream",
    "fluid_pp_upload_state", "fluid_pp_upload_state_device", "fluid_pp_project", "fluid_pp_project_async",
    "fluid_pp_upload_solids", "fluid_pp_get_level_faces", "fluid_pp_lcp_opts_default", "fluid_pp_project_lcp",
    "fluid_pp_extrapolate_velocity", "fluid_pp_tall_set_graphs", "fluid_pp_transport_opts_default",
    "fluid_pp_transport_density", "fluid_pp_set_gamma", "fluid_pp_get_gamma", "fluid_pp_get_vof",
    "fluid_pp_atlas_plan", "fluid_pp_atlas_create", "fluid_pp_atlas_destroy", "fluid_pp_atlas_set_stream", "fluid_pp_atlas_set_graphs",
    "fluid_pp_atlas_upload", "fluid_pp_atlas_project", "fluid_pp_atlas_download", "fluid_pp_atlas_last_error",
    "fluid_pp_receipt_read", "fluid_pp_download", "fluid_pp_device_arrays", "fluid_pp_last_error",
    "fluid_pp_prepare", "fluid_pp_level_dims", "fluid_pp_get_level", "fluid_pp_get_rhs",
    "fluid_pp_apply_operator", "fluid_pp_apply_vcycle", "fluid_pp_apply_fcycle", "fluid_pp_get_pressure_cells",
    "fluid_pp_batch_create", "fluid_pp_batch_destroy", "fluid_pp_batch_project",
    "fluid_pp_kernel_launches", "fluid_pp_set_profiling", "fluid_pp_profile_read",
    "fluid_pp_batch_set_profiling", "fluid_pp_batch_profile_read",
    "fluid_pp_apply_operator_noalloc",
    "fluid_pp_tall_choose_base", "fluid_pp_tall_limit_bases", "fluid_pp_tall_plan", "fluid_pp_tall_create",
    "fluid_pp_tall_destroy", "fluid_pp_tall_set_stream", "fluid_pp_tall_upload_state",
    "fluid_pp_tall_upload_state_device", "fluid_pp_tall_project", "fluid_pp_tall_download",
    "fluid_pp_tall_prepare", "fluid_pp_tall_get_rhs", "fluid_pp_tall_get_labels", "fluid_pp_tall_apply_operator",
    "fluid_pp_tall_get_pressure", "fluid_pp_tall_last_error", "fluid_pp_required_bytes",
    "fluid_pp_tall_required_bytes", "fluid_pp_batch_set_graphs",
    "fluid_pp_set_allocation_cache", "fluid_pp_allocation_cache_bytes", "fluid_pp_reserve_allocation",
    "fluid_pp_tall_project_begin", "fluid_pp_tall_project_continue", "fluid_pp_tall_project_end",
    "fluid_pp_batch_project_async", "fluid_pp_batch_receipts_read", "fluid_pp_download_async",
    "fluid_pp_synchronize", "fluid_pp_batch_tuning_default", "fluid_pp_batch_create_tuned",
    "fluid_pp_batch_upload_state", "fluid_pp_batch_download_async", "fluid_pp_tall_solve_rhs",
)
STAGES = ("reset", "label", "coarsen", "bake", "factor", "init", "smooth0", "smoothc", "residual0", "residualc",
          "restrict0", "restrictc", "coarse", "prolong0", "prolongc", "dot", "dir", "spmv", "update", "true",
          "grad", "receipt", "down0", "downc", "up0", "upc", "dirspmv")


class Config(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("h", ctypes.c_float),
                ("rho", ctypes.c_float), ("open_top", ctypes.c_int), ("precision", ctypes.c_int),
                ("device", ctypes.c_int)]


class TallConfig(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("nz", ctypes.c_int), ("fine_ny", ctypes.c_int), ("band", ctypes.c_int),
                ("h", ctypes.c_float), ("rho", ctypes.c_float), ("precision", ctypes.c_int),
                ("device", ctypes.c_int)]


class SolveOpts(ctypes.Structure):
    _fields_ = [("rel_tol", ctypes.c_double), ("abs_tol", ctypes.c_double), ("max_iters", ctypes.c_int),
                ("pre_sweeps", ctypes.c_int), ("post_sweeps", ctypes.c_int),
                ("true_residual_every", ctypes.c_int), ("warm_start", ctypes.c_int),
                ("rel_tol_inf", ctypes.c_double), ("cycle", ctypes.c_int)]


class LcpOpts(ctypes.Structure):
    _fields_ = [("full_cycles", ctypes.c_int), ("v_cycles", ctypes.c_int), ("pre_sweeps", ctypes.c_int),
                ("post_sweeps", ctypes.c_int), ("constraint_levels", ctypes.c_int), ("coarse_sweeps", ctypes.c_int),
                ("coarse_tol", ctypes.c_double), ("warm_start", ctypes.c_int)]


class AtlasConfig(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("h", ctypes.c_float),
                ("rho", ctypes.c_float), ("device", ctypes.c_int)]


class TransportOpts(ctypes.Structure):
    _fields_ = [("gamma_diffusion_iterations", ctypes.c_int), ("sharpening", ctypes.c_int),
                ("sharpening_mass_return", ctypes.c_int), ("sharpening_strength", ctypes.c_float),
                ("sharpening_distance", ctypes.c_float)]


class TransportReceipt(ctypes.Structure):
    _fields_ = [("mass_before", ctypes.c_double), ("mass_after", ctypes.c_double), ("rho_min", ctypes.c_float),
                ("rho_max", ctypes.c_float)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class BatchTuning(ctypes.Structure):
    _fields_ = [("fill_tiles", ctypes.c_int), ("chunk_planes", ctypes.c_int), ("box_shape", ctypes.c_int),
                ("parts", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Receipt(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("iterations", ctypes.c_int), ("liquid_cells", ctypes.c_int),
                ("levels", ctypes.c_int), ("b_norm", ctypes.c_double), ("rel_residual", ctypes.c_double),
                ("true_rel_residual", ctypes.c_double), ("max_div_before", ctypes.c_double),
                ("max_div_after", ctypes.c_double), ("l2_div_before", ctypes.c_double),
                ("l2_div_after", ctypes.c_double)]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["status_name"] = STATUS_NAMES.get(self.status, str(self.status))
        return d


_lib = None


def load():
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"fluid_b200 CUDA library missing: {LIB_PATH} (run python -m fluid_b200.build)")
    L = ctypes.CDLL(LIB_PATH)
    vp, ci, cf = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    pi = ctypes.POINTER(ctypes.c_int)
    L.fluid_pp_plan_hierarchy.argtypes = [ci, ci, ci, pi, vp, pi, pi, pi]
    L.fluid_pp_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(vp)]
    L.fluid_pp_destroy.argtypes = [vp]
    L.fluid_pp_destroy.restype = None
    L.fluid_pp_set_stream.argtypes = [vp, vp]
    L.fluid_pp_upload_state.argtypes = [vp, vp, vp, vp, vp]
    L.fluid_pp_upload_solids.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
    L.fluid_pp_get_level_faces.argtypes = [vp, ci, vp]
    L.fluid_pp_lcp_opts_default.argtypes = [vp]
    L.fluid_pp_lcp_opts_default.restype = None
    L.fluid_pp_project_lcp.argtypes = [vp, ctypes.c_float, vp, vp]
    L.fluid_pp_extrapolate_velocity.argtypes = [vp, vp]
    L.fluid_pp_tall_set_graphs.argtypes = [vp, ci]
    L.fluid_pp_transport_opts_default.argtypes = [vp]
    L.fluid_pp_transport_opts_default.restype = None
    L.fluid_pp_transport_density.argtypes = [vp, cf, vp, vp]
    L.fluid_pp_set_gamma.argtypes = [vp, vp]
    L.fluid_pp_get_gamma.argtypes = [vp, vp]
    L.fluid_pp_get_vof.argtypes = [vp, vp]
    L.fluid_pp_atlas_plan.argtypes = [ci, ci, ci, ci, vp, vp, vp, vp, vp, vp]
    L.fluid_pp_atlas_create.argtypes = [vp, vp]
    L.fluid_pp_atlas_destroy.argtypes = [vp]
    L.fluid_pp_atlas_destroy.restype = None
    L.fluid_pp_atlas_set_stream.argtypes = [vp, vp]
    L.fluid_pp_atlas_set_graphs.argtypes = [vp, ci]
    L.fluid_pp_atlas_upload.argtypes = [vp, ci, vp, vp, vp]
    L.fluid_pp_atlas_project.argtypes = [vp, cf, vp, vp]
    L.fluid_pp_atlas_download.argtypes = [vp, vp, vp]
    L.fluid_pp_atlas_last_error.argtypes = [vp]
    L.fluid_pp_atlas_last_error.restype = ctypes.c_char_p
    L.fluid_pp_upload_state_device.argtypes = [vp, vp, vp, vp, vp]
    L.fluid_pp_project.argtypes = [vp, cf, ctypes.POINTER(SolveOpts), ctypes.POINTER(Receipt)]
    L.fluid_pp_project_async.argtypes = [vp, cf, ctypes.POINTER(SolveOpts)]
    L.fluid_pp_receipt_read.argtypes = [vp, ctypes.POINTER(Receipt)]
    L.fluid_pp_download.argtypes = [vp, vp, vp, vp, vp]
    L.fluid_pp_device_arrays.argtypes = [vp] + [ctypes.POINTER(vp)] * 5
    L.fluid_pp_last_error.argtypes = [vp]
    L.fluid_pp_last_error.restype = ctypes.c_char_p
    L.fluid_pp_prepare.argtypes = [vp, cf]
    L.fluid_pp_level_dims.argtypes = [vp, ci, vp]
    L.fluid_pp_get_level.argtypes = [vp, ci, vp, vp, vp]
    L.fluid_pp_get_rhs.argtypes = [vp, vp]
    L.fluid_pp_apply_operator.argtypes = [vp, vp, vp]
    L.fluid_pp_apply_vcycle.argtypes = [vp, vp, vp, ci, ci]
    L.fluid_pp_apply_fcycle.argtypes = [vp, vp, vp, ci, ci, vp]
    L.fluid_pp_get_pressure_cells.argtypes = [vp, vp]
    L.fluid_pp_batch_create.argtypes = [ctypes.POINTER(vp), ci, ctypes.POINTER(vp)]
    L.fluid_pp_batch_destroy.argtypes = [vp]
    L.fluid_pp_batch_destroy.restype = None
    L.fluid_pp_batch_project.argtypes = [vp, vp, ctypes.POINTER(SolveOpts), ctypes.POINTER(Receipt)]
    L.fluid_pp_batch_project_async.argtypes = [vp, vp, ctypes.POINTER(SolveOpts)]
    L.fluid_pp_batch_upload_state.argtypes = [vp, vp, vp, vp, vp]
    L.fluid_pp_batch_download_async.argtypes = [vp, vp, vp, vp, vp]
    L.fluid_pp_batch_tuning_default.argtypes = [ctypes.POINTER(BatchTuning)]
    L.fluid_pp_batch_tuning_default.restype = None
    L.fluid_pp_batch_create_tuned.argtypes = [ctypes.POINTER(vp), ci, ctypes.POINTER(BatchTuning), ctypes.POINTER(vp)]
    L.fluid_pp_batch_receipts_read.argtypes = [vp, ctypes.POINTER(Receipt)]
    L.fluid_pp_download_async.argtypes = [vp, vp, vp, vp, vp]
    L.fluid_pp_synchronize.argtypes = [vp]
    L.fluid_pp_kernel_launches.argtypes = []
    L.fluid_pp_kernel_launches.restype = ctypes.c_ulonglong
    L.fluid_pp_set_profiling.argtypes = [vp, ci]
    L.fluid_pp_profile_read.argtypes = [vp, vp, vp, ci]
    L.fluid_pp_batch_set_profiling.argtypes = [vp, ci]
    L.fluid_pp_batch_set_graphs.argtypes = [vp, ci]
    L.fluid_pp_batch_profile_read.argtypes = [vp, vp, vp, ci]
    L.fluid_pp_apply_operator_noalloc.argtypes = [ci, ci, ci, vp, vp, vp, vp, vp, vp]
    L.fluid_pp_set_allocation_cache.argtypes = [ci, ctypes.c_ulonglong]
    L.fluid_pp_allocation_cache_bytes.argtypes = [ci, ctypes.POINTER(ctypes.c_ulonglong)]
    L.fluid_pp_reserve_allocation.argtypes = [ci, ctypes.c_ulonglong]
    L.fluid_pp_tall_choose_base.argtypes = [ci, ci, ci, ci, ci, ci]
    L.fluid_pp_tall_limit_bases.argtypes = [vp, ci, ci, ci, ci]
    L.fluid_pp_tall_plan.argtypes = [ci, ci, ci, ci, vp, pi, vp]
    L.fluid_pp_tall_create.argtypes = [ctypes.POINTER(TallConfig), vp, ctypes.POINTER(vp)]
    L.fluid_pp_tall_destroy.argtypes = [vp]
    L.fluid_pp_tall_destroy.restype = None
    L.fluid_pp_tall_set_stream.argtypes = [vp, vp]
    L.fluid_pp_tall_upload_state.argtypes = [vp, vp, vp, vp, vp]
    L.fluid_pp_tall_upload_state_device.argtypes = [vp, vp, vp, vp, vp]
    L.fluid_pp_tall_project.argtypes = [vp, cf, ctypes.POINTER(SolveOpts), ctypes.POINTER(Receipt)]
    L.fluid_pp_tall_project_begin.argtypes = [vp, cf, ctypes.POINTER(SolveOpts)]
    L.fluid_pp_tall_project_continue.argtypes = [vp, ci, ctypes.POINTER(ctypes.c_int)]
    L.fluid_pp_tall_project_end.argtypes = [vp, ctypes.POINTER(Receipt)]
    L.fluid_pp_tall_download.argtypes = [vp, vp, vp, vp, vp]
    L.fluid_pp_tall_prepare.argtypes = [vp, cf]
    L.fluid_pp_tall_get_rhs.argtypes = [vp, vp]
    L.fluid_pp_tall_get_labels.argtypes = [vp, ci, vp]
    L.fluid_pp_tall_apply_operator.argtypes = [vp, vp, vp]
    L.fluid_pp_tall_get_pressure.argtypes = [vp, vp]
    L.fluid_pp_tall_solve_rhs.argtypes = [vp, cf, vp, ctypes.POINTER(SolveOpts), vp, ctypes.POINTER(Receipt)]
    L.fluid_pp_tall_last_error.argtypes = [vp]
    L.fluid_pp_tall_last_error.restype = ctypes.c_char_p
    L.fluid_pp_required_bytes.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_ulonglong)]
    L.fluid_pp_tall_required_bytes.argtypes = [ctypes.POINTER(TallConfig), vp, ctypes.POINTER(ctypes.c_ulonglong)]
    _lib = L
    return L


def ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)
