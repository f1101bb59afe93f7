"""ctypes binding of the C-ABI in include/ash3d_b200.h.

The shared library is built in-tree (``libash3d_b200.so`` next to this file)
by ``build.py``.  There is no CPU path: loading fails loudly when the library
is missing, and every call that fails raises ``A3GError`` with the library's
own message.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libash3d_b200.so"

A3G_OK = 0
ERR_NAMES = {
    1: "A3G_ERR_ARG", 2: "A3G_ERR_CUDA", 3: "A3G_ERR_NOMEM", 4: "A3G_ERR_BC_CODE",
    5: "A3G_ERR_SUBGRID", 6: "A3G_ERR_PIVOT", 7: "A3G_ERR_STATE",
    8: "A3G_ERR_UNSUPPORTED", 9: "A3G_ERR_NONFINITE", 10: "A3G_ERR_TIMEOUT",
}
LIMITERS = {"none": 0, "laxwen": 1, "bw": 2, "fromm": 3, "minmod": 4, "superbee": 5, "mc": 6}

# every symbol include/ash3d_b200.h declares (checked by the CPU test suite)
EXPORTED = [
    "a3g_default_params", "a3g_abi_version", "a3g_last_error", "a3g_create", "a3g_destroy",
    "a3g_sync", "a3g_device_bytes", "a3g_set_geometry", "a3g_set_diffusivity",
    "a3g_set_fall_velocity", "a3g_set_aloft", "a3g_set_winds", "a3g_set_met_steps",
    "a3g_interp_winds", "a3g_upload_concen", "a3g_download_concen", "a3g_upload_outflow",
    "a3g_download_outflow", "a3g_output_ashcon", "a3g_restart_load", "a3g_step_prologue",
    "a3g_set_dt", "a3g_add_source_column",
    "a3g_set_bc", "a3g_advect_horz", "a3g_advect_x", "a3g_advect_y", "a3g_advect_vert",
    "a3g_diffuse_horz", "a3g_diffuse_vert", "a3g_adjust_dt", "a3g_timestep_totals",
    "a3g_get_minmax_index", "a3g_set_subgrid", "a3g_get_subgrid", "a3g_step",
    "a3g_kernel_launches", "a3g_get_stream", "a3g_kernel_timing", "a3g_kernel_times",
    "a3g_cfl_maxima", "a3g_adjust_dt_from_maxima", "a3g_cfl_maxima_device",
    "a3g_adjust_dt_device_maxima_async", "a3g_selftest_div", "a3g_set_variant",
    "a3g_get_variant", "a3g_mass_aloft_noalloc",
    "a3g_adj_enable", "a3g_adj_zero", "a3g_adj_set_lambda", "a3g_adj_get_lambda",
    "a3g_adj_set_lambda_dep", "a3g_adj_get_lambda_dep", "a3g_adj_advect_x", "a3g_adj_advect_y",
    "a3g_adj_advect_vert", "a3g_adj_diffuse_horz", "a3g_adj_diffuse_vert", "a3g_adj_step",
    "a3g_adj_vent_column", "a3g_cloud_load", "a3g_adj_add_cloud_load", "a3g_snapshot_alloc",
    "a3g_snapshot_save", "a3g_snapshot_load", "a3g_set_output_params", "a3g_output_reset",
    "a3g_output_vars", "a3g_set_topo", "a3g_set_umbrella", "a3g_add_umbrella_winds",
    "a3g_add_source_umbrella", "a3g_vprofiles", "a3g_adjust_dt_async", "a3g_wait_dt",
    "a3g_timestep_totals_async", "a3g_totals_get", "a3g_set_source_pulses", "a3g_add_source_scheduled",
    "a3g_prefetch_met_step", "a3g_advance_met_step", "a3g_met_prefetch_fence",
    "a3g_add_source_column_devdt", "a3g_adj_grad_reset", "a3g_adj_vent_accumulate", "a3g_adj_grad_get",
    "a3g_set_fall_velocity_meso", "a3g_cfl_maxima_meso", "a3g_adjust_dt_meso",
    "a3g_adjust_dt_meso_from_maxima", "a3g_fast_dt_async",
    "a3g_inv_setup", "a3g_forward_checkpointed", "a3g_adjoint", "a3g_tangent_linear",
    "a3g_inv_observations", "a3g_checkpoint_cost",
]
KERNEL_CLASSES = ["advect_x", "advect_y", "advect_z", "diff_x", "diff_y", "diff_z", "cn_table",
                  "cn_solve_x", "cn_solve_y", "cn_solve_z", "cfl", "totals", "winds", "other",
                  "adjoint"]


class A3GError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class GridDesc(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("ns", C.c_int32),
                ("periodic", C.c_int32), ("latlon", C.c_int32), ("dx", C.c_double), ("dy", C.c_double)]


class InvDesc(C.Structure):
    _fields_ = [("ivent", C.c_int32), ("jvent", C.c_int32), ("nbins", C.c_int32), ("misfit", C.c_int32),
                ("fast_dt", C.c_int32), ("load_from", C.c_int32), ("dep_from", C.c_int32), ("adj_from", C.c_int32),
                ("sim_hours", C.c_double), ("snapshot_bytes", C.c_double), ("met_cache", C.c_int32)]


MISFIT_LOAD, MISFIT_DEPOSIT = 1, 2
FP = C.POINTER(C.c_float)
MET_PROVIDER = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.POINTER(FP), C.POINTER(FP), C.POINTER(FP))


class Params(C.Structure):
    _fields_ = [("limiter", C.c_int32), ("use_cn", C.c_int32), ("use_diffusion", C.c_int32),
                ("fast_subgrid", C.c_int32), ("nocycle", C.c_int32), ("zscaling_id", C.c_int32),
                ("cfl", C.c_double), ("dt_min", C.c_double), ("dt_max", C.c_double),
                ("imp_fac", C.c_double), ("imp_dt_fac", C.c_double), ("eps_thresh", C.c_double),
                ("eps_small", C.c_double), ("cloudcon_grid_thresh", C.c_double),
                ("magma_density", C.c_double)]


_lib = None


def load(path: os.PathLike | str | None = None) -> C.CDLL:
    """Loads the in-tree library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = pathlib.Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(
            f"{p} is missing: build it with `python __graft_entry__.py build` "
            "(the transport path has no CPU fallback)")
    lib = C.CDLL(str(p))
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    F = C.POINTER(C.c_float)
    I = C.POINTER(C.c_int32)
    sig = {
        "a3g_default_params": (None, [C.POINTER(Params)]),
        "a3g_abi_version": (C.c_int, []),
        "a3g_last_error": (C.c_char_p, []),
        "a3g_create": (C.c_int, [C.POINTER(GridDesc), C.POINTER(Params), C.c_int, C.POINTER(P)]),
        "a3g_destroy": (C.c_int, [P]),
        "a3g_sync": (C.c_int, [P]),
        "a3g_device_bytes": (C.c_int, [P, C.POINTER(C.c_size_t)]),
        "a3g_set_geometry": (C.c_int, [P, D, D, D, D, D]),
        "a3g_set_diffusivity": (C.c_int, [P, D, D, D]),
        "a3g_set_fall_velocity": (C.c_int, [P, D]),
        "a3g_set_aloft": (C.c_int, [P, I]),
        "a3g_set_winds": (C.c_int, [P, D, D, D]),
        "a3g_set_met_steps": (C.c_int, [P, F, F, F, F, F, F]),
        "a3g_interp_winds": (C.c_int, [P, C.c_double]),
        "a3g_set_topo": (C.c_int, [P, D, D, D, D, D, C.c_double]),
        "a3g_set_umbrella": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, D]),
        "a3g_add_umbrella_winds": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, D, D]),
        "a3g_add_source_umbrella": (C.c_int, [P, D, C.c_double]),
        "a3g_vprofiles": (C.c_int, [P, C.c_int32, I, I, D, I]),
        "a3g_adjust_dt_async": (C.c_int, [P, C.c_double, C.c_double, C.c_double]),
        "a3g_wait_dt": (C.c_int, [P, D]),
        "a3g_timestep_totals_async": (C.c_int, [P, C.POINTER(C.c_int64)]),
        "a3g_totals_get": (C.c_int, [P, C.c_int64, D, D]),
        "a3g_set_source_pulses": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, D, D, D, D, D]),
        "a3g_add_source_scheduled": (C.c_int, [P, C.c_double]),
        "a3g_prefetch_met_step": (C.c_int, [P, F, F, F]),
        "a3g_advance_met_step": (C.c_int, [P]),
        "a3g_met_prefetch_fence": (C.c_int, [P]),
        "a3g_add_source_column_devdt": (C.c_int, [P, C.c_int32, C.c_int32, D]),
        "a3g_adj_grad_reset": (C.c_int, [P, C.c_int32]),
        "a3g_adj_vent_accumulate": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, C.c_double]),
        "a3g_adj_grad_get": (C.c_int, [P, D]),
        "a3g_upload_concen": (C.c_int, [P, D]),
        "a3g_download_concen": (C.c_int, [P, D]),
        "a3g_upload_outflow": (C.c_int, [P, D, D, D, D, D, D]),
        "a3g_download_outflow": (C.c_int, [P, D, D, D, D, D, D, D]),
        # FP32 arrays as addresses: host (numpy) or device (a tensor's data_ptr)
        "a3g_output_ashcon": (C.c_int, [P, P, P]),
        "a3g_restart_load": (C.c_int, [P, P, P]),
        "a3g_step_prologue": (C.c_int, [P]),
        "a3g_set_dt": (C.c_int, [P, C.c_double]),
        "a3g_add_source_column": (C.c_int, [P, C.c_int32, C.c_int32, D, C.c_double]),
        "a3g_set_bc": (C.c_int, [P, C.c_int32]),
        "a3g_advect_horz": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
        "a3g_advect_x": (C.c_int, [P]),
        "a3g_advect_y": (C.c_int, [P]),
        "a3g_advect_vert": (C.c_int, [P]),
        "a3g_diffuse_horz": (C.c_int, [P, C.c_int32]),
        "a3g_diffuse_vert": (C.c_int, [P]),
        "a3g_adjust_dt": (C.c_int, [P, C.c_double, C.c_double, C.c_double, D]),
        "a3g_timestep_totals": (C.c_int, [P, D, D]),
        "a3g_cfl_maxima": (C.c_int, [P, D]),
        "a3g_set_variant": (C.c_int, [P, C.c_int32, C.c_int32]),
        "a3g_get_variant": (C.c_int, [P, C.c_int32, C.POINTER(C.c_int32)]),
        "a3g_mass_aloft_noalloc": (C.c_int, [C.c_int, D, D, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                             C.c_int64, D, C.c_void_p]),
        "a3g_selftest_div": (C.c_int, [C.c_int, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64)]),
        "a3g_adjust_dt_from_maxima": (C.c_int, [P, D, C.c_int32, C.c_double, C.c_double, C.c_double, D]),
        "a3g_cfl_maxima_device": (C.c_int, [P, C.POINTER(D)]),
        "a3g_adjust_dt_device_maxima_async": (C.c_int, [P, C.c_int32, C.c_double, C.c_double, C.c_double]),
        "a3g_set_fall_velocity_meso": (C.c_int, [P, F, C.c_int32]),
        "a3g_cfl_maxima_meso": (C.c_int, [P, C.c_int32, D]),
        "a3g_adjust_dt_meso": (C.c_int, [P, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, D]),
        "a3g_adjust_dt_meso_from_maxima": (C.c_int, [P, D, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                                     C.c_double, D]),
        "a3g_fast_dt_async": (C.c_int, [P, C.c_double, C.c_double, C.c_double, C.c_double]),
        "a3g_inv_setup": (C.c_int, [P, C.POINTER(InvDesc), MET_PROVIDER, C.c_void_p, D, D]),
        "a3g_forward_checkpointed": (C.c_int, [P, D, D, C.POINTER(C.c_int32)]),
        "a3g_adjoint": (C.c_int, [P, D, D, D]),
        "a3g_tangent_linear": (C.c_int, [P, D, D, D, D]),
        "a3g_inv_observations": (C.c_int, [P, D, D, C.POINTER(C.c_int64)]),
        "a3g_checkpoint_cost": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
        "a3g_get_minmax_index": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, I]),
        "a3g_set_subgrid": (C.c_int, [P, I]),
        "a3g_get_subgrid": (C.c_int, [P, I]),
        "a3g_step": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, D]),
        "a3g_kernel_launches": (C.c_int, [P, C.POINTER(C.c_uint64)]),
        "a3g_get_stream": (C.c_int, [P, C.POINTER(C.c_void_p)]),
        "a3g_kernel_timing": (C.c_int, [P, C.c_int32]),
        "a3g_kernel_times": (C.c_int, [P, D, C.POINTER(C.c_uint64)]),
        "a3g_adj_enable": (C.c_int, [P]), "a3g_adj_zero": (C.c_int, [P]),
        "a3g_adj_set_lambda": (C.c_int, [P, D]), "a3g_adj_get_lambda": (C.c_int, [P, D]),
        "a3g_adj_set_lambda_dep": (C.c_int, [P, D]), "a3g_adj_get_lambda_dep": (C.c_int, [P, D]),
        "a3g_adj_advect_x": (C.c_int, [P]), "a3g_adj_advect_y": (C.c_int, [P]),
        "a3g_adj_advect_vert": (C.c_int, [P]), "a3g_adj_diffuse_horz": (C.c_int, [P, C.c_int32]),
        "a3g_adj_diffuse_vert": (C.c_int, [P]), "a3g_adj_step": (C.c_int, [P, C.c_int32]),
        "a3g_adj_vent_column": (C.c_int, [P, C.c_int32, C.c_int32, D]),
        "a3g_cloud_load": (C.c_int, [P, D]), "a3g_adj_add_cloud_load": (C.c_int, [P, D]),
        "a3g_snapshot_alloc": (C.c_int, [P, C.c_int32]), "a3g_snapshot_save": (C.c_int, [P, C.c_int32]),
        "a3g_snapshot_load": (C.c_int, [P, C.c_int32]),
        "a3g_set_output_params": (C.c_int, [P, D, C.c_double, C.c_double, C.c_double, C.c_double]),
        "a3g_output_reset": (C.c_int, [P]),
        "a3g_output_vars": (C.c_int, [P, C.c_double, D, D, D, D, I, D, I, D, D, D]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != A3G_OK:
        msg = _lib.a3g_last_error().decode() if _lib is not None else ""
        raise A3GError(rc, msg)


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.flags.c_contiguous), "need a contiguous float64 array"
    return a.ctypes.data_as(C.POINTER(C.c_double))


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and (a.flags.f_contiguous or a.flags.c_contiguous)
    return a.ctypes.data_as(C.POINTER(C.c_float))


def iptr(a: np.ndarray):
    assert a.dtype == np.int32
    return a.ctypes.data_as(C.POINTER(C.c_int32))
