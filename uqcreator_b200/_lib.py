"""ctypes binding of the C ABI in include/uqc.h (libuqc_b200.so, built in-tree).

There is no CPU fallback: if the extension is missing or a CUDA device is not
available, calls raise.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libuqc_b200.so"
_lib = None

UQC_OK = 0
ERRORS = {-1: "argument", -2: "config", -3: "cuda", -4: "not converged", -5: "memory", -6: "state", -7: "capacity"}
LAYOUT_REF, LAYOUT_STATE_MAJOR = 0, 1
FP64, MIXED = 0, 1
CELL_CODES = {0: "converged", 1: "max iterations", 2: "line search", 3: "not positive definite", 4: "non-finite"}

# every symbol include/uqc.h declares
EXPORTS = [
    "uqc_create_from_file", "uqc_create_from_string", "uqc_destroy", "uqc_last_error", "uqc_get_info",
    "uqc_set_precision", "uqc_set_newton", "uqc_get_tables", "uqc_get_geometry", "uqc_init_state",
    "uqc_upload_state", "uqc_download_state", "uqc_solve_closure", "uqc_cell_status", "uqc_step", "uqc_run",
    "uqc_mean_var", "uqc_closure_solve_host", "uqc_closure_solve_device", "uqc_last_timing", "uqc_device_state",
    "uqc_last_launch_count", "uqc_stream", "uqc_mesh_tri_jitter", "uqc_closure_solve_device_noalloc",
    "uqc_set_option", "uqc_step_async", "uqc_step_query", "uqc_device_bytes", "uqc_server_create",
    "uqc_server_destroy", "uqc_server_last_error", "uqc_server_submit", "uqc_server_progress",
    "uqc_server_request", "uqc_server_release", "uqc_server_request_error", "uqc_export_state", "uqc_write_vtk",
    "uqc_debug_mixed_inverse", "uqc_server_set_option", "uqc_solve_closure_cells", "uqc_moments_mean_var",
    "uqc_partition", "uqc_get_shard", "uqc_shard_buffers", "uqc_halo_pack", "uqc_step_phase",
    "uqc_config_defaults", "uqc_create_from_config", "uqc_step_host",
]
REQ_STATES = {0: "queued", 1: "running", 2: "done", 3: "failed"}
NOALLOC_MAX_CELLS = 65536


class UqcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"uqc error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class Info(C.Structure):
    _fields_ = [("n_cells", C.c_int), ("n_states", C.c_int), ("n_total", C.c_int), ("n_quad", C.c_int),
                ("n_levels", C.c_int), ("dim_xi", C.c_int), ("n_faces", C.c_int), ("mesh_dim", C.c_int),
                ("n_total_level", C.c_int * 16), ("precision", C.c_int), ("newton_mode", C.c_int),
                ("t", C.c_double), ("steps", C.c_longlong), ("mixed_form", C.c_int), ("mixed_rounds", C.c_int)]


class Config(C.Structure):
    """uqc_config (include/uqc.h): the input file's keys as a struct."""
    _fields_ = [("problem", C.c_char_p), ("restart_file", C.c_char_p), ("import_dual_state", C.c_int),
                ("mesh_dimension", C.c_int), ("n_cells", C.c_int), ("a", C.c_double), ("b", C.c_double),
                ("su2_file", C.c_char_p), ("n_su2_bc", C.c_int), ("su2_bc_marker", C.POINTER(C.c_char_p)),
                ("su2_bc_type", C.POINTER(C.c_char_p)), ("dim_xi", C.c_int), ("sigma", C.c_double * 4),
                ("cfl", C.c_double), ("t_end", C.c_double), ("min_residual", C.c_double), ("gamma", C.c_double),
                ("closure", C.c_char_p), ("max_degree", C.c_int), ("n_levels", C.c_int), ("degree", C.c_int * 16),
                ("quad_points", C.c_int * 16), ("max_iterations", C.c_int), ("epsilon", C.c_double), ("n_ic", C.c_int),
                ("ic", C.c_double * 8), ("bounds", C.c_double * 2), ("nx", C.c_int), ("ny", C.c_int),
                ("jitter", C.c_double), ("seed", C.c_ulonglong), ("precision", C.c_int), ("newton_mode", C.c_int),
                ("steps", C.c_int)]


class ShardInfo(C.Structure):
    _fields_ = [("rank", C.c_int), ("n_ranks", C.c_int), ("n_global", C.c_int), ("n_owned", C.c_int),
                ("n_halo", C.c_int), ("n_peers", C.c_int), ("n_send", C.c_int), ("row_doubles", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class StepInfo(C.Structure):
    _fields_ = [("t", C.c_double), ("dt", C.c_double), ("residual", C.c_double), ("steps", C.c_int),
                ("failed_cells", C.c_int), ("newton_iterations", C.c_longlong), ("line_search_trials", C.c_longlong),
                ("active_cells", C.c_int), ("fallback_cells", C.c_longlong), ("running", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class RequestInfo(C.Structure):
    _fields_ = [("id", C.c_longlong), ("state", C.c_int), ("status", C.c_int), ("n_cells", C.c_int),
                ("n_states", C.c_int), ("steps", C.c_int), ("t", C.c_double), ("newton_iterations", C.c_longlong),
                ("device_bytes", C.c_ulonglong), ("submit_ms", C.c_double), ("admit_ms", C.c_double),
                ("done_ms", C.c_double)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["state"] = REQ_STATES.get(d["state"], d["state"])
        return d


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_up = C.POINTER(C.c_uint)
_vp = C.c_void_p


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is not built; run `python -m uqcreator_b200.build` "
                          "(there is no CPU fallback for the hot path)")
    L = C.CDLL(str(LIB_PATH))
    sig = {
        "uqc_create_from_file": ([C.c_char_p, _vp, C.POINTER(_vp), C.c_char_p, C.c_int], C.c_int),
        "uqc_create_from_string": ([C.c_char_p, _vp, C.POINTER(_vp), C.c_char_p, C.c_int], C.c_int),
        "uqc_destroy": ([_vp], None),
        "uqc_last_error": ([_vp], C.c_char_p),
        "uqc_get_info": ([_vp, C.POINTER(Info)], C.c_int),
        "uqc_set_precision": ([_vp, C.c_int], C.c_int),
        "uqc_set_newton": ([_vp, C.c_int, C.c_double, C.c_int], C.c_int),
        "uqc_get_tables": ([_vp, _dp, _dp, _dp, _dp], C.c_int),
        "uqc_get_geometry": ([_vp, _dp, _dp, _dp, _dp, _dp, _ip, _ip], C.c_int),
        "uqc_init_state": ([_vp], C.c_int),
        "uqc_upload_state": ([_vp, _dp, _dp, _up, C.c_int, C.c_double], C.c_int),
        "uqc_download_state": ([_vp, _dp, _dp, _up, C.c_int], C.c_int),
        "uqc_solve_closure": ([_vp, C.POINTER(StepInfo)], C.c_int),
        "uqc_cell_status": ([_vp, _ip, _ip], C.c_int),
        "uqc_step": ([_vp, C.c_int, C.POINTER(StepInfo)], C.c_int),
        "uqc_run": ([_vp, C.c_double, C.POINTER(StepInfo)], C.c_int),
        "uqc_step_host": ([_vp, _dp, _dp, _up, C.c_double, _dp, _dp, _up, C.POINTER(StepInfo)], C.c_int),
        "uqc_mean_var": ([_vp, _dp], C.c_int),
        "uqc_closure_solve_host": ([_vp, C.c_int, _dp, _dp, _up, C.c_int, _ip], C.c_int),
        "uqc_closure_solve_device": ([_vp, C.c_int, _vp, _vp, _vp, _vp], C.c_int),
        "uqc_last_timing": ([_vp, C.POINTER(C.c_float)], C.c_int),
        "uqc_device_state": ([_vp, C.POINTER(_vp), C.POINTER(_vp)], C.c_int),
        "uqc_last_launch_count": ([_vp], C.c_int),
        "uqc_stream": ([_vp], _vp),
        "uqc_mesh_tri_jitter": ([C.c_int, C.c_int, C.c_double, C.c_ulonglong, _dp, _ip, _ip], C.c_int),
        "uqc_closure_solve_device_noalloc": ([_vp, C.c_int, _vp, _vp, _vp, _vp, _vp], C.c_int),
        "uqc_set_option": ([_vp, C.c_char_p, C.c_double], C.c_int),
        "uqc_step_async": ([_vp, C.c_int], C.c_int),
        "uqc_step_query": ([_vp, C.POINTER(StepInfo)], C.c_int),
        "uqc_device_bytes": ([_vp, C.POINTER(C.c_ulonglong)], C.c_int),
        "uqc_server_create": ([C.c_ulonglong, C.c_int, C.c_int, C.POINTER(_vp)], C.c_int),
        "uqc_server_destroy": ([_vp], None),
        "uqc_server_last_error": ([_vp], C.c_char_p),
        "uqc_server_submit": ([_vp, C.c_char_p, C.c_int, C.POINTER(C.c_longlong)], C.c_int),
        "uqc_server_progress": ([_vp, _ip, _ip, _ip], C.c_int),
        "uqc_server_request": ([_vp, C.c_longlong, C.POINTER(RequestInfo), _dp], C.c_int),
        "uqc_server_release": ([_vp, C.c_longlong], C.c_int),
        "uqc_server_request_error": ([_vp, C.c_longlong], C.c_char_p),
        "uqc_export_state": ([_vp, C.c_char_p], C.c_int),
        "uqc_write_vtk": ([_vp, C.c_char_p], C.c_int),
        "uqc_debug_mixed_inverse": ([_vp, C.c_int, _ip, C.c_int, C.POINTER(C.c_float)], C.c_int),
        "uqc_server_set_option": ([_vp, C.c_char_p, C.c_double], C.c_int),
        "uqc_solve_closure_cells": ([_vp, _up, C.c_int, C.c_double, C.c_int, C.POINTER(StepInfo)], C.c_int),
        "uqc_moments_mean_var": ([_vp, _dp], C.c_int),
        "uqc_config_defaults": ([C.POINTER(Config)], None),
        "uqc_create_from_config": ([C.POINTER(Config), _vp, C.POINTER(_vp), C.c_char_p, C.c_int], C.c_int),
        "uqc_partition": ([_vp, C.c_int, C.c_int], C.c_int),
        "uqc_get_shard": ([_vp, C.POINTER(ShardInfo), _ip, _ip, _ip, _ip, _ip], C.c_int),
        "uqc_shard_buffers": ([_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp)], C.c_int),
        "uqc_halo_pack": ([_vp, _vp], C.c_int),
        "uqc_step_phase": ([_vp, C.c_int, C.POINTER(StepInfo)], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def ptr(a, t=_dp):
    return None if a is None else a.ctypes.data_as(t)


def check(h, rc: int):
    if rc != UQC_OK:
        msg = lib().uqc_last_error(h).decode() if h else ""
        raise UqcError(rc, msg)
    return rc


def mesh_tri_jitter(nx: int, ny: int, jitter: float, seed: int):
    """The product's own seeded triangle mesh (host code, no GPU needed)."""
    nn = (nx + 1) * (ny + 1)
    xy = np.zeros((nn, 2)); bnd = np.zeros(nn, dtype=np.int32); tri = np.zeros((2 * nx * ny, 3), dtype=np.int32)
    rc = lib().uqc_mesh_tri_jitter(nx, ny, jitter, seed, ptr(xy), ptr(bnd, _ip), ptr(tri, _ip))
    if rc != 0:
        raise UqcError(rc, "mesh")
    return dict(xy=xy, node_boundary=bnd, tri=tri)
