"""ctypes binding of libadi_b200.so (include/adi_b200.h).

The shared library is built in-tree by ``cmc-fluid-solver_b200/build_adi.py``.  There is
no fallback: if the library is missing or fails to load, importing the binding
raises, so nothing can silently run a CPU path in its place.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libadi_b200.so")

ADI_OK = 0
STATUS_NAMES = {
    0: "ADI_OK", 1: "ADI_ERR_BAD_ARG", 2: "ADI_ERR_CAPACITY", 3: "ADI_ERR_NONFINITE",
    4: "ADI_ERR_NOT_CONVERGED", 5: "ADI_ERR_CUDA", 6: "ADI_ERR_TIMEOUT", 7: "ADI_ERR_DIVERGENCE",
    8: "ADI_ERR_STATE", 9: "ADI_ERR_NO_DEVICE",
}
globals().update({name: code for code, name in STATUS_NAMES.items()})
ADI_FP32, ADI_FP64 = 4, 8
ADI_SOLVER_EXACT, ADI_SOLVER_FAST = 0, 1
ADI_FAULT_NONE, ADI_FAULT_SKIP_TILE_LOADS = 0, 1
ADI_BATCH_PERSISTENT, ADI_BATCH_MEMBER_GRAPHS = 0, 1

# every entry point include/adi_b200.h declares
EXPORTED = [
    "adi_fluid_params_normalized", "adi_fluid_params_dimensional", "adi_create", "adi_destroy",
    "adi_set_stream", "adi_set_solver", "adi_last_error_string", "adi_set_mask", "adi_build_segments",
    "adi_get_segments", "adi_update_boundaries", "adi_time_step", "adi_step", "adi_run", "adi_get_state",
    "adi_set_state", "adi_get_layer", "adi_div_error", "adi_device_pointers", "adi_version",
    "adi_set_profiling", "adi_get_profile", "adi_get_fast_shape", "adi_set_fast_shape", "adi_autotune",
    "adi_sweep_exact_static", "adi_static_scratch_bytes", "adi_step_tol", "adi_set_graphs",
    "adi_batch_create", "adi_batch_destroy", "adi_batch_set_stream", "adi_batch_step", "adi_batch_div_errors",
    "adi_batch_set_chunk", "adi_batch_get_chunk", "adi_batch_autotune", "adi_batch_set_graphs",
    "adi_batch_launches", "adi_batch_last_error_string", "adi_batch_time_sweeps", "adi_batch_set_schedule",
    "adi_batch_get_schedule", "adi_batch_time_step", "adi_step_io", "adi_io_wait", "adi_batch_step_io", "adi_batch_io_wait", "adi_nc_write_header", "adi_nc_write_layer", "adi_adjoint_run",
    "adi_set_node_values", "adi_set_adjoint_chunk", "adi2d_create", "adi2d_destroy", "adi2d_set_stream", "adi2d_set_grid",
    "adi2d_set_segments", "adi2d_step_tol",
    "adi2d_update_boundaries", "adi2d_time_step", "adi2d_step", "adi2d_get_state", "adi2d_set_state",
    "adi2d_get_layer", "adi2d_last_error", "adi2d_last_error_string",
    "adi_mask_shape3d", "adi_mask_sea", "adi_mask_extrude2d", "adi_get_mask", "adi_mask_shape2d",
    "adi_set_fault_injection", "adi_phase_begin", "adi_phase_sweep", "adi_phase_div_sum", "adi_phase_end",
    "adi_role_pointers",
]

K_NUM = 7
KERNEL_CLASSES = ["step_begin", "sweep_x", "sweep_y", "sweep_z", "merge", "div_error", "other"]


class GridDesc(C.Structure):
    _fields_ = [("dimx", C.c_int), ("dimy", C.c_int), ("dimz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("precision", C.c_int)]


class FluidParams(C.Structure):
    _fields_ = [("v_T", C.c_double), ("v_vis", C.c_double), ("t_vis", C.c_double), ("t_phi", C.c_double)]


class SegStats(C.Structure):
    _fields_ = [("num_segments", C.c_int64 * 3), ("num_nodes", C.c_int64 * 3), ("max_size", C.c_int32 * 3),
                ("max_per_line", C.c_int32 * 3), ("num_in", C.c_int64)]


class StaticSweepArgs(C.Structure):
    """adi_static_sweep_args: one allocation-free exact sweep on caller-owned device arrays."""
    _fields_ = [("dir", C.c_int), ("dimx", C.c_int), ("dimy", C.c_int), ("dimz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
                ("params", FluidParams), ("precision", C.c_int), ("merges", C.c_int),
                ("node_type", C.c_void_p), ("bc_vel", C.c_void_p), ("bc_temp", C.c_void_p),
                ("node_value", C.c_void_p * 4), ("cur", C.c_void_p * 4), ("temp_in", C.c_void_p * 4),
                ("next", C.c_void_p * 4), ("temp_out", C.c_void_p * 4), ("stream", C.c_void_p)]


class Profile(C.Structure):
    _fields_ = [("launches", C.c_int64 * 7), ("ms", C.c_double * 7), ("bytes", C.c_int64 * 7)]


class AdiError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with cmc-fluid-solver_b200/build_adi.py")
    lib = C.CDLL(LIB_PATH)
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    sig = {
        "adi_fluid_params_normalized": [d, d, d, C.POINTER(FluidParams)],
        "adi_fluid_params_dimensional": [d, d, d, d, d, C.POINTER(FluidParams)],
        "adi_create": [C.POINTER(GridDesc), C.POINTER(FluidParams), C.POINTER(vp)],
        "adi_destroy": [vp],
        "adi_set_stream": [vp, vp],
        "adi_set_solver": [vp, i],
        "adi_set_fault_injection": [vp, i],
        "adi_phase_begin": [vp, i],
        "adi_phase_sweep": [vp, i, C.c_double, i],
        "adi_phase_div_sum": [vp, i, C.POINTER(C.c_double), C.POINTER(C.c_uint64)],
        "adi_phase_end": [vp],
        "adi_role_pointers": [vp, i, C.c_void_p],
        "adi_set_mask": [vp] + [vp] * 7,
        "adi_mask_shape3d": [vp, vp, i, vp, i, d, C.POINTER(i)],
        "adi_mask_sea": [vp, vp, i, i, C.c_float, d, vp, d],
        "adi_mask_extrude2d": [vp, vp, vp, vp, i, d, d],
        "adi_get_mask": [vp] + [vp] * 7,
        "adi_mask_shape2d": [vp, vp, i, i, i, d, vp, vp, vp, vp, vp],
        "adi_build_segments": [vp, C.POINTER(SegStats)],
        "adi_get_segments": [vp, i, vp, C.c_int64, C.POINTER(C.c_int64)],
        "adi_update_boundaries": [vp],
        "adi_time_step": [vp, d, i, i, i],
        "adi_step": [vp, d, i, i, i],
        "adi_run": [vp, d, i, i, i, i],
        "adi_step_tol": [vp, d, i, i, d, i, C.POINTER(i), C.POINTER(d)],
        "adi_set_graphs": [vp, i],
        "adi_batch_create": [vp, i, C.POINTER(vp)],
        "adi_batch_destroy": [vp],
        "adi_batch_set_stream": [vp, vp],
        "adi_batch_step": [vp, d, i, i, i],
        "adi_batch_div_errors": [vp, vp],
        "adi_batch_set_chunk": [vp, i, i],
        "adi_batch_get_chunk": [vp, i, C.POINTER(i)],
        "adi_batch_autotune": [vp, d, i],
        "adi_batch_set_graphs": [vp, i],
        "adi_batch_launches": [vp, C.POINTER(C.c_int64)],
        "adi_batch_time_sweeps": [vp, d, i, vp],
        "adi_batch_set_schedule": [vp, i, i],
        "adi_batch_get_schedule": [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)],
        "adi_batch_time_step": [vp, d, i, i, i, C.POINTER(C.c_float)],
        "adi_step_io": [vp, C.POINTER(vp), C.POINTER(vp), d, i, i, i],
        "adi_io_wait": [vp],
        "adi_batch_step_io": [vp, C.POINTER(vp), C.POINTER(vp), d, i, i, i],
        "adi_batch_io_wait": [vp],
        "adi_nc_write_header": [C.c_char_p, vp, vp, i, i, d, d, i, i, i, C.c_char_p, i],
        "adi_nc_write_layer": [C.c_char_p, vp, i, vp, i, i, i, i, C.c_char_p],
        "adi_adjoint_run": [vp, d, i, i, i, i, vp, vp, C.POINTER(d), vp, vp],
        "adi_set_node_values": [vp, vp, vp, vp, vp],
        "adi_set_adjoint_chunk": [vp, i],
        "adi2d_create": [i, i, d, d, i, C.POINTER(FluidParams), C.POINTER(vp)],
        "adi2d_destroy": [vp],
        "adi2d_set_stream": [vp, vp],
        "adi2d_set_grid": [vp, vp, vp, vp, vp, vp, d],
        "adi2d_set_segments": [vp, i],
        "adi2d_step_tol": [vp, d, i, i, d, C.POINTER(i), C.POINTER(d)],
        "adi2d_update_boundaries": [vp],
        "adi2d_time_step": [vp, d, i, i, C.POINTER(i)],
        "adi2d_step": [vp, d, i, i, C.POINTER(i)],
        "adi2d_get_state": [vp, i, vp, vp, vp],
        "adi2d_set_state": [vp, vp, vp, vp],
        "adi2d_get_layer": [vp, i, i, vp, vp],
        "adi2d_last_error": [vp, C.POINTER(d), C.POINTER(i)],
        "adi_get_state": [vp, i, vp, vp, vp, vp],
        "adi_set_state": [vp, vp, vp, vp, vp],
        "adi_get_layer": [vp, i, i, i, vp, vp],
        "adi_div_error": [vp, C.POINTER(d)],
        "adi_device_pointers": [vp, C.POINTER(vp * 8)],
        "adi_sweep_exact_static": [C.POINTER(StaticSweepArgs)],
        "adi_set_profiling": [vp, i],
        "adi_get_fast_shape": [vp, i, C.POINTER(i), C.POINTER(i), C.POINTER(i)],
        "adi_set_fast_shape": [vp, i, i, i],
        "adi_autotune": [vp, i],
        "adi_get_profile": [vp, C.POINTER(Profile), i],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    lib.adi_last_error_string.argtypes = [vp]
    lib.adi_last_error_string.restype = C.c_char_p
    lib.adi2d_last_error_string.argtypes = [vp]
    lib.adi2d_last_error_string.restype = C.c_char_p
    lib.adi_batch_last_error_string.argtypes = [vp]
    lib.adi_batch_last_error_string.restype = C.c_char_p
    lib.adi_version.argtypes = []
    lib.adi_version.restype = C.c_char_p
    lib.adi_static_scratch_bytes.argtypes = []
    lib.adi_static_scratch_bytes.restype = C.c_size_t
    _lib = lib
    return lib


def check(status: int, handle=None) -> None:
    if status != ADI_OK:
        msg = ""
        if handle:
            raw = load().adi_last_error_string(handle)
            msg = raw.decode() if raw else ""
        raise AdiError(status, msg)
