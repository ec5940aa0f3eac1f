"""ctypes binding of libpvb200.so (the C ABI declared in include/pvb200.h).

The shared library is built in-tree by ``python pointvortex_b200/build.py``. Importing this module
without it raises ImportError: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpvb200.so")

PV_OK = 0
PV_ERROR_INVALID_ARGUMENT = 1
PV_ERROR_OUT_OF_RANGE = 2
PV_ERROR_RUNTIME = 3
PV_ERROR_LOGIC = 4
PV_ERROR_CUDA = 5

GEOMETRY_INFINITE = 0
GEOMETRY_PERIODIC = 1
GEOMETRY_DISK = 2
PRECISION_FP64 = 0
PRECISION_FP32C = 1


class PvParams(ctypes.Structure):
    _fields_ = [
        ("geometry", ctypes.c_int),
        ("core_radius", ctypes.c_double),
        ("box_length_x", ctypes.c_double),
        ("box_length_y", ctypes.c_double),
        ("image_layers", ctypes.c_int),
        ("disk_radius", ctypes.c_double),
        ("precision", ctypes.c_int),
    ]


class PvStepResult(ctypes.Structure):
    _fields_ = [
        ("accepted_time_step", ctypes.c_double),
        ("suggested_time_step", ctypes.c_double),
        ("normalized_error", ctypes.c_double),
        ("rejected_steps", ctypes.c_uint),
    ]


class PvDipoleCandidate(ctypes.Structure):
    _fields_ = [
        ("first", ctypes.c_uint64),
        ("second", ctypes.c_uint64),
        ("distance_squared", ctypes.c_double),
    ]


class PvDipoleConfig(ctypes.Structure):
    _fields_ = [
        ("removal", ctypes.c_int),
        ("distance", ctypes.c_double),
        ("reinjection", ctypes.c_int),
        ("random_seed", ctypes.c_uint64),
    ]


REINJECTION = {"none": 0, "independent": 1, "paired": 2}

class PvPlanInfo(ctypes.Structure):
    _fields_ = [("symmetric", ctypes.c_int), ("rows", ctypes.c_int),
                ("targets_per_thread", ctypes.c_int), ("chunk", ctypes.c_int),
                ("symmetric_min_ctas", ctypes.c_int), ("symmetric_targets", ctypes.c_int),
                ("symmetric_grid_ctas", ctypes.c_int)]


TRAJECTORY_ROW_MAX = 192   # PV_TRAJECTORY_ROW_MAX
CHECKPOINT_ROW_MAX = 80    # PV_CHECKPOINT_ROW_MAX

PV_ERROR_CAPACITY = 6
SIM_RUNNING, SIM_DONE, SIM_FAILED, SIM_BUDGET = 1, 2, 3, 4


class PvBatchConfig(ctypes.Structure):
    _fields_ = [("capacity_vortices", ctypes.c_size_t), ("max_simulations", ctypes.c_uint32),
                ("device", ctypes.c_int), ("max_steps_per_simulation", ctypes.c_uint64),
                ("partial_chunks_per_vortex_slot", ctypes.c_size_t)]


class PvBatchSolve(ctypes.Structure):
    _fields_ = [("t_end", ctypes.c_double), ("dt", ctypes.c_double),
                ("absolute_tolerance", ctypes.c_double), ("relative_tolerance", ctypes.c_double),
                ("minimum_time_step", ctypes.c_double), ("maximum_time_step", ctypes.c_double),
                ("max_steps", ctypes.c_uint64)]


class PvBatchSimInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int), ("status", ctypes.c_int), ("time", ctypes.c_double),
                ("suggested_time_step", ctypes.c_double), ("accepted_steps", ctypes.c_uint64),
                ("rejected_steps", ctypes.c_uint64), ("population", ctypes.c_uint32),
                ("failure", ctypes.c_int), ("targets_per_thread", ctypes.c_int)]


class PvBatchTotals(ctypes.Structure):
    _fields_ = [("attempts", ctypes.c_uint64), ("work_items", ctypes.c_uint32),
                ("free_vortices", ctypes.c_size_t), ("running", ctypes.c_uint32),
                ("occupied_slots", ctypes.c_uint32)]


KERNEL_KINDS = ("velocity", "stage", "accept", "invariants", "dipole", "output", "near")


class PvKernelStats(ctypes.Structure):
    _fields_ = [
        ("launches", ctypes.c_uint64 * len(KERNEL_KINDS)),
        ("timed_launches", ctypes.c_uint64 * len(KERNEL_KINDS)),
        ("milliseconds", ctypes.c_double * len(KERNEL_KINDS)),
    ]


_D = ctypes.POINTER(ctypes.c_double)
_SZ = ctypes.c_size_t
_CTX = ctypes.c_void_p
_ST = ctypes.c_int

# name -> (restype, argtypes): every function of include/pvb200.h
SIGNATURES = {
    "pv_context_create": (_ST, [ctypes.POINTER(PvParams), ctypes.c_int, ctypes.POINTER(_CTX)]),
    "pv_context_destroy": (None, [_CTX]),
    "pv_last_error": (ctypes.c_char_p, [_CTX]),
    "pv_backend_name": (ctypes.c_char_p, []),
    "pv_runtime_details": (_ST, [ctypes.c_int, ctypes.c_char_p, _SZ]),
    "pv_evaluate_range": (_ST, [_CTX, _D, _D, _D, _SZ, _SZ, _SZ, _D, _D]),
    "pv_evaluate": (_ST, [_CTX, _D, _D, _D, _SZ, _D, _D]),
    "pv_hamiltonian": (_ST, [_CTX, _D, _D, _D, _SZ, _D]),
    "pv_invariants": (_ST, [_CTX, _D, _D, _D, _SZ, _D]),
    "pv_upload_state": (_ST, [_CTX, _D, _D, _D, _SZ]),
    "pv_download_state": (_ST, [_CTX, _D, _D, _SZ]),
    "pv_evaluate_state": (_ST, [_CTX, _D, _D, _SZ]),
    "pv_rk4_step": (_ST, [_CTX, ctypes.c_double]),
    "pv_dopri5_step": (_ST, [_CTX, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                             ctypes.c_double, ctypes.c_double, ctypes.POINTER(PvStepResult)]),
    "pv_invalidate_derivative": (_ST, [_CTX]),
    "pv_state_invariants": (_ST, [_CTX, _D]),
    "pv_dipole_scan": (_ST, [_CTX, ctypes.c_double, ctypes.POINTER(PvDipoleCandidate), _SZ,
                             ctypes.POINTER(_SZ)]),
    "pv_dipole_configure": (_ST, [_CTX, ctypes.POINTER(PvDipoleConfig)]),
    "pv_dipole_process": (_ST, [_CTX, ctypes.POINTER(_SZ)]),
    "pv_dipole_state": (_ST, [_CTX, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                              ctypes.c_char_p, _SZ, ctypes.POINTER(_SZ)]),
    "pv_dipole_restore": (_ST, [_CTX, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_char_p]),
    "pv_download_circulation": (_ST, [_CTX, _D, _SZ]),
    "pv_format_trajectory": (_ST, [_CTX, ctypes.c_double, ctypes.c_uint64, ctypes.c_char_p, _SZ,
                                   ctypes.POINTER(_SZ)]),
    "pv_format_trajectory_host": (_ST, [_CTX, ctypes.c_double, ctypes.c_uint64, _D, _D, _D, _D, _D,
                                        _SZ, ctypes.c_char_p, _SZ, ctypes.POINTER(_SZ)]),
    "pv_format_checkpoint_vortices": (_ST, [_CTX, ctypes.c_char_p, _SZ, ctypes.POINTER(_SZ)]),
    "pv_state_plan": (_ST, [_CTX, ctypes.POINTER(PvPlanInfo)]),
    "pv_state_size": (_ST, [_CTX, ctypes.POINTER(_SZ)]),
    "pv_evaluation_count": (_ST, [_CTX, ctypes.POINTER(ctypes.c_uint64)]),
    "pv_rk4_advance": (_ST, [_CTX, ctypes.c_double, ctypes.c_uint64]),
    "pv_evaluate_device_noalloc": (_ST, [ctypes.POINTER(PvParams), ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, _SZ, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]),
    "pv_batch_create": (_ST, [ctypes.POINTER(PvBatchConfig), ctypes.POINTER(ctypes.c_void_p)]),
    "pv_batch_destroy": (None, [ctypes.c_void_p]),
    "pv_batch_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "pv_batch_add": (_ST, [ctypes.c_void_p, ctypes.POINTER(PvParams), _D, _D, _D, _SZ,
                           ctypes.POINTER(PvBatchSolve), ctypes.POINTER(ctypes.c_uint32)]),
    "pv_batch_advance": (_ST, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]),
    "pv_batch_info": (_ST, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(PvBatchSimInfo)]),
    "pv_batch_result": (_ST, [ctypes.c_void_p, ctypes.c_uint32, _D, _D, _SZ]),
    "pv_batch_release": (_ST, [ctypes.c_void_p, ctypes.c_uint32]),
    "pv_batch_status": (_ST, [ctypes.c_void_p, ctypes.POINTER(PvBatchTotals)]),
    "pv_batch_stream": (_ST, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "pv_probe_peak": (_ST, [ctypes.c_int, ctypes.c_int, _D]),
    "pv_context_stream": (_ST, [_CTX, ctypes.POINTER(ctypes.c_void_p)]),
    "pv_set_tuning": (_ST, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "pv_get_tuning": (_ST, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "pv_set_symmetric_tuning": (_ST, [ctypes.c_int] * 6),
    "pv_get_symmetric_tuning": (_ST, [ctypes.c_int, ctypes.c_int, ctypes.c_int] +
                                [ctypes.POINTER(ctypes.c_int)] * 3),
    "pv_set_symmetric_grid": (_ST, [ctypes.c_int] * 4),
    "pv_get_symmetric_grid": (_ST, [ctypes.c_int] * 3 + [ctypes.POINTER(ctypes.c_int)]),
    "pv_set_batch_tuning": (_ST, [ctypes.c_int] * 4),
    "pv_get_batch_tuning": (_ST, [ctypes.c_int] * 3 + [ctypes.POINTER(ctypes.c_int)]),
    "pv_set_profiling": (_ST, [_CTX, ctypes.c_int]),
    "pv_set_wait_limits": (_ST, [_CTX, ctypes.c_int64, ctypes.c_int64]),
    "pv_set_near_field": (_ST, [_CTX, ctypes.c_double]),
    "pv_get_near_field": (_ST, [_CTX, _D]),
    "pv_get_kernel_stats": (_ST, [_CTX, ctypes.POINTER(PvKernelStats)]),
    "pv_reset_kernel_stats": (_ST, [_CTX]),
}


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build the CUDA library with `python pointvortex_b200/build.py` "
            "(there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = load()
