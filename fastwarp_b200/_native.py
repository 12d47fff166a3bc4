"""ctypes binding of ``libfastwarp_cuda.so`` (the C ABI declared in include/fastwarp_cuda.h).

The shared library is built in-tree (``fastwarp_b200/csrc/Makefile``) for sm_100a only. There is
no CPU fallback: importing works anywhere, but every call that needs the device fails with
``FastwarpError`` when no sm_100 GPU is present, and ``lib()`` raises when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfastwarp_cuda.so")
CSRC = os.path.join(_HERE, "csrc")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "fastwarp_cuda.h")

FW_OK = 0
FW_ERR_INVALID = -1
FW_ERR_CUDA = -2
FW_ERR_MEMORY = -3
FW_ERR_NOT_FINITE = -4
FW_ERR_TIMEOUT = -5
FW_ERR_CANCELLED = -6

MAX_LEVELS = 8
MAX_CHANNELS = 4


class Grid(C.Structure):
    _fields_ = [("size", C.c_int64 * 3), ("spacing", C.c_double * 3),
                ("origin", C.c_double * 3), ("direction", C.c_double * 9)]


class Affine(C.Structure):
    _fields_ = [("matrix", C.c_double * 9), ("offset", C.c_double * 3)]


class InvertParams(C.Structure):
    _fields_ = [("max_iterations", C.c_int32), ("mean_error_tolerance", C.c_double),
                ("max_error_tolerance", C.c_double), ("enforce_boundary_condition", C.c_int32)]


class InvertStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("mean_error_norm", C.c_double),
                ("max_error_norm", C.c_double)]


class MiBinning(C.Structure):
    _fields_ = [("bins", C.c_int32), ("fixed_min", C.c_double), ("fixed_max", C.c_double),
                ("moving_min", C.c_double), ("moving_max", C.c_double),
                ("fixed_bin_size", C.c_double), ("moving_bin_size", C.c_double),
                ("fixed_normalized_min", C.c_double), ("moving_normalized_min", C.c_double)]


class LinearTransform(C.Structure):
    _fields_ = [("outer_matrix", C.c_double * 9), ("outer_translation", C.c_double * 3),
                ("outer_center", C.c_double * 3), ("kind", C.c_int32), ("zyx", C.c_int32),
                ("parameters", C.c_double * 12), ("center", C.c_double * 3)]


class CgSettings(C.Structure):
    _fields_ = [("max_step_mm", C.c_double), ("lower_limit", C.c_double),
                ("upper_limit", C.c_double), ("epsilon", C.c_double),
                ("max_line_search_iterations", C.c_int32), ("iterations", C.c_int32),
                ("convergence_threshold", C.c_double), ("convergence_window", C.c_int32),
                ("small_parameter_variation", C.c_double)]


class CgTrace(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32),
                ("converged_value", C.c_double), ("best_value", C.c_double),
                ("initial_learning_rate", C.c_double), ("final_learning_rate", C.c_double),
                ("line_search_evaluations", C.c_uint64), ("scales", C.c_double * 12),
                ("nvalues", C.c_int64)]


class LinearRecipe(C.Structure):
    _fields_ = [("levels", C.c_int32), ("iterations", C.c_uint32 * 8),
                ("shrink_factors", C.c_uint32 * 8), ("smoothing_sigmas", C.c_double * 8),
                ("sigma_units_mm", C.c_int32), ("gradient_step", C.c_double),
                ("convergence_threshold", C.c_double), ("convergence_window", C.c_int32),
                ("bins", C.c_int32), ("sampling_percentage", C.c_float), ("seed", C.c_uint32)]


class LinearLevelTrace(C.Structure):
    _fields_ = [("level", C.c_int32), ("shrink_factors", C.c_uint32 * 3),
                ("grid_size", C.c_int64 * 3), ("samples", C.c_int64), ("skipped", C.c_int32),
                ("cg", CgTrace), ("parameters", C.c_double * 12),
                ("prepare_ms", C.c_double), ("optimize_ms", C.c_double),
                ("samples_cached", C.c_int32)]


class LinearChainResult(C.Structure):
    _fields_ = [("initial_matrix", C.c_double * 9), ("initial_translation", C.c_double * 3),
                ("initial_center", C.c_double * 3), ("rigid", LinearTransform),
                ("affine", LinearTransform), ("rigid_levels", LinearLevelTrace * 8),
                ("affine_levels", LinearLevelTrace * 8), ("total_matrix", C.c_double * 9),
                ("total_translation", C.c_double * 3), ("total_center", C.c_double * 3),
                ("initial_ms", C.c_double)]


METRIC_VALUE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(LinearTransform),
                              C.POINTER(C.c_double))
METRIC_VALUE_DERIVATIVE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(LinearTransform),
                                         C.POINTER(C.c_double), C.POINTER(C.c_double))


class TransformElem(C.Structure):
    """fw_transform_elem (include/fastwarp_transform_io.h)."""
    _fields_ = [("kind", C.c_int32), ("matrix", C.c_double * 9),
                ("translation", C.c_double * 3), ("center", C.c_double * 3), ("grid", Grid),
                ("field", C.c_void_p)]


class SynRecipe(C.Structure):
    _fields_ = [("gradient_step", C.c_double), ("update_field_variance", C.c_double),
                ("total_field_variance", C.c_double), ("cc_radius", C.c_int32),
                ("levels", C.c_int32), ("iterations", C.c_uint32 * MAX_LEVELS),
                ("shrink_factors", C.c_uint32 * MAX_LEVELS),
                ("smoothing_sigmas", C.c_double * MAX_LEVELS), ("sigma_units_mm", C.c_int32),
                ("convergence_threshold", C.c_double), ("convergence_window", C.c_int32),
                ("channels", C.c_int32), ("channel_weights", C.c_double * MAX_CHANNELS),
                ("channel_metrics", C.c_int32 * MAX_CHANNELS), ("mi_bins", C.c_int32)]


class SynIteration(C.Structure):
    _fields_ = [("level", C.c_int32), ("energy", C.c_double), ("energy_weighted", C.c_double),
                ("convergence_value", C.c_double), ("fixed_update_scale", C.c_double),
                ("moving_update_scale", C.c_double), ("inversions", InvertStats * 4)]


class BatchSubject(C.Structure):
    """fw_batch_subject (include/fastwarp_cuda.h)."""
    _fields_ = [("moving", C.c_void_p * MAX_CHANNELS), ("initial", Affine),
                ("has_initial", C.c_int32)]


class BatchTuning(C.Structure):
    _fields_ = [("level", C.c_int32), ("grid_size", C.c_int64 * 3),
                ("warp_zchunk", C.c_int32), ("warp_blocks_per_sm", C.c_int32),
                ("compose_zchunk", C.c_int32), ("compose_blocks_per_sm", C.c_int32),
                ("cc_zchunk", C.c_int32), ("cc_blocks_per_sm", C.c_int32),
                ("measure_zchunk", C.c_int32), ("measure_blocks_per_sm", C.c_int32),
                ("body_blocks_per_sm", C.c_int32), ("smooth_blocks_per_sm", C.c_int32),
                ("from_cache", C.c_int32), ("tune_ms", C.c_double),
                ("kernel_ms", C.c_double * 6)]


class BatchReport(C.Structure):
    _fields_ = [("subjects", C.c_int32), ("levels", C.c_int32),
                ("tuning", BatchTuning * MAX_LEVELS), ("level_ms", C.c_double * MAX_LEVELS),
                ("device_bytes", C.c_uint64), ("prepare_ms", C.c_double * MAX_LEVELS),
                ("finish_ms", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("kernel_launches", C.c_uint64), ("graph_launches", C.c_uint64),
                ("host_syncs", C.c_uint64), ("bytes_uploaded", C.c_uint64),
                ("bytes_downloaded", C.c_uint64), ("peak_device_bytes", C.c_uint64),
                ("live_device_bytes", C.c_uint64)]


class FastwarpError(RuntimeError):
    """A failed call of the engine; `code` is the FW_ERR_* status."""

    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


_lib = None


def build(quiet: bool = True) -> None:
    """Compiles the CUDA library (nvcc, sm_100a) with its Makefile."""
    subprocess.run(["make", "-C", CSRC, "-j8"], check=True,
                   capture_output=quiet)


def lib():
    """The loaded library; raises FileNotFoundError when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `make -C {CSRC}` "
                "(the engine has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        L.fw_last_error.restype = C.c_char_p
        L.fw_backend_name.restype = C.c_char_p
        L.fw_ctx_stream.restype = C.c_void_p
        L.fw_image_device_ptr.restype = C.c_void_p
        L.fw_field_device_ptr.restype = C.c_void_p
        L.fw_ctx_destroy.restype = None
        L.fw_image_free.restype = None
        L.fw_field_free.restype = None
        L.fw_mi_level_free.restype = None
        L.fw_ctx_reset_stats.restype = None
        L.fw_abi_struct_size.restype = C.c_size_t
        L.fw_abi_struct_size.argtypes = [C.c_char_p]
        L.fw_lookup3.restype = C.c_uint32
        L.fw_lookup3.argtypes = [C.c_char_p, C.c_size_t]
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != 0:
        raise FastwarpError(rc, lib().fw_last_error().decode())


def exported_symbols():
    """The function names include/fastwarp_cuda.h declares."""
    import re
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(fw_[a-z0-9_]+)\s*\(", text)))
