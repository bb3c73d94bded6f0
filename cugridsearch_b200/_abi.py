"""ctypes binding of ``libcgs_b200.so`` (declared in ``include/cugridsearch_b200.h``).

The library is the product: if it is missing or cannot be loaded this module raises,
there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcgs_b200.so")

COSTS = {
    "SAD_AVG": 0, "SAD_AVG_H": 1, "SAD_SUM_T": 2, "SAD_SUM_T_REF": 3, "SQD_REF": 4,
    "NCC_REF": 5, "SQD_ALT": 6, "NCC_ALT": 7, "MI_ALT": 8, "ZNCC": 9, "MI": 10,
}
PIXEL_F32, PIXEL_U8, PIXEL_F64, PIXEL_U16 = 0, 1, 2, 3
FLAG_NATURAL_ORDER = 1
FLAG_EXACT_SAMPLES = 2
FLAG_FAST_SAMPLES = 4
FLAG_QUAD_TAPS = 8
FLAG_TEXTURE_TAPS = 16
FLAG_PER_SAMPLE_DECISIONS = 32
FLAG_NO_VERIFY = 64
VERIFY_MAX = 64

STATUS = {
    0: "CGS_SUCCESS", 1: "CGS_ERROR_INVALID_VALUE", 2: "CGS_ERROR_UNSUPPORTED",
    3: "CGS_ERROR_GRID_TOO_LARGE", 4: "CGS_ERROR_OUT_OF_MEMORY", 5: "CGS_ERROR_CUDA",
    6: "CGS_ERROR_NO_DEVICE", 7: "CGS_ERROR_DEVICE_TIMEOUT",
}

# Every symbol the header declares; tests check the library exports all of them.
EXPORTS = [
    "cgs_grid_update", "cgs_grid_num_elements", "cgs_grid_point", "cgs_search",
    "cgs_argmin_f32", "cgs_search_sync", "cgs_status_string", "cgs_last_error", "cgs_version",
    "cgs_mi_histogram", "cgs_search_noalloc", "cgs_covariance", "cgs_search_refine",
    "cgs_homography", "cgs_transform_image", "cgs_fuse_aligned", "cgs_filter_image", "cgs_quantize_image",
    "cgs_batch_create", "cgs_batch_launch", "cgs_batch_set_plan", "cgs_batch_get_plan", "cgs_batch_autotune",
    "cgs_batch_pair_times", "cgs_batch_kernel_launches", "cgs_batch_destroy", "cgs_search_batched", "cgs_autotune",
    "cgs_net_param_count", "cgs_net_create", "cgs_net_destroy", "cgs_net_get_params", "cgs_net_set_params",
    "cgs_net_get_grads", "cgs_net_forward", "cgs_net_backward", "cgs_net_adam_step", "cgs_grid_window",
    "cgs_proposal_window",
]


class CgsImage(C.Structure):
    _fields_ = [("data", C.c_void_p), ("height", C.c_int32), ("width", C.c_int32),
                ("channels", C.c_int32), ("pixel", C.c_int32)]


class CgsGrid(C.Structure):
    _fields_ = [("dims", C.c_int32), ("start", C.c_float * 8), ("end", C.c_float * 8),
                ("resolution", C.c_float * 8), ("count", C.c_float * 8)]


class CgsOptions(C.Structure):
    _fields_ = [("cost", C.c_int32), ("mi_bins", C.c_int32), ("overlap_gate", C.c_float),
                ("points_per_warp", C.c_int32), ("warps_per_block", C.c_int32), ("flags", C.c_int32)]


class CgsArgmin(C.Structure):
    _fields_ = [("cost", C.c_float), ("valid", C.c_int32), ("index", C.c_int64),
                ("params", C.c_float * 8), ("status", C.c_int32), ("verified", C.c_int32),
                ("candidates", C.c_int32), ("reserved", C.c_int32), ("index_fp64", C.c_int64),
                ("cost_fp64", C.c_double), ("err_fp64", C.c_double), ("max_err_fp64", C.c_double)]


class CgsPair(C.Structure):
    _fields_ = [("moving", CgsImage), ("fixed", CgsImage), ("grid", CgsGrid), ("options", CgsOptions),
                ("costs", C.c_void_p), ("result", C.c_void_p)]


class CgsBatchPlan(C.Structure):
    _fields_ = [("points_per_warp", C.c_int32), ("warps_per_block", C.c_int32), ("block_split", C.c_int32),
                ("reserved", C.c_int32)]


class CgsTuneEntry(C.Structure):
    _fields_ = [("plan", CgsBatchPlan), ("ms", C.c_float), ("status", C.c_int32)]


class CgsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


_lock = threading.Lock()
_lib = None


def load() -> C.CDLL:
    """Load the sm_100a library (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cugridsearch_b200.build`")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        L.cgs_grid_update.restype = C.c_int
        L.cgs_grid_update.argtypes = [P(CgsGrid), C.c_int32]
        L.cgs_grid_num_elements.restype = C.c_int
        L.cgs_grid_num_elements.argtypes = [P(CgsGrid), P(C.c_uint64)]
        L.cgs_grid_point.restype = C.c_int
        L.cgs_grid_point.argtypes = [P(CgsGrid), C.c_int64, P(C.c_float)]
        L.cgs_search.restype = C.c_int
        L.cgs_search.argtypes = [P(CgsImage), P(CgsImage), P(CgsGrid), P(CgsOptions), C.c_void_p, C.c_void_p,
                                 C.c_void_p]
        L.cgs_search_noalloc.restype = C.c_int
        L.cgs_search_noalloc.argtypes = [P(CgsImage), P(CgsImage), P(CgsGrid), P(CgsOptions), C.c_void_p,
                                         C.c_void_p, C.c_void_p]
        L.cgs_search_sync.restype = C.c_int
        L.cgs_search_sync.argtypes = [P(CgsImage), P(CgsImage), P(CgsGrid), P(CgsOptions), C.c_void_p,
                                      P(CgsArgmin), C.c_void_p]
        L.cgs_argmin_f32.restype = C.c_int
        L.cgs_argmin_f32.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
        L.cgs_mi_histogram.restype = C.c_int
        L.cgs_mi_histogram.argtypes = [P(CgsImage), P(CgsImage), P(C.c_float), C.c_int32, C.c_void_p, C.c_void_p]
        L.cgs_covariance.restype = C.c_int
        L.cgs_covariance.argtypes = [P(CgsGrid), C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
        L.cgs_search_refine.restype = C.c_int
        L.cgs_search_refine.argtypes = [P(CgsImage), P(CgsImage), P(CgsGrid), P(CgsOptions), C.c_int32,
                                        P(CgsArgmin), P(CgsGrid), C.c_void_p]
        L.cgs_homography.restype = C.c_int
        L.cgs_homography.argtypes = [P(C.c_float), C.c_float, C.c_float, C.c_int32, P(C.c_float)]
        L.cgs_transform_image.restype = C.c_int
        L.cgs_transform_image.argtypes = [P(C.c_float), C.c_int32, C.c_int32, P(CgsImage), P(CgsImage), C.c_void_p]
        L.cgs_fuse_aligned.restype = C.c_int
        L.cgs_fuse_aligned.argtypes = [P(C.c_float), P(C.c_float), P(CgsImage), P(CgsImage), P(CgsImage), C.c_int32,
                                       C.c_void_p]
        L.cgs_filter_image.restype = C.c_int
        L.cgs_filter_image.argtypes = [P(CgsImage), P(CgsImage), P(CgsImage), P(C.c_int32), C.c_void_p]
        L.cgs_quantize_image.restype = C.c_int
        L.cgs_quantize_image.argtypes = [P(CgsImage), C.c_float, C.c_void_p]
        L.cgs_batch_create.restype = C.c_int
        L.cgs_batch_create.argtypes = [P(CgsPair), C.c_int32, P(CgsBatchPlan), P(C.c_void_p)]
        L.cgs_batch_launch.restype = C.c_int
        L.cgs_batch_launch.argtypes = [C.c_void_p, C.c_void_p]
        L.cgs_batch_set_plan.restype = C.c_int
        L.cgs_batch_set_plan.argtypes = [C.c_void_p, P(CgsBatchPlan)]
        L.cgs_batch_get_plan.restype = C.c_int
        L.cgs_batch_get_plan.argtypes = [C.c_void_p, P(CgsBatchPlan)]
        L.cgs_batch_autotune.restype = C.c_int
        L.cgs_batch_autotune.argtypes = [C.c_void_p, C.c_int32, P(CgsTuneEntry), C.c_int32, P(C.c_int32),
                                         P(CgsBatchPlan)]
        L.cgs_batch_pair_times.restype = C.c_int
        L.cgs_batch_pair_times.argtypes = [C.c_void_p, P(C.c_uint64), P(C.c_uint64)]
        L.cgs_batch_kernel_launches.restype = C.c_int
        L.cgs_batch_kernel_launches.argtypes = [C.c_void_p, P(C.c_int32)]
        L.cgs_batch_destroy.restype = C.c_int
        L.cgs_batch_destroy.argtypes = [C.c_void_p]
        L.cgs_search_batched.restype = C.c_int
        L.cgs_search_batched.argtypes = [P(CgsPair), C.c_int32, P(CgsBatchPlan), C.c_void_p]
        L.cgs_autotune.restype = C.c_int
        L.cgs_autotune.argtypes = [P(CgsPair), C.c_int32, C.c_int32, P(CgsBatchPlan)]
        L.cgs_net_param_count.restype = C.c_int64
        L.cgs_net_param_count.argtypes = []
        L.cgs_net_create.restype = C.c_int
        L.cgs_net_create.argtypes = [C.c_int32, C.c_uint64, P(C.c_void_p)]
        L.cgs_net_destroy.restype = C.c_int
        L.cgs_net_destroy.argtypes = [C.c_void_p]
        for fn in ("cgs_net_get_params", "cgs_net_set_params", "cgs_net_get_grads"):
            getattr(L, fn).restype = C.c_int
            getattr(L, fn).argtypes = [C.c_void_p, P(C.c_float)]
        L.cgs_net_forward.restype = C.c_int
        L.cgs_net_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                                      C.c_void_p]
        L.cgs_net_backward.restype = C.c_int
        L.cgs_net_backward.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.cgs_net_adam_step.restype = C.c_int
        L.cgs_net_adam_step.argtypes = [C.c_void_p, C.c_float, C.c_void_p]
        L.cgs_grid_window.restype = C.c_int
        L.cgs_grid_window.argtypes = [P(CgsGrid), P(C.c_int32), P(C.c_int32), P(CgsGrid)]
        L.cgs_proposal_window.restype = C.c_int
        L.cgs_proposal_window.argtypes = [P(CgsGrid), P(C.c_float), C.c_int32, C.c_int32, P(C.c_int32),
                                          P(C.c_int32)]
        L.cgs_status_string.restype = C.c_char_p
        L.cgs_status_string.argtypes = [C.c_int]
        L.cgs_last_error.restype = C.c_char_p
        L.cgs_last_error.argtypes = []
        L.cgs_version.restype = C.c_int32
        L.cgs_version.argtypes = []
        _lib = L
        return L


def check(status: int) -> None:
    if status != 0:
        msg = load().cgs_last_error().decode(errors="replace")
        raise CgsError(status, msg)
