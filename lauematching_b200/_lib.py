"""ctypes binding of liblmb200.so (the C ABI declared in include/lmb200.h).

The library is loaded from this package directory.  There is no CPU
fallback: if the shared library is missing or no CUDA device is usable, the
calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblmb200.so")

LMB_OK = 0
LMB_ERR_INVALID = -1
LMB_ERR_CUDA = -2
LMB_ERR_OOM = -3
LMB_ERR_OVERFLOW = -4
LMB_ERR_TIMEOUT = -5
LMB_MAX_SLOTS = 64
LMB_F64, LMB_F32, LMB_U8, LMB_U16 = 0, 1, 2, 3
LMB_THR_ADAPTIVE, LMB_THR_PERCENTILE, LMB_THR_FIXED = 0, 1, 2
LMB_PRE_STAGES = 8
LMB_VALUE_U8, LMB_VALUE_F64 = 0, 1
LMB_BUILD_EXACT_FP64 = 1
LMB_BUILD_SYNTH_HEX_FZ = 2
LMB_NOALLOC_ORDER_MAX = 1 << 20

# Every function the header declares (checked by the CPU test suite).
EXPORTS = [
    "lmb_version", "lmb_last_error", "lmb_device_info", "lmb_geometry_init", "lmb_engine_create",
    "lmb_engine_destroy", "lmb_engine_stream", "lmb_engine_set_tuning",
    "lmb_engine_get_tuning", "lmb_engine_layout_info", "lmb_engine_set_sparse_uploads",
    "lmb_engine_set_dense_share",
    "lmb_db_upload", "lmb_db_build",
    "lmb_db_build_ex", "lmb_db_build_synthetic", "lmb_synth_orientations",
    "lmb_db_build_synthetic_ex", "lmb_synth_orientations_ex", "lmb_db_download", "lmb_db_info", "lmb_image_load",
    "lmb_image_load_batch",
    "lmb_match", "lmb_results", "lmb_results_batch", "lmb_last_pass_ms", "lmb_engine_bytes",
    "lmb_post_process", "lmb_post_free", "lmb_merge_clusters",
    "lmb_order_survivors_noalloc",
    "lmb_host_alloc", "lmb_host_free",
    "lmb_pre_create", "lmb_pre_destroy", "lmb_pre_median", "lmb_pre_set_background",
    "lmb_pre_get_background", "lmb_pre_segment", "lmb_pre_segment_thresholded",
    "lmb_pre_centres", "lmb_pre_stats", "lmb_pre_images", "lmb_pre_blur", "lmb_pre_timings",
    "lmb_pre_blur_to_slot",
    "lmb_refine_create", "lmb_refine_destroy", "lmb_refine_dims", "lmb_refine_set_images",
    "lmb_refine_set_grains", "lmb_refine_start", "lmb_refine_evaluate", "lmb_refine_fit",
    "lmb_refine_last_stats", "lmb_post_last_refine_stats",
]


class LmbGeometry(C.Structure):
    _fields_ = [
        ("recip", C.c_double * 9), ("rot_t", C.c_double * 9), ("p", C.c_double * 3),
        ("px_x", C.c_double), ("px_y", C.c_double), ("elo", C.c_double), ("ehi", C.c_double),
        ("nr_px_x", C.c_int32), ("nr_px_y", C.c_int32), ("max_nr_spots", C.c_int32),
        ("reserved", C.c_int32),
    ]


class LmbSurvivor(C.Structure):
    _fields_ = [("id", C.c_uint64), ("n_spots", C.c_int32), ("sum_u8", C.c_int32),
                ("tot_int", C.c_double), ("score", C.c_double)]


class LmbPostParams(C.Structure):
    _fields_ = [("lattice", C.c_double * 6), ("space_group", C.c_int32),
                ("max_nr_spots", C.c_int32), ("tol_latc", C.c_double * 6),
                ("tol_c_over_a", C.c_double), ("max_angle", C.c_double),
                ("min_nr_spots", C.c_int32), ("image_num", C.c_int32),
                ("num_threads", C.c_int32), ("optimizer", C.c_int32),
                ("max_results", C.c_int32), ("merge_on_device", C.c_int32)]


class LmbPostOutput(C.Structure):
    _fields_ = [("solutions", C.c_void_p), ("solutions_len", C.c_uint64),
                ("spots", C.c_void_p), ("spots_len", C.c_uint64), ("n_unique", C.c_int32)]


class LmbPreParams(C.Structure):
    _fields_ = [("threshold_method", C.c_int32), ("min_area", C.c_int32),
                ("threshold_value", C.c_double), ("threshold_percentile", C.c_double),
                ("override_thresh", C.c_double)]


class LmbPreCounts(C.Structure):
    _fields_ = [("threshold", C.c_double), ("min_dist2", C.c_double), ("n_labels", C.c_int32),
                ("n_centres", C.c_int32)]


class LmbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"lmb200 error {code}: {msg}")
        self.code = code


class OverflowError_(LmbError):
    pass


class TimeoutError_(LmbError):
    """A bounded device wait gave up (LMB_ERR_TIMEOUT)."""


_lib = None


def lib():
    """Load liblmb200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m lauematching_b200.build` "
            "(the B200 library has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, u64, i32, dbl = C.c_void_p, C.c_uint64, C.c_int32, C.c_double
    dp = C.POINTER(C.c_double)
    sig = {
        "lmb_version": ([], C.c_char_p),
        "lmb_last_error": ([], C.c_char_p),
        "lmb_device_info": ([i32, C.POINTER(u64), C.POINTER(u64), C.POINTER(i32),
                             C.POINTER(i32)], C.c_int),
        "lmb_geometry_init": ([dp, i32, dp, dp, dbl, dbl, i32, i32, dbl, dbl, i32,
                               C.POINTER(LmbGeometry)], C.c_int),
        "lmb_engine_create": ([i32, C.POINTER(LmbGeometry), u64, C.POINTER(vp)], C.c_int),
        "lmb_engine_destroy": ([vp], C.c_int),
        "lmb_engine_stream": ([vp], vp),
        "lmb_engine_set_tuning": ([vp, C.POINTER(i32), i32], C.c_int),
        "lmb_engine_get_tuning": ([vp, C.POINTER(i32), i32], C.c_int),
        "lmb_engine_layout_info": ([vp, C.POINTER(i32), C.POINTER(u64), C.POINTER(i32),
                                    C.POINTER(i32)], C.c_int),
        "lmb_engine_set_sparse_uploads": ([vp, i32], C.c_int),
        "lmb_engine_set_dense_share": ([vp, dbl], C.c_int),
        "lmb_db_upload": ([vp, vp, u64], C.c_int),
        "lmb_db_build": ([vp, vp, u64, vp, i32], C.c_int),
        "lmb_db_build_ex": ([vp, vp, u64, vp, i32, C.c_uint32], C.c_int),
        "lmb_db_build_synthetic": ([vp, u64, u64, vp, i32, vp], C.c_int),
        "lmb_synth_orientations": ([vp, u64, u64, u64, vp], C.c_int),
        "lmb_db_build_synthetic_ex": ([vp, u64, u64, vp, i32, vp, C.c_uint32], C.c_int),
        "lmb_synth_orientations_ex": ([vp, u64, u64, u64, vp, C.c_uint32], C.c_int),
        "lmb_db_download": ([vp, u64, u64, vp], C.c_int),
        "lmb_db_info": ([vp, C.POINTER(u64), C.POINTER(i32)], C.c_int),
        "lmb_image_load": ([vp, i32, vp, i32, i32, dp], C.c_int),
        "lmb_image_load_batch": ([vp, vp, vp, i32, i32, dp], C.c_int),
        "lmb_match": ([vp, u64, i32, dbl, i32], C.c_int),
        "lmb_results": ([vp, i32, vp, u64, C.POINTER(u64), C.POINTER(u64)], C.c_int),
        "lmb_results_batch": ([vp, vp, i32, vp, u64, vp, vp], C.c_int),
        "lmb_last_pass_ms": ([vp, C.POINTER(C.c_float), C.POINTER(C.c_float)], C.c_int),
        "lmb_engine_bytes": ([vp, C.POINTER(u64), C.POINTER(u64)], C.c_int),
        "lmb_post_process": ([C.POINTER(LmbGeometry), C.POINTER(LmbPostParams), vp, u64, vp, vp,
                              C.c_int64, vp, vp, i32, C.POINTER(LmbPostOutput)], C.c_int),
        "lmb_post_free": ([C.POINTER(LmbPostOutput)], None),
        "lmb_merge_clusters": ([i32, i32, dbl, dbl, vp, u64, vp, vp, C.c_int64, i32,
                                C.POINTER(i32), vp, vp, vp], C.c_int),
        "lmb_order_survivors_noalloc": ([vp, u64, vp, vp], C.c_int),
        "lmb_host_alloc": ([u64, C.POINTER(vp)], C.c_int),
        "lmb_host_free": ([vp], C.c_int),
        "lmb_pre_create": ([i32, i32, i32, C.POINTER(vp)], C.c_int),
        "lmb_pre_destroy": ([vp], C.c_int),
        "lmb_pre_median": ([vp, vp, i32, i32, i32, vp], C.c_int),
        "lmb_pre_set_background": ([vp, vp], C.c_int),
        "lmb_pre_get_background": ([vp, vp], C.c_int),
        "lmb_pre_segment": ([vp, vp, i32, C.POINTER(LmbPreParams), C.POINTER(LmbPreCounts)],
                            C.c_int),
        "lmb_pre_segment_thresholded": ([vp, vp, i32, C.POINTER(LmbPreCounts)], C.c_int),
        "lmb_pre_centres": ([vp, vp, i32], C.c_int),
        "lmb_pre_stats": ([vp, vp, i32], C.c_int),
        "lmb_pre_images": ([vp, vp, vp, vp, vp], C.c_int),
        "lmb_pre_blur": ([vp, vp, i32, vp, i32], C.c_int),
        "lmb_pre_timings": ([vp, vp, i32], C.c_int),
        "lmb_pre_blur_to_slot": ([vp, vp, i32, vp, i32, i32, dp], C.c_int),
        "lmb_refine_create": ([i32, C.POINTER(LmbGeometry), C.POINTER(LmbPostParams), vp, i32,
                               C.POINTER(vp)], C.c_int),
        "lmb_refine_destroy": ([vp], C.c_int),
        "lmb_refine_dims": ([vp, C.POINTER(i32)], C.c_int),
        "lmb_refine_set_images": ([vp, vp, i32], C.c_int),
        "lmb_refine_set_grains": ([vp, vp, vp, i32, vp], C.c_int),
        "lmb_refine_start": ([vp, vp, vp, vp], C.c_int),
        "lmb_refine_evaluate": ([vp, vp, vp, C.c_int64, vp], C.c_int),
        "lmb_refine_fit": ([vp, i32, i32, dbl, vp, vp, vp], C.c_int),
        "lmb_refine_last_stats": ([vp, C.POINTER(C.c_int64), C.POINTER(i32),
                                   C.POINTER(C.c_float)], C.c_int),
        "lmb_post_last_refine_stats": ([C.POINTER(i32), C.POINTER(C.c_int64), C.POINTER(i32),
                                        C.POINTER(C.c_float)], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def device_info(device: int = 0) -> dict:
    fr, tot = C.c_uint64(), C.c_uint64()
    l2, sms = C.c_int32(), C.c_int32()
    check(lib().lmb_device_info(int(device), C.byref(fr), C.byref(tot), C.byref(l2), C.byref(sms)))
    return {"free": fr.value, "total": tot.value, "l2": l2.value, "sms": sms.value}


def check(rc: int) -> int:
    if rc != LMB_OK:
        msg = lib().lmb_last_error().decode(errors="replace")
        if rc == LMB_ERR_OVERFLOW:
            raise OverflowError_(rc, msg)
        if rc == LMB_ERR_TIMEOUT:
            raise TimeoutError_(rc, msg)
        raise LmbError(rc, msg)
    return rc
