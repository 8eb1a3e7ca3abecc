"""ctypes binding of liblre_cuda.so (the C ABI in include/lre_cuda.h).

The library is built in-tree by ``python -m libraw_enhanced_b200.build`` (or
``__graft_entry__.build()``).  There is no CPU fallback: if the library is
missing, or no sm_100 device is present, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblre_cuda.so")

LRE_OK = 0
STATUS_NAMES = {
    0: "LRE_OK",
    1: "LRE_ERR_INVALID_ARGUMENT",
    2: "LRE_ERR_CUDA",
    3: "LRE_ERR_OUT_OF_MEMORY",
    4: "LRE_ERR_NO_DEVICE",
    5: "LRE_ERR_TIMEOUT",
    6: "LRE_ERR_INJECTED",
    7: "LRE_ERR_BUSY",
}
FILTERS_XTRANS = 9


class LibRawError(RuntimeError):
    """Failure reported by the CUDA develop backend (mirrors libraw_enhanced's
    LibRawError, core/python_bindings.cpp:503-505)."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


class DevelopParams(C.Structure):
    _fields_ = [
        ("filters", C.c_uint32),
        ("xtrans", C.c_char * 36),
        ("cam_mul", C.c_float * 4),
        ("maximum_value", C.c_float),
        ("xtrans_passes", C.c_int),
        ("lateral_ca_correction", C.c_int),
        ("lateral_ca_cell_size", C.c_int),
        ("lateral_ca_max_iterations", C.c_int),
        ("lateral_ca_max_shift", C.c_float),
        ("lateral_ca_min_confidence", C.c_float),
        ("lateral_ca_pyramid_levels", C.c_int),
        ("axial_ca_correction", C.c_int),
        ("axial_ca_radius", C.c_int),
        ("axial_ca_epsilon", C.c_float),
        ("axial_ca_strength", C.c_float),
        ("defringe", C.c_int),
        ("defringe_radius", C.c_float),
        ("defringe_edge_threshold", C.c_float),
        ("defringe_chroma_threshold", C.c_float),
        ("defringe_strength", C.c_float),
        ("defringe_green", C.c_int),
        ("defringe_green_strength", C.c_float),
        ("tone_mapping", C.c_int),
        ("tone_after_scale", C.c_float),
        ("output_bits", C.c_int),
        ("stage_order", C.c_int),
        ("demosaic_algorithm", C.c_int),
        ("highlight_recovery", C.c_int),
        ("highlight_threshold", C.c_float),
    ]


class WbInputs(C.Structure):
    _fields_ = [
        ("user_mul", C.c_float * 4),
        ("pre_mul", C.c_float * 4),
        ("cam_mul", C.c_float * 4),
        ("white", (C.c_ushort * 8) * 8),
        ("cblack", C.c_uint * 4),
        ("use_auto_wb", C.c_int),
        ("use_camera_wb", C.c_int),
        ("camerawb_fallback_to_daylight", C.c_int),
        ("as_shot_wb_applied", C.c_int),
        ("colors", C.c_int),
        ("no_auto_scale", C.c_int),
    ]


class WbResult(C.Structure):
    _fields_ = [
        ("scale_mul", C.c_float * 4),
        ("pre_mul", C.c_float * 4),
        ("maximum", C.c_uint),
        ("auto_wb", C.c_int),
        ("bad_camera_wb", C.c_int),
    ]


class RawFrame(C.Structure):
    _fields_ = [
        ("raw_width", C.c_size_t),
        ("raw_height", C.c_size_t),
        ("raw_pitch", C.c_size_t),
        ("top_margin", C.c_size_t),
        ("left_margin", C.c_size_t),
        ("width", C.c_size_t),
        ("height", C.c_size_t),
        ("shrink", C.c_int),
        ("filters", C.c_uint32),
        ("xtrans", C.c_char * 36),
        ("cblack", C.c_uint * 42),
        ("black", C.c_uint),
        ("maximum", C.c_uint),
        ("green_matching", C.c_int),
        ("wb", C.c_float * 4),
        ("adjust_maximum_thr", C.c_float),
        ("data_maximum", C.c_float),
        ("derive_wb", C.c_int),
        ("wb_in", WbInputs),
        ("fuji_width", C.c_int),
        ("fuji_layout", C.c_int),
    ]


class Tuning(C.Structure):
    _fields_ = [("lanes", C.c_int), ("axial_strip", C.c_int), ("axial_rows", C.c_int), ("blur_tile", C.c_int)]


class Image(C.Structure):
    _fields_ = [
        ("mosaic", C.c_void_p),
        ("out", C.c_void_p),
        ("width", C.c_size_t),
        ("height", C.c_size_t),
        ("params", DevelopParams),
    ]


class BatchConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("lanes", C.c_int), ("use_graph", C.c_int), ("autotune", C.c_int)]


class BatchStats(C.Structure):
    _fields_ = [
        ("ms", C.c_double),
        ("graph", C.c_int),
        ("lanes", C.c_int),
        ("launches", C.c_uint64),
        ("tune_ms", C.c_double),
    ]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("lanes", C.c_int), ("device_budget_bytes", C.c_size_t),
                ("decode_threads", C.c_int)]


class RequestStats(C.Structure):
    _fields_ = [
        ("status", C.c_int),
        ("lane", C.c_int),
        ("queue_ms", C.c_double),
        ("run_ms", C.c_double),
        ("total_ms", C.c_double),
        ("device_bytes", C.c_size_t),
        ("decode_ms", C.c_double),
    ]


# lre_decode_fn: status (void* user, float* mosaic, size_t width, size_t height)
DECODE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_float), C.c_size_t, C.c_size_t)


_p = C.c_void_p
_sz = C.c_size_t
_f = C.c_float
_i = C.c_int
_st = C.c_int

# name -> (restype, argtypes); every symbol include/lre_cuda.h declares.
SIGNATURES = {
    "lre_create": (_st, [_i, C.POINTER(_p)]),
    "lre_destroy": (None, [_p]),
    "lre_last_error": (C.c_char_p, [_p]),
    "lre_device_info": (_st, [_p, C.c_char_p, _sz]),
    "lre_is_available": (_i, []),
    "lre_abi_version": (_i, []),
    "lre_set_stream": (_st, [_p, _p]),
    "lre_get_stream": (_p, [_p]),
    "lre_synchronize": (_st, [_p]),
    "lre_reserve_workspace": (_st, [_p, _sz]),
    "lre_workspace_bytes": (_sz, [_p]),
    "lre_launch_count": (C.c_uint64, [_p]),
    "lre_host_alloc": (_st, [_p, _sz, C.POINTER(_p)]),
    "lre_host_free": (_st, [_p, _p]),
    "lre_inject_fault": (None, [_p, _i]),
    "lre_set_wait_limit": (_st, [_p, C.c_longlong]),
    "lre_inject_sweep_stall": (None, [_p, _i]),
    "lre_demosaic_bayer_amaze": (_st, [_p, _p, _p, _sz, _sz, C.c_uint32, _p, _f]),
    "lre_demosaic_xtrans_1pass": (_st, [_p, _p, _p, _sz, _sz, _p, _p, _f]),
    "lre_demosaic_xtrans_3pass": (_st, [_p, _p, _p, _sz, _sz, _p, _p, _f]),
    "lre_apply_white_balance": (_st, [_p, _p, _p, _sz, _sz, _p, C.c_uint32, _p]),
    "lre_tone_mapping": (_st, [_p, _p, _p, _sz, _sz, _f]),
    "lre_detail_tonemap": (_st, [_p, _p, _p, _sz, _sz]),
    "lre_enhance_micro_contrast": (_st, [_p, _p, _p, _sz, _sz, _f, _f, _f, _p]),
    "lre_ca_register_lateral": (_st, [_p, _p, _p, _sz, _sz, _i, _i, _f, _f, _i]),
    "lre_ca_axial_cleanup": (_st, [_p, _p, _p, _sz, _sz, _i, _f, _f]),
    "lre_defringe": (_st, [_p, _p, _p, _sz, _sz, _f, _f, _f, _f, _i, _f]),
    "lre_black_level": (_st, [_p, _p, _sz, _sz, _p, _sz, C.c_uint, C.c_uint]),
    "lre_adjust_maximum": (_st, [_p, _p, _sz, _sz, C.c_uint32, _f, C.POINTER(_f), C.POINTER(_f)]),
    "lre_quantize_u16": (_st, [_p, _p, _p, _sz]),
    "lre_quantize_u8": (_st, [_p, _p, _p, _sz]),
    "lre_dev_demosaic_bayer_amaze": (_st, [_p, _p, _p, _sz, _sz, C.c_uint32, _p, _f]),
    "lre_dev_demosaic_xtrans": (_st, [_p, _p, _p, _sz, _sz, _p, _f, _i]),
    "lre_dev_tone_mapping": (_st, [_p, _p, _p, _sz, _sz, _f]),
    "lre_dev_detail_tonemap": (_st, [_p, _p, _p, _sz, _sz]),
    "lre_dev_enhance_micro_contrast": (_st, [_p, _p, _p, _sz, _sz, _f, _f, _f, _p]),
    "lre_dev_ca_register_lateral": (_st, [_p, _p, _p, _sz, _sz, _i, _i, _f, _f, _i]),
    "lre_dev_ca_axial_cleanup": (_st, [_p, _p, _p, _sz, _sz, _i, _f, _f]),
    "lre_dev_defringe": (_st, [_p, _p, _p, _sz, _sz, _f, _f, _f, _f, _i, _f]),
    "lre_dev_quantize_u16": (_st, [_p, _p, _p, _sz]),
    "lre_dev_ca_axial_cleanup_noalloc": (_st, [_p, _p, _sz, _sz, _i, _f, _f, _p]),
    "lre_develop_params_default": (None, [C.POINTER(DevelopParams)]),
    "lre_develop": (_st, [_p, _p, _p, _sz, _sz, C.POINTER(DevelopParams)]),
    "lre_dev_develop": (_st, [_p, _p, _p, _sz, _sz, C.POINTER(DevelopParams)]),
    "lre_demosaic_bayer_linear": (_st, [_p, _p, _p, _sz, _sz, C.c_uint32, _f]),
    "lre_dev_demosaic_bayer_linear": (_st, [_p, _p, _p, _sz, _sz, C.c_uint32, _f]),
    "lre_demosaic_bayer_dcb": (_st, [_p, _p, _p, _sz, _sz, C.c_uint32, _f, C.c_int, C.c_int]),
    "lre_dev_demosaic_bayer_dcb": (_st, [_p, _p, _p, _sz, _sz, C.c_uint32, _f, C.c_int, C.c_int]),
    "lre_demosaic_bayer_aahd": (_st, [_p, _p, _p, _sz, _sz, C.c_uint32, _f]),
    "lre_recover_highlights": (_st, [_p, _p, _p, _sz, _sz, _f, _p, _p, _p]),
    "lre_dev_recover_highlights": (_st, [_p, _p, _p, _sz, _sz, _f, _p, _p, _p]),
    "lre_dev_demosaic_bayer_aahd": (_st, [_p, _p, _p, _sz, _sz, C.c_uint32, _f]),
    "lre_convert_color_space": (_st, [_p, _p, _p, _sz, _sz, _p]),
    "lre_gamma_correct": (_st, [_p, _p, _p, _sz, _sz, _f, _f, _i]),
    "lre_dev_convert_color_space": (_st, [_p, _p, _p, _sz, _sz, _p]),
    "lre_dev_gamma_correct": (_st, [_p, _p, _p, _sz, _sz, _f, _f, _i]),
    "lre_output_epilogue": (_st, [_p, _p, _p, _sz, _sz, _p, _f, _f, _i, _i]),
    "lre_dev_output_epilogue": (_st, [_p, _p, _p, _sz, _sz, _p, _f, _f, _i, _i]),
    "lre_raw2image": (_st, [_p, _p, C.POINTER(RawFrame), _p]),
    "lre_green_matching": (_st, [_p, _p, _sz, _sz, C.c_uint32, C.c_uint]),
    "lre_develop_raw": (_st, [_p, _p, C.POINTER(RawFrame), _p, C.POINTER(DevelopParams), C.POINTER(_f)]),
    "lre_dev_develop_raw": (_st, [_p, _p, C.POINTER(RawFrame), _p, C.POINTER(DevelopParams), C.POINTER(_f)]),
    "lre_wb_needs_channel_sums": (_i, [C.POINTER(WbInputs)]),
    "lre_wb_multipliers": (_st, [C.POINTER(WbInputs), C.c_uint32, C.c_uint, C.c_uint, _p, _p, C.POINTER(WbResult)]),
    "lre_channel_sums": (_st, [_p, _p, _sz, _sz, C.c_uint32, _p, _p, _p]),
    "lre_dev_channel_sums": (_st, [_p, _p, _sz, _sz, C.c_uint32, _p, _p, _p]),
    "lre_fuji_rotate_size": (_st, [_i, _i, _sz, _sz, C.POINTER(_sz), C.POINTER(_sz)]),
    "lre_fuji_rotate": (_st, [_p, _p, _sz, _sz, _i, _i, _p]),
    "lre_dev_fuji_rotate": (_st, [_p, _p, _sz, _sz, _i, _i, _p]),
    "lre_set_tuning": (_st, [_p, C.POINTER(Tuning)]),
    "lre_get_tuning": (_st, [_p, C.POINTER(Tuning)]),
    "lre_batch_create": (_st, [C.POINTER(BatchConfig), C.POINTER(_p)]),
    "lre_batch_destroy": (None, [_p]),
    "lre_batch_last_error": (C.c_char_p, [_p]),
    "lre_batch_run": (_st, [_p, C.POINTER(Image), _sz, C.POINTER(BatchStats)]),
    "lre_dev_batch_run": (_st, [_p, C.POINTER(Image), _sz, C.POINTER(BatchStats)]),
    "lre_batch_get_tuning": (_st, [_p, C.POINTER(Tuning)]),
    "lre_batch_set_tuning": (_st, [_p, C.POINTER(Tuning)]),
    "lre_server_create": (_st, [C.POINTER(ServerConfig), C.POINTER(_p)]),
    "lre_server_destroy": (None, [_p]),
    "lre_server_last_error": (C.c_char_p, [_p]),
    "lre_server_submit": (_st, [_p, C.POINTER(Image), C.POINTER(C.c_uint64)]),
    "lre_server_submit_decode": (_st, [_p, C.POINTER(Image), DECODE_FN, _p, C.POINTER(C.c_uint64)]),
    "lre_server_wait": (_st, [_p, C.c_uint64, C.c_double, C.POINTER(RequestStats)]),
    "lre_server_memory": (_st, [_p, C.POINTER(_sz), C.POINTER(_sz)]),
}

_lib = None
_lock = threading.Lock()


def load() -> C.CDLL:
    """Load liblre_cuda.so (raises if it was not built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is missing: build it with `python -m libraw_enhanced_b200.build` "
                    "(there is no CPU fallback for the develop backend)"
                )
            lib = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib
