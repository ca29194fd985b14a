"""ctypes binding of ``libslm_b200.so`` (the C ABI declared in ``include/slm_b200.h``).

There is no fallback: if the library is missing or no CUDA device is visible,
every product call raises.  Build it with ``python -m slm_b200.build``.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libslm_b200.so")

SLM_OK = 0
SLM_ERR_ARGS = 1
SLM_ERR_CUDA = 2
SLM_ERR_CAPACITY = 3
SLM_ERR_ITERATION_CAP = 4
SLM_ERR_UNSUPPORTED = 5

SLM_RK2 = 2
SLM_RK4 = 4
SLM_SCHED_PLAIN = 0
SLM_SCHED_PERSISTENT = 1


class SlmLaunch(ctypes.Structure):
    _fields_ = [("schedule", ctypes.c_int32), ("integrator", ctypes.c_int32),
                ("block_threads", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
                ("chunk", ctypes.c_int32), ("reserved", ctypes.c_int32 * 3)]


class SlmTile(ctypes.Structure):
    _fields_ = [("grid_offset", ctypes.c_uint64), ("nx_padded", ctypes.c_uint32),
                ("ny_padded", ctypes.c_uint32), ("seed_begin", ctypes.c_uint32),
                ("n_seeds", ctypes.c_uint32), ("grid_scale", ctypes.c_float),
                ("combo_factor", ctypes.c_float), ("dt_max", ctypes.c_float),
                ("reserved", ctypes.c_uint32)]


class SlmPreprocessParams(ctypes.Structure):
    _fields_ = [("pixel_size", ctypes.c_double), ("vecsum_threshold", ctypes.c_double),
                ("divergence_threshold", ctypes.c_double), ("curl_threshold", ctypes.c_double),
                ("pad_width", ctypes.c_uint32), ("do_normalize_speed", ctypes.c_uint32)]


class SlmError(RuntimeError):
    def __init__(self, code, message):
        super().__init__("slm_b200 error {}: {}".format(code, message))
        self.code = code


_P = ctypes.c_void_p
_I = ctypes.c_int32
_U = ctypes.c_uint32

# name -> (restype, argtypes); every symbol of include/slm_b200.h
SIGNATURES = {
    "slm_version": (ctypes.c_char_p, []),
    "slm_last_error": (ctypes.c_char_p, []),
    "slm_device_count": (ctypes.c_int, []),
    "slm_fields_workspace_words": (ctypes.c_size_t, []),
    "slm_integrate_fields": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "slm_integrate_fields_noalloc": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "slm_integrate_fields_scheduled": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "slm_integrate_fields_pair": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, ctypes.c_uint64, _P, _P, _P, _P]),
    "slm_integrate_fields_batched": (ctypes.c_int, [_P, _P, _P, _U, _U, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "slm_fields_finish": (ctypes.c_int, [_P, _U, _U, ctypes.c_double, ctypes.c_double, _I, _P, _U, _P, _P,
                                         _P, _P]),
    "slm_integrate_trajectory": (ctypes.c_int, [_P, _I, _U, _P, _P, _P, _P, _P, _P, _P, _P]),
    "slm_histogram_univariate": (ctypes.c_int, [_P, _P, _U, _P, _P]),
    "slm_histogram_bivariate": (ctypes.c_int, [_P, _P, _U, _P, _P]),
    "slm_pdf_univariate": (ctypes.c_int, [_P, _P, _P, _P]),
    "slm_pdf_bivariate_rows": (ctypes.c_int, [_P, _P, _P, _P]),
    "slm_pdf_bivariate_cols": (ctypes.c_int, [_P, _P, _P, _P]),
    "slm_connect_channels": (ctypes.c_int, [_P, _U, _P, _P, _P, _P, _P, _P]),
    "slm_map_channel_heads": (ctypes.c_int, [_P, _U, _P, _P, _P, _P, _P]),
    "slm_prune_channel_heads": (ctypes.c_int, [_P, _U, _P, _P, _P, _P, _P]),
    "slm_count_downchannels_workspace": (ctypes.c_size_t, [_U, ctypes.c_uint64]),
    "slm_count_downchannels": (ctypes.c_int, [_P, _U, _P, _P, _P, _P, _P, _P, _P, ctypes.c_size_t, _P, _P]),
    "slm_flag_downchannels_workspace": (ctypes.c_size_t, [_U, _U]),
    "slm_flag_downchannels": (ctypes.c_int, [_P, _U, _P, _P, _P, _P, _P, _P, _P, ctypes.c_size_t, _P, _P]),
    "slm_label_confluences": (ctypes.c_int, [_P, _U, _P, _P, _P, _P, _P, _P, _P, _P]),
    "slm_segment_downchannels": (ctypes.c_int, [_P, _U, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "slm_segment_hillslopes": (ctypes.c_int, [_P, _U, _P, _P, _P, _P, _P, _P, _P, _P]),
    "slm_subsegment_channel_edges": (ctypes.c_int, [_P, _U, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "slm_subsegment_flanks": (ctypes.c_int, [_P, _U, _P, _P, _P, _P, _P, _P, _P, _P]),
    "slm_fix_flanks_workspace": (ctypes.c_size_t, [_U, _U, ctypes.c_uint64]),
    "slm_fix_right_flanks": (ctypes.c_int, [_P, _U, _P, _P, _P, _P, _P, _P, _P, _P, ctypes.c_size_t, _P, _P]),
    "slm_fix_left_flanks": (ctypes.c_int, [_P, _U, _P, _P, _P, _P, _P, _P, _P, _P, ctypes.c_size_t, _P, _P]),
    "slm_hillslopes": (ctypes.c_int, [_P, _U, _P, _P, _P, _P, _P, _P, _P]),
    "slm_hillslope_lengths": (ctypes.c_int, [_P, _U, _P, _P, _P, _P, _P, _P, _P]),
    "slm_thin": (ctypes.c_int, [_P, _P, _U, _U, _U, _P, _P, _P]),
    "slm_create_seeds": (ctypes.c_int, [_P, _U, _U, _U, ctypes.c_int, _U, _P, ctypes.c_uint64, _P, _P]),
    "slm_create_seeds_device_workspace": (ctypes.c_size_t, [ctypes.c_uint64]),
    "slm_selftest_div6": (ctypes.c_int, [_P, _P]),
    "slm_exclusive_scan_u64_scratch": (ctypes.c_size_t, [ctypes.c_uint32]),
    "slm_exclusive_scan_u64": (ctypes.c_int, [_P, ctypes.c_uint32, _P, _P, ctypes.c_size_t, _P]),
    "slm_selftest_cvt_i8": (ctypes.c_int, [_P, _P]),
    "slm_fmm_lengths": (ctypes.c_int, [_P, _P, ctypes.c_int, ctypes.c_int, _U, _P, _P, _P, ctypes.c_int,
                                       ctypes.c_int64, ctypes.c_int, ctypes.c_double, _P, _P, _P, _P, _P, _P, _P,
                                       _P, _P, _P]),
    "slm_create_seeds_device": (ctypes.c_int, [_P, _U, _U, _U, ctypes.c_int, _U, _P, ctypes.c_uint64, _P, _P,
                                               _P, ctypes.c_size_t, _P]),
    "slm_preprocess": (ctypes.c_int, [_P, ctypes.c_int, _U, _U, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "slm_pick_seeds_workspace": (ctypes.c_size_t, [_U]),
    "slm_pick_seeds": (ctypes.c_int, [_P, _P, _U, _I, _U, _U, _U, _P, _U, _P, _P, ctypes.c_size_t, _P]),
    "slm_map_channels": (ctypes.c_int, [_P, _P, ctypes.c_float, _U, _U, _P, _P]),
    "slm_flag_op": (ctypes.c_int, [_P, _P, _U, _I, _U, _U, _P]),
    "slm_relabel_workspace": (ctypes.c_size_t, [_U]),
    "slm_relabel": (ctypes.c_int, [_P, _U, _P, ctypes.c_size_t, _P, _P]),
    "slm_signed_labels": (ctypes.c_int, [_P, _U, _U, _P]),
    "slm_cnn_gather": (ctypes.c_int, [_P, _U, _U, _U, _P, _P, _U, _P, _P]),
    "slm_cnn_rearrange": (ctypes.c_int, [_P, _U, _P, _I, _P]),
    "slm_gemm": (ctypes.c_int, [_I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _I, _I, _I, _P, _P, _P]),
    "slm_relu_backward": (ctypes.c_int, [_P, _P, ctypes.c_uint64, _P, _P]),
    "slm_bias_grad": (ctypes.c_int, [_P, ctypes.c_uint64, _I, _P, _P]),
    "slm_mse": (ctypes.c_int, [_P, _P, _P, ctypes.c_uint64, ctypes.c_float, _P, _P, _P]),
    "slm_adam": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_uint64, ctypes.c_float, ctypes.c_float,
                                ctypes.c_float, ctypes.c_float, _I, _I, _P]),
    "slm_cnn_infer": (ctypes.c_int, [_P, _U, _U, _U, _P, _P, _U, _P, _P, _P, _P, _P, _P, _P, _P]),
    "slm_order_spatial_bins": (ctypes.c_uint32, [_U, _U, _U, _I]),
    "slm_order_spatial": (ctypes.c_int, [_P, _U, _U, _U, _U, _P, _U, _U, ctypes.c_float, _P, _U, _P, _P]),
    "slm_order_by_prediction": (ctypes.c_int, [_P, _U, _U, _U, ctypes.c_float, ctypes.c_float, _U,
                                               _P, _P, _P]),
}

_lock = threading.Lock()
_lib = None


def load():
    """Load the library and bind every entry point (raises if it is missing)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    "{} is not built; run `python -m slm_b200.build` (nvcc, sm_100a)".format(LIB_PATH))
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
        return _lib


def check(rc):
    if rc != SLM_OK:
        msg = load().slm_last_error()
        raise SlmError(rc, msg.decode() if msg else "")


def ptr(t):
    """Device (or host) address of a torch tensor / numpy array, or None."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return ctypes.c_void_p(t.data_ptr())
    return ctypes.c_void_p(t.ctypes.data)


def sref(struct):
    return ctypes.cast(ctypes.byref(struct), ctypes.c_void_p)
