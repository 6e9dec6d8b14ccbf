"""ctypes binding of libtomgpu.so (include/tomgpu.h).

The library is built in-tree (``tom_b200/build_ext.py``) and loaded from this
package directory.  There is no fallback: if the library is missing or no GPU
is present, the calls raise.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtomgpu.so")
HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "tomgpu.h")

c_int_p = ctypes.POINTER(ctypes.c_int)
c_float_p = ctypes.POINTER(ctypes.c_float)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_void_p = ctypes.c_void_p

TOMGPU_OK = 0
TOMGPU_ERR_ARG = 1
TOMGPU_ERR_UNSUPPORTED = 2
TOMGPU_ERR_OOM = 3
TOMGPU_ERR_CUDA = 4
TOMGPU_ERR_STATE = 5
TOMGPU_ERR_DEVICE = 6
TOMGPU_ERR_TIMEOUT = 7
KERNEL_CLASSES = ("rotate", "filter", "spec_x", "spec_z", "corr_y", "inv_z", "c2r_flcf")
TOMGPU_EULER_DEG = 1
TOMGPU_MATRIX = 3


class TomGpuError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"tomgpu error {status}: {msg}")
        self.status = status


class MatchParams(ctypes.Structure):
    _fields_ = [("batch", ctypes.c_int), ("wedge_fp64", ctypes.c_int), ("path", ctypes.c_int),
                ("reserved", ctypes.c_int * 5)]


class AlignJob(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int * 3), ("ref", ctypes.c_void_p), ("part", ctypes.c_void_p),
                ("mask", ctypes.c_void_p), ("mask_ccf", ctypes.c_void_p), ("wedge_ref", ctypes.c_void_p),
                ("wedge_part", ctypes.c_void_p), ("phi", ctypes.c_float * 3), ("psi", ctypes.c_float * 3),
                ("theta", ctypes.c_float * 3)]


class AlignParams(ctypes.Structure):
    _fields_ = [("path", ctypes.c_int), ("batch_bytes", ctypes.c_size_t)]


class AvgItem(ctypes.Structure):
    _fields_ = [("particle", ctypes.c_void_p), ("wedge", ctypes.c_void_p), ("shift", ctypes.c_float * 3),
                ("angles", ctypes.c_float * 3)]


class WedgeSpec(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("angle_deg", ctypes.c_float), ("volume", ctypes.c_void_p)]


# name -> (restype, argtypes)
_SIGS = {
    "tomgpu_version": (ctypes.c_char_p, []),
    "tomgpu_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "tomgpu_last_error": (ctypes.c_char_p, [c_void_p]),
    "tomgpu_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(c_void_p)]),
    "tomgpu_ctx_destroy": (ctypes.c_int, [c_void_p]),
    "tomgpu_ctx_set_stream": (ctypes.c_int, [c_void_p, c_void_p]),
    "tomgpu_ctx_synchronize": (ctypes.c_int, [c_void_p]),
    "tomgpu_ctx_trim": (ctypes.c_int, [c_void_p]),
    "tomgpu_ctx_launch_count": (ctypes.c_int64, [c_void_p]),
    "tomgpu_ctx_profile": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "tomgpu_ctx_profile_read": (ctypes.c_int, [c_void_p, ctypes.c_int, c_double_p, ctypes.POINTER(ctypes.c_int64)]),
    "tomgpu_rotate3d": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_int_p, c_float_p, ctypes.c_int, c_float_p]),
    "tomgpu_rotate3d_batch_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_int_p, c_float_p, ctypes.c_int,
                                                 c_float_p, c_void_p]),
    "tomgpu_euler_matrix": (ctypes.c_int, [c_float_p, c_float_p]),
    "tomgpu_peak": (ctypes.c_int, [c_void_p, c_void_p, c_int_p, c_float_p, c_int_p]),
    "tomgpu_peak_dev": (ctypes.c_int, [c_void_p, c_void_p, c_int_p, c_float_p, c_int_p]),
    "tomgpu_topk_dev": (ctypes.c_int, [c_void_p, c_void_p, c_int_p, ctypes.c_int, ctypes.c_double, c_float_p,
                                       c_int_p]),
    "tomgpu_peak_radius_dev": (ctypes.c_int, [c_void_p, c_void_p, c_int_p, ctypes.c_double, c_float_p, c_int_p]),
    "tomgpu_topk_noalloc_dev": (ctypes.c_int, [c_void_p, c_void_p, c_int_p, ctypes.c_int, ctypes.c_double,
                                               c_void_p, c_void_p]),
    "tomgpu_peak_spline_dev": (ctypes.c_int, [c_void_p, c_void_p, c_int_p, c_int_p, c_double_p, c_double_p]),
    "tomgpu_weight3d": (ctypes.c_int, [c_void_p, c_int_p, c_double_p, ctypes.c_int, ctypes.c_double, c_void_p]),
    "tomgpu_wedge_dev": (ctypes.c_int, [c_void_p, c_int_p, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                        c_void_p]),
    "tomgpu_em_read": (ctypes.c_int, [ctypes.c_char_p, c_int_p, c_void_p, ctypes.c_size_t]),
    "tomgpu_em_write": (ctypes.c_int, [ctypes.c_char_p, c_void_p, c_int_p, ctypes.c_char_p]),
    "tomgpu_apply_weight_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_int_p, c_void_p]),
    "tomgpu_fft3d_c2c_dev": (ctypes.c_int, [c_void_p, c_void_p, c_int_p, ctypes.c_int, ctypes.c_int]),
    "tomgpu_fft3d_r2c_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_int_p, ctypes.c_int]),
    "tomgpu_fft3d_c2r_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_int_p, ctypes.c_int]),
    "tomgpu_match_plan_create": (ctypes.c_int, [c_void_p, c_int_p, c_int_p, ctypes.POINTER(MatchParams),
                                                ctypes.POINTER(c_void_p)]),
    "tomgpu_match_plan_destroy": (ctypes.c_int, [c_void_p]),
    "tomgpu_match_plan_bytes": (ctypes.c_int64, [c_void_p]),
    "tomgpu_match_set_volume_dev": (ctypes.c_int, [c_void_p, c_void_p]),
    "tomgpu_match_set_template_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "tomgpu_match_init_results_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p]),
    "tomgpu_match_run_dev": (ctypes.c_int, [c_void_p, c_float_p, ctypes.c_int, ctypes.c_int, c_void_p, c_void_p]),
    "tomgpu_match_corr_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p]),
    "tomgpu_match_autotune": (ctypes.c_int, [c_void_p, c_float_p, ctypes.c_int, c_int_p, ctypes.c_int, c_int_p,
                                             c_float_p]),
    "tomgpu_match_set_template_raw_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p]),
    "tomgpu_match_init_analysis_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "tomgpu_match_run_analysis_dev": (ctypes.c_int, [c_void_p, c_float_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                     c_void_p, c_void_p, c_void_p, c_void_p]),
    "tomgpu_av3_average_add_dev": (ctypes.c_int, [c_void_p, c_int_p, ctypes.POINTER(AvgItem), ctypes.c_int,
                                                  c_void_p, c_void_p]),
    "tomgpu_av3_average_final_dev": (ctypes.c_int, [c_void_p, c_int_p, c_void_p, c_void_p, c_void_p]),
    "tomgpu_corr3d_peaks_dev": (ctypes.c_int, [c_void_p, c_int_p, ctypes.POINTER(c_void_p), ctypes.c_int,
                                               ctypes.POINTER(c_void_p), ctypes.c_int, c_double_p, ctypes.c_int,
                                               c_void_p, ctypes.POINTER(WedgeSpec), ctypes.POINTER(WedgeSpec),
                                               c_void_p, c_double_p, c_double_p, c_int_p]),
    "tomgpu_corr3d_peaks": (ctypes.c_int, [c_void_p, c_int_p, ctypes.POINTER(c_void_p), ctypes.c_int,
                                           ctypes.POINTER(c_void_p), ctypes.c_int, c_double_p, ctypes.c_int,
                                           c_void_p, ctypes.POINTER(WedgeSpec), ctypes.POINTER(WedgeSpec),
                                           c_void_p, c_double_p, c_double_p, c_int_p]),
    "tomgpu_cnn_conv3d_fwd_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, c_int_p, c_void_p, c_void_p,
                                                 ctypes.c_int, ctypes.c_int, ctypes.c_int, c_void_p]),
    "tomgpu_cnn_conv3d_bwd_data_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, c_int_p, c_void_p,
                                                      ctypes.c_int, ctypes.c_int, c_void_p]),
    "tomgpu_cnn_conv3d_bwd_weight_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, c_int_p, c_void_p,
                                                        ctypes.c_int, ctypes.c_int, c_void_p, c_void_p]),
    "tomgpu_cnn_dense_fwd_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int64, ctypes.c_int, c_void_p]),
    "tomgpu_cnn_dense_bwd_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int64, c_void_p, c_void_p, c_void_p]),
    "tomgpu_cnn_relu_bwd_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_int64]),
    "tomgpu_cnn_bce_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_int64, ctypes.c_float, c_void_p,
                                          c_void_p]),
    "tomgpu_cnn_softmax_ce_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_int, ctypes.c_int, c_void_p,
                                                 c_void_p]),
    "tomgpu_cnn_adam_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_int64,
                                           ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                           ctypes.c_int]),
    "tomgpu_cnn_gather_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, ctypes.c_int64, c_void_p, ctypes.c_int,
                                             c_void_p]),
    "tomgpu_cnn_scatter_add_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, ctypes.c_int64, c_void_p,
                                                  ctypes.c_int, c_void_p]),
    "tomgpu_unet_pack_weights_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                    c_void_p]),
    "tomgpu_unet_conv3_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_int_p,
                                             c_void_p, ctypes.c_int, c_void_p, ctypes.c_int, c_void_p, ctypes.c_int,
                                             ctypes.c_int, c_void_p, ctypes.c_int, ctypes.c_int]),
    "tomgpu_unet_conv3_wgrad_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                   c_int_p, c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                   c_void_p]),
    "tomgpu_unet_conv_first_dev": (ctypes.c_int, [c_void_p, c_void_p, c_int_p, c_void_p, c_void_p, c_void_p]),
    "tomgpu_unet_conv_first_wgrad_dev": (ctypes.c_int, [c_void_p, c_void_p, c_int_p, c_void_p, c_void_p, c_void_p]),
    "tomgpu_unet_head_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int64, c_void_p, ctypes.c_int, c_void_p]),
    "tomgpu_unet_head_bwd_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int64, c_void_p, c_void_p, c_void_p,
                                                c_void_p]),
    "tomgpu_unet_pool_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_int_p,
                                            c_void_p]),
    "tomgpu_unet_pool_bwd_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, c_int_p, c_void_p, ctypes.c_int,
                                                ctypes.c_int, c_void_p, ctypes.c_int]),
    "tomgpu_unet_upsample_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, c_int_p, c_void_p, ctypes.c_int,
                                                ctypes.c_int]),
    "tomgpu_unet_upsample_bwd_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                    c_int_p, c_void_p]),
    "tomgpu_unet_channel_sum_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                   ctypes.c_int64, c_void_p]),
    "tomgpu_unet_normalise_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int64, c_void_p]),
    "tomgpu_unet_bin2_dev": (ctypes.c_int, [c_void_p, c_void_p, c_int_p, c_void_p]),
    "tomgpu_unet_gather_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, c_void_p, ctypes.c_int, c_void_p]),
    "tomgpu_unet_scatter_add_dev": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, c_void_p, ctypes.c_int,
                                                   c_void_p, c_void_p]),
    "tomgpu_analyze_psr_dev": (ctypes.c_int, [c_void_p, c_void_p, c_int_p, c_int_p, c_void_p]),
    "tomgpu_template_autocorr_dev": (ctypes.c_int, [c_void_p, c_void_p, c_int_p, c_void_p]),
    "tomgpu_analyze_autocorr_dev": (ctypes.c_int, [c_void_p, c_void_p, c_int_p, c_void_p, c_int_p, c_void_p,
                                                   c_void_p]),
    "tomgpu_match_rescore_fp64_dev": (ctypes.c_int, [c_void_p, c_void_p, c_float_p, c_int_p, ctypes.c_int,
                                                     c_double_p]),
    "tomgpu_match_stats_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p]),
    "tomgpu_corr_dev": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_int_p, c_void_p, c_void_p, c_void_p,
                                       c_void_p]),
    "tomgpu_av3_align_dev": (ctypes.c_int, [c_void_p, ctypes.POINTER(AlignJob), ctypes.c_int, c_float_p, c_float_p,
                                            c_float_p]),
    "tomgpu_av3_align_ex_dev": (ctypes.c_int, [c_void_p, ctypes.POINTER(AlignJob), ctypes.c_int,
                                                ctypes.POINTER(AlignParams), c_float_p, c_float_p, c_float_p]),
    "tomgpu_av3_align": (ctypes.c_int, [c_void_p, ctypes.POINTER(AlignJob), ctypes.c_int, ctypes.POINTER(AlignParams),
                                        c_float_p, c_float_p, c_float_p]),
    "tomgpu_match": (ctypes.c_int, [c_void_p, c_void_p, c_int_p, c_void_p, c_int_p, c_void_p, c_void_p, c_float_p,
                                    ctypes.c_int, ctypes.POINTER(MatchParams), c_void_p, c_void_p]),
}

_lib = None


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not found: build it with `python -m tom_b200.build_ext` "
                              "(or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def declared_symbols():
    """Entry points declared in include/tomgpu.h."""
    import re
    txt = open(HEADER_PATH).read()
    return sorted(set(re.findall(r"\b(tomgpu_[a-z0-9_]+)\s*\(", txt)))


def check(status: int, ctx_handle=None):
    if status != TOMGPU_OK:
        msg = lib().tomgpu_last_error(ctx_handle)
        raise TomGpuError(status, (msg or b"").decode() or lib().tomgpu_status_string(status).decode())
