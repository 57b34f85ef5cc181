"""ctypes binding of ``include/ads_gpu.h`` (libads_gpu.so).

This is the binding a Python caller of the C ABI needs; the reference-shaped
classes in ``api.py`` sit on top of it.  Loading fails loudly when the native
library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import atexit
import ctypes as C
import os

from . import build as _build

ADS_OK = 0
ADS_ERR_INVALID_ARGUMENT = 1
ADS_ERR_OUT_OF_MEMORY = 2
ADS_ERR_CUDA = 3
ADS_ERR_DEVICE_TIMEOUT = 4
ADS_ERR_INTERNAL = 5
ADS_MEM_HOST = 0
ADS_MEM_DEVICE = 1
ADS_PRECISION_FP32 = 0
ADS_PRECISION_BF16 = 1

vp = C.c_void_p
i64 = C.c_int64
i32 = C.c_int32
f32 = C.c_float


class AdsRawArrays(C.Structure):
    _fields_ = [
        ("location", i32),
        ("n_spectra", i64),
        ("spectrum_delta_scan_idx", vp),
        ("isolation_lower_mz", vp),
        ("isolation_upper_mz", vp),
        ("spectrum_peak_start_idx", vp),
        ("spectrum_peak_stop_idx", vp),
        ("spectrum_cycle_idx", vp),
        ("spectrum_rt", vp),
        ("n_peaks", i64),
        ("peak_mz", vp),
        ("peak_intensity", vp),
        ("cycle", vp),
        ("cycle_shape", i64 * 4),
    ]


class AdsLibArrays(C.Structure):
    _fields_ = [
        ("location", i32),
        ("n_precursors", i64),
        ("precursor_idx", vp),
        ("precursor_mz_library", vp),
        ("precursor_mz", vp),
        ("precursor_rt_library", vp),
        ("precursor_rt", vp),
        ("precursor_naa", vp),
        ("flat_frag_start_idx", vp),
        ("flat_frag_stop_idx", vp),
        ("n_fragments", i64),
        ("fragment_mz_library", vp),
        ("fragment_mz", vp),
        ("fragment_intensity", vp),
        ("fragment_cardinality", vp),
        ("fragment_charge", vp),
        ("fragment_loss_type", vp),
        ("fragment_number", vp),
        ("fragment_position", vp),
        ("fragment_type", vp),
        ("precursor_rt_tolerance", vp),
    ]


class AdsSelectionParams(C.Structure):
    _fields_ = [
        ("fwhm_rt", f32),
        ("kernel_size", i64),
        ("peak_length", i64),
        ("mass_tolerance", f32),
        ("rt_tolerance", f32),
        ("candidate_count", i64),
        ("top_k_fragments", i64),
    ]


class AdsScoringParams(C.Structure):
    _fields_ = [
        ("mass_tolerance", f32),
        ("top_k_fragments", i64),
    ]


class AdsQuantParams(C.Structure):
    _fields_ = [
        ("tolerance_ppm", f32),
        ("top_k_fragments", i64),
    ]


class AdsEngineOptions(C.Structure):
    _fields_ = [
        ("precision", i32),
        ("verbose", i32),
        ("use_graph", i32),
        ("warps_per_block", i32),
        ("blocks_per_sm", i32),
        ("gather_mode", i32),
        ("time_stages", i32),
        ("cycles_per_lane", i32),
        ("stream", i64),
    ]


# name -> (restype, argtypes); every symbol declared in include/ads_gpu.h
SIGNATURES = {
    "ads_last_error": (C.c_char_p, []),
    "ads_version": (C.c_char_p, []),
    "ads_device_count": (C.c_int, []),
    "ads_dia_create": (C.c_int, [C.POINTER(AdsRawArrays), C.c_int, C.POINTER(vp)]),
    "ads_dia_destroy": (C.c_int, [vp]),
    "ads_dia_num_observations": (i64, [vp]),
    "ads_dia_memory_footprint_bytes": (i64, [vp]),
    "ads_dia_rt_values": (C.c_int, [vp, vp, i64, C.POINTER(i64)]),
    "ads_dia_cycle": (C.c_int, [vp, vp, i64, C.POINTER(i64 * 4)]),
    "ads_dia_rt_index": (C.c_int, [vp, vp, i64, C.POINTER(i64), C.POINTER(f32)]),
    "ads_dia_observation_info": (C.c_int, [vp, i64, C.POINTER(f32), C.POINTER(f32), C.POINTER(i64), C.POINTER(i64)]),
    "ads_dia_copy_observation": (C.c_int, [vp, i64, vp, vp, vp]),
    "ads_mz_grid_len": (i64, []),
    "ads_mz_grid": (C.c_int, [vp, i64]),
    "ads_lib_create": (C.c_int, [C.POINTER(AdsLibArrays), C.c_int, C.POINTER(vp)]),
    "ads_lib_destroy": (C.c_int, [vp]),
    "ads_lib_num_precursors": (i64, [vp]),
    "ads_lib_num_fragments": (i64, [vp]),
    "ads_selection_params_default": (None, [C.POINTER(AdsSelectionParams)]),
    "ads_engine_options_default": (None, [C.POINTER(AdsEngineOptions)]),
    "ads_gaussian_kernel": (C.c_int, [f32, f32, i64, f32, vp, i64, C.POINTER(i64)]),
    "ads_selftest_ln": (C.c_int, [C.c_int, C.c_uint32, C.c_uint32, C.POINTER(i64), C.POINTER(i64)]),
    "ads_selection_create": (C.c_int, [C.POINTER(AdsSelectionParams), C.POINTER(AdsEngineOptions), C.c_int, C.POINTER(vp)]),
    "ads_selection_destroy": (C.c_int, [vp]),
    "ads_selection_kernel": (C.c_int, [vp, vp, i64, C.POINTER(i64)]),
    "ads_select": (C.c_int, [vp, vp, vp, C.POINTER(vp)]),
    "ads_select_async": (C.c_int, [vp, vp, vp, vp]),
    "ads_selection_autotune": (C.c_int, [vp, vp, vp, i32, C.POINTER(i32), C.POINTER(i32),
                                         C.POINTER(C.c_float)]),
    # allocation-free search: dia, lib, params*, stream, capacity, six device output
    # columns, device int64 count, device int32 flags (nullable)
    "ads_dia_device_bytes": (i64, [vp]),
    "ads_dia_keep_bf16_only": (C.c_int, [vp]),
    "ads_select_noalloc": (C.c_int, [vp, vp, C.POINTER(AdsSelectionParams), i64, i64,
                                     vp, vp, vp, vp, vp, vp, vp, vp]),
    "ads_candidates_create": (C.c_int, [vp, C.POINTER(vp)]),
    "ads_selection_stream": (i64, [vp]),
    "ads_selection_last_launches": (i64, [vp]),
    "ads_selection_set_stats": (C.c_int, [vp, C.c_int]),
    "ads_selection_last_stats": (C.c_int, [vp, vp, i64]),
    "ads_selection_stage_times": (C.c_int, [vp, vp, i64]),
    "ads_candidates_size": (i64, [vp]),
    "ads_candidates_copy_out": (C.c_int, [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "ads_candidates_destroy": (C.c_int, [vp]),
    "ads_scoring_params_default": (None, [C.POINTER(AdsScoringParams)]),
    "ads_score": (C.c_int, [C.POINTER(AdsScoringParams), vp, vp, vp, C.c_int, C.POINTER(vp)]),
    "ads_score_arrays": (C.c_int, [C.POINTER(AdsScoringParams), vp, vp, i64, vp, vp, vp, vp, vp, vp,
                                   C.c_int, C.c_int, C.POINTER(vp)]),
    "ads_features_size": (i64, [vp]),
    "ads_features_kernel_ms": (C.c_float, [vp]),
    "ads_features_copy_out": (C.c_int, [vp, vp, vp, vp]),
    "ads_features_destroy": (C.c_int, [vp]),
    "ads_feature_names": (C.c_int, [C.POINTER(C.c_char_p), C.c_int]),
    "ads_quant_params_default": (None, [C.POINTER(AdsQuantParams)]),
    "ads_quantify": (C.c_int, [C.POINTER(AdsQuantParams), vp, vp, vp, C.c_int, C.POINTER(vp)]),
    "ads_quantify_arrays": (C.c_int, [C.POINTER(AdsQuantParams), vp, vp, i64, vp, vp, vp, vp, vp,
                                      C.c_int, C.c_int, C.POINTER(vp)]),
    "ads_quant_sizes": (C.c_int, [vp, C.POINTER(i64), C.POINTER(i64)]),
    "ads_quant_kernel_ms": (C.c_float, [vp]),
    "ads_quant_copy_out": (C.c_int, [vp] + [vp] * 13),
    "ads_quant_destroy": (C.c_int, [vp]),
    "ads_idf_bins": (i64, []),
    "ads_lib_idf_counts": (C.c_int, [vp, vp, C.c_int]),
    "ads_lib_set_idf": (C.c_int, [vp, vp, C.c_double, C.c_int]),
}

_lib = None
_finalizing = False


def _mark_finalizing():
    global _finalizing
    _finalizing = True


atexit.register(_mark_finalizing)


def alive() -> bool:
    """False once the interpreter is shutting down: handles are then left to the
    process exit instead of being destroyed through a runtime that may already be
    torn down."""
    return _lib is not None and not _finalizing


class AdsError(RuntimeError):
    pass


def library_path() -> str:
    return _build.lib_path()


def load(build_if_missing: bool = True):
    """Load libads_gpu.so (building it from csrc/ when it is absent and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        if not build_if_missing:
            raise ImportError(f"{path} is missing; build it with `python -m alphadia_search_rs_b200.build`")
        _build.build()
    L = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc: int) -> None:
    if rc == ADS_OK:
        return
    msg = (load().ads_last_error() or b"").decode(errors="replace")
    if rc == ADS_ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    if rc == ADS_ERR_OUT_OF_MEMORY:
        raise MemoryError(msg)
    raise AdsError(f"ads error {rc}: {msg}")
