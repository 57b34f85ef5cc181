"""CPU oracle for the peak-group-selection path -- TEST INFRASTRUCTURE ONLY.

ctypes bindings over ``oracle/_build/liboracle.so`` (built from ``oracle.cpp`` by
``oracle/Makefile``), a C++17 restatement of the reference crate's scalar CPU path.
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` import
this package, as the checker or as the timed CPU baseline.  The product
(``alphadia_search_rs_b200``) never imports it.

Parity pin: the reference crate's own known-answer tests for this path are ported
in ``tests/test_oracle_known_answers.py`` and run against this library.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

LOG_GLIBC = 0  # glibc logf, what the reference's f32::ln calls on Linux
LOG_RN = 1  # correctly rounded logf: (float)log((double)x)

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_i64 = C.c_int64
_f32 = C.c_float


class OrcParams(C.Structure):
    _fields_ = [
        ("fwhm_rt", C.c_float),
        ("kernel_size", C.c_int64),
        ("peak_length", C.c_int64),
        ("mass_tolerance", C.c_float),
        ("rt_tolerance", C.c_float),
        ("candidate_count", C.c_int64),
        ("top_k_fragments", C.c_int64),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    vp = C.c_void_p
    sig = {
        "orc_ppm_index_len": (_i64, [_f32, _f32, _f32]),
        "orc_ppm_index": (None, [_f32, _f32, _f32, _f32p]),
        "orc_find_closest_index": (_i64, [_f32p, _i64, _f32]),
        "orc_mz_range_indices": (None, [_f32p, _i64, _f32, _f32, C.POINTER(_i64), C.POINTER(_i64)]),
        "orc_mean_delta_t": (_f32, [_f32p, _i64]),
        "orc_rt_limits": (None, [_f32p, _i64, _f32, _f32, _f32, _i64, C.POINTER(_i64), C.POINTER(_i64)]),
        "orc_rust_binary_search_u16": (_i64, [_u16p, _i64, C.c_uint16]),
        "orc_gaussian_kernel": (_i64, [_f32, _f32, _i64, _f32, _f32p]),
        "orc_convolution": (None, [_f32p, _i64, _f32p, _i64, _i64, _f32p]),
        "orc_log_dot": (None, [_f32p, _i64, _i64, _f32p, _f32p, C.c_int]),
        "orc_local_maxima": (_i64, [_f32p, _i64, _i64, _i64p, _f32p]),
        "orc_filter_sort_fragments": (_i64, [_i64, _f32p, _f32p, _u8p, _u8p, C.c_int, C.c_int, _i64, _i64p]),
        "orc_dia_build": (vp, [_i64, _i64p, _f32p, _f32p, _i64p, _i64p, _i64p, _f32p, _i64, _f32p, _f32p, C.c_int]),
        "orc_dia_free": (None, [vp]),
        "orc_dia_num_obs": (_i64, [vp]),
        "orc_dia_grid_len": (_i64, [vp]),
        "orc_dia_grid": (C.POINTER(C.c_float), [vp]),
        "orc_dia_rt_len": (_i64, [vp]),
        "orc_dia_rt": (C.POINTER(C.c_float), [vp]),
        "orc_dia_delta_t": (_f32, [vp]),
        "orc_dia_obs_window": (None, [vp, _i64, C.POINTER(_f32), C.POINTER(_f32)]),
        "orc_dia_obs_num_cycles": (_i64, [vp, _i64]),
        "orc_dia_obs_num_peaks": (_i64, [vp, _i64]),
        "orc_dia_obs_slice_starts": (C.POINTER(C.c_uint32), [vp, _i64]),
        "orc_dia_obs_cycles": (C.POINTER(C.c_uint16), [vp, _i64]),
        "orc_dia_obs_intensities": (C.POINTER(C.c_float), [vp, _i64]),
        "orc_dia_valid_observations": (_i64, [vp, _f32, _i64p, _i64]),
        "orc_fill_xic_slice_raw": (None, [np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS"), _i64, _u16p,
                                           _f32p, _f32p, _i64, _f32p, _i64, _i64, _f32, _f32]),
        "orc_dense_xic": (None, [vp, _f32, _i64, _i64, _f32, _f32p, _i64, _f32p]),
        "orc_lib_build": (vp, [_i64, _u64p, _f32p, _f32p, _u64p, _u64p, _i64, _f32p, _f32p, _u8p, _u8p]),
        "orc_lib_free": (None, [vp]),
        "orc_lib_num_precursors": (_i64, [vp]),
        "orc_search": (vp, [vp, vp, C.POINTER(OrcParams), vp, vp, _i64, C.c_int, C.c_int, C.c_int]),
        "orc_result_len": (_i64, [vp]),
        "orc_result_copy": (None, [vp, _u64p, _u64p, _f32p, _f64p, _u64p, _u64p, _u64p]),
        "orc_result_free": (None, [vp]),
        "orc_trace_precursor": (_i64, [vp, vp, C.POINTER(OrcParams), _f32, _i64, C.c_int,
                                        C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64),
                                        _f32p, _f32p, _f32p, _i64]),
        "orc_scores_f64_at": (C.c_double, [vp, vp, C.POINTER(OrcParams), _f32, _i64, _i64p, _i64, _f64p]),
        # PeakGroupScoring
        "orc_lib_set_scoring": (None, [vp, _u8p, _i64, _f32p]),
        "orc_score": (vp, [vp, vp, _f32, _i64, _u64p, _u64p, _f32p, _u64p, _u64p, _u64p, _i64,
                           C.c_int, C.c_int]),
        "orc_features_len": (_i64, [vp]),
        "orc_features_copy": (None, [vp, _u64p, _u64p, _f32p]),
        "orc_features_free": (None, [vp]),
        "orc_quantify": (vp, [vp, vp, _f32, _i64, _u64p, _u64p, _u64p, _u64p, _u64p, _i64, C.c_int]),
        "orc_quant_sizes": (None, [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "orc_quant_copy": (None, [vp, _u64p, _u64p, _u64p, _f32p, _u64p, _u64p, _u64p, _f32p, _f32p,
                                  _f32p, _f32p, _u64p, _u64p]),
        "orc_quant_free": (None, [vp]),
        "orc_sc_normalize_profiles": (None, [_f32p, _i64, _i64, _i64, _f32p]),
        "orc_sc_median_axis0": (None, [_f32p, _i64, _i64, C.c_int, _f32p]),
        "orc_sc_correlation": (_f32, [_f32p, _f32p, _i64]),
        "orc_sc_gamma_ln": (_f32, [_f32, C.c_int]),
        "orc_sc_hyperscore": (_f32, [_u8p, _f32p, _u8p, vp, _i64, C.c_int]),
        "orc_sc_longest_ion_series": (None, [_u8p, _u8p, _u8p, _i64, C.POINTER(C.c_uint8),
                                              C.POINTER(C.c_uint8)]),
        "orc_sc_intensity_ion_series": (_f32, [_u8p, _f32p, _u8p, _i64, C.c_uint8]),
        "orc_sc_fwhm_rt": (_f32, [_f32p, _i64, _i64, _f32p]),
        "orc_sc_fragment_mz_errors": (None, [_f32p, _f32p, _i64, _i64, _f32p, _f32p, _f32p]),
        "orc_sc_weighted_mae": (_f32, [_f32p, _f32p, _i64]),
        "orc_sc_median": (_f32, [_f32p, _i64]),
        "orc_sc_std": (_f32, [_f32p, _i64]),
        "orc_sc_ranked_mask": (None, [_f32p, _i64, _i64, _i64, _u8p]),
        "orc_sc_count_above": (_i64, [_f32p, _i64, _f32, vp]),
        "orc_sc_dot": (_f32, [_f32p, _f32p, _i64]),
        "orc_sc_dense_xic_mz": (None, [vp, _f32, _i64, _i64, _f32, _f32p, _i64, _f32p, _f32p]),
        "orc_sc_idf": (None, [vp, vp, _f32p, _i64, C.c_int, _f32p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _f32a(x):
    return np.ascontiguousarray(x, dtype=np.float32)


# ------------------------------------------------------------------ primitives

def ppm_index(resolution_ppm=1.0, mz_start=150.0, mz_end=2000.0) -> np.ndarray:
    L = lib()
    n = L.orc_ppm_index_len(resolution_ppm, mz_start, mz_end)
    out = np.empty(n, np.float32)
    L.orc_ppm_index(resolution_ppm, mz_start, mz_end, out)
    return out


def find_closest_index(grid, mz) -> int:
    g = _f32a(grid)
    return int(lib().orc_find_closest_index(g, len(g), float(mz)))


def mz_range_indices(grid, lower_mz, upper_mz) -> range:
    g = _f32a(grid)
    s, e = _i64(), _i64()
    lib().orc_mz_range_indices(g, len(g), float(lower_mz), float(upper_mz), C.byref(s), C.byref(e))
    return range(s.value, e.value)


def mean_delta_t(rt) -> float:
    r = _f32a(rt)
    return float(lib().orc_mean_delta_t(r, len(r)))


def rt_limits(rt, delta_t, precursor_rt, rt_tolerance, padding):
    r = _f32a(rt)
    lo, hi = _i64(), _i64()
    lib().orc_rt_limits(r, len(r), float(delta_t), float(precursor_rt), float(rt_tolerance),
                        int(padding), C.byref(lo), C.byref(hi))
    return lo.value, hi.value


def rust_binary_search_u16(a, x) -> int:
    arr = np.ascontiguousarray(a, dtype=np.uint16)
    return int(lib().orc_rust_binary_search_u16(arr, len(arr), int(x)))


def gaussian_kernel(fwhm_rt, sigma_scale_rt, kernel_width, rt_resolution) -> np.ndarray:
    out = np.zeros(int(kernel_width) + 2, np.float32)
    n = lib().orc_gaussian_kernel(float(fwhm_rt), float(sigma_scale_rt), int(kernel_width),
                                  float(rt_resolution), out)
    return out[:n].copy()


def convolution(kernel, xic) -> np.ndarray:
    k = _f32a(kernel)
    x = _f32a(np.atleast_2d(xic)) if np.ndim(xic) else _f32a(xic)
    F, Cn = x.shape
    out = np.zeros((F, Cn), np.float32)
    lib().orc_convolution(k, len(k), x.reshape(-1), F, Cn, out.reshape(-1))
    return out


def log_dot(array, weights, log_mode=LOG_GLIBC) -> np.ndarray:
    a = _f32a(array)
    F, Cn = a.shape
    w = _f32a(weights)
    assert len(w) == F, "Number of rows in array must match the length of weights vector"
    out = np.zeros(Cn, np.float32)
    lib().orc_log_dot(a.reshape(-1), F, Cn, w, out, int(log_mode))
    return out


def local_maxima(array, offset=0):
    a = _f32a(array)
    idx = np.zeros(max(len(a), 1), np.int64)
    val = np.zeros(max(len(a), 1), np.float32)
    n = lib().orc_local_maxima(a, len(a), int(offset), idx, val)
    return idx[:n].copy(), val[:n].copy()


def filter_sort_fragments(mz, intensity, number, ftype, non_zero, filter_y1, top_k) -> np.ndarray:
    n = len(mz)
    out = np.zeros(max(n, 1), np.int64)
    k = lib().orc_filter_sort_fragments(
        n, _f32a(mz), _f32a(intensity), np.ascontiguousarray(number, np.uint8),
        np.ascontiguousarray(ftype, np.uint8), int(non_zero), int(filter_y1),
        int(min(top_k, 2**62)), out)
    return out[:k].copy()


def fill_xic_slice_raw(slice_starts, cycles, intensities, grid, xic, cycle_start, cycle_stop,
                       mass_tolerance, mz):
    """Adds into ``xic`` (float32, length cycle_stop - cycle_start) in place."""
    ss = np.ascontiguousarray(slice_starts, np.uint32)
    cy = np.ascontiguousarray(cycles, np.uint16)
    it = _f32a(intensities)
    g = _f32a(grid)
    assert xic.dtype == np.float32 and xic.flags.c_contiguous
    lib().orc_fill_xic_slice_raw(ss, len(ss) - 1, cy if len(cy) else np.zeros(1, np.uint16),
                                 it if len(it) else np.zeros(1, np.float32), g, len(g), xic,
                                 int(cycle_start), int(cycle_stop), float(mass_tolerance), float(mz))
    return xic


# ------------------------------------------------------------------ DIA + lib

class Dia:
    """Oracle DIAData (src/dia_data_builder/mod.rs:11-139)."""

    def __init__(self, spectrum_delta_scan_idx, isolation_lower_mz, isolation_upper_mz,
                 spectrum_peak_start_idx, spectrum_peak_stop_idx, spectrum_cycle_idx,
                 spectrum_rt, peak_mz, peak_intensity, n_threads=0):
        L = lib()
        n_threads = n_threads or os.cpu_count() or 1
        ds = np.ascontiguousarray(spectrum_delta_scan_idx, np.int64)
        self._keep = [ds,
                      _f32a(isolation_lower_mz), _f32a(isolation_upper_mz),
                      np.ascontiguousarray(spectrum_peak_start_idx, np.int64),
                      np.ascontiguousarray(spectrum_peak_stop_idx, np.int64),
                      np.ascontiguousarray(spectrum_cycle_idx, np.int64),
                      _f32a(spectrum_rt), _f32a(peak_mz), _f32a(peak_intensity)]
        k = self._keep
        self._h = L.orc_dia_build(len(ds), k[0], k[1], k[2], k[3], k[4], k[5], k[6],
                                  len(k[7]), k[7], k[8], int(n_threads))
        self._keep = None

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                lib().orc_dia_free(self._h)
            except TypeError:  # interpreter shutdown: module globals already cleared
                pass
            self._h = None

    @property
    def num_observations(self) -> int:
        return int(lib().orc_dia_num_obs(self._h))

    @property
    def rt(self) -> np.ndarray:
        L = lib()
        n = L.orc_dia_rt_len(self._h)
        return np.ctypeslib.as_array(L.orc_dia_rt(self._h), (n,)).copy() if n else np.zeros(0, np.float32)

    @property
    def delta_t(self) -> float:
        return float(lib().orc_dia_delta_t(self._h))

    def window(self, obs):
        lo, hi = _f32(), _f32()
        lib().orc_dia_obs_window(self._h, obs, C.byref(lo), C.byref(hi))
        return lo.value, hi.value

    def num_cycles(self, obs) -> int:
        return int(lib().orc_dia_obs_num_cycles(self._h, obs))

    def slice_starts(self, obs) -> np.ndarray:
        L = lib()
        g = L.orc_dia_grid_len(self._h)
        return np.ctypeslib.as_array(L.orc_dia_obs_slice_starts(self._h, obs), (g + 1,)).copy()

    def cycles(self, obs) -> np.ndarray:
        L = lib()
        n = L.orc_dia_obs_num_peaks(self._h, obs)
        if n == 0:
            return np.zeros(0, np.uint16)
        return np.ctypeslib.as_array(L.orc_dia_obs_cycles(self._h, obs), (n,)).copy()

    def intensities(self, obs) -> np.ndarray:
        L = lib()
        n = L.orc_dia_obs_num_peaks(self._h, obs)
        if n == 0:
            return np.zeros(0, np.float32)
        return np.ctypeslib.as_array(L.orc_dia_obs_intensities(self._h, obs), (n,)).copy()

    def slice_data(self, obs, mz_idx):
        ss = self.slice_starts(obs)
        s, e = int(ss[mz_idx]), int(ss[mz_idx + 1])
        return self.cycles(obs)[s:e], self.intensities(obs)[s:e]

    def valid_observations(self, precursor_mz):
        out = np.zeros(max(self.num_observations, 1), np.int64)
        n = lib().orc_dia_valid_observations(self._h, float(precursor_mz), out, len(out))
        return [int(v) for v in out[:n]]

    def dense_xic(self, precursor_mz, cycle_start, cycle_stop, mass_tolerance, fragment_mz):
        f = _f32a(fragment_mz)
        out = np.zeros((len(f), cycle_stop - cycle_start), np.float32)
        lib().orc_dense_xic(self._h, float(precursor_mz), int(cycle_start), int(cycle_stop),
                            float(mass_tolerance), f if len(f) else np.zeros(1, np.float32), len(f),
                            out.reshape(-1) if out.size else np.zeros(1, np.float32))
        return out


class Lib:
    """Oracle SpecLibFlat (src/speclib_flat/mod.rs:100-188)."""

    def __init__(self, precursor_idx, precursor_mz, precursor_rt, flat_frag_start_idx,
                 flat_frag_stop_idx, fragment_mz, fragment_intensity, fragment_number,
                 fragment_type):
        L = lib()
        a = [np.ascontiguousarray(precursor_idx, np.uint64), _f32a(precursor_mz), _f32a(precursor_rt),
             np.ascontiguousarray(flat_frag_start_idx, np.uint64),
             np.ascontiguousarray(flat_frag_stop_idx, np.uint64),
             _f32a(fragment_mz), _f32a(fragment_intensity),
             np.ascontiguousarray(fragment_number, np.uint8), np.ascontiguousarray(fragment_type, np.uint8)]
        nf = len(a[5])
        if nf == 0:
            a[5], a[6] = np.zeros(1, np.float32), np.zeros(1, np.float32)
            a[7], a[8] = np.zeros(1, np.uint8), np.zeros(1, np.uint8)
        self._h = L.orc_lib_build(len(a[0]), a[0], a[1], a[2], a[3], a[4], nf, a[5], a[6], a[7], a[8])
        self.num_precursors = len(a[0])
        self.sorted_order = np.argsort(a[0], kind="stable")

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                lib().orc_lib_free(self._h)
            except TypeError:  # interpreter shutdown: module globals already cleared
                pass
            self._h = None


@dataclass
class Params:
    fwhm_rt: float = 3.0
    kernel_size: int = 20
    peak_length: int = 5
    mass_tolerance: float = 7.0
    rt_tolerance: float = 200.0
    candidate_count: int = 3
    top_k_fragments: int = 12

    def c(self) -> OrcParams:
        return OrcParams(self.fwhm_rt, self.kernel_size, self.peak_length, self.mass_tolerance,
                         self.rt_tolerance, self.candidate_count, self.top_k_fragments)


def search(dia: Dia, lb: Lib, params: Params, rt_tolerance_per_precursor=None, subset=None,
           log_mode=LOG_GLIBC, precision=0, n_threads=0) -> dict:
    """src/peak_group_selection/mod.rs:94-128.  ``rt_tolerance_per_precursor`` and
    ``subset`` are indexed in sorted-library order.  Returns the candidate arrays."""
    L = lib()
    n_threads = n_threads or os.cpu_count() or 1
    p = params.c()
    tol = None if rt_tolerance_per_precursor is None else _f32a(rt_tolerance_per_precursor)
    sub = None if subset is None else np.ascontiguousarray(subset, np.int64)
    h = L.orc_search(dia._h, lb._h, C.byref(p),
                     tol.ctypes.data if tol is not None else None,
                     sub.ctypes.data if sub is not None else None,
                     0 if sub is None else len(sub), int(log_mode), int(precision), int(n_threads))
    try:
        n = L.orc_result_len(h)
        m = max(n, 1)
        out = {k: np.zeros(m, np.uint64) for k in ("precursor_idx", "rank", "cycle_center", "cycle_start", "cycle_stop")}
        out["score"] = np.zeros(m, np.float32)
        out["score_f64"] = np.zeros(m, np.float64)
        L.orc_result_copy(h, out["precursor_idx"], out["rank"], out["score"], out["score_f64"],
                          out["cycle_center"], out["cycle_start"], out["cycle_stop"])
        return {k: v[:n] for k, v in out.items()}
    finally:
        L.orc_result_free(h)


def trace_precursor(dia: Dia, lb: Lib, params: Params, lib_pos, rt_tolerance=None, log_mode=LOG_GLIBC,
                    cap=1 << 22):
    L = lib()
    p = params.c()
    xic = np.zeros(cap, np.float32)
    conv = np.zeros(cap, np.float32)
    score = np.zeros(cap, np.float32)
    cs, ce, nf = _i64(), _i64(), _i64()
    tol = params.rt_tolerance if rt_tolerance is None else rt_tolerance
    c = L.orc_trace_precursor(dia._h, lb._h, C.byref(p), float(tol), int(lib_pos), int(log_mode),
                              C.byref(cs), C.byref(ce), C.byref(nf), xic, conv, score, cap)
    F = nf.value
    Cn = max(int(c), 0)
    return dict(cycle_start=cs.value, cycle_stop=ce.value, n_frag=F,
                xic=xic[:F * Cn].reshape(F, Cn), conv=conv[:F * Cn].reshape(F, Cn), score=score[:Cn])


def scores_f64_at(dia: Dia, lb: Lib, params: Params, lib_pos, cycles, rt_tolerance=None):
    p = params.c()
    cyc = np.ascontiguousarray(cycles, np.int64)
    out = np.zeros(max(len(cyc), 1), np.float64)
    tol = params.rt_tolerance if rt_tolerance is None else rt_tolerance
    mx = lib().orc_scores_f64_at(dia._h, lb._h, C.byref(p), float(tol), int(lib_pos),
                                 cyc if len(cyc) else np.zeros(1, np.int64), len(cyc), out)
    return out[:len(cyc)], float(mx)


# ------------------------------------------------------------ PeakGroupScoring

# src/candidate/features.rs:6-48
FEATURE_NAMES = (
    "score", "mean_correlation", "median_correlation", "correlation_std", "intensity_correlation",
    "num_fragments", "num_scans", "num_over_95", "num_over_90", "num_over_80", "num_over_50",
    "num_over_0", "num_over_0_rank_0_5", "num_over_0_rank_6_11", "num_over_0_rank_12_17",
    "num_over_0_rank_18_23", "num_over_50_rank_0_5", "num_over_50_rank_6_11",
    "num_over_50_rank_12_17", "num_over_50_rank_18_23", "hyperscore_intensity_observation",
    "hyperscore_intensity_library", "hyperscore_inverse_mass_error", "rt_observed", "delta_rt",
    "longest_b_series", "longest_y_series", "naa", "weighted_mass_error", "log10_b_ion_intensity",
    "log10_y_ion_intensity", "fwhm_rt", "idf_hyperscore", "idf_xic_dot_product",
    "idf_intensity_dot_product", "median_profile_sum", "median_profile_sum_filtered",
    "num_profiles", "num_profiles_filtered", "num_over_0_top6_idf", "num_over_50_top6_idf",
)


def lib_set_scoring(lb: "Lib", precursor_naa, fragment_mz_library) -> None:
    """Adds SpecLibFlat's precursor_naa (input order) and fragment_mz_library."""
    naa = np.ascontiguousarray(precursor_naa, np.uint8)
    fml = _f32a(fragment_mz_library)
    if len(fml) == 0:
        fml = np.zeros(1, np.float32)
        n = 0
    else:
        n = len(fml)
    if len(naa) == 0:
        naa = np.zeros(1, np.uint8)
    lib().orc_lib_set_scoring(lb._h, naa, n, fml)


def score(dia: "Dia", lb: "Lib", candidates: dict, mass_tolerance: float = 7.0,
          top_k_fragments: int = 100, log_mode: int = LOG_GLIBC, n_threads: int = 0) -> dict:
    """PeakGroupScoring.score (src/peak_group_scoring/mod.rs:42-101): a dict of
    precursor_idx, rank and the 41 feature columns (src/candidate/features.rs:220-411)."""
    L = lib()
    n = len(candidates["precursor_idx"])
    cols = [np.ascontiguousarray(candidates[k], np.uint64) for k in ("precursor_idx", "rank")]
    sc = _f32a(candidates["score"])
    cyc = [np.ascontiguousarray(candidates[k], np.uint64) for k in ("cycle_center", "cycle_start", "cycle_stop")]
    if n == 0:
        cols = [np.zeros(1, np.uint64)] * 2
        sc = np.zeros(1, np.float32)
        cyc = [np.zeros(1, np.uint64)] * 3
    h = L.orc_score(dia._h, lb._h, float(mass_tolerance), int(top_k_fragments), cols[0], cols[1], sc,
                    cyc[0], cyc[1], cyc[2], n, int(log_mode), int(n_threads or os.cpu_count() or 1))
    try:
        m = L.orc_features_len(h)
        pidx = np.zeros(max(m, 1), np.uint64)
        rank = np.zeros(max(m, 1), np.uint64)
        feats = np.zeros((max(m, 1), len(FEATURE_NAMES)), np.float32)
        L.orc_features_copy(h, pidx, rank, feats)
    finally:
        L.orc_features_free(h)
    out = {"precursor_idx": pidx[:m], "rank": rank[:m]}
    for k, name in enumerate(FEATURE_NAMES):
        out[name] = np.ascontiguousarray(feats[:m, k])
    return out


QUANT_PRECURSOR_KEYS = ("precursor_idx", "mz_library", "mz", "rt_library", "rt", "naa", "rank",
                        "rt_observed", "flat_frag_start_idx", "flat_frag_stop_idx")
QUANT_FRAGMENT_KEYS = ("mz_library", "mz", "intensity", "cardinality", "charge", "loss_type", "number",
                       "position", "type", "mz_observed", "correlation_observed", "mass_error_observed",
                       "precursor_idx", "rank")


def quantify(dia: "Dia", lb: "Lib", candidates: dict, library: dict, tolerance_ppm: float = 7.0,
             top_k_fragments: int = 10000, n_threads: int = 0):
    """PeakGroupQuantification.quantify (src/peak_group_quantification/mod.rs:49-168) as
    SpecLibFlatQuantified.to_dict_arrays (src/speclib_flat_quantified/mod.rs:126-210):
    (precursor dict, fragment dict).  ``library`` holds the SpecLibFlat.from_arrays
    inputs, from which the pass-through columns are taken."""
    L = lib()
    n = len(candidates["precursor_idx"])
    cols = [np.ascontiguousarray(candidates[k], np.uint64) for k in
            ("precursor_idx", "rank", "cycle_center", "cycle_start", "cycle_stop")]
    if n == 0:
        cols = [np.zeros(1, np.uint64)] * 5
    h = L.orc_quantify(dia._h, lb._h, float(tolerance_ppm), int(min(top_k_fragments, 2**63 - 1)),
                       *cols, n, int(n_threads or os.cpu_count() or 1))
    try:
        np_, nf_ = C.c_int64(), C.c_int64()
        L.orc_quant_sizes(h, C.byref(np_), C.byref(nf_))
        P, NF = np_.value, nf_.value
        pu = [np.zeros(max(P, 1), np.uint64) for _ in range(5)]
        prt = np.zeros(max(P, 1), np.float32)
        fu = [np.zeros(max(NF, 1), np.uint64) for _ in range(3)]
        ff = [np.zeros(max(NF, 1), np.float32) for _ in range(4)]
        L.orc_quant_copy(h, pu[0], pu[1], pu[2], prt, pu[3], pu[4], fu[0], ff[0], ff[1], ff[2], ff[3],
                         fu[1], fu[2])
    finally:
        L.orc_quant_free(h)
    prow, frow = pu[1][:P].astype(np.int64), fu[0][:NF].astype(np.int64)
    g = lambda k, rows: np.asarray(library[k])[rows]
    prec = {"precursor_idx": pu[0][:P], "mz_library": g("precursor_mz_library", prow),
            "mz": g("precursor_mz", prow), "rt_library": g("precursor_rt_library", prow),
            "rt": g("precursor_rt", prow), "naa": g("precursor_naa", prow), "rank": pu[2][:P],
            "rt_observed": prt[:P], "flat_frag_start_idx": pu[3][:P], "flat_frag_stop_idx": pu[4][:P]}
    frag = {"mz_library": g("fragment_mz_library", frow), "mz": g("fragment_mz", frow),
            "intensity": ff[0][:NF], "cardinality": g("fragment_cardinality", frow),
            "charge": g("fragment_charge", frow), "loss_type": g("fragment_loss_type", frow),
            "number": g("fragment_number", frow), "position": g("fragment_position", frow),
            "type": g("fragment_type", frow), "mz_observed": ff[1][:NF],
            "correlation_observed": ff[2][:NF], "mass_error_observed": ff[3][:NF],
            "precursor_idx": fu[1][:NF], "rank": fu[2][:NF]}
    return prec, frag


def sc_normalize_profiles(x, dilations: int = 1) -> np.ndarray:
    x = _f32a(np.atleast_2d(x))
    out = np.zeros_like(x)
    lib().orc_sc_normalize_profiles(x, x.shape[0], x.shape[1], dilations, out)
    return out


def sc_median_axis0(x, non_zero_only: bool = False) -> np.ndarray:
    x = _f32a(x).reshape(-1, np.shape(x)[-1]) if np.size(x) else np.zeros((0, np.shape(x)[-1]), np.float32)
    out = np.zeros(max(x.shape[1], 1), np.float32)
    lib().orc_sc_median_axis0(x if x.size else np.zeros(1, np.float32), x.shape[0], x.shape[1],
                              int(non_zero_only), out)
    return out[:x.shape[1]]


def _nz(a, dtype):
    a = np.ascontiguousarray(a, dtype)
    return a if a.size else np.zeros(1, dtype)


def sc_correlation(x, y) -> float:
    x, y = _f32a(x), _f32a(y)
    if len(x) != len(y):
        return 0.0
    return float(lib().orc_sc_correlation(_nz(x, np.float32), _nz(y, np.float32), len(x)))


def sc_gamma_ln(x: float, log_mode: int = LOG_GLIBC) -> float:
    return float(lib().orc_sc_gamma_ln(float(x), int(log_mode)))


def sc_hyperscore(types, intensities, mask, weights=None, log_mode: int = LOG_GLIBC) -> float:
    n = len(types)
    if len(intensities) != n or len(mask) != n or (weights is not None and len(weights) != n):
        return 0.0  # src/peak_group_scoring/utils.rs:199-209
    w = None if weights is None else _nz(weights, np.float32)
    return float(lib().orc_sc_hyperscore(_nz(types, np.uint8), _nz(intensities, np.float32),
                                         _nz(mask, np.uint8), w.ctypes.data if w is not None else None,
                                         n, int(log_mode)))


def sc_longest_ion_series(types, numbers, mask):
    n = len(types)
    if len(mask) != n or len(numbers) != n:
        return (0, 0)  # src/peak_group_scoring/utils.rs:319-322
    b, y = C.c_uint8(), C.c_uint8()
    lib().orc_sc_longest_ion_series(_nz(types, np.uint8), _nz(numbers, np.uint8), _nz(mask, np.uint8), n,
                                    C.byref(b), C.byref(y))
    return (b.value, y.value)


def sc_intensity_ion_series(types, intensities, mask, target: int) -> float:
    n = len(types)
    if len(intensities) != n or len(mask) != n:
        return 0.0
    return float(lib().orc_sc_intensity_ion_series(_nz(types, np.uint8), _nz(intensities, np.float32),
                                                   _nz(mask, np.uint8), n, int(target)))


def sc_fwhm_rt(profile, cycle_start: int, rt) -> float:
    return float(lib().orc_sc_fwhm_rt(_nz(profile, np.float32), len(profile), int(cycle_start), _nz(rt, np.float32)))


def sc_fragment_mz_errors(dense_mz, dense_xic, mz_library):
    dm, dx = _f32a(np.atleast_2d(dense_mz)), _f32a(np.atleast_2d(dense_xic))
    F, Cn = dm.shape
    mo, err = np.zeros(max(F, 1), np.float32), np.zeros(max(F, 1), np.float32)
    lib().orc_sc_fragment_mz_errors(_nz(dm, np.float32), _nz(dx, np.float32), F, Cn,
                                    _nz(mz_library, np.float32), mo, err)
    return mo[:F], err[:F]


def sc_weighted_mae(errors, weights) -> float:
    if len(errors) != len(weights):
        return 0.0
    return float(lib().orc_sc_weighted_mae(_nz(errors, np.float32), _nz(weights, np.float32), len(errors)))


def sc_median(v) -> float:
    return float(lib().orc_sc_median(_nz(v, np.float32), len(v)))


def sc_std(v) -> float:
    return float(lib().orc_sc_std(_nz(v, np.float32), len(v)))


def sc_ranked_mask(v, r1: int, r2: int) -> np.ndarray:
    out = np.zeros(max(len(v), 1), np.uint8)
    lib().orc_sc_ranked_mask(_nz(v, np.float32), len(v), int(r1), int(r2), out)
    return out[:len(v)].astype(bool)


def sc_count_above(v, threshold: float, mask=None) -> int:
    if mask is not None and len(mask) != len(v):
        return 0
    m = None if mask is None else _nz(mask, np.uint8)
    return int(lib().orc_sc_count_above(_nz(v, np.float32), len(v), float(threshold),
                                        m.ctypes.data if m is not None else None))


def sc_dot(a, b) -> float:
    if len(a) != len(b):
        return 0.0
    return float(lib().orc_sc_dot(_nz(a, np.float32), _nz(b, np.float32), len(a)))


def sc_dense_xic_mz(dia: "Dia", precursor_mz: float, cycle_start: int, cycle_stop: int,
                    mass_tolerance: float, fragment_mz):
    fmz = _f32a(fragment_mz)
    F, Cn = len(fmz), cycle_stop - cycle_start
    xic = np.zeros(max(F * Cn, 1), np.float32)
    mz = np.zeros(max(F * Cn, 1), np.float32)
    lib().orc_sc_dense_xic_mz(dia._h, float(precursor_mz), int(cycle_start), int(cycle_stop),
                              float(mass_tolerance), _nz(fmz, np.float32), F, xic, mz)
    return xic[:F * Cn].reshape(F, Cn), mz[:F * Cn].reshape(F, Cn)


def sc_idf(dia: "Dia", lb: "Lib", mz, log_mode: int = LOG_GLIBC) -> np.ndarray:
    mz = _f32a(mz)
    out = np.zeros(max(len(mz), 1), np.float32)
    lib().orc_sc_idf(dia._h, lb._h, _nz(mz, np.float32), len(mz), int(log_mode), out)
    return out[:len(mz)]
