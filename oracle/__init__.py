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
