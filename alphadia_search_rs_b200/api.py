"""Python classes with the reference module's names and behaviour.

Mirrors the pyo3 classes of MannLabs/alphadia-search-rs (src/lib.rs:74-93) that
the selection path uses: ``DIAData``, ``SpecLibFlat``, ``SelectionParameters``,
``PeakGroupSelection`` and ``CandidateCollection``.  Every call goes through the
C ABI of ``include/ads_gpu.h``; the work runs on the GPU.  Extensions beyond the
reference API are keyword-only arguments with defaults that keep the reference
behaviour.
"""
from __future__ import annotations

import ctypes as C
from typing import Any

import numpy as np

from . import _ffi as F

_DEFAULT_DEVICE = 0


def _lib():
    return F.load()


def _release(obj, destroy: str) -> None:
    """Frees a native handle from __del__; silent during interpreter shutdown, when
    module globals may already be gone."""
    h = getattr(obj, "_h", None)
    obj._h = None
    if not h:
        return
    try:
        if F.alive():
            getattr(_lib(), destroy)(h)
    except Exception:
        pass


def _is_device_tensor(x: Any) -> bool:
    return hasattr(x, "is_cuda") and bool(getattr(x, "is_cuda"))


def _as_np(name: str, x: Any, dtype) -> np.ndarray:
    """numpy view of ``x`` with exactly ``dtype`` (pyo3's PyReadonlyArray1<T>
    rejects other dtypes with TypeError)."""
    if not isinstance(x, np.ndarray):
        raise TypeError(f"argument '{name}': expected numpy.ndarray of {np.dtype(dtype).name}, got {type(x).__name__}")
    if x.dtype != np.dtype(dtype):
        raise TypeError(f"argument '{name}': expected dtype {np.dtype(dtype).name}, got {x.dtype.name}")
    return np.ascontiguousarray(x)


_PINNED = None  # torch when page-locked host memory can be had, else False


def _host_empty(n: int, dtype) -> np.ndarray:
    """An uninitialised host array of n elements for device-to-host copies.  With torch
    and a CUDA device it is page-locked memory from torch's caching host allocator
    (freed blocks are reused, so steady-state calls do not pin new pages), which the
    copy engines fill at full link speed; otherwise a plain numpy array."""
    global _PINNED
    if _PINNED is None:
        try:
            import torch

            _PINNED = torch if torch.cuda.is_available() else False
        except Exception:  # no torch: pageable numpy memory
            _PINNED = False
    if _PINNED is False:
        return np.empty(n, dtype)
    t = _PINNED
    tdt = {np.dtype(np.uint64): t.uint64, np.dtype(np.float32): t.float32,
           np.dtype(np.uint8): t.uint8, np.dtype(np.int64): t.int64}[np.dtype(dtype)]
    return t.empty(n, dtype=tdt, pin_memory=True).numpy()


def _dev_ptr(name: str, t: Any, dtype, device: int) -> int:
    import torch

    want = {np.float32: torch.float32, np.int64: torch.int64, np.uint8: torch.uint8,
            np.uint64: torch.uint64}[dtype]
    if t.dtype != want:
        raise TypeError(f"argument '{name}': expected dtype {want}, got {t.dtype}")
    if t.device.index != device:
        raise ValueError(f"argument '{name}': tensor on cuda:{t.device.index}, expected cuda:{device}")
    if not t.is_contiguous():
        raise ValueError(f"argument '{name}': tensor must be contiguous")
    return int(t.data_ptr())


class DIAData:
    """DIAData (src/dia_data/mod.rs:15-136), device resident."""

    def __init__(self):
        self._h = None
        self._n_obs = 0
        self._iso = np.zeros((0, 2), np.float32)
        self._num_peaks = np.zeros(0, np.int64)
        self._rt_values = np.zeros(0, np.float32)
        self._cycle = np.zeros((0, 0, 0, 0), np.float32)
        self.device = _DEFAULT_DEVICE

    def __del__(self):
        _release(self, "ads_dia_destroy")

    @staticmethod
    def from_arrays(spectrum_delta_scan_idx, isolation_lower_mz, isolation_upper_mz,
                    spectrum_peak_start_idx, spectrum_peak_stop_idx, spectrum_cycle_idx,
                    spectrum_rt, peak_mz, peak_intensity, cycle, *, device: int | None = None,
                    intensity_storage: str = "f32"):
        """DIAData::from_arrays (src/dia_data/mod.rs:41-72).  The first nine arrays
        may instead all be CUDA tensors on ``device`` (same dtypes).

        ``intensity_storage="bf16"`` (an addition) keeps the intensities as bfloat16
        only, for runs searched with ``precision="bf16"``: 4 instead of 6 device bytes
        per peak; FP32 searches, scoring and quantification of such a run raise
        ValueError."""
        if intensity_storage not in ("f32", "bf16"):
            raise ValueError("intensity_storage must be 'f32' or 'bf16'")
        L = _lib()
        names = ["spectrum_delta_scan_idx", "isolation_lower_mz", "isolation_upper_mz",
                 "spectrum_peak_start_idx", "spectrum_peak_stop_idx", "spectrum_cycle_idx",
                 "spectrum_rt", "peak_mz", "peak_intensity"]
        dtypes = [np.int64, np.float32, np.float32, np.int64, np.int64, np.int64, np.float32,
                  np.float32, np.float32]
        arrays = [spectrum_delta_scan_idx, isolation_lower_mz, isolation_upper_mz,
                  spectrum_peak_start_idx, spectrum_peak_stop_idx, spectrum_cycle_idx,
                  spectrum_rt, peak_mz, peak_intensity]
        cyc = _as_np("cycle", cycle, np.float32)
        if cyc.ndim != 4:
            raise TypeError("argument 'cycle': expected a 4-D float32 array")
        on_dev = [_is_device_tensor(a) for a in arrays]
        if any(on_dev) and not all(on_dev):
            raise ValueError("spectrum and peak arrays must be all host arrays or all CUDA tensors")
        raw = F.AdsRawArrays()
        keep = []
        if all(on_dev):
            dev = arrays[0].device.index if device is None else device
            raw.location = F.ADS_MEM_DEVICE
            ptrs = [_dev_ptr(n, a, t, dev) for n, a, t in zip(names, arrays, dtypes)]
            lens = [int(a.numel()) for a in arrays]
        else:
            dev = _DEFAULT_DEVICE if device is None else device
            raw.location = F.ADS_MEM_HOST
            np_arrays = [_as_np(n, a, t) for n, a, t in zip(names, arrays, dtypes)]
            keep.extend(np_arrays)
            ptrs = [a.ctypes.data for a in np_arrays]
            lens = [a.size for a in np_arrays]
        n_spec = lens[0]
        if any(n != n_spec for n in lens[1:7]):
            raise ValueError("spectrum arrays must have the same length")
        if lens[7] != lens[8]:
            raise ValueError("peak_mz and peak_intensity must have the same length")
        raw.n_spectra = n_spec
        (raw.spectrum_delta_scan_idx, raw.isolation_lower_mz, raw.isolation_upper_mz,
         raw.spectrum_peak_start_idx, raw.spectrum_peak_stop_idx, raw.spectrum_cycle_idx,
         raw.spectrum_rt, raw.peak_mz, raw.peak_intensity) = ptrs
        raw.n_peaks = lens[7]
        raw.cycle = cyc.ctypes.data if cyc.size else None
        for i in range(4):
            raw.cycle_shape[i] = cyc.shape[i]
        h = C.c_void_p()
        F.check(L.ads_dia_create(C.byref(raw), int(dev), C.byref(h)))
        d = DIAData()
        d._h = h.value
        d.device = int(dev)
        if intensity_storage == "bf16":
            F.check(L.ads_dia_keep_bf16_only(d._h))
        d._load_meta()
        return d

    def _load_meta(self):
        L = _lib()
        self._n_obs = int(L.ads_dia_num_observations(self._h))
        iso = np.zeros((self._n_obs, 2), np.float32)
        npk = np.zeros(self._n_obs, np.int64)
        lo, hi, nc, n = C.c_float(), C.c_float(), C.c_int64(), C.c_int64()
        for w in range(self._n_obs):
            F.check(L.ads_dia_observation_info(self._h, w, C.byref(lo), C.byref(hi), C.byref(nc), C.byref(n)))
            iso[w] = (lo.value, hi.value)
            npk[w] = n.value
        self._iso, self._num_peaks = iso, npk
        cnt = C.c_int64()
        F.check(L.ads_dia_rt_values(self._h, None, 0, C.byref(cnt)))
        rtv = np.zeros(max(cnt.value, 1), np.float32)
        F.check(L.ads_dia_rt_values(self._h, rtv.ctypes.data, cnt.value, C.byref(cnt)))
        self._rt_values = rtv[:cnt.value].copy()
        shape = (C.c_int64 * 4)()
        F.check(L.ads_dia_cycle(self._h, None, 0, C.byref(shape)))
        cyc = np.zeros(tuple(shape), np.float32)
        if cyc.size:
            F.check(L.ads_dia_cycle(self._h, cyc.ctypes.data, cyc.size, C.byref(shape)))
        self._cycle = cyc

    # ---- getters (src/dia_data/mod.rs:74-135)
    @property
    def num_observations(self) -> int:
        return self._n_obs

    def get_valid_observations(self, precursor_mz: float) -> list[int]:
        """src/dia_data/mod.rs:79-87: windows with lower <= mz <= upper, in order."""
        mz = np.float32(precursor_mz)
        return [i for i in range(self._n_obs) if self._iso[i, 0] <= mz and self._iso[i, 1] >= mz]

    def memory_footprint_bytes(self) -> int:
        return int(_lib().ads_dia_memory_footprint_bytes(self._h)) if self._h else 24

    def memory_footprint_mb(self) -> float:
        return self.memory_footprint_bytes() / (1024.0 * 1024.0)

    def device_bytes(self) -> int:
        """Device memory the run holds (an addition; memory_footprint_bytes keeps the
        reference's own accounting)."""
        return int(_lib().ads_dia_device_bytes(self._h)) if self._h else 0

    @property
    def has_mobility(self) -> bool:
        return False

    @property
    def has_ms1(self) -> bool:
        return False

    @property
    def mobility_values(self) -> list[float]:
        return [1e-6, 0.0]

    @property
    def rt_values(self) -> np.ndarray:
        return self._rt_values.copy()

    @property
    def cycle(self) -> np.ndarray:
        return self._cycle.copy()

    # ---- engine extras
    def rt_index(self) -> tuple[np.ndarray, float]:
        L = _lib()
        n, dt = C.c_int64(), C.c_float()
        F.check(L.ads_dia_rt_index(self._h, None, 0, C.byref(n), C.byref(dt)))
        out = np.zeros(max(n.value, 1), np.float32)
        F.check(L.ads_dia_rt_index(self._h, out.ctypes.data, n.value, C.byref(n), C.byref(dt)))
        return out[:n.value].copy(), float(dt.value)

    def observation(self, obs: int) -> dict:
        """CSR of one quadrupole observation copied to host (slice_starts,
        cycle_indices, intensities)."""
        L = _lib()
        g = int(L.ads_mz_grid_len())
        n = int(self._num_peaks[obs])
        ss = np.zeros(g + 1, np.uint32)
        cy = np.zeros(max(n, 1), np.uint16)
        it = np.zeros(max(n, 1), np.float32)
        F.check(L.ads_dia_copy_observation(self._h, obs, ss.ctypes.data, cy.ctypes.data, it.ctypes.data))
        return dict(isolation_window=tuple(self._iso[obs]), slice_starts=ss,
                    cycle_indices=cy[:n], intensities=it[:n])


_QUANT_PASSTHROUGH = ("precursor_mz_library", "precursor_mz", "precursor_rt_library", "precursor_rt",
                      "precursor_naa", "fragment_mz_library", "fragment_mz", "fragment_cardinality",
                      "fragment_charge", "fragment_loss_type", "fragment_number", "fragment_position",
                      "fragment_type")


class SpecLibFlat:
    """SpecLibFlat (src/speclib_flat/mod.rs:6-199), device resident."""

    def __init__(self):
        self._passthrough = None
        self._h = None
        self._n_prec = 0
        self._n_frag = 0
        self.device = _DEFAULT_DEVICE

    def __del__(self):
        _release(self, "ads_lib_destroy")

    @staticmethod
    def from_arrays(precursor_idx, precursor_mz_library, precursor_mz, precursor_rt_library,
                    precursor_rt, precursor_naa, flat_frag_start_idx, flat_frag_stop_idx,
                    fragment_mz_library, fragment_mz, fragment_intensity, fragment_cardinality,
                    fragment_charge, fragment_loss_type, fragment_number, fragment_position,
                    fragment_type, *, precursor_rt_tolerance=None, device: int | None = None):
        """SpecLibFlat::from_arrays (src/speclib_flat/mod.rs:98-188).
        ``precursor_rt_tolerance`` (extension): per-precursor RT half-window in
        seconds replacing SelectionParameters.rt_tolerance."""
        L = _lib()
        spec = [("precursor_idx", precursor_idx, np.uint64), ("precursor_mz_library", precursor_mz_library, np.float32),
                ("precursor_mz", precursor_mz, np.float32), ("precursor_rt_library", precursor_rt_library, np.float32),
                ("precursor_rt", precursor_rt, np.float32), ("precursor_naa", precursor_naa, np.uint8),
                ("flat_frag_start_idx", flat_frag_start_idx, np.uint64), ("flat_frag_stop_idx", flat_frag_stop_idx, np.uint64),
                ("fragment_mz_library", fragment_mz_library, np.float32), ("fragment_mz", fragment_mz, np.float32),
                ("fragment_intensity", fragment_intensity, np.float32), ("fragment_cardinality", fragment_cardinality, np.uint8),
                ("fragment_charge", fragment_charge, np.uint8), ("fragment_loss_type", fragment_loss_type, np.uint8),
                ("fragment_number", fragment_number, np.uint8), ("fragment_position", fragment_position, np.uint8),
                ("fragment_type", fragment_type, np.uint8)]
        if precursor_rt_tolerance is not None:
            spec.append(("precursor_rt_tolerance", precursor_rt_tolerance, np.float32))
        on_dev = [_is_device_tensor(a) for _, a, _ in spec]
        if any(on_dev) and not all(on_dev):
            raise ValueError("library arrays must be all host arrays or all CUDA tensors")
        arr = F.AdsLibArrays()
        keep = []
        if all(on_dev):
            dev = spec[0][1].device.index if device is None else device
            arr.location = F.ADS_MEM_DEVICE
            ptr = {n: _dev_ptr(n, a, t, dev) for n, a, t in spec}
            lens = {n: int(a.numel()) for n, a, _ in spec}
        else:
            dev = _DEFAULT_DEVICE if device is None else device
            arr.location = F.ADS_MEM_HOST
            conv = {n: _as_np(n, a, t) for n, a, t in spec}
            keep.append(conv)
            ptr = {n: a.ctypes.data for n, a in conv.items()}
            lens = {n: a.size for n, a in conv.items()}
        n_prec = lens["precursor_idx"]
        n_frag = lens["fragment_mz"]
        for n, _, _ in spec:
            want = n_prec if n.startswith("precursor") or n.startswith("flat") else n_frag
            if lens[n] != want:
                raise ValueError(f"argument '{n}': length {lens[n]}, expected {want}")
        arr.n_precursors = n_prec
        arr.n_fragments = n_frag
        for n, _, _ in spec:
            setattr(arr, n, ptr[n] if lens[n] else None)
        h = C.c_void_p()
        F.check(L.ads_lib_create(C.byref(arr), int(dev), C.byref(h)))
        lib = SpecLibFlat()
        lib._h = h.value
        lib._n_prec = n_prec
        lib._n_frag = n_frag
        lib.device = int(dev)
        # the columns PeakGroupQuantification passes through (read at quantify time)
        src = {n: a for n, a, _ in spec} if all(on_dev) else conv
        lib._passthrough = {n: src[n] for n in _QUANT_PASSTHROUGH}
        return lib

    @property
    def num_precursors(self) -> int:
        return self._n_prec

    @property
    def num_fragments(self) -> int:
        return self._n_frag

    def idf_counts(self, out=None):
        """Extension: the fragments of this library per m/z grid bin, the document
        counts of scoring's IDF (src/idf/mod.rs:13-33), as a uint32 numpy array, or
        written into ``out`` (a contiguous 32-bit CUDA tensor of ads_idf_bins()
        elements) without leaving the device."""
        L = _lib()
        n = int(L.ads_idf_bins())
        if out is not None:
            if not _is_device_tensor(out) or out.numel() != n or out.element_size() != 4 or \
                    not out.is_contiguous():
                raise ValueError(f"out must be a contiguous 32-bit CUDA tensor of {n} elements")
            F.check(L.ads_lib_idf_counts(self._h, out.data_ptr(), F.ADS_MEM_DEVICE))
            return out
        counts = np.empty(n, np.uint32)
        F.check(L.ads_lib_idf_counts(self._h, counts.ctypes.data, F.ADS_MEM_HOST))
        return counts

    def set_idf(self, counts, total_fragments: int) -> None:
        """Extension: replaces the histogram and fragment total that scoring's IDF uses
        (the sums over the shards of a library split across ranks)."""
        L = _lib()
        n = int(L.ads_idf_bins())
        if _is_device_tensor(counts):
            if counts.numel() != n or counts.element_size() != 4 or not counts.is_contiguous():
                raise ValueError(f"counts must be a contiguous 32-bit tensor of {n} elements")
            F.check(L.ads_lib_set_idf(self._h, counts.data_ptr(), float(total_fragments), F.ADS_MEM_DEVICE))
            return
        c = np.ascontiguousarray(counts, np.uint32)
        if c.size != n:
            raise ValueError(f"counts must hold {n} elements")
        F.check(L.ads_lib_set_idf(self._h, c.ctypes.data, float(total_fragments), F.ADS_MEM_HOST))


_FLOAT_KEYS = ("fwhm_rt", "mass_tolerance", "rt_tolerance")
_USIZE_KEYS = ("kernel_size", "peak_length", "candidate_count", "top_k_fragments")
# the order in which update() reads the keys (parameters.rs:45-68)
_SELECTION_UPDATE_ORDER = ("fwhm_rt", "kernel_size", "peak_length", "mass_tolerance", "rt_tolerance",
                           "candidate_count", "top_k_fragments")


def _extract_f32(val) -> float:
    """pyo3's extract::<f32>: any object with __float__ (or __index__), rounded to f32."""
    if not (hasattr(val, "__float__") or hasattr(val, "__index__")):
        raise TypeError(f"'{type(val).__name__}' object cannot be converted to 'PyFloat'")
    return float(np.float32(float(val)))


def _extract_usize(val) -> int:
    """pyo3's extract::<usize>: integers only (no floats), 0 <= v < 2**64."""
    if isinstance(val, (float, np.floating)) or not hasattr(val, "__index__"):
        raise TypeError(f"'{type(val).__name__}' object cannot be interpreted as an integer")
    iv = int(val.__index__())
    if iv < 0:
        raise OverflowError("can't convert negative int to unsigned")
    if iv >= 2**64:
        raise OverflowError("int too big to convert")
    return iv


_F32_PARAMS = frozenset(_FLOAT_KEYS + ("tolerance_ppm",))


def _update_in_order(obj, config: dict, order) -> None:
    """Reads the keys present in ``config`` in the reference's order; the first
    value that does not convert raises, and the keys read before it stay set."""
    for k in order:
        if k in config:
            conv = _extract_f32 if k in _F32_PARAMS else _extract_usize
            v = dict(object.__getattribute__(obj, "_v"))
            v[k] = conv(config[k])
            object.__setattr__(obj, "_v", v)


class SelectionParameters:
    """SelectionParameters (src/peak_group_selection/parameters.rs:4-75): read-only
    attributes, defaults of ``new``, and ``update(dict)``."""

    __slots__ = ("_v",)

    def __init__(self):
        p = F.AdsSelectionParams()
        _lib().ads_selection_params_default(C.byref(p))
        object.__setattr__(self, "_v", {k: getattr(p, k) for k, _ in F.AdsSelectionParams._fields_})
        for k in _FLOAT_KEYS:
            self._v[k] = float(np.float32(self._v[k]))

    def __getattr__(self, name):
        v = object.__getattribute__(self, "_v")
        if name in v:
            return v[name]
        raise AttributeError(name)

    def __setattr__(self, name, value):
        raise AttributeError(f"attribute '{name}' of 'SelectionParameters' objects is not writable")

    def update(self, config: dict) -> None:
        """Sets any of the seven keys present in ``config`` (parameters.rs:45-68)."""
        _update_in_order(self, config, _SELECTION_UPDATE_ORDER)

    def _c(self) -> F.AdsSelectionParams:
        p = F.AdsSelectionParams()
        for k, _ in F.AdsSelectionParams._fields_:
            v = self._v[k]
            if k in _USIZE_KEYS:
                v = min(v, 2**63 - 1)
            setattr(p, k, v)
        return p

    def __repr__(self):
        return "SelectionParameters(" + ", ".join(f"{k}={v!r}" for k, v in self._v.items()) + ")"


class CandidateCollection:
    """CandidateCollection (src/candidate/entry.rs:41-193)."""

    _COLS = ("precursor_idx", "rank", "score", "scan_center", "scan_start", "scan_stop",
             "cycle_center", "cycle_start", "cycle_stop")

    def __init__(self):
        self._h = None
        self._arrays = {c: np.zeros(0, np.float32 if c == "score" else np.uint64) for c in self._COLS}
        self._n = 0

    def __del__(self):
        _release(self, "ads_candidates_destroy")

    @classmethod
    def _from_handle(cls, h: int) -> "CandidateCollection":
        c = cls()
        c._h = h
        n = int(_lib().ads_candidates_size(h))
        if n < 0:
            F.check(F.ADS_ERR_INTERNAL)
        c._n = n
        c._arrays = None
        return c

    def _materialize(self) -> dict:
        if self._arrays is None:
            n = self._n
            cols = {c: np.zeros(n, np.float32 if c == "score" else np.uint64) for c in self._COLS}
            if n:
                ptr = [cols[c].ctypes.data for c in self._COLS]
                for i in (3, 4, 5):  # scan_* stay zero (np.zeros), as in the reference
                    ptr[i] = None
                F.check(_lib().ads_candidates_copy_out(self._h, *ptr))
            self._arrays = cols
            _lib().ads_candidates_destroy(self._h)
            self._h = None
        return self._arrays

    @staticmethod
    def from_arrays(precursor_idxs, ranks, scores, scan_center, scan_start, scan_stop,
                    cycle_center, cycle_start, cycle_stop) -> "CandidateCollection":
        """src/candidate/entry.rs:70-120 (ValueError when lengths differ)."""
        cols = [precursor_idxs, ranks, scores, scan_center, scan_start, scan_stop, cycle_center,
                cycle_start, cycle_stop]
        n = len(cols[0])
        if not all(len(c) == n for c in cols[1:]):
            raise ValueError("All input arrays must have the same length")
        c = CandidateCollection()
        c._arrays = {name: np.asarray(v, dtype=np.float32 if name == "score" else np.uint64).copy()
                     for name, v in zip(CandidateCollection._COLS, cols)}
        c._n = n
        return c

    def len(self) -> int:
        return self._n

    def __len__(self) -> int:
        return self._n

    def is_empty(self) -> bool:
        return self._n == 0

    def to_arrays(self, *, out=None):
        """Nine arrays in the reference's tuple order (src/candidate/entry.rs:124-173):
        precursor_idx, rank, score, scan_center, scan_start, scan_stop, cycle_center,
        cycle_start, cycle_stop.

        ``out`` (extension): nine preallocated arrays (for example views of pinned
        memory) of at least len() elements; the first len() entries are written and
        views of them returned."""
        if out is not None and self._h is not None and self._arrays is None:
            n = self._n
            if len(out) != 9 or any(len(o) < n for o in out):
                raise ValueError("out must be nine arrays of at least len() elements")
            for o, c in zip(out, self._COLS):
                want = np.float32 if c == "score" else np.uint64
                if o.dtype != want or not o.flags.c_contiguous:
                    raise TypeError(f"out array for {c} must be contiguous {np.dtype(want).name}")
            if n:
                F.check(_lib().ads_candidates_copy_out(self._h, *[o.ctypes.data for o in out]))
            return tuple(o[:n] for o in out)
        a = self._materialize()
        return tuple(a[c].copy() for c in self._COLS)


class PeakGroupSelection:
    """PeakGroupSelection (src/peak_group_selection/mod.rs:66-90) on the GPU."""

    def __init__(self, params: SelectionParameters, *, precision: str = "fp32", verbose: bool = True,
                 device: int | None = None, warps_per_block: int = 0, blocks_per_sm: int = 0,
                 gather_mode: int = 0, time_stages: bool = False, stream: int = 0,
                 cycles_per_lane: int = 0, use_graph: bool = False):
        if not isinstance(params, SelectionParameters):
            raise TypeError("argument 'params': expected SelectionParameters")
        L = _lib()
        self.params = params
        self.device = _DEFAULT_DEVICE if device is None else int(device)
        o = F.AdsEngineOptions()
        L.ads_engine_options_default(C.byref(o))
        o.precision = {"fp32": F.ADS_PRECISION_FP32, "bf16": F.ADS_PRECISION_BF16}[precision]
        o.verbose = 1 if verbose else 0
        o.warps_per_block = warps_per_block
        o.blocks_per_sm = blocks_per_sm
        o.gather_mode = gather_mode
        o.time_stages = 1 if time_stages else 0
        o.cycles_per_lane = int(cycles_per_lane)
        o.use_graph = 1 if use_graph else 0
        o.stream = int(stream)
        self._opts = o
        p = params._c()
        h = C.c_void_p()
        F.check(L.ads_selection_create(C.byref(p), C.byref(o), self.device, C.byref(h)))
        self._h = h.value

    def __del__(self):
        _release(self, "ads_selection_destroy")

    def search(self, dia_data: DIAData, lib: SpecLibFlat) -> CandidateCollection:
        if not isinstance(dia_data, DIAData) or not isinstance(lib, SpecLibFlat):
            raise TypeError("search(dia_data: DIAData, lib: SpecLibFlat)")
        if dia_data._h is None or lib._h is None:
            raise ValueError("DIAData and SpecLibFlat must be built with from_arrays")
        out = C.c_void_p()
        F.check(_lib().ads_select(self._h, dia_data._h, lib._h, C.byref(out)))
        return CandidateCollection._from_handle(out.value)

    # ---- engine extras
    def kernel(self) -> np.ndarray:
        n = C.c_int64()
        F.check(_lib().ads_selection_kernel(self._h, None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 1), np.float32)
        F.check(_lib().ads_selection_kernel(self._h, out.ctypes.data, n.value, C.byref(n)))
        return out[:n.value].copy()

    @property
    def stream(self) -> int:
        return int(_lib().ads_selection_stream(self._h))

    @property
    def last_launches(self) -> int:
        return int(_lib().ads_selection_last_launches(self._h))

    def search_into(self, dia_data: DIAData, lib: SpecLibFlat, cand: "DeviceCandidates") -> None:
        """Enqueue a search without waiting, reusing ``cand``'s device buffers."""
        F.check(_lib().ads_select_async(self._h, dia_data._h, lib._h, cand._h))

    def autotune(self, dia_data: DIAData, lib: SpecLibFlat, repeats: int = 2) -> dict:
        """Times the launch shapes on this run and library and keeps the fastest
        (cached per workload shape for the process); returns the choice."""
        w, c, ms = C.c_int32(), C.c_int32(), C.c_float()
        F.check(_lib().ads_selection_autotune(self._h, dia_data._h, lib._h, int(repeats),
                                               C.byref(w), C.byref(c), C.byref(ms)))
        return dict(warps_per_block=w.value, cycles_per_lane=c.value, ms=ms.value)

    def new_candidates(self) -> "DeviceCandidates":
        return DeviceCandidates(self)

    def stage_times(self) -> dict:
        """Summed device ms per stage over the searches since the last call
        (needs time_stages=True)."""
        out = np.zeros(4, np.float32)
        F.check(_lib().ads_selection_stage_times(self._h, out.ctypes.data, 4))
        return dict(prep_ms=float(out[0]), search_ms=float(out[1]), compaction_ms=float(out[2]),
                    searches=int(out[3]))

    def enable_stats(self, on: bool = True) -> None:
        F.check(_lib().ads_selection_set_stats(self._h, 1 if on else 0))

    def last_stats(self) -> dict:
        out = np.zeros(7, np.int64)
        F.check(_lib().ads_selection_last_stats(self._h, out.ctypes.data, 7))
        return dict(pairs=int(out[0]), bins_plus_one=int(out[1]), fragments=int(out[2]),
                    entries_read=int(out[3]), entries_accumulated=int(out[4]),
                    offsets_read=int(out[5]), xic_cells=int(out[6]))


class DeviceCandidates:
    """A reusable device-side candidate buffer for PeakGroupSelection.search_into."""

    def __init__(self, sel: PeakGroupSelection):
        h = C.c_void_p()
        F.check(_lib().ads_candidates_create(sel._h, C.byref(h)))
        self._h = h.value

    def __del__(self):
        _release(self, "ads_candidates_destroy")

    def size(self) -> int:
        n = int(_lib().ads_candidates_size(self._h))
        if n < 0:
            F.check(F.ADS_ERR_INTERNAL)
        return n

    def copy_out(self, out: dict) -> int:
        """Copies into preallocated arrays keyed by column name (missing keys skipped)."""
        n = self.size()
        cols = CandidateCollection._COLS
        ptr = [out[c].ctypes.data if c in out else None for c in cols]
        F.check(_lib().ads_candidates_copy_out(self._h, *ptr))
        return n


def gaussian_kernel(fwhm_rt: float, sigma_scale_rt: float, kernel_width: int,
                    rt_resolution: float) -> np.ndarray:
    """GaussianKernel::new(...).kernel_array (src/kernel/mod.rs:13-56)."""
    L = _lib()
    n = C.c_int64()
    F.check(L.ads_gaussian_kernel(fwhm_rt, sigma_scale_rt, int(kernel_width), rt_resolution, None, 0, C.byref(n)))
    out = np.zeros(max(n.value, 1), np.float32)
    F.check(L.ads_gaussian_kernel(fwhm_rt, sigma_scale_rt, int(kernel_width), rt_resolution,
                                  out.ctypes.data, n.value, C.byref(n)))
    return out[:n.value].copy()


def mz_grid() -> np.ndarray:
    """The global 1-ppm m/z grid (src/mz_index/mod.rs:4-27)."""
    L = _lib()
    n = int(L.ads_mz_grid_len())
    out = np.zeros(n, np.float32)
    F.check(L.ads_mz_grid(out.ctypes.data, n))
    return out


def device_count() -> int:
    return int(_lib().ads_device_count())


# ------------------------------------------------------------------ scoring

class ScoringParameters:
    """ScoringParameters (src/peak_group_scoring/parameters.rs:4-40): read-only
    mass_tolerance and top_k_fragments, defaults of ``new``, and ``update(dict)``."""

    __slots__ = ("_v",)

    def __init__(self):
        p = F.AdsScoringParams()
        _lib().ads_scoring_params_default(C.byref(p))
        object.__setattr__(self, "_v", {"mass_tolerance": float(np.float32(p.mass_tolerance)),
                                        "top_k_fragments": int(p.top_k_fragments)})

    def __getattr__(self, name):
        v = object.__getattribute__(self, "_v")
        if name in v:
            return v[name]
        raise AttributeError(name)

    def __setattr__(self, name, value):
        raise AttributeError(f"attribute '{name}' of 'ScoringParameters' objects is not writable")

    def update(self, config: dict) -> None:
        """Sets mass_tolerance and/or top_k_fragments (parameters.rs:28-37)."""
        _update_in_order(self, config, ("mass_tolerance", "top_k_fragments"))

    def _c(self) -> F.AdsScoringParams:
        p = F.AdsScoringParams()
        p.mass_tolerance = self._v["mass_tolerance"]
        p.top_k_fragments = min(self._v["top_k_fragments"], 2**63 - 1)
        return p

    def __repr__(self):
        return "ScoringParameters(" + ", ".join(f"{k}={v!r}" for k, v in self._v.items()) + ")"


def _feature_names() -> tuple:
    names = (C.c_char_p * 64)()
    n = _lib().ads_feature_names(names, 64)
    return tuple(names[k].decode() for k in range(n))


class CandidateFeatureCollection:
    """CandidateFeatureCollection (src/candidate/features.rs:192-431)."""

    def __init__(self):
        self._h = None
        self._n = 0

    def __del__(self):
        _release(self, "ads_features_destroy")

    @classmethod
    def _from_handle(cls, h: int) -> "CandidateFeatureCollection":
        c = cls()
        c._h = h
        c._n = int(_lib().ads_features_size(h))
        return c

    def len(self) -> int:
        return self._n

    def __len__(self) -> int:
        return self._n

    def is_empty(self) -> bool:
        return self._n == 0

    def kernel_ms(self) -> float:
        """Extension: device time of the scoring kernel in milliseconds."""
        return float(_lib().ads_features_kernel_ms(self._h)) if self._h is not None else 0.0

    def to_dict_arrays(self) -> dict:
        """precursor_idx and rank (uint64) and the 41 float32 feature columns
        (src/candidate/features.rs:220-411)."""
        # fresh arrays on every call (as the reference builds them from its vectors):
        # one device-to-host copy, the feature columns are rows of one block
        n = self._n
        names = _feature_names()
        pidx = _host_empty(max(n, 1), np.uint64)
        rank = _host_empty(max(n, 1), np.uint64)
        feats = _host_empty(len(names) * max(n, 1), np.float32).reshape(len(names), max(n, 1))
        if self._h is not None and n:
            F.check(_lib().ads_features_copy_out(self._h, pidx.ctypes.data, rank.ctypes.data,
                                                 feats.ctypes.data))
        d = {"precursor_idx": pidx[:n], "rank": rank[:n]}
        for k, name in enumerate(names):
            d[name] = feats[k, :n]
        return d

    @staticmethod
    def get_feature_names() -> list:
        """src/candidate/features.rs:413-416"""
        return list(_feature_names())


class PeakGroupScoring:
    """PeakGroupScoring (src/peak_group_scoring/mod.rs:29-101) on the GPU."""

    def __init__(self, params: ScoringParameters, *, verbose: bool = True):
        if not isinstance(params, ScoringParameters):
            raise TypeError("argument 'params': expected ScoringParameters")
        self.params = params
        self.verbose = verbose

    def score(self, dia_data: DIAData, lib: SpecLibFlat,
              candidates: CandidateCollection) -> CandidateFeatureCollection:
        """Features of every candidate whose precursor_idx is in ``lib``.  Extension:
        ``candidates`` may also be a DeviceCandidates buffer (search_into)."""
        if not isinstance(dia_data, DIAData) or not isinstance(lib, SpecLibFlat) or \
                not isinstance(candidates, (CandidateCollection, DeviceCandidates)):
            raise TypeError("score(dia_data: DIAData, lib: SpecLibFlat, candidates: CandidateCollection)")
        if dia_data._h is None or lib._h is None:
            raise ValueError("DIAData and SpecLibFlat must be built with from_arrays")
        p = self.params._c()
        out = C.c_void_p()
        L = _lib()
        if isinstance(candidates, DeviceCandidates) or (candidates._h is not None and
                                                         candidates._arrays is None):
            F.check(L.ads_score(C.byref(p), dia_data._h, lib._h, candidates._h, int(self.verbose),
                                C.byref(out)))
        else:
            a = candidates._materialize()
            cols = [np.ascontiguousarray(a[k], np.uint64) for k in
                    ("precursor_idx", "rank", "cycle_center", "cycle_start", "cycle_stop")]
            sc = np.ascontiguousarray(a["score"], np.float32)
            n = len(cols[0])
            F.check(L.ads_score_arrays(C.byref(p), dia_data._h, lib._h, n, cols[0].ctypes.data,
                                       cols[1].ctypes.data, sc.ctypes.data, cols[2].ctypes.data,
                                       cols[3].ctypes.data, cols[4].ctypes.data, F.ADS_MEM_HOST,
                                       int(self.verbose), C.byref(out)))
        return CandidateFeatureCollection._from_handle(out.value)


# ------------------------------------------------------------------ quantification

class QuantificationParameters:
    """QuantificationParameters (src/peak_group_quantification/parameters.rs:4-44):
    tolerance_ppm and top_k_fragments, readable and writable, the defaults of ``new``
    and ``update(dict)``."""

    __slots__ = ("_v",)

    def __init__(self):
        p = F.AdsQuantParams()
        _lib().ads_quant_params_default(C.byref(p))
        object.__setattr__(self, "_v", {"tolerance_ppm": float(np.float32(p.tolerance_ppm)),
                                        "top_k_fragments": int(p.top_k_fragments)})

    def __getattr__(self, name):
        v = object.__getattribute__(self, "_v")
        if name in v:
            return v[name]
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name not in ("tolerance_ppm", "top_k_fragments"):
            raise AttributeError(f"'QuantificationParameters' object has no attribute '{name}'")
        _update_in_order(self, {name: value}, (name,))

    def __delattr__(self, name):
        raise TypeError("can't delete attribute")

    def update(self, config: dict) -> None:
        """Sets tolerance_ppm and/or top_k_fragments (parameters.rs:30-37)."""
        _update_in_order(self, config, ("tolerance_ppm", "top_k_fragments"))

    def _c(self) -> F.AdsQuantParams:
        p = F.AdsQuantParams()
        p.tolerance_ppm = self._v["tolerance_ppm"]
        p.top_k_fragments = min(self._v["top_k_fragments"], 2**63 - 1)
        return p

    def __repr__(self):
        return (f"QuantificationParameters(tolerance_ppm={self.tolerance_ppm}, "
                f"top_k_fragments={self.top_k_fragments})")


_QUANT_PRECURSOR_KEYS = ("precursor_idx", "mz_library", "mz", "rt_library", "rt", "naa", "rank",
                         "rt_observed", "flat_frag_start_idx", "flat_frag_stop_idx")
_QUANT_FRAGMENT_KEYS = ("mz_library", "mz", "intensity", "cardinality", "charge", "loss_type", "number",
                        "position", "type", "mz_observed", "correlation_observed", "mass_error_observed",
                        "precursor_idx", "rank")
_QUANT_DTYPES = {"precursor_idx": np.uint64, "rank": np.uint64, "flat_frag_start_idx": np.uint64,
                 "flat_frag_stop_idx": np.uint64, "naa": np.uint8, "cardinality": np.uint8,
                 "charge": np.uint8, "loss_type": np.uint8, "number": np.uint8, "position": np.uint8,
                 "type": np.uint8}


class SpecLibFlatQuantified:
    """SpecLibFlatQuantified (src/speclib_flat_quantified/mod.rs:19-210): quantified
    precursors sorted by precursor_idx, their fragments in candidate order."""

    def __init__(self):
        self._prec = {k: np.zeros(0, _QUANT_DTYPES.get(k, np.float32)) for k in _QUANT_PRECURSOR_KEYS}
        self._frag = {k: np.zeros(0, _QUANT_DTYPES.get(k, np.float32)) for k in _QUANT_FRAGMENT_KEYS}
        self._kernel_ms = 0.0

    @property
    def num_precursors(self) -> int:
        return len(self._prec["mz"])

    @property
    def num_fragments(self) -> int:
        return len(self._frag["mz"])

    def to_dict_arrays(self) -> tuple:
        """(precursor dict, fragment dict) (src/speclib_flat_quantified/mod.rs:126-210)."""
        return ({k: self._prec[k].copy() for k in _QUANT_PRECURSOR_KEYS},
                {k: self._frag[k].copy() for k in _QUANT_FRAGMENT_KEYS})

    def kernel_ms(self) -> float:
        """Extension: device time of the quantification kernel in milliseconds."""
        return self._kernel_ms


class _Rows:
    """Row indices for the pass-through gathers, moved to a CUDA device at most once.
    Gathers from CUDA tensors are copied into page-locked host arrays without waiting;
    finish() waits for all of them."""

    def __init__(self, rows: np.ndarray):
        self.rows = rows
        self._dev = {}
        self._streams = []

    def take(self, src) -> np.ndarray:
        """src[rows] for a numpy array or a CUDA tensor, as a numpy array (valid after
        finish())."""
        if _is_device_tensor(src):
            import torch

            key = src.device
            if key not in self._dev:
                self._dev[key] = torch.from_numpy(self.rows).to(src.device, non_blocking=False)
            sel = src.index_select(0, self._dev[key])
            out = torch.empty(sel.shape, dtype=sel.dtype, pin_memory=True)
            out.copy_(sel, non_blocking=True)
            self._streams.append(torch.cuda.current_stream(src.device))
            return out.numpy()
        return np.asarray(src)[self.rows]

    def finish(self) -> None:
        for st in set(self._streams):
            st.synchronize()
        self._streams.clear()


class PeakGroupQuantification:
    """PeakGroupQuantification (src/peak_group_quantification/mod.rs:24-168) on the GPU."""

    def __init__(self, params: QuantificationParameters, *, verbose: bool = True):
        if not isinstance(params, QuantificationParameters):
            raise TypeError("argument 'params': expected QuantificationParameters")
        self.params = params
        self.verbose = verbose

    def quantify(self, dia_data: DIAData, lib: SpecLibFlat, candidates) -> SpecLibFlatQuantified:
        """Quantifies every candidate whose precursor is in ``lib``.  ``candidates`` is a
        CandidateCollection, or (extension) a DeviceCandidates buffer.  The library's
        pass-through columns are read from the arrays given to SpecLibFlat.from_arrays."""
        if not isinstance(dia_data, DIAData) or not isinstance(lib, SpecLibFlat) or \
                not isinstance(candidates, (CandidateCollection, DeviceCandidates)):
            raise TypeError("quantify(dia_data: DIAData, lib: SpecLibFlat, candidates: CandidateCollection)")
        if dia_data._h is None or lib._h is None:
            raise ValueError("DIAData and SpecLibFlat must be built with from_arrays")
        p = self.params._c()
        h = C.c_void_p()
        L = _lib()
        if isinstance(candidates, DeviceCandidates) or (candidates._h is not None and
                                                         candidates._arrays is None):
            F.check(L.ads_quantify(C.byref(p), dia_data._h, lib._h, candidates._h, int(self.verbose),
                                   C.byref(h)))
        else:
            a = candidates._materialize()
            cols = [np.ascontiguousarray(a[k], np.uint64) for k in
                    ("precursor_idx", "rank", "cycle_center", "cycle_start", "cycle_stop")]
            F.check(L.ads_quantify_arrays(C.byref(p), dia_data._h, lib._h, len(cols[0]),
                                          *[c.ctypes.data for c in cols], F.ADS_MEM_HOST,
                                          int(self.verbose), C.byref(h)))
        out = SpecLibFlatQuantified()
        try:
            n_p, n_f = C.c_int64(), C.c_int64()
            F.check(L.ads_quant_sizes(h, C.byref(n_p), C.byref(n_f)))
            P, NF = n_p.value, n_f.value
            out._kernel_ms = float(L.ads_quant_kernel_ms(h))
            u = lambda m: _host_empty(max(m, 1), np.uint64)
            f = lambda m: _host_empty(max(m, 1), np.float32)
            pidx, prow, prank, prt, pfs, pfe = u(P), u(P), u(P), f(P), u(P), u(P)
            frow, fint, fmzo, fcorr, ferr, fpidx, frank = u(NF), f(NF), f(NF), f(NF), f(NF), u(NF), u(NF)
            if P:
                F.check(L.ads_quant_copy_out(h, *[x.ctypes.data for x in (
                    pidx, prow, prank, prt, pfs, pfe, frow, fint, fmzo, fcorr, ferr, fpidx, frank)]))
        finally:
            L.ads_quant_destroy(h)
        src = lib._passthrough
        pr, fr = _Rows(prow[:P].view(np.int64)), _Rows(frow[:NF].view(np.int64))
        out._prec = {"precursor_idx": pidx[:P], "mz_library": pr.take(src["precursor_mz_library"]),
                     "mz": pr.take(src["precursor_mz"]),
                     "rt_library": pr.take(src["precursor_rt_library"]),
                     "rt": pr.take(src["precursor_rt"]), "naa": pr.take(src["precursor_naa"]),
                     "rank": prank[:P], "rt_observed": prt[:P], "flat_frag_start_idx": pfs[:P],
                     "flat_frag_stop_idx": pfe[:P]}
        out._frag = {"mz_library": fr.take(src["fragment_mz_library"]), "mz": fr.take(src["fragment_mz"]),
                     "intensity": fint[:NF], "cardinality": fr.take(src["fragment_cardinality"]),
                     "charge": fr.take(src["fragment_charge"]),
                     "loss_type": fr.take(src["fragment_loss_type"]),
                     "number": fr.take(src["fragment_number"]),
                     "position": fr.take(src["fragment_position"]), "type": fr.take(src["fragment_type"]),
                     "mz_observed": fmzo[:NF], "correlation_observed": fcorr[:NF],
                     "mass_error_observed": ferr[:NF], "precursor_idx": fpidx[:NF], "rank": frank[:NF]}
        pr.finish()
        fr.finish()
        for d in (out._prec, out._frag):
            for k, v in d.items():
                d[k] = np.ascontiguousarray(v, _QUANT_DTYPES.get(k, np.float32))
        return out
