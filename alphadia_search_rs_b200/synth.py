"""Seeded synthetic DIA runs and spectral libraries with the shapes of the
benchmark configurations (no public dataset is used or reproduced).

Run layout (per cycle c): one MS1 spectrum (delta_scan_idx 0, isolation [-1, -1],
no peaks, rt = c * cycle_time seconds, cycle_time 1 s unless a configuration says
otherwise) followed by W MS2 spectra (delta_scan_idx 1..W) with
contiguous isolation windows.  Each MS2 spectrum has N random peaks (m/z uniform
in [150, 1800], intensity log-normal(mu=8, sigma=2)) plus the planted signal.

Library: P precursors (precursor_idx a seeded permutation of 0..P-1), F fragments
each (m/z uniform 150-1800, intensities Dirichlet(1), fragment numbers >= 2 so
the y1 filter is a no-op).  A fraction ``planted`` of the targets elutes: for
every fragment and cycle within apex +- 4 sigma a peak is inserted at the
fragment m/z (+ N(0, 2 ppm) jitter) into the windows holding the precursor m/z
with intensity A * lib_int * exp(-(c - apex)^2 / (2 sigma^2)) * LogNormal(0, 0.3),
A = 1e6, sigma = 4 cycles.  Library RT = (apex + N(0, 20)) * cycle_time.  Decoys (if any) have
their fragment m/z shifted by U(-50, 50), clamped to [150, 1800].

Backends: ``torch`` (on a CUDA device; used for the large configurations) and
``numpy`` (CPU, for small cases).  Both follow the same steps with their own
random streams; each is deterministic for a given seed.
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace

import numpy as np

PLANT_AMPLITUDE = 1.0e6
PLANT_SIGMA = 4.0
PLANT_NOISE_SIGMA = 0.3
PLANT_PPM_JITTER = 2.0
RT_LIB_SIGMA = 20.0
PEAK_MZ_RANGE = (150.0, 1800.0)


@dataclass(frozen=True)
class SynthConfig:
    name: str
    n_cycles: int
    n_windows: int
    window_width: float
    window_start: float
    peaks_per_spectrum: int
    n_precursors: int
    frag_min: int
    frag_max: int
    precursor_mz_range: tuple
    charge_range: tuple
    rt_half_window: tuple          # (lo, hi) seconds; lo == hi -> global rt_tolerance
    mass_tolerance: float
    sigma_cycles: float            # Gaussian kernel sigma (fwhm = 2.3548 * sigma)
    kernel_size: int
    candidate_count: int
    top_k_fragments: int
    decoy_fraction: float = 0.0
    planted: float = 0.6
    seed: int = 0
    precision: str = "fp32"
    cycle_time: float = 1.0        # seconds per cycle (spectrum RT = cycle * cycle_time)

    @property
    def fwhm_rt(self) -> float:
        return float(np.float32(self.sigma_cycles * 2.3548))

    @property
    def per_precursor_tolerance(self) -> bool:
        return self.rt_half_window[0] != self.rt_half_window[1]

    def params_dict(self) -> dict:
        return dict(fwhm_rt=self.fwhm_rt, kernel_size=self.kernel_size, peak_length=5,
                    mass_tolerance=self.mass_tolerance, rt_tolerance=float(self.rt_half_window[1]),
                    candidate_count=self.candidate_count, top_k_fragments=self.top_k_fragments)

    @property
    def n_ms2_peaks(self) -> int:
        return self.n_cycles * self.n_windows * self.peaks_per_spectrum


CONFIGS = {
    # small cases for tests
    "tiny": SynthConfig("tiny", 160, 4, 25.0, 400.0, 300, 300, 12, 12, (400.0, 500.0), (2, 3),
                        (40.0, 40.0), 15.0, 2.0, 21, 3, 12, seed=11),
    "tiny_uneven": SynthConfig("tiny_uneven", 400, 6, 10.0, 400.0, 400, 600, 4, 24, (400.0, 460.0),
                               (2, 4), (30.0, 160.0), 15.0, 2.0, 21, 3, 24, decoy_fraction=0.5, seed=12),
    # cfg4's search settings (kernel sigma 3 / width 31, 10 ppm, top-5, 4-24 fragments,
    # RT half-windows up to 300 cycles: several length classes, multi-pass rows)
    # precursors with 20-60 library fragments, 40 kept: more than one warp's worth of
    # fragments in the library preparation and the search
    "tiny_many": SynthConfig("tiny_many", 300, 4, 25.0, 400.0, 300, 300, 20, 60, (400.0, 500.0),
                             (2, 3), (40.0, 120.0), 15.0, 2.0, 21, 3, 40, decoy_fraction=0.3,
                             seed=14),
    "tiny_cfg4": SynthConfig("tiny_cfg4", 700, 6, 8.0, 400.0, 400, 400, 4, 24, (400.0, 448.0),
                             (2, 4), (30.0, 300.0), 10.0, 3.0, 31, 5, 24, decoy_fraction=0.5,
                             seed=13),
    # long RT windows: per-precursor half-windows of 400-1100 cycles on a 2600-cycle run
    # (length classes up to cfg2/3's 801 and cfg4's 1201 cycles, the widest shared-memory
    # plan at 2048 cycles and windows beyond it)
    "tiny_long": SynthConfig("tiny_long", 2600, 4, 25.0, 400.0, 200, 300, 4, 24, (400.0, 500.0),
                             (2, 4), (400.0, 1100.0), 15.0, 2.0, 21, 3, 24, decoy_fraction=0.5,
                             seed=15),
    # 6000 cycles of 0.5 s searched with rt_tolerance 1000 s: every window spans about
    # 4000 cycles
    "long_rt": SynthConfig("long_rt", 6000, 3, 25.0, 400.0, 150, 200, 12, 12, (400.0, 475.0),
                           (2, 3), (1000.0, 1000.0), 15.0, 2.0, 21, 3, 12, seed=16,
                           cycle_time=0.5),
    # the benchmark configurations
    "cfg0": SynthConfig("cfg0", 1000, 8, 25.0, 400.0, 1500, 2000, 12, 12, (400.0, 600.0), (2, 3),
                        (100.0, 100.0), 15.0, 2.0, 21, 3, 12, seed=100),
    "cfg1": SynthConfig("cfg1", 3000, 300, 2.0, 380.0, 1000, 200_000, 12, 12, (380.0, 980.0), (2, 3),
                        (150.0, 150.0), 15.0, 2.0, 21, 3, 12, seed=101),
    # cfg1's densities on 60 of its 300 windows (380-500 m/z): a profiling-sized case
    "cfg1_prof": SynthConfig("cfg1_prof", 3000, 60, 2.0, 380.0, 1000, 40_000, 12, 12, (380.0, 500.0),
                             (2, 3), (150.0, 150.0), 15.0, 2.0, 21, 3, 12, seed=101),
    # cfg3's densities on 60 of its 300 windows (380-500 m/z): a profiling-sized case
    "cfg3_prof": SynthConfig("cfg3_prof", 3000, 60, 2.0, 380.0, 1000, 100_000, 4, 24, (380.0, 500.0),
                             (2, 4), (30.0, 400.0), 15.0, 2.0, 21, 3, 24, decoy_fraction=0.5, seed=102,
                             precision="bf16"),
    "cfg2": SynthConfig("cfg2", 3000, 300, 2.0, 380.0, 1000, 500_000, 4, 24, (380.0, 980.0), (2, 4),
                        (30.0, 400.0), 15.0, 2.0, 21, 3, 24, decoy_fraction=0.5, seed=102),
    "cfg3": SynthConfig("cfg3", 3000, 300, 2.0, 380.0, 1000, 500_000, 4, 24, (380.0, 980.0), (2, 4),
                        (30.0, 400.0), 15.0, 2.0, 21, 3, 24, decoy_fraction=0.5, seed=102,
                        precision="bf16"),
    "cfg4": SynthConfig("cfg4", 6000, 400, 1.5, 380.0, 1500, 2_000_000, 4, 24, (380.0, 980.0), (2, 4),
                        (30.0, 600.0), 10.0, 3.0, 31, 5, 24, decoy_fraction=0.5, seed=104,
                        precision="bf16"),
}


def get_config(name: str, **overrides) -> SynthConfig:
    c = CONFIGS[name]
    return replace(c, **overrides) if overrides else c


# ------------------------------------------------------------------ backend

class _NP:
    def __init__(self, seed):
        self.rng = np.random.default_rng(seed)
        self.lib = np

    def rand(self, n):
        return self.rng.random(n, dtype=np.float64)

    def randn(self, n):
        return self.rng.standard_normal(n)

    def randint(self, lo, hi, n):
        return self.rng.integers(lo, hi, n)

    def perm(self, n):
        return self.rng.permutation(n)

    def arange(self, n):
        return np.arange(n, dtype=np.int64)

    def repeat(self, x, counts):
        return np.repeat(x, counts)

    def cumsum(self, x):
        return np.cumsum(x)

    def stable_argsort(self, x):
        return np.argsort(x, kind="stable")

    def to_numpy(self, x):
        return np.asarray(x)

    def f32(self, x):
        return np.asarray(x, dtype=np.float32)

    def i64(self, x):
        return np.asarray(x, dtype=np.int64)

    def f64(self, x):
        return np.asarray(x, dtype=np.float64)

    def cat(self, xs):
        return np.concatenate(xs)

    def zeros_i64(self, n):
        return np.zeros(n, np.int64)

    def full(self, n, v, kind):
        return np.full(n, v, dtype={"f32": np.float32, "i64": np.int64}[kind])

    def scatter_add_count(self, idx, n):
        return np.bincount(idx, minlength=n).astype(np.int64)

    def exp(self, x):
        return np.exp(x)

    def clip(self, x, lo, hi):
        return np.clip(x, lo, hi)


class _TORCH:
    def __init__(self, seed, device):
        import torch

        self.t = torch
        self.dev = torch.device(device)
        self.g = torch.Generator(device=self.dev)
        self.g.manual_seed(int(seed))

    def rand(self, n):
        return self.t.rand(int(n), generator=self.g, device=self.dev, dtype=self.t.float64)

    def randn(self, n):
        return self.t.randn(int(n), generator=self.g, device=self.dev, dtype=self.t.float64)

    def randint(self, lo, hi, n):
        return self.t.randint(int(lo), int(hi), (int(n),), generator=self.g, device=self.dev)

    def perm(self, n):
        return self.t.randperm(int(n), generator=self.g, device=self.dev)

    def arange(self, n):
        return self.t.arange(int(n), device=self.dev, dtype=self.t.int64)

    def repeat(self, x, counts):
        return self.t.repeat_interleave(x, counts)

    def cumsum(self, x):
        return self.t.cumsum(x, 0)

    def stable_argsort(self, x):
        return self.t.sort(x, stable=True).indices

    def to_numpy(self, x):
        return x.cpu().numpy()

    def f32(self, x):
        return x.to(self.t.float32)

    def i64(self, x):
        return x.to(self.t.int64)

    def f64(self, x):
        return x.to(self.t.float64)

    def cat(self, xs):
        return self.t.cat(xs)

    def zeros_i64(self, n):
        return self.t.zeros(int(n), device=self.dev, dtype=self.t.int64)

    def full(self, n, v, kind):
        return self.t.full((int(n),), v, device=self.dev,
                           dtype={"f32": self.t.float32, "i64": self.t.int64}[kind])

    def scatter_add_count(self, idx, n):
        return self.t.bincount(idx, minlength=int(n)).to(self.t.int64)

    def exp(self, x):
        return self.t.exp(x)

    def clip(self, x, lo, hi):
        return self.t.clamp(x, lo, hi)


def _backend(backend, seed, device):
    if backend == "numpy":
        return _NP(seed)
    if backend == "torch":
        return _TORCH(seed, device)
    raise ValueError(backend)


# ------------------------------------------------------------------ library

def make_library(cfg: SynthConfig, backend="numpy", device="cuda:0") -> dict:
    """Spectral library arrays in the argument order of SpecLibFlat.from_arrays plus
    the generator's ground truth (apex, planted, decoy) in sorted-library order."""
    B = _backend(backend, cfg.seed * 7919 + 1, device)
    P = cfg.n_precursors
    nfrag = B.randint(cfg.frag_min, cfg.frag_max + 1, P)
    stop = B.cumsum(nfrag)
    start = stop - nfrag
    NF = int(B.to_numpy(stop[-1])) if P else 0
    lo, hi = cfg.precursor_mz_range
    pmz = B.f32(lo + (hi - lo) * B.rand(P))
    charge = B.randint(cfg.charge_range[0], cfg.charge_range[1] + 1, P)
    apex = B.rand(P) * (cfg.n_cycles - 1)
    prt = B.f32((apex + RT_LIB_SIGMA * B.randn(P)) * cfg.cycle_time)
    is_decoy = B.rand(P) < cfg.decoy_fraction
    planted = (~is_decoy) & (B.rand(P) < cfg.planted)
    owner = B.repeat(B.arange(P), nfrag)
    fmz = PEAK_MZ_RANGE[0] + (PEAK_MZ_RANGE[1] - PEAK_MZ_RANGE[0]) * B.rand(NF)
    shift = (B.rand(NF) * 100.0 - 50.0)
    decoy_f = is_decoy[owner]
    fmz = B.clip(fmz + shift * decoy_f, PEAK_MZ_RANGE[0], PEAK_MZ_RANGE[1])
    e = -B.lib.log(B.rand(NF) + 1e-300) if backend == "numpy" else -B.t.log(B.rand(NF) + 1e-300)
    denom = B.zeros_i64(P).to(B.t.float64) if backend == "torch" else np.zeros(P)
    if backend == "torch":
        denom.index_add_(0, owner, e)
    else:
        np.add.at(denom, owner, e)
    fint = B.f32(e / denom[owner])
    fnum = B.randint(2, 21, NF)
    ftype = B.cat([B.full(0, 0, "i64")]) if NF == 0 else B.randint(0, 2, NF)
    ftype = ftype * (121 - 98) + 98  # b or y
    pidx = B.perm(P)
    rt_tol = None
    if cfg.per_precursor_tolerance:
        rt_tol = B.f32(cfg.rt_half_window[0] + (cfg.rt_half_window[1] - cfg.rt_half_window[0]) * B.rand(P))
    out = dict(
        precursor_idx=pidx, precursor_mz=pmz, precursor_rt=prt, flat_frag_start_idx=start,
        flat_frag_stop_idx=stop, fragment_mz=B.f32(fmz), fragment_intensity=fint,
        fragment_number=fnum, fragment_type=ftype, charge=charge, apex=apex, planted=planted,
        is_decoy=is_decoy, rt_tolerance=rt_tol, n_fragments=NF, backend=backend,
    )
    return out


def library_arrays(lib: dict) -> dict:
    """Keyword arrays for SpecLibFlat.from_arrays with the reference dtypes (numpy)."""
    if lib["backend"] == "torch":
        n = {k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in lib.items()}
    else:
        n = lib
    P = len(n["precursor_idx"])
    NF = len(n["fragment_mz"])
    out = dict(
        precursor_idx=np.asarray(n["precursor_idx"], np.uint64),
        precursor_mz_library=np.asarray(n["precursor_mz"], np.float32),
        precursor_mz=np.asarray(n["precursor_mz"], np.float32),
        precursor_rt_library=np.asarray(n["precursor_rt"], np.float32),
        precursor_rt=np.asarray(n["precursor_rt"], np.float32),
        precursor_naa=np.full(P, 10, np.uint8),
        flat_frag_start_idx=np.asarray(n["flat_frag_start_idx"], np.uint64),
        flat_frag_stop_idx=np.asarray(n["flat_frag_stop_idx"], np.uint64),
        fragment_mz_library=np.asarray(n["fragment_mz"], np.float32),
        fragment_mz=np.asarray(n["fragment_mz"], np.float32),
        fragment_intensity=np.asarray(n["fragment_intensity"], np.float32),
        fragment_cardinality=np.ones(NF, np.uint8),
        fragment_charge=np.ones(NF, np.uint8),
        fragment_loss_type=np.zeros(NF, np.uint8),
        fragment_number=np.asarray(n["fragment_number"], np.uint8),
        fragment_position=np.ones(NF, np.uint8),
        fragment_type=np.asarray(n["fragment_type"], np.uint8),
    )
    if n.get("rt_tolerance") is not None:
        out["precursor_rt_tolerance"] = np.asarray(n["rt_tolerance"], np.float32)
    return out


# -------------------------------------------------------------------- run

# Random MS2 peaks generated and sorted at once by the torch backend; larger runs
# are generated in blocks of consecutive cycles (the sort of ~1e9 float64 keys with
# its index arrays is what bounds device memory).
TORCH_BLOCK_PEAKS = 1_200_000_000


def make_run(cfg: SynthConfig, lib: dict, backend="numpy", device="cuda:0") -> dict:
    """DIA run arrays in the argument order of DIAData.from_arrays (on the
    backend's device); ``cycle`` is a host array."""
    if backend == "torch" and cfg.n_ms2_peaks > TORCH_BLOCK_PEAKS:
        return _make_run_torch_blocked(cfg, lib, device)
    B = _backend(backend, cfg.seed * 104729 + 7, device)
    W, NC, N = cfg.n_windows, cfg.n_cycles, cfg.peaks_per_spectrum
    n_spec = NC * (W + 1)
    sidx = B.arange(n_spec)
    cyc = sidx // (W + 1)
    dsi = sidx % (W + 1)
    wlo = cfg.window_start + (dsi - 1).clamp(min=0) * cfg.window_width if backend == "torch" else \
        cfg.window_start + np.maximum(dsi - 1, 0) * cfg.window_width
    iso_lo = B.f32(wlo)
    iso_hi = B.f32(wlo + cfg.window_width)
    ms1 = dsi == 0
    if backend == "torch":
        iso_lo = iso_lo.masked_fill(ms1, -1.0)
        iso_hi = iso_hi.masked_fill(ms1, -1.0)
    else:
        iso_lo = np.where(ms1, np.float32(-1.0), iso_lo).astype(np.float32)
        iso_hi = np.where(ms1, np.float32(-1.0), iso_hi).astype(np.float32)
    rt = B.f32((cyc.to(B.t.float64) if backend == "torch" else cyc.astype(np.float64)) * cfg.cycle_time)

    # random peaks: spectrum id of MS2 spectra only
    ms2_ids = sidx[~ms1]
    n_rand = ms2_ids.shape[0] * N
    r_spec = B.repeat(ms2_ids, B.full(ms2_ids.shape[0], N, "i64"))
    r_mz = PEAK_MZ_RANGE[0] + (PEAK_MZ_RANGE[1] - PEAK_MZ_RANGE[0]) * B.rand(n_rand)
    r_int = B.exp(8.0 + 2.0 * B.randn(n_rand))

    # planted peaks
    to_dev = (lambda x: x.to(B.dev)) if backend == "torch" else (lambda x: np.asarray(x))
    planted = to_dev(lib["planted"])
    apex = to_dev(lib["apex"])
    pmz = to_dev(lib["precursor_mz"])
    fst = to_dev(lib["flat_frag_start_idx"])
    fsp = to_dev(lib["flat_frag_stop_idx"])
    fmz_all = to_dev(lib["fragment_mz"])
    fint_all = to_dev(lib["fragment_intensity"])
    pl_ids = B.arange(planted.shape[0])[planted]
    half = int(np.ceil(4 * PLANT_SIGMA))
    span = 2 * half + 1
    nfr = (fsp - fst)[pl_ids]
    # (precursor, fragment) pairs
    pf_prec = B.repeat(pl_ids, nfr)
    first = B.cumsum(nfr) - nfr
    pair_rank = B.arange(pf_prec.shape[0]) - B.repeat(first, nfr)
    pf_frag = fst[pf_prec] + pair_rank
    # windows holding the precursor m/z (contiguous windows: at most two)
    pm = pmz[pf_prec].to(B.t.float64) if backend == "torch" else pmz[pf_prec].astype(np.float64)
    wf = (pm - cfg.window_start) / cfg.window_width
    w_a = wf.floor() if backend == "torch" else np.floor(wf)
    w_a = B.i64(w_a) + 1  # dsi of the window starting at or below mz
    pairs_w = []
    for dw in (0, -1):
        w = w_a + dw
        ok = (w >= 1) & (w <= W)
        wc = w.clamp(1, W) if backend == "torch" else np.clip(w, 1, W)
        lo_w = B.f32(cfg.window_start + (wc - 1) * cfg.window_width)
        hi_w = B.f32(cfg.window_start + (wc - 1) * cfg.window_width + cfg.window_width)
        pmf = pmz[pf_prec]
        ok = ok & (lo_w <= pmf) & (hi_w >= pmf)
        pairs_w.append((ok, wc))
    recs_spec, recs_mz, recs_int = [], [], []
    for ok, wc in pairs_w:
        sel = B.arange(ok.shape[0])[ok]
        if sel.shape[0] == 0:
            continue
        k = sel.shape[0]
        rep = B.repeat(sel, B.full(k, span, "i64"))
        off = (B.arange(k * span) % span) - half
        prec = pf_prec[rep]
        ap = apex[prec]
        apr = ap.round() if backend == "torch" else np.round(ap)
        c = B.i64(apr) + off
        good = (c >= 0) & (c < NC)
        rep, c, ap = rep[good], c[good], ap[good]
        m = rep.shape[0]
        frag = pf_frag[rep]
        d = c.to(B.t.float64) - ap if backend == "torch" else c.astype(np.float64) - ap
        inten = PLANT_AMPLITUDE * fint_all[frag] * B.exp(-(d * d) / (2 * PLANT_SIGMA ** 2)) * \
            B.exp(PLANT_NOISE_SIGMA * B.randn(m))
        mzj = fmz_all[frag] * (1.0 + PLANT_PPM_JITTER * 1e-6 * B.randn(m))
        recs_spec.append(c * (W + 1) + wc[rep])
        recs_mz.append(mzj)
        recs_int.append(inten)
    all_spec = B.cat([r_spec] + recs_spec)
    all_mz = B.f32(B.cat([r_mz] + [B.f64(x) for x in recs_mz]))
    all_int = B.f32(B.cat([r_int] + [B.f64(x) for x in recs_int]))
    # one stable sort on the exact key spectrum * 2048 + m/z (m/z < 2048)
    key = B.f64(all_spec) * 2048.0 + B.f64(all_mz)
    order = B.stable_argsort(key)
    all_spec = all_spec[order]
    peak_mz = all_mz[order]
    peak_int = all_int[order]
    counts = B.scatter_add_count(all_spec, n_spec)
    stop = B.cumsum(counts)
    start = stop - counts
    cycle_arr = np.zeros((W + 1, 1, 1, 1), np.float32)
    return dict(spectrum_delta_scan_idx=B.i64(dsi), isolation_lower_mz=iso_lo, isolation_upper_mz=iso_hi,
                spectrum_peak_start_idx=B.i64(start), spectrum_peak_stop_idx=B.i64(stop),
                spectrum_cycle_idx=B.i64(cyc), spectrum_rt=rt, peak_mz=peak_mz, peak_intensity=peak_int,
                cycle=cycle_arr)


def _make_run_torch_blocked(cfg: SynthConfig, lib: dict, device: str) -> dict:
    """make_run for runs too large to generate at once (torch backend): the same
    distributions, with the planted peaks drawn first and the random peaks drawn,
    merged and sorted one block of consecutive cycles at a time, each block written
    into the preallocated peak arrays.  Only the block being sorted holds float64
    keys, so device memory stays near the size of the final f32 arrays."""
    import torch

    B = _TORCH(cfg.seed * 104729 + 11, device)
    t = torch
    dev = B.dev
    W, NC, N = cfg.n_windows, cfg.n_cycles, cfg.peaks_per_spectrum
    S1 = W + 1
    n_spec = NC * S1
    sidx = t.arange(n_spec, device=dev)
    cyc = sidx // S1
    dsi = sidx % S1
    wlo = cfg.window_start + (dsi - 1).clamp(min=0) * cfg.window_width
    ms1 = dsi == 0
    iso_lo = wlo.to(t.float32).masked_fill(ms1, -1.0)
    iso_hi = (wlo + cfg.window_width).to(t.float32).masked_fill(ms1, -1.0)
    rt = (cyc.to(t.float64) * cfg.cycle_time).to(t.float32)
    del sidx, wlo

    # planted peaks (spectrum id, m/z, intensity), all cycles at once
    planted = lib["planted"].to(dev)
    apex = lib["apex"].to(dev)
    pmz = lib["precursor_mz"].to(dev)
    fst = lib["flat_frag_start_idx"].to(dev)
    fsp = lib["flat_frag_stop_idx"].to(dev)
    fmz_all = lib["fragment_mz"].to(dev)
    fint_all = lib["fragment_intensity"].to(dev)
    pl_ids = t.arange(planted.shape[0], device=dev)[planted]
    half = int(np.ceil(4 * PLANT_SIGMA))
    span = 2 * half + 1
    nfr = (fsp - fst)[pl_ids]
    pf_prec = t.repeat_interleave(pl_ids, nfr)
    first = t.cumsum(nfr, 0) - nfr
    pf_frag = fst[pf_prec] + (t.arange(pf_prec.shape[0], device=dev) - t.repeat_interleave(first, nfr))
    pm = pmz[pf_prec]
    w_a = ((pm.to(t.float64) - cfg.window_start) / cfg.window_width).floor().to(t.int64) + 1
    p_spec, p_mz, p_int = [], [], []
    for dw in (0, -1):
        w = w_a + dw
        wc = w.clamp(1, W)
        lo_w = (cfg.window_start + (wc - 1) * cfg.window_width).to(t.float32)
        hi_w = (cfg.window_start + (wc - 1) * cfg.window_width + cfg.window_width).to(t.float32)
        ok = (w >= 1) & (w <= W) & (lo_w <= pm) & (hi_w >= pm)
        sel = t.nonzero(ok).flatten()
        if sel.numel() == 0:
            continue
        rep = t.repeat_interleave(sel, span)
        off = (t.arange(rep.numel(), device=dev) % span) - half
        ap = apex[pf_prec[rep]]
        c = ap.round().to(t.int64) + off
        good = (c >= 0) & (c < NC)
        rep, c, ap = rep[good], c[good], ap[good]
        frag = pf_frag[rep]
        d = c.to(t.float64) - ap
        inten = PLANT_AMPLITUDE * fint_all[frag].to(t.float64) * t.exp(-(d * d) / (2 * PLANT_SIGMA ** 2)) * \
            t.exp(PLANT_NOISE_SIGMA * B.randn(rep.numel()))
        mzj = fmz_all[frag].to(t.float64) * (1.0 + PLANT_PPM_JITTER * 1e-6 * B.randn(rep.numel()))
        p_spec.append(c * S1 + wc[rep])
        p_mz.append(mzj.to(t.float32))
        p_int.append(inten.to(t.float32))
        del rep, off, ap, c, good, frag, d, inten, mzj
    p_spec = t.cat(p_spec) if p_spec else t.zeros(0, dtype=t.int64, device=dev)
    p_mz = t.cat(p_mz) if p_mz else t.zeros(0, dtype=t.float32, device=dev)
    p_int = t.cat(p_int) if p_int else t.zeros(0, dtype=t.float32, device=dev)
    del pf_prec, pf_frag, pm, w_a, first, nfr, pl_ids

    counts = t.bincount(p_spec, minlength=n_spec).to(t.int64)
    counts[~ms1] += N
    stop = t.cumsum(counts, 0)
    start = stop - counts
    total = int(stop[-1].item()) if n_spec else 0
    peak_mz = t.empty(total, dtype=t.float32, device=dev)
    peak_int = t.empty(total, dtype=t.float32, device=dev)

    # blocks of consecutive cycles: their spectra, and so their peaks, are contiguous
    cyc_per_block = max(1, TORCH_BLOCK_PEAKS // max(1, W * N))
    p_cyc = p_spec // S1
    for c0 in range(0, NC, cyc_per_block):
        c1 = min(NC, c0 + cyc_per_block)
        s0, s1 = c0 * S1, c1 * S1
        ms2_ids = t.arange(s0, s1, device=dev)
        ms2_ids = ms2_ids[(ms2_ids % S1) != 0]
        n_rand = ms2_ids.numel() * N
        r_spec = t.repeat_interleave(ms2_ids, N)
        r_mz = (PEAK_MZ_RANGE[0] + (PEAK_MZ_RANGE[1] - PEAK_MZ_RANGE[0]) * B.rand(n_rand)).to(t.float32)
        r_int = t.exp(8.0 + 2.0 * B.randn(n_rand)).to(t.float32)
        sel = t.nonzero((p_cyc >= c0) & (p_cyc < c1)).flatten()
        spec = t.cat([r_spec, p_spec[sel]])
        mz = t.cat([r_mz, p_mz[sel]])
        inten = t.cat([r_int, p_int[sel]])
        del r_spec, r_mz, r_int, ms2_ids, sel
        key = (spec - s0).to(t.float64) * 2048.0 + mz.to(t.float64)
        order = t.sort(key, stable=True).indices
        del key, spec
        o0 = int(start[s0].item())
        peak_mz[o0:o0 + order.numel()] = mz[order]
        peak_int[o0:o0 + order.numel()] = inten[order]
        del order, mz, inten
    cycle_arr = np.zeros((W + 1, 1, 1, 1), np.float32)
    return dict(spectrum_delta_scan_idx=dsi, isolation_lower_mz=iso_lo, isolation_upper_mz=iso_hi,
                spectrum_peak_start_idx=start, spectrum_peak_stop_idx=stop, spectrum_cycle_idx=cyc,
                spectrum_rt=rt, peak_mz=peak_mz, peak_intensity=peak_int, cycle=cycle_arr)


def run_to_numpy(run: dict) -> dict:
    return {k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in run.items()}


def make_workload(name: str, backend="numpy", device="cuda:0", **overrides):
    cfg = get_config(name, **overrides)
    lib = make_library(cfg, backend, device)
    run = make_run(cfg, lib, backend, device)
    return cfg, lib, run
