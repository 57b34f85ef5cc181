#!/usr/bin/env python
"""Benchmark: precursors/s of peak-group selection (XIC + convolution + score +
top-k + compaction) on B200.

Workload (default ``cfg3``): a synthetic Astral-scale DIA run of 3000 cycles x 300
MS2 windows of 2 Th (380-980 m/z), 1000 peaks per spectrum (~0.95 G peaks incl.
planted signal, ~8.8 GB resident), and 500,000 precursors (half decoys) with 4-24
fragments and per-precursor RT half-windows of 30-400 s; 15 ppm, Gaussian sigma 2
cycles (kernel_size 21), top-3.  The headline searches it with BF16 intensity
storage (f32 arithmetic); the same process times the plain FP32 path on the same
run, library and settings (cfg2) and reports both and their ratio.  ``--workload
cfg1`` is the 200,000-precursor plain FP32 case.  Data are generated on the device
from a fixed seed (no dataset is used).

One step = one PeakGroupSelection.search over the whole library with inputs
resident in HBM.  Inputs are far larger than L2 (126 MB), so no L2 flush is
needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 the script runs one rank per GPU (torchrun); every rank searches its own
library of the same size against its own copy of the run (weak scaling, no
collective on the data path); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

RUN_KEYS = ("spectrum_delta_scan_idx", "isolation_lower_mz", "isolation_upper_mz",
            "spectrum_peak_start_idx", "spectrum_peak_stop_idx", "spectrum_cycle_idx",
            "spectrum_rt", "peak_mz", "peak_intensity")
METRIC = "precursors/s (XIC+conv+score+top-k) on 1 B200: batched-BF16 vs plain FP32"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg3",
                    help="synthetic configuration (default cfg3: BF16 storage, timed beside the "
                         "plain FP32 path on the same data)")
    ap.add_argument("--e2e-steps", type=int, default=7)
    ap.add_argument("--cpu-windows", type=int, default=0,
                    help="MS2 windows in the CPU-baseline sample (0: about 72 M peaks' worth)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-scoring", action="store_true",
                    help="skip the scoring and quantification figures added to the JSON line")
    ap.add_argument("--warps-per-block", type=int, default=0)
    ap.add_argument("--blocks-per-sm", type=int, default=0)
    ap.add_argument("--cycles-per-lane", type=int, default=0)
    ap.add_argument("--gather-mode", type=int, default=0, choices=[0, 1, 2],
                    help="0 automatic, 1 scan every bin range, 2 binary-search every bin")
    ap.add_argument("--graph", dest="graph", action="store_true", default=True,
                    help="replay a captured CUDA graph per search (the default; stage times "
                         "then come from a second, directly enqueued pass)")
    ap.add_argument("--no-graph", dest="graph", action="store_false",
                    help="enqueue every search's kernels directly")
    ap.add_argument("--autotune", dest="autotune", action="store_true", default=None,
                    help="pick warps per block and cycles per lane with the engine's autotuner, "
                         "untimed, before the timed region (default: on for the batched uneven "
                         "workloads cfg2-cfg4)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false")
    ap.add_argument("--precision", choices=["fp32", "bf16"], default=None,
                    help="override the workload's precision (cfg3/cfg4: bf16 storage)")
    return ap.parse_args()


# ----------------------------------------------------------------- clocks

class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    def __init__(self, device_index: int):
        self.samples = []
        self._stop = threading.Event()
        self._thr = None
        self.max_mhz = None
        try:
            import pynvml

            pynvml.nvmlInit()
            import torch

            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            h = None
            for i in range(pynvml.nvmlDeviceGetCount()):
                hh = pynvml.nvmlDeviceGetHandleByIndex(i)
                u = pynvml.nvmlDeviceGetUUID(hh)
                u = u.decode() if isinstance(u, bytes) else u
                if u.replace("GPU-", "") == uuid.replace("GPU-", ""):
                    h = hh
            self.h = h if h is not None else pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.nv = pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # no NVML: clocks reported as unavailable
            self.nv = None
            self.err = str(e)

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((sm, int(reasons)))
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        if self.nv is not None:
            self._thr = threading.Thread(target=self._run, daemon=True)
            self._thr.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._thr:
            self._thr.join()

    def summary(self):
        if self.nv is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        nv = self.nv
        names = {
            getattr(nv, "nvmlClocksEventReasonGpuIdle", 0x1): "gpu_idle",
            getattr(nv, "nvmlClocksEventReasonApplicationsClocksSetting", 0x2): "applications_clocks_setting",
            getattr(nv, "nvmlClocksEventReasonSwPowerCap", 0x4): "sw_power_cap",
            getattr(nv, "nvmlClocksEventReasonHwSlowdown", 0x8): "hw_slowdown",
            getattr(nv, "nvmlClocksEventReasonSyncBoost", 0x10): "sync_boost",
            getattr(nv, "nvmlClocksEventReasonSwThermalSlowdown", 0x20): "sw_thermal_slowdown",
            getattr(nv, "nvmlClocksEventReasonHwThermalSlowdown", 0x40): "hw_thermal_slowdown",
            getattr(nv, "nvmlClocksEventReasonHwPowerBrakeSlowdown", 0x80): "hw_power_brake_slowdown",
            getattr(nv, "nvmlClocksEventReasonDisplayClockSetting", 0x100): "display_clock_setting",
        }
        seen = 0
        for _, r in self.samples:
            seen |= r
        reasons = sorted(n for bit, n in names.items() if seen & bit)
        share = {n: round(sum(1 for _, r in self.samples if r & bit) / len(self.samples), 4)
                 for bit, n in names.items() if seen & bit}
        med = statistics.median([s for s, _ in self.samples]) if self.samples else None
        return {"sm_mhz": med, "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "reason_share": share, "samples": len(self.samples)}


# --------------------------------------------------------------- workload

def make_device_workload(name: str, device: str, lib_seed_offset: int = 0):
    from alphadia_search_rs_b200 import synth

    cfg = synth.get_config(name)
    lib_cfg = synth.get_config(name, seed=cfg.seed + 1000 * lib_seed_offset) if lib_seed_offset else cfg
    lib = synth.make_library(lib_cfg, "torch", device)
    run = synth.make_run(cfg, lib, "torch", device)
    import torch

    torch.cuda.synchronize()
    torch.cuda.empty_cache()  # the generator's temporaries: the engine allocates outside torch
    return cfg, lib, run


def library_tensors(lib: dict, device: str):
    """SpecLibFlat.from_arrays keyword tensors on the device (reference dtypes)."""
    import torch

    P = lib["precursor_idx"].numel()
    NF = lib["fragment_mz"].numel()
    d = torch.device(device)
    out = dict(
        precursor_idx=lib["precursor_idx"].to(torch.uint64),
        precursor_mz_library=lib["precursor_mz"], precursor_mz=lib["precursor_mz"],
        precursor_rt_library=lib["precursor_rt"], precursor_rt=lib["precursor_rt"],
        precursor_naa=torch.full((P,), 10, dtype=torch.uint8, device=d),
        flat_frag_start_idx=lib["flat_frag_start_idx"].to(torch.uint64),
        flat_frag_stop_idx=lib["flat_frag_stop_idx"].to(torch.uint64),
        fragment_mz_library=lib["fragment_mz"], fragment_mz=lib["fragment_mz"],
        fragment_intensity=lib["fragment_intensity"],
        fragment_cardinality=torch.ones(NF, dtype=torch.uint8, device=d),
        fragment_charge=torch.ones(NF, dtype=torch.uint8, device=d),
        fragment_loss_type=torch.zeros(NF, dtype=torch.uint8, device=d),
        fragment_number=lib["fragment_number"].to(torch.uint8),
        fragment_position=torch.ones(NF, dtype=torch.uint8, device=d),
        fragment_type=lib["fragment_type"].to(torch.uint8),
    )
    out = {k: v.contiguous() for k, v in out.items()}
    if lib.get("rt_tolerance") is not None:
        out["precursor_rt_tolerance"] = lib["rt_tolerance"].contiguous()
    return out


def host_copies(tensors: dict, copy) -> dict:
    """copy(t) of every tensor, one copy per distinct tensor: columns that are the same
    array (the synthetic library's m/z and library m/z, RT and library RT) stay one
    array on the host, as a caller's would."""
    done = {}
    return {k: done.setdefault(id(v), copy(v)) for k, v in tensors.items()}


def sample_windows(cfg, requested: int) -> int:
    """MS2 windows of the CPU sample: as requested, else about 72 M peaks' worth
    (24 windows at 3000 cycles x 1000 peaks)."""
    if requested > 0:
        return min(requested, cfg.n_windows)
    per_window = cfg.n_cycles * cfg.peaks_per_spectrum
    return max(1, min(cfg.n_windows, round(72e6 / per_window)))


def window_subset(cfg, run: dict, lib: dict, n_windows: int):
    """Host copy of the MS1 spectra plus ``n_windows`` consecutive MS2 windows from
    the middle of the run, and the library precursors whose every valid window lies
    in that subset (strictly inside its m/z span).  Windows are renumbered 1..n."""
    import torch

    W = cfg.n_windows
    w0 = max(1, (W - n_windows) // 2 + 1)
    w1 = min(W, w0 + n_windows - 1)
    dsi = run["spectrum_delta_scan_idx"]
    keep = (dsi == 0) | ((dsi >= w0) & (dsi <= w1))
    sidx = torch.nonzero(keep).flatten()
    st, sp = run["spectrum_peak_start_idx"], run["spectrum_peak_stop_idx"]
    counts = (sp - st)[sidx]
    # peaks of the kept spectra, in spectrum order
    owner = torch.repeat_interleave(torch.arange(sidx.numel(), device=dsi.device), counts)
    first = torch.cumsum(counts, 0) - counts
    pk = st[sidx][owner] + (torch.arange(owner.numel(), device=dsi.device) - first[owner])
    new_stop = torch.cumsum(counts, 0)
    new_start = new_stop - counts
    new_dsi = dsi[sidx].clone()
    new_dsi[new_dsi > 0] -= (w0 - 1)
    host = dict(
        spectrum_delta_scan_idx=new_dsi.cpu().numpy().astype(np.int64),
        isolation_lower_mz=run["isolation_lower_mz"][sidx].cpu().numpy(),
        isolation_upper_mz=run["isolation_upper_mz"][sidx].cpu().numpy(),
        spectrum_peak_start_idx=new_start.cpu().numpy().astype(np.int64),
        spectrum_peak_stop_idx=new_stop.cpu().numpy().astype(np.int64),
        spectrum_cycle_idx=run["spectrum_cycle_idx"][sidx].cpu().numpy().astype(np.int64),
        spectrum_rt=run["spectrum_rt"][sidx].cpu().numpy(),
        peak_mz=run["peak_mz"][pk].cpu().numpy(),
        peak_intensity=run["peak_intensity"][pk].cpu().numpy(),
        cycle=np.zeros((n_windows + 1, 1, 1, 1), np.float32),
    )
    lo = np.float32(cfg.window_start + (w0 - 1) * cfg.window_width)
    hi = np.float32(cfg.window_start + w1 * cfg.window_width)
    pmz = lib["precursor_mz"].cpu().numpy()
    sel = np.nonzero((pmz > lo) & (pmz < hi))[0]
    fs = lib["flat_frag_start_idx"].cpu().numpy()
    fe = lib["flat_frag_stop_idx"].cpu().numpy()
    nf = fe[sel] - fs[sel]
    fidx = np.concatenate([np.arange(a, b) for a, b in zip(fs[sel], fe[sel])]) if len(sel) else np.zeros(0, np.int64)
    new_fe = np.cumsum(nf)
    sub = dict(
        precursor_idx=lib["precursor_idx"].cpu().numpy()[sel].astype(np.uint64),
        precursor_mz=pmz[sel], precursor_rt=lib["precursor_rt"].cpu().numpy()[sel],
        flat_frag_start_idx=(new_fe - nf).astype(np.uint64), flat_frag_stop_idx=new_fe.astype(np.uint64),
        fragment_mz=lib["fragment_mz"].cpu().numpy()[fidx],
        fragment_intensity=lib["fragment_intensity"].cpu().numpy()[fidx],
        fragment_number=lib["fragment_number"].cpu().numpy()[fidx].astype(np.uint8),
        fragment_type=lib["fragment_type"].cpu().numpy()[fidx].astype(np.uint8),
    )
    if lib.get("rt_tolerance") is not None:
        sub["rt_tolerance"] = lib["rt_tolerance"].cpu().numpy()[sel]
    return host, sub, (w0, w1)


def bf16_agreement(got: dict, ref: dict, eps_rel_max: float = 1e-3):
    """(fraction of the FP64 oracle's (precursor, rank) rows whose cycle the GPU
    found too, relative score errors over those rows).  The error of a row is taken
    against max(|s64|, eps_rel_max * the precursor's largest |s64|), since scores
    near zero are common at the RT-window edges."""
    ref_max = {}
    for p, s64 in zip(ref["precursor_idx"], ref["score_f64"]):
        ref_max[int(p)] = max(ref_max.get(int(p), 0.0), abs(float(s64)))
    mine = {(int(p), int(r)): (int(c), float(s)) for p, r, c, s in
            zip(got["precursor_idx"], got["rank"], got["cycle_center"], got["score"])}
    same, errs = 0, []
    for p, r, c, s64 in zip(ref["precursor_idx"], ref["rank"], ref["cycle_center"], ref["score_f64"]):
        m = mine.get((int(p), int(r)))
        if m is None or m[0] != int(c):
            continue
        same += 1
        den = max(abs(float(s64)), eps_rel_max * ref_max[int(p)])
        errs.append(abs(m[1] - float(s64)) / den if den > 0 else 0.0)
    return same / max(len(ref["rank"]), 1), np.asarray(errs if errs else [0.0])


def sub_library_arrays(sub: dict) -> dict:
    """SpecLibFlat.from_arrays keywords (numpy, reference dtypes) of a window
    subset's library, with the same constant columns as library_tensors."""
    P, NF = len(sub["precursor_idx"]), len(sub["fragment_mz"])
    out = dict(
        precursor_idx=sub["precursor_idx"], precursor_mz_library=sub["precursor_mz"],
        precursor_mz=sub["precursor_mz"], precursor_rt_library=sub["precursor_rt"],
        precursor_rt=sub["precursor_rt"], precursor_naa=np.full(P, 10, np.uint8),
        flat_frag_start_idx=sub["flat_frag_start_idx"], flat_frag_stop_idx=sub["flat_frag_stop_idx"],
        fragment_mz_library=sub["fragment_mz"], fragment_mz=sub["fragment_mz"],
        fragment_intensity=sub["fragment_intensity"],
        fragment_cardinality=np.ones(NF, np.uint8), fragment_charge=np.ones(NF, np.uint8),
        fragment_loss_type=np.zeros(NF, np.uint8), fragment_number=sub["fragment_number"],
        fragment_position=np.ones(NF, np.uint8), fragment_type=sub["fragment_type"])
    if "rt_tolerance" in sub:
        out["precursor_rt_tolerance"] = sub["rt_tolerance"]
    return out


CAND_COLS = ("precursor_idx", "rank", "score", "scan_center", "scan_start", "scan_stop",
             "cycle_center", "cycle_start", "cycle_stop")


def scoring_figures(ads, dia, slib, cand, out_np, steps: int = 3) -> dict:
    """PeakGroupScoring.score of the search's candidates: the scoring kernel's device
    time (CUDA events), the call on the device-resident collection, and end to end
    from pinned host arrays to host feature arrays."""
    import torch

    scorer = ads.PeakGroupScoring(ads.ScoringParameters(), verbose=False)
    scorer.score(dia, slib, cand)  # warm-up: IDF histogram of the library, scratch pool
    k_ms, call_s = [], []
    n = 0
    for _ in range(steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f = scorer.score(dia, slib, cand)
        call_s.append(time.perf_counter() - t0)
        k_ms.append(f.kernel_ms())
        n = len(f)
        del f
    nc = cand.copy_out(dict(zip(CAND_COLS, out_np)))
    arrs = tuple(o[:nc] for o in out_np)
    e2e_s = []
    d2h = 0
    for i in range(steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cc = ads.CandidateCollection.from_arrays(*arrs)
        f = scorer.score(dia, slib, cc)
        d = f.to_dict_arrays()
        dt = time.perf_counter() - t0
        d2h = len(f) * (2 * 8 + 4 * 41) + nc  # precursor_idx, rank, 41 features; found flags
        del cc, f, d
        if i > 0:
            e2e_s.append(dt)
    kms = statistics.median(k_ms)
    return {"metric": "candidates scored per second (PeakGroupScoring.score, 41 features)",
            "value": n / (kms / 1e3), "unit": "candidates/s", "candidates": int(n),
            "kernel_ms": kms, "call_ms": 1e3 * statistics.median(call_s),
            "call_value": n / statistics.median(call_s),
            "e2e": {"value": n / statistics.median(e2e_s), "unit": "candidates/s",
                    "h2d_bytes_per_step": int(nc * (5 * 8 + 4)), "d2h_bytes_per_step": int(d2h),
                    "path": "CandidateCollection.from_arrays(pinned host arrays) + "
                            "PeakGroupScoring.score + CandidateFeatureCollection.to_dict_arrays"},
            "timing": f"median of {steps} calls after one warm-up"}


def quant_figures(ads, dia, slib, cand, steps: int = 3) -> dict:
    """PeakGroupQuantification.quantify of the search's candidates: the kernel's device
    time and the whole call (kernel, copy-out, assembly of SpecLibFlatQuantified with
    its pass-through columns)."""
    import torch

    q = ads.PeakGroupQuantification(ads.QuantificationParameters(), verbose=False)
    q.quantify(dia, slib, cand)  # warm-up
    k_ms, call_s = [], []
    n_prec = n_frag = 0
    for _ in range(steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = q.quantify(dia, slib, cand)
        call_s.append(time.perf_counter() - t0)
        k_ms.append(r.kernel_ms())
        n_prec, n_frag = r.num_precursors, r.num_fragments
        # released before the next call, as a caller consuming one result at a time
        # would: its page-locked arrays go back to the host allocator's cache
        del r
    n = cand.size()
    kms = statistics.median(k_ms)
    return {"metric": "candidates quantified per second (PeakGroupQuantification.quantify)",
            "value": n / (kms / 1e3), "unit": "candidates/s", "candidates": int(n),
            "precursors_out": int(n_prec), "fragments_out": int(n_frag),
            "kernel_ms": kms, "call_ms": 1e3 * statistics.median(call_s),
            "call_value": n / statistics.median(call_s),
            "timing": f"median of {steps} calls after one warm-up; the call includes the "
                      f"device-to-host copy and the SpecLibFlatQuantified assembly"}


def quant_cpu_and_parity(ads, oracle, dsub, lsub, od, ol, la: dict, res: dict, n_threads: int,
                         steps: int = 3):
    """The oracle's PeakGroupQuantification on the CPU sample's candidates (timed), and
    the device's result for the same candidates against it, every column bit for bit."""
    cols = {k: res[k] for k in ("precursor_idx", "rank", "score", "cycle_center", "cycle_start",
                                "cycle_stop")}
    oracle.quantify(od, ol, cols, la, n_threads=n_threads)
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        ref = oracle.quantify(od, ol, cols, la, n_threads=n_threads)
        ts.append(time.perf_counter() - t0)
    nc = len(cols["rank"])
    cpu = {"value": nc / statistics.mean(ts), "unit": "candidates/s", "cores": n_threads,
           "kind": "port", "sample": f"the {nc} candidates of the search CPU sample, mean of "
                                     f"{steps} timed calls"}
    z = np.zeros(nc, np.uint64)
    cc = ads.CandidateCollection.from_arrays(cols["precursor_idx"], cols["rank"], cols["score"], z, z, z,
                                             cols["cycle_center"], cols["cycle_start"], cols["cycle_stop"])
    gp, gf = ads.PeakGroupQuantification(ads.QuantificationParameters(),
                                         verbose=False).quantify(dsub, lsub, cc).to_dict_arrays()
    diff = []
    for part, g, r in (("precursor", gp, ref[0]), ("fragment", gf, ref[1])):
        for k in r:
            a, b = np.asarray(g[k]), np.asarray(r[k])
            same = len(a) == len(b) and (np.array_equal(a.view(np.uint32), b.view(np.uint32))
                                         if a.dtype == np.float32 else np.array_equal(a, b))
            if not same:
                diff.append(f"{part}.{k}")
    parity = {"candidates": int(nc), "precursors": int(len(ref[0]["precursor_idx"])),
              "fragments": int(len(ref[1]["mz"])), "bit_identical": not diff, "columns_differing": diff}
    return cpu, parity


def scoring_cpu_and_parity(ads, oracle, host: dict, sub: dict, od, ol, res: dict, n_threads: int,
                           local_rank: int, steps: int = 3):
    """The oracle's PeakGroupScoring on the CPU sample's candidates (timed), and the
    device's features of the same candidates against it (correctly rounded logs:
    every feature bit for bit)."""
    la = sub_library_arrays(sub)
    oracle.lib_set_scoring(ol, la["precursor_naa"], la["fragment_mz_library"])
    cols = {k: res[k] for k in ("precursor_idx", "rank", "score", "cycle_center", "cycle_start",
                                "cycle_stop")}
    oracle.score(od, ol, cols, n_threads=n_threads)
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        oracle.score(od, ol, cols, n_threads=n_threads)
        ts.append(time.perf_counter() - t0)
    nc = len(cols["rank"])
    cpu = {"value": nc / statistics.mean(ts), "unit": "candidates/s", "cores": n_threads,
           "kind": "port", "sample": f"the {nc} candidates of the search CPU sample, mean of "
                                     f"{steps} timed calls"}
    ref = oracle.score(od, ol, cols, log_mode=oracle.LOG_RN, n_threads=n_threads)
    kw = dict(la)
    tol = kw.pop("precursor_rt_tolerance", None)
    dsub = ads.DIAData.from_arrays(*(host[k] for k in RUN_KEYS), host["cycle"], device=local_rank)
    lsub = ads.SpecLibFlat.from_arrays(**kw, precursor_rt_tolerance=tol, device=local_rank)
    z = np.zeros(nc, np.uint64)
    cc = ads.CandidateCollection.from_arrays(cols["precursor_idx"], cols["rank"], cols["score"], z, z, z,
                                             cols["cycle_center"], cols["cycle_start"], cols["cycle_stop"])
    got = ads.PeakGroupScoring(ads.ScoringParameters(), verbose=False).score(dsub, lsub, cc).to_dict_arrays()
    same_rows = len(got["rank"]) == len(ref["rank"]) and all(
        np.array_equal(got[k], ref[k]) for k in ("precursor_idx", "rank"))
    diff = [k for k in oracle.FEATURE_NAMES
            if not same_rows or not np.array_equal(got[k].view(np.uint32), ref[k].view(np.uint32))]
    parity = {"candidates": int(nc), "rows_identical": bool(same_rows),
              "features_bit_identical": len(diff) == 0, "features_differing": diff}
    del cc
    return cpu, parity, (dsub, lsub, la)


def oracle_setup(host: dict, sub: dict, n_threads: int):
    import oracle

    od = oracle.Dia(**{k: host[k] for k in RUN_KEYS}, n_threads=n_threads)
    ol = oracle.Lib(sub["precursor_idx"], sub["precursor_mz"], sub["precursor_rt"],
                    sub["flat_frag_start_idx"], sub["flat_frag_stop_idx"], sub["fragment_mz"],
                    sub["fragment_intensity"], sub["fragment_number"], sub["fragment_type"])
    tol = None
    if "rt_tolerance" in sub:
        tol = np.asarray(sub["rt_tolerance"], np.float32)[ol.sorted_order]
    return od, ol, tol


def time_oracle(od, ol, tol, params, n_threads, steps, warmup):
    import oracle

    p = oracle.Params(**params)
    res = None
    for _ in range(warmup):
        res = oracle.search(od, ol, p, rt_tolerance_per_precursor=tol, n_threads=n_threads)
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        res = oracle.search(od, ol, p, rt_tolerance_per_precursor=tol, n_threads=n_threads)
        ts.append(time.perf_counter() - t0)
    return ts, res


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def load_traffic(name: str, precision: str):
    """DRAM bytes of one search's search_kernel launches (all length classes) for this
    workload and precision, from the committed ncu summary (profiles/), or None."""
    key = f"traffic_bytes_per_search_{precision}:"
    for fname in (f"search_kernel_{name}_prof.md", f"search_kernel_{name}.md"):
        try:
            with open(os.path.join(ROOT, "profiles", fname)) as f:
                for line in f:
                    if line.strip().startswith(key):
                        return float(line.split(":", 1)[1].strip())
        except OSError:
            pass
    return None


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------- the line's config

def workload_text(cfg) -> str:
    return (f"{cfg.name}: {cfg.n_cycles} cycles x {cfg.n_windows} MS2 windows of {cfg.window_width} Th, "
            f"{cfg.peaks_per_spectrum} peaks/spectrum, {cfg.n_precursors} precursors x "
            f"{cfg.frag_min}-{cfg.frag_max} fragments"
            + (f" ({int(cfg.decoy_fraction * 100)}% decoys)" if cfg.decoy_fraction else ""))


def bench_config(cfg, precision: str, world: int) -> dict:
    """The ``config`` object of the JSON line; both arms print the same one."""
    compared = ("bf16 storage (f32 arithmetic) against the plain f32 path on the same data "
                "and settings" if precision == "bf16" else "plain f32")
    return {"workload": workload_text(cfg), "params": cfg.params_dict(),
            "rt_tolerance": ("per precursor, uniform %g-%g s" % cfg.rt_half_window
                             if cfg.per_precursor_tolerance else "%g s" % cfg.rt_half_window[1]),
            "precision": compared,
            "l2": "inputs larger than L2 (resident run of ~0.9-4 G peaks), no flush",
            "parallelism": f"replicated run, {world} library shard(s)"}


# ------------------------------------------------------------- reference arm

def run_reference(args, rank, world):
    if rank != 0:
        return
    import torch

    device = "cuda:0"
    cfg, lib, run = make_device_workload(args.workload, device)
    precision = args.precision or cfg.precision
    host, sub, (w0, w1) = window_subset(cfg, run, lib, sample_windows(cfg, args.cpu_windows))
    del run
    torch.cuda.empty_cache()
    n = cpu_threads()
    od, ol, tol = oracle_setup(host, sub, n)
    ts, res = time_oracle(od, ol, tol, cfg.params_dict(), n, args.steps, args.warmup)
    P = len(sub["precursor_idx"])
    mean = statistics.mean(ts)
    value = P / mean
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "precursors/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": mean * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded, generated on the device)",
        "config": bench_config(cfg, precision, world),
        "cpu_baseline": {"value": value, "unit": "precursors/s", "cores": n, "kind": "port",
                         "sample": sample_text(cfg, sub, host, w0, w1, args.steps),
                         "cpu_model": cpu_model()},
        "e2e": {"value": value, "unit": "precursors/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "candidates_per_step": int(len(res["rank"])),
        "reference_note": "the reference crate is Rust and cannot be built here (no cargo); its scalar "
                          "path (the only one it has on x86-64, f32) is timed as the C++ restatement "
                          "in oracle/ with all host threads",
    }
    print(json.dumps(line), flush=True)


def sample_text(cfg, sub, host, w0, w1, n_timed) -> str:
    return (f"{len(sub['precursor_idx'])} of the {cfg.n_precursors} precursors: those whose m/z lies "
            f"strictly inside MS2 windows {w0}-{w1} ({w1 - w0 + 1} of {cfg.n_windows}), searched against "
            f"those windows' {len(host['peak_mz'])} peaks (the same candidates as in the full search); "
            f"precursors/s is the sample's precursors over the mean of {n_timed} timed searches")


# ------------------------------------------------------------------ our arm

def timed_search(ads, params, precision, dia, slib, args, local_rank, dist, tune: bool):
    """One precision's timed region: W warm-up searches, then K searches (graph
    replays by default) bracketed by a barrier and a synchronize, timed with CUDA
    events on the selection's stream; then a second, directly enqueued pass for the
    stage times.  Returns the figures and the collection of the last search."""
    import torch

    device = f"cuda:{local_rank}"
    sel = ads.PeakGroupSelection(params, verbose=False, device=local_rank, time_stages=True,
                                 precision=precision, use_graph=args.graph,
                                 warps_per_block=args.warps_per_block,
                                 cycles_per_lane=args.cycles_per_lane,
                                 blocks_per_sm=args.blocks_per_sm, gather_mode=args.gather_mode)
    tuned = sel.autotune(dia, slib) if tune else None
    sel_opts = ((tuned["warps_per_block"], tuned["cycles_per_lane"]) if tuned
                else (args.warps_per_block, args.cycles_per_lane))
    cand = sel.new_candidates()
    stream = torch.cuda.ExternalStream(sel.stream, device=device)
    for _ in range(args.warmup):
        sel.search_into(dia, slib, cand)
    n_cand = cand.size()
    try:
        sel.stage_times()  # discard warm-up stage timings
    except ValueError:  # graph replays record none
        pass
    launches = sel.last_launches
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if dist:
        import torch.distributed as td

        td.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            sel.search_into(dia, slib, cand)
        ev1.record(stream)
        torch.cuda.synchronize()
    if dist:
        td.barrier()
    ms = ev0.elapsed_time(ev1)
    if cand.size() != n_cand:
        raise RuntimeError("candidate count changed between searches")
    if not args.graph:
        st = sel.stage_times()
    else:
        # graph replays record no stage events: time the stages on a second pass of
        # the same searches enqueued directly
        sel_st = ads.PeakGroupSelection(params, verbose=False, device=local_rank, time_stages=True,
                                        precision=precision, warps_per_block=sel_opts[0],
                                        cycles_per_lane=sel_opts[1], blocks_per_sm=args.blocks_per_sm,
                                        gather_mode=args.gather_mode)
        cand_st = sel_st.new_candidates()
        for _ in range(args.warmup):
            sel_st.search_into(dia, slib, cand_st)
        cand_st.size()
        sel_st.stage_times()
        for _ in range(args.steps):
            sel_st.search_into(dia, slib, cand_st)
        cand_st.size()
        st = sel_st.stage_times()
        del cand_st, sel_st
    ms_t = torch.tensor([ms], device=device, dtype=torch.float64)
    if dist:
        td.all_reduce(ms_t, op=td.ReduceOp.MAX)
    return {"ms": float(ms_t.item()), "stages": st, "tuned": tuned, "opts": sel_opts,
            "launches": launches, "n_cand": n_cand, "clocks": clk, "sel": sel, "cand": cand,
            "kernel": sel.kernel()}


def e2e_search(ads, params, precision, dia, lib_np, n_cand, steps, local_rank, dist):
    """End to end through the public API with pinned host buffers:
    SpecLibFlat.from_arrays (H2D of the library) + search + to_arrays(out=pinned)."""
    import torch

    device = f"cuda:{local_rank}"
    cap = max(n_cand, 1)
    out_t = [torch.empty(cap, dtype=torch.float32 if i == 2 else torch.uint64).pin_memory() for i in range(9)]
    out_np = tuple(t.numpy() for t in out_t)
    sel_e2e = ads.PeakGroupSelection(params, verbose=False, device=local_rank, precision=precision)
    # what SpecLibFlat.from_arrays uploads (the arrays the reference's other columns
    # name are kept on the host); fragment_mz_library only when it is its own array
    copied = ["precursor_idx", "precursor_mz", "precursor_rt", "precursor_naa", "flat_frag_start_idx",
              "flat_frag_stop_idx", "fragment_mz", "fragment_intensity", "fragment_number",
              "fragment_type", "precursor_rt_tolerance"]
    h2d = sum(lib_np[k].nbytes for k in copied if k in lib_np)
    if lib_np["fragment_mz_library"].ctypes.data != lib_np["fragment_mz"].ctypes.data:
        h2d += lib_np["fragment_mz_library"].nbytes
    times = []
    d2h = 0
    for i in range(steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        l2 = ads.SpecLibFlat.from_arrays(**lib_np, device=local_rank)
        c2 = sel_e2e.search(dia, l2)
        arrs = c2.to_arrays(out=out_np)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        d2h = len(arrs[0]) * (5 * 8 + 4)
        del l2, c2
        if i > 0:  # first call warms up allocations
            times.append(dt)
    # median: one step is tens of milliseconds of host work and copies, whose outliers
    # (page faults, another process's transfers) say nothing about the engine
    t = torch.tensor([statistics.median(times)], device=device, dtype=torch.float64)
    if dist:
        import torch.distributed as td

        td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item()), int(h2d), int(d2h), out_np


def e2e_stream(ads, params, precision, dia, lib_np, n_cand, steps, local_rank, dist, h2d):
    """End to end through the public API with the steps overlapped, as a caller
    streaming libraries through one selection would run it: step i uploads its library
    (SpecLibFlat.from_arrays of pinned host arrays) and enqueues its search
    (PeakGroupSelection.search_into) while step i-1's search runs, then reads step i-1's
    candidates back (DeviceCandidates.copy_out into pinned arrays) while step i's runs;
    two candidate collections alternate.  Every step's upload, search and read-back
    lies inside the timed region (wall clock from the first upload to the last
    read-back, over the steps), which follows one untimed pass of the same length.  The
    libraries are released after each pass."""
    import torch

    device = f"cuda:{local_rank}"
    cap = max(n_cand, 1)
    outs = [{c: torch.empty(cap, dtype=torch.float32 if c == "score" else torch.uint64).pin_memory().numpy()
             for c in CAND_COLS} for _ in range(2)]
    sel = ads.PeakGroupSelection(params, verbose=False, device=local_rank, precision=precision)
    cands = [sel.new_candidates(), sel.new_candidates()]

    def run(n_steps):
        libs, d2h = [], 0
        for i in range(n_steps + 1):
            if i < n_steps:
                lib = ads.SpecLibFlat.from_arrays(**lib_np, device=local_rank)
                libs.append(lib)
                sel.search_into(dia, lib, cands[i % 2])
            if i >= 1:
                n = cands[(i - 1) % 2].copy_out(outs[(i - 1) % 2])
                d2h = n * (5 * 8 + 4)  # five u64 columns and the f32 score (scan_* are zero)
        return libs, d2h

    # an untimed pass of the same length first: it sizes the selection's and the
    # collections' buffers and grows the device memory pool to hold a pass's libraries
    # (the first pass at cfg4 took up to 0.8 s in one allocation; later passes reuse)
    warm, _ = run(steps)
    del warm
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    libs, d2h = run(steps)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    del libs
    t = torch.tensor([dt * 1e3 / steps], device=device, dtype=torch.float64)
    if dist:
        import torch.distributed as td

        td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item()) / 1e3, int(h2d), int(d2h)


def search_roofline(stats, stages, precision, kernel, P, nf_raw, n_cand, ms_per_step, peak, peak_kind,
                    sm_max_mhz, traffic):
    """Roofline of search_kernel: algorithmic gather bytes (4 per CSR offset, 2 per
    cycle and s_I per intensity of every accumulated entry, counted by the kernel's
    statistics pass) over its CUDA-event time per launch."""
    n_searches = max(stages["searches"], 1)
    search_ms = stages["search_ms"] / n_searches
    s_i = 2 if precision == "bf16" else 4
    gather_bytes = 4 * stats["bins_plus_one"] + (2 + s_i) * stats["entries_accumulated"]
    path_bytes = 8 * P + 8 * nf_raw + gather_bytes + 68 * n_cand
    h = len(kernel) // 2
    dense_flops = stats.get("xic_cells", 0) * (3 * h + 2)
    fp32_peak = 148 * 128 * 2 * (sm_max_mhz or 1965) * 1e6 / 1e12
    achieved = gather_bytes / (search_ms / 1e3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "peak_source": f"{peak_kind} hbm_gbs",
            "kernel": "search_kernel", "bytes_per_intensity": s_i,
            "launch_unit": "one search: the search_kernel launches of its RT-window length "
                           "classes together (per_launch fields are per search)",
            "traffic_source": "ncu DRAM bytes of a profiling-sized case at the same densities, "
                              "scaled by the precursor count (profiles/)",
            "algorithmic_bytes_per_launch": gather_bytes,
            "kernel_ms_per_launch": search_ms,
            "path_bytes_per_step": path_bytes,
            "path_gbs": path_bytes / (ms_per_step / 1e3) / 1e9,
            # the stencil and score work: XIC cells x (3h + 2) flops, h the kernel's
            # half width; against the FP32 CUDA-core peak (148 SMs x 128 lanes x 2 x
            # the max SM clock)
            "dense_flops_per_launch": dense_flops,
            "dense_tflops": dense_flops / (search_ms / 1e3) / 1e12,
            "fp32_peak_tflops_nominal": fp32_peak,
            "stage_ms": {"prep": stages["prep_ms"] / n_searches, "search": search_ms,
                         "compaction": stages["compaction_ms"] / n_searches}}


def merge_clocks(*samplers) -> dict:
    samples = [s for c in samplers for s in c.samples]
    out = samplers[0].summary()
    if samplers[0].nv is not None and samples:
        merged = ClockSampler.__new__(ClockSampler)
        merged.samples, merged.nv, merged.max_mhz = samples, samplers[0].nv, samplers[0].max_mhz
        out = merged.summary()
    return out


def sample_parity_fp32(got: dict, mask, res: dict) -> dict:
    same = {k: bool(np.array_equal(got[k][mask], res[k])) for k in
            ("precursor_idx", "rank", "cycle_center", "cycle_start", "cycle_stop")}
    rel = 0.0
    if mask.sum() == len(res["score"]) and len(res["score"]):
        rel = float(np.max(np.abs(got["score"][mask].astype(np.float64) - res["score"]) /
                           np.maximum(np.abs(res["score"]).astype(np.float64), 1e-30)))
    return {"candidates": int(len(res["rank"])),
            "indices_identical": all(same.values()) and int(mask.sum()) == len(res["rank"]),
            "max_score_rel_err_vs_glibc_logf": rel}


CAND_NAMES = ("precursor_idx", "rank", "score", "sc", "ss", "sp", "cycle_center", "cycle_start",
              "cycle_stop")


def run_ours(args, rank, world, local_rank):
    import torch

    import alphadia_search_rs_b200 as ads

    device = f"cuda:{local_rank}"
    torch.cuda.set_device(local_rank)
    dist = world > 1
    t_setup = time.perf_counter()
    cfg, lib, run = make_device_workload(args.workload, device, lib_seed_offset=rank)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_setup
    t0 = time.perf_counter()
    dia = ads.DIAData.from_arrays(*(run[k] for k in RUN_KEYS), run["cycle"], device=local_rank)
    t_dia = time.perf_counter() - t0
    ltens = library_tensors(lib, device)
    t0 = time.perf_counter()
    slib = ads.SpecLibFlat.from_arrays(**ltens, device=local_rank)
    t_lib = time.perf_counter() - t0
    P = slib.num_precursors
    params = ads.SelectionParameters()
    params.update(cfg.params_dict())
    precision = args.precision or cfg.precision
    bf16 = precision == "bf16"
    # the plain FP32 path on the same data and settings (cfg3 -> cfg2's search)
    arms = ["bf16", "fp32"] if bf16 else ["fp32"]

    # counters pass (untimed): algorithmic bytes of the gather; the full result of
    # each precision is kept for the parity check on the CPU sample
    keep_inputs = rank == 0 and world == 1 and not args.no_cpu_baseline
    stats, full = None, {}
    for prec in arms:
        sel_stats = ads.PeakGroupSelection(params, verbose=False, device=local_rank, precision=prec)
        sel_stats.enable_stats(True)
        cand_full = sel_stats.search(dia, slib)
        if stats is None:
            stats = sel_stats.last_stats()
        if keep_inputs:
            full[prec] = dict(zip(CAND_NAMES, cand_full.to_arrays()))
        del cand_full, sel_stats
    n_peaks_total = int(run["peak_mz"].numel())
    nf_raw = int(lib["fragment_mz"].numel())
    if not keep_inputs:  # the device copies inside DIAData/SpecLibFlat are all the search needs
        lib_host_src = host_copies(ltens, lambda v: v.cpu())
        del run, ltens
        ltens = lib_host_src
        torch.cuda.empty_cache()

    tune = args.autotune if args.autotune is not None else cfg.per_precursor_tolerance
    timed = {prec: timed_search(ads, params, prec, dia, slib, args, local_rank, dist, tune)
             for prec in arms}
    head = timed[arms[0]]
    value = P * world * args.steps / (head["ms"] / 1e3)

    lib_host = host_copies(ltens, lambda v: v.cpu().pin_memory())
    lib_np = {k: v.numpy() for k, v in lib_host.items()}
    e2e = {prec: e2e_search(ads, params, prec, dia, lib_np, timed[prec]["n_cand"], args.e2e_steps,
                            local_rank, dist) for prec in arms}
    out_np = e2e[arms[0]][3]
    e2e_s = {prec: e2e_stream(ads, params, prec, dia, lib_np, timed[prec]["n_cand"], args.e2e_steps,
                              local_rank, dist, e2e[prec][1]) for prec in arms}

    if rank != 0:
        return

    peak, peak_kind = measured_peak()
    clocks = merge_clocks(*(timed[p]["clocks"] for p in arms))
    roof = {prec: search_roofline(stats, timed[prec]["stages"], prec, timed[prec]["kernel"], P, nf_raw,
                                  timed[prec]["n_cand"], timed[prec]["ms"] / args.steps, peak, peak_kind,
                                  clocks.get("sm_max_mhz"),
                                  load_traffic(cfg.name, prec))
            for prec in arms}

    # ---- CPU baseline (oracle port on the host cores, bounded sample) and the
    #      parity of the GPU results for the same precursors
    cpu = parity = None
    scoring = quant = None
    cand = head["cand"]
    if world == 1 and not args.no_scoring:
        scoring = scoring_figures(ads, dia, slib, cand, out_np)
        quant = quant_figures(ads, dia, slib, cand)
    if world == 1 and not args.no_cpu_baseline:
        import oracle

        host, sub, (w0, w1) = window_subset(cfg, run, lib, sample_windows(cfg, args.cpu_windows))
        n = cpu_threads()
        od, ol, tol = oracle_setup(host, sub, n)
        ts, res = time_oracle(od, ol, tol, cfg.params_dict(), n, steps=3, warmup=1)
        Ps = len(sub["precursor_idx"])
        cpu = {"value": Ps / statistics.mean(ts), "unit": "precursors/s", "cores": n, "kind": "port",
               "sample": sample_text(cfg, sub, host, w0, w1, 3), "cpu_model": cpu_model()}
        parity = {"precursors": int(Ps)}
        got32 = full["fp32"]
        mask = np.isin(got32["precursor_idx"], sub["precursor_idx"])
        parity["fp32"] = sample_parity_fp32(got32, mask, res)
        if bf16:
            # BF16 storage is compared with the FP64 oracle: top-K cycle agreement and
            # relative score error (against max(|s64|, 1e-3 * the precursor's largest |s64|))
            ref64 = oracle.search(od, ol, oracle.Params(**cfg.params_dict()),
                                  rt_tolerance_per_precursor=tol, log_mode=oracle.LOG_RN,
                                  precision=1, n_threads=n)
            g16 = full["bf16"]
            m16 = np.isin(g16["precursor_idx"], sub["precursor_idx"])
            agree, errs = bf16_agreement({k: v[m16] for k, v in g16.items()}, ref64)
            parity["bf16"] = {"candidates_fp64_oracle": int(len(ref64["rank"])),
                              "topk_cycle_agreement_vs_fp64": agree,
                              "score_rel_err_vs_fp64_max": float(errs.max()),
                              "score_rel_err_vs_fp64_p99": float(np.quantile(errs, 0.99)),
                              "score_rel_err_vs_fp64_median": float(np.median(errs)),
                              "bound_note": "target 1e-3 relative: met by p99 and median; the max "
                                            "is bounded by bfloat16's u = 2^-8 = 3.9e-3"}
        if scoring is not None:
            scoring["cpu_baseline"], scoring["parity_sample"], (dsub, lsub, la_sub) = \
                scoring_cpu_and_parity(ads, oracle, host, sub, od, ol, res, n, local_rank)
            quant["cpu_baseline"], quant["parity_sample"] = quant_cpu_and_parity(
                ads, oracle, dsub, lsub, od, ol, la_sub, res, n)
            del dsub, lsub

    def launch_info(t):
        return {"cuda_graph": bool(args.graph), "autotuned": t["tuned"],
                "gather_mode": args.gather_mode,
                "warps_per_block": t["opts"][0] or "default",
                "cycles_per_lane": t["opts"][1] or "length classes"}

    e_head, es_head = e2e[arms[0]], e2e_s[arms[0]]
    stream_path = ("per step: SpecLibFlat.from_arrays(pinned host arrays) + "
                   "PeakGroupSelection.search_into + DeviceCandidates.copy_out(pinned), steps "
                   "overlapped (step i's upload and search enqueued before step i-1's read-back)")
    serial_path = ("per step, one after the other: SpecLibFlat.from_arrays(pinned host arrays) + "
                   "PeakGroupSelection.search + CandidateCollection.to_arrays(out=pinned)")
    line = {
        "metric": METRIC, "value": value, "unit": "precursors/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16-storage/f32-compute" if bf16 else "f32",
        "data": "synthetic (seeded, generated on the device)",
        "config": bench_config(cfg, precision, world),
        "e2e": {"value": P * world / es_head[0], "unit": "precursors/s", "h2d_bytes_per_step": es_head[1],
                "d2h_bytes_per_step": es_head[2], "path": stream_path,
                "serial": {"value": P * world / e_head[0], "unit": "precursors/s",
                           "h2d_bytes_per_step": e_head[1], "d2h_bytes_per_step": e_head[2],
                           "path": serial_path}},
        "gpu_launches": int(head["launches"] * args.steps),
        "roofline": roof[arms[0]],
    }
    if bf16:
        t32, e32, es32 = timed["fp32"], e2e["fp32"], e2e_s["fp32"]
        v32 = P * world * args.steps / (t32["ms"] / 1e3)
        line["bf16_vs_fp32"] = value / v32
        line["bf16_vs_fp32_e2e"] = es32[0] / es_head[0]
        line["fp32_companion"] = {
            "what": "the plain FP32 GPU path (bit-exact indices) on the same run, library and "
                    "settings, timed the same way in the same process (cfg3's data searched as cfg2)",
            "value": v32, "unit": "precursors/s", "ms_per_step": t32["ms"] / args.steps,
            "e2e": {"value": P * world / es32[0], "unit": "precursors/s", "h2d_bytes_per_step": es32[1],
                    "d2h_bytes_per_step": es32[2],
                    "serial": {"value": P * world / e32[0], "unit": "precursors/s"}},
            "gpu_launches": int(t32["launches"] * args.steps),
            "roofline": roof["fp32"], "launch": launch_info(t32),
            "candidates_per_step": int(t32["n_cand"])}
    line.update({
        "cpu_baseline": cpu,
        "parity_sample": parity,
        "launch": launch_info(head),
        "workload_stats": {"peaks": n_peaks_total, "candidates_per_step": int(head["n_cand"]),
                           "precursors_per_gpu": int(P),
                           "resident_run_gb": dia.device_bytes() / 1e9,
                           "resident_run_gb_bf16_only": (dia.device_bytes() -
                                                         4 * int(n_peaks_total)) / 1e9},
        "scoring": scoring,
        "quantification": quant,
        "clocks": clocks,
        "setup_s": {"generate": t_gen, "dia_build": t_dia, "lib_build": t_lib},
        "counters": stats,
    })
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus and world > 1:
        print(f"WORLD_SIZE={world} but --gpus {args.gpus}", file=sys.stderr)
    if world > 1:
        import datetime

        import torch
        import torch.distributed as td

        torch.cuda.set_device(local_rank)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                              device_id=torch.device(f"cuda:{local_rank}"))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as td

            td.destroy_process_group()


if __name__ == "__main__":
    main()
