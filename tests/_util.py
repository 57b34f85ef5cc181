"""Shared helpers for the parity tests (runs the product and the oracle on the
same inputs).  Not a test module."""
from __future__ import annotations

import numpy as np

import oracle
from alphadia_search_rs_b200 import (CandidateCollection, DIAData, PeakGroupSelection,
                                     SelectionParameters, SpecLibFlat, synth)

COLS = ("precursor_idx", "rank", "score", "scan_center", "scan_start", "scan_stop",
        "cycle_center", "cycle_start", "cycle_stop")
INDEX_COLS = ("precursor_idx", "rank", "cycle_center", "cycle_start", "cycle_stop")
# scores of the f32 path vs the reference (glibc logf): relative tolerance
SCORE_RTOL = 1e-5

RUN_KEYS = ("spectrum_delta_scan_idx", "isolation_lower_mz", "isolation_upper_mz",
            "spectrum_peak_start_idx", "spectrum_peak_stop_idx", "spectrum_cycle_idx",
            "spectrum_rt", "peak_mz", "peak_intensity")


def params_from(d: dict) -> SelectionParameters:
    p = SelectionParameters()
    p.update(d)
    return p


def oracle_inputs(run: dict, la: dict, n_threads=0):
    od = oracle.Dia(**{k: run[k] for k in RUN_KEYS}, n_threads=n_threads)
    ol = oracle.Lib(la["precursor_idx"], la["precursor_mz"], la["precursor_rt"],
                    la["flat_frag_start_idx"], la["flat_frag_stop_idx"], la["fragment_mz"],
                    la["fragment_intensity"], la["fragment_number"], la["fragment_type"])
    tol = None
    if "precursor_rt_tolerance" in la:
        tol = np.asarray(la["precursor_rt_tolerance"], np.float32)[ol.sorted_order]
    return od, ol, tol


def oracle_search(run: dict, la: dict, params: dict, log_mode=oracle.LOG_GLIBC, od=None, ol=None,
                  tol=None, subset=None):
    if od is None:
        od, ol, tol = oracle_inputs(run, la)
    r = oracle.search(od, ol, oracle.Params(**params), rt_tolerance_per_precursor=tol,
                      log_mode=log_mode, subset=subset)
    n = len(r["rank"])
    out = dict(precursor_idx=r["precursor_idx"], rank=r["rank"], score=r["score"],
               scan_center=np.zeros(n, np.uint64), scan_start=np.zeros(n, np.uint64),
               scan_stop=np.zeros(n, np.uint64), cycle_center=r["cycle_center"],
               cycle_start=r["cycle_start"], cycle_stop=r["cycle_stop"])
    return out


def product_search(run: dict, la: dict, params: dict, **engine):
    dia = DIAData.from_arrays(*(run[k] for k in RUN_KEYS), run["cycle"])
    lib_kw = dict(la)
    tol = lib_kw.pop("precursor_rt_tolerance", None)
    lib = SpecLibFlat.from_arrays(**lib_kw, precursor_rt_tolerance=tol)
    sel = PeakGroupSelection(params_from(params), verbose=False, **engine)
    cand = sel.search(dia, lib)
    arrs = dict(zip(COLS, cand.to_arrays()))
    return arrs, dia, lib, sel


def assert_candidates_equal(got: dict, ref: dict, exact_scores: bool, where=""):
    n_got, n_ref = len(got["rank"]), len(ref["rank"])
    if n_got != n_ref:
        # locate the first differing precursor for the message
        m = min(n_got, n_ref)
        bad = np.nonzero(got["precursor_idx"][:m] != ref["precursor_idx"][:m])[0]
        first = int(bad[0]) if len(bad) else m
        raise AssertionError(f"{where}: {n_got} candidates vs {n_ref} in the reference; first "
                             f"difference at row {first}")
    for c in INDEX_COLS + ("scan_center", "scan_start", "scan_stop"):
        g, r = np.asarray(got[c]), np.asarray(ref[c])
        assert g.dtype == np.uint64, (c, g.dtype)
        if not np.array_equal(g, r):
            i = int(np.nonzero(g != r)[0][0])
            raise AssertionError(f"{where}: column {c} differs at row {i}: {g[i]} vs {r[i]} "
                                 f"(precursor {ref['precursor_idx'][i]})")
    gs, rs = np.asarray(got["score"]), np.asarray(ref["score"])
    assert gs.dtype == np.float32
    if exact_scores:
        if not np.array_equal(gs.view(np.uint32), rs.view(np.uint32)):
            i = int(np.nonzero(gs.view(np.uint32) != rs.view(np.uint32))[0][0])
            raise AssertionError(f"{where}: score bits differ at row {i}: {gs[i]!r} vs {rs[i]!r}")
    else:
        rel = np.abs(gs.astype(np.float64) - rs) / np.maximum(np.abs(rs.astype(np.float64)), 1e-30)
        assert float(rel.max(initial=0.0)) <= SCORE_RTOL, f"{where}: max rel score err {rel.max()}"


def edge_case_workload():
    """Hand-built run + library exercising the corners of the reference path."""
    rng = np.random.default_rng(5)
    W = 4  # delta_scan_idx 0..4, window 3 has no spectra (empty observation)
    n_cyc = 100
    iso = {1: (400.0, 425.0), 2: (425.0, 450.0), 4: (430.0, 440.0)}
    spectra = []
    for c in range(n_cyc):
        spectra.append((0, -1.0, -1.0, c))
        for w in (1, 2, 4):
            spectra.append((w, iso[w][0], iso[w][1], c))
    # spectra of cycle 50 listed out of cycle order (the builder must keep
    # (bin, cycle) order with ties in visit order)
    i50 = [i for i, s in enumerate(spectra) if s[3] == 50]
    i60 = [i for i, s in enumerate(spectra) if s[3] == 60]
    for a, b in zip(i50, i60):
        spectra[a], spectra[b] = spectra[b], spectra[a]
    frag_mz = np.array([300.0, 350.0, 500.0, 650.0, 800.0, 820.0, 900.5, 1000.25], np.float32)
    peaks_mz, peaks_int, starts, stops = [], [], [], []
    for (w, lo, hi, c) in spectra:
        starts.append(sum(len(p) for p in peaks_mz))
        mz = list(rng.uniform(150, 1800, 60).astype(np.float32))
        it = list(rng.lognormal(8, 2, 60).astype(np.float32))
        if w == 0:  # MS1 with peaks: observation 0 is built like any other
            pass
        else:
            for k, f in enumerate(frag_mz):
                a = 5e4 * np.exp(-((c - 40 - 3 * k) ** 2) / 18.0)
                if a > 1.0:
                    mz.append(np.float32(f * (1 + 1e-6 * rng.normal())))
                    it.append(np.float32(a * rng.lognormal(0, 0.2)))
            if c in (19, 29):  # two peaks in one 1-ppm bin at a window's first cycle
                for f in frag_mz[:3]:
                    mz += [np.float32(f), np.float32(f * (1 + 1e-8))]
                    it += [np.float32(1000.0 + c), np.float32(7.0 + c)]
            if c % 7 == 0:  # zero-intensity peaks
                mz.append(np.float32(frag_mz[4]))
                it.append(np.float32(0.0))
        order = np.argsort(np.array(mz, np.float32), kind="stable")
        peaks_mz.append(np.array(mz, np.float32)[order])
        peaks_int.append(np.array(it, np.float32)[order])
        stops.append(starts[-1] + len(order))
    run = dict(
        spectrum_delta_scan_idx=np.array([s[0] for s in spectra], np.int64),
        isolation_lower_mz=np.array([s[1] for s in spectra], np.float32),
        isolation_upper_mz=np.array([s[2] for s in spectra], np.float32),
        spectrum_peak_start_idx=np.array(starts, np.int64),
        spectrum_peak_stop_idx=np.array(stops, np.int64),
        spectrum_cycle_idx=np.array([s[3] for s in spectra], np.int64),
        spectrum_rt=np.array([s[3] * 1.0 for s in spectra], np.float32),
        peak_mz=np.concatenate(peaks_mz), peak_intensity=np.concatenate(peaks_int),
        cycle=np.zeros((W + 1, 1, 1, 1), np.float32),
    )
    # library: (mz, rt, fragments as (mz, intensity, number, type))
    F = frag_mz
    prec = [
        (410.0, 50.0, [(f, 1.0 + i, 2, 98) for i, f in enumerate(F)]),        # window 1
        (425.0, 50.0, [(f, 2.0 + i, 3, 121) for i, f in enumerate(F)]),       # windows 1 and 2
        (435.0, 45.0, [(f, 3.0 + i, 4, 98) for i, f in enumerate(F)]),        # windows 2 and 4
        (999.0, 50.0, [(f, 1.0, 2, 98) for f in F]),                          # no window
        (410.0, 900.0, [(f, 1.0, 2, 98) for f in F]),                         # RT outside the run
        (410.0, 50.0, []),                                                    # no fragments
        (410.0, 50.0, [(f, 0.0, 2, 98) for f in F]),                          # all intensities 0
        (410.0, 50.0, [(f, 1.0 + i, 1, 121) for i, f in enumerate(F)]),       # all y1: filtered
        (410.0, 50.0, [(f, 5.0 if i % 2 else 1.0 + i, 2, 98) for i, f in enumerate(F)] * 2),  # ties, >top_k
        (410.0, 60.0, [(F[i], 1.0 + i, 2, 98) for i in (7, 0, 5, 2, 1)]),    # unsorted m/z
        (410.0, 3.0, [(f, 1.0 + i, 2, 98) for i, f in enumerate(F)]),         # window clipped at 0
        (410.0, 97.0, [(f, 1.0 + i, 2, 98) for i, f in enumerate(F)]),        # clipped at the end
        (410.0, 50.0, [(f, 1.0 + i, 2, 98) for i, f in enumerate(F)]),        # duplicate idx below
    ]
    pidx = [7, 3, 11, 5, 1, 9, 2, 8, 0, 4, 10, 6, 7]
    frag_rows, starts, stops = [], [], []
    for (_, _, frs) in prec:
        starts.append(len(frag_rows))
        frag_rows += frs
        stops.append(len(frag_rows))
    fr = np.array(frag_rows, dtype=object) if frag_rows else np.zeros((0, 4))
    NF = len(frag_rows)
    la = dict(
        precursor_idx=np.array(pidx, np.uint64),
        precursor_mz_library=np.array([p[0] for p in prec], np.float32),
        precursor_mz=np.array([p[0] for p in prec], np.float32),
        precursor_rt_library=np.array([p[1] for p in prec], np.float32),
        precursor_rt=np.array([p[1] for p in prec], np.float32),
        precursor_naa=np.full(len(prec), 9, np.uint8),
        flat_frag_start_idx=np.array(starts, np.uint64),
        flat_frag_stop_idx=np.array(stops, np.uint64),
        fragment_mz_library=np.array([r[0] for r in frag_rows], np.float32),
        fragment_mz=np.array([r[0] for r in frag_rows], np.float32),
        fragment_intensity=np.array([r[1] for r in frag_rows], np.float32),
        fragment_cardinality=np.ones(NF, np.uint8), fragment_charge=np.ones(NF, np.uint8),
        fragment_loss_type=np.zeros(NF, np.uint8),
        fragment_number=np.array([r[2] for r in frag_rows], np.uint8),
        fragment_position=np.ones(NF, np.uint8),
        fragment_type=np.array([r[3] for r in frag_rows], np.uint8),
    )
    del fr
    return run, la
