"""The oracle's PeakGroupQuantification (src/peak_group_quantification/mod.rs:49-168)
and SpecLibFlatQuantified assembly (src/speclib_flat_quantified/mod.rs:212-333).

The per-fragment values are recomputed here from the oracle's helpers on raw arrays
(dense XIC/m/z, mass errors, normalisation, median of the non-zero rows, correlation),
which the reference's own unit-test values pin (test_oracle_scoring_known_answers.py);
the assembly rules follow the reference's SpecLibFlatQuantified tests
(src/speclib_flat_quantified/tests.rs:29-157).  CPU only."""
import numpy as np
import pytest

import oracle
from alphadia_search_rs_b200 import synth

from _util import oracle_inputs, oracle_search


def _ndarray_row_sum(x: np.ndarray) -> np.float32:
    """ndarray's contiguous row sum (8 partial sums, pairwise combined, then the tail)."""
    x = np.asarray(x, np.float32)
    p = np.zeros(8, np.float32)
    i = 0
    while len(x) - i >= 8:
        for k in range(8):
            p[k] = np.float32(p[k] + x[i + k])
        i += 8
    acc = np.float32(0.0)
    for a, b in ((0, 4), (1, 5), (2, 6), (3, 7)):
        acc = np.float32(acc + np.float32(p[a] + p[b]))
    for k in range(i, len(x)):
        acc = np.float32(acc + x[k])
    return acc


@pytest.fixture(scope="module")
def tiny():
    cfg, lib, run = synth.make_workload("tiny", "numpy")
    la = synth.library_arrays(lib)
    rng = np.random.default_rng(4)
    la["precursor_naa"] = rng.integers(6, 40, len(la["precursor_idx"])).astype(np.uint8)
    la["fragment_cardinality"] = rng.integers(1, 3, len(la["fragment_mz"])).astype(np.uint8)
    la["fragment_position"] = rng.integers(0, 30, len(la["fragment_mz"])).astype(np.uint8)
    od, ol, tol = oracle_inputs(run, la)
    cand = oracle_search(run, la, cfg.params_dict(), oracle.LOG_RN, od, ol, tol)
    return cfg, run, la, od, ol, cand


def test_values_match_the_pinned_helpers(tiny):
    cfg, run, la, od, ol, cand = tiny
    prec, frag = oracle.quantify(od, ol, cand, la, tolerance_ppm=7.0, top_k_fragments=10000)
    order = np.asarray(ol.sorted_order)
    pos_of = {int(p): i for i, p in enumerate(np.asarray(la["precursor_idx"])[order])}
    fs_all, fe_all = la["flat_frag_start_idx"], la["flat_frag_stop_idx"]
    expect_f = {k: [] for k in ("row", "intensity", "mz_observed", "correlation_observed",
                                "mass_error_observed")}
    kept_candidates = []
    for q in range(len(cand["rank"])):
        i = pos_of[int(cand["precursor_idx"][q])]
        row = int(order[i])
        s, e = int(fs_all[row]), int(fe_all[row])
        keep = oracle.filter_sort_fragments(la["fragment_mz"][s:e], la["fragment_intensity"][s:e],
                                            la["fragment_number"][s:e], la["fragment_type"][s:e],
                                            True, True, 10000)
        fmz = la["fragment_mz"][s:e][keep]
        cs, ce = int(cand["cycle_start"][q]), int(cand["cycle_stop"][q])
        xic, mzo = oracle.sc_dense_xic_mz(od, la["precursor_mz"][row], cs, ce, 7.0, fmz)
        mz_obs, err = oracle.sc_fragment_mz_errors(mzo, xic, fmz)
        norm = oracle.sc_normalize_profiles(xic, 1)
        med = oracle.sc_median_axis0(norm, non_zero_only=True)
        obs = np.array([_ndarray_row_sum(r) for r in xic], np.float32)
        corr = np.array([oracle.sc_correlation(r, med) for r in norm], np.float32)
        ok = obs > 0
        if not ok.any():
            continue
        kept_candidates.append(q)
        expect_f["row"] += list(s + keep[ok])
        expect_f["intensity"] += list(obs[ok])
        expect_f["mz_observed"] += list(np.asarray(mz_obs, np.float32)[ok])
        expect_f["correlation_observed"] += list(corr[ok])
        expect_f["mass_error_observed"] += list(np.asarray(err, np.float32)[ok])
    assert len(kept_candidates) == len(prec["precursor_idx"]) > 0
    assert np.array_equal(frag["mz"], la["fragment_mz"][np.asarray(expect_f["row"], np.int64)])
    for k in ("intensity", "mz_observed", "correlation_observed", "mass_error_observed"):
        got = np.asarray(frag[k], np.float32).view(np.uint32)
        want = np.asarray(expect_f[k], np.float32).view(np.uint32)
        assert np.array_equal(got, want), k


def test_assembly_order_and_ranges(tiny):
    """Fragments stay in candidate order; precursors are sorted by precursor_idx with
    equal indices in candidate order; each precursor's range covers its fragments and
    the fragment precursor_idx / rank columns repeat the precursor's
    (src/speclib_flat_quantified/tests.rs:111-157)."""
    cfg, run, la, od, ol, cand = tiny
    prec, frag = oracle.quantify(od, ol, cand, la)
    P, NF = len(prec["precursor_idx"]), len(frag["mz"])
    assert np.all(np.diff(prec["precursor_idx"].astype(np.int64)) >= 0)
    assert int((prec["flat_frag_stop_idx"] - prec["flat_frag_start_idx"]).sum()) == NF
    for j in range(P):
        a, b = int(prec["flat_frag_start_idx"][j]), int(prec["flat_frag_stop_idx"][j])
        assert b > a
        assert np.all(frag["precursor_idx"][a:b] == prec["precursor_idx"][j])
        assert np.all(frag["rank"][a:b] == prec["rank"][j])
    # candidate order: the fragment ranges, read in start order, follow the candidates
    by_start = np.argsort(prec["flat_frag_start_idx"], kind="stable")
    assert np.all(np.diff(prec["flat_frag_start_idx"][by_start].astype(np.int64)) > 0)
    # equal precursor_idx (one precursor's candidates): ranks in candidate order
    for p in np.unique(prec["precursor_idx"]):
        sel = np.nonzero(prec["precursor_idx"] == p)[0]
        assert np.all(np.diff(prec["flat_frag_start_idx"][sel].astype(np.int64)) > 0)
    # pass-through columns
    rows = {int(p): i for i, p in enumerate(la["precursor_idx"])}
    for j in range(P):
        r = rows[int(prec["precursor_idx"][j])]
        assert prec["mz"][j] == la["precursor_mz"][r] and prec["naa"][j] == la["precursor_naa"][r]
    assert prec["rt_observed"].dtype == np.float32 and frag["position"].dtype == np.uint8


def test_dropped_candidates(tiny):
    """None in the reference: unknown precursor, empty cycle range, centre outside the
    range, no fragment with a positive observed intensity."""
    cfg, run, la, od, ol, cand = tiny
    base = {k: np.asarray(v)[:4].copy() for k, v in cand.items()}
    prec0, frag0 = oracle.quantify(od, ol, base, la)
    bad = {k: np.concatenate([v, v[:1], v[:1], v[:1]]) for k, v in base.items()}
    n = len(base["rank"])
    bad["precursor_idx"][n] = np.uint64(10**9)                     # not in the library
    bad["cycle_stop"][n + 1] = bad["cycle_start"][n + 1]           # zero cycles
    bad["cycle_center"][n + 2] = bad["cycle_stop"][n + 2]          # centre at the stop
    prec, frag = oracle.quantify(od, ol, bad, la)
    assert len(prec["precursor_idx"]) == len(prec0["precursor_idx"])
    assert len(frag["mz"]) == len(frag0["mz"])
    # a cycle range with no peaks at all (before any signal: cycles 0..1 of a precursor
    # whose fragments are absent there) drops the precursor when every row sums to 0
    empty = {k: np.asarray(v)[:1].copy() for k, v in base.items()}
    empty["cycle_start"][0], empty["cycle_stop"][0], empty["cycle_center"][0] = 0, 1, 0
    p1, f1 = oracle.quantify(od, ol, empty, la, tolerance_ppm=1e-6)
    assert len(p1["precursor_idx"]) == 0 and len(f1["mz"]) == 0


def test_top_k_and_tolerance_change_the_fragments(tiny):
    cfg, run, la, od, ol, cand = tiny
    p_all, f_all = oracle.quantify(od, ol, cand, la)
    p3, f3 = oracle.quantify(od, ol, cand, la, top_k_fragments=3)
    assert np.all(p3["flat_frag_stop_idx"] - p3["flat_frag_start_idx"] <= 3)
    assert len(f3["mz"]) < len(f_all["mz"])
    p0, f0 = oracle.quantify(od, ol, cand, la, top_k_fragments=0)
    assert len(p0["precursor_idx"]) == 0 and len(f0["mz"]) == 0


def test_empty_candidates(tiny):
    cfg, run, la, od, ol, cand = tiny
    prec, frag = oracle.quantify(od, ol, {k: np.asarray(v)[:0] for k, v in cand.items()}, la)
    assert set(prec) == set(oracle.QUANT_PRECURSOR_KEYS) and set(frag) == set(oracle.QUANT_FRAGMENT_KEYS)
    assert all(len(v) == 0 for v in prec.values()) and all(len(v) == 0 for v in frag.values())
