"""GPU parity of PeakGroupScoring (src/peak_group_scoring/mod.rs:42-101): the 41
candidate features computed on the device, through the C ABI, against the oracle's
restatement on the same candidates.

  * oracle with a correctly rounded logf / log10f (what the kernel computes): every
    row and every feature identical, bit for bit;
  * oracle with glibc logf (the reference's numerics on Linux): rows identical,
    features within FEATURE_RTOL relative (FEATURE_ATOL absolute near zero).
"""
import numpy as np
import pytest

import oracle
from alphadia_search_rs_b200 import (CandidateCollection, CandidateFeatureCollection, DIAData,
                                     PeakGroupScoring, PeakGroupSelection, ScoringParameters,
                                     SpecLibFlat, synth)

from _util import COLS, RUN_KEYS, edge_case_workload, oracle_inputs, params_from

pytestmark = pytest.mark.gpu

FEATURE_RTOL = 1e-5
FEATURE_ATOL = 1e-6


def scoring_library(la: dict, seed: int) -> dict:
    """The synthetic library with per-precursor amino-acid counts and library
    fragment m/z a few ppm away from the searched (calibrated) m/z, so that the IDF
    bins and the naa-based features see values of their own."""
    la = dict(la)
    rng = np.random.default_rng(seed)
    P, NF = len(la["precursor_idx"]), len(la["fragment_mz"])
    la["precursor_naa"] = rng.integers(6, 40, P).astype(np.uint8)
    la["fragment_mz_library"] = (la["fragment_mz"].astype(np.float64) *
                                 (1.0 + 3e-6 * rng.standard_normal(NF))).astype(np.float32)
    return la


def build(run: dict, la: dict):
    dia = DIAData.from_arrays(*(run[k] for k in RUN_KEYS), run["cycle"])
    kw = dict(la)
    tol = kw.pop("precursor_rt_tolerance", None)
    lib = SpecLibFlat.from_arrays(**kw, precursor_rt_tolerance=tol)
    od, ol, _ = oracle_inputs(run, la)
    oracle.lib_set_scoring(ol, la["precursor_naa"], la["fragment_mz_library"])
    return dia, lib, od, ol


def candidate_dict(cand: CandidateCollection) -> dict:
    return dict(zip(COLS, cand.to_arrays()))


def _ordered(bits: np.ndarray) -> np.ndarray:
    """float32 bit patterns mapped to integers in the order of the floats."""
    b = bits.astype(np.int64)
    return np.where(b & 0x80000000, 0x80000000 - (b & 0x7FFFFFFF), b)


def assert_features_equal(got: dict, ref: dict, exact: bool, where: str):
    n_got, n_ref = len(got["rank"]), len(ref["rank"])
    assert n_got == n_ref, f"{where}: {n_got} feature rows vs {n_ref} in the oracle"
    for c in ("precursor_idx", "rank"):
        assert got[c].dtype == np.uint64
        assert np.array_equal(got[c], ref[c]), f"{where}: column {c} differs"
    report = []
    for name in oracle.FEATURE_NAMES:
        g, r = np.asarray(got[name]), np.asarray(ref[name], np.float32)
        assert g.dtype == np.float32, (name, g.dtype)
        both_nan = np.isnan(g) & np.isnan(r)
        if exact:
            bad = (g.view(np.uint32) != r.view(np.uint32)) & ~both_nan
        else:
            d = np.abs(g.astype(np.float64) - r.astype(np.float64))
            lim = FEATURE_ATOL + FEATURE_RTOL * np.abs(r.astype(np.float64))
            bad = ~((d <= lim) | both_nan | (g == r))
        if bad.any():
            i = int(np.nonzero(bad)[0][0])
            ulp = np.abs(_ordered(g.view(np.uint32)) - _ordered(r.view(np.uint32)))[bad]
            report.append(f"{name}: {int(bad.sum())} rows, first row {i} "
                          f"(precursor {ref['precursor_idx'][i]}): {g[i]!r} vs {r[i]!r}, "
                          f"max {int(ulp.max())} ulp")
    assert not report, f"{where}:\n  " + "\n  ".join(report)


@pytest.fixture(scope="module", params=["tiny", "tiny_uneven", "tiny_cfg4", "tiny_many", "cfg0"])
def scored(request):
    """Search on the device, score the collection still on the device, and the
    oracle's features of the same candidates."""
    cfg, lib, run = synth.make_workload(request.param, "numpy")
    la = scoring_library(synth.library_arrays(lib), seed=21)
    dia, slib, od, ol = build(run, la)
    sel = PeakGroupSelection(params_from(cfg.params_dict()), verbose=False)
    cand = sel.search(dia, slib)
    sp = ScoringParameters()
    feats = PeakGroupScoring(sp, verbose=False).score(dia, slib, cand)
    cd = candidate_dict(cand)
    return dict(cfg=cfg, run=run, la=la, dia=dia, lib=slib, od=od, ol=ol, cand=cd,
                got=feats.to_dict_arrays(), n=len(feats), sp=sp)


def test_features_bit_exact_vs_rn_oracle(scored):
    s = scored
    assert len(s["cand"]["rank"]) > 0 and s["n"] == len(s["cand"]["rank"])
    ref = oracle.score(s["od"], s["ol"], s["cand"], log_mode=oracle.LOG_RN)
    assert_features_equal(s["got"], ref, exact=True, where=s["cfg"].name)


def test_features_close_to_glibc_oracle(scored):
    s = scored
    ref = oracle.score(s["od"], s["ol"], s["cand"], log_mode=oracle.LOG_GLIBC)
    assert_features_equal(s["got"], ref, exact=False, where=s["cfg"].name)


def test_host_arrays_path_matches_device_collection(scored):
    """A collection built from host arrays (ads_score_arrays) scores the same as
    the search's device-resident collection (ads_score)."""
    s = scored
    c = s["cand"]
    cc = CandidateCollection.from_arrays(*(c[k] for k in COLS))
    got = PeakGroupScoring(s["sp"], verbose=False).score(s["dia"], s["lib"], cc).to_dict_arrays()
    assert_features_equal(got, s["got"], exact=True, where=s["cfg"].name + "/arrays")


@pytest.mark.parametrize("mass_tolerance,top_k", [(15.0, 3), (3.0, 100), (7.0, 0)])
def test_other_parameters_bit_exact(scored, mass_tolerance, top_k):
    s = scored
    sp = ScoringParameters()
    sp.update({"mass_tolerance": mass_tolerance, "top_k_fragments": top_k})
    got = PeakGroupScoring(sp, verbose=False).score(
        s["dia"], s["lib"], CandidateCollection.from_arrays(*(s["cand"][k] for k in COLS)))
    ref = oracle.score(s["od"], s["ol"], s["cand"], mass_tolerance=mass_tolerance,
                       top_k_fragments=top_k, log_mode=oracle.LOG_RN)
    assert_features_equal(got.to_dict_arrays(), ref, exact=True,
                          where=f"{s['cfg'].name}/tol{mass_tolerance}/k{top_k}")


def test_unknown_precursor_is_skipped(scored):
    """Candidates whose precursor_idx is not in the library are dropped
    (src/peak_group_scoring/mod.rs:60-70), the others keep their order."""
    s = scored
    c = {k: v.copy() for k, v in s["cand"].items()}
    n = len(c["rank"])
    missing = np.uint64(int(s["la"]["precursor_idx"].max()) + 1000)
    ins = [0, n // 2, n]
    for k in COLS:
        fill = missing if k == "precursor_idx" else c[k][:1].repeat(1)[0]
        c[k] = np.insert(c[k], ins, fill)
    got = PeakGroupScoring(s["sp"], verbose=False).score(
        s["dia"], s["lib"], CandidateCollection.from_arrays(*(c[k] for k in COLS)))
    assert len(got) == n
    assert_features_equal(got.to_dict_arrays(), s["got"], exact=True, where="unknown precursor")


def test_invalid_cycle_range_raises(scored):
    s = scored
    c = {k: v[:3].copy() for k, v in s["cand"].items()}
    c["cycle_stop"][1] = np.uint64(len(s["od"].rt) + 5)
    with pytest.raises(ValueError, match="cycle range"):
        PeakGroupScoring(s["sp"], verbose=False).score(
            s["dia"], s["lib"], CandidateCollection.from_arrays(*(c[k] for k in COLS)))


def test_empty_collection(scored):
    s = scored
    got = PeakGroupScoring(s["sp"], verbose=False).score(s["dia"], s["lib"], CandidateCollection())
    assert got.is_empty() and len(got) == 0
    d = got.to_dict_arrays()
    assert set(d) == {"precursor_idx", "rank", *oracle.FEATURE_NAMES}
    assert all(len(v) == 0 for v in d.values())


def test_edge_case_library_bit_exact():
    """Hand-built corners: precursors without fragments, all-zero intensities,
    duplicated precursor_idx, unsorted fragment m/z, windows clipped at the ends."""
    run, la = edge_case_workload()
    la = scoring_library(la, seed=3)
    dia, slib, od, ol = build(run, la)
    params = dict(fwhm_rt=3.0, kernel_size=20, peak_length=5, mass_tolerance=20.0,
                  rt_tolerance=30.0, candidate_count=3, top_k_fragments=6)
    sel = PeakGroupSelection(params_from(params), verbose=False)
    cand = sel.search(dia, slib)
    feats = PeakGroupScoring(ScoringParameters(), verbose=False).score(dia, slib, cand)
    cd = candidate_dict(cand)
    assert len(cd["rank"]) > 0
    ref = oracle.score(od, ol, cd, log_mode=oracle.LOG_RN)
    assert_features_equal(feats.to_dict_arrays(), ref, exact=True, where="edge cases")


def test_feature_names_match_reference_order():
    assert CandidateFeatureCollection.get_feature_names() == list(oracle.FEATURE_NAMES)


def test_device_buffer_scores_like_collection(scored):
    """A reusable DeviceCandidates buffer (search_into) is scored in place, twice in a
    row, with the same features as the search's collection."""
    s = scored
    sel = PeakGroupSelection(params_from(s["cfg"].params_dict()), verbose=False)
    buf = sel.new_candidates()
    scorer = PeakGroupScoring(s["sp"], verbose=False)
    for call in range(2):
        sel.search_into(s["dia"], s["lib"], buf)
        f = scorer.score(s["dia"], s["lib"], buf)
        assert f.kernel_ms() > 0.0
        assert_features_equal(f.to_dict_arrays(), s["got"], exact=True,
                              where=f"{s['cfg'].name}/buffer/{call}")


def test_whole_run_cycle_ranges(scored):
    """Candidates spanning the whole run (a scratch of several thousand words per
    candidate) still match the oracle."""
    s = scored
    n_rt = len(s["od"].rt)
    c = {k: v[:64].copy() for k, v in s["cand"].items()}
    c["cycle_start"][:] = 0
    c["cycle_stop"][:] = n_rt
    c["cycle_center"][:] = np.minimum(c["cycle_center"], n_rt - 1)
    got = PeakGroupScoring(s["sp"], verbose=False).score(
        s["dia"], s["lib"], CandidateCollection.from_arrays(*(c[k] for k in COLS)))
    ref = oracle.score(s["od"], s["ol"], c, log_mode=oracle.LOG_RN)
    assert_features_equal(got.to_dict_arrays(), ref, exact=True, where=s["cfg"].name + "/long")


def test_sharded_scoring_with_merged_idf():
    """A library split in two shards, each searched and scored on its own with the two
    shards' IDF histograms summed (the all-reduce of a multi-GPU run, done here on one
    GPU), gives the unsplit library's features, in the same order."""
    import torch

    from alphadia_search_rs_b200 import _ffi, sharding

    cfg, lib, run = synth.make_workload("tiny_uneven", "numpy")
    la = scoring_library(synth.library_arrays(lib), seed=8)
    dia, whole, od, ol = build(run, la)
    params = params_from(cfg.params_dict())
    ref = PeakGroupScoring(ScoringParameters(), verbose=False).score(
        dia, whole, PeakGroupSelection(params, verbose=False).search(dia, whole)).to_dict_arrays()
    n_bins = int(_ffi.load().ads_idf_bins())
    shards, total = [], 0
    counts = torch.zeros(n_bins, dtype=torch.int32, device="cuda:0")
    for r in range(2):
        sa = sharding.shard_library(la, r, 2)
        kw = dict(sa)
        tol = kw.pop("precursor_rt_tolerance", None)
        sl = SpecLibFlat.from_arrays(**kw, precursor_rt_tolerance=tol)
        own = torch.empty(n_bins, dtype=torch.int32, device="cuda:0")
        sl.idf_counts(out=own)
        assert np.array_equal(own.cpu().numpy().view(np.uint32), sl.idf_counts())
        counts += own
        total += sl.num_fragments
        shards.append(sl)
    assert np.array_equal(counts.cpu().numpy().view(np.uint32), whole.idf_counts())
    parts = []
    for r, sl in enumerate(shards):
        (sl.set_idf(counts, total) if r == 0 else sl.set_idf(counts.cpu().numpy().view(np.uint32), total))
        cand = PeakGroupSelection(params, verbose=False).search(dia, sl)
        parts.append(PeakGroupScoring(ScoringParameters(), verbose=False).score(dia, sl, cand).to_dict_arrays())
    got = {k: np.concatenate([p[k] for p in parts]) for k in ref}
    assert_features_equal(got, ref, exact=True, where="2 shards")


@pytest.mark.parametrize("case", ["inf_library_intensity", "huge_peaks"])
def test_extreme_values(case):
    """Scoring and quantification with an infinite library intensity (top-k ranks,
    intensity correlation and hyperscore see it) or peaks near the f32 range (sums
    overflow to inf in the XIC): device and oracle still agree bit for bit."""
    from test_gpu_quant import assert_quant_equal, quant_library

    from alphadia_search_rs_b200 import PeakGroupQuantification, QuantificationParameters

    run, la = edge_case_workload()
    la = quant_library(la, seed=11)
    run = dict(run)
    if case == "inf_library_intensity":
        fi = np.array(la["fragment_intensity"], np.float32, copy=True)
        fi[3] = np.inf
        la["fragment_intensity"] = fi
    else:
        pi = np.array(run["peak_intensity"], np.float32, copy=True)
        pi[::7] = np.float32(3e38)
        run["peak_intensity"] = pi
    dia, slib, od, ol = build(run, la)
    params = dict(fwhm_rt=3.0, kernel_size=20, peak_length=5, mass_tolerance=20.0,
                  rt_tolerance=30.0, candidate_count=3, top_k_fragments=6)
    cand = PeakGroupSelection(params_from(params), verbose=False).search(dia, slib)
    cd = candidate_dict(cand)
    assert len(cd["rank"]) > 0
    feats = PeakGroupScoring(ScoringParameters(), verbose=False).score(dia, slib, cand)
    assert_features_equal(feats.to_dict_arrays(), oracle.score(od, ol, cd, log_mode=oracle.LOG_RN),
                          exact=True, where=case)
    q = PeakGroupQuantification(QuantificationParameters(), verbose=False).quantify(dia, slib, cand)
    assert_quant_equal(q, oracle.quantify(od, ol, cd, la), case)


def test_concurrent_threads_share_run_and_library():
    """Four host threads search, score and quantify against the same DIAData and
    SpecLibFlat at once (each call on its thread's stream; the library's IDF histogram
    is built once under a lock); every thread gets the serial result."""
    import threading

    from test_gpu_quant import quant_library

    from alphadia_search_rs_b200 import PeakGroupQuantification, QuantificationParameters

    cfg, lib, run = synth.make_workload("tiny_uneven", "numpy")
    la = quant_library(synth.library_arrays(lib), seed=2)
    dia, slib, od, ol = build(run, la)
    params = params_from(cfg.params_dict())

    def job():
        cand = PeakGroupSelection(params, verbose=False).search(dia, slib)
        f = PeakGroupScoring(ScoringParameters(), verbose=False).score(dia, slib, cand).to_dict_arrays()
        q = PeakGroupQuantification(QuantificationParameters(), verbose=False).quantify(dia, slib, cand)
        return f, q.to_dict_arrays()

    results, errors = [None] * 4, []

    def run_one(i):
        try:
            results[i] = job()
        except Exception as e:  # reported below
            errors.append(repr(e))

    threads = [threading.Thread(target=run_one, args=(i,)) for i in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    ref_f, ref_q = job()
    for f, q in results:
        assert_features_equal(f, ref_f, exact=True, where="thread")
        for part, g, r in ((0, q[0], ref_q[0]), (1, q[1], ref_q[1])):
            for k in r:
                assert np.array_equal(np.asarray(g[k]).view(np.uint8), np.asarray(r[k]).view(np.uint8)), (part, k)
