"""GPU parity of PeakGroupQuantification (src/peak_group_quantification/mod.rs:49-168):
the SpecLibFlatQuantified arrays computed on the device, through the C ABI, against the
oracle's restatement on the same candidates, every column identical (no logarithm is
involved, so bit for bit)."""
import numpy as np
import pytest

import oracle
from alphadia_search_rs_b200 import (CandidateCollection, PeakGroupQuantification,
                                     PeakGroupSelection, QuantificationParameters, synth)

from _util import COLS, edge_case_workload, params_from
from test_gpu_scoring import build, candidate_dict, scoring_library

pytestmark = pytest.mark.gpu


def quant_library(la: dict, seed: int) -> dict:
    """Scoring's library plus fragment annotations of their own, so that the
    pass-through columns are checked on values that differ between fragments."""
    la = scoring_library(la, seed)
    rng = np.random.default_rng(seed + 1)
    NF = len(la["fragment_mz"])
    for k in ("fragment_cardinality", "fragment_charge", "fragment_loss_type", "fragment_position"):
        la[k] = rng.integers(0, 5, NF).astype(np.uint8)
    la["precursor_mz_library"] = (la["precursor_mz"] - np.float32(0.01)).astype(np.float32)
    la["precursor_rt_library"] = (la["precursor_rt"] + np.float32(1.5)).astype(np.float32)
    return la


def assert_quant_equal(got, ref, where: str):
    gp, gf = got.to_dict_arrays() if hasattr(got, "to_dict_arrays") else got
    rp, rf = ref
    assert list(gp) == list(oracle.QUANT_PRECURSOR_KEYS) and list(gf) == list(oracle.QUANT_FRAGMENT_KEYS)
    for part, g, r in (("precursor", gp, rp), ("fragment", gf, rf)):
        for k in r:
            a, b = np.asarray(g[k]), np.asarray(r[k])
            assert a.dtype == b.dtype, f"{where}: {part} {k} dtype {a.dtype} vs {b.dtype}"
            assert len(a) == len(b), f"{where}: {part} {k}: {len(a)} rows vs {len(b)}"
            # floats bit for bit; NaN matches NaN (its payload differs between the
            # device and the host's SSE arithmetic and carries no information)
            same = ((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))
                    if a.dtype == np.float32 else a == b)
            if not np.all(same):
                i = int(np.nonzero(~same)[0][0])
                raise AssertionError(f"{where}: {part} {k} differs at row {i}: {a[i]!r} vs {b[i]!r}")


@pytest.fixture(scope="module", params=["tiny", "tiny_uneven", "tiny_cfg4", "tiny_many", "cfg0"])
def quantified(request):
    cfg, lib, run = synth.make_workload(request.param, "numpy")
    la = quant_library(synth.library_arrays(lib), seed=31)
    dia, slib, od, ol = build(run, la)
    sel = PeakGroupSelection(params_from(cfg.params_dict()), verbose=False)
    cand = sel.search(dia, slib)
    qp = QuantificationParameters()
    got = PeakGroupQuantification(qp, verbose=False).quantify(dia, slib, cand)
    return dict(cfg=cfg, la=la, dia=dia, lib=slib, od=od, ol=ol, cand=candidate_dict(cand), got=got,
                qp=qp)


def test_quantified_library_matches_oracle(quantified):
    s = quantified
    ref = oracle.quantify(s["od"], s["ol"], s["cand"], s["la"])
    assert len(ref[0]["precursor_idx"]) > 0
    assert s["got"].num_precursors == len(ref[0]["precursor_idx"])
    assert s["got"].num_fragments == len(ref[1]["mz"])
    assert_quant_equal(s["got"], ref, s["cfg"].name)


def test_host_arrays_path(quantified):
    s = quantified
    cc = CandidateCollection.from_arrays(*(s["cand"][k] for k in COLS))
    got = PeakGroupQuantification(s["qp"], verbose=False).quantify(s["dia"], s["lib"], cc)
    assert_quant_equal(got, s["got"].to_dict_arrays(), s["cfg"].name + "/arrays")


@pytest.mark.parametrize("tol,top_k", [(15.0, 3), (2.0, 10000), (7.0, 0)])
def test_other_parameters(quantified, tol, top_k):
    s = quantified
    qp = QuantificationParameters()
    qp.update({"tolerance_ppm": tol, "top_k_fragments": top_k})
    got = PeakGroupQuantification(qp, verbose=False).quantify(
        s["dia"], s["lib"], CandidateCollection.from_arrays(*(s["cand"][k] for k in COLS)))
    ref = oracle.quantify(s["od"], s["ol"], s["cand"], s["la"], tolerance_ppm=tol, top_k_fragments=top_k)
    assert_quant_equal(got, ref, f"{s['cfg'].name}/tol{tol}/k{top_k}")


def test_dropped_candidates(quantified):
    """Unknown precursors, empty cycle ranges and centres outside the range are dropped
    as in the reference; the remaining order is kept."""
    s = quantified
    c = {k: np.asarray(v)[:40].copy() for k, v in s["cand"].items()}
    c["precursor_idx"][3] = np.uint64(int(s["la"]["precursor_idx"].max()) + 7)
    c["cycle_stop"][5] = c["cycle_start"][5]
    c["cycle_center"][7] = c["cycle_stop"][7]
    c["cycle_start"][9], c["cycle_stop"][9] = c["cycle_stop"][9], c["cycle_start"][9]
    got = PeakGroupQuantification(s["qp"], verbose=False).quantify(
        s["dia"], s["lib"], CandidateCollection.from_arrays(*(c[k] for k in COLS)))
    ref = oracle.quantify(s["od"], s["ol"], c, s["la"])
    assert_quant_equal(got, ref, s["cfg"].name + "/dropped")


def test_range_beyond_the_run_raises(quantified):
    s = quantified
    c = {k: np.asarray(v)[:3].copy() for k, v in s["cand"].items()}
    c["cycle_stop"][1] = np.uint64(len(s["od"].rt) + 4)
    with pytest.raises(ValueError, match="RT index"):
        PeakGroupQuantification(s["qp"], verbose=False).quantify(
            s["dia"], s["lib"], CandidateCollection.from_arrays(*(c[k] for k in COLS)))


def test_device_buffer(quantified):
    s = quantified
    sel = PeakGroupSelection(params_from(s["cfg"].params_dict()), verbose=False)
    buf = sel.new_candidates()
    q = PeakGroupQuantification(s["qp"], verbose=False)
    for call in range(2):
        sel.search_into(s["dia"], s["lib"], buf)
        got = q.quantify(s["dia"], s["lib"], buf)
        assert got.kernel_ms() > 0.0
        assert_quant_equal(got, s["got"].to_dict_arrays(), f"{s['cfg'].name}/buffer/{call}")


def test_empty_collection(quantified):
    s = quantified
    got = PeakGroupQuantification(s["qp"], verbose=False).quantify(s["dia"], s["lib"], CandidateCollection())
    assert got.num_precursors == 0 and got.num_fragments == 0
    p, f = got.to_dict_arrays()
    assert all(len(v) == 0 for v in p.values()) and all(len(v) == 0 for v in f.values())


def test_edge_case_library():
    run, la = edge_case_workload()
    la = quant_library(la, seed=5)
    dia, slib, od, ol = build(run, la)
    params = dict(fwhm_rt=3.0, kernel_size=20, peak_length=5, mass_tolerance=20.0,
                  rt_tolerance=30.0, candidate_count=3, top_k_fragments=6)
    cand = PeakGroupSelection(params_from(params), verbose=False).search(dia, slib)
    got = PeakGroupQuantification(QuantificationParameters(), verbose=False).quantify(dia, slib, cand)
    cd = candidate_dict(cand)
    assert len(cd["rank"]) > 0
    assert_quant_equal(got, oracle.quantify(od, ol, cd, la), "edge cases")


def test_device_resident_candidate_arrays(quantified):
    """ads_score_arrays and ads_quantify_arrays with ADS_MEM_DEVICE (candidate columns
    already in device memory) give what the host-array calls give."""
    import ctypes as C

    import torch

    from alphadia_search_rs_b200 import CandidateFeatureCollection, ScoringParameters
    from alphadia_search_rs_b200 import _ffi as F

    s = quantified
    L = F.load()
    c = s["cand"]
    n = len(c["rank"])
    dev = {k: torch.as_tensor(np.asarray(c[k]).view(np.int64) if c[k].dtype == np.uint64 else c[k],
                              device="cuda:0") for k in COLS}
    ptr = lambda k: dev[k].data_ptr()
    # scoring
    sp = ScoringParameters()._c()
    h = C.c_void_p()
    F.check(L.ads_score_arrays(C.byref(sp), s["dia"]._h, s["lib"]._h, n, ptr("precursor_idx"),
                               ptr("rank"), ptr("score"), ptr("cycle_center"), ptr("cycle_start"),
                               ptr("cycle_stop"), F.ADS_MEM_DEVICE, 0, C.byref(h)))
    got = CandidateFeatureCollection._from_handle(h.value).to_dict_arrays()
    from alphadia_search_rs_b200 import PeakGroupScoring

    ref = PeakGroupScoring(ScoringParameters(), verbose=False).score(
        s["dia"], s["lib"], CandidateCollection.from_arrays(*(c[k] for k in COLS))).to_dict_arrays()
    for k in ref:
        assert np.array_equal(np.asarray(got[k]).view(np.uint8), np.asarray(ref[k]).view(np.uint8)), k
    # quantification
    qp = s["qp"]._c()
    hq = C.c_void_p()
    F.check(L.ads_quantify_arrays(C.byref(qp), s["dia"]._h, s["lib"]._h, n, ptr("precursor_idx"),
                                  ptr("rank"), ptr("cycle_center"), ptr("cycle_start"), ptr("cycle_stop"),
                                  F.ADS_MEM_DEVICE, 0, C.byref(hq)))
    try:
        n_p, n_f = C.c_int64(), C.c_int64()
        F.check(L.ads_quant_sizes(hq, C.byref(n_p), C.byref(n_f)))
        rp, rf = s["got"].to_dict_arrays()
        assert n_p.value == len(rp["precursor_idx"]) and n_f.value == len(rf["mz"])
        out = [np.empty(max(n_p.value, 1), np.uint64) for _ in range(3)]
        F.check(L.ads_quant_copy_out(hq, out[0].ctypes.data, None, out[1].ctypes.data, None, None,
                                     out[2].ctypes.data, None, None, None, None, None, None, None))
        assert np.array_equal(out[0][:n_p.value], rp["precursor_idx"])
        assert np.array_equal(out[1][:n_p.value], rp["rank"])
        assert np.array_equal(out[2][:n_p.value], rp["flat_frag_stop_idx"])
    finally:
        L.ads_quant_destroy(hq)
