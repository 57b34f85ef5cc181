"""GPU: the search at the benchmark configurations' full sizes (cfg1: 0.95 G peaks,
200,000 precursors; cfg3: the same run, 500,000 precursors with 4-24 fragments and
per-precursor RT windows), generated on the device.

The oracle cannot search these in seconds, so the checks are properties that hold at
any size, plus the oracle on the subset the bench uses: the precursors strictly inside
24 consecutive MS2 windows, searched against those windows' peaks, which must give
exactly the full search's candidates for those precursors.
"""
import os
import sys

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from _util import COLS, RUN_KEYS, SCORE_RTOL, params_from  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["cfg1", "cfg3"])
def full(request):
    import torch

    import alphadia_search_rs_b200 as ads

    cfg, lib, run = bench.make_device_workload(request.param, "cuda:0")
    dia = ads.DIAData.from_arrays(*(run[k] for k in RUN_KEYS), run["cycle"], device=0)
    slib = ads.SpecLibFlat.from_arrays(**bench.library_tensors(lib, "cuda:0"), device=0)
    yield cfg, lib, run, dia, slib
    del dia, slib, run, lib
    torch.cuda.empty_cache()


def _search(ads, cfg, dia, slib, **engine):
    sel = ads.PeakGroupSelection(params_from(cfg.params_dict()), verbose=False, **engine)
    return dict(zip(COLS, sel.search(dia, slib).to_arrays()))


def test_full_size_output_properties(full):
    """Library order, ranks 0.. per precursor, best first, valid cycle ranges."""
    import alphadia_search_rs_b200 as ads

    cfg, lib, run, dia, slib = full
    got = _search(ads, cfg, dia, slib)
    n = len(got["rank"])
    assert n > cfg.n_precursors  # most precursors give their top-3
    pidx, rank, score = got["precursor_idx"], got["rank"], got["score"]
    assert np.all(np.diff(pidx.astype(np.int64)) >= 0)  # library order (sorted precursor_idx)
    first = np.r_[True, pidx[1:] != pidx[:-1]]
    assert np.all(rank[first] == 0)
    assert np.all(rank[~first] == rank[np.nonzero(~first)[0] - 1] + 1)
    assert rank.max() < cfg.candidate_count
    same = ~first
    prev = np.nonzero(same)[0] - 1
    assert np.all(score[same] <= score[prev])  # value descending within a precursor
    n_rt = len(dia.rt_index()[0])
    c, s, e = got["cycle_center"], got["cycle_start"], got["cycle_stop"]
    assert np.all((s <= c) & (c < e) & (e <= n_rt))
    assert np.all(e - s <= 2 * 5 + 1)  # peak_length 5
    assert np.all(np.isfinite(score))
    for k in ("scan_center", "scan_start", "scan_stop"):
        assert not got[k].any()


def test_full_size_graph_replay_and_repeat_identical(full):
    import alphadia_search_rs_b200 as ads

    cfg, lib, run, dia, slib = full
    a = _search(ads, cfg, dia, slib)
    sel = ads.PeakGroupSelection(params_from(cfg.params_dict()), verbose=False, use_graph=True)
    cand = sel.new_candidates()
    for _ in range(3):  # direct, then two graph replays into the same buffers
        sel.search_into(dia, slib, cand)
        n = cand.size()
        got = {c: np.zeros(n, np.float32 if c == "score" else np.uint64) for c in COLS}
        cand.copy_out(got)
        for k in COLS:
            assert np.array_equal(np.asarray(got[k]).view(np.uint8), np.asarray(a[k]).view(np.uint8)), k


def test_full_size_bf16_agrees_with_fp32(full):
    """BF16 storage against the exact FP32 path on the same data: top-K cycles."""
    import alphadia_search_rs_b200 as ads

    cfg, lib, run, dia, slib = full
    f32 = _search(ads, cfg, dia, slib)
    b16 = _search(ads, cfg, dia, slib, precision="bf16")
    key32 = set(zip(f32["precursor_idx"].tolist(), f32["rank"].tolist(), f32["cycle_center"].tolist()))
    key16 = set(zip(b16["precursor_idx"].tolist(), b16["rank"].tolist(), b16["cycle_center"].tolist()))
    assert len(key32 & key16) / len(key32) >= 0.99


def test_full_size_window_subset_matches_oracle(full):
    """The full search's candidates of the precursors inside 24 middle windows equal the
    oracle's search of those windows: indices exactly, scores bit for bit against the
    correctly rounded log and within 1e-5 relative against glibc logf."""
    import alphadia_search_rs_b200 as ads

    cfg, lib, run, dia, slib = full
    got = _search(ads, cfg, dia, slib)
    host, sub, _ = bench.window_subset(cfg, run, lib, 24)
    od, ol, tol = bench.oracle_setup(host, sub, bench.cpu_threads())
    mask = np.isin(got["precursor_idx"], sub["precursor_idx"])
    for log_mode in (oracle.LOG_RN, oracle.LOG_GLIBC):
        ref = oracle.search(od, ol, oracle.Params(**cfg.params_dict()), rt_tolerance_per_precursor=tol,
                            log_mode=log_mode, n_threads=bench.cpu_threads())
        assert int(mask.sum()) == len(ref["rank"]) > 1000
        for k in ("precursor_idx", "rank", "cycle_center", "cycle_start", "cycle_stop"):
            assert np.array_equal(got[k][mask], ref[k]), k
        gs, rs = got["score"][mask], ref["score"]
        if log_mode == oracle.LOG_RN:
            assert np.array_equal(gs.view(np.uint32), rs.view(np.uint32))
        else:
            rel = np.abs(gs.astype(np.float64) - rs) / np.maximum(np.abs(rs.astype(np.float64)), 1e-30)
            assert float(rel.max()) <= SCORE_RTOL
