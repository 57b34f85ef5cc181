"""GPU: searches streamed through one selection (step i's library uploaded and its
search enqueued before step i-1's candidates are read back, two candidate
collections alternating), as the end-to-end benchmark runs them.  Every read-back
equals a search of the same library on its own."""
import numpy as np
import pytest

from alphadia_search_rs_b200 import DIAData, PeakGroupSelection, SpecLibFlat, synth

from _util import COLS, RUN_KEYS, params_from

pytestmark = pytest.mark.gpu


def _libraries():
    cfg, lib, run = synth.make_workload("tiny_uneven", "numpy")
    la = synth.library_arrays(lib)
    tol = la.pop("precursor_rt_tolerance")
    # a second library: every other precursor, fragments re-based
    keep = np.arange(0, len(la["precursor_idx"]), 2)
    fs, fe = la["flat_frag_start_idx"][keep], la["flat_frag_stop_idx"][keep]
    frag = np.concatenate([np.arange(int(a), int(b)) for a, b in zip(fs, fe)]).astype(np.int64)
    n = (fe - fs).astype(np.uint64)
    start = np.concatenate([[0], np.cumsum(n)[:-1]]).astype(np.uint64)
    lb = {k: (v[keep] if k.startswith("precursor") else v[frag]) for k, v in la.items()
          if not k.startswith("flat")}
    lb["flat_frag_start_idx"], lb["flat_frag_stop_idx"] = start, start + n
    return cfg, run, [(la, tol), (lb, tol[keep])]


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_streamed_searches_match_serial(precision):
    cfg, run, libs = _libraries()
    dia = DIAData.from_arrays(*(run[k] for k in RUN_KEYS), run["cycle"])
    params = params_from(cfg.params_dict())
    expect = []
    for la, tol in libs:
        sl = SpecLibFlat.from_arrays(**la, precursor_rt_tolerance=tol)
        expect.append(dict(zip(COLS, PeakGroupSelection(params, verbose=False, precision=precision)
                               .search(dia, sl).to_arrays())))
    sel = PeakGroupSelection(params, verbose=False, precision=precision)
    cands = [sel.new_candidates(), sel.new_candidates()]
    cap = max(len(e["rank"]) for e in expect)
    outs = [{c: np.zeros(cap, np.float32 if c == "score" else np.uint64) for c in COLS} for _ in range(2)]
    held = []
    steps = 6
    for i in range(steps + 1):
        if i < steps:
            la, tol = libs[i % 2]
            sl = SpecLibFlat.from_arrays(**la, precursor_rt_tolerance=tol)
            held.append(sl)
            sel.search_into(dia, sl, cands[i % 2])
        if i >= 1:
            j = i - 1
            n = cands[j % 2].copy_out(outs[j % 2])
            ref = expect[j % 2]
            assert n == len(ref["rank"])
            for c in COLS:
                assert np.array_equal(outs[j % 2][c][:n].view(np.uint8), np.asarray(ref[c]).view(np.uint8)), (j, c)


def test_graph_replay_after_library_replaced():
    """use_graph: a library released and another built in its place (the handle may land
    at the same address) is searched afresh, not through the old library's graph."""
    cfg, run, libs = _libraries()
    dia = DIAData.from_arrays(*(run[k] for k in RUN_KEYS), run["cycle"])
    params = params_from(cfg.params_dict())
    sel = PeakGroupSelection(params, verbose=False, use_graph=True)
    cand = sel.new_candidates()
    for j in (0, 1, 0):
        la, tol = libs[j]
        sl = SpecLibFlat.from_arrays(**la, precursor_rt_tolerance=tol)
        ref = dict(zip(COLS, PeakGroupSelection(params, verbose=False).search(dia, sl).to_arrays()))
        for _ in range(2):  # captured, then replayed
            sel.search_into(dia, sl, cand)
            n = cand.size()
            got = {c: np.zeros(max(n, 1), np.float32 if c == "score" else np.uint64) for c in COLS}
            cand.copy_out(got)
            assert n == len(ref["rank"])
            for c in COLS:
                assert np.array_equal(got[c][:n].view(np.uint8), np.asarray(ref[c]).view(np.uint8)), (j, c)
        del sl
