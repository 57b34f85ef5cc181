"""ads_select_noalloc, the allocation-free search entry point, against ads_select.

The entry point exists for callers that may not allocate device memory while they
search (their device memory belongs to another allocator, or cudaFree's implicit
synchronisation is unaffordable); it works in a fixed scratch array that keeps the
previous call's contents, so every check here runs two calls in a row.  The file
name makes pytest collect it last: a run that stops at the first failure has run
every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

from alphadia_search_rs_b200 import _ffi as F
from alphadia_search_rs_b200 import synth

from _util import RUN_KEYS, assert_candidates_equal, edge_case_workload, params_from, product_search

pytestmark = pytest.mark.gpu

OUT_COLS = ("precursor_idx", "rank", "score", "cycle_center", "cycle_start", "cycle_stop")


def noalloc_search(dia, lib, params: dict, capacity=None):
    """One call through the C ABI into torch-owned device arrays; returns the
    candidate columns (scan_* zero, as in the reference) and the error flags."""
    import torch

    prm = params_from(params)
    P = lib.num_precursors
    cap = P * prm.candidate_count if capacity is None else capacity
    dev = torch.device("cuda", 0)
    cols = {c: torch.empty(max(cap, 1), dtype=torch.float32 if c == "score" else torch.int64,
                           device=dev) for c in OUT_COLS}
    count = torch.full((1,), -7, dtype=torch.int64, device=dev)
    flags = torch.full((1,), -7, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    c_params = prm._c()
    rc = F.load().ads_select_noalloc(dia._h, lib._h, C.byref(c_params), stream.cuda_stream, cap,
                                     *[cols[c].data_ptr() for c in OUT_COLS], count.data_ptr(),
                                     flags.data_ptr())
    F.check(rc)
    stream.synchronize()
    n = int(count.item())
    out = {c: cols[c][:n].cpu().numpy() for c in OUT_COLS}
    for c in OUT_COLS:
        if c != "score":
            out[c] = out[c].view(np.uint64)
    for c in ("scan_center", "scan_start", "scan_stop"):
        out[c] = np.zeros(n, np.uint64)
    return out, int(flags.item())


def _check_twice(run, la, params):
    ref, dia, lib, _ = product_search(run, la, params)
    assert len(ref["rank"]) > 0
    for call in (1, 2):
        got, flags = noalloc_search(dia, lib, params)
        assert flags == 0
        # same kernels, same order of operations: identical bits
        assert_candidates_equal(got, ref, exact_scores=True, where=f"call {call}")


@pytest.mark.parametrize("name", ["tiny", "tiny_uneven", "cfg0"])
def test_noalloc_matches_select(name):
    cfg, lib, run = synth.make_workload(name, "numpy")
    _check_twice(run, synth.library_arrays(lib), cfg.params_dict())


def test_noalloc_matches_select_edge_cases():
    run, la = edge_case_workload()
    params = dict(fwhm_rt=3.0, kernel_size=20, peak_length=5, mass_tolerance=20.0,
                  rt_tolerance=30.0, candidate_count=3, top_k_fragments=6)
    _check_twice(run, la, params)


def test_noalloc_rejects_small_capacity():
    cfg, lib, run = synth.make_workload("tiny", "numpy")
    params = cfg.params_dict()
    _, dia, slib, _ = product_search(run, synth.library_arrays(lib), params)
    need = slib.num_precursors * params["candidate_count"]
    with pytest.raises(ValueError, match="capacity"):
        noalloc_search(dia, slib, params, capacity=need - 1)


def test_noalloc_rejects_search_beyond_scratch():
    """A library whose working memory exceeds the fixed scratch is refused with a
    message, before anything is enqueued."""
    from alphadia_search_rs_b200 import DIAData, SpecLibFlat

    cfg, _, run = synth.make_workload("tiny", "numpy")
    dia = DIAData.from_arrays(*(run[k] for k in RUN_KEYS), run["cycle"])
    P, nfrag = 200_000, 12
    rng = np.random.default_rng(3)
    NF = P * nfrag
    start = np.arange(P, dtype=np.uint64) * nfrag
    lib = SpecLibFlat.from_arrays(
        precursor_idx=np.arange(P, dtype=np.uint64),
        precursor_mz_library=np.full(P, 450.0, np.float32), precursor_mz=np.full(P, 450.0, np.float32),
        precursor_rt_library=np.full(P, 80.0, np.float32), precursor_rt=np.full(P, 80.0, np.float32),
        precursor_naa=np.full(P, 10, np.uint8),
        flat_frag_start_idx=start, flat_frag_stop_idx=start + nfrag,
        fragment_mz_library=rng.uniform(200, 1500, NF).astype(np.float32),
        fragment_mz=rng.uniform(200, 1500, NF).astype(np.float32),
        fragment_intensity=rng.uniform(0.1, 1.0, NF).astype(np.float32),
        fragment_cardinality=np.ones(NF, np.uint8), fragment_charge=np.ones(NF, np.uint8),
        fragment_loss_type=np.zeros(NF, np.uint8), fragment_number=np.full(NF, 3, np.uint8),
        fragment_position=np.ones(NF, np.uint8), fragment_type=np.full(NF, 98, np.uint8))
    with pytest.raises(ValueError, match="scratch"):
        noalloc_search(dia, lib, cfg.params_dict())
