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


def output_arrays(cap: int):
    """Caller-owned device arrays for one call (torch allocates them, not the library)."""
    import torch

    dev = torch.device("cuda", 0)
    cols = {c: torch.empty(max(cap, 1), dtype=torch.float32 if c == "score" else torch.int64,
                           device=dev) for c in OUT_COLS}
    count = torch.full((1,), -7, dtype=torch.int64, device=dev)
    flags = torch.full((1,), -7, dtype=torch.int32, device=dev)
    return cols, count, flags


def noalloc_search(dia, lib, params: dict, capacity=None, outputs=None, flags_ptr=None):
    """One call through the C ABI into torch-owned device arrays; returns the
    candidate columns (scan_* zero, as in the reference) and the error flags."""
    import torch

    prm = params_from(params)
    P = lib.num_precursors
    cap = P * prm.candidate_count if capacity is None else capacity
    cols, count, flags = outputs if outputs is not None else output_arrays(cap)
    stream = torch.cuda.current_stream(torch.device("cuda", 0))
    c_params = prm._c()
    rc = F.load().ads_select_noalloc(dia._h, lib._h, C.byref(c_params), stream.cuda_stream, cap,
                                     *[cols[c].data_ptr() for c in OUT_COLS], count.data_ptr(),
                                     flags.data_ptr() if flags_ptr is None else flags_ptr)
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


@pytest.mark.parametrize("name", ["tiny", "tiny_uneven", "tiny_cfg4", "cfg0", "tiny_long", "long_rt"])
def test_noalloc_matches_select(name):
    cfg, lib, run = synth.make_workload(name, "numpy")
    _check_twice(run, synth.library_arrays(lib), cfg.params_dict())


def test_noalloc_matches_select_edge_cases():
    run, la = edge_case_workload()
    params = dict(fwhm_rt=3.0, kernel_size=20, peak_length=5, mass_tolerance=20.0,
                  rt_tolerance=30.0, candidate_count=3, top_k_fragments=6)
    _check_twice(run, la, params)


def test_noalloc_matches_select_wide_kernel():
    """A kernel wider than 62: its taps go into the scratch array too."""
    cfg, lib, run = synth.make_workload("tiny_long", "numpy")
    _check_twice(run, synth.library_arrays(lib), dict(cfg.params_dict(), kernel_size=128, fwhm_rt=30.0))


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


def test_noalloc_after_a_larger_different_search():
    """The scratch keeps whatever the previous call left: a long-window search over a
    larger library fills it first, then a smaller search of another run must still
    give exactly what ads_select gives."""
    cfg_a, lib_a, run_a = synth.make_workload("tiny_long", "numpy")
    _, dia_a, slib_a, _ = product_search(run_a, synth.library_arrays(lib_a), cfg_a.params_dict())
    noalloc_search(dia_a, slib_a, cfg_a.params_dict())
    cfg_b, lib_b, run_b = synth.make_workload("tiny", "numpy")
    ref, dia_b, slib_b, _ = product_search(run_b, synth.library_arrays(lib_b), cfg_b.params_dict())
    got, flags = noalloc_search(dia_b, slib_b, cfg_b.params_dict())
    assert flags == 0
    assert_candidates_equal(got, ref, exact_scores=True, where="after a larger search")


def test_noalloc_allocates_nothing():
    """After its first call on the device (which looks up the scratch array), a call
    leaves the device's free memory and torch's caching allocator untouched."""
    import torch

    cfg, lib, run = synth.make_workload("tiny_uneven", "numpy")
    params = cfg.params_dict()
    ref, dia, slib, _ = product_search(run, synth.library_arrays(lib), params)
    cap = slib.num_precursors * params["candidate_count"]
    outputs = output_arrays(cap)
    noalloc_search(dia, slib, params, outputs=outputs)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    reserved0 = torch.cuda.memory_reserved(0)
    F.load()  # no library calls between the two measurements but the search
    got, flags = noalloc_search(dia, slib, params, outputs=outputs)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert torch.cuda.memory_reserved(0) == reserved0
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"
    assert flags == 0
    assert_candidates_equal(got, ref, exact_scores=True, where="allocation check")


def test_noalloc_rejects_null_flags():
    """The kernels report internal errors through *flags, so it may not be NULL."""
    cfg, lib, run = synth.make_workload("tiny", "numpy")
    params = cfg.params_dict()
    _, dia, slib, _ = product_search(run, synth.library_arrays(lib), params)
    with pytest.raises(ValueError, match="flags"):
        noalloc_search(dia, slib, params, flags_ptr=0)
