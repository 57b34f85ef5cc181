"""GPU parity: the CUDA search (through the C ABI) against the CPU oracle.

Two comparisons per workload:
  * oracle with a correctly rounded logf (what the kernel computes): every column
    identical, scores bit for bit -- this pins the kernel's summation order;
  * oracle with glibc logf (the reference's numerics on Linux): every index
    column identical, scores within SCORE_RTOL (1e-5) relative.
"""
import numpy as np
import pytest

import oracle
from alphadia_search_rs_b200 import synth

from _util import (RUN_KEYS, assert_candidates_equal, edge_case_workload, oracle_inputs,
                   oracle_search, product_search)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["tiny", "tiny_uneven", "tiny_cfg4", "tiny_many", "cfg0",
                                        "tiny_long", "long_rt"])
def workload(request):
    cfg, lib, run = synth.make_workload(request.param, "numpy")
    la = synth.library_arrays(lib)
    od, ol, tol = oracle_inputs(run, la)
    return cfg, run, la, (od, ol, tol)


def test_dia_csr_matches_builder(workload):
    """DIAData built on the device is word-identical to the restated builder
    (src/dia_data_builder/mod.rs:52-139)."""
    cfg, run, la, (od, ol, tol) = workload
    from alphadia_search_rs_b200 import DIAData

    dia = DIAData.from_arrays(*(run[k] for k in RUN_KEYS), run["cycle"])
    assert dia.num_observations == od.num_observations
    rt, dt = dia.rt_index()
    assert np.array_equal(rt, od.rt) and np.float32(dt) == np.float32(od.delta_t)
    for w in range(od.num_observations):
        o = dia.observation(w)
        assert o["isolation_window"] == od.window(w)
        assert np.array_equal(o["slice_starts"], od.slice_starts(w)), w
        assert np.array_equal(o["cycle_indices"], od.cycles(w)), w
        assert np.array_equal(o["intensities"].view(np.uint32), od.intensities(w).view(np.uint32)), w


@pytest.mark.parametrize("gather_mode", [0, 1, 2])
def test_search_bit_exact_vs_rn_oracle(workload, gather_mode):
    cfg, run, la, (od, ol, tol) = workload
    got, *_ = product_search(run, la, cfg.params_dict(), gather_mode=gather_mode)
    ref = oracle_search(run, la, cfg.params_dict(), oracle.LOG_RN, od, ol, tol)
    assert len(ref["rank"]) > 0
    assert_candidates_equal(got, ref, exact_scores=True, where=f"{cfg.name}/mode{gather_mode}")


@pytest.mark.parametrize("cycles_per_lane", [4, 8, 10, 12, 16])
def test_search_bit_exact_every_lane_width(workload, cycles_per_lane):
    """Every compiled cycles-per-lane instance gives the same bits (one pass or
    several per RT window)."""
    cfg, run, la, (od, ol, tol) = workload
    got, *_ = product_search(run, la, cfg.params_dict(), cycles_per_lane=cycles_per_lane)
    ref = oracle_search(run, la, cfg.params_dict(), oracle.LOG_RN, od, ol, tol)
    assert_candidates_equal(got, ref, exact_scores=True, where=f"{cfg.name}/S{cycles_per_lane}")


def test_graph_replay_matches_direct(workload):
    """use_graph: the first search runs directly and is captured; the next ones
    replay the graph (into the same collection) and give the same candidates."""
    cfg, run, la, _ = workload
    ref, dia, lib, _ = product_search(run, la, cfg.params_dict())
    from alphadia_search_rs_b200 import PeakGroupSelection

    from _util import COLS, params_from

    sel = PeakGroupSelection(params_from(cfg.params_dict()), verbose=False, use_graph=True)
    cand = sel.new_candidates()
    for call in range(3):
        sel.search_into(dia, lib, cand)
        n = cand.size()
        got = {c: np.zeros(n, np.float32 if c == "score" else np.uint64) for c in COLS}
        cand.copy_out(got)
        assert_candidates_equal(got, ref, exact_scores=True, where=f"{cfg.name}/graph call {call}")


def test_autotune_keeps_results(workload):
    """The autotuner only changes launch shapes: the tuned search gives the same
    candidates, and a second call is served from the cache."""
    cfg, run, la, _ = workload
    ref, dia, lib, _ = product_search(run, la, cfg.params_dict())
    from alphadia_search_rs_b200 import PeakGroupSelection

    from _util import COLS, params_from

    sel = PeakGroupSelection(params_from(cfg.params_dict()), verbose=False)
    choice = sel.autotune(dia, lib, repeats=1)
    assert choice["warps_per_block"] in (2, 4, 8)
    assert choice["cycles_per_lane"] in (0, 4, 8, 10, 12, 16)
    assert choice["ms"] > 0
    assert sel.autotune(dia, lib) == choice
    got = dict(zip(COLS, sel.search(dia, lib).to_arrays()))
    assert_candidates_equal(got, ref, exact_scores=True, where=f"{cfg.name}/tuned {choice}")


def test_search_vs_reference_numerics(workload):
    cfg, run, la, (od, ol, tol) = workload
    got, *_ = product_search(run, la, cfg.params_dict())
    ref = oracle_search(run, la, cfg.params_dict(), oracle.LOG_GLIBC, od, ol, tol)
    assert_candidates_equal(got, ref, exact_scores=False, where=cfg.name)


def test_search_deterministic(workload):
    cfg, run, la, _ = workload
    a, *_ = product_search(run, la, cfg.params_dict())
    b, *_ = product_search(run, la, cfg.params_dict(), warps_per_block=2)
    for k in a:
        assert np.array_equal(np.asarray(a[k]).view(np.uint8), np.asarray(b[k]).view(np.uint8)), k


@pytest.mark.parametrize("variant", [
    dict(),
    dict(peak_length=15),              # center - peak_length wraps as usize
    dict(kernel_size=9, fwhm_rt=2.0),
    dict(kernel_size=62),              # widest kernel with taps in kernel parameters
    dict(kernel_size=63),              # taps from device memory, bitmap read below cycle 0
    dict(kernel_size=70, fwhm_rt=12.0),
    dict(kernel_size=101),             # wider than the run: no output anywhere
    dict(kernel_size=21),              # unrolled stencil, half width 11
    dict(kernel_size=31, fwhm_rt=7.0), # unrolled stencil, half width 16
    dict(kernel_size=14),              # generic stencil, half width 7
    dict(candidate_count=0),
    dict(candidate_count=50),
    dict(top_k_fragments=0),
    dict(top_k_fragments=3),
    dict(mass_tolerance=200.0),        # wide bin ranges (binary-search gather)
    dict(rt_tolerance=5.0),            # minimum tolerance (10 + kernel_size) * delta_t applies
    dict(rt_tolerance=1000.0),
])
def test_edge_cases(variant):
    run, la = edge_case_workload()
    params = dict(fwhm_rt=3.0, kernel_size=20, peak_length=5, mass_tolerance=20.0,
                  rt_tolerance=30.0, candidate_count=3, top_k_fragments=6)
    params.update(variant)
    got, *_ = product_search(run, la, params)
    ref = oracle_search(run, la, params, oracle.LOG_RN)
    assert_candidates_equal(got, ref, exact_scores=True, where=str(variant))
    ref_g = oracle_search(run, la, params, oracle.LOG_GLIBC)
    assert_candidates_equal(got, ref_g, exact_scores=False, where=str(variant))


@pytest.mark.parametrize("value", [np.inf, 1e-30])
def test_extreme_library_intensity(value):
    """An infinite library intensity makes ln(0 + 1) * inf = NaN in every column
    of the score, as in the reference; a tiny one only scales its row."""
    run, la = edge_case_workload()
    la = dict(la)
    fi = np.array(la["fragment_intensity"], dtype=np.float32, copy=True)
    fi[1] = value
    la["fragment_intensity"] = fi
    params = dict(fwhm_rt=3.0, kernel_size=20, peak_length=5, mass_tolerance=20.0,
                  rt_tolerance=30.0, candidate_count=3, top_k_fragments=6)
    got, *_ = product_search(run, la, params)
    ref = oracle_search(run, la, params, oracle.LOG_RN)
    assert_candidates_equal(got, ref, exact_scores=True, where=f"intensity {value}")


def test_edge_case_csr():
    run, la = edge_case_workload()
    from alphadia_search_rs_b200 import DIAData

    od, _, _ = oracle_inputs(run, la)
    dia = DIAData.from_arrays(*(run[k] for k in RUN_KEYS), run["cycle"])
    assert dia.num_observations == od.num_observations == 5
    for w in range(5):
        o = dia.observation(w)
        assert np.array_equal(o["slice_starts"], od.slice_starts(w))
        assert np.array_equal(o["cycle_indices"], od.cycles(w))
    assert dia.get_valid_observations(425.0) == od.valid_observations(425.0) == [1, 2]


def test_empty_library():
    run, la = edge_case_workload()
    la = {k: v[:0] for k, v in la.items()}
    got, *_ = product_search(run, la, dict(candidate_count=3))
    assert all(len(v) == 0 for v in got.values())


def test_device_inputs_match_host_inputs():
    import torch

    from alphadia_search_rs_b200 import DIAData, PeakGroupSelection, SpecLibFlat

    from _util import params_from

    cfg, lib, run = synth.make_workload("tiny", "numpy")
    la = synth.library_arrays(lib)
    host, *_ = product_search(run, la, cfg.params_dict())
    dev = {k: torch.from_numpy(np.ascontiguousarray(run[k])).cuda() for k in RUN_KEYS}
    dia = DIAData.from_arrays(*(dev[k] for k in RUN_KEYS), run["cycle"])
    ldev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in la.items()}
    sl = SpecLibFlat.from_arrays(**ldev)
    cand = PeakGroupSelection(params_from(cfg.params_dict()), verbose=False).search(dia, sl)
    arrs = cand.to_arrays()
    for k, a in zip(host, arrs):
        assert np.array_equal(np.asarray(host[k]).view(np.uint8), a.view(np.uint8)), k


def test_verbose_prints_reference_lines(capfd):
    from alphadia_search_rs_b200 import PeakGroupSelection

    from _util import params_from

    cfg, lib, run = synth.make_workload("tiny", "numpy")
    la = synth.library_arrays(lib)
    _, dia, sl, _ = product_search(run, la, cfg.params_dict())
    cand = PeakGroupSelection(params_from(cfg.params_dict())).search(dia, sl)
    out = capfd.readouterr().out
    assert "Precursors per second:" in out
    assert f"Found {cand.len()} candidates" in out


def test_statistics_pass_counts(workload):
    """The statistics pass: every searched fragment row spans at least one and at most
    all cycles, and each accumulated entry was read."""
    cfg, run, la, _ = workload
    from alphadia_search_rs_b200 import PeakGroupSelection

    from _util import params_from

    _, dia, lib, _ = product_search(run, la, cfg.params_dict())
    sel = PeakGroupSelection(params_from(cfg.params_dict()), verbose=False)
    sel.enable_stats(True)
    sel.search(dia, lib)
    st = sel.last_stats()
    n_cycles = len(dia.rt_index()[0])
    assert st["fragments"] > 0
    assert st["fragments"] <= st["xic_cells"] <= st["fragments"] * n_cycles
    assert st["entries_accumulated"] <= st["entries_read"]


@pytest.mark.parametrize("where", ["host", "device"])
@pytest.mark.parametrize("fault", ["range", "rt_nan", "rt_inf"])
def test_library_validation(where, fault):
    """SpecLibFlat.from_arrays rejects what the reference would panic on (a fragment
    range outside the fragment arrays, a non-finite precursor RT) with ValueError,
    for host arrays and for CUDA tensors, and the library built afterwards works."""
    import torch

    from alphadia_search_rs_b200 import SpecLibFlat

    cfg, lib, run = synth.make_workload("tiny", "numpy")
    la = {k: np.array(v, copy=True) for k, v in synth.library_arrays(lib).items()}
    if fault == "range":
        la["flat_frag_stop_idx"][5] = np.uint64(len(la["fragment_mz"]) + 3)
    else:
        la["precursor_rt"][7] = np.float32(np.nan if fault == "rt_nan" else np.inf)
    if where == "device":
        la = {k: torch.as_tensor(v.view(np.int64) if v.dtype == np.uint64 else v, device="cuda:0")
              for k, v in la.items()}
        for k in ("precursor_idx", "flat_frag_start_idx", "flat_frag_stop_idx"):
            la[k] = la[k].view(torch.uint64)
    with pytest.raises(ValueError, match="fragment range|RT is not finite"):
        SpecLibFlat.from_arrays(**la)
    ok = SpecLibFlat.from_arrays(**synth.library_arrays(lib))
    assert ok.num_precursors == len(synth.library_arrays(lib)["precursor_idx"])


@pytest.mark.parametrize("top_k", [6, 12, 32, 33, 60])
def test_many_fragments_top_k(top_k):
    """Precursors with 20-60 library fragments searched with top-k below, at and above
    one warp's worth of fragments: the library preparation's multi-pass selection and
    the search kernel's fragments past the first 32 stay bit-exact."""
    cfg, lib, run = synth.make_workload("tiny_many", "numpy")
    la = synth.library_arrays(lib)
    params = dict(cfg.params_dict(), top_k_fragments=top_k)
    got, *_ = product_search(run, la, params)
    ref = oracle_search(run, la, params, oracle.LOG_RN)
    assert len(ref["rank"]) > 0
    assert_candidates_equal(got, ref, exact_scores=True, where=f"top-{top_k}")



@pytest.mark.parametrize("kernel_size,fwhm_rt", [(63, 10.0), (128, 30.0), (301, 60.0)])
def test_wide_kernels(kernel_size, fwhm_rt):
    """Gaussian kernels wider than 62 (the reference accepts any width,
    src/kernel/mod.rs:13-30) on windows of up to 2300 cycles: bit-exact against the
    oracle, in shared-memory and global-memory classes."""
    cfg, lib, run = synth.make_workload("tiny_long", "numpy")
    la = synth.library_arrays(lib)
    params = dict(cfg.params_dict(), kernel_size=kernel_size, fwhm_rt=fwhm_rt)
    got, *_ = product_search(run, la, params)
    ref = oracle_search(run, la, params, oracle.LOG_RN)
    assert len(ref["rank"]) > 0
    assert_candidates_equal(got, ref, exact_scores=True, where=f"kernel_size {kernel_size}")


def test_statistics_pass_with_wide_kernel_and_long_windows():
    """The statistics pass runs the generic-half-width instances with the counters
    compiled in: same candidates as the search, and counts that add up."""
    from alphadia_search_rs_b200 import PeakGroupSelection

    from _util import COLS, params_from

    cfg, lib, run = synth.make_workload("tiny_long", "numpy")
    la = synth.library_arrays(lib)
    params = dict(cfg.params_dict(), kernel_size=101, fwhm_rt=25.0)
    ref, dia, slib, _ = product_search(run, la, params)
    sel = PeakGroupSelection(params_from(params), verbose=False)
    sel.enable_stats(True)
    got = dict(zip(COLS, sel.search(dia, slib).to_arrays()))
    assert_candidates_equal(got, ref, exact_scores=True, where="statistics pass")
    st = sel.last_stats()
    assert st["pairs"] > 0 and st["entries_accumulated"] <= st["entries_read"]
    assert st["fragments"] <= st["xic_cells"]
