"""GPU: the BF16-storage search (peak intensities read as bfloat16, FP32 arithmetic
with the hardware log2) against the FP64 oracle.

Relative score error is taken against max(|s64|, 1e-3 * max |s64| of the
precursor), because scores near zero are common at the RT-window edges.  Bounds:
  * top-k candidate cycles: at least 99.5% identical to the oracle's (99% on the
    few-hundred-precursor cases);
  * scores: the target bound, 1e-3 relative, holds for the 99th percentile
    and the median, and is asserted there.  It cannot hold for the maximum:
    bfloat16 keeps 8 significant bits, so a stored intensity may be off by up to
    u = 2^-8 = 3.9e-3 relative (just above a power of two), and a score column fed
    by one such entry (a noise peak, or the tail of the Gaussian kernel, where
    ln(1 + c) ~ c) carries that error unchanged.  Conversely u bounds every score:
    a convolved value of non-negative intensities is within u, each ln(c + 1) term
    within u (ln(1 + c) >= c / (1 + c)), and the score, a positive-weighted sum of
    such terms, within u.  The maximum is asserted against u (plus f32 noise).
"""
import numpy as np
import pytest

import oracle
from alphadia_search_rs_b200 import synth

from _util import oracle_inputs, product_search

pytestmark = pytest.mark.gpu

BF16_U = 2.0 ** -8
SCORE_MAX_BF16 = BF16_U * 1.01
SCORE_P99_BF16 = 1e-3
EPS_REL_MAX = 1e-3


def compare_to_fp64(got: dict, ref: dict):
    """(fraction of the oracle's (precursor, rank) rows with the same cycle, the
    relative score errors over those rows)."""
    ref_max = {}
    for p, s in zip(ref["precursor_idx"], ref["score_f64"]):
        ref_max[int(p)] = max(ref_max.get(int(p), 0.0), abs(float(s)))
    mine = {(int(p), int(r)): (int(c), float(s)) for p, r, c, s in
            zip(got["precursor_idx"], got["rank"], got["cycle_center"], got["score"])}
    same, errs = 0, []
    for p, r, c, s in zip(ref["precursor_idx"], ref["rank"], ref["cycle_center"], ref["score_f64"]):
        m = mine.get((int(p), int(r)))
        if m is None or m[0] != int(c):
            continue
        same += 1
        den = max(abs(float(s)), EPS_REL_MAX * ref_max[int(p)])
        errs.append(abs(m[1] - float(s)) / den if den > 0 else 0.0)
    return same / max(len(ref["rank"]), 1), np.asarray(errs if errs else [0.0])


@pytest.mark.parametrize("name,min_agree", [("tiny", 0.99), ("tiny_uneven", 0.99), ("tiny_cfg4", 0.99),
                                            ("tiny_many", 0.99), ("tiny_long", 0.99),
                                            ("long_rt", 0.99), ("cfg0", 0.995)])
def test_bf16_against_fp64_oracle(name, min_agree):
    cfg, lib, run = synth.make_workload(name, "numpy")
    la = synth.library_arrays(lib)
    got, *_ = product_search(run, la, cfg.params_dict(), precision="bf16")
    od, ol, tol = oracle_inputs(run, la)
    ref = oracle.search(od, ol, oracle.Params(**cfg.params_dict()), rt_tolerance_per_precursor=tol,
                        log_mode=oracle.LOG_RN, precision=1)
    assert len(ref["rank"]) > 0
    agree, errs = compare_to_fp64(got, ref)
    assert agree >= min_agree, f"{name}: top-k cycle agreement {agree:.4f}"
    assert errs.max() <= SCORE_MAX_BF16, f"{name}: max relative score error {errs.max():.2e}"
    p99 = float(np.quantile(errs, 0.99))
    assert p99 <= SCORE_P99_BF16, f"{name}: 99th percentile relative score error {p99:.2e}"
    assert float(np.median(errs)) <= SCORE_P99_BF16


@pytest.mark.parametrize("name", ["tiny_uneven", "long_rt"])
def test_bf16_deterministic(name):
    """Every operation runs in a fixed order (XIC cells in CSR order, the stencil's taps,
    scores in fragment order), so the result does not depend on the launch shape."""
    cfg, lib, run = synth.make_workload(name, "numpy")
    la = synth.library_arrays(lib)
    a, *_ = product_search(run, la, cfg.params_dict(), precision="bf16")
    b, *_ = product_search(run, la, cfg.params_dict(), precision="bf16", warps_per_block=2)
    c, *_ = product_search(run, la, cfg.params_dict(), precision="bf16", warps_per_block=8)
    for k in a:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
        assert np.array_equal(np.asarray(a[k]), np.asarray(c[k])), k


def test_bf16_non_finite_library_intensity():
    """An infinite library intensity makes every column of the score NaN (ln(1) * inf),
    as in the FP32 path and the reference: no candidates for that precursor."""
    from _util import edge_case_workload

    run, la = edge_case_workload()
    la = dict(la)
    fi = np.array(la["fragment_intensity"], dtype=np.float32, copy=True)
    fi[1] = np.inf
    la["fragment_intensity"] = fi
    params = dict(fwhm_rt=3.0, kernel_size=20, peak_length=5, mass_tolerance=20.0,
                  rt_tolerance=30.0, candidate_count=3, top_k_fragments=6)
    f32, *_ = product_search(run, la, params)
    b16, *_ = product_search(run, la, params, precision="bf16")
    assert set(f32["precursor_idx"].tolist()) == set(b16["precursor_idx"].tolist())
    assert not np.isnan(b16["score"]).any()


def test_bf16_only_run_storage():
    """A run built with BF16-only intensity storage gives the same BF16 search as the
    f32 run (the same round-to-nearest values), holds less device memory, and refuses
    what needs f32 intensities."""
    from alphadia_search_rs_b200 import (DIAData, PeakGroupQuantification, PeakGroupScoring,
                                         PeakGroupSelection, QuantificationParameters,
                                         ScoringParameters, SpecLibFlat)

    from _util import COLS, RUN_KEYS, params_from

    cfg, lib, run = synth.make_workload("tiny_uneven", "numpy")
    la = synth.library_arrays(lib)
    ref, dia32, slib, _ = product_search(run, la, cfg.params_dict(), precision="bf16")
    dia16 = DIAData.from_arrays(*(run[k] for k in RUN_KEYS), run["cycle"], intensity_storage="bf16")
    assert dia16.device_bytes() < dia32.device_bytes()
    sel = PeakGroupSelection(params_from(cfg.params_dict()), verbose=False, precision="bf16")
    cand = sel.search(dia16, slib)
    got = dict(zip(COLS, cand.to_arrays()))
    for k in COLS:
        assert np.array_equal(np.asarray(got[k]).view(np.uint8), np.asarray(ref[k]).view(np.uint8)), k
    o32, o16 = dia32.observation(1), dia16.observation(1)
    assert np.array_equal(o32["cycle_indices"], o16["cycle_indices"])
    bits = o32["intensities"].view(np.uint32).astype(np.int64)  # finite, so no carry into NaN
    rne = ((bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    assert np.array_equal(o16["intensities"].view(np.uint32), rne)
    with pytest.raises(ValueError, match="bfloat16"):
        PeakGroupSelection(params_from(cfg.params_dict()), verbose=False).search(dia16, slib)
    with pytest.raises(ValueError, match="bfloat16"):
        PeakGroupScoring(ScoringParameters(), verbose=False).score(dia16, slib, cand)
    with pytest.raises(ValueError, match="bfloat16"):
        PeakGroupQuantification(QuantificationParameters(), verbose=False).quantify(dia16, slib, cand)


@pytest.mark.parametrize("kernel_size,fwhm_rt", [(64, 12.0), (128, 30.0)])
def test_bf16_wide_kernels_against_fp64_oracle(kernel_size, fwhm_rt):
    """BF16 storage with Gaussian kernels wider than 62 (taps from device memory)."""
    cfg, lib, run = synth.make_workload("tiny_long", "numpy")
    la = synth.library_arrays(lib)
    params = dict(cfg.params_dict(), kernel_size=kernel_size, fwhm_rt=fwhm_rt)
    got, *_ = product_search(run, la, params, precision="bf16")
    od, ol, tol = oracle_inputs(run, la)
    ref = oracle.search(od, ol, oracle.Params(**params), rt_tolerance_per_precursor=tol,
                        log_mode=oracle.LOG_RN, precision=1)
    assert len(ref["rank"]) > 0
    agree, errs = compare_to_fp64(got, ref)
    assert agree >= 0.99, f"kernel_size {kernel_size}: top-k cycle agreement {agree:.4f}"
    assert errs.max() <= SCORE_MAX_BF16
    assert float(np.quantile(errs, 0.99)) <= SCORE_P99_BF16
