"""Host-side helpers of bench.py that shape the reported line (no GPU needed)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from alphadia_search_rs_b200 import synth  # noqa: E402


def test_cpu_sample_windows_are_bounded_by_peaks():
    # about 72 M peaks' worth of consecutive MS2 windows, whatever the run's shape
    assert bench.sample_windows(synth.get_config("cfg1"), 0) == 24
    assert bench.sample_windows(synth.get_config("cfg4"), 0) == 8
    assert bench.sample_windows(synth.get_config("cfg0"), 0) == 8  # all of its windows
    assert bench.sample_windows(synth.get_config("cfg1"), 5) == 5
    assert bench.sample_windows(synth.get_config("cfg0"), 50) == 8


def _rows(*rows):
    keys = ("precursor_idx", "rank", "cycle_center", "score")
    return {k: np.array([r[i] for r in rows]) for i, k in enumerate(keys)}


def test_bf16_agreement_counts_matching_cycles_and_relative_errors():
    ref = _rows((7, 0, 100, 10.0), (7, 1, 200, 5.0), (9, 0, 50, 2.0))
    ref["score_f64"] = ref.pop("score").astype(np.float64)
    got = _rows((7, 0, 100, 10.01), (7, 1, 201, 5.0), (9, 0, 50, 2.0))
    agree, errs = bench.bf16_agreement(got, ref)
    assert abs(agree - 2 / 3) < 1e-12
    assert np.allclose(sorted(errs), [0.0, 0.001])


def test_bf16_agreement_floors_the_denominator_near_zero():
    # a score of 1e-9 next to the precursor's 10.0 is compared against 1e-3 * 10.0
    ref = _rows((3, 0, 10, 10.0), (3, 1, 20, 1e-9))
    ref["score_f64"] = ref.pop("score").astype(np.float64)
    got = _rows((3, 0, 10, 10.0), (3, 1, 20, 1e-4))
    agree, errs = bench.bf16_agreement(got, ref)
    assert agree == 1.0
    assert abs(max(errs) - (1e-4 - 1e-9) / 1e-2) < 1e-9


def test_traffic_comes_from_the_committed_profiles():
    # DRAM bytes of one search's search_kernel launches, per workload and precision
    assert bench.load_traffic("cfg3", "bf16") > bench.load_traffic("cfg3", "fp32") * 0.5
    assert bench.load_traffic("cfg1", "fp32") > 0
    assert bench.load_traffic("cfg1", "bf16") is None


def test_both_arms_print_the_same_config():
    cfg = synth.get_config("cfg3")
    a = bench.bench_config(cfg, "bf16", 1)
    assert a == bench.bench_config(cfg, "bf16", 1)
    assert a["workload"].startswith("cfg3") and "per precursor" in a["rt_tolerance"]


def test_host_copies_keep_shared_columns_shared():
    """Columns that are one array (the synthetic library's m/z and library m/z) stay
    one array after the host copy: the library upload then copies the m/z once, and
    the bench's H2D count leaves the second name out."""
    import torch

    mz = torch.arange(5, dtype=torch.float32)
    other = torch.ones(5)
    out = bench.host_copies({"fragment_mz": mz, "fragment_mz_library": mz, "fragment_intensity": other},
                            lambda t: t.clone())
    assert out["fragment_mz"] is out["fragment_mz_library"]
    assert out["fragment_intensity"] is not out["fragment_mz"]
    assert torch.equal(out["fragment_mz"], mz) and out["fragment_mz"] is not mz
