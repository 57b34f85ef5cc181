"""The oracle's restatement of PeakGroupScoring and its helpers, pinned by the values
of the reference crate's own unit tests (src/peak_group_scoring/tests.rs,
src/utils/tests.rs, src/idf/tests.rs), plus structural checks of the dense XIC/m/z
extraction (src/quadrupole_observation/mod.rs:152-211) on a synthetic run."""
import math

import numpy as np
import pytest

B, Y, A, Cc, X, Z = 98, 121, 97, 99, 120, 122  # src/constants.rs:4-9


def f32(x):
    return float(np.float32(x))


def test_median_axis_0(orc):  # src/peak_group_scoring/tests.rs:13-34
    assert orc.sc_median_axis0(np.array([[1, 2, 3], [4, 5, 6], [7, 8, 9]])).tolist() == [4, 5, 6]
    assert orc.sc_median_axis0(np.array([[1, 2], [3, 4], [5, 6], [7, 8]])).tolist() == [4, 5]
    assert orc.sc_median_axis0(np.array([[1, 2], [3, 4], [5, 6]])).tolist() == [3, 4]
    # no rows: zeros (utils.rs:39-42); non-zero rows only (utils.rs:7-29)
    assert orc.sc_median_axis0(np.array([[0, 0], [0, 0]]), non_zero_only=True).tolist() == [0, 0]
    assert orc.sc_median_axis0(np.array([[0, 0], [2, 4], [6, 8]]), non_zero_only=True).tolist() == [4, 6]


def test_normalize_profiles(orc):  # src/peak_group_scoring/tests.rs:37-103
    r = orc.sc_normalize_profiles(np.array([[1, 2, 3, 4, 5], [2, 4, 6, 8, 10], [0, 0, 0, 0, 0]]))
    assert r[0].tolist() == [f32(1 / 3), f32(2 / 3), 1.0, f32(4 / 3), f32(5 / 3)]
    assert r[1].tolist() == [f32(np.float32(2) / np.float32(6)), f32(np.float32(4) / np.float32(6)), 1.0,
                             f32(np.float32(8) / np.float32(6)), f32(np.float32(10) / np.float32(6))]
    assert r[2].tolist() == [0.0] * 5
    r = orc.sc_normalize_profiles(np.array([[1, 2], [3, 4]]))
    assert r[0].tolist() == [f32(np.float32(1) / np.float32(1.5)), f32(np.float32(2) / np.float32(1.5))]
    assert r[1].tolist() == [f32(np.float32(3) / np.float32(3.5)), f32(np.float32(4) / np.float32(3.5))]
    r = orc.sc_normalize_profiles(np.array([[1, 0, 3], [1, 2, 3]]), dilations=0)  # zero center
    assert r[0].tolist() == [0.0, 0.0, 0.0]
    assert r[1].tolist() == [0.5, 1.0, 1.5]


def test_correlation(orc):  # src/peak_group_scoring/tests.rs:106-190
    med = [1.0, 2.0, 3.0]
    assert abs(orc.sc_correlation(med, [1, 2, 3]) - 1.0) < 1e-6
    assert abs(orc.sc_correlation(med, [2, 4, 6]) - 1.0) < 1e-6
    assert abs(orc.sc_correlation(med, [3, 2, 1]) + 1.0) < 1e-6
    assert orc.sc_correlation(med, [0, 0, 0]) == 0.0
    assert abs(orc.sc_correlation([1, 2], [1, 2]) - 1.0) < 1e-6
    assert orc.sc_correlation([1, 2], [1, 1]) == 0.0
    assert orc.sc_correlation([1, 2], [0, 0]) == 0.0
    assert orc.sc_correlation(med, [1, 2]) == 0.0
    assert orc.sc_correlation([1, 2, 3], [1, 1, 1]) == 0.0
    assert orc.sc_correlation([0, 0, 0], [1, 2, 3]) == 0.0


def test_hyperscore(orc):  # src/peak_group_scoring/tests.rs:193-345
    assert orc.sc_hyperscore([B, Y, B, Y, A], [100, 200, 150, 250, 50], [1, 1, 1, 1, 0]) > 0
    assert orc.sc_hyperscore([B, Y, B, Y], [100, 200, 150, 250], [0, 0, 0, 0]) == 0.0
    assert orc.sc_hyperscore([B, B, B], [100, 200, 150], [1, 1, 1]) > 0
    assert orc.sc_hyperscore([Y, Y, Y], [100, 200, 150], [1, 1, 1]) > 0
    assert orc.sc_hyperscore([B, Y, Cc, X, B, Y], [100, 200, 50, 75, 150, 250], [1] * 6) > 0
    h = orc.sc_hyperscore([B, B, Y, Y], [100, 200, 150, 250], [1, 1, 1, 1])
    assert 10.0 < h < 20.0
    # the same value written out: Stirling's ln(2!) twice plus ln(300) + ln(400)
    g = orc.sc_gamma_ln(3.0)
    expect = np.float32(np.float32(np.float32(g + g) + np.float32(math.log(300))) + np.float32(math.log(400)))
    assert abs(h - float(expect)) <= 2e-6 * abs(h)
    h1 = orc.sc_hyperscore([B, Y], [50, 75], [1, 1])
    assert 7.0 < h1 < 10.0
    assert abs(h1 - (math.log(50) + math.log(75))) < 1e-5  # ln(1!) = 0 exactly (utils.rs:302-304)


def test_gamma_ln_special_cases(orc):  # src/peak_group_scoring/utils.rs:293-312
    assert orc.sc_gamma_ln(0.0) == 0.0 and orc.sc_gamma_ln(-1.0) == 0.0
    assert orc.sc_gamma_ln(1.0) == 0.0 and orc.sc_gamma_ln(2.0) == 0.0
    x = np.float32(5.0)
    expect = (x - np.float32(0.5)) * np.float32(math.log(5.0)) - x + np.float32(0.5) * np.float32(1.837877)
    assert abs(orc.sc_gamma_ln(5.0) - float(expect)) < 1e-5


@pytest.mark.parametrize("types,numbers,mask,expect", [  # src/peak_group_scoring/tests.rs:347-611
    ([B, B, B, Y, Y, Y], [1, 2, 3, 1, 2, 3], [1] * 6, (3, 3)),
    ([B, B, B, Y, Y], [1, 3, 4, 1, 3], [1] * 5, (2, 1)),
    ([B, B, B, B, Y, Y, Y], [1, 2, 3, 4, 1, 2, 3], [1, 0, 1, 1, 1, 1, 0], (2, 2)),
    ([B, Y, B], [1, 1, 2], [0, 0, 0], (0, 0)),
    ([B, B, B, B], [1, 2, 4, 5], [1] * 4, (2, 0)),
    ([Y, Y, Y, Y], [2, 3, 4, 6], [1] * 4, (0, 3)),
    ([], [], [], (0, 0)),
    ([B, B, B], [3, 1, 2], [1, 1, 1], (3, 0)),
    ([B, B, B, B, Y, Y], [2, 2, 2, 2, 3, 3], [1] * 6, (1, 1)),
])
def test_longest_ion_series(orc, types, numbers, mask, expect):
    assert orc.sc_longest_ion_series(types, numbers, mask) == expect


def test_longest_ion_series_mismatched_lengths(orc):
    assert orc.sc_longest_ion_series([B, Y], [1, 2, 3], [1, 1]) == (0, 0)


def test_hyperscore_inverse_mass_error(orc):  # src/peak_group_scoring/tests.rs:614-749
    def inv(errs):
        return [1.0 / (abs(np.float32(e)) + np.float32(0.1)) for e in errs]

    s = orc.sc_hyperscore([B, B, Y, Y], [100, 200, 150, 250], [1] * 4, inv([1.0, 2.0, 0.5, 3.0]))
    assert s > 0 and math.isfinite(s)
    assert orc.sc_hyperscore([B, B, Y, Y], [100, 0, 150, 0], [1] * 4, inv([1.0, 2.0, 0.5, 3.0])) > 0
    assert orc.sc_hyperscore([B, Y], [0, 0], [1, 1], inv([1.0, 2.0])) == 0.0
    s = orc.sc_hyperscore([B, Y], [100, 100], [1, 1], inv([1000.0, 2000.0]))
    assert s != 0.0 and math.isfinite(s)
    small = orc.sc_hyperscore([B, Y], [100, 100], [1, 1], inv([0.01, 0.02]))
    large = orc.sc_hyperscore([B, Y], [100, 100], [1, 1], inv([10.0, 20.0]))
    assert small > large


def test_intensity_ion_series(orc):  # src/peak_group_scoring/tests.rs:752-910
    t, i = [B, B, Y, Y, A], [100, 200, 150, 250, 75]
    assert orc.sc_intensity_ion_series(t, i, [1] * 5, B) == 300.0
    assert orc.sc_intensity_ion_series(t, i, [1] * 5, Y) == 400.0
    assert orc.sc_intensity_ion_series([B, Y], [100, 200], [0, 1], B) == 0.0
    assert orc.sc_intensity_ion_series([B, Y], [100, 200], [0, 1], Y) == 200.0
    assert orc.sc_intensity_ion_series([B, Y], [0, 200], [1, 1], B) == 0.0
    assert orc.sc_intensity_ion_series([], [], [], B) == 0.0
    t, i = [A, B, Cc, X, Y, Z], [50, 100, 75, 80, 200, 60]
    for typ, v in zip(t, i):
        assert orc.sc_intensity_ion_series(t, i, [1] * 6, typ) == v
    assert orc.sc_intensity_ion_series([B, Y, A], [100, 200, 50], [1, 1, 1], Cc) == 0.0


def test_fwhm_and_dot(orc):  # src/peak_group_scoring/tests.rs:913-980
    fw = orc.sc_fwhm_rt([0, 50, 100, 50, 0], 10, np.arange(17, dtype=np.float32))
    assert 0.0 < fw < 5.0 and fw == 2.0
    assert orc.sc_fwhm_rt([], 0, np.arange(6, dtype=np.float32)) == 0.0
    assert orc.sc_dot([1, 2, 3], [4, 5, 6]) == 32.0
    assert orc.sc_dot([], []) == 0.0
    assert orc.sc_dot([1, 2], [3, 4, 5]) == 0.0
    assert orc.sc_dot([1, 2, 3], [0, 0, 0]) == 0.0


def test_weighted_mean_and_mass_errors(orc):  # src/utils/tests.rs:5-272
    def wmean(values, weights):
        mo, _ = orc.sc_fragment_mz_errors(np.array(values), np.array(weights), np.ones(len(values)))
        return mo

    r = wmean([[10, 20, 30], [5, 15, 25]], [[1, 2, 3], [4, 0, 2]])
    assert abs(r[0] - 23.333334) < 1e-5 and abs(r[1] - 11.666667) < 1e-5
    r = wmean([[10, 20, 30], [5, 15, 25]], [[1, 2, 3], [0, 0, 0]])
    assert abs(r[0] - 23.333334) < 1e-5 and r[1] == 0.0
    assert wmean([[42.0]], [[2.5]]).tolist() == [42.0]
    r = wmean([[100, 200, 300, 400], [10, 20, 30, 40]], [[1, 0, 3, 0], [0, 2, 0, 4]])
    assert r[0] == 250.0 and abs(r[1] - 33.333332) < 1e-5
    mo, err = orc.sc_fragment_mz_errors(np.array([[200.01, 200.02, 200.03], [300.05, 300.10, 300.15], [0, 0, 0]]),
                                        np.array([[1000, 2000, 3000], [500, 1000, 500], [0, 0, 0]]),
                                        [200.0, 300.0, 400.0])
    assert abs(mo[0] - 200.02333) < 1e-5 and abs(err[0] - 116.67) < 0.1
    assert abs(mo[1] - 300.1) < 1e-5 and abs(err[1] - 333.33) < 0.1
    assert mo[2] == 0.0 and err[2] == 0.0
    mo, err = orc.sc_fragment_mz_errors(np.array([[250.005]]), np.array([[1500.0]]), [250.0])
    assert mo[0] == f32(250.005) and abs(err[0] - 20.0) < 0.1
    mo, err = orc.sc_fragment_mz_errors(np.array([[150.01, 0, 150.03, 0], [0, 200.02, 0, 200.04]]),
                                        np.array([[1000, 0, 2000, 0], [0, 3000, 0, 1000]]), [150.0, 200.0])
    assert abs(mo[0] - 150.02333) < 1e-5 and abs(err[0] - 155.56) < 0.2
    assert abs(mo[1] - 200.025) < 1e-5 and abs(err[1] - 125.0) < 0.1


def test_weighted_mean_absolute_error(orc):  # src/utils/tests.rs:89-195
    assert abs(orc.sc_weighted_mae([10, -20, 30, -40], [1, 2, 3, 4]) - 30.0) < 1e-5
    assert abs(orc.sc_weighted_mae([10, -20, 30, -40], [1, 0, 3, 0]) - 25.0) < 1e-5
    assert abs(orc.sc_weighted_mae([10, 0, 30, 0], [1, 2, 3, 4]) - 25.0) < 1e-5
    assert orc.sc_weighted_mae([10, -20, 30], [0, 0, 0]) == 0.0
    assert orc.sc_weighted_mae([], []) == 0.0
    assert orc.sc_weighted_mae([10, -20], [1, 2, 3]) == 0.0
    assert orc.sc_weighted_mae([25.0], [2.0]) == 25.0
    assert abs(orc.sc_weighted_mae([10, 20, 30], [1, -2, 3]) - 25.0) < 1e-5


def test_median_std(orc):  # src/utils/tests.rs:275-293
    assert orc.sc_median([3, 1, 4, 1, 5]) == 3.0
    assert orc.sc_median([2, 4, 1, 3]) == 2.5
    assert orc.sc_median([42.0]) == 42.0
    assert orc.sc_median([]) == 0.0
    assert orc.sc_median([-3, 1, -1, 3, 0]) == 0.0
    assert math.isnan(orc.sc_median([1.0, float("nan"), 3.0]))
    assert abs(orc.sc_std([1, 2, 3, 4, 5]) - 1.5811) < 1e-4
    assert orc.sc_std([42.0]) == 0.0 and orc.sc_std([]) == 0.0
    assert abs(orc.sc_std([1, 5]) - 2.8284) < 1e-4
    assert orc.sc_std([7, 7, 7]) == 0.0
    assert orc.sc_std([-2, 0, 2]) == 2.0


@pytest.mark.parametrize("values,r1,r2,expect", [  # src/utils/tests.rs:295-400
    ([1, 3, 2], 0, 2, [0, 1, 1]),
    ([1, 1, 1], 0, 2, [1, 1, 0]),
    ([1, 2, 3], 0, 0, [0, 0, 0]),
    ([], 0, 5, []),
    ([1, 2, 3], 0, 5, [1, 1, 1]),
    ([42.0], 0, 1, [1]),
    ([42.0], 0, 0, [0]),
    ([42.0], 1, 2, [0]),
    ([5, 4, 3, 2, 1], 0, 3, [1, 1, 1, 0, 0]),
    ([1, 2, 3, 4, 5], 0, 3, [0, 0, 1, 1, 1]),
    ([-1, 2, -3, 4], 0, 2, [0, 1, 0, 1]),
    ([5, 1, 3, 2, 4], 0, 2, [1, 0, 0, 0, 1]),
    ([5, 1, 3, 2, 4], 1, 3, [0, 0, 1, 0, 1]),
    ([5, 1, 3, 2, 4], 3, 5, [0, 1, 0, 1, 0]),
])
def test_ranked_mask(orc, values, r1, r2, expect):
    assert orc.sc_ranked_mask(values, r1, r2).tolist() == [bool(e) for e in expect]


def test_count_values_above(orc):  # src/utils/tests.rs:402-440
    assert orc.sc_count_above([1, 2, 3, 4], 2.5) == 2
    assert orc.sc_count_above([1, 2, 3, 4], 0.0) == 4
    assert orc.sc_count_above([1, 2, 3, 4], 5.0) == 0
    assert orc.sc_count_above([], 1.0) == 0
    assert orc.sc_count_above([2, 2, 2], 2.0) == 0
    assert orc.sc_count_above([1, 2, 3, 4], 1.5, [1, 0, 1, 0]) == 1
    assert orc.sc_count_above([1, 2, 3, 4], 1.5, [1, 1, 1, 1]) == 3
    assert orc.sc_count_above([1, 2, 3, 4], 0.0, [0, 0, 0, 0]) == 0
    assert orc.sc_count_above([1, 2, 3, 4], 0.0, [1, 1]) == 0


def _tiny_run(orc):
    from alphadia_search_rs_b200 import synth

    cfg, lib, run = synth.make_workload("tiny", "numpy")
    keys = ("spectrum_delta_scan_idx", "isolation_lower_mz", "isolation_upper_mz", "spectrum_peak_start_idx",
            "spectrum_peak_stop_idx", "spectrum_cycle_idx", "spectrum_rt", "peak_mz", "peak_intensity")
    return cfg, lib, run, orc.Dia(**{k: run[k] for k in keys})


def _lib_with_fragments(orc, mz_library):
    n = len(mz_library)
    lb = orc.Lib(np.array([0], np.uint64), [500.0], [10.0], np.array([0], np.uint64),
                 np.array([n], np.uint64), np.asarray(mz_library, np.float32), np.ones(n, np.float32),
                 np.full(n, 2, np.uint8), np.full(n, B, np.uint8))
    orc.lib_set_scoring(lb, [7], mz_library)
    return lb


def test_idf(orc):  # src/idf/tests.rs:4-41
    _, _, _, dia = _tiny_run(orc)
    v = orc.sc_idf(dia, _lib_with_fragments(orc, [100.0, 100.0]), [100.0, 200.0])
    assert abs(v[0]) < 1e-6 and abs(v[1] - math.log(2.0)) < 1e-6
    assert orc.sc_idf(dia, _lib_with_fragments(orc, []), [100.0, 200.0, 300.0]).tolist() == [1.0, 1.0, 1.0]
    assert abs(orc.sc_idf(dia, _lib_with_fragments(orc, [150.0]), [150.0])[0]) < 1e-6


def test_dense_xic_mz_matches_dense_xic(orc):
    """The XIC half of the m/z-weighted extraction equals the plain XIC extraction
    (same bins, same entries, same order); the m/z half is a weighted mean of grid m/z
    values, so it lies inside each fragment's tolerance window wherever there is signal."""
    cfg, lib, run, dia = _tiny_run(orc)
    pmz = float(lib["precursor_mz"][0])
    fmz = np.asarray(lib["fragment_mz"][:12], np.float32)
    cs, ce = 20, 120
    xic, mz = orc.sc_dense_xic_mz(dia, pmz, cs, ce, 15.0, fmz)
    ref = dia.dense_xic(pmz, cs, ce, 15.0, fmz)
    assert np.array_equal(xic.view(np.uint32), np.asarray(ref, np.float32).reshape(xic.shape).view(np.uint32))
    assert (xic > 0).any()
    tol = fmz[:, None] * 15e-6 * 1.01
    sig = xic > 0
    assert np.all(np.abs(mz - fmz[:, None])[sig] <= np.broadcast_to(tol, mz.shape)[sig])
    assert np.all(mz[~sig] == 0)


def test_score_end_to_end_shapes(orc):
    """score() on the tiny run's own selection output: one row per candidate, in the
    candidates' order, with the counts and ranges the definitions imply."""
    cfg, lib, run, dia = _tiny_run(orc)
    from alphadia_search_rs_b200 import synth

    la = synth.library_arrays(lib)
    lb = orc.Lib(la["precursor_idx"], la["precursor_mz"], la["precursor_rt"], la["flat_frag_start_idx"],
                 la["flat_frag_stop_idx"], la["fragment_mz"], la["fragment_intensity"], la["fragment_number"],
                 la["fragment_type"])
    orc.lib_set_scoring(lb, la["precursor_naa"], la["fragment_mz_library"])
    cand = orc.search(dia, lb, orc.Params(**cfg.params_dict()))
    feats = orc.score(dia, lb, cand, mass_tolerance=15.0, top_k_fragments=12)
    n = len(cand["rank"])
    assert n > 0 and len(feats["rank"]) == n
    assert np.array_equal(feats["precursor_idx"], cand["precursor_idx"])
    assert np.array_equal(feats["rank"], cand["rank"])
    assert np.array_equal(feats["score"], cand["score"])
    assert np.all(feats["num_scans"] == (cand["cycle_stop"] - cand["cycle_start"]).astype(np.float32))
    assert np.all(feats["num_fragments"] == 12) and np.all(feats["num_profiles"] == 12)
    assert np.all(feats["num_profiles_filtered"] <= 12)
    for k in ("mean_correlation", "median_correlation", "intensity_correlation"):
        assert np.all(np.abs(feats[k]) <= 1.0)
    assert np.all(feats["num_over_95"] <= feats["num_over_50"])
    assert np.all(feats["num_over_50"] <= feats["num_over_0"])
    assert np.all(feats["naa"] == 10)
    rt = dia.rt
    assert np.array_equal(feats["rt_observed"], rt[cand["cycle_center"].astype(np.int64)])
    # candidates whose precursor is not in the library are skipped
    bad = dict(cand)
    bad["precursor_idx"] = cand["precursor_idx"].copy()
    bad["precursor_idx"][0] = np.uint64(10**9)
    assert len(orc.score(dia, lb, bad, mass_tolerance=15.0, top_k_fragments=12)["rank"]) == n - 1
