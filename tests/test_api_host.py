"""Host-side behaviour of the reference-shaped Python API (no GPU needed).
Ports src/peak_group_selection/tests.rs:48-97, src/candidate/tests.rs:43-157 and
src/dia_data/tests.rs:214-300."""
import numpy as np
import pytest

import alphadia_search_rs_b200 as ads


def test_selection_parameter_defaults():  # src/peak_group_selection/tests.rs:48-59
    p = ads.SelectionParameters()
    assert p.fwhm_rt == 3.0 and p.kernel_size == 20 and p.peak_length == 5
    assert p.mass_tolerance == 7.0 and p.rt_tolerance == 200.0 and p.candidate_count == 3
    assert p.top_k_fragments == 12


def test_selection_parameter_update_partial():  # src/peak_group_selection/tests.rs:82-97
    p = ads.SelectionParameters()
    p.update({"rt_tolerance": 150.0})
    assert p.rt_tolerance == 150.0 and p.fwhm_rt == 3.0
    p.update({"fwhm_rt": 5, "kernel_size": 30, "peak_length": 8, "mass_tolerance": 12.0,
              "candidate_count": 4, "top_k_fragments": 24, "unknown_key": 1})
    assert (p.fwhm_rt, p.kernel_size, p.peak_length, p.mass_tolerance, p.candidate_count,
            p.top_k_fragments) == (5.0, 30, 8, 12.0, 4, 24)
    assert p.fwhm_rt == float(np.float32(5.0))
    p.update({"fwhm_rt": 0.1})
    assert p.fwhm_rt == float(np.float32(0.1))  # stored as f32


def test_selection_parameter_errors():
    p = ads.SelectionParameters()
    with pytest.raises(AttributeError):
        p.rt_tolerance = 1.0  # pyo3(get) only
    with pytest.raises(TypeError):
        p.update({"kernel_size": 2.5})
    with pytest.raises(OverflowError):
        p.update({"top_k_fragments": -1})
    with pytest.raises(TypeError):
        p.update({"fwhm_rt": "x"})
    assert p.kernel_size == 20  # failed updates leave the object unchanged


def test_selection_update_reads_keys_in_order():  # src/peak_group_selection/parameters.rs:45-68
    p = ads.SelectionParameters()
    with pytest.raises(TypeError):
        p.update({"top_k_fragments": 7.5, "fwhm_rt": 4.0, "candidate_count": 9})
    # fwhm_rt and candidate_count are read before the failing key
    assert (p.fwhm_rt, p.candidate_count, p.top_k_fragments) == (4.0, 9, 12)
    p.update({"fwhm_rt": True})  # extract::<f32> takes bool like int
    assert p.fwhm_rt == 1.0


def test_scoring_parameter_defaults():  # src/peak_group_scoring/parameters.rs:16-25
    p = ads.ScoringParameters()
    assert p.mass_tolerance == 7.0 and p.top_k_fragments == 100


def test_scoring_parameter_update():  # src/peak_group_scoring/parameters.rs:28-37
    p = ads.ScoringParameters()
    p.update({"mass_tolerance": 12, "other": "ignored"})
    assert p.mass_tolerance == 12.0 and p.top_k_fragments == 100
    p.update({"mass_tolerance": 0.1, "top_k_fragments": np.int64(24)})
    assert p.mass_tolerance == float(np.float32(0.1)) and p.top_k_fragments == 24
    with pytest.raises(AttributeError):
        p.mass_tolerance = 3.0
    with pytest.raises(TypeError):
        p.update({"mass_tolerance": 5.0, "top_k_fragments": 2.0})
    assert (p.mass_tolerance, p.top_k_fragments) == (5.0, 24)  # set before the failing key
    with pytest.raises(OverflowError):
        p.update({"top_k_fragments": -3})
    with pytest.raises(TypeError):
        p.update({"mass_tolerance": "7"})


def test_feature_names():  # src/candidate/features.rs:6-48, 413-416
    import oracle

    names = ads.CandidateFeatureCollection.get_feature_names()
    assert names == list(oracle.FEATURE_NAMES) and len(names) == 41
    assert names[0] == "score" and names[-1] == "num_over_50_top6_idf"


def test_empty_feature_collection():
    f = ads.CandidateFeatureCollection()
    assert f.is_empty() and len(f) == 0 and f.len() == 0 and f.kernel_ms() == 0.0
    d = f.to_dict_arrays()
    assert list(d)[:2] == ["precursor_idx", "rank"] and len(d) == 43
    assert d["precursor_idx"].dtype == np.uint64 and d["score"].dtype == np.float32


def test_scoring_argument_types():
    s = ads.PeakGroupScoring(ads.ScoringParameters(), verbose=False)
    with pytest.raises(TypeError):
        s.score(None, None, ads.CandidateCollection())
    with pytest.raises(TypeError):
        ads.PeakGroupScoring({"mass_tolerance": 7.0})


def test_quantification_parameters():  # src/peak_group_quantification/tests.rs:15-90
    p = ads.QuantificationParameters()
    assert p.tolerance_ppm == 7.0 and p.top_k_fragments == 10000
    p.tolerance_ppm = 12.0
    p.top_k_fragments = 50
    assert (p.tolerance_ppm, p.top_k_fragments) == (12.0, 50)
    p.update({"tolerance_ppm": 15.0})
    assert (p.tolerance_ppm, p.top_k_fragments) == (15.0, 50)
    p.update({"tolerance_ppm": 20.0, "top_k_fragments": 200})
    assert (p.tolerance_ppm, p.top_k_fragments) == (20.0, 200)
    p.update({})
    assert (p.tolerance_ppm, p.top_k_fragments) == (20.0, 200)
    with pytest.raises(TypeError):
        p.top_k_fragments = 1.5
    with pytest.raises(OverflowError):
        p.update({"top_k_fragments": -1})
    with pytest.raises(AttributeError):
        p.other = 1


def test_empty_quantified_library():  # src/speclib_flat_quantified/tests.rs:29-41
    q = ads.SpecLibFlatQuantified()
    assert q.num_precursors == 0 and q.num_fragments == 0
    prec, frag = q.to_dict_arrays()
    assert list(prec) == ["precursor_idx", "mz_library", "mz", "rt_library", "rt", "naa", "rank",
                          "rt_observed", "flat_frag_start_idx", "flat_frag_stop_idx"]
    assert list(frag) == ["mz_library", "mz", "intensity", "cardinality", "charge", "loss_type",
                          "number", "position", "type", "mz_observed", "correlation_observed",
                          "mass_error_observed", "precursor_idx", "rank"]
    with pytest.raises(TypeError):
        ads.PeakGroupQuantification(ads.QuantificationParameters(), verbose=False).quantify(None, None, None)


def test_candidate_collection_roundtrip():  # src/candidate/tests.rs:104-156
    cols = dict(precursor_idxs=[1, 2], ranks=[10, 20], scores=[0.1, 0.2], scan_center=[11, 21],
                scan_start=[12, 22], scan_stop=[13, 23], cycle_center=[14, 24], cycle_start=[15, 25],
                cycle_stop=[16, 26])
    c = ads.CandidateCollection.from_arrays(**cols)
    assert c.len() == 2 and not c.is_empty()
    out = c.to_arrays()
    assert len(out) == 9
    for a, (k, v) in zip(out, cols.items()):
        assert a.dtype == (np.float32 if k == "scores" else np.uint64)
        assert np.array_equal(a, np.asarray(v, a.dtype))


def test_candidate_collection_dtypes_and_order():  # src/candidate/tests.rs:43-102
    c = ads.CandidateCollection.from_arrays([42], [7], [1.5], [101], [100], [102], [201], [200], [202])
    p, r, s, sc, ss, so, cc, cs, co = c.to_arrays()
    assert (p[0], r[0], sc[0], ss[0], so[0], cc[0], cs[0], co[0]) == (42, 7, 101, 100, 102, 201, 200, 202)
    assert abs(s[0] - 1.5) < 1e-6


def test_candidate_collection_length_mismatch():  # src/candidate/entry.rs:85-102
    with pytest.raises(ValueError, match="same length"):
        ads.CandidateCollection.from_arrays([1], [1, 2], [0.1], [0], [0], [0], [0], [0], [0])


def test_empty_collection():
    c = ads.CandidateCollection()
    assert c.len() == 0 and c.is_empty()
    assert all(len(a) == 0 for a in c.to_arrays())


def test_empty_dia_data():  # src/dia_data/tests.rs:214-300
    d = ads.DIAData()
    assert d.num_observations == 0
    assert d.has_mobility is False and d.has_ms1 is False
    assert d.mobility_values == [1e-6, 0.0]
    assert len(d.rt_values) == 0
    assert d.cycle.shape == (0, 0, 0, 0)
    assert d.get_valid_observations(100.0) == []


def test_from_arrays_dtype_checks():
    z64 = np.zeros(1, np.int64)
    z32 = np.zeros(1, np.float32)
    cyc = np.zeros((1, 1, 1, 1), np.float32)
    with pytest.raises(TypeError):
        ads.DIAData.from_arrays(z64.astype(np.int32), z32, z32, z64, z64, z64, z32, z32, z32, cyc)
    with pytest.raises(TypeError):
        ads.DIAData.from_arrays(z64, z32, z32, z64, z64, z64, z32, z32, z32, np.zeros(1, np.float32))
    u8 = np.zeros(1, np.uint8)
    u64 = np.zeros(1, np.uint64)
    with pytest.raises(TypeError):
        ads.SpecLibFlat.from_arrays(u64.astype(np.int64), z32, z32, z32, z32, u8, u64, u64, z32, z32, z32,
                                    u8, u8, u8, u8, u8, u8)


def test_empty_speclib():
    lib = ads.SpecLibFlat()
    assert lib.num_precursors == 0 and lib.num_fragments == 0
