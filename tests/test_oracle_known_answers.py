"""Pins the CPU oracle to the reference crate's own known-answer tests.

Each test restates one reference test (file:line in MannLabs/alphadia-search-rs)
with the same inputs and the same expected values, run against the oracle
(oracle/oracle.cpp).  These are CPU-only.
"""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def grid(orc):
    return orc.ppm_index(1.0, 150.0, 2000.0)


# ---------------------------------------------------------------- mz_index
def test_ppm_index_len(orc):  # src/mz_index/tests.rs:80-84
    assert len(orc.ppm_index(1.0, 100.0, 2000.0)) == 2995974


def test_global_grid_len(grid):  # global grid (src/mz_index/mod.rs:4-6): 150..2000 at 1 ppm
    assert len(grid) == 2590781


@pytest.mark.parametrize("res,start,end", [(1.0, 100.0, 1000.0), (0.5, 200.0, 300.0), (2.0, 500.0, 600.0),
                                           (0.1, 500.0, 600.0), (10.0, 500.0, 600.0)])
def test_ppm_index_properties(orc, res, start, end):  # src/mz_index/tests.rs:86-172
    r = orc.ppm_index(res, start, end)
    assert len(r) > 1 and r[0] >= start and r[-1] <= end * 1.01
    ratio = np.float32(1.0) + np.float32(res) / np.float32(1e6)
    for i in range(1, min(10, len(r))):
        assert abs(float(r[i] / r[i - 1]) - float(ratio)) < 1e-6


def test_ppm_index_small_range_and_clamp(orc):  # src/mz_index/tests.rs:130-148
    r = orc.ppm_index(1.0, 100.0, 101.0)
    assert r[0] >= 100.0 and r[-1] <= 101.1
    assert orc.ppm_index(1.0, 10.0, 100.0)[0] == 50.0


def test_find_closest_index(orc, grid):  # src/mz_index/tests.rs:174-213
    assert orc.find_closest_index(grid, grid[100]) == 100
    assert orc.find_closest_index(grid, grid[0]) == 0
    assert orc.find_closest_index(grid, grid[-1]) == len(grid) - 1
    assert orc.find_closest_index(grid, 0.0) == 0
    assert orc.find_closest_index(grid, 3000.0) == len(grid) - 1
    between = (grid[100] + grid[101]) / np.float32(2.0)
    assert orc.find_closest_index(grid, between) in (100, 101)


def test_mz_range_indices(orc, grid):  # src/mz_index/tests.rs:215-280
    assert list(orc.mz_range_indices(grid, grid[100], grid[105])) == list(range(100, 106))
    assert list(orc.mz_range_indices(grid, grid[100], grid[100])) == [100]
    below = grid[0] - np.float32(10.0)
    assert len(orc.mz_range_indices(grid, below, below)) == 0
    above = grid[-1] + np.float32(10.0)
    assert len(orc.mz_range_indices(grid, above, above + np.float32(10.0))) == 0
    assert orc.mz_range_indices(grid, below, above) == range(0, len(grid))
    assert orc.mz_range_indices(grid, below, grid[50]) == range(0, 51)
    s = len(grid) - 50
    assert orc.mz_range_indices(grid, grid[s], above) == range(s, len(grid))
    assert len(orc.mz_range_indices(grid, 400.0, 600.0)) > 0  # :282-303


# ---------------------------------------------------------------- rt_index
@pytest.fixture(scope="module")
def rt_realistic(orc):  # src/rt_index/tests.rs:35-44
    rt = (np.arange(101, dtype=np.float32) * np.float32(0.5)).astype(np.float32)
    return rt, orc.mean_delta_t(rt)


def test_rt_limits_known_values(orc, rt_realistic):  # src/rt_index/tests.rs:108-190
    rt, dt = rt_realistic
    lo, hi = orc.rt_limits(rt, dt, 25.0, 2.0, 5)
    assert 33 <= lo <= 37 and 63 <= hi <= 67
    lo, hi = orc.rt_limits(rt, dt, 25.0, 10.0, 5)
    assert 28 <= lo <= 32 and 68 <= hi <= 72
    l1, u1 = orc.rt_limits(rt, dt, 25.0, 1.0, 2)
    l2, u2 = orc.rt_limits(rt, dt, 25.0, 1.0, 10)
    assert u2 - l2 > u1 - l1 and 22 <= u1 - l1 <= 26 and 38 <= u2 - l2 <= 42
    assert orc.rt_limits(rt, dt, 25.0, 15.0, 0) == (20, 80)
    assert orc.rt_limits(rt, dt, 5.0, 15.0, 0) == (0, 40)
    assert orc.rt_limits(rt, dt, 45.0, 15.0, 0) == (60, 101)
    assert orc.rt_limits(rt, dt, -20.0, 5.0, 0) == (0, 0)
    assert orc.rt_limits(rt, dt, 70.0, 5.0, 0) == (101, 101)
    assert orc.rt_limits(np.zeros(0, np.float32), 1.0, 25.0, 5.0, 5) == (0, 0)


def test_rt_limits_binary_search_cases(orc, rt_realistic):  # src/rt_index/tests.rs:192-243
    rt, dt = rt_realistic
    for prt, tol, pad in [(25.0, 10.0, 2), (10.0, 5.0, 0), (40.0, 7.5, 1)]:
        lo, hi = orc.rt_limits(rt, dt, prt, tol, pad)
        assert lo <= len(rt) and hi <= len(rt) and lo <= hi and hi - lo > 0


def _alpha_raw_rt(total, cycle_len):  # src/rt_index/tests.rs:60-88
    ds = (np.arange(total) % cycle_len).astype(np.int64)
    rt = (np.arange(total, dtype=np.float32) * np.float32(0.1)).astype(np.float32)
    z = np.zeros(total, np.int64)
    return dict(spectrum_delta_scan_idx=ds, isolation_lower_mz=np.full(total, 400, np.float32),
                isolation_upper_mz=np.full(total, 500, np.float32), spectrum_peak_start_idx=z,
                spectrum_peak_stop_idx=z, spectrum_cycle_idx=z, spectrum_rt=rt,
                peak_mz=np.zeros(0, np.float32), peak_intensity=np.zeros(0, np.float32))


def test_rt_from_alpha_raw(orc):  # src/rt_index/tests.rs:245-279
    d = orc.Dia(**_alpha_raw_rt(30, 10))
    assert list(d.rt) == [0.0, np.float32(1.0), np.float32(2.0)]
    d = orc.Dia(**_alpha_raw_rt(9, 3))
    assert len(d.rt) == 3 and abs(d.delta_t - 0.3) < 1e-6


# ---------------------------------------------------- rust binary search
def test_rust_binary_search_semantics(orc):
    # Rust >= 1.82 binary search: Ok(last equal) / Err(insertion point)
    s = [0, 1, 1, 1, 1, 2, 3, 5, 8, 13, 21, 34, 55]
    assert orc.rust_binary_search_u16(s, 13) == 9
    assert orc.rust_binary_search_u16(s, 4) == 7
    assert orc.rust_binary_search_u16(s, 100) == 13
    assert orc.rust_binary_search_u16(s, 1) == 4
    assert orc.rust_binary_search_u16([], 3) == 0
    assert orc.rust_binary_search_u16([5, 5, 5], 5) == 2


# ------------------------------------------------------------ dia_data
def _three_windows():  # src/dia_data/tests.rs:88-118
    return dict(
        spectrum_delta_scan_idx=np.array([0, 0, 1, 1, 2, 2]),
        isolation_lower_mz=np.array([100, 100, 200, 200, 300, 300], np.float32),
        isolation_upper_mz=np.array([125, 125, 225, 225, 325, 325], np.float32),
        spectrum_peak_start_idx=np.array([0, 2, 4, 6, 8, 10]),
        spectrum_peak_stop_idx=np.array([2, 4, 6, 8, 10, 12]),
        spectrum_cycle_idx=np.array([0, 1, 0, 1, 0, 1]),
        spectrum_rt=np.array([1.0, 1.1, 2.0, 2.1, 3.0, 3.1], np.float32),
        peak_mz=np.array([110, 115, 111, 116, 210, 215, 211, 216, 310, 315, 311, 316], np.float32),
        peak_intensity=np.array([1000, 1100, 1200, 1300, 2000, 2100, 2200, 2300, 3000, 3100, 3200, 3300],
                                np.float32))


def test_valid_observations(orc):  # src/dia_data/tests.rs:87-146
    d = orc.Dia(**_three_windows())
    assert d.num_observations == 3
    assert d.valid_observations(112.0) == [0]
    assert d.valid_observations(212.0) == [1]
    assert d.valid_observations(312.0) == [2]
    assert d.valid_observations(100.0) == [0]
    assert d.valid_observations(125.0) == [0]
    assert d.valid_observations(50.0) == []
    assert d.valid_observations(175.0) == []


def test_isolation_windows(orc):  # src/dia_data/tests.rs:148-212, src/dia_data_builder/tests.rs:84-129
    d = orc.Dia(**_three_windows())
    assert [d.window(i) for i in range(3)] == [(100.0, 125.0), (200.0, 225.0), (300.0, 325.0)]
    assert len(d.rt) > 0


def test_builder_cycle_ordering(orc):  # src/dia_data_builder/tests.rs:221-269
    d = orc.Dia(spectrum_delta_scan_idx=np.array([0, 0, 0]),
                isolation_lower_mz=np.full(3, 100, np.float32), isolation_upper_mz=np.full(3, 150, np.float32),
                spectrum_peak_start_idx=np.array([0, 1, 2]), spectrum_peak_stop_idx=np.array([1, 2, 3]),
                spectrum_cycle_idx=np.array([2, 0, 1]), spectrum_rt=np.array([1.0, 1.1, 1.2], np.float32),
                peak_mz=np.full(3, 120.0, np.float32),
                peak_intensity=np.array([1000, 2000, 3000], np.float32))
    grid = orc.ppm_index()
    b = orc.find_closest_index(grid, 120.0)
    cyc, it = d.slice_data(0, b)
    assert list(cyc) == [0, 1, 2]
    assert list(it) == [2000.0, 3000.0, 1000.0]


def test_builder_deterministic(orc):  # src/dia_data_builder/tests.rs:178-219
    a, b = orc.Dia(**_three_windows()), orc.Dia(**_three_windows())
    for w in range(3):
        assert np.array_equal(a.slice_starts(w), b.slice_starts(w))
        assert np.array_equal(a.cycles(w), b.cycles(w))


# ------------------------------------------------- quadrupole observation
def test_fill_xic_slice_basic(orc, grid):  # src/quadrupole_observation/tests.rs:85-121
    ss = np.array([0, 1, 2, 3, 4, 5, 5, 5, 5, 5, 5], np.uint32)
    cy = np.arange(5, dtype=np.uint16)
    it = (np.arange(5, dtype=np.float32) + 1) * 100
    xic = np.zeros(5, np.float32)
    orc.fill_xic_slice_raw(ss, cy, it, grid, xic, 0, 5, 0.1, grid[0])
    assert xic[0] == 100.0


def test_fill_xic_slice_cycle_range(orc, grid):  # src/quadrupole_observation/tests.rs:123-158
    ss = np.array([0] + [10] * 10, np.uint32)
    cy = np.arange(10, dtype=np.uint16)
    it = np.arange(10, dtype=np.float32) * 100
    xic = np.zeros(4, np.float32)
    orc.fill_xic_slice_raw(ss, cy, it, grid, xic, 2, 6, 0.1, grid[0])
    assert list(xic) == [200.0, 300.0, 400.0, 500.0]


def test_fill_xic_slice_mass_tolerance(orc, grid):  # src/quadrupole_observation/tests.rs:160-190
    ss = np.arange(6, dtype=np.uint32)
    cy = np.ones(5, np.uint16)
    it = 100.0 * (np.arange(5, dtype=np.float32) + 1)
    xic = np.zeros(3, np.float32)
    orc.fill_xic_slice_raw(ss, cy, it, grid, xic, 0, 3, 0.1, grid[2])
    assert xic[1] == 300.0 and xic[0] == 0.0 and xic[2] == 0.0


def test_fill_xic_duplicate_first_cycle_quirk(orc, grid):
    # Two peaks at the window's first cycle in one bin: the Rust binary search
    # lands on the last of them, so only that one is summed.
    ss = np.array([0, 3], np.uint32)
    cy = np.array([4, 4, 5], np.uint16)
    it = np.array([1.0, 2.0, 4.0], np.float32)
    xic = np.zeros(2, np.float32)
    orc.fill_xic_slice_raw(ss, cy, it, grid, xic, 4, 6, 0.1, grid[0])
    assert list(xic) == [2.0, 4.0]
    xic = np.zeros(3, np.float32)
    orc.fill_xic_slice_raw(ss, cy, it, grid, xic, 3, 6, 0.1, grid[0])
    assert list(xic) == [0.0, 3.0, 4.0]


# ------------------------------------------------------------ dense XIC
def _simple_raw():  # src/dense_xic_observation/tests.rs:6-30
    return dict(spectrum_delta_scan_idx=np.array([0]), isolation_lower_mz=np.array([199.0], np.float32),
                isolation_upper_mz=np.array([201.0], np.float32), spectrum_peak_start_idx=np.array([0]),
                spectrum_peak_stop_idx=np.array([2]), spectrum_cycle_idx=np.array([10]),
                spectrum_rt=np.array([100.0], np.float32), peak_mz=np.array([200.0, 200.1], np.float32),
                peak_intensity=np.array([1000.0, 2000.0], np.float32))


def test_dense_xic_shapes(orc):  # src/dense_xic_observation/tests.rs:32-107
    d = orc.Dia(**_simple_raw())
    assert d.dense_xic(200.0, 10, 12, 20.0, [200.0]).shape == (1, 2)
    assert d.dense_xic(200.0, 10, 11, 20.0, [200.0]).shape == (1, 1)
    assert d.dense_xic(200.0, 10, 12, 20.0, []).shape == (0, 2)
    assert d.dense_xic(200.0, 10, 12, 20.0, [200.0, 200.1, 205.0]).shape == (3, 2)
    assert d.valid_observations(200.0) == [0]


def test_dense_xic_sums(orc):  # src/dense_xic_observation/tests.rs:126-143,246-325
    d = orc.Dia(**_simple_raw())
    assert d.dense_xic(200.0, 10, 11, 1000.0, [200.05])[0, 0] == 3000.0
    x = d.dense_xic(200.0, 10, 11, 20.0, [200.0, 200.1, 300.0])
    assert (x[0, 0], x[1, 0], x[2, 0]) == (1000.0, 2000.0, 0.0)
    assert d.dense_xic(200.0, 10, 12, 20.0, [300.0]).sum() == 0.0
    assert d.dense_xic(200.0, 10, 11, 20.0, [200.0])[0, 0] == 1000.0
    x = d.dense_xic(200.0, 10, 11, 1000.0, [200.0, 200.05])
    assert x[0, 0] == 3000.0 and x[1, 0] == 3000.0
    assert d.dense_xic(200.0, 10, 11, 20.0, [100.0])[0, 0] == 0.0
    assert d.dense_xic(200.0, 10, 11, 400.0, [200.05])[0, 0] == 3000.0


def test_dense_xic_weighted_and_zero(orc):  # src/dense_xic_observation/tests.rs:145-227
    d = orc.Dia(spectrum_delta_scan_idx=np.array([0]), isolation_lower_mz=np.array([249.0], np.float32),
                isolation_upper_mz=np.array([251.0], np.float32), spectrum_peak_start_idx=np.array([0]),
                spectrum_peak_stop_idx=np.array([3]), spectrum_cycle_idx=np.array([5]),
                spectrum_rt=np.array([50.0], np.float32), peak_mz=np.array([249.9, 250.0, 250.1], np.float32),
                peak_intensity=np.array([500.0, 1000.0, 1500.0], np.float32))
    assert d.dense_xic(250.0, 5, 6, 2000.0, [250.0])[0, 0] == 3000.0
    d = orc.Dia(spectrum_delta_scan_idx=np.array([0, 1]), isolation_lower_mz=np.array([299.0, 299.0], np.float32),
                isolation_upper_mz=np.array([301.0, 301.0], np.float32), spectrum_peak_start_idx=np.array([0, 2]),
                spectrum_peak_stop_idx=np.array([2, 4]), spectrum_cycle_idx=np.array([0, 1]),
                spectrum_rt=np.array([10.0, 20.0], np.float32),
                peak_mz=np.array([300.0, 300.1, 300.0, 300.1], np.float32),
                peak_intensity=np.array([1000.0, 0.0, 0.0, 2000.0], np.float32))
    x = d.dense_xic(300.0, 0, 2, 2000.0, [300.05])
    assert x[0, 0] == 1000.0 and x[0, 1] == 2000.0


# --------------------------------------------------------------- kernel
def test_gaussian_kernel(orc):  # src/kernel/tests.rs:4-26
    k = orc.gaussian_kernel(10.0, 1.0, 30, 60.0)
    assert len(k) == 30
    assert abs(float(np.sum(k.astype(np.float64))) - 1.0) < 1e-6
    assert all(k[i] <= k[15] for i in range(30))
    assert len(orc.gaussian_kernel(2 * 2.3548, 1.0, 21, 1.0)) == 22  # width rounded up to even
    assert len(orc.gaussian_kernel(3.0, 1.0, 31, 1.0)) == 32


# ---------------------------------------------------------- convolution
def test_convolution_shapes(orc):  # src/convolution/tests.rs:6-164
    k5 = orc.gaussian_kernel(0.5, 1.0, 5, 1.0)
    assert orc.convolution(k5, np.array([[0, 0, 1, 0, 0]], np.float32)).shape == (1, 5)
    k7 = orc.gaussian_kernel(0.5, 1.0, 7, 1.0)
    assert orc.convolution(k7, np.array([[0, 1, 0]], np.float32)).shape == (1, 3)
    assert orc.convolution(k5, np.zeros((0, 10), np.float32)).shape == (0, 10)
    assert orc.convolution(k5, np.zeros((5, 0), np.float32)).shape == (5, 0)
    for ks in (3, 5, 7, 9, 11):
        kk = orc.gaussian_kernel(1.0, 1.0, ks, 1.0)
        for n in (1, 2, 3, 5, 10):
            x = np.zeros((1, n), np.float32)
            x[0, n // 2] = 1.0
            assert orc.convolution(kk, x).shape == (1, n)
    out = orc.convolution(orc.gaussian_kernel(1.0, 1.0, 11, 1.0), np.ones((1, 5), np.float32))
    assert out.shape == (1, 5) and not out.any()


def test_convolution_values_and_edges(orc):
    # valid region [h, C-h) only; edges stay 0 (src/convolution/scalar.rs:33-50)
    k = orc.gaussian_kernel(0.5, 1.0, 5, 1.0)  # len 6, h = 3
    x = np.linspace(0.1, 1.0, 10, dtype=np.float32)[None, :]
    out = orc.convolution(k, x)
    h = len(k) // 2
    assert not out[0, :h].any() and not out[0, len(x[0]) - h:].any()
    i = 5
    s = np.float32(x[0, i] * k[h])
    for j in range(h):
        s = np.float32(s + np.float32(np.float32(x[0, i - (h - j)] + x[0, i + (h - j)]) * k[j]))
    assert out[0, i] == s


# ---------------------------------------------------------------- score
def test_log_dot_known_values(orc):  # src/score/tests.rs:5-18
    a = np.array([[0.0, 1.0, 2.0], [3.0, 4.0, 5.0]], np.float32)
    r = orc.log_dot(a, [0.5, 1.5])
    assert np.allclose(r, [2.0794415, 2.7607305, 3.2369454], atol=1e-5, rtol=0)
    r1 = orc.log_dot(a, [0.5, 1.5], log_mode=orc.LOG_RN)
    assert np.allclose(r1, r, atol=1e-6, rtol=0)


# ---------------------------------------------------------- local maxima
def test_local_maxima(orc):  # src/peak_group_selection/tests.rs:7-46
    i, v = orc.local_maxima([1, 2, 3, 2, 5, 3, 2, 4, 7, 5, 3, 2], 10)
    assert list(i) == [18] and list(v) == [7.0]
    assert len(orc.local_maxima([1, 2, 3, 4, 5, 6, 7])[0]) == 0
    assert len(orc.local_maxima([1, 2, 3, 4])[0]) == 0
    assert len(orc.local_maxima([1, 2, 5, 5, 5, 2, 1])[0]) == 0


def test_local_maxima_order_is_value_desc_stable(orc):
    a = [0, 1, 5, 1, 0, 1, 9, 1, 0, 1, 5, 1, 0]
    i, v = orc.local_maxima(a, 0)
    assert list(i) == [6, 2, 10] and list(v) == [9, 5, 5]


# --------------------------------------------------------- fragment filter
B, Y = 98, 121


def _ffs(orc, mz, inten, non_zero, top_k, number=None, ftype=None, filter_y1=False):
    n = len(mz)
    number = np.ones(n, np.uint8) if number is None else number
    ftype = np.full(n, B, np.uint8) if ftype is None else ftype
    k = orc.filter_sort_fragments(mz, inten, number, ftype, non_zero, filter_y1, top_k)
    return list(np.asarray(mz, np.float32)[k]), list(np.asarray(inten, np.float32)[k])


def test_filter_sort_fragments(orc):  # src/speclib_flat/tests.rs:5-345
    big = 2**62
    mz = [100.0, 200.0, 300.0, 400.0, 500.0]
    assert _ffs(orc, mz, [0, 15, 10, 20, 5], False, big, filter_y1=True) == (mz, [0, 15, 10, 20, 5])
    assert _ffs(orc, mz, [0, 15, 10, 0, 5], True, big) == ([200, 300, 500], [15, 10, 5])
    assert _ffs(orc, mz, [5, 15, 10, 20, 8], False, 3) == ([200, 300, 400], [15, 10, 20])
    assert _ffs(orc, mz, [0, 15, 10, 0, 20], True, 2) == ([200, 500], [15, 20])
    assert _ffs(orc, [600, 200, 800, 100, 400], [15, 25, 5, 30, 20], False, 3) == ([100, 200, 400], [30, 25, 20])
    m, i = _ffs(orc, mz, [10, 15, 10, 10, 10], False, 3)
    assert len(m) == 3 and 15.0 in i and i.count(10.0) == 2 and m == sorted(m)
    assert _ffs(orc, [], [], False, 5) == ([], [])
    assert _ffs(orc, [500.0], [10.0], False, 5) == ([500.0], [10.0])
    assert _ffs(orc, [500.0], [0.0], True, 5) == ([], [])
    assert _ffs(orc, mz, [0, 0, 0, 0, 0], True, 5) == ([], [])
    assert _ffs(orc, mz, [5, 15, 10, 20, 8], False, 0) == ([], [])
    assert _ffs(orc, mz, [5, 15, 10, 20, 8], False, 10) == (mz, [5, 15, 10, 20, 8])


def test_filter_y1(orc):  # src/speclib_flat/tests.rs:613-676
    mz = [150.0, 200.0, 300.0, 400.0, 500.0]
    k = orc.filter_sort_fragments(mz, [10, 15, 20, 25, 30], np.array([1, 2, 3, 1, 2], np.uint8),
                                  np.array([Y, Y, B, Y, B], np.uint8), False, True, 2**62)
    assert list(np.array(mz)[k]) == [200.0, 300.0, 500.0]


def test_filter_invariants(orc):  # src/speclib_flat/tests.rs:347-413
    rng = np.random.default_rng(0)
    for _ in range(50):
        n = int(rng.integers(0, 30))
        mz = rng.uniform(100, 1000, n).astype(np.float32)
        it = rng.uniform(0, 10, n).astype(np.float32)
        it[rng.random(n) < 0.2] = 0
        for k in (1, 3, 12, 100):
            for nz in (False, True):
                kk = orc.filter_sort_fragments(mz, it, np.ones(n, np.uint8), np.full(n, B, np.uint8), nz, False, k)
                assert len(kk) <= k
                if nz:
                    assert (it[kk] > 0).all()
                assert (np.diff(mz[kk]) >= 0).all()


def test_speclib_sorting_and_filtered_precursor(orc):  # src/speclib_flat/tests.rs:414-611
    lb = orc.Lib(precursor_idx=[3, 1, 4, 2], precursor_mz=[300, 100, 400, 200], precursor_rt=[30, 10, 40, 20],
                 flat_frag_start_idx=[6, 0, 9, 3], flat_frag_stop_idx=[9, 3, 12, 6],
                 fragment_mz=np.arange(12, dtype=np.float32) + 100, fragment_intensity=np.ones(12, np.float32),
                 fragment_number=np.ones(12, np.uint8), fragment_type=np.full(12, B, np.uint8))
    assert list(np.array([3, 1, 4, 2])[lb.sorted_order]) == [1, 2, 3, 4]
