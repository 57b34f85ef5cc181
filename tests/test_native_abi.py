"""The C-ABI library: builds, loads, exports every declared symbol; host-only
entry points agree with the oracle bit for bit.  CPU only (no kernel launches)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "ads_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(ads_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from alphadia_search_rs_b200 import _ffi

    return _ffi.load()


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("ads_dia_create", "ads_lib_create", "ads_selection_create", "ads_select",
                 "ads_candidates_size", "ads_candidates_copy_out", "ads_candidates_destroy",
                 "ads_last_error"):
        assert must in names


def test_every_declared_symbol_is_exported(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    from alphadia_search_rs_b200 import _ffi

    assert set(declared_functions()) == set(_ffi.SIGNATURES)


def test_library_is_sm100a_build():
    from alphadia_search_rs_b200 import build

    assert build.ARCH_FLAGS == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert os.path.exists(build.lib_path())


def test_grid_matches_oracle(orc):
    import alphadia_search_rs_b200 as ads

    g = ads.mz_grid()
    og = orc.ppm_index()
    assert len(g) == 2590781
    assert np.array_equal(g.view(np.uint32), og.view(np.uint32))


@pytest.mark.parametrize("args", [(3.0, 1.0, 20, 1.0), (4.7096, 1.0, 21, 1.0), (7.0644, 1.0, 31, 1.0),
                                  (10.0, 1.0, 30, 60.0), (0.5, 1.0, 5, 1.0), (1.0, 1.0, 3, 1.0),
                                  (2.0, 1.0, 62, 1.0), (5.0, 2.0, 17, 0.5)])
def test_gaussian_kernel_matches_oracle(orc, args):
    import alphadia_search_rs_b200 as ads

    k = ads.gaussian_kernel(*args)
    ok = orc.gaussian_kernel(*args)
    assert np.array_equal(k.view(np.uint32), ok.view(np.uint32))


def test_default_parameters(lib):
    from alphadia_search_rs_b200 import _ffi

    p = _ffi.AdsSelectionParams()
    lib.ads_selection_params_default(C.byref(p))
    # src/peak_group_selection/parameters.rs:24-43
    assert (p.fwhm_rt, p.kernel_size, p.peak_length, p.mass_tolerance, p.rt_tolerance,
            p.candidate_count, p.top_k_fragments) == (3.0, 20, 5, 7.0, 200.0, 3, 12)


def test_errors_are_reported_not_thrown(lib):
    from alphadia_search_rs_b200 import _ffi

    h = C.c_void_p()
    rc = lib.ads_dia_create(None, 0, C.byref(h))
    assert rc == _ffi.ADS_ERR_INVALID_ARGUMENT
    assert b"null" in lib.ads_last_error()
    assert lib.ads_candidates_size(None) == -1
    assert lib.ads_dia_destroy(None) == _ffi.ADS_OK


def test_no_silent_cpu_fallback(lib):
    """Without a GPU every compute entry point fails loudly."""
    if lib.ads_device_count() > 0:
        pytest.skip("a GPU is present")
    import alphadia_search_rs_b200 as ads

    with pytest.raises(Exception):
        ads.PeakGroupSelection(ads.SelectionParameters())
    z64 = np.zeros(1, np.int64)
    z32 = np.zeros(1, np.float32)
    with pytest.raises(Exception):
        ads.DIAData.from_arrays(z64, z32, z32, z64, z64, z64, z32, z32, z32,
                                np.zeros((1, 1, 1, 1), np.float32))
