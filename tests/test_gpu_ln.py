"""The search kernel's logarithm equals ln rounded once from double precision for
every finite float >= 1 (1 + a convolved intensity), checked exhaustively on the
device."""
import ctypes as C
import struct

import pytest

pytestmark = pytest.mark.gpu


def _bits(x: float) -> int:
    return struct.unpack("<I", struct.pack("<f", x))[0]


def test_ln_fast_equals_double_rounded_ln_exhaustive():
    from alphadia_search_rs_b200 import _ffi

    L = _ffi.load()
    bad, slow = C.c_int64(), C.c_int64()
    lo, hi = _bits(1.0), _bits(float("inf"))
    _ffi.check(L.ads_selftest_ln(0, lo, hi, C.byref(bad), C.byref(slow)))
    n = hi - lo
    assert bad.value == 0
    assert slow.value < n * 1e-3  # the slow path is rare


def test_ln_special_values():
    from alphadia_search_rs_b200 import _ffi

    L = _ffi.load()
    bad, slow = C.c_int64(), C.c_int64()
    # zero, subnormals and (0, 1): handled by the reference path
    _ffi.check(L.ads_selftest_ln(0, 0, _bits(1.0) + 1, C.byref(bad), C.byref(slow)))
    assert bad.value == 0
    # the largest finite floats, +inf and NaNs
    _ffi.check(L.ads_selftest_ln(0, _bits(2.0 ** 120), 0x7FC00010, C.byref(bad), C.byref(slow)))
    assert bad.value == 0
