"""Device unit tests of the float helpers (tests/cuda/ht_selftest.cu).

The render path replaces groups of IEEE divisions that share a divisor by one correctly
rounded reciprocal plus Markstein's FMA correction step; these tests show the result is
bit-identical to IEEE division, value by value and through the whole Moebius ray map."""
import ctypes
import os

import pytest

pytestmark = pytest.mark.gpu

LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cuda", "libht_selftest.so")


@pytest.fixture(scope="module")
def selftest(built):
    lib = ctypes.CDLL(LIB)
    lib.ht_selftest_div.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong)]
    lib.ht_selftest_raymap.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_ulonglong)]
    lib.ht_selftest_monotone.argtypes = [ctypes.POINTER(ctypes.c_ulonglong)]
    return lib


@pytest.mark.parametrize("mode,n", [(0, 1 << 32), (1, 1 << 28), (2, 1 << 28), (3, 1 << 30)])
def test_shared_reciprocal_division_is_ieee(selftest, mode, n):
    out = (ctypes.c_ulonglong * 2)()
    assert selftest.ht_selftest_div(n, 0x1234 + mode, mode, out) == 0
    fast, mism = out[0], out[1]
    assert fast > n // 4, "fast path barely used"
    assert mism == 0, f"{mism} of {fast} fast-path quotients differ from IEEE division"


def test_fast_ray_map_is_bit_identical(selftest):
    out = (ctypes.c_ulonglong * 2)()
    assert selftest.ht_selftest_raymap(1 << 26, 77, out) == 0
    assert out[0] == 1 << 26
    assert out[1] == 0, f"{out[1]} ray maps differ from the IEEE-division form"


def test_distance_is_monotone_in_x(selftest):
    """log(x + sqrt(x^2 - 1)) as compiled is non-decreasing over every float in [1, inf):
    the object scan may compare x instead of the distance (exhaustive, 2^30 values)."""
    out = (ctypes.c_ulonglong * 2)()
    assert selftest.ht_selftest_monotone(out) == 0
    assert out[0] == 0x7f800000 - 0x3f800000
    assert out[1] == 0, f"{out[1]} decreasing steps"
