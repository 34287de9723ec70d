"""The tree builder's device primitives (sort.cu): the stable LSD radix sort
of (64-bit key, int value) pairs against a stable host sort, and the
exclusive scan against host prefix sums, through the C ABI.  Stability
matters: the tree's point orders follow from it (points of one box keep
their relative order)."""
import ctypes

import pytest

import elfmmlib3d_b200 as E


@pytest.mark.gpu
@pytest.mark.parametrize("n,bits", [(0, 8), (1, 8), (7, 3), (255, 8), (256, 9), (4095, 12), (4097, 20),
                                    (100_003, 23), (1_000_000, 40), (300_000, 64)])
def test_radix_sort_and_scan_match_host(gpu, n, bits):
    f = E.load().efmm_sort_selfcheck_device
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.POINTER(ctypes.c_longlong)]
    bad = ctypes.c_longlong(-1)
    assert f(n, bits, 17, ctypes.byref(bad)) == 0
    assert bad.value == 0
