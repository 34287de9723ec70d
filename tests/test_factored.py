"""Factored translations (rotation, shift along z, rotation back) against the
dense per-offset operators, on the CPU (host construction, no device).  The
error is measured in the normalised basis, where the harmonics are O(1)."""
import ctypes

import pytest


@pytest.mark.parametrize("p,eps,stride", [(6, 0.5e-2, 1), (14, 0.5e-3, 1), (26, 0.5e-6, 9), (39, 0.5e-9, 40)])
def test_factored_equals_dense(lib, p, eps, stride):
    L = lib.load()
    f = L.efmm_factored_selfcheck
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    worst = ctypes.c_double(1.0)
    n = f(p, eps, stride, ctypes.byref(worst))
    assert n == 316 + 16
    assert worst.value < 1e-12
