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


def test_u_kernel_m2l_selfcheck(lib):
    # M2L of the half-space kernel U = z log(r + z) - r through its J table
    # (the device operators' code, run on the host): errors fall with the
    # order as for 1/r, at offsets above, level with and far from the sources
    import ctypes
    f = lib.load().efmm_u_m2l_selfcheck
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_uint]
    for X in [(2.0, 1.0, 1.0), (0.0, 0.0, 2.0), (3.0, -2.0, 0.0), (-1.0, 3.0, 3.0)]:
        e8 = f(8, *X, 20, 3)
        e20 = f(20, *X, 20, 3)
        assert 0 <= e20 < 1e-6 and e20 < e8, (X, e8, e20)
    assert f(0, 2.0, 0, 0, 5, 1) == -1.0


@pytest.mark.parametrize("p,eps,stride", [(6, 0.5e-2, 1), (14, 0.5e-3, 1), (26, 0.5e-6, 9), (30, 5e-8, 13), (31, 5e-8, 29)])
def test_parity_split_equals_dense(lib, p, eps, stride):
    """The translations as Rz, the re / im blocks of Ry, the shift's re / im
    blocks, Ry back and Rz back: in double against the dense operators, and
    the packed FP32 pool of the device kernel applied on the host as the
    kernel reads it (FP32 operator rounding only)."""
    L = lib.load()
    f = L.efmm_split_selfcheck
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    worst = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    assert f(p, eps, stride, worst) == 316 + 16
    assert worst[0] < 1e-12
    assert worst[1] < 1e-6


@pytest.mark.parametrize("p,eps,stride", [(6, 0.5e-2, 1), (14, 0.5e-3, 3), (30, 5e-8, 17), (39, 5e-10, 41)])
def test_u_kernel_m2l_parity_split(lib, p, eps, stride):
    """The half-space U-kernel M2L as Rz out, the re / im blocks of the
    operator at the offset rotated into the xz plane, Rz in: in double
    against the dense operator, and the packed FP32 pool as the kernel reads
    it; the dropped re / im coupling is zero (U is even in y)."""
    L = lib.load()
    f = L.efmm_usplit_selfcheck
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    worst = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    assert f(p, eps, stride, worst) == 178
    assert worst[0] < 1e-12
    assert worst[1] < 1e-6
    assert worst[2] < 1e-12
