"""The FP32 factored translations on the tensor cores (k_rot_tc: the three
factors Fw, Z, Bk of 32 columns at a time in shared memory, M = 64 operator
rows x N = 32 columns per MMA) against the factored product of the same FP32
operators in FP64 (host), through the C ABI; and the host emulation of the
kernel's arithmetic (tiles, padded rows, row maps; CPU, no device)."""
import ctypes

import pytest

import elfmmlib3d_b200 as E


def _lib():
    L = E.load()
    L.efmm_rot_tc_selfcheck.restype = ctypes.c_int
    L.efmm_rot_tc_selfcheck.argtypes = [ctypes.c_int, ctypes.c_uint, ctypes.POINTER(ctypes.c_double)]
    L.efmm_rot_tc_selfcheck_device.restype = ctypes.c_int
    L.efmm_rot_tc_selfcheck_device.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint,
                                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
    return L


@pytest.mark.parametrize("p", [1, 2, 7, 14, 26, 30, 31])
def test_rot_tc_host_emulation(p):
    """Tiles, canonical-layout addressing and the row maps between the
    stages, emulated on the host with the kernel's split and FP32 sums."""
    r = ctypes.c_double()
    assert _lib().efmm_rot_tc_selfcheck(p, 3, ctypes.byref(r)) == 0
    assert r.value < 5e-7


@pytest.mark.gpu
@pytest.mark.parametrize("p,C,npair", [(3, 40, 3), (14, 256, 2), (20, 96, 3), (26, 64, 5), (30, 256, 3), (31, 7, 20)])
def test_rot_tc_device_matches_fp64_product(gpu, p, C, npair):
    r, to = ctypes.c_double(), ctypes.c_int()
    assert _lib().efmm_rot_tc_selfcheck_device(p, C, npair, 11, ctypes.byref(r), ctypes.byref(to)) == 0
    print(f"p={p} C={C} npair={npair}: rel {r.value:.2e}")
    assert to.value == 0
    assert r.value < 5e-7
