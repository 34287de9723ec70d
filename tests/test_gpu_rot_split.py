"""The FP32 translations in the parity-split form (k_translate_rot_s: Rz,
the re / im blocks of Ry and of the shift along z, Ry back, Rz back; one
warp per block) against the same FP32 operators applied in FP64 on the
host, through the C ABI, for M2L, M2M and L2L groups (one M2L offset along
-z), and against the full-block kernels on the same inputs."""
import ctypes

import pytest

import elfmmlib3d_b200 as E


def _lib():
    L = E.load()
    L.efmm_rot_split_selfcheck_device.restype = ctypes.c_int
    L.efmm_rot_split_selfcheck_device.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint,
                                                  ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.efmm_rot_split_bench.restype = ctypes.c_int
    L.efmm_rot_split_bench.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_double)]
    return L


@pytest.mark.gpu
@pytest.mark.parametrize("p,C,npair", [(1, 5, 3), (3, 40, 3), (8, 17, 2), (14, 256, 2), (16, 64, 3), (20, 96, 3),
                                       (26, 64, 5), (30, 256, 3), (31, 7, 20)])
def test_split_kernel_matches_fp64_product(gpu, p, C, npair):
    r = ctypes.c_double(1.0)
    assert _lib().efmm_rot_split_selfcheck_device(p, C, npair, 5, 0, ctypes.byref(r)) == 0
    print(f"p={p} C={C} npair={npair}: rel {r.value:.2e}")
    assert r.value < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("p", [12, 30])
def test_split_kernel_timing_beside_full_blocks(gpu, p):
    """Both kernels on the same groups and columns; the split form does about
    half the multiply-adds (printed, not asserted beyond a sanity bound)."""
    L = _lib()
    ms = [ctypes.c_double(), ctypes.c_double()]
    for e in (0, 1):
        assert L.efmm_rot_split_bench(p, 256, 64, e, 5, ctypes.byref(ms[e])) == 0
    print(f"p={p}: split {ms[0].value:.3f} ms, full blocks {ms[1].value:.3f} ms")
    assert 0 < ms[0].value < 2.0 * ms[1].value
