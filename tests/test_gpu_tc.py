"""The tensor-core FP32 product (tcgen05.mma kind::tf32 with the 3-term
head/tail split) against an FP64 host product: FP32-level accuracy on full
tiles, ragged edges (M, N not multiples of 128, K not a multiple of 32) and
an empty K; in both forms of the kernel (operands streamed by cp.async into
a ring of raw tiles, the default, and register staging)."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(params=[1, 0], ids=["ring", "registers"], autouse=True)
def variant(request, gpu):
    f = gpu.load().efmm_tc_variant
    f.restype = ctypes.c_int
    old = f(request.param)
    yield request.param
    f(old)


def _check(gpu, M, N, K, seed, bn=128, aligned=0):
    f = gpu.load().efmm_tc_gemm_selfcheck_tile
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint,
                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
    rel, to = ctypes.c_double(), ctypes.c_int()
    ier = f(M, N, K, bn, aligned, seed, ctypes.byref(rel), ctypes.byref(to))
    return ier, rel.value, to.value


@pytest.mark.parametrize("M,N,K", [(128, 128, 32), (256, 128, 512), (300, 200, 1000), (1640, 256, 4000), (5, 7, 3)])
def test_tc_product_fp32_accuracy(gpu, M, N, K):
    ier, rel, to = _check(gpu, M, N, K, 11)
    print(f"tc product {M}x{N}x{K}: rel {rel:.2e}")
    assert ier == 0 and to == 0
    # FP32 products of K terms in [-1, 1): FP32 rounding ~ 1e-7
    assert rel < 2e-6


def test_tc_product_empty_k(gpu):
    ier, rel, to = _check(gpu, 130, 10, 0, 3)
    assert ier == 0 and to == 0 and rel == 0.0


@pytest.mark.parametrize("M,N,K", [(128, 64, 32), (1640, 64, 1250), (300, 50, 77), (256, 130, 600)])
def test_tc_product_64_wide_tiles(gpu, M, N, K):
    ier, rel, to = _check(gpu, M, N, K, 5, bn=64)
    print(f"tc product (64-wide tiles) {M}x{N}x{K}: rel {rel:.2e}")
    assert ier == 0 and to == 0 and rel < 2e-6


@pytest.mark.parametrize("bn", [64, 128])
@pytest.mark.parametrize("M,N,K", [(128, 64, 32), (1640, 64, 1250), (300, 50, 77), (992, 130, 4000)])
def test_tc_product_aligned_rows(gpu, M, N, K, bn):
    # 16-byte rows: vector loads of B, zero fill at the edges
    ier, rel, to = _check(gpu, M, N, K, 9, bn=bn, aligned=1)
    print(f"tc product (aligned, {bn}-wide) {M}x{N}x{K}: rel {rel:.2e}")
    assert ier == 0 and to == 0 and rel < 2e-6
