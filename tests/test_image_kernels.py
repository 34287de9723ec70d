"""The product's generated image kernels (mindlin_gen.cuh, evaluated on the
host through efmm_mindlin_image_kernel) against the oracle's C kernels
(oracle/image_gen.h, printed from oracle/mindlin.py's symbolic
expressions): the two derivations of Mindlin's image part agree to
rounding at random source / target pairs in z < 0.  No device is used."""
import ctypes

import numpy as np
import pytest

_dp = ctypes.POINTER(ctypes.c_double)


def _kernels(lib, oracle):
    L = ctypes.CDLL(lib.library_path())
    L.efmm_mindlin_image_kernel.restype = ctypes.c_int
    O = oracle.lib()
    O.oracle_image_kernel.restype = ctypes.c_int

    def call(f, layer, lam, mu, x, s, n):
        out = np.zeros(27)
        ier = f(ctypes.c_int(layer), ctypes.c_double(lam), ctypes.c_double(mu), x.ctypes.data_as(_dp),
                s.ctypes.data_as(_dp), n.ctypes.data_as(_dp), out.ctypes.data_as(_dp))
        assert ier == 0
        return out
    return (lambda *a: call(L.efmm_mindlin_image_kernel, *a)), (lambda *a: call(O.oracle_image_kernel, *a))


@pytest.mark.parametrize("layer", [0, 1])
def test_product_image_kernels_match_oracle(lib, oracle, layer):
    prod, orc = _kernels(lib, oracle)
    rng = np.random.default_rng(21 + layer)
    worst = 0.0
    for _ in range(400):
        lam, mu = rng.uniform(0.2, 3.0, 2)
        x = np.array([*rng.uniform(-3, 3, 2), -rng.uniform(0.01, 4.0)])
        s = np.array([*rng.uniform(-3, 3, 2), -rng.uniform(0.01, 4.0)])
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        a, b = prod(layer, lam, mu, x, s, n), orc(layer, lam, mu, x, s, n)
        for k in range(3):  # per source direction: displacement, then strain
            for blk in (slice(9 * k, 9 * k + 3), slice(9 * k + 3, 9 * k + 9)):
                scale = np.abs(b[blk]).max()
                worst = max(worst, np.abs(a[blk] - b[blk]).max() / scale)
    assert worst < 1e-12, worst


def test_product_image_kernel_rejects_bad_layer(lib):
    L = ctypes.CDLL(lib.library_path())
    L.efmm_mindlin_image_kernel.restype = ctypes.c_int
    x = np.array([0.0, 0.0, -1.0])
    out = np.zeros(27)
    ier = L.efmm_mindlin_image_kernel(ctypes.c_int(2), ctypes.c_double(1.0), ctypes.c_double(1.0),
                                      x.ctypes.data_as(_dp), x.ctypes.data_as(_dp), x.ctypes.data_as(_dp),
                                      out.ctypes.data_as(_dp))
    assert ier == 16
