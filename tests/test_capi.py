"""CPU tests of the C ABI and the host layer (no GPU compute)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def _header_symbols():
    syms = []
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            syms += re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", src)
    keep = [s for s in syms if s.startswith(("el", "efmm"))]
    return sorted(set(keep))


def test_library_exports_every_declared_symbol(lib):
    L = ctypes.CDLL(lib.library_path())
    syms = _header_symbols()
    assert "elfmm3dtriatarg_" in syms and "efmm_plan_evaluate" in syms
    for s in syms:
        assert hasattr(L, s), s
    for s in lib.EXPORTS:
        assert s in syms


def test_no_cpu_fallback_without_gpu(lib):
    if lib.device_count() > 0:
        pytest.skip("a GPU is visible")
    tri = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]]], float)
    with pytest.raises(lib.ElfmmError):
        lib.elfmm3dtriatarg(2, 1.0, 1.0, tri, [[0, 0, 1]], tri.mean(1), sigma_sl=[[1, 0, 0]])


def test_fortran_abi_returns_ier_without_device(lib):
    """The Fortran-ABI symbol reports ier (1024: no device) instead of failing silently."""
    if lib.device_count() > 0:
        pytest.skip("a GPU is visible")
    L = ctypes.CDLL(lib.library_path())
    dp = ctypes.POINTER(ctypes.c_double)
    tri = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0], float)
    nrm = np.array([0, 0, 1.0])
    src = np.array([1 / 3, 1 / 3, 0])
    sig = np.array([1.0, 0, 0])
    out = np.zeros(9)
    ier = ctypes.c_int(-5)
    i = lambda v: ctypes.byref(ctypes.c_int(v))
    d = lambda v: ctypes.byref(ctypes.c_double(v))
    L.elfmm3dtria_(ctypes.byref(ier), i(2), d(1.0), d(1.0), tri.ctypes.data_as(dp), nrm.ctypes.data_as(dp),
                   i(1), src.ctypes.data_as(dp), i(1), sig.ctypes.data_as(dp), i(0), sig.ctypes.data_as(dp),
                   i(1), out.ctypes.data_as(dp), i(1), out.ctypes.data_as(dp))
    assert ier.value == 1024


def test_iprec_tables():
    """iprec -> (eps, nbox, p) as the reference (elfmm3dtria.f:702-722, l3dterms.f:42)."""
    import math
    def p_for(eps):
        z1, z2 = 1.5, math.sqrt(3) / 2
        jf, hf = z2, 1 / z1 ** 2
        for j in range(2, 1000):
            hf /= z1
            jf *= z2
            if jf * hf < eps:
                return j
    assert [p_for(e) for e in (.5e-3, .5e-6, .5e-9, .5e-12)] == [14, 26, 39, 51]


def test_halfspace_total_checks_arguments_before_the_device(lib):
    """elhfmm3dtria_total_ rejects points above z = 0 with ier 16 before it
    touches a device; valid input without a device gives 1024."""
    if lib.device_count() > 0:
        pytest.skip("a GPU is visible")
    L = ctypes.CDLL(lib.library_path())
    dp = ctypes.POINTER(ctypes.c_double)
    tri = np.array([0, 0, -1, 1, 0, -1, 0, 1, -1], float)
    nrm = np.array([0, 0, 1.0])
    src = np.array([1 / 3, 1 / 3, -1.0])
    sig = np.array([1.0, 0, 0])
    out = np.zeros(18)
    i = lambda v: ctypes.byref(ctypes.c_int(v))
    d = lambda v: ctypes.byref(ctypes.c_double(v))
    for tgt, want in ((np.array([0.2, 0.2, 0.5]), 16), (np.array([0.2, 0.2, -0.5]), 1024)):
        ier = ctypes.c_int(-5)
        L.elhfmm3dtria_total_(ctypes.byref(ier), i(2), d(1.0), d(1.0), tri.ctypes.data_as(dp),
                              nrm.ctypes.data_as(dp), i(1), src.ctypes.data_as(dp), i(0), sig.ctypes.data_as(dp),
                              i(1), sig.ctypes.data_as(dp), i(1), out.ctypes.data_as(dp), i(1),
                              out.ctypes.data_as(dp), i(1), tgt.ctypes.data_as(dp), i(1), out.ctypes.data_as(dp),
                              i(1), out.ctypes.data_as(dp))
        assert ier.value == want
