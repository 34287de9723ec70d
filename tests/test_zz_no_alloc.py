"""The allocation-free direct sum (efmm_direct_noalloc) against the regular
direct-sum entry point, through the C ABI, on two calls in a row.

The entry point exists for callers that cannot allocate device memory when
they need the result (their memory pool already holds the device's free
memory, or their loop cannot afford an allocation's synchronisation); it keeps
its intermediates in fixed scratch arrays, so two consecutive calls must not
see each other's leftovers, and a warm call must take no device memory.  This
file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from conftest import rel
from elfmmlib3d_b200 import geometry as G

pytestmark = pytest.mark.gpu

SHAPES = lambda n, m: ((n, 3), (n, 3, 3), (m, 3), (m, 3, 3))


def _noalloc(L, n, dtri, dcen, ssl, sdl, m, dtg, out):
    ptr = lambda t: t.data_ptr() if t is not None else None
    return L.efmm_direct_noalloc(1.3, 0.7, n, dtri.data_ptr(), dcen.data_ptr(), ptr(ssl), ptr(sdl), m,
                                 ptr(dtg), *[ptr(t) for t in out], None)


# output masks (u_src, e_src, u_tgt, e_tgt) and target counts: all outputs,
# target-only (the target scratch still starts after the n centroids),
# displacement at targets alone, strain at the centroids alone, no targets
CASES = [((1, 1, 1, 1), 300), ((0, 0, 1, 1), 300), ((0, 0, 1, 0), 300), ((0, 1, 0, 0), 300),
         ((1, 1, 0, 0), 0), ((1, 0, 1, 0), 0)]


@pytest.mark.parametrize("mask,m", CASES)
def test_noalloc_matches_direct_two_calls(gpu, mask, m):
    import torch
    L = gpu.load()
    tri, nrm, cen = G.sphere_triangles(3)
    n = len(cen)
    tg = G.box_targets(m, 4) if m else None
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    dtri, dnrm, dcen = d(tri), d(nrm), d(cen)
    dtg = d(tg) if m else None
    P = gpu.Plan(0)
    P.set_geometry(dtri, dnrm, dcen, dtg, iprec=2)
    rng = np.random.default_rng(12)
    for call in range(2):
        ssl = d(rng.normal(size=(n, 3)))
        sdl = d(rng.normal(size=(n, 3))) if call == 0 else None
        ref = [torch.zeros(s, dtype=torch.float64, device="cuda") if (k and s[0]) else None
               for k, s in zip(mask, SHAPES(n, m))]
        P.evaluate(1.3, 0.7, ssl, sdl, *ref, direct=True)
        out = [torch.full(s, np.nan, dtype=torch.float64, device="cuda") if (k and s[0]) else None
               for k, s in zip(mask, SHAPES(n, m))]
        torch.cuda.synchronize()
        assert _noalloc(L, n, dtri, dcen, ssl, sdl, m, dtg, out) == 0
        torch.cuda.synchronize()
        for a, b in zip(out, ref):
            if b is not None:
                assert rel(a.cpu().numpy(), b.cpu().numpy()) < 1e-13
    P.close()


def test_noalloc_warm_call_takes_no_device_memory(gpu):
    """After one warm-up call (which loads the scratch on this device), a
    second call changes neither the device's free memory nor torch's
    allocation count."""
    import torch
    L = gpu.load()
    tri, nrm, cen = G.sphere_triangles(2)
    n = len(cen)
    tg = G.box_targets(50, 5)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    dtri, dcen, dtg = d(tri), d(cen), d(tg)
    rng = np.random.default_rng(3)
    ssl, sdl = d(rng.normal(size=(n, 3))), d(rng.normal(size=(n, 3)))
    out = [torch.zeros(s, dtype=torch.float64, device="cuda") for s in SHAPES(n, len(tg))]
    assert _noalloc(L, n, dtri, dcen, ssl, sdl, len(tg), dtg, out) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    assert _noalloc(L, n, dtri, dcen, ssl, sdl, len(tg), dtg, out) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0


def test_noalloc_rejects_oversize(gpu):
    L = gpu.load()
    ier = L.efmm_direct_noalloc(1.0, 1.0, 40000, 1, 1, 1, None, 0, None, 1, None, None, None, None)
    assert ier == 16
