"""The allocation-free direct sum (efmm_direct_noalloc) against the regular
direct-sum entry point, through the C ABI, on two calls in a row.

The entry point exists for callers that cannot allocate device memory when
they need the result (their memory pool already holds the device's free
memory, or their loop cannot afford an allocation's synchronisation); it keeps
its intermediates in fixed scratch arrays, so two consecutive calls must not
see each other's leftovers.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from conftest import rel
from elfmmlib3d_b200 import geometry as G

pytestmark = pytest.mark.gpu


def test_noalloc_matches_direct_two_calls(gpu):
    import torch
    L = gpu.load()
    tri, nrm, cen = G.sphere_triangles(3)
    tg = G.box_targets(300, 4)
    n, m = len(cen), len(tg)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    dtri, dnrm, dcen, dtg = d(tri), d(nrm), d(cen), d(tg)
    P = gpu.Plan(0)
    P.set_geometry(dtri, dnrm, dcen, dtg, iprec=2)
    rng = np.random.default_rng(12)
    for call in range(2):
        ssl = d(rng.normal(size=(n, 3)))
        sdl = d(rng.normal(size=(n, 3))) if call == 0 else None
        ref = [torch.zeros(s, dtype=torch.float64, device="cuda") for s in ((n, 3), (n, 3, 3), (m, 3), (m, 3, 3))]
        P.evaluate(1.3, 0.7, ssl, sdl, *ref, direct=True)
        out = [torch.full(s, np.nan, dtype=torch.float64, device="cuda") for s in ((n, 3), (n, 3, 3), (m, 3), (m, 3, 3))]
        torch.cuda.synchronize()
        ier = L.efmm_direct_noalloc(1.3, 0.7, n, dtri.data_ptr(), dcen.data_ptr(), ssl.data_ptr(),
                                    sdl.data_ptr() if sdl is not None else None, m, dtg.data_ptr(),
                                    *[t.data_ptr() for t in out], None)
        torch.cuda.synchronize()
        assert ier == 0
        for a, b in zip(out, ref):
            assert rel(a.cpu().numpy(), b.cpu().numpy()) < 1e-13
    P.close()


def test_noalloc_rejects_oversize(gpu):
    L = gpu.load()
    ier = L.efmm_direct_noalloc(1.0, 1.0, 40000, 1, 1, 1, None, 0, None, 1, None, None, None, None)
    assert ier == 16
