"""Repeated batched evaluations replayed as one CUDA graph
(efmm_plan_evaluate_batch_graph / efmm_plan_evaluate_image_graph): new
densities written into the same buffers give the results of the plain
calls, for the free-space batch (stored and analytic near field) and the
half-space image batch."""
import numpy as np
import pytest

from conftest import rel
from elfmmlib3d_b200 import geometry as G

pytestmark = pytest.mark.gpu


def test_graph_batch_and_image_replay(gpu):
    import torch
    tri, nrm, cen, _ = G.planar_fault(40, 20)
    n, R = len(cen), 40
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    dtri, dnrm, dcen = d(tri), d(nrm), d(cen)
    F, I = gpu.Plan(0), gpu.Plan(0)
    F.set_geometry(dtri, dnrm, dcen, None, iprec=3, iter=True)
    I.set_geometry(dtri, dnrm, dcen, d(cen * np.array([1, 1, -1.0])), iprec=3, iter=True, mindlin=True)
    rng = np.random.default_rng(4)
    sdl = d(rng.normal(size=(R, n, 3)))
    z = lambda *s: torch.zeros(s, dtype=torch.float64, device="cuda")
    u, e, ui, ei = z(R, n, 3), z(R, n, 3, 3), z(R, n, 3), z(R, n, 3, 3)
    F.evaluate_batch(1.0, 1.0, R, None, sdl, u, e, precision=1, mode=1)
    I.evaluate_image(1.0, 1.0, R, None, sdl, ui, ei, precision=1, mode=1)
    u0, e0, ui0, ei0 = z(R, n, 3), z(R, n, 3, 3), z(R, n, 3), z(R, n, 3, 3)
    for it in range(3):
        sdl.copy_(d(rng.normal(size=(R, n, 3))))
        F.evaluate_batch(1.0, 1.0, R, None, sdl, u0, e0, precision=1, mode=2)
        I.evaluate_image(1.0, 1.0, R, None, sdl, ui0, ei0, precision=1, mode=2)
        l0 = gpu.kernel_launches()
        F.evaluate_batch(1.0, 1.0, R, None, sdl, u, e, precision=1, mode=2, graph=True)
        I.evaluate_image(1.0, 1.0, R, None, sdl, ui, ei, precision=1, mode=2, graph=True)
        assert gpu.kernel_launches() > l0
        for a, b in ((u, u0), (e, e0), (ui, ui0), (ei, ei0)):
            assert rel(a.cpu().numpy(), b.cpu().numpy()) < 1e-12
    # analytic near field (mode 0), FP64
    F2 = gpu.Plan(0)
    F2.set_geometry(dtri, dnrm, dcen, None, iprec=2)
    F2.evaluate_batch(1.0, 1.0, R, None, sdl, u0, e0, precision=0)
    F2.evaluate_batch(1.0, 1.0, R, None, sdl, u, e, precision=0, graph=True)
    F2.evaluate_batch(1.0, 1.0, R, None, sdl, u, e, precision=0, graph=True)
    assert rel(u.cpu().numpy(), u0.cpu().numpy()) < 1e-12 and rel(e.cpu().numpy(), e0.cpu().numpy()) < 1e-12
    for P in (F, I, F2):
        P.close()


def test_graph_rejects_chunked_calls(gpu):
    # more than 64 right-hand sides run as several passes: not replayed
    # (IER 16), the plain call serves them
    import torch
    tri, nrm, cen, _ = G.planar_fault(10, 5)
    n, R = len(cen), 70
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    F = gpu.Plan(0)
    F.set_geometry(d(tri), d(nrm), d(cen), None, iprec=2)
    sdl = d(np.random.default_rng(2).normal(size=(R, n, 3)))
    u = torch.zeros((R, n, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(gpu.ElfmmError) as ex:
        F.evaluate_batch(1.0, 1.0, R, None, sdl, u, None, precision=1, graph=True)
    assert ex.value.ier == 16
    F.evaluate_batch(1.0, 1.0, R, None, sdl, u, None, precision=1)
    assert float(u.abs().sum()) > 0
    F.close()
