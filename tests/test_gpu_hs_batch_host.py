"""The half-space many-right-hand-side host entry point
(elhfmm3dtria_batch_host) against the reference-shaped single calls: for each
right-hand side the half-space total of elhfmm3dtria_total_ (direct arrival
through the free-space FMM plus the image part through the image FMM), the
sum the reference's drivers form from an elfmm3dtriatarg and an
elhfmm3dtriatargiter call (examples/elhfmm3dtria_self_iter_dr.f:331-385).
The store call (icomp_type 2) and two replays with new densities
(icomp_type 3, CUDA-graph replay) are checked; FP64 to the FMM's own error
at iprec 3 (the batched and the single-column passes take different routes
to it: 2e-10 displacement, 6e-10 strain measured), the mixed form to its
stated 1e-6 (displacement) / 1e-5 (strain)."""
import numpy as np
import pytest

from conftest import rel
from elfmmlib3d_b200 import geometry as G

pytestmark = pytest.mark.gpu


def _fault():
    return G.planar_fault(30, 12, length=12.0, width=6.0, dip_deg=45.0, top_depth=0.5)


@pytest.mark.parametrize("precision", [0, 1])
def test_hs_batch_host_store_and_replay(gpu, precision):
    tri, nrm, cen, _ = _fault()
    n, R = len(cen), 3
    rng = np.random.default_rng(5 + precision)
    ws = np.zeros(8)
    tol_u, tol_e = (2e-9, 5e-9) if precision == 0 else (1e-6, 1e-5)
    for call, icomp in enumerate((2, 3, 3)):
        sdl = rng.normal(size=(R, n, 3))
        ssl = rng.normal(size=(R, n, 3)) if precision == 0 else None
        ier, u, e = gpu.hs_batch_host(3, 1.3, 0.7, tri, nrm, cen, ssl, sdl, precision=precision, icomp_type=icomp,
                                      wsave=ws)
        assert ier == 0
        for r in range(R):
            ier, ur, er, _, _ = gpu.elhfmm3dtria_total(3, 1.3, 0.7, tri, nrm, cen, None if ssl is None else ssl[r],
                                                       sdl[r])
            assert ier == 0
            eu, ee = rel(u[r], ur), rel(e[r], er)
            assert eu < tol_u and ee < tol_e, (call, r, eu, ee)
    assert gpu.iter_release(ws) == 0


def test_hs_batch_host_rejects_a_changed_call(gpu):
    tri, nrm, cen, _ = _fault()
    n = len(cen)
    rng = np.random.default_rng(9)
    ws = np.zeros(8)
    sdl = rng.normal(size=(2, n, 3))
    ier, _, _ = gpu.hs_batch_host(2, 1.0, 1.0, tri, nrm, cen, None, sdl, precision=1, icomp_type=2, wsave=ws)
    assert ier == 0
    # another right-hand-side count, another precision, moved geometry: the handle does not match
    ier, _, _ = gpu.hs_batch_host(2, 1.0, 1.0, tri, nrm, cen, None, sdl[:1], precision=1, icomp_type=3, wsave=ws)
    assert ier == 512
    ier, _, _ = gpu.hs_batch_host(2, 1.0, 1.0, tri, nrm, cen, None, sdl, precision=0, icomp_type=3, wsave=ws)
    assert ier == 512
    ier, _, _ = gpu.hs_batch_host(2, 1.0, 1.0, tri - np.array([0, 0, 0.1]), nrm, cen - np.array([0, 0, 0.1]), None,
                                  sdl, precision=1, icomp_type=3, wsave=ws)
    assert ier == 512
    # a source above the surface
    ier, _, _ = gpu.hs_batch_host(2, 1.0, 1.0, tri + np.array([0, 0, 5.0]), nrm, cen + np.array([0, 0, 5.0]), None,
                                  sdl, precision=1, icomp_type=1)
    assert ier == 16
    assert gpu.iter_release(ws) == 0
