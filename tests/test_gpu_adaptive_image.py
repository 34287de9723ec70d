"""Error control of the image quadrature: the GPU direct image sum and the
image FMM (whose stored near field uses the same quadrature) against the
oracle's independent adaptive integration (tria3adam's scheme,
src/tria3adamar.f:33-395, at eps 1e-10), on faults that reach or nearly
reach the surface, where the reflected targets come close to the triangles
and the distance refinement alone runs into its depth cap."""
import numpy as np
import pytest

from conftest import rel
from elfmmlib3d_b200 import geometry as G

pytestmark = pytest.mark.gpu

CASES = {
    "surface-breaking-60": dict(dip=60.0, top=0.0),
    "surface-breaking-vertical": dict(dip=90.0, top=0.0),
    "shallow-15-near-surface": dict(dip=15.0, top=0.05),
}


def _case(name, nl=8, nw=4):
    c = CASES[name]
    tri, nrm, cen, _ = G.planar_fault(nl, nw, length=6.0, width=3.0, dip_deg=c["dip"], top_depth=c["top"])
    rng = np.random.default_rng(17)
    ssl, sdl = rng.normal(size=cen.shape), rng.normal(size=cen.shape)
    near = np.array([[0.3, 0.05, -1e-3], [1.0, 0.4, -0.01], [-1.5, 0.2, -0.05], [2.0, 1.0, -0.3]])
    return tri, nrm, cen, ssl, sdl, np.vstack([cen, near])


@pytest.mark.parametrize("name", list(CASES))
def test_direct_image_sum_against_adaptive_oracle(gpu, oracle, name):
    tri, nrm, cen, ssl, sdl, tg = _case(name)
    gpu.hs_capped()
    for a, b in ((ssl, sdl), (None, sdl), (ssl, None)):
        ier, u, e = gpu.hs_image_direct(1.3, 0.7, tri, nrm, a, b, tg)
        assert ier == 0
        uo, eo, cap = oracle.image_direct_adaptive(1.3, 0.7, tri, nrm, a, b, tg, eps=1e-10)
        assert cap == 0
        eu, ee = rel(u, uo), rel(e, eo)
        print(f"{name}: u {eu:.2e} strain {ee:.2e}")
        assert eu < 1e-7 and ee < 1e-7
    assert gpu.hs_capped() == 0


@pytest.mark.parametrize("name", ["surface-breaking-60", "shallow-15-near-surface"])
def test_image_fmm_store_against_adaptive_oracle(gpu, oracle, name):
    """elhfmm3dtriatargiter at iprec 3 (the stored image near field with its
    adaptive quadrature, the image far field) against the oracle."""
    tri, nrm, cen, ssl, sdl, tg = _case(name, nl=24, nw=10)
    w = np.zeros(8)
    gpu.hs_capped()
    ier, _, u, e = gpu.elhfmm3dtriatargiter(3, 1.3, 0.7, tri, nrm, cen, ssl, sdl, tg, icomp_type=2, wsave=w)
    assert ier == 0
    sub = np.concatenate([np.arange(0, len(cen), 7), np.arange(len(cen), len(tg))])
    uo, eo, cap = oracle.image_direct_adaptive(1.3, 0.7, tri, nrm, ssl, sdl, tg[sub], eps=1e-10)
    eu, ee = rel(u[sub], uo), rel(e[sub], eo)
    print(f"{name} image FMM vs adaptive oracle: u {eu:.2e} strain {ee:.2e}")
    assert cap == 0 and gpu.hs_capped() == 0
    assert eu < 1e-7 and ee < 1e-7
    assert gpu.iter_release(w) == 0
