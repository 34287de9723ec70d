"""The oracle's C image direct sum (oracle/image.c over the kernels that
oracle/gen_image_c.py prints from oracle/mindlin.py) against the numpy
lambdification of the same expressions (mindlin.image_direct), and its
adaptive refinement against fine uniform subdivision."""
import numpy as np
import pytest

from conftest import rel
from elfmmlib3d_b200 import geometry as G


@pytest.fixture(scope="module")
def fault():
    tri, nrm, cen, _ = G.planar_fault(3, 2, length=4.0, width=3.0, dip_deg=45.0, top_depth=1.0)
    rng = np.random.default_rng(11)
    ssl, sdl = rng.normal(size=cen.shape), rng.normal(size=cen.shape)
    extra = np.array([[0.3, 0.4, -0.5], [-1.2, 2.0, -3.0], [2.5, -0.5, -0.05]])
    return tri, nrm, np.vstack([cen, extra]), ssl, sdl


@pytest.mark.parametrize("layers", ["both", "sl", "dl"])
def test_c_image_matches_numpy(oracle, fault, layers):
    from oracle import mindlin as M
    tri, nrm, tg, ssl, sdl = fault
    ssl = ssl if layers in ("both", "sl") else None
    sdl = sdl if layers in ("both", "dl") else None
    uc, ec = oracle.image_direct(1.3, 0.7, tri, nrm, ssl, sdl, tg, level=1)
    un, en = M.image_direct(1.3, 0.7, tri, nrm, ssl, sdl, tg, level=1)
    assert rel(uc, un) < 1e-12 and rel(ec, en) < 1e-12
    assert np.array_equal(ec, ec.transpose(0, 2, 1))


def test_c_image_adaptive_converged(oracle, fault):
    tri, nrm, tg, ssl, sdl = fault
    ua, ea = oracle.image_direct(1.0, 1.0, tri, nrm, ssl, sdl, tg, level=-1)
    uf, ef = oracle.image_direct(1.0, 1.0, tri, nrm, ssl, sdl, tg, level=5)
    assert rel(ua, uf) < 1e-10 and rel(ea, ef) < 1e-10


def test_c_image_rejects_bad_level(oracle, fault):
    tri, nrm, tg, ssl, sdl = fault
    with pytest.raises(ValueError):
        oracle.image_direct(1.0, 1.0, tri, nrm, ssl, sdl, tg, level=13)


def test_c_adaptive_converges_and_matches_refinement(oracle, fault):
    """The oracle's tria3adam-style adaptive mode (src/tria3adamar.f:33-395):
    tighter tolerances converge, and the result agrees with the distance
    refinement; no pair reaches the depth cap."""
    tri, nrm, tg, ssl, sdl = fault
    ur, er = oracle.image_direct(1.3, 0.7, tri, nrm, ssl, sdl, tg, level=-1)
    u6, e6, c6 = oracle.image_direct_adaptive(1.3, 0.7, tri, nrm, ssl, sdl, tg, eps=1e-6)
    u12, e12, c12 = oracle.image_direct_adaptive(1.3, 0.7, tri, nrm, ssl, sdl, tg, eps=1e-12)
    assert c6 == 0 and c12 == 0
    assert rel(u6, u12) < 1e-7 and rel(e6, e12) < 1e-7
    assert rel(ur, u12) < 1e-10 and rel(er, e12) < 1e-10


def test_c_adaptive_surface_breaking_fault(oracle):
    """A fault whose top edge lies on the surface, targets down to 1e-3 below
    it: the adaptive sum converges (1e-9 against 1e-12) without the cap."""
    tri, nrm, cen, _ = G.planar_fault(4, 2, length=4.0, width=2.0, dip_deg=60.0, top_depth=0.0)
    rng = np.random.default_rng(5)
    sdl = rng.normal(size=cen.shape)
    tg = np.vstack([cen, [[0.3, 0.05, -1e-3], [1.1, -0.2, -0.02]]])
    u9, e9, c9 = oracle.image_direct_adaptive(1.0, 1.0, tri, nrm, None, sdl, tg, eps=1e-9)
    u12, e12, c12 = oracle.image_direct_adaptive(1.0, 1.0, tri, nrm, None, sdl, tg, eps=1e-12)
    assert c9 == 0 and c12 == 0
    assert rel(u9, u12) < 1e-8 and rel(e9, e12) < 1e-8
