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
