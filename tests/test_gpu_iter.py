"""ITER entry point (src/elfmm3dtria_iter_1.f:160): store the near-field
interactions once, reuse them with new densities.  Parity is against the plain
evaluation on the same tree (icomp_type 1), against the oracle's golden
fixture, and against the handle rules (mismatch -> ier 512)."""
import numpy as np
import pytest

from conftest import golden, rel
from elfmmlib3d_b200 import geometry as G

pytestmark = pytest.mark.gpu

# stored blocks x densities vs the analytic near field: same integrals,
# different summation order
SAME = 1e-12


def _case(seed=0, level=3, ntarg=150):
    tri, nrm, cen = G.sphere_triangles(level)
    tg = G.box_targets(ntarg, 11 + seed)
    rng = np.random.default_rng(seed)
    return tri, nrm, cen, tg, rng.normal(size=cen.shape), rng.normal(size=cen.shape)


def test_iter_store_and_replay_match_plain(gpu):
    tri, nrm, cen, tg, ssl, sdl = _case(0)
    w = np.zeros(8)
    ier, lused, *a = gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, cen, ssl, sdl, tg, icomp_type=2, wsave=w)
    assert ier == 0 and lused == 8 and w[0] != 0
    ier, _, *b = gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, cen, ssl, sdl, tg, icomp_type=1)
    assert ier == 0
    for x, y in zip(a, b):
        assert rel(x, y) < SAME
    assert gpu.iter_stored_bytes(w) > 0
    # new densities through the stored operator
    rng = np.random.default_rng(7)
    for _ in range(2):
        s2, d2 = rng.normal(size=cen.shape), rng.normal(size=cen.shape)
        ier, _, *c = gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, cen, s2, d2, tg, icomp_type=3, wsave=w)
        assert ier == 0
        ier, _, *d = gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, cen, s2, d2, tg, icomp_type=1)
        assert ier == 0
        for x, y in zip(c, d):
            assert rel(x, y) < SAME
    assert gpu.iter_release(w) == 0
    assert gpu.iter_release(w) == 512


def test_iter_golden(gpu):
    g = golden("golden_sphere320.npz")
    w = np.zeros(8)
    ier, _, pt, st, ptt, stt = gpu.elfmm3dtriatargiter(2, float(g["rlam"]), float(g["rmu"]), g["tri"], g["nrm"],
                                                       g["cen"], g["ssl"], g["sdl"], g["tgt"], icomp_type=2,
                                                       wsave=w)
    assert ier == 0
    assert rel(pt, g["pt"]) < 0.5e-6 and rel(ptt, g["ptt"]) < 0.5e-6
    assert rel(st, g["st"]) < 0.5e-5 and rel(stt, g["stt"]) < 0.5e-5
    ier, _, pt3, st3, ptt3, stt3 = gpu.elfmm3dtriatargiter(2, float(g["rlam"]), float(g["rmu"]), g["tri"],
                                                           g["nrm"], g["cen"], g["ssl"], g["sdl"], g["tgt"],
                                                           icomp_type=3, wsave=w)
    assert ier == 0
    assert rel(pt3, pt) < SAME and rel(st3, st) < SAME and rel(ptt3, ptt) < SAME and rel(stt3, stt) < SAME
    gpu.iter_release(w)


def test_iter_single_layer_displacement_only(gpu):
    tri, nrm, cen, tg, ssl, _ = _case(1, level=2, ntarg=40)
    w = np.zeros(10)
    ier, _, pt, _, ptt, _ = gpu.elfmm3dtriatargiter(1, 1.0, 1.0, tri, nrm, cen, ssl, None, tg, icomp_type=2,
                                                    wsave=w, ifstrain=0, ifstraintarg=0)
    assert ier == 0
    s2 = np.random.default_rng(3).normal(size=cen.shape)
    ier, _, pt3, _, ptt3, _ = gpu.elfmm3dtriatargiter(1, 1.0, 1.0, tri, nrm, cen, s2, None, tg, icomp_type=3,
                                                      wsave=w, ifstrain=0, ifstraintarg=0)
    assert ier == 0
    ier, _, pt1, _, ptt1, _ = gpu.elfmm3dtriatargiter(1, 1.0, 1.0, tri, nrm, cen, s2, None, tg, icomp_type=1,
                                                      ifstrain=0, ifstraintarg=0)
    assert rel(pt3, pt1) < SAME and rel(ptt3, ptt1) < SAME
    # a replay asking for strain the store does not hold is a handle mismatch
    ier, *_ = gpu.elfmm3dtriatargiter(1, 1.0, 1.0, tri, nrm, cen, s2, None, tg, icomp_type=3, wsave=w)
    assert ier == 512
    gpu.iter_release(w)


def test_iter_handle_mismatch(gpu):
    tri, nrm, cen, tg, ssl, sdl = _case(2, level=2, ntarg=30)
    w = np.zeros(8)
    assert gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, cen, ssl, sdl, tg, icomp_type=2, wsave=w)[0] == 0
    moved = cen.copy()
    moved[0, 0] += 1e-9
    assert gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, moved, ssl, sdl, tg, icomp_type=3, wsave=w)[0] == 512
    assert gpu.elfmm3dtriatargiter(1, 3.2, 2.3, tri, nrm, cen, ssl, sdl, tg, icomp_type=3, wsave=w)[0] == 512
    assert gpu.elfmm3dtriatargiter(2, 3.0, 2.3, tri, nrm, cen, ssl, sdl, tg, icomp_type=3, wsave=w)[0] == 512
    assert gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, cen, ssl, None, tg, icomp_type=3, wsave=w)[0] == 512
    assert gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, cen, ssl, sdl, tg, icomp_type=3,
                                   wsave=np.zeros(8))[0] == 512
    # the store is still good after the rejected calls
    assert gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, cen, ssl, sdl, tg, icomp_type=3, wsave=w)[0] == 0
    gpu.iter_release(w)
    assert gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, cen, ssl, sdl, tg, icomp_type=3, wsave=w)[0] == 512


def test_iter_modes_0_4_5_and_short_wsave(gpu):
    # large enough (5120 triangles) for the tree to have a far field
    tri, nrm, cen, tg, ssl, sdl = _case(3, level=4, ntarg=30)
    ier, lused, pt, *_ = gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, cen, ssl, sdl, tg, icomp_type=0)
    assert ier == 0 and lused == 8 and not pt.any()
    w = np.zeros(8)
    ier, lused, pt, *_ = gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, cen, ssl, sdl, tg, icomp_type=4, wsave=w)
    assert ier == 0 and lused == 8 and not pt.any() and w[0] == 0
    ref = gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, cen, ssl, sdl, tg, icomp_type=1)
    # wsave too short for the handle: plain evaluation, no handle written
    short = np.zeros(4)
    out = gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, cen, ssl, sdl, tg, icomp_type=2, wsave=short)
    assert out[0] == 0 and not short.any()
    for x, y in zip(out[2:], ref[2:]):
        assert rel(x, y) < SAME
    # icomp 5 stores the near field only; a replay adds the far field
    ier, _, ptn, *_ = gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, cen, ssl, sdl, tg, icomp_type=5, wsave=w)
    assert ier == 0 and rel(ptn, ref[2]) > 1e-8
    out = gpu.elfmm3dtriatargiter(2, 3.2, 2.3, tri, nrm, cen, ssl, sdl, tg, icomp_type=3, wsave=w)
    assert out[0] == 0
    for x, y in zip(out[2:], ref[2:]):
        assert rel(x, y) < SAME
    gpu.iter_release(w)


def test_iter_eviction(gpu):
    tri, nrm, cen, tg, ssl, sdl = _case(4, level=1, ntarg=10)
    ws = [np.zeros(8) for _ in range(5)]
    for w in ws:
        assert gpu.elfmm3dtriatargiter(2, 1.0, 1.0, tri, nrm, cen, ssl, sdl, tg, icomp_type=2, wsave=w)[0] == 0
    # four stores stay live; the first (least recently used) was evicted
    assert gpu.elfmm3dtriatargiter(2, 1.0, 1.0, tri, nrm, cen, ssl, sdl, tg, icomp_type=3, wsave=ws[0])[0] == 512
    for w in ws[1:]:
        assert gpu.elfmm3dtriatargiter(2, 1.0, 1.0, tri, nrm, cen, ssl, sdl, tg, icomp_type=3, wsave=w)[0] == 0
        assert gpu.iter_release(w) == 0


def test_iter_on_surface_variant(gpu):
    tri, nrm, cen, _, ssl, sdl = _case(5, level=2, ntarg=1)
    w = np.zeros(8)
    ier, lused, pt, st = gpu.elfmm3dtriaiter(2, 3.2, 2.3, tri, nrm, cen, ssl, sdl, icomp_type=2, wsave=w)
    assert ier == 0 and lused == 8
    ier, _, pt3, st3 = gpu.elfmm3dtriaiter(2, 3.2, 2.3, tri, nrm, cen, ssl, sdl, icomp_type=3, wsave=w)
    assert ier == 0 and rel(pt3, pt) < SAME and rel(st3, st) < SAME
    ier, pt1, st1 = gpu.elfmm3dtria(2, 3.2, 2.3, tri, nrm, cen, ssl, sdl)
    # the ITER tree has twice the leaf capacity: same answer within iprec 2
    assert ier == 0 and rel(pt, pt1) < 0.5e-6 and rel(st, st1) < 0.5e-5
    gpu.iter_release(w)
