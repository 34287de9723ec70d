"""Half-space image part as an FMM (efmm_plan_evaluate_image) against the
direct image sum (all pairs, the same refined quadrature), at the iprec
tolerance: the anti-image passes, the 1/r potentials of the C piece and the
U potential of the B piece through the far field, the near lists through
the stored image blocks."""
import numpy as np
import pytest

from conftest import rel
from elfmmlib3d_b200 import geometry as G

pytestmark = pytest.mark.gpu


def _t():
    import torch
    return torch


def _setup(gpu, nl=50, nw=20, iprec=2, extra=True, seed=0):
    torch = _t()
    tri, nrm, cen, us = G.planar_fault(nl, nw)
    tg = cen.copy()
    if extra:
        rng = np.random.default_rng(seed)
        gx, gy = np.meshgrid(np.linspace(-25, 25, 11), np.linspace(-5, 20, 6))
        surf = np.stack([gx.ravel(), gy.ravel(), np.zeros(gx.size)], axis=1)
        below = np.stack([rng.uniform(-25, 25, 60), rng.uniform(-5, 20, 60), -rng.uniform(0.1, 16, 60)], axis=1)
        tg = np.vstack([tg, surf, below])
    tgr = tg * np.array([1.0, 1.0, -1.0])
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    P = gpu.Plan(0)
    P.set_geometry(d(tri), d(nrm), d(cen), d(tgr), iprec=iprec, mindlin=True)
    return P, tri, nrm, cen, tg, d


def _image(P, d, R, ssl, sdl, m, precision=0, mode=0, strain=True, rlam=1.3, rmu=0.7):
    torch = _t()
    u = torch.zeros((R, m, 3), dtype=torch.float64, device="cuda")
    e = torch.zeros((R, m, 3, 3), dtype=torch.float64, device="cuda") if strain else None
    P.evaluate_image(rlam, rmu, R, d(ssl) if ssl is not None else None, d(sdl) if sdl is not None else None, u, e,
                     precision=precision, mode=mode)
    return u.cpu().numpy(), (e.cpu().numpy() if strain else None)


@pytest.mark.parametrize("layers", ["sl", "dl", "both"])
def test_image_fmm_matches_direct(gpu, layers):
    P, tri, nrm, cen, tg, d = _setup(gpu)
    assert P.info()["nlev"] >= 3 if "nlev" in P.info() else True
    rng = np.random.default_rng(1)
    ssl = rng.normal(size=cen.shape) if layers in ("sl", "both") else None
    sdl = rng.normal(size=cen.shape) if layers in ("dl", "both") else None
    u, e = _image(P, d, 1, None if ssl is None else ssl[None], None if sdl is None else sdl[None], len(tg))
    ier, ud, ed = gpu.hs_image_direct(1.3, 0.7, tri, nrm, ssl, sdl, tg)
    assert ier == 0
    eu, ee = rel(u[0], ud), rel(e[0], ed)
    print(f"image FMM vs direct ({layers}): u {eu:.2e}  strain {ee:.2e}")
    assert eu < 2e-6 and ee < 2e-6
    P.close()


def test_image_fmm_iprec3_and_forms(gpu):
    # iprec 3: tighter than iprec 2; the mixed form within its FP32 error;
    # batches equal single evaluations; the stored blocks replay exactly
    P, tri, nrm, cen, tg, d = _setup(gpu, nl=40, nw=20, iprec=3, seed=3)
    m = len(tg)
    rng = np.random.default_rng(5)
    R = 5
    ssl, sdl = rng.normal(size=(R,) + cen.shape), rng.normal(size=(R,) + cen.shape)
    u, e = _image(P, d, R, ssl, sdl, m)
    ier, ud, ed = gpu.hs_image_direct(1.3, 0.7, tri, nrm, ssl[R - 1], sdl[R - 1], tg)
    assert ier == 0
    eu, ee = rel(u[R - 1], ud), rel(e[R - 1], ed)
    print(f"iprec 3 image FMM vs direct: u {eu:.2e}  strain {ee:.2e}")
    assert eu < 5e-7 and ee < 5e-7
    u1, e1 = _image(P, d, 1, ssl[2:3], sdl[2:3], m)
    assert rel(u1[0], u[2]) < 1e-12 and rel(e1[0], e[2]) < 1e-12
    um, em = _image(P, d, R, ssl, sdl, m, precision=1)
    print(f"mixed vs FP64: u {rel(um, u):.2e}  strain {rel(em, e):.2e}")
    assert rel(um, u) < 1e-6 and rel(em, e) < 1e-6 and rel(um, u) > 1e-13
    # store on the first call, replay with new densities
    _image(P, d, R, ssl, sdl, m, mode=1)
    assert P.stored_bytes() > 0
    s2, d2 = rng.normal(size=(R,) + cen.shape), rng.normal(size=(R,) + cen.shape)
    ur, er = _image(P, d, R, s2, d2, m, mode=2)
    u0, e0 = _image(P, d, R, s2, d2, m, mode=0)
    assert rel(ur, u0) < 1e-12 and rel(er, e0) < 1e-12
    with pytest.raises(gpu.ElfmmError) as ex:
        _image(P, d, R, s2, d2, m, mode=2, rlam=1.4)
    assert ex.value.ier == 512
    P.close()


def test_image_p2m_unit_multipoles_match_node_products(gpu, monkeypatch):
    # image plan: the seven columns (anti-image, C piece, U piece) through
    # per-triangle unit-density multipoles equal the node-feature products
    P, tri, nrm, cen, tg, d = _setup(gpu, nl=40, nw=20, iprec=3, seed=4)
    monkeypatch.setenv("ELFMM3D_P2M", "nodes")
    Pn, *_ = _setup(gpu, nl=40, nw=20, iprec=3, seed=4)
    monkeypatch.delenv("ELFMM3D_P2M")
    m = len(tg)
    rng = np.random.default_rng(6)
    R = 12
    ssl, sdl = rng.normal(size=(R,) + cen.shape), rng.normal(size=(R,) + cen.shape)
    u, e = _image(P, d, R, ssl, sdl, m)
    un, en = _image(Pn, d, R, ssl, sdl, m)
    print(f"unit vs nodes (FP64): u {rel(u, un):.2e}  strain {rel(e, en):.2e}")
    assert rel(u, un) < 1e-12 and rel(e, en) < 1e-12
    um, em = _image(P, d, R, ssl, sdl, m, precision=1)
    unm, enm = _image(Pn, d, R, ssl, sdl, m, precision=1)
    print(f"unit vs nodes (mixed): u {rel(um, unm):.2e}  strain {rel(em, enm):.2e}")
    assert rel(um, unm) < 1e-6 and rel(em, enm) < 1e-6
    assert rel(um, u) < 1e-6 and rel(em, e) < 1e-6
    P.close()
    Pn.close()


def test_image_fmm_traction_free_surface(gpu):
    # the total field (free-space FMM + image FMM) has zero traction on z = 0
    torch = _t()
    tri, nrm, cen, us = G.planar_fault(30, 15)
    gx, gy = np.meshgrid(np.linspace(-30, 30, 13), np.linspace(-10, 25, 8))
    surf = np.stack([gx.ravel(), gy.ravel(), np.zeros(gx.size)], axis=1)
    rng = np.random.default_rng(8)
    sdl = rng.normal(size=cen.shape)
    lam, mu = 1.3, 0.7
    _, _, ufree, efree = gpu.el3dtriadirecttarg(lam, mu, tri, nrm, cen, None, sdl, surf)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    P = gpu.Plan(0)
    P.set_geometry(d(tri), d(nrm), d(cen), d(surf), iprec=3, mindlin=True)
    _, eimg = _image(P, d, 1, None, sdl[None], len(surf), rlam=lam, rmu=mu)

    def traction(e):
        tr = np.trace(e, axis1=1, axis2=2)
        sig = lam * tr[:, None, None] * np.eye(3)[None] + 2 * mu * e
        return sig[:, :, 2]

    t_free = traction(efree)
    t_tot = traction(efree + eimg[0])
    print(f"surface traction / free traction: {np.abs(t_tot).max() / np.abs(t_free).max():.2e}")
    assert np.abs(t_tot).max() < 1e-6 * np.abs(t_free).max()
    P.close()


def test_image_fmm_rejects_non_halfspace_plan(gpu):
    torch = _t()
    tri, nrm, cen, us = G.planar_fault(4, 3)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    P = gpu.Plan(0)
    P.set_geometry(d(tri), d(nrm), d(cen), d(cen * np.array([1, 1, -1.0])), iprec=2)  # mindlin not set
    with pytest.raises(gpu.ElfmmError) as ex:
        _image(P, d, 1, None, np.ones((1,) + cen.shape), len(cen))
    assert ex.value.ier == 16
    P.close()


def test_image_fmm_matches_c_oracle(gpu, oracle):
    # the image FMM at iprec 3 against the oracle's C image sum (its own
    # kernels and refinement, independent of the product's direct sum) on
    # every 40th centroid and all off-surface and surface targets
    P, tri, nrm, cen, tg, d = _setup(gpu, nl=40, nw=20, iprec=3, seed=3)
    rng = np.random.default_rng(9)
    ssl, sdl = rng.normal(size=cen.shape), rng.normal(size=cen.shape)
    u, e = _image(P, d, 1, ssl[None], sdl[None], len(tg))
    P.close()
    sub = np.concatenate([np.arange(0, len(cen), 40), np.arange(len(cen), len(tg))])
    uo, eo = oracle.image_direct(1.3, 0.7, tri, nrm, ssl, sdl, tg[sub], level=-1)
    eu, ee = rel(u[0][sub], uo), rel(e[0][sub], eo)
    print(f"iprec 3 image FMM vs C oracle: u {eu:.2e}  strain {ee:.2e}")
    # the FMM's own error at iprec 3 (2e-11 displacement, 5e-10 strain against
    # the direct image sum, which equals the oracle's sum to rounding)
    assert eu < 1e-9 and ee < 2e-9
