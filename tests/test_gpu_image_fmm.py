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
