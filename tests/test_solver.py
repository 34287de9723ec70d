"""The iterative solver loop (efmm_plan_solve / efmm_gcr_dense_host): the
minimal-residual iteration of the reference's matlab/gmres_simple.m.

CPU: the library's iteration on a dense matrix against a line-by-line numpy
restatement of gmres_simple (same iterates) and against numpy's direct
solve.  GPU: free-space and half-space fault operators (traction of the
slip, displacement of the traction) through the stored near fields: the
solution reproduces the density that made the right-hand side."""
import numpy as np
import pytest

import elfmmlib3d_b200 as E
from conftest import rel
from elfmmlib3d_b200 import geometry as G


def gmres_simple(A, b, tol, maxit):
    """matlab/gmres_simple.m restated in numpy (x0 = 0), one right-hand side."""
    n = len(b)
    Ae = np.zeros((n, maxit))
    e = np.zeros((n, maxit))
    x = np.zeros(n)
    r = b.copy()
    er0 = np.linalg.norm(r)
    for i in range(maxit):
        if (i + 1) % 10 == 0:
            r = b - A @ x
        w = A @ r
        wp, rp = w.copy(), r.copy()
        for j in range(i):
            d = Ae[:, j] @ wp
            wp = wp - d * Ae[:, j]
            rp = rp - d * e[:, j]
        d = 1.0 / np.sqrt(wp @ wp)
        Ae[:, i] = d * wp
        e[:, i] = d * rp
        for j in range(i):
            d = Ae[:, j] @ Ae[:, i]
            Ae[:, i] -= d * Ae[:, j]
            e[:, i] -= d * e[:, j]
        d = 1.0 / np.sqrt(Ae[:, i] @ Ae[:, i])
        Ae[:, i] *= d
        e[:, i] *= d
        d = Ae[:, i] @ r
        r = r - d * Ae[:, i]
        er1 = np.linalg.norm(r)
        if er1 >= er0:
            return x, 8, i + 1
        er0 = er1
        x = x + d * e[:, i]
        if np.linalg.norm(r) < tol * np.linalg.norm(b):
            return x, 0, i + 1
    return x, 4, maxit


def test_dense_iteration_matches_restatement_and_direct_solve():
    rng = np.random.default_rng(2)
    n = 60
    A = np.eye(n) + 0.4 * rng.normal(size=(n, n)) / np.sqrt(n)
    B = rng.normal(size=(3, n))
    X, its, res, ier = E.gcr_dense_host(A, B, tol=1e-12, maxit=60)
    for c in range(3):
        xr, ir, kr = gmres_simple(A, B[c], 1e-12, 60)
        assert ier[c] == ir == 0 and its[c] == kr
        assert rel(X[c], xr) < 1e-10
        assert rel(X[c], np.linalg.solve(A, B[c])) < 1e-10
        assert res[c] < 1e-12


def test_dense_iteration_reports_maxit_and_zero_columns():
    rng = np.random.default_rng(3)
    n = 40
    A = np.eye(n) + 2.0 * rng.normal(size=(n, n)) / np.sqrt(n)  # slow to converge
    B = np.vstack([rng.normal(size=n), np.zeros(n)])
    X, its, res, ier = E.gcr_dense_host(A, B, tol=1e-14, maxit=5)
    xr, ir, kr = gmres_simple(A, B[0], 1e-14, 5)
    assert ier[0] == ir and its[0] == kr and rel(X[0], xr) < 1e-10
    assert ier[1] == 0 and np.all(X[1] == 0)


def _fault_plans(gpu, half, nl=16, nw=8):
    import torch
    top = 0.5 if half else 0.0
    tri, nrm, cen, _ = G.planar_fault(nl, nw, length=8.0, width=4.0, dip_deg=45.0, top_depth=top)
    if not half:
        tri, cen = tri - np.array([0, 0, 10.0]), cen - np.array([0, 0, 10.0])
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    F = gpu.Plan(0)
    F.set_geometry(d(tri), d(nrm), d(cen), None, iprec=3, iter=True)
    I = None
    if half:
        I = gpu.Plan(0)
        I.set_geometry(d(tri), d(nrm), d(cen), d(cen * np.array([1.0, 1.0, -1.0])), iprec=3, iter=True, mindlin=True)
    return tri, nrm, cen, F, I, d


@pytest.mark.gpu
@pytest.mark.parametrize("half", [False, True])
@pytest.mark.parametrize("kind", [0, 1])
def test_solve_recovers_density(gpu, half, kind):
    import torch
    tri, nrm, cen, F, I, d = _fault_plans(gpu, half)
    n, R = len(cen), 3
    rng = np.random.default_rng(7)
    # smooth densities: tapered along strike and dip, plus a little noise
    taper = np.cos(np.pi * (cen[:, 0] / 8.0)) ** 2
    x_true = np.stack([taper[:, None] * rng.normal(size=3)[None, :] + 0.05 * rng.normal(size=(n, 3))
                       for _ in range(R)])
    dx, dn = d(x_true), d(nrm)
    # right-hand side: the operator applied once through the same plans
    u = torch.zeros((R, n, 3), dtype=torch.float64, device="cuda")
    e = torch.zeros((R, n, 3, 3), dtype=torch.float64, device="cuda")
    ssl, sdl = (None, dx) if kind == 0 else (dx, None)
    F.evaluate_batch(1.0, 1.0, R, ssl, sdl, u, e, mode=1)
    if I is not None:
        ui, ei = torch.zeros_like(u), torch.zeros_like(e)
        I.evaluate_image(1.0, 1.0, R, ssl, sdl, ui, ei, mode=1)
        u, e = u + ui, e + ei
    if kind == 0:
        E_ = e.cpu().numpy()
        tr = np.trace(E_, axis1=2, axis2=3)
        rhs = tr[..., None] * nrm[None] + 2.0 * np.einsum("rnij,nj->rni", E_, nrm)
    else:
        rhs = u.cpu().numpy()
    x = torch.zeros((R, n, 3), dtype=torch.float64, device="cuda")
    its, res, ier = F.solve(I, kind, 1.0, 1.0, R, dn, d(rhs), x, tol=1e-10, maxit=60)
    print(f"half={half} kind={kind}: iterations {its}, residual {res}, ier {ier}")
    assert np.all(ier == 0) and np.all(res < 1e-10)
    assert rel(x.cpu().numpy(), x_true) < 1e-6
    F.close()
    if I is not None:
        I.close()
