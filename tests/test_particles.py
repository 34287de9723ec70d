"""The particle FMM (elfmm3dpart / elfmm3dparttarg / el3dpartdirecttarg,
src/elfmm3dpart.f).

CPU: the particle pair kernel (efmm_part_pair_host, the decomposition the
device near field runs) against Kelvin's point-force solution written out,
and against the triangle layer potentials of the same library on a tiny
triangle carrying the same total force or jump (the point limit of the
triangle layers, whose closed forms are pinned against the oracle's
integration in test_near_pair_host.py).
GPU: the particle FMM against the particle direct sum at iprec 1..3, and the
direct sum against host pair sums."""
import ctypes

import numpy as np
import pytest

import elfmmlib3d_b200 as E
from conftest import rel

_dp = ctypes.POINTER(ctypes.c_double)


def kelvin(rlam, rmu, x, y, f):
    """Point force f at y, displacement at x, no 1/(4 pi) (the reference's
    normalisation): ((lam + 3 mu) f / r + (lam + mu) (f.rho) rho / r^3) /
    (2 mu (lam + 2 mu))."""
    rho = np.asarray(x, float) - np.asarray(y, float)
    r = np.linalg.norm(rho)
    return ((rlam + 3 * rmu) * f / r + (rlam + rmu) * (f @ rho) * rho / r ** 3) / (2 * rmu * (rlam + 2 * rmu))


def kelvin_strain(rlam, rmu, x, y, f, h=1e-4):
    """Symmetric gradient of kelvin() in x by a fourth-order difference."""
    G = np.zeros((3, 3))
    for b in range(3):
        e = np.zeros(3)
        e[b] = h
        G[:, b] = (-kelvin(rlam, rmu, x + 2 * e, y, f) + 8 * kelvin(rlam, rmu, x + e, y, f)
                   - 8 * kelvin(rlam, rmu, x - e, y, f) + kelvin(rlam, rmu, x - 2 * e, y, f)) / (12 * h)
    return 0.5 * (G + G.T)


def tiny_triangle(y, nu, h):
    """Equilateral triangle of side ~h centred at y, vertex-order normal nu."""
    nu = np.asarray(nu, float) / np.linalg.norm(nu)
    a = np.cross(nu, [1.0, 0.0, 0.0] if abs(nu[0]) < 0.9 else [0.0, 1.0, 0.0])
    a /= np.linalg.norm(a)
    b = np.cross(nu, a)
    ang = 2 * np.pi / 3 * np.arange(3)
    v = np.array([y + h * (np.cos(t) * a + np.sin(t) * b) for t in ang])
    area = 0.5 * np.linalg.norm(np.cross(v[1] - v[0], v[2] - v[0]))
    assert np.cross(v[1] - v[0], v[2] - v[0]) @ nu > 0
    return v, area


def tri_pair(rlam, rmu, tri, ssl, sdl, x):
    L = E.load()
    u, e6 = np.zeros(3), np.zeros(6)
    keep = [np.ascontiguousarray(a, float) if a is not None else None for a in (tri, ssl, sdl, x)]
    p = lambda a: a.ctypes.data_as(_dp) if a is not None else None
    L.efmm_pair_eval_host.restype = ctypes.c_int
    ier = L.efmm_pair_eval_host(ctypes.c_double(rlam), ctypes.c_double(rmu), p(keep[0]), p(keep[1]), p(keep[2]),
                                p(keep[3]), ctypes.c_int(0), u.ctypes.data_as(_dp), e6.ctypes.data_as(_dp))
    assert ier == 0
    return u, np.array([[e6[0], e6[3], e6[4]], [e6[3], e6[1], e6[5]], [e6[4], e6[5], e6[2]]])


def test_point_force_is_kelvin():
    rng = np.random.default_rng(1)
    for _ in range(5):
        x, y, f = rng.normal(size=3), rng.normal(size=3), rng.normal(size=3)
        rlam, rmu = rng.uniform(0.5, 3.0, size=2)
        u, e = E.part_pair_host(rlam, rmu, x, y, sl=f)
        assert rel(u, kelvin(rlam, rmu, x, y, f)) < 1e-13
        assert rel(e, kelvin_strain(rlam, rmu, x, y, f)) < 1e-8


@pytest.mark.parametrize("layer", ["sl", "dl"])
def test_point_limit_of_a_tiny_triangle(layer):
    """A triangle of side h carrying density s / area acts like a particle of
    strength s (orientation = its normal) up to O((h / r)^2)."""
    rng = np.random.default_rng(2)
    for _ in range(4):
        y, nu, s = rng.normal(size=3), rng.normal(size=3), rng.normal(size=3)
        x = y + rng.normal(size=3) * 2.0
        tri, area = tiny_triangle(y, nu, 1e-3)
        nu_t = np.cross(tri[1] - tri[0], tri[2] - tri[0])
        nu_t /= np.linalg.norm(nu_t)
        if layer == "sl":
            u_p, e_p = E.part_pair_host(1.3, 0.7, x, y, sl=s)
            u_t, e_t = tri_pair(1.3, 0.7, tri, s / area, None, x)
        else:
            u_p, e_p = E.part_pair_host(1.3, 0.7, x, y, dl=s, nu=nu_t)
            u_t, e_t = tri_pair(1.3, 0.7, tri, None, s / area, x)
        assert rel(u_p, u_t) < 1e-6 and rel(e_p, e_t) < 1e-6


def test_coincident_points_contribute_nothing():
    u, e = E.part_pair_host(1.0, 1.0, [0.1, 0.2, 0.3], [0.1, 0.2, 0.3], sl=[1.0, 2.0, 3.0])
    assert np.all(u == 0) and np.all(e == 0)


def _cloud(n, m, seed):
    rng = np.random.default_rng(seed)
    src = rng.uniform(-1, 1, size=(n, 3))
    tgt = rng.uniform(-1.5, 1.5, size=(m, 3))
    sl, dl = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    dv = rng.normal(size=(n, 3))
    dv /= np.linalg.norm(dv, axis=1, keepdims=True)
    return src, tgt, sl, dl, dv


@pytest.mark.gpu
def test_particle_direct_matches_host_pairs(gpu):
    src, tgt, sl, dl, dv = _cloud(60, 20, 3)
    ier, u, e, ut, et = gpu.elfmm3dparttarg(2, 1.3, 0.7, src, sl, dl, dv, tgt, direct=True)
    for pts, uu, ee, self_ in ((src, u, e, True), (tgt, ut, et, False)):
        ur, er = np.zeros_like(uu), np.zeros_like(ee)
        for i, x in enumerate(pts):
            for j in range(len(src)):
                if self_ and i == j:
                    continue
                a, b = gpu.part_pair_host(1.3, 0.7, x, src[j], sl=sl[j], dl=dl[j], nu=dv[j])
                ur[i] += a
                er[i] += b
        assert rel(uu, ur) < 1e-12 and rel(ee, er) < 1e-12


TOL = {1: 0.5e-3, 2: 0.5e-6, 3: 0.5e-9}


@pytest.mark.gpu
@pytest.mark.parametrize("iprec", [1, 2, 3])
@pytest.mark.parametrize("layers", ["sl", "dl", "both"])
def test_particle_fmm_within_iprec_tolerance(gpu, iprec, layers):
    src, tgt, sl, dl, dv = _cloud(20000, 3000, 4 + iprec)
    sl = sl if layers in ("sl", "both") else None
    dl = dl if layers in ("dl", "both") else None
    d = gpu.elfmm3dparttarg(iprec, 1.3, 0.7, src, sl, dl, dv, tgt, direct=True)
    ier, u, e, ut, et = gpu.elfmm3dparttarg(iprec, 1.3, 0.7, src, sl, dl, dv, tgt)
    assert ier == 0
    errs = [rel(u, d[1]), rel(e, d[2]), rel(ut, d[3]), rel(et, d[4])]
    print(f"particles iprec {iprec} {layers}: {errs}")
    assert errs[0] < 2 * TOL[iprec] and errs[2] < 2 * TOL[iprec]
    assert errs[1] < 10 * TOL[iprec] and errs[3] < 10 * TOL[iprec]


def _halfspace_cloud(n, m, seed):
    src, tgt, sl, dl, dv = _cloud(n, m, seed)
    src[:, 2] = -np.abs(src[:, 2]) - 0.05
    tgt[:, 2] = -np.abs(tgt[:, 2]) - 0.01
    return src, tgt, sl, dl, dv


@pytest.mark.gpu
@pytest.mark.parametrize("iprec", [2, 3])
def test_halfspace_particle_fmm_matches_direct(gpu, iprec):
    src, tgt, sl, dl, dv = _halfspace_cloud(8000, 1500, 9 + iprec)
    d = gpu.elfmm3dparttarg(iprec, 1.3, 0.7, src, sl, dl, dv, tgt, direct=True, halfspace=True)
    ier, u, e, ut, et = gpu.elfmm3dparttarg(iprec, 1.3, 0.7, src, sl, dl, dv, tgt, halfspace=True)
    assert ier == 0
    errs = [rel(u, d[1]), rel(e, d[2]), rel(ut, d[3]), rel(et, d[4])]
    print(f"half-space particles iprec {iprec}: {errs}")
    assert errs[0] < 2 * TOL[iprec] and errs[2] < 2 * TOL[iprec]
    assert errs[1] < 10 * TOL[iprec] and errs[3] < 10 * TOL[iprec]


@pytest.mark.gpu
def test_halfspace_particles_traction_free_surface(gpu):
    """The total field of particles below the surface carries no traction
    on z = 0 (lam tr(e) n + 2 mu e n with n = e_z), relative to the
    free-space traction there."""
    src, _, sl, dl, dv = _halfspace_cloud(400, 1, 3)
    g = np.linspace(-1.5, 1.5, 9)
    surf = np.array([[x, y, 0.0] for x in g for y in g])
    ier, _, _, _, et = gpu.elfmm3dparttarg(3, 1.3, 0.7, src, sl, dl, dv, surf, ifptfrc=0, ifstrain=0,
                                           halfspace=True)
    assert ier == 0
    _, _, _, _, ef = gpu.elfmm3dparttarg(3, 1.3, 0.7, src, sl, dl, dv, surf, ifptfrc=0, ifstrain=0)
    tr = lambda E_: 1.3 * np.trace(E_, axis1=1, axis2=2)[:, None] * np.array([0, 0, 1.0]) + 2 * 0.7 * E_[:, :, 2]
    assert np.abs(tr(et)).max() < 1e-7 * np.abs(tr(ef)).max()


@pytest.mark.gpu
def test_halfspace_particles_reject_points_above_the_surface(gpu):
    src, tgt, sl, dl, dv = _halfspace_cloud(20, 3, 1)
    src[0, 2] = 0.5
    ier, *_ = gpu.elfmm3dparttarg(2, 1.0, 1.0, src, sl, None, None, tgt, halfspace=True)
    assert ier == 16
