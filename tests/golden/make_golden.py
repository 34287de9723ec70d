"""Generate the golden fixtures under tests/golden/.

  golden_tables.npz   R/B derivative tables of a flat triangle at five targets,
                      integrated by adaptive quadrature (scipy, rel. tol 1e-13) directly from the kernel
                      definitions of the reference (src/triahquad.f:127-200):
                      pins the oracle's integrals to the documented definitions.
  golden_sphere320.npz  oracle direct sum (el3dtriadirecttarg restated) on the
                      level-2 icosphere (320 triangles) + 40 targets, the
                      reference driver's Lame constants (elfmm3dtria_dr.f:131).
  golden_fault100.npz oracle direct sum on a flat 10x5 fault (100 triangles,
                      coplanar neighbours, targets collinear with edges) + 20
                      targets.
  golden_c1_sphere5120.npz  the free-space configuration at its own size:
                      icosphere level 4 (5,120 triangles), 1,000 targets
                      uniform in [-2,2]^3 with |x| > 1.1, lambda = mu = 1,
                      single and double layer N(0,1) (seed 1); the oracle
                      direct sum at 256 sampled centroids and 256 sampled
                      targets (the geometry is regenerated from
                      elfmmlib3d_b200.geometry and checked by its SHA-256).

Run from the repository root:  python tests/golden/make_golden.py [c1]
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from elfmmlib3d_b200 import geometry as G  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

TRI = np.array([[0.1, 0.2, 0.05], [1.2, 0.1, -0.1], [0.4, 1.1, 0.2]])
# targets in the triangle frame (x, y, z)
LOCAL_TARGETS = np.array([[0.3, 0.4, 0.7], [2.0, -1.0, 0.5], [0.5, 0.3, -0.05], [1.5, 0.9, 0.25],
                          [-0.4, 0.2, -0.3]])
R_IDX = [(a, b, c) for a in range(3) for b in range(3) for c in range(3) if a + b + c <= 2]
B_IDX = [(a, b, c) for a in range(5) for b in range(5) for c in range(5) if 2 <= a + b + c <= 4]


def quad_tables(v, x0, y0, z0):
    """Adaptive double quadrature (scipy QUADPACK, relative tolerance 1e-13)
    of the kernel derivatives, differentiated symbolically (sympy) from 1/r
    and r: independent of the oracle's polar/Gauss schemes."""
    import sympy as sp
    from scipy import integrate
    X, Y, Z = sp.symbols("X Y Z")
    r = sp.sqrt(X ** 2 + Y ** 2 + Z ** 2)
    (ax, ay), (bx, by), (cx, cy) = [(float(p[0]), float(p[1])) for p in v]
    area2 = abs((bx - ax) * (cy - ay) - (cx - ax) * (by - ay))
    out = {}
    for kind, base, idx in (("R", 1 / r, R_IDX), ("B", r, B_IDX)):
        for a in idx:
            e = sp.diff(base, X, a[0], Y, a[1], Z, a[2]) if sum(a) else base
            fn = sp.lambdify((X, Y, Z), e, "math")

            def f(t, u):
                s = (1 - u) * t
                px = ax + u * (bx - ax) + s * (cx - ax)
                py = ay + u * (by - ay) + s * (cy - ay)
                # source minus target, source at z = 0
                return fn(px - x0, py - y0, -z0) * (1 - u)
            val, err = integrate.dblquad(f, 0, 1, 0, 1, epsabs=0, epsrel=1e-13)
            out[(kind,) + a] = val * area2
    return out


def c1():
    """Oracle direct sum on the free-space configuration (sphere 5,120 +
    1,000 box targets) at sampled points.  The oracle evaluates a
    contiguous range of centroids, so the triangles are permuted to put the
    sampled ones first (the sum over triangles does not depend on their
    order)."""
    tri, nrm, cen = G.sphere_triangles(4)
    tg = G.box_targets(1000, 2)
    rng = np.random.default_rng(1)
    ssl = rng.normal(size=cen.shape)
    sdl = rng.normal(size=cen.shape)
    pick = np.random.default_rng(11)
    ic = np.sort(pick.choice(len(cen), 256, replace=False))
    it = np.sort(pick.choice(len(tg), 256, replace=False))
    order = np.concatenate([ic, np.setdiff1d(np.arange(len(cen)), ic)])
    pt, st, _, _ = O.direct(1.0, 1.0, tri[order], cen[order], ssl[order], sdl[order], None,
                            rows=(0, len(ic)), trows=(0, 0))
    _, _, ptt, stt = O.direct(1.0, 1.0, tri, cen, ssl, sdl, tg[it], rows=(0, 0))
    np.savez_compressed(os.path.join(OUT, "golden_c1_sphere5120.npz"), rlam=1.0, rmu=1.0, ssl=ssl, sdl=sdl,
                        tgt=tg, idx_c=ic, idx_t=it, u_c=pt[:len(ic)], e_c=st[:len(ic)], u_t=ptt, e_t=stt,
                        tri_sha256=hashlib.sha256(np.ascontiguousarray(tri).tobytes()).hexdigest())
    print("c1", flush=True)


def main():
    rot, v = O.frame(TRI)
    targets = np.array([TRI[0] + rot @ xl for xl in LOCAL_TARGETS])
    R = np.zeros((len(targets), len(R_IDX)))
    B = np.zeros((len(targets), len(B_IDX)))
    for i, xl in enumerate(LOCAL_TARGETS):
        t = quad_tables(v, *xl)
        R[i] = [t[("R",) + a] for a in R_IDX]
        B[i] = [t[("B",) + a] for a in B_IDX]
        print("tables", i, flush=True)
    np.savez(os.path.join(OUT, "golden_tables.npz"), tri=TRI, targets=targets, R=R, B=B,
             r_idx=np.array(R_IDX), b_idx=np.array(B_IDX))

    rlam, rmu = 3.2, 2.3
    rng = np.random.default_rng(20260101)
    tri, nrm, cen = G.sphere_triangles(2)
    tg = G.box_targets(40, 11)
    ssl = rng.normal(size=cen.shape)
    sdl = rng.normal(size=cen.shape)
    pt, st, ptt, stt = O.direct(rlam, rmu, tri, cen, ssl, sdl, tg)
    np.savez(os.path.join(OUT, "golden_sphere320.npz"), rlam=rlam, rmu=rmu, tri=tri, nrm=nrm, cen=cen,
             tgt=tg, ssl=ssl, sdl=sdl, pt=pt, st=st, ptt=ptt, stt=stt)
    print("sphere320", flush=True)

    tri, nrm, cen, us = G.planar_fault(10, 5, length=10.0, width=5.0, dip_deg=30.0, top_depth=1.0)
    tg = np.array(cen[::5] + 0.3 * nrm[::5])
    ssl = rng.normal(size=cen.shape)
    sdl = rng.normal(size=cen.shape)
    pt, st, ptt, stt = O.direct(rlam, rmu, tri, cen, ssl, sdl, tg)
    np.savez(os.path.join(OUT, "golden_fault100.npz"), rlam=rlam, rmu=rmu, tri=tri, nrm=nrm, cen=cen,
             tgt=tg, ssl=ssl, sdl=sdl, pt=pt, st=st, ptt=ptt, stt=stt)
    print("fault100", flush=True)


if __name__ == "__main__":
    if sys.argv[1:] == ["c1"]:
        c1()
    else:
        main()
        c1()
