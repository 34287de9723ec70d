"""Oracle (test infrastructure only): image part of Mindlin's half-space
Green's functions, restated from the reference and evaluated with numpy.

Nothing in the product imports this module.  The reference builds the image
of a point force f at xi (xi_3 < 0) seen at x (x_3 < 0) from three pieces
(src/el3greenh.f:643-787):

  A  the anti-image: the Kelvin solution with lambda' = lambda + 4 mu and
     mu' = -mu at the reflected target (x_1, x_2, -x_3), sign flipped
     (src/el3greenh.f:683-713; Kelvin kernel src/el3green.f:619-748,
     reflected strain src/el3green.f:749-878);
  B  (1 - alpha)/alpha (-f_1 U_i1 - f_2 U_i2 + f_3 U_i3) / mu, U_ij second
     derivatives of U = R_3 log(R + R_3) - R with R = x - (xi_1, xi_2, -xi_3)
     and R_3 = -(x_3 + xi_3) (src/mindlinpieces.f:29-185);
  C  x_3 P_i / mu, P from V = 1/R (src/mindlinpieces.f:368-500):
     P_1 = -(2 - alpha) f_3 V_1 + h alpha (f_1 V_11 + f_2 V_12 + f_3 V_13),
     P_2 = -(2 - alpha) f_3 V_2 + h alpha (f_1 V_12 + f_2 V_22 + f_3 V_23),
     P_3 = -(2 - alpha)(f_1 V_1 + f_2 V_2) - h alpha (f_1 V_13 + f_2 V_23 + f_3 V_33),
     h = -xi_3,

alpha = (lambda + mu)/(lambda + 2 mu), no 1/(4 pi).  The double layer (jump
b on a surface with normal n) is sum C_pqkl b_p n_q d/dxi_l G_ki, which with
the free-space kernel reproduces the analytic double layer of oracle.c.

These expressions are evaluated here through sympy/numpy, independently of
the product's generated CUDA code.  They are pinned by the physics the
reference's image must satisfy (tests/test_mindlin_oracle.py): zero traction
on z = 0 for the total (free + image) field of both layers, reciprocity of
the total Green's function, and consistency of the double layer with the
analytic free-space double layer.  Parity against numbers produced by the
reference itself is unpinned (no Fortran compiler on this image).
"""
import functools

import numpy as np
import sympy as sp

_x, _y, _z, _s1, _s2, _s3 = sp.symbols('x y z s1 s2 s3', real=True)
_lam, _mu = sp.symbols('lam mu', positive=True)
_n = sp.symbols('n1 n2 n3', real=True)
_X, _S = [_x, _y, _z], [_s1, _s2, _s3]


def _kelvin(ca, cb, d, k, mu):
    r = sp.sqrt(d[0] ** 2 + d[1] ** 2 + d[2] ** 2)
    return [(ca * (1 if i == k else 0) / r + cb * d[k] * d[i] / r ** 3) / (2 * mu) for i in range(3)]


def _alpha():
    return (_lam + _mu) / (_lam + 2 * _mu)


def free_force(k):
    """Free-space displacement of a unit force along k (src/el3green.f:619)."""
    al = _alpha()
    return _kelvin(2 - al, al, [_X[i] - _S[i] for i in range(3)], k, _mu)


def image_force(k):
    """Image displacement of a unit force along k (pieces A + B + C)."""
    al = _alpha()
    ua = _kelvin(al, 2 - al, [_x - _s1, _y - _s2, -_z - _s3], k, _mu)
    R = [_x - _s1, _y - _s2, -_z - _s3]
    Rn = sp.sqrt(R[0] ** 2 + R[1] ** 2 + R[2] ** 2)
    # derivatives with respect to R_j; since R is linear in x with
    # dR/dx = diag(1, 1, -1), d/dR_j = sign_j d/dx_j
    sgn = [1, 1, -1]
    U = R[2] * sp.log(Rn + R[2]) - Rn
    dU = lambda i, j: sgn[i] * sgn[j] * sp.diff(U, _X[i], _X[j])
    f = [1 if j == k else 0 for j in range(3)]
    sc = (1 - al) / al
    ub = [sc * (-f[0] * dU(i, 0) - f[1] * dU(i, 1) + f[2] * dU(i, 2)) / _mu for i in range(3)]
    V = 1 / Rn
    V1 = [sgn[i] * sp.diff(V, _X[i]) for i in range(3)]
    V2 = [[sgn[i] * sgn[j] * sp.diff(V, _X[i], _X[j]) for j in range(3)] for i in range(3)]
    h = -_s3
    P = [-(2 - al) * f[2] * V1[0] + h * al * (f[0] * V2[0][0] + f[1] * V2[0][1] + f[2] * V2[0][2]),
         -(2 - al) * f[2] * V1[1] + h * al * (f[0] * V2[0][1] + f[1] * V2[1][1] + f[2] * V2[1][2]),
         -(2 - al) * (f[0] * V1[0] + f[1] * V1[1]) - h * al * (f[0] * V2[0][2] + f[1] * V2[1][2] + f[2] * V2[2][2])]
    uc = [_z * P[i] / _mu for i in range(3)]
    return [ua[i] + ub[i] + uc[i] for i in range(3)]


def _cijkl(p, q, k, l):
    d = lambda a, c: 1 if a == c else 0
    return _lam * d(p, q) * d(k, l) + _mu * (d(p, k) * d(q, l) + d(p, l) * d(q, k))


def _dl(G, p):
    return [sum(_cijkl(p, q, k, l) * _n[q] * sp.diff(G[k][i], _S[l])
                for q in range(3) for k in range(3) for l in range(3) if _cijkl(p, q, k, l) != 0)
            for i in range(3)]


def _disp_strain(u):
    g = [[sp.diff(u[i], _X[j]) for j in range(3)] for i in range(3)]
    return list(u) + [g[0][0], g[1][1], g[2][2], (g[0][1] + g[1][0]) / 2, (g[0][2] + g[2][0]) / 2,
                      (g[1][2] + g[2][1]) / 2]


@functools.lru_cache(maxsize=None)
def kernels(part="image"):
    """numpy kernels (sl, dl): sl(lam, mu, x, y, z, s1, s2, s3) and
    dl(lam, mu, x, y, z, s1, s2, s3, n1, n2, n3) return 27 arrays: per source
    direction (force e_k or jump e_p) displacement (3) then strain (6)."""
    G = [image_force(k) if part == "image" else free_force(k) for k in range(3)]
    sl = sum((_disp_strain(G[k]) for k in range(3)), [])
    dl = sum((_disp_strain(_dl(G, p)) for p in range(3)), [])
    args = (_lam, _mu, _x, _y, _z, _s1, _s2, _s3)
    fsl = sp.lambdify(args, sl, 'numpy')
    fdl = sp.lambdify(args + tuple(_n), dl, 'numpy')
    return fsl, fdl


@functools.lru_cache(maxsize=None)
def traction_on_surface():
    """numpy function of (lam, mu, x, y, s1, s2, s3, b1, b2, b3, n1, n2, n3,
    f1, f2, f3) returning the traction sigma . e_z at (x, y, 0) of the total
    (free + image) field of a force f plus a jump b with normal n."""
    b = sp.symbols('b1 b2 b3', real=True)
    f = sp.symbols('f1 f2 f3', real=True)
    G = [[free_force(k)[i] + image_force(k)[i] for i in range(3)] for k in range(3)]
    u = [sum(f[k] * G[k][i] for k in range(3)) + sum(b[p] * _dl(G, p)[i] for p in range(3)) for i in range(3)]
    eps = [[(sp.diff(u[i], _X[j]) + sp.diff(u[j], _X[i])) / 2 for j in range(3)] for i in range(3)]
    tr = eps[0][0] + eps[1][1] + eps[2][2]
    t = [_lam * tr * (1 if i == 2 else 0) + 2 * _mu * eps[i][2] for i in range(3)]
    t = [ti.subs(_z, 0) for ti in t]
    return sp.lambdify((_lam, _mu, _x, _y, _s1, _s2, _s3) + tuple(b) + tuple(_n) + tuple(f), t, 'numpy')


# 12-node degree-6 symmetric rule on the triangle (barycentric nodes, weights
# summing to 1): the rule of oracle.c / the product's P2M.
def _quad12():
    a1, w1 = 0.2492867451709104212916386, 0.1167862757263793660252896
    a2, w2 = 0.0630890144915022283403316, 0.05084490637020681692093681
    b3, c3, w3 = 0.05314504984481694735324967, 0.3103524510337844054166077, 0.08285107561837357519355346
    B, W = [], []
    for a, w in ((a1, w1), (a2, w2)):
        o = 1 - 2 * a
        B += [[o, a, a], [a, o, a], [a, a, o]]
        W += [w] * 3
    o = 1 - b3 - c3
    for p in ((o, b3, c3), (o, c3, b3), (b3, o, c3), (c3, o, b3), (b3, c3, o), (c3, b3, o)):
        B.append(list(p))
        W.append(w3)
    return np.array(B), np.array(W)


def _subdivide(tri, level):
    """4**level congruent sub-triangles of tri (3, 3)."""
    tris = [np.asarray(tri, float)]
    for _ in range(level):
        nxt = []
        for t in tris:
            a, b, c = t
            ab, bc, ca = (a + b) / 2, (b + c) / 2, (c + a) / 2
            nxt += [np.array([a, ab, ca]), np.array([ab, b, bc]), np.array([ca, bc, c]), np.array([ab, bc, ca])]
        tris = nxt
    return np.array(tris)


def image_direct(rlam, rmu, tri, nrm, ssl, sdl, tgt, level=2, part="image"):
    """Image displacement (m, 3) and strain (m, 3, 3) at targets tgt (m, 3)
    of piecewise-constant layers on triangles tri (n, 3, 3): single layer
    ssl (n, 3) and/or double layer sdl (n, 3) with normals nrm (n, 3)
    (None disables a layer).  Each triangle is split into 4**level
    sub-triangles with the 12-node rule on each.  part="free" integrates the
    free-space kernels instead (targets away from the triangles only)."""
    fsl, fdl = kernels(part)
    B, W = _quad12()
    tgt = np.asarray(tgt, float)
    u = np.zeros((len(tgt), 3))
    e6 = np.zeros((len(tgt), 6))
    for t in range(len(tri)):
        sub = _subdivide(tri[t], level)
        area = 0.5 * np.linalg.norm(np.cross(sub[:, 1] - sub[:, 0], sub[:, 2] - sub[:, 0]), axis=1)
        pts = np.einsum('qv,svd->sqd', B, sub).reshape(-1, 3)
        wts = (area[:, None] * W[None, :]).reshape(-1)
        X = tgt[:, None, :]
        P = pts[None, :, :]
        args = (rlam, rmu, X[..., 0], X[..., 1], X[..., 2], P[..., 0], P[..., 1], P[..., 2])
        if ssl is not None:
            o = fsl(*args)
            for k in range(3):
                for c in range(9):
                    v = np.broadcast_to(o[9 * k + c], (len(tgt), len(pts)))
                    val = (v * wts[None, :]).sum(axis=1) * ssl[t][k]
                    if c < 3:
                        u[:, c] += val
                    else:
                        e6[:, c - 3] += val
        if sdl is not None:
            o = fdl(*args, nrm[t][0], nrm[t][1], nrm[t][2])
            for p in range(3):
                for c in range(9):
                    v = np.broadcast_to(o[9 * p + c], (len(tgt), len(pts)))
                    val = (v * wts[None, :]).sum(axis=1) * sdl[t][p]
                    if c < 3:
                        u[:, c] += val
                    else:
                        e6[:, c - 3] += val
    e = np.zeros((len(tgt), 3, 3))
    e[:, 0, 0], e[:, 1, 1], e[:, 2, 2] = e6[:, 0], e6[:, 1], e6[:, 2]
    e[:, 0, 1] = e[:, 1, 0] = e6[:, 3]
    e[:, 0, 2] = e[:, 2, 0] = e6[:, 4]
    e[:, 1, 2] = e[:, 2, 1] = e6[:, 5]
    return u, e
