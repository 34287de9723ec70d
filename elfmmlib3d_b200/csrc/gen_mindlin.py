"""Generate mindlin_gen.cuh: the image part of Mindlin's half-space Green's
functions for a point force (single layer) and a point displacement jump
(double layer), with their strains.

The image of a point force f at xi (xi_3 < 0) at target x (x_3 < 0) is the
sum of three pieces (src/el3greenh.f:643-787, src/mindlinpieces.f):
  A  the "anti-image": the Kelvin solution with lambda' = lambda + 4 mu,
     mu' = -mu at the reflected target (x_1, x_2, -x_3), sign flipped
     (src/el3greenh.f:683-713, src/el3green.f:749);
  B  (1 - alpha)/alpha sum_j s_j f_j d_i d_j U / mu with
     U = R_3 log(R + R_3) - R, R = (x_1 - xi_1, x_2 - xi_2, -x_3 - xi_3),
     s = (-1, -1, 1) (src/mindlinpieces.f:29-250);
  C  x_3 P_i / mu with P built from V = 1/R and its first and second
     derivatives (src/mindlinpieces.f:368-520),
alpha = (lambda + mu)/(lambda + 2 mu).  The double layer (jump b, normal n)
is the elastic contraction  sum C_pqkl b_p n_q d/dxi_l G_ki  of the source
derivatives of the point-force kernel (the convention of the free-space
double layer of this library).  Outputs carry no 1/(4 pi), like the rest of
the library.  Strain = symmetrised target gradient; order xx yy zz xy xz yz.

    python gen_mindlin.py   (writes mindlin_gen.cuh next to this file)
"""
import os

import sympy as sp
from sympy.printing.c import C99CodePrinter

x, y, z, s1, s2, s3 = sp.symbols('x y z s1 s2 s3', real=True)
lam, mu = sp.symbols('lam mu', positive=True)
n1, n2, n3 = sp.symbols('n1 n2 n3', real=True)
X, S, NN = [x, y, z], [s1, s2, s3], [n1, n2, n3]
al = (lam + mu) / (lam + 2 * mu)


def kelvin(cA, cB, d, k):
    r = sp.sqrt(d[0] ** 2 + d[1] ** 2 + d[2] ** 2)
    return [(cA * (1 if i == k else 0) / r + cB * d[k] * d[i] / r ** 3) / (2 * mu) for i in range(3)]


def image_force(k):
    """Image displacement (3 components) of a unit force along axis k."""
    uA = kelvin(al, 2 - al, [x - s1, y - s2, -z - s3], k)
    r1, r2, r3 = sp.symbols('r1 r2 r3', real=True)
    rs = [r1, r2, r3]
    sub = {r1: x - s1, r2: y - s2, r3: -z - s3}
    rr = sp.sqrt(r1 ** 2 + r2 ** 2 + r3 ** 2)
    U = r3 * sp.log(rr + r3) - rr
    f = [1 if j == k else 0 for j in range(3)]
    sg = [-1, -1, 1]
    scale = (1 - al) / al
    uB = [scale * sum(sg[j] * f[j] * sp.diff(U, rs[i], rs[j]) for j in range(3)).subs(sub) / mu for i in range(3)]
    V = 1 / rr
    v = [sp.diff(V, q) for q in rs]
    vv = [[sp.diff(V, a, c) for c in rs] for a in rs]
    h = -s3  # height of the image source
    P = [-(2 - al) * f[2] * v[0] + h * al * (f[0] * vv[0][0] + f[1] * vv[0][1] + f[2] * vv[0][2]),
         -(2 - al) * f[2] * v[1] + h * al * (f[0] * vv[0][1] + f[1] * vv[1][1] + f[2] * vv[1][2]),
         -(2 - al) * (f[0] * v[0] + f[1] * v[1]) - h * al * (f[0] * vv[0][2] + f[1] * vv[1][2] + f[2] * vv[2][2])]
    uC = [z * Pi.subs(sub) / mu for Pi in P]
    return [uA[i] + uB[i] + uC[i] for i in range(3)]


def cijkl(p, q, k, l):
    d = lambda a, c: 1 if a == c else 0
    return lam * d(p, q) * d(k, l) + mu * (d(p, k) * d(q, l) + d(p, l) * d(q, k))


def disp_strain(u):
    g = [[sp.diff(u[i], X[j]) for j in range(3)] for i in range(3)]
    e = [g[0][0], g[1][1], g[2][2], (g[0][1] + g[1][0]) / 2, (g[0][2] + g[2][0]) / 2, (g[1][2] + g[2][1]) / 2]
    return list(u) + e


class _Printer(C99CodePrinter):
    """Integer and half-integer powers as products, sqrt and one division
    (no general pow in device code)."""

    def _print_Pow(self, expr):
        b, e = expr.base, expr.exp
        if e.is_Integer or (e.is_Rational and e.q == 2):
            num = abs(int(e.p))
            base = self._print(b)
            if e.is_Integer:
                fac = [f'({base})'] * num
            else:
                fac = [f'sqrt({base})'] * num
            prod = '*'.join(fac) if fac else '1.0'
            return f'({prod})' if e > 0 else f'(1.0/({prod}))'
        return super()._print_Pow(expr)


_pr = _Printer()


def main():
    G = [image_force(k) for k in range(3)]  # G[k][i]
    f = sp.symbols('f1 f2 f3', real=True)
    b = sp.symbols('b1 b2 b3', real=True)
    sl = disp_strain([sum(f[k] * G[k][i] for k in range(3)) for i in range(3)])
    dl = disp_strain([sum(cijkl(p, q, k, l) * b[p] * NN[q] * sp.diff(G[k][i], S[l])
                          for p in range(3) for q in range(3) for k in range(3) for l in range(3)
                          if cijkl(p, q, k, l) != 0) for i in range(3)])
    # unit-density blocks (27 doubles: per direction k of the force or jump,
    # displacement then strain): the stored near-field form
    sl_blk = sum((disp_strain(G[k]) for k in range(3)), [])
    dl_blk = sum((disp_strain([sum(cijkl(p, q, k, l) * NN[q] * sp.diff(G[k][i], S[l])
                                   for q in range(3) for k in range(3) for l in range(3)
                                   if cijkl(p, q, k, l) != 0) for i in range(3)]) for p in range(3)), [])
    out = ['// mindlin_gen.cuh -- generated by gen_mindlin.py; do not edit.',
           '// Image part of the half-space Green\'s functions of a point force f',
           '// (single layer) and of a point displacement jump b with normal n',
           '// (double layer) at source s, seen at target (x, y, z): 9 doubles,',
           '// displacement (3) then strain (xx yy zz xy xz yz).  The _blk forms',
           '// return the responses to the three unit forces / unit jumps, 27 doubles',
           '// (direction-major, 9 each).',
           '#pragma once', '#include "tri_index.cuh"', '', 'namespace efmm {', '']
    for name, exprs, extra in (('mindlin_image_sl', sl, ', double f1, double f2, double f3'),
                               ('mindlin_image_dl', dl, ', double b1, double b2, double b3, double n1, double n2, '
                                                        'double n3'),
                               ('mindlin_image_sl_blk', sl_blk, ''),
                               ('mindlin_image_dl_blk', dl_blk, ', double n1, double n2, double n3')):
        rep, red = sp.cse(exprs, symbols=sp.numbered_symbols('t'), optimizations='basic')
        out.append(f'EFMM_HD void {name}(double lam, double mu, double x, double y, double z, double s1, '
                   f'double s2, double s3{extra}, double* o) {{')
        for sym, ex in rep:
            out.append(f'  const double {sym} = {_pr.doprint(ex)};')
        for i, ex in enumerate(red):
            out.append(f'  o[{i}] = {_pr.doprint(ex)};')
        out.append('}')
        out.append('')
    out.append('}  // namespace efmm')
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'mindlin_gen.cuh')
    with open(path, 'w') as fh:
        fh.write('\n'.join(out) + '\n')
    print(path, sum(len(l) for l in out))


if __name__ == '__main__':
    main()
