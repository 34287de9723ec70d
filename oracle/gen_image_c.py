"""Generate image_gen.h (TEST INFRASTRUCTURE ONLY): the oracle's image part
of Mindlin's half-space Green's functions as plain C, printed from the
symbolic expressions of oracle/mindlin.py (image_force, _dl, _disp_strain;
src/el3greenh.f:643-787, src/mindlinpieces.f) with common subexpressions
shared.  image.c sums these kernels over refined triangle quadrature; the
numpy lambdification of the same expressions (mindlin.kernels) is the check
of the generated file (tests/test_oracle_image_c.py).

    python oracle/gen_image_c.py   (writes oracle/image_gen.h; about a minute)
"""
import os

import sympy as sp
from sympy.printing.c import C99CodePrinter

import mindlin as M  # this directory is on sys.path when run as a script


def main():
    G = [M.image_force(k) for k in range(3)]
    sl = sum((M._disp_strain(G[k]) for k in range(3)), [])
    dl = sum((M._disp_strain(M._dl(G, p)) for p in range(3)), [])
    pr = C99CodePrinter()
    names = {M._lam: 'lam', M._mu: 'mu', M._x: 'x', M._y: 'y', M._z: 'z', M._s1: 's1', M._s2: 's2',
             M._s3: 's3', M._n[0]: 'n1', M._n[1]: 'n2', M._n[2]: 'n3'}
    assert all(str(k) == v for k, v in names.items())
    out = ['/* image_gen.h -- generated by gen_image_c.py from oracle/mindlin.py; do not edit.',
           ' * TEST INFRASTRUCTURE ONLY (the oracle).  Image part of the half-space',
           ' * Green\'s functions (no 1/(4 pi)) at target (x, y, z) of the three unit',
           ' * point forces (oracle_image_sl) or unit displacement jumps with normal n',
           ' * (oracle_image_dl) at source (s1, s2, s3): 27 doubles, per direction',
           ' * displacement (3) then strain (xx yy zz xy xz yz). */',
           '#include <math.h>', '']
    for name, exprs, extra in (('oracle_image_sl', sl, ''),
                               ('oracle_image_dl', dl, ', double n1, double n2, double n3')):
        rep, red = sp.cse(exprs, symbols=sp.numbered_symbols('t'), optimizations='basic')
        out.append(f'static void {name}(double lam, double mu, double x, double y, double z, double s1, '
                   f'double s2, double s3{extra}, double* o) {{')
        for sym, ex in rep:
            out.append(f'  const double {sym} = {pr.doprint(ex)};')
        for i, ex in enumerate(red):
            out.append(f'  o[{i}] = {pr.doprint(ex)};')
        out.append('}')
        out.append('')
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'image_gen.h')
    with open(path, 'w') as fh:
        fh.write('\n'.join(out))
    print(path, sum(len(line) + 1 for line in out))


if __name__ == '__main__':
    main()
