"""Generate edge_gen.cuh: accumulation of one triangle edge's contribution to
the near-field derivative tables, from the edge-frame derivatives of the line
integrals L1 = int 1/r dl (orders 0..2) and Lr = int r dl (orders 1..3).

Edge frame: u along the edge (unit tangent t), v along the outward in-plane
normal m = (t_y, -t_x), h along the triangle normal.  Triangle-frame target
derivatives are d_x = t_x d_u + m_x d_v, d_y = t_y d_u + m_y d_v, d_h = d_h.
The divergence theorem gives, for |a| >= 1 with an in-plane index d,
    X(a) = sum_edges m_d (-1)^(|a|-1) D^(a - e_d) L_edge.
Run: python gen_edge.py > edge_gen.cuh
"""
import re

import sympy as sp


def cc(e):
    """C code without pow() for small integer powers."""
    s = sp.ccode(e)
    s = re.sub(r"pow\((\w+), 2\)", r"(\1*\1)", s)
    s = re.sub(r"pow\((\w+), 3\)", r"(\1*\1*\1)", s)
    s = re.sub(r"pow\((\w+), 4\)", r"((\1*\1)*(\1*\1))", s)
    assert "pow" not in s, s
    return s


def jidx(a, b, c):
    n = a + b + c
    off = n * (n + 1) * (n + 2) // 6
    pos = 0
    for ap in range(n, a, -1):
        pos += n - ap + 1
    pos += (n - a) - b
    return off + pos


def multi(N, lo=0):
    return [(a, b, c) for n in range(lo, N + 1) for a in range(n, -1, -1) for b in range(n - a, -1, -1)
            for c in [n - a - b]]


tx, ty = sp.symbols("tx ty")
mx, my = ty, -tx
Du, Dv, Dh = sp.symbols("Du Dv Dh")
EL1 = {t: sp.Symbol(f"L1[{jidx(*t)}]") for t in multi(2)}
ELr = {t: sp.Symbol(f"Lr[{jidx(*t)}]") for t in multi(3)}


def D(beta, E):
    bx, by, bh = beta
    poly = sp.expand((tx * Du + mx * Dv) ** bx * (ty * Du + my * Dv) ** by * Dh ** bh)
    out = 0
    for term in sp.Add.make_args(poly):
        c, mon = term.as_coeff_Mul()
        pw = sp.Poly(mon, Du, Dv, Dh).monoms()[0] if mon != 1 else (0, 0, 0)
        coef = sp.Poly(term, Du, Dv, Dh).coeffs()[0]
        out += coef * E[tuple(pw)]
    return sp.expand(out)


def main():
    lines = []
    exprs = []
    targets = []
    for (ix, iy, iz) in multi(4, 1):
        if ix + iy == 0:
            continue
        n = ix + iy + iz
        sgn = 1 if n % 2 == 1 else -1
        if ix >= 1:
            d, m = (ix - 1, iy, iz), mx
        else:
            d, m = (ix, iy - 1, iz), my
        if n >= 2:
            exprs.append(sgn * m * D(d, ELr))
            targets.append(f"B[{jidx(ix, iy, iz)}] +=")
        if n <= 2:
            exprs.append(sgn * m * D(d, EL1))
            targets.append(f"R[{jidx(ix, iy, iz)}] +=")
    exprs.append(mx * D((1, 0, 1), EL1) + my * D((0, 1, 1), EL1))
    targets.append("sh +=")
    rep, red = sp.cse(exprs, symbols=sp.numbered_symbols("q"))
    print("// edge_gen.cuh -- GENERATED by gen_edge.py; do not edit by hand.")
    print("#pragma once")
    print("// included from tri_integrals.cuh (needs EFMM_HD)")
    print("namespace efmm {")
    print("// Add one edge's contribution to the in-plane table entries R (|a| = 1, 2),")
    print("// B (|a| = 2..4) and to sh = d_h (d_xx + d_yy) int 1/r.  L1: edge-frame")
    print("// derivatives of int 1/r dl (|b| <= 2), Lr: of int r dl (1 <= |b| <= 3),")
    print("// both indexed by jidx(u, v, h); (tx, ty): unit edge tangent.")
    print("EFMM_HD void edge_tables_gen(double tx, double ty, const double* __restrict__ L1,")
    print("                             const double* __restrict__ Lr, double* __restrict__ R,")
    print("                             double* __restrict__ B, double& sh) {")
    for s, e in rep:
        print(f"  const double {s} = {cc(e)};")
    for t, e in zip(targets, red):
        print(f"  {t} {cc(e)};")
    print("}")
    print("}  // namespace efmm")


if __name__ == "__main__":
    main()
