"""Generate assemble_gen.cuh: straight-line code for the local-frame single
and double layer assembly of the analytic near field from the R/B tables.

The index arithmetic of the assembly is resolved here once and emitted as
plain statements.  Run: python gen_assemble.py > assemble_gen.cuh
"""


def jidx(a, b, c):
    n = a + b + c
    off = n * (n + 1) * (n + 2) // 6
    pos = 0
    for ap in range(n, a, -1):
        pos += n - ap + 1
    pos += (n - a) - b
    return off + pos


def multi(N):
    return [(a, b, c) for n in range(N + 1) for a in range(n, -1, -1) for b in range(n - a, -1, -1)
            for c in [n - a - b]]


def fact(n):
    r = 1
    for k in range(2, n + 1):
        r *= k
    return r


def e(*ax):
    c = [0, 0, 0]
    for a in ax:
        c[a] += 1
    return jidx(*c)


def emit_assemble():
    L = []
    L.append("// Local-frame single/double layer displacement and symmetric")
    L.append("// strain from the R/B tables; pair_eval (tri_integrals.cuh) rotates and scales.")
    L.append("EFMM_HD void assemble_gen(const double* __restrict__ R, const double* __restrict__ B,")
    L.append("    double rlam, double rmu, double c1, const double* ssl, const double* sdl,")
    L.append("    bool dosl, bool dodl, bool dostrain, double* __restrict__ ul, double* __restrict__ el) {")
    L.append("  for (int i = 0; i < 3; i++) ul[i] = 0.0;")
    L.append("  for (int i = 0; i < 6; i++) el[i] = 0.0;")
    sym = {(0, 0): 0, (1, 1): 1, (2, 2): 2, (0, 1): 3, (1, 0): 3, (0, 2): 4, (2, 0): 4, (1, 2): 5, (2, 1): 5}
    # single layer
    L.append("  if (dosl) {")
    L.append("    const double s0 = ssl[0], s1 = ssl[1], s2 = ssl[2];")
    for i in range(3):
        terms = []
        for k in range(3):
            t = f"-c1 * B[{e(i, k)}]"
            if i == k:
                t += f" + 2.0 * R[0]"
            terms.append(f"s{k} * ({t})")
        L.append(f"    ul[{i}] += " + " + ".join(terms) + ";")
    L.append("    if (dostrain) {")
    for q, (i, j) in enumerate([(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]):
        terms = []
        for k in range(3):
            # 0.5*(m_ij + m_ji), m_ij = -c1 B(i+j+k) + 2 d_ik R(j)
            t = f"-c1 * B[{e(i, j, k)}]"
            extra = []
            if i == k:
                extra.append(f"R[{e(j)}]")
            if j == k:
                extra.append(f"R[{e(i)}]")
            if extra:
                t += " + (" + " + ".join(extra) + ")"
            terms.append(f"s{k} * ({t})")
        L.append(f"      el[{q}] += " + " + ".join(terms) + ";")
    L.append("    }")
    L.append("  }")
    # double layer: U(i,k,m) = -c1 B(i+k+m) + 2 d_ik R(m)
    def U(i, k, m):
        t = f"(-c1 * B[{e(i, k, m)}]"
        if i == k:
            t += f" + 2.0 * R[{e(m)}]"
        return t + ")"

    def D(i, k, j, m):
        t = f"(-c1 * B[{e(i, k, j, m)}]"
        if i == k:
            t += f" + 2.0 * R[{e(j, m)}]"
        return t + ")"
    L.append("  if (dodl) {")
    L.append("    const double s0 = sdl[0], s1 = sdl[1], s2 = sdl[2];")
    for a in range(3):
        terms = []
        for k in range(3):
            t = f"rmu * ({U(k, a, 2)} + {U(2, a, k)})"
            if k == 2:
                t += f" + rlam * ({U(0, a, 0)} + {U(1, a, 1)} + {U(2, a, 2)})"
            terms.append(f"s{k} * ({t})")
        L.append(f"    ul[{a}] += " + " + ".join(terms) + ";")
    L.append("    if (dostrain) {")
    for q, (a, b) in enumerate([(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]):
        terms = []
        for k in range(3):
            def S(a_, b_):
                t = f"rmu * ({D(k, a_, 2, b_)} + {D(2, a_, k, b_)})"
                if k == 2:
                    t += f" + rlam * ({D(0, a_, 0, b_)} + {D(1, a_, 1, b_)} + {D(2, a_, 2, b_)})"
                return t
            if a == b:
                terms.append(f"s{k} * ({S(a, b)})")
            else:
                terms.append(f"s{k} * 0.5 * ({S(a, b)} + {S(b, a)})")
        L.append(f"      el[{q}] += " + " + ".join(terms) + ";")
    L.append("    }")
    L.append("  }")
    L.append("}")
    return "\n".join(L)


if __name__ == "__main__":
    print("// assemble_gen.cuh -- GENERATED by gen_assemble.py; do not edit by hand.")
    print("#pragma once")
    print("// included from tri_integrals.cuh (needs EFMM_HD)")
    print("namespace efmm {")
    print(emit_assemble())
    print("}  // namespace efmm")
