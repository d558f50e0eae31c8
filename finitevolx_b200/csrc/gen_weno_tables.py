"""Generate weno_tables.cuh: WENO7/WENO9 finite-volume tables.

The tables (candidate reconstruction weights, optimal linear weights and
Jiang-Shu smoothness quadratic forms) are derived here from their
definition with exact rational arithmetic:

* candidate k of an r-cell scheme is the polynomial whose averages over its
  r cells equal the data, evaluated at the east face x = +1/2 of the target
  cell [-1/2, 1/2];
* the optimal weights make the candidates' blend equal the (2r-1)-cell
  reconstruction;
* beta_k = sum_l int_{-1/2}^{1/2} (d^l p_k/dx^l)^2 dx, l = 1..r-1.

finitevolX uses the same published scheme (advection/weno.py:7-253); the
right-biased tables are the mirror images (advection/weno.py:525-535).
Run: ``python gen_weno_tables.py > weno_tables.cuh``.
"""

import math
from fractions import Fraction


def _inverse(r, k):
    shift = r - 1 - k
    A = []
    for j in range(r):
        o = j - shift
        hi, lo = Fraction(2 * o + 1, 2), Fraction(2 * o - 1, 2)
        A.append([(hi ** (a + 1) - lo ** (a + 1)) / (a + 1) for a in range(r)])
    M = [A[i][:] + [Fraction(int(i == j)) for j in range(r)] for i in range(r)]
    for c in range(r):
        p = next(i for i in range(c, r) if M[i][c] != 0)
        M[c], M[p] = M[p], M[c]
        pv = M[c][c]
        M[c] = [x / pv for x in M[c]]
        for i in range(r):
            if i != c and M[i][c] != 0:
                f = M[i][c]
                M[i] = [x - f * y for x, y in zip(M[i], M[c])]
    return [row[r:] for row in M]


def face_coeffs(r, k):
    Ai = _inverse(r, k)
    return [sum(Ai[a][j] * Fraction(1, 2) ** a for a in range(r)) for j in range(r)]


def linear_weights(r):
    big = face_coeffs(2 * r - 1, r - 1)
    small = [face_coeffs(r, k) for k in range(r)]
    d = []
    for p in range(r):
        acc = sum(d[k] * small[k][p - k] for k in range(p))
        d.append((big[p] - acc) / small[p][0])
    return d


def beta_matrix(r, k):
    Ai = _inverse(r, k)
    B = [[Fraction(0)] * r for _ in range(r)]
    for l in range(1, r):
        for a in range(l, r):
            fa = Fraction(math.factorial(a), math.factorial(a - l))
            for b in range(l, r):
                fb = Fraction(math.factorial(b), math.factorial(b - l))
                e = (a - l) + (b - l)
                integ = (Fraction(1, 2) ** (e + 1) - Fraction(-1, 2) ** (e + 1)) / (e + 1)
                for i in range(r):
                    for j in range(r):
                        B[i][j] += fa * fb * integ * Ai[a][i] * Ai[b][j]
    return B


def lit(x):
    x = Fraction(x)
    return f"({x.numerator}.0/{x.denominator}.0)"


def emit(r, name, ctype="double", suffix=""):
    out = []
    C = [face_coeffs(r, k) for k in range(r)]
    W = linear_weights(r)
    Bs = [beta_matrix(r, k) for k in range(r)]
    out.append(f"// {2 * r - 1}-point WENO: {r} candidates of {r} cells (left-biased).")
    out.append(f"__device__ __constant__ {ctype} k{name}_C{suffix}[{r}][{r}] = {{")
    for row in C:
        out.append("  {" + ", ".join(lit(x) for x in row) + "},")
    out.append("};")
    out.append(f"__device__ __constant__ {ctype} k{name}_W{suffix}[{r}] = {{" + ", ".join(lit(x) for x in W) + "};")
    out.append(f"__device__ __constant__ {ctype} k{name}_B{suffix}[{r}][{r}][{r}] = {{")
    for B in Bs:
        out.append("  {")
        for row in B:
            out.append("    {" + ", ".join(lit(x) for x in row) + "},")
        out.append("  },")
    out.append("};")
    return "\n".join(out)


if __name__ == "__main__":
    print("// Generated by gen_weno_tables.py -- do not edit.")
    print("#pragma once")
    for ctype, sfx in (("double", ""), ("float", "f")):
        print(emit(4, "W7", ctype, sfx))
        print(emit(5, "W9", ctype, sfx))
