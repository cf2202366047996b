"""Generate ``bicubic_gen.cuh``: the bicubic coefficient map as explicit sums.

A bicubic patch p(t, u) = sum_{n,m<4} c[n*4+m] t^n u^m on the unit cell is fixed
by 16 values at the four corners (counter-clockwise from (0,0)): p, dp/dt,
dp/du and d2p/dtdu, stored x[type*4 + corner].  The constraint matrix M (rows:
those 16 functionals applied to each monomial) is inverted exactly with
rational arithmetic; W = M^-1 is integer.  The coarse-to-fine transfer of the
reference forms c = W x with a dense 16-term loop per coefficient
(``bcucof_opt.c:55-61``, ``xx += wt[i][k]*x[k]`` for k = 0..15).  Adding a zero
product leaves a non-zero partial sum unchanged, so the emitted code keeps only
the non-zero terms, in ascending k, left-associated — the same rounding
sequence without the 60% of multiply-adds that are zero.  Weights of +-1 become
an addition or subtraction (1 x and -1 x are exact), and power-of-two weights
(+-2, +-4) a fused multiply-add: their product is exact, so rounding once after
the add is what rounding the product and then the sum gives.

Run: ``python gen_bicubic.py`` (writes next to this file).
"""
from fractions import Fraction
from pathlib import Path

CORNERS = [(0, 0), (1, 0), (1, 1), (0, 1)]


def constraint_matrix():
    rows = []
    for typ in range(4):              # value, d/dt, d/du, d2/dtdu
        dn, dm = typ in (1, 3), typ in (2, 3)
        for (t, u) in CORNERS:
            row = []
            for n in range(4):
                for m in range(4):
                    if n < dn or m < dm:
                        row.append(Fraction(0))
                        continue
                    v = Fraction(1)
                    if dn:
                        v *= n
                    if dm:
                        v *= m
                    v *= Fraction(t) ** (n - dn) * Fraction(u) ** (m - dm)
                    row.append(v)
            rows.append(row)
    return rows


def invert(M):
    n = len(M)
    A = [row[:] + [Fraction(int(i == j)) for j in range(n)] for i, row in enumerate(M)]
    for col in range(n):
        piv = next(r for r in range(col, n) if A[r][col] != 0)
        A[col], A[piv] = A[piv], A[col]
        d = A[col][col]
        A[col] = [x / d for x in A[col]]
        for r in range(n):
            if r != col and A[r][col] != 0:
                f = A[r][col]
                A[r] = [a - f * b for a, b in zip(A[r], A[col])]
    return [row[n:] for row in A]


def weights():
    W = invert(constraint_matrix())
    out = []
    for row in W:
        assert all(x.denominator == 1 for x in row)
        out.append([int(x) for x in row])
    return out


def emit(path: Path):
    W = weights()
    lines = [
        "// GENERATED by gen_bicubic.py — bicubic coefficients c[n*4+m] of t^n u^m",
        "// from x[type*4+corner] (type: value, d/dt, d/du, d2/dtdu; corners",
        "// counter-clockwise from (0,0)).  Non-zero terms only, ascending k,",
        "// left-associated (the rounding sequence of a dense k = 0..15 loop).",
        "// A weight of +-1 is an exact sign; a weight that is a power of two",
        "// makes the product exact, so fma(w, x, s) rounds as s + w x does.",
        "#pragma once",
        "#define DNS_BICUBIC_COEFFS(c, x) \\",
    ]
    def body(suffix):
        out = []
        for r, row in enumerate(W):
            nz = [(k, w) for k, w in enumerate(row) if w != 0]
            k0, w0 = nz[0]
            expr = f"(x)[{k0}]" if w0 == 1 else (f"(-(x)[{k0}])" if w0 == -1 else f"({float(w0)!r}{suffix} * (x)[{k0}])")
            for k, w in nz[1:]:
                if w == 1:
                    expr = f"({expr} + (x)[{k}])"
                elif w == -1:
                    expr = f"({expr} - (x)[{k}])"
                elif abs(w) & (abs(w) - 1) == 0:   # +-2, +-4, ...: the product is exact
                    expr = f"fma({float(w)!r}{suffix}, (x)[{k}], {expr})"
                else:
                    expr = f"({expr} + ({float(w)!r}{suffix} * (x)[{k}]))"
            out.append(f"  (c)[{r}] = {expr};")
        return out
    lines.append(" \\\n".join(body("")))
    lines.append("")
    path.write_text("\n".join(lines))


if __name__ == "__main__":
    emit(Path(__file__).resolve().parent / "bicubic_gen.cuh")
