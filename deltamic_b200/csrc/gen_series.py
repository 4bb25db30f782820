"""Generate the centroid-series coefficients of series_coeffs.cuh.

For a triangle with vertex phases x_v, centroid x_g and deviations
d_v = x_v - x_g (sum d_v = 0), the triangle term is F = e^{-i x_g} H with

    H = sum_n (-i)^n h_n(d_a, d_b, d_c) / (n+2)!

(h_n the complete homogeneous symmetric polynomials: F is minus the second
divided difference of exp(-i x)).  With p2 = sum d^2, p3 = sum d^3 and e1 = 0 the
Newton identities give h_n = (p2/2) h_{n-2} + (p3/3) h_{n-3}, h_0 = 1, h_1 = 0.
Grouping by powers of p3:  Re H = P0(p2) + p3^2 P2(p2) + p3^4 P4(p2),
Im H = p3 Q1(p2) + p3^3 Q3(p2).  Terms up to n = NMAX are formed, then every
monomial whose largest value over the series domain (largest phase difference
D <= DMAX, so p2 <= 2 D^2/3 and |p3| <= 2 D^3/9) is below DROP is dropped.

Two sets are written: DM_SERIES_* for the whole series domain (D <= 3.5) and
DM_SERIES_LO_* for D <= 1.5, where fewer terms reach the same truncation error
(the kernels pick the short set when every lane of a warp qualifies).  A part
with no term left has length 0.

    python deltamic_b200/csrc/gen_series.py > deltamic_b200/csrc/series_coeffs.cuh
"""
from fractions import Fraction
from math import factorial

NMAX = 14
DMAX = 3.5
DROP = 1e-9


def h_polys(nmax):
    # polynomial = dict {(j, k): coeff} for p2^j p3^k
    h = [{(0, 0): Fraction(1)}, {}]
    for n in range(2, nmax + 1):
        out = {}
        for (j, k), c in h[n - 2].items():
            out[(j + 1, k)] = out.get((j + 1, k), 0) + c / 2
        if n >= 3:
            for (j, k), c in h[n - 3].items():
                out[(j, k + 1)] = out.get((j, k + 1), 0) + c / 3
        h.append(out)
    return h


def series(nmax=NMAX):
    h = h_polys(nmax)
    re, im = {}, {}
    for n in range(nmax + 1):
        # (-i)^n = 1, -i, -1, i
        sgn = [1, -1, -1, 1][n % 4]
        tgt = re if n % 2 == 0 else im
        for (j, k), c in h[n].items():
            tgt[(j, k)] = tgt.get((j, k), 0) + sgn * c / factorial(n + 2)
    return re, im


def poly(d, k, dmax=None):
    """Coefficients (ascending in p2) of the p3^k part, truncated by DROP."""
    dmax = DMAX if dmax is None else dmax
    p2max, p3max = 2 * dmax ** 2 / 3, 2 * dmax ** 3 / 9
    js = [j for (j, kk), c in d.items()
          if kk == k and abs(float(c)) * p2max ** j * p3max ** k >= DROP]
    if not js:
        return []
    return [d.get((j, k), Fraction(0)) for j in range(max(js) + 1)]


DMAX_LO = 1.5


def main():
    re, im = series()
    print("// Generated by gen_series.py (do not edit): centroid-series coefficients,")
    print(f"// terms n <= {NMAX}, monomials below {DROP:g} dropped: DM_SERIES_* for")
    print(f"// D <= {DMAX}, DM_SERIES_LO_* for D <= {DMAX_LO}.  Ascending powers of p2.")
    print("#pragma once")
    for tag, dmax in (("", DMAX), ("LO_", DMAX_LO)):
        for name, d, k in (("P0", re, 0), ("P2", re, 2), ("P4", re, 4), ("Q1", im, 1),
                           ("Q3", im, 3)):
            c = poly(d, k, dmax)
            vals = ", ".join(f"{float(x):.9e}f" for x in (c or [Fraction(0)]))
            print(f"#define DM_SERIES_{tag}{name}_N {len(c)}")
            print(f"#define DM_SERIES_{tag}{name} {{{vals}}}")


if __name__ == "__main__":
    main()
