"""Generates phi_series.h: the power series in m^2 (m = pi s) of the
reference's closed-form basis transforms (meshless_vis/fourier_transform.cu:
31-60), for the h-binned tensor form, which needs Phi^ without its branch.

Below its branch point (s = 0.06 SPH, 0.24 Wendland) the reference replaces
the closed form by a quadratic fit whose slope differs from the closed form's
at the branch point.  The h-binned form interpolates the closed form C(s) on
all s (smooth: the transform of a compact kernel is entire) and sums the small
difference Q(s) - C(s) below the branch point separately.  C(s) is evaluated
from this series below the branch point, where the closed form cancels in
FP64 (its numerator is O(m^8) for Wendland, O(m^6) for SPH), and from the
closed form above.

The coefficients are exact rationals, printed as doubles:
  Wendland: N(m) = 4 m^2 - 6 + (6 - m^2) cos 2m + 4.5 m sin 2m = sum_{n>=4} a_n m^(2n),
            C = (7.5 pi) sum_n a_n m^(2n-8);
  SPH:      (cos 2m - 1)(cos 2m + m sin 2m - 1) = sum_{n>=3} b_n m^(2n),
            C = (3 pi / 4) sum_n b_n m^(2n-6).
Terms: 24 each; at the branch point (m <= 0.76) the last term is below 1e-40.
Run:  python gen_phi_series.py > phi_series.h
"""
from fractions import Fraction as Fr
from math import factorial

TERMS = 24


def cos2m(k):  # coefficient of m^(2k) in cos 2m
    return Fr((-1) ** k * 4 ** k, factorial(2 * k))


def sin2m(k):  # coefficient of m^(2k+1) in sin 2m
    return Fr((-1) ** k * 2 ** (2 * k + 1), factorial(2 * k + 1))


def wendland():
    n = TERMS + 4
    a = [Fr(0)] * (n + 2)
    a[0] += -6
    a[1] += 4
    for k in range(n + 1):
        a[k] += 6 * cos2m(k)
        a[k + 1] += -cos2m(k)
        a[k + 1] += Fr(9, 2) * sin2m(k)
    assert all(x == 0 for x in a[:4])
    return a[4:4 + TERMS]


def sph():
    n = TERMS + 4
    A = [cos2m(k) for k in range(n)]
    A[0] -= 1
    B = [cos2m(k) for k in range(n)]
    B[0] -= 1
    for k in range(n - 1):
        B[k + 1] += sin2m(k)
    P = [Fr(0)] * n
    for i in range(n):
        for j in range(n - i):
            P[i + j] += A[i] * B[j]
    assert all(x == 0 for x in P[:3])
    return P[3:3 + TERMS]


def main():
    print("/* Generated by gen_phi_series.py; do not edit. */")
    print("#pragma once")
    print(f"#define MV_PHI_SERIES_TERMS {TERMS}")
    for name, coef in (("WENDLAND", wendland()), ("SPH", sph())):
        vals = ", ".join(repr(float(c)) for c in coef)
        print(f"/* coefficient of m^(2n), n = 0 .. {TERMS - 1}, of the closed form's numerator over its m power */")
        print(f"static __device__ const double MV_{name}_SERIES[{TERMS}] = {{{vals}}};")


if __name__ == "__main__":
    main()
