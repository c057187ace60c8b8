"""Generates phi_poly.h: polynomial forms of the reference's closed-form basis
transforms on the interval just above each branch point, where the closed form
evaluated in FP32 cancels badly (meshless_vis/fourier_transform.cu:31-60 keep
the closed form there; in FP32 it is off by up to 3e-4 of Phi^(0) for the
Wendland D3 C2 transform on [0.24, 0.5] and 7e-5 for SPH on [0.06, 0.24]).

The polynomial is a least-squares Chebyshev fit, in the variable
x = (s^2 - t_mid) / t_half, of the exact closed form evaluated with mpmath at
40 digits on Chebyshev nodes; it is then converted to monomial coefficients in
x for Horner evaluation.  The fit error is printed and must stay below 1e-9 of
Phi^(0).  Run:  python gen_phi_poly.py > phi_poly.h
"""
import numpy as np
from numpy.polynomial import chebyshev as C
from numpy.polynomial import polynomial as P
import mpmath as mp

mp.mp.dps = 40


def wendland(s):
    m = mp.pi * s
    return (mp.pi * mp.mpf(7.5)) / m**8 * (4 * m**2 - 6 + (6 - m**2) * mp.cos(2 * m) + mp.mpf(4.5) * m * mp.sin(2 * m))


def sph(s):
    m = mp.pi * s
    c, sn = mp.cos(2 * m), mp.sin(2 * m)
    return (mp.mpf("2.3561944901923448") / m**6) * (c - 1) * (c + m * sn - 1)


def fit(f, a, b, deg, phi0, name):
    ta, tb = mp.mpf(a) ** 2, mp.mpf(b) ** 2
    tm, th = (ta + tb) / 2, (tb - ta) / 2
    nodes = np.cos(np.pi * (np.arange(600) + 0.5) / 600)
    ys = np.array([float(f(mp.sqrt(tm + th * mp.mpf(float(x))))) for x in nodes])
    c = C.chebfit(nodes, ys, deg)
    mono = C.cheb2poly(c)
    xt = np.linspace(-1, 1, 4001)
    ref = np.array([float(f(mp.sqrt(tm + th * mp.mpf(float(x))))) for x in xt])
    # FP32 Horner, as the kernel evaluates it
    m32 = mono.astype(np.float32)
    x32 = xt.astype(np.float32)
    acc = np.full_like(x32, m32[-1])
    for k in range(len(m32) - 2, -1, -1):
        acc = (acc * x32 + m32[k]).astype(np.float32)
    fit_err = np.abs(P.polyval(xt, mono) - ref).max() / phi0
    f32_err = np.abs(acc.astype(np.float64) - ref).max() / phi0
    assert fit_err < 1e-9, (name, fit_err)
    out = []
    out.append(f"/* {name}: s in [{a}, {b}), x = (s*s - {float(tm)!r}) * {float(1/th)!r};")
    out.append(f"   fit error {fit_err:.2e}, FP32 Horner error {f32_err:.2e} (units of Phi^(0)) */")
    out.append(f"#define {name}_T_MID {float(tm)!r}f")
    out.append(f"#define {name}_T_INV_HALF {float(1/th)!r}f")
    out.append(f"#define {name}_DEG {deg}")
    coeffs = ", ".join(f"{float(v)!r}f" for v in mono)
    out.append(f"static __device__ __constant__ const float {name}_C[{deg + 1}] = {{{coeffs}}};")
    return "\n".join(out)


if __name__ == "__main__":
    print("/* Generated by gen_phi_poly.py; do not edit. */")
    print("#pragma once")
    print(fit(wendland, 0.24, 1.0, 9, 0.2992, "MV_WENDLAND_POLY"))
    print(fit(sph, 0.06, 0.5, 9, np.pi, "MV_SPH_POLY"))
