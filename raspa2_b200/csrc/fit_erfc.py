"""Generates erfc_fit.h: the FP32 complementary error function of the
mixed-precision real-space Ewald term.

Method: erfc(x) = exp(-x^2) * R(t) with t = 1 / (1 + P*x), the form of
Abramowitz & Stegun 7.1.26 (Hastings), but with R a degree-8 polynomial in t
fitted here by Chebyshev least squares to R(x) = erfc(x) exp(x^2) on
x in [0, XMAX], using Python's double-precision math.erfc as the target.
XMAX = 3.7 covers alpha * r_c for alpha <= 0.3 / A and r_c = 12 A.

Run `python fit_erfc.py` to regenerate the header; it prints the maximum
relative error of the polynomial evaluated in FP32 (Horner) against erfc,
excluding the exp(-x^2) factor (evaluated on the GPU with exp2f).
"""
import math
import os

import numpy as np
from numpy.polynomial import chebyshev as C

P = 0.5
XMAX = 3.7
DEG = 8


def fit():
    xs = np.linspace(0.0, XMAX, 40001)
    R = np.array([math.erfc(x) * math.exp(x * x) for x in xs])
    t = 1.0 / (1.0 + P * xs)
    tmin = 1.0 / (1.0 + P * XMAX)
    u = (2.0 * t - (1.0 + tmin)) / (1.0 - tmin)
    c = C.chebfit(u, R, DEG)
    a, b = 2.0 / (1.0 - tmin), -(1.0 + tmin) / (1.0 - tmin)
    poly = np.polynomial.Polynomial(C.cheb2poly(c))(np.polynomial.Polynomial([b, a]))
    coef = poly.coef.astype(np.float32)
    # FP32 Horner check
    tf = (np.float32(1.0) / (np.float32(1.0) + np.float32(P) * xs.astype(np.float32))).astype(np.float32)
    acc = np.full_like(tf, coef[-1])
    for k in range(len(coef) - 2, -1, -1):
        acc = (acc * tf + coef[k]).astype(np.float32)
    err = float(np.max(np.abs(acc.astype(np.float64) - R) / R))
    return coef, err


def main():
    coef, err = fit()
    here = os.path.dirname(os.path.abspath(__file__))
    lines = [
        "/* Generated by fit_erfc.py: erfc(x) ~= exp(-x^2) * sum_k c_k t^k, t = 1/(1+P x).",
        f" * Fitted on x in [0, {XMAX}]; max relative error of the FP32 polynomial part {err:.2e}. */",
        "#ifndef RGPU_ERFC_FIT_H", "#define RGPU_ERFC_FIT_H",
        f"#define RGPU_ERFC_P {P:.9g}f",
        f"#define RGPU_ERFC_XMAX {XMAX:.9g}f",
        f"#define RGPU_ERFC_DEG {DEG}",
        f"#define RGPU_ERFC_MAXREL {err:.3e}",
    ] + [f"#define RGPU_ERFC_C{k} {float(c):.9e}f" for k, c in enumerate(coef)] + [
        "#endif", "",
    ]
    with open(os.path.join(here, "erfc_fit.h"), "w") as fh:
        fh.write("\n".join(lines))
    print(f"max relative error {err:.3e}")


if __name__ == "__main__":
    main()
