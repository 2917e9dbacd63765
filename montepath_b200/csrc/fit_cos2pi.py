"""Coefficients of the FP32 cos(2 pi t) polynomial used by the fused
counter-hash normal (cos_2pi_fast in mpc_device.cuh).

cos(2 pi t) on t in [-1/2, 1/2] as a degree-8 polynomial in x = t^2, fitted
by Chebyshev least squares on a dense grid of x in [0, 1/4] and rounded to
float32.  Prints the coefficients (constant term first) and the maximum
absolute error of a float32 Horner evaluation (about 3.3e-7).

    python montepath_b200/csrc/fit_cos2pi.py
"""

import numpy as np


def fit(deg: int = 8):
    x = np.linspace(0.0, 0.25, 200001)
    f = np.cos(2.0 * np.pi * np.sqrt(x))
    cheb = np.polynomial.chebyshev.Chebyshev.fit(x, f, deg, domain=[0.0, 0.25])
    poly = cheb.convert(kind=np.polynomial.Polynomial, domain=[0.0, 0.25], window=[0.0, 0.25])
    coef = poly.coef.astype(np.float32)
    xs = x.astype(np.float32)
    acc = np.full_like(xs, coef[-1])
    for a in coef[-2::-1]:
        acc = (acc.astype(np.float64) * xs.astype(np.float64) + np.float64(a)).astype(np.float32)
    return coef, float(np.max(np.abs(acc.astype(np.float64) - f)))


if __name__ == "__main__":
    coef, err = fit()
    for c in coef:
        print(f"{float(c):.9e}f")
    print("max abs error", err)
