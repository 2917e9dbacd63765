"""Fits the FP32 inverse normal CDF used by the fused kernels.

    z = Phi^{-1}(u) = x * g(w),  x = 2u - 1,  w = -ln(4 u (1 - u)) = -ln(1 - x^2)

g is smooth in w.  Central region w < W_SPLIT: g = P(w - W_MID) (Horner,
one branch for >99% of samples); tail w >= W_SPLIT: g = Q(sqrt(w) - S_MID).
The polynomials are Chebyshev least-squares fits in float64 against
scipy.special.ndtri, checked here under float32 Horner evaluation.

Run: python montepath_b200/csrc/gen_icdf_coeffs.py  (prints the C constants)
"""

import numpy as np
from scipy.special import ndtri

W_SPLIT = 5.0
W_MAX = 23.0  # u down to 2^-33
DEG_C, DEG_T = 9, 9


def g_of_w(w):
    # invert w -> x: 1 - x^2 = exp(-w), x = sqrt(1 - exp(-w)) (positive branch)
    x = np.sqrt(-np.expm1(-w))
    u = 0.5 * (1.0 + x)
    return ndtri(u) / x


def fit(var_lo, var_hi, transform, deg, center):
    k = np.arange(4096)
    nodes = np.cos(np.pi * (k + 0.5) / 4096)  # Chebyshev nodes
    v = 0.5 * (var_lo + var_hi) + 0.5 * (var_hi - var_lo) * nodes
    w = transform(v)
    y = g_of_w(w)
    coef = np.polynomial.polynomial.polyfit(v - center, y, deg)
    return coef


def horner32(coef, t):
    t = np.float32(t)
    p = np.float32(coef[-1])
    for c in coef[-2::-1]:
        p = np.float32(np.float64(p) * np.float64(t) + np.float64(np.float32(c)))  # one rounding, like FMA
    return p


def main():
    w_mid = 2.5
    cc = fit(1e-9, W_SPLIT, lambda v: v, DEG_C, w_mid)
    s_lo, s_hi = np.sqrt(W_SPLIT), np.sqrt(W_MAX)
    s_mid = 0.5 * (s_lo + s_hi)
    ct = fit(s_lo, s_hi, lambda v: v * v, DEG_T, s_mid)
    # float32 evaluation check over u
    u = np.concatenate([np.linspace(1e-7, 1 - 1e-7, 200001), np.geomspace(2**-33, 0.01, 20001)])
    u32 = u.astype(np.float32).astype(np.float64)
    x = 2 * u32 - 1
    w = -np.log(4 * u32 * (1 - u32))
    g = np.where(w < W_SPLIT, [float(horner32(cc, wi - w_mid)) for wi in w],
                 [float(horner32(ct, np.sqrt(wi) - s_mid)) for wi in w])
    z = x * g
    ref = ndtri(u32)
    rel = np.abs(z - ref) / np.maximum(np.abs(ref), 1e-3)
    print(f"// max relative error (float32 evaluation, exact w): {rel.max():.3e}")
    print(f"#define MPC_ICDF_W_SPLIT {W_SPLIT:.1f}f")
    print(f"#define MPC_ICDF_W_MID {w_mid:.1f}f")
    print(f"#define MPC_ICDF_S_MID {s_mid:.9g}f")
    print("static __device__ const float kIcdfCentral[] = {" + ", ".join(f"{c:.9e}f" for c in cc) + "};")
    print("static __device__ const float kIcdfTail[] = {" + ", ".join(f"{c:.9e}f" for c in ct) + "};")


if __name__ == "__main__":
    main()
