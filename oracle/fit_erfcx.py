"""Fit of the scaled complementary error function used by the pair kernels.

erfcx(x) = erfc(x) * exp(x^2) is smooth and bounded on [0, 4]; it is
approximated by a degree-8 polynomial in t = 1 / (1 + x/2), fitted here by
weighted least squares (relative error) against scipy's double-precision
erfcx.  The kernels then form erfc(x) = erfcx(x) * exp(-x^2), reusing the
exp(-x^2) factor the Coulomb force needs anyway.  Run this file to print the
coefficients pasted into snb_common.cuh and the achieved error bound.
"""

import numpy as np
from scipy.special import erfcx

P = 0.5
DEG = 8
XMAX = 4.0


def fit():
    x = np.linspace(0.0, XMAX, 40001)
    t = 1.0 / (1.0 + P * x)
    y = erfcx(x)
    A = np.vander(t, DEG + 1, increasing=True)
    w = 1.0 / y
    coef, *_ = np.linalg.lstsq(A * w[:, None], y * w, rcond=None)
    return coef


def f32_error(coef):
    x = np.linspace(0.0, XMAX, 400001).astype(np.float32)
    t = (np.float32(1) / (np.float32(1) + np.float32(P) * x)).astype(np.float32)
    acc = np.zeros_like(t)
    for c in coef.astype(np.float32)[::-1]:
        acc = (acc * t + c).astype(np.float32)
    y = erfcx(x.astype(np.float64))
    return float(np.max(np.abs(acc - y) / y))


if __name__ == "__main__":
    c = fit()
    for k, v in enumerate(c):
        print(f"  c{k} = {np.float32(v)!r}f")
    print("max relative error of the float32 evaluation on [0, 4]:", f32_error(c))
