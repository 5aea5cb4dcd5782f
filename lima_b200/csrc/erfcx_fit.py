"""Coefficients of the pair kernel's energy-step erfc (nonbonded.cu, EC_*).

erfc(x) e^{x^2} is fitted as t (c0 + c1 t + ... + c9 t^9) with
t = 1 / (1 + p x), p = 0.3275911 (the same t as the force's Abramowitz & Stegun
7.1.26 form, so an energy step reuses the force's reciprocal and e^{-x^2}):
weighted least squares for the relative error on 6,000 Chebyshev nodes of t
over x in [0, 7].  Maximum relative error 7e-10 in exact arithmetic, 2e-7
with the polynomial evaluated by Horner's rule in FP32.

    python lima_b200/csrc/erfcx_fit.py
"""
import numpy as np
from scipy.special import erfcx

P = 0.3275911
X_MAX = 7.0
DEG = 9


def fit():
    tmin = 1.0 / (1.0 + P * X_MAX)
    k = np.arange(6000)
    t = 0.5 * (1 + tmin) + 0.5 * (1 - tmin) * np.cos(np.pi * (k + 0.5) / len(k))
    f = erfcx((1.0 / t - 1.0) / P)
    a = np.vstack([t ** (i + 1) for i in range(DEG + 1)]).T
    c, *_ = np.linalg.lstsq(a / f[:, None], np.ones_like(f), rcond=None)
    return c


if __name__ == "__main__":
    c = fit()
    tmin = 1.0 / (1.0 + P * X_MAX)
    t = np.linspace(tmin, 1.0, 400001)
    g = sum(c[i] * t ** (i + 1) for i in range(DEG + 1))
    print("max relative error", np.max(np.abs(g / erfcx((1 / t - 1) / P) - 1)))
    for i, v in enumerate(c):
        print(f"constexpr float EC{i} = {float(np.float32(v)):.9g}f;   // {v:.17g}")
