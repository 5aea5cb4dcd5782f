"""Coefficients of the pair kernel's energy-step erfc (nonbonded.cu, EC_*).

erfc(x) e^{x^2} is fitted as t (c0 + c1 t + ... + c7 t^7) with
t = 1 / (1 + p x), p = 0.3275911 (the same t as the force's Abramowitz & Stegun
7.1.26 form, so an energy step reuses the force's reciprocal and e^{-x^2}):
weighted least squares for the relative error on 6,000 Chebyshev nodes of t
over x in [0, 5.5].  Maximum relative error 6e-8 in exact arithmetic, 4.4e-7
with t, the polynomial (Horner's rule) and the product in FP32 — the same as a
degree-9 fit over [0, 7], whose extra accuracy the FP32 evaluation loses.
Past x = 5.5 (erfc < 1e-14, nothing a sum of pair energies can see) the
polynomial is extrapolated, within 2e-4 relative up to x = 30.

    python lima_b200/csrc/erfcx_fit.py
"""
import numpy as np
from scipy.special import erfcx

P = 0.3275911
X_MAX = 5.5
DEG = 7


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
