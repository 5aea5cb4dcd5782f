"""The pair kernel's two erfc forms, evaluated on the CPU in the kernel's FP32
order from the constants in its source (no GPU needed):

* forces: Abramowitz & Stegun 7.1.26, t (a1 + t (a2 + ...)) e^{-x^2} with
  t = 1/(1 + p x): absolute error at most 1.5e-7 in exact arithmetic (their
  published bound), 5.1e-7 with t and the polynomial in FP32 (near x = 0,
  where erfc is 1 and an FP32 ulp is 1.2e-7);
* energy steps: t P7(t) e^{-x^2} on the same t, this build's fit of
  erfc(x) e^{x^2} (lima_b200/csrc/erfcx_fit.py), relative error below 5e-7
  over x in [0, 5.5] with t and the polynomial in FP32, and the fit's
  extrapolation past 5.5 within 2e-4 relative up to x = 30.
"""
import os
import re

import numpy as np
from scipy.special import erfc, erfcx

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "lima_b200", "csrc")


def constants():
    txt = open(os.path.join(SRC, "nonbonded.cu")).read() + open(os.path.join(SRC, "engine.h")).read()
    vals = dict((k, float(v)) for k, v in re.findall(r"\b(AS_P|AS_A\d|EC\d)\s*=\s*([-+0-9.eE]+)f", txt))
    a = [vals[f"AS_A{i}"] for i in range(1, 6)]
    ec = [vals[f"EC{i}"] for i in range(10) if f"EC{i}" in vals]
    return vals["AS_P"], a, ec


def t32(x, p):
    x = x.astype(np.float32)
    return (np.float32(1) / (np.float32(1) + np.float32(p) * x)).astype(np.float32)


def horner32(coef, t):
    """sum_i coef[i] t^i in FP32, highest power first (the kernel's order)."""
    c = np.asarray(coef, np.float32)
    q = (c[-1] * t + c[-2]).astype(np.float32)
    for ci in c[-3::-1]:
        q = (q * t + ci).astype(np.float32)
    return q


def test_force_form_absolute_error():
    p, a, _ = constants()
    x = np.linspace(0.0, 6.0, 200001)
    t = t32(x, p)
    poly = (t * horner32([a[0], a[1], a[2], a[3], a[4]], t)).astype(np.float32)
    approx = poly.astype(np.float64) * np.exp(-x * x)
    assert np.max(np.abs(approx - erfc(x))) < 6.0e-7
    t64 = 1.0 / (1.0 + p * x)
    exact = t64 * (a[0] + t64 * (a[1] + t64 * (a[2] + t64 * (a[3] + t64 * a[4])))) * np.exp(-x * x)
    assert np.max(np.abs(exact - erfc(x))) < 1.5e-7


def test_energy_form_relative_error():
    p, _, ec = constants()
    assert len(ec) == 8
    x = np.linspace(0.0, 5.5, 400001)
    t = t32(x, p)
    g = (horner32(ec, t) * t).astype(np.float32)
    assert np.max(np.abs(g / erfcx(x) - 1.0)) < 5e-7
    xs = np.linspace(5.5, 30.0, 100001)
    ts = 1.0 / (1.0 + p * xs)
    gs = ts * sum(c * ts ** i for i, c in enumerate(ec))
    assert np.max(np.abs(gs / erfcx(xs) - 1.0)) < 2.5e-4
