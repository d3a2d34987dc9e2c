"""Fits the polynomial coefficients of myrt_b200/csrc/glmath.hpp.

Each kernel is a near-minimax polynomial for the relative error of the final
float function, found by Lawson's algorithm (iteratively reweighted least
squares, C. L. Lawson 1961) on 4,000 Chebyshev nodes of the reduced interval,
in float64, then rounded to float32. Run:

    python -m myrt_b200.glmath_fit

It prints the coefficient table that glmath.hpp holds and the relative error of
each float64 fit. The float32 functions themselves are measured against float64
numpy references by tests/test_glmath.py.
"""
from __future__ import annotations

import numpy as np


def lawson(basis, target, weight, iters: int = 400):
    """Coefficients c minimising max |weight * (basis @ c - target)| (approx.)."""
    w = np.ones(len(target))
    c = None
    for _ in range(iters):
        A = basis * (w * weight)[:, None]
        b = target * w * weight
        c, *_ = np.linalg.lstsq(A, b, rcond=None)
        err = np.abs(weight * (basis @ c - target))
        w = w * err
        w = w / w.sum() * len(w)
        w = np.sqrt(w)  # damped update
    return c


def cheb(a: float, b: float, n: int = 4000) -> np.ndarray:
    k = np.arange(n)
    return 0.5 * (a + b) + 0.5 * (b - a) * np.cos((2 * k + 1) * np.pi / (2 * n))


def fit_sin():
    # sin(r) = r + r^3 * P(r^2), r in [0, pi/4]; error relative to sin(r)
    r = cheb(1e-4, np.pi / 4)
    z = r * r
    basis = np.stack([r ** 3 * z ** j for j in range(4)], 1)
    return lawson(basis, np.sin(r) - r, 1.0 / np.sin(r))


def fit_cos():
    # cos(r) = 1 - r^2 / 2 + r^4 * Q(r^2), r in [0, pi/4]
    r = cheb(1e-4, np.pi / 4)
    z = r * r
    basis = np.stack([z * z * z ** j for j in range(4)], 1)
    return lawson(basis, np.cos(r) - 1 + z / 2, 1.0 / np.cos(r))


def fit_atan():
    # atan(t) = t + t^3 * A(t^2), |t| <= tan(pi / 8)
    t = cheb(1e-4, np.tan(np.pi / 8))
    z = t * t
    basis = np.stack([t ** 3 * z ** j for j in range(6)], 1)
    return lawson(basis, np.arctan(t) - t, 1.0 / np.arctan(t))


def fit_log():
    # log(m) = 2 s + s^3 * L(s^2), s = (m - 1) / (m + 1), m in [sqrt(1/2), sqrt(2)]
    s_max = (np.sqrt(2) - 1) / (np.sqrt(2) + 1)
    s = cheb(1e-4, s_max)
    z = s * s
    m = (1 + s) / (1 - s)
    basis = np.stack([s ** 3 * z ** j for j in range(4)], 1)
    return lawson(basis, np.log(m) - 2 * s, 1.0 / np.log(m))


def fit_exp2():
    # 2^f = 1 + f * E(f), f in [-0.5, 0.5] (a little wider for rounding)
    f = cheb(-0.5005, 0.5005)
    basis = np.stack([f ** (j + 1) for j in range(7)], 1)
    return lawson(basis, np.exp2(f) - 1, 1.0 / np.exp2(f))


def rel_error(name, coef):
    c = np.asarray(coef, np.float32).astype(np.float64)
    if name == "sin":
        r = np.linspace(1e-4, np.pi / 4, 100001)
        z = r * r
        v = r + r ** 3 * np.polyval(c[::-1], z)
        return np.max(np.abs(v / np.sin(r) - 1))
    if name == "cos":
        r = np.linspace(0, np.pi / 4, 100001)
        z = r * r
        v = 1 - z / 2 + z * z * np.polyval(c[::-1], z)
        return np.max(np.abs(v / np.cos(r) - 1))
    if name == "atan":
        t = np.linspace(1e-4, np.tan(np.pi / 8), 100001)
        z = t * t
        v = t + t ** 3 * np.polyval(c[::-1], z)
        return np.max(np.abs(v / np.arctan(t) - 1))
    if name == "log":
        s = np.linspace(1e-4, (np.sqrt(2) - 1) / (np.sqrt(2) + 1), 100001)
        z = s * s
        m = (1 + s) / (1 - s)
        v = 2 * s + s ** 3 * np.polyval(c[::-1], z)
        return np.max(np.abs(v / np.log(m) - 1))
    f = np.linspace(-0.5, 0.5, 100001)
    v = 1 + f * np.polyval(c[::-1], f)
    return np.max(np.abs(v / np.exp2(f) - 1))


def main():
    fits = {"sin": fit_sin(), "cos": fit_cos(), "atan": fit_atan(), "log": fit_log(), "exp2": fit_exp2()}
    for name, c in fits.items():
        c32 = np.asarray(c, np.float32)
        print(f"{name}: rel. error {rel_error(name, c32):.3e}")
        print("  " + ", ".join(f"{float(x):.9e}f" for x in c32))


if __name__ == "__main__":
    main()
