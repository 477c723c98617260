"""Regenerates the polynomial coefficients of the FP32 atan2 and atanh of the compensated
path (lenstool-hpc_b200/csrc/lt_profiles32.cuh: fatan2, fatanh_third) by a Remez exchange
on the relative error, in float64 with numpy.

  fatan2:       atan(a) = a P(a^2),  P of degree 7, a in [0, 1]
  fatanh_third: atanh(s) = s (1 + x Q(x)),  x = s^2 in [0, 1/9],  Q of degree 3
                (the constant term is fixed at 1 so that atanh(s) ~ s stays exact to first order)

Each fit minimises max |s P - f| / |f| over the interval.  The exchange alternates
between solving for the polynomial that equioscillates on n + 2 reference points and
moving the points to the extrema of the new error curve, until the error's extrema
agree to 1e-6 of their size.

  python tests/golden/fit_fast_math.py      prints the coefficients as C float literals
"""
from __future__ import annotations

import numpy as np


def remez(g, w, basis, lo, hi, n_coef, iters=60, grid=200001):
    """Minimax fit of g(x) ~ sum_k c_k basis_k(x) with error weight 1/w(x) (w > 0) on
    [lo, hi]: returns (coefficients, max weighted error)."""
    xs = np.linspace(lo, hi, grid)
    m = n_coef + 1
    # Chebyshev points as the first reference
    ref = 0.5 * (lo + hi) - 0.5 * (hi - lo) * np.cos(np.pi * np.arange(m) / (m - 1))
    E = 0.
    for _ in range(iters):
        A = np.column_stack([basis(ref, k) for k in range(n_coef)] + [(-1.) ** np.arange(m) * w(ref)])
        sol = np.linalg.solve(A, g(ref))
        c, E = sol[:-1], sol[-1]
        err = (sum(c[k] * basis(xs, k) for k in range(n_coef)) - g(xs)) / w(xs)
        # the extrema of the error: one per sign run, the endpoints included
        sgn = np.sign(err)
        sgn[sgn == 0] = 1
        runs = np.flatnonzero(np.diff(sgn)) + 1
        bounds = np.concatenate([[0], runs, [xs.size]])
        ext = np.array([b0 + np.argmax(np.abs(err[b0:b1])) for b0, b1 in zip(bounds[:-1], bounds[1:])])
        if ext.size > m:  # keep the m largest while alternating: drop the smallest ends
            while ext.size > m:
                if abs(err[ext[0]]) < abs(err[ext[-1]]):
                    ext = ext[1:]
                else:
                    ext = ext[:-1]
        if ext.size < m:
            break
        new = xs[ext]
        emax = np.max(np.abs(err[ext]))
        if np.max(np.abs(np.abs(err[ext]) - emax)) <= 1e-6 * emax:
            ref = new
            break
        ref = new
    err = (sum(c[k] * basis(xs, k) for k in range(n_coef)) - g(xs)) / w(xs)
    return c, float(np.max(np.abs(err)))


def fit_atan():
    """atan(a)/a = P(a^2) on a in [0, 1]; relative error of a P(a^2) against atan a."""
    def g(s):  # s = a^2
        a = np.sqrt(s)
        with np.errstate(invalid="ignore", divide="ignore"):
            r = np.where(a > 0, np.arctan(a) / np.where(a > 0, a, 1.), 1.)
        return r
    c, e = remez(g, g, lambda s, k: s ** k, 0., 1., 8)
    return c, e


def fit_atanh_third():
    """atanh(s)/s = 1 + x Q(x), x = s^2 in [0, 1/9]: fit x Q(x) to atanh(s)/s - 1 with the
    relative error of the whole atanh(s)/s."""
    def f(x):
        s = np.sqrt(x)
        with np.errstate(invalid="ignore", divide="ignore"):
            return np.where(s > 0, np.arctanh(s) / np.where(s > 0, s, 1.), 1.)
    c, e = remez(lambda x: f(x) - 1., f, lambda x, k: x ** (k + 1), 0., 1. / 9., 4)
    return np.concatenate([[1.], c]), e


def main():
    ca, ea = fit_atan()
    ct, et = fit_atanh_third()
    print(f"fatan2: P(s), s = a^2, highest degree first (max relative error {ea:.2e}):")
    print("  " + ", ".join(f"{float(np.float32(v)):.9e}f" for v in ca[::-1]))
    print(f"fatanh_third: 1 + c1 x + ... + c4 x^4, highest first (max relative error {et:.2e}):")
    print("  " + ", ".join(f"{float(np.float32(v)):.9e}f" for v in ct[::-1]))


if __name__ == "__main__":
    main()
