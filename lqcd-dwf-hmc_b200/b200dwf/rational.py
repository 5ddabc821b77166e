"""Partial-fraction rational approximations for the RHMC action.

The reference reads pre-computed coefficient files (Math_Rational,
src/lib/Tools/math_Rational.cpp:126-180) holding
    x^(p/q) ~ a0 + sum_i b_i / (x + c_i)   on [lo, hi].
This module computes such coefficients itself for x^(-1/2) (one flavour of
det(DdagD)^(1/2)): the shifts c_i are optimised by variable projection —
for fixed shifts the residues b_i are the linear least-squares solution of the
relative-error equations on a logarithmic grid, and the log-shifts are fitted
with Levenberg-Marquardt on the remaining relative error.  With 16 poles on
[1e-4, 10] the maximum relative error is about 4e-9 (the reference's shipped
16-pole file states 5e-10 for the same interval).
"""
import numpy as np


def inv_sqrt_partial_fractions(lo=1e-4, hi=10.0, n=16, grid=600):
    """(a0, b, c) with x^-1/2 ~ a0 + sum b_i / (x + c_i) on [lo, hi]; a0 = 0."""
    from scipy.optimize import least_squares
    x = np.logspace(np.log10(lo), np.log10(hi), grid)
    f = x ** -0.5

    def residues(logc):
        c = np.exp(logc)
        a = 1.0 / (x[:, None] + c[None, :]) / f[:, None]
        b, *_ = np.linalg.lstsq(a, np.ones_like(x), rcond=None)
        return b, c

    def rel_err(logc):
        b, c = residues(logc)
        return (1.0 / (x[:, None] + c[None, :]) @ b) / f - 1.0

    logc0 = np.linspace(np.log(lo / 3), np.log(hi * 3), n)
    sol = least_squares(rel_err, logc0, method="lm", max_nfev=4000)
    b, c = residues(sol.x)
    order = np.argsort(c)
    return 0.0, b[order], c[order]


def max_rel_error(a0, b, c, lo, hi, power=-0.5, n=20000):
    x = np.logspace(np.log10(lo), np.log10(hi), n)
    r = a0 + (1.0 / (x[:, None] + np.asarray(c)[None, :])) @ np.asarray(b)
    return float(np.max(np.abs(r / x ** power - 1.0)))
