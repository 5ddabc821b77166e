"""Partial-fraction rational approximations for the RHMC actions.

The reference reads pre-computed coefficient files (Math_Rational,
src/lib/Tools/math_Rational.cpp:126-180) holding
    x^(n/d) ~ a0 + sum_i b_i / (x + c_i)   on [lo, hi]
for the powers its rational actions need: x^(-1/2) (one flavour of
det(DdagD)^(1/2)), x^(1/4) for the Pauli-Villars numerator and x^(+-1/4) for
the pseudofermion heatbath (Action_F_Rational_Ratio_eo::set_parameters,
src/lib/Action/Fermion/action_F_Rational_Ratio_eo.cpp:20-55).

This module computes such coefficients itself.  For fixed shifts c_i the
constant a0 and the residues b_i are the linear least-squares solution of the
relative-error equations on a logarithmic grid; the log-shifts are fitted with
Levenberg-Marquardt on the remaining relative error (variable projection),
then re-fitted a few times with Lawson-style weights that push the error
towards equal ripple.  Pole counts are reached by continuation (each fit
starts from the interpolated shifts of a smaller one).  Reached maximum
relative errors on [1e-4, 10]: about 2e-6 (10 poles), 5e-10 to 1e-9
(16 poles) and 1e-11 to 7e-10 (24 poles); each table states its own error.

Tables are written and read in the reference's file format and naming
(``parameter_rational.<|n|>_<d>[inv]_<Np>_<lo>_<hi>``), so the same files can
be handed to the reference's Math_Rational.  The committed tables live in
``rational_tables/`` beside this module; ``python -m b200dwf.rational``
regenerates them.
"""
import os

import numpy as np

TABLE_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rational_tables")
# the grids of pole counts the committed tables are generated along
CHAIN = (10, 13, 16, 20, 24)


def _fit(power, lo, hi, n, init=None, grid=1200, lawson=10):
    from scipy.optimize import least_squares
    x = np.logspace(np.log10(lo), np.log10(hi), grid)
    f = x ** power
    w = np.ones_like(x)

    def design(logc):
        c = np.exp(logc)
        return np.concatenate([np.ones((x.size, 1)), 1.0 / (x[:, None] + c[None, :])],
                              axis=1) / f[:, None]

    def linear(logc):
        a = design(logc)
        coef, *_ = np.linalg.lstsq(a * w[:, None], w, rcond=None)
        return coef, a

    def residual(logc):
        coef, a = linear(logc)
        return w * (a @ coef - 1.0)

    if init is None:
        logc = np.linspace(np.log(lo) - 1.0, np.log(hi) + 1.0, n)
    else:
        li = np.sort(np.log(np.asarray(init, np.float64)))
        logc = np.interp(np.linspace(0.0, 1.0, n), np.linspace(0.0, 1.0, li.size), li)
    best = None
    for _ in range(lawson + 1):
        sol = least_squares(residual, logc, method="lm", max_nfev=20000,
                            ftol=1e-15, xtol=1e-15, gtol=1e-15)
        logc = sol.x
        coef, a = linear(logc)
        e = np.abs(a @ coef - 1.0)
        if best is None or e.max() < best[0]:
            best = (e.max(), coef, logc.copy())
        w = w * np.sqrt(e / e.max()) + 1e-4
        w /= w.max()
    _, coef, logc = best
    c = np.exp(logc)
    order = np.argsort(c)
    return float(coef[0]), coef[1:][order], c[order]


def max_rel_error(a0, b, c, lo, hi, power=-0.5, n=40000):
    x = np.logspace(np.log10(lo), np.log10(hi), n)
    r = a0 + (1.0 / (x[:, None] + np.asarray(c)[None, :])) @ np.asarray(b)
    return float(np.max(np.abs(r / x ** power - 1.0)))


def partial_fractions(n_exp, d_exp, lo, hi, n):
    """(a0, b, c, err): x^(n_exp/d_exp) ~ a0 + sum b_i/(x + c_i) on [lo, hi]."""
    power = n_exp / d_exp
    prev = None
    for m in [k for k in CHAIN if k < n] + [n]:
        a0, b, c = _fit(power, lo, hi, m, init=prev)
        prev = c
    return a0, b, c, max_rel_error(a0, b, c, lo, hi, power)


def inv_sqrt_partial_fractions(lo=1e-4, hi=10.0, n=16):
    """(a0, b, c) with x^-1/2 ~ a0 + sum b_i / (x + c_i) on [lo, hi]."""
    try:
        return load(-1, 2, n, lo, hi)[:3]
    except FileNotFoundError:
        return partial_fractions(-1, 2, lo, hi, n)[:3]


def table_name(n_exp, d_exp, n, lo, hi):
    """Math_Rational::read_file's file name for x^(n_exp/d_exp), n poles."""
    return "parameter_rational.%1d_%1d%s_%02d_%010.8f_%07.3f" % (
        abs(n_exp), d_exp, "inv" if n_exp < 0 else "", n, lo, hi)


def write_table(path, n_exp, d_exp, lo, hi, a0, b, c, err):
    with open(path, "w") as f:
        f.write("%6d %5d %5d\n" % (len(b), n_exp, d_exp))
        f.write("  %.16e  %.16e\n" % (lo, hi))
        f.write("  %.6e\n" % err)
        f.write("  %.16e\n" % a0)
        for bi, ci in zip(b, c):
            f.write("  %.16e  %.16e\n" % (bi, ci))


def read_table(path):
    """(n_exp, d_exp, lo, hi, err, a0, b, c) of a Math_Rational-format file."""
    tok = open(path).read().split()
    n, n_exp, d_exp = int(tok[0]), int(tok[1]), int(tok[2])
    lo, hi, err, a0 = (float(t) for t in tok[3:7])
    rest = np.array([float(t) for t in tok[7:7 + 2 * n]]).reshape(n, 2)
    return n_exp, d_exp, lo, hi, err, a0, rest[:, 0].copy(), rest[:, 1].copy()


def load(n_exp, d_exp, n, lo, hi, directory=TABLE_DIR):
    """(a0, b, c, err) from a committed table (FileNotFoundError if absent)."""
    path = os.path.join(directory, table_name(n_exp, d_exp, n, lo, hi))
    ne, de, _, _, err, a0, b, c = read_table(path)
    if (ne, de, len(b)) != (n_exp, d_exp, n):
        raise ValueError("inconsistent table " + path)
    return a0, b, c, err


class Rational:
    """Fopr_Rational's coefficients (src/lib/Fopr/afopr_Rational-tmpl.h:
    140-180): the bounds are given as the square roots of the spectral
    interval (lower_bound, upper_bound) and squared here, as there."""

    def __init__(self, n_poles, n_exp, d_exp, lower_bound, upper_bound, directory=TABLE_DIR):
        self.n_exp, self.d_exp = n_exp, d_exp
        self.lo, self.hi = lower_bound ** 2, upper_bound ** 2
        self.a0, self.b, self.c, self.err = load(n_exp, d_exp, n_poles, self.lo, self.hi,
                                                 directory)

    def __call__(self, x):
        x = np.asarray(x, np.float64)
        return self.a0 + (1.0 / (x[..., None] + self.c)) @ self.b


def main():
    os.makedirs(TABLE_DIR, exist_ok=True)
    lo, hi = 1e-4, 10.0
    for n_exp, d_exp in ((1, 4), (-1, 4), (-1, 2)):
        prev = None
        for n in CHAIN:
            a0, b, c = _fit(n_exp / d_exp, lo, hi, n, init=prev)
            prev = c
            if n in (10, 16, 24):
                err = max_rel_error(a0, b, c, lo, hi, n_exp / d_exp)
                write_table(os.path.join(TABLE_DIR, table_name(n_exp, d_exp, n, lo, hi)),
                            n_exp, d_exp, lo, hi, a0, b, c, err)
                print(table_name(n_exp, d_exp, n, lo, hi), "max rel error %.2e" % err)


if __name__ == "__main__":
    main()
