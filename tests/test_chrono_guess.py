"""The minimal residual extrapolation of the MD solves' starting guess
(b200dwf.hmc.Solver with chrono_depth > 1), its host logic on the CPU: an
operator stand-in whose DdagD is a seeded symmetric positive definite matrix
and whose fields are numpy vectors, with the solve itself replaced by an
exact one that records the start it was handed."""
import numpy as np

from b200dwf.hmc import Solver


class Vec:
    def __init__(self, n):
        self.a = np.zeros(n)

    def zero(self):
        self.a[:] = 0.0


class FakeOp:
    """DdagD = A (n x n SPD); dot, axpby and new_field as the plan has them."""

    def __init__(self, n, seed):
        rng = np.random.default_rng(seed)
        q = rng.standard_normal((n, n))
        self.A = q @ q.T + n * np.eye(n)
        self.n = n
        self.starts = []

    def new_field(self, prec=0):
        return Vec(self.n)

    def mult(self, v, w, mode):
        assert mode == "DdagD"
        v.a[:] = self.A @ w.a

    def dot(self, x, y):
        return float(x.a @ y.a)

    def axpby(self, y, a, x, b):
        y.a[:] = a * x.a + (b * y.a if b != 0.0 else 0.0)

    def set_initial_guess(self, use):
        pass

    def cg(self, x, b, tol2, maxiter):
        self.starts.append(x.a.copy())
        x.a[:] = np.linalg.solve(self.A, b.a)
        return 1, 0.0, 0


def test_guess_minimises_the_a_norm_error_over_the_history():
    op = FakeOp(40, 3)
    s = Solver("cg", 1e-20, chrono=True, chrono_depth=3)
    rng = np.random.default_rng(4)
    b0 = rng.standard_normal(op.n)
    x, b = Vec(op.n), Vec(op.n)
    sols = []
    for k in range(4):                  # slowly moving right-hand sides, as in MD
        b.a[:] = b0 + 0.05 * k * rng.standard_normal(op.n)
        s.solve(op, x, b, guess=(k > 0))
        sols.append(x.a.copy())
    # the 4th solve started from the combination of the three earlier
    # solutions closest to its own solution in the A norm
    start = op.starts[-1]
    xs = sols[-1]
    V = np.stack(sols[:3], axis=1)
    c = np.linalg.solve(V.T @ op.A @ V, V.T @ op.A @ xs)
    best = V @ c
    assert np.allclose(start, best, rtol=1e-8, atol=1e-10)
    err = lambda y: float((y - xs) @ op.A @ (y - xs))
    assert err(start) <= err(sols[2]) + 1e-12   # never worse than the previous solution


def test_forget_drops_the_history():
    op = FakeOp(20, 5)
    s = Solver("cg", 1e-20, chrono=True, chrono_depth=4)
    x, b = Vec(op.n), Vec(op.n)
    b.a[:] = 1.0
    s.solve(op, x, b)
    s.solve(op, x, b, guess=True)
    assert len(s._hist) == 2
    s.forget()
    assert len(s._hist) == 0
    x.a[:] = 7.0
    s.solve(op, x, b, guess=True)       # one stored solution: x itself is the start
    assert np.allclose(op.starts[-1], 7.0)


def test_repeated_system_is_reproduced_by_the_extrapolation():
    op = FakeOp(30, 6)
    s = Solver("cg", 1e-20, chrono=True, chrono_depth=3)
    x, b = Vec(op.n), Vec(op.n)
    b.a[:] = np.linspace(-1, 1, op.n)
    s.solve(op, x, b)
    s.solve(op, x, b, guess=True)
    x.zero()
    s.solve(op, x, b, guess=True)       # two identical solutions in the history
    assert np.allclose(op.starts[-1], np.linalg.solve(op.A, b.a), rtol=1e-10)
