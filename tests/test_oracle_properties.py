"""Algebraic identities of the even/odd DWF operator, checked on the oracle
(size-independent properties used again on the GPU at full sizes)."""
import numpy as np
import pytest

from b200dwf import synth
from oracle.oracle import OracleDWF


@pytest.fixture(scope="module")
def op():
    lat = [4, 4, 4, 8]
    o = OracleDWF(lat, 8, 0.04, 1.8, 1.0, 0.0, 1.0, (1, 1, 1, -1))
    o.set_links(synth.gauge_field(lat, 7, "hot"))
    return o


def rand(op, seed):
    return synth.spinor_field(op.lattice, op.Ls, seed)


def test_adjointness(op):
    x, y = rand(op, 1), rand(op, 2)
    for mode in ("Deo", "Doe", "Dee", "Dee_inv", "D", "H"):
        lhs = np.dot(x, op.mult(mode, y))
        rhs = np.dot(op.mult(mode, x, dag=True), y)
        assert abs(lhs - rhs) < 1e-12 * abs(lhs) + 1e-10, mode


def test_dee_inverse(op):
    x = rand(op, 3)
    y = op.mult("Dee_inv", op.mult("Dee", x))
    assert np.linalg.norm(y - x) / np.linalg.norm(x) < 1e-13
    y = op.mult("Dee_inv", op.mult("Dee", x, dag=True), dag=True)
    assert np.linalg.norm(y - x) / np.linalg.norm(x) < 1e-13


def test_ddagd_positive(op):
    x = rand(op, 6)
    assert np.dot(x, op.mult("DdagD", x)) > 0
