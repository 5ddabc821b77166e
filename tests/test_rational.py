"""The partial-fraction approximation of x^-1/2 used by the RHMC action
(computed here; the reference reads coefficient files of the same form,
Math_Rational, src/lib/Tools/math_Rational.cpp:126-180)."""
from b200dwf.rational import inv_sqrt_partial_fractions, max_rel_error


def test_sixteen_poles_on_the_reference_interval():
    a0, b, c = inv_sqrt_partial_fractions(1e-4, 10.0, 16)
    assert len(b) == len(c) == 16
    assert min(c) > 0 and min(b) > 0          # shifted CG needs positive shifts
    assert max_rel_error(a0, b, c, 1e-4, 10.0) < 2e-8


def test_fewer_poles_are_less_accurate():
    e12 = max_rel_error(*inv_sqrt_partial_fractions(1e-4, 10.0, 12), 1e-4, 10.0)
    e16 = max_rel_error(*inv_sqrt_partial_fractions(1e-4, 10.0, 16), 1e-4, 10.0)
    assert e16 < e12 < 1e-5
