"""GPU solvers through the C ABI against the CPU oracle: multishift CG and the
mixed-precision Richardson with f32 / f16 / bf16 inner solves."""
import numpy as np
import pytest

from b200dwf import synth

pytestmark = pytest.mark.gpu

LAT, LS = [4, 4, 4, 8], 8


def make(seed=5):
    import b200dwf
    from oracle.oracle import OracleDWF
    u = synth.gauge_field(LAT, seed, "near", eps=0.3)
    ora = OracleDWF(LAT, LS, 0.02, 1.8)
    ora.set_links(u)
    dev = b200dwf.DomainWall(LAT, LS, 0.02, 1.8)
    dev.set_config(u)
    return ora, dev


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_multishift_matches_oracle():
    ora, dev = make()
    b = synth.spinor_field(LAT, LS, 9)
    sigma = [0.005, 0.05, 0.5, 5.0]
    fb = dev.new_field(0)
    dev.convert(fb, b)
    xs = [dev.new_field(0) for _ in sigma]
    n, diff, rc = dev.shiftcg(xs, sigma, fb, 1e-22, 3000)
    assert rc == 0
    xr, nr, dr, rcr = ora.shiftcg(b, sigma, 1e-22, 3000)
    assert rcr == 0
    assert abs(n - nr) <= 1
    assert diff < 1e-9
    for i in range(len(sigma)):
        assert rel(dev.reverse(xs[i]), xr[i]) < 1e-9, i


@pytest.mark.parametrize("inner", [1, 2, 3])
def test_mixed_precision_richardson(inner):
    ora, dev = make(6)
    b = synth.spinor_field(LAT, LS, 10)
    fb, fx = dev.new_field(0), dev.new_field(0)
    dev.convert(fb, b)
    tol_inner = 1e-8 if inner == 1 else 1e-4
    nout, nin, diff, rc = dev.richardson(fx, fb, inner, 1e-20, 60, tol_inner, 5000)
    assert rc == 0, (nout, nin, diff)
    assert diff < 1e-10
    xr, _, _, _ = ora.cg(b, 1e-24, 5000)
    assert rel(dev.reverse(fx), xr) < 1e-8


def test_zero_rhs_and_nonconvergence_status():
    _, dev = make()
    fb, fx = dev.new_field(0), dev.new_field(0)
    n, diff, rc = dev.cg(fx, fb, 1e-20, 100)
    assert rc == 0 and n == 0 and diff == 0.0
    b = synth.spinor_field(LAT, LS, 3)
    dev.convert(fb, b)
    n, diff, rc = dev.cg(fx, fb, 1e-30, 3)   # cannot converge in 3 iterations
    assert rc == -4 and n == 3 and diff > 1e-6
