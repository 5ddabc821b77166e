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


@pytest.mark.parametrize("window", [0, 3, 8, 16])
def test_multishift_matches_oracle(window):
    """Per-iteration shift updates (window 0) and deferred updates from a
    window of stored residuals (8, the default 16; 3 exercises windows that end
    mid-solve and shifts pruned inside a window) against the oracle."""
    ora, dev = make()
    dev.set_shift_window(window)
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


def test_multishift_window_agrees_with_per_iteration_updates():
    """Sixteen shifts spanning 1e-4..64 (the rational poles' range): the
    windowed solver reproduces the per-iteration one to rounding, iteration
    count included, and rejects windows outside [0, 16]."""
    import b200dwf
    _, dev = make(7)
    b = synth.spinor_field(LAT, LS, 11)
    fb = dev.new_field(0)
    dev.convert(fb, b)
    sigma = list(np.logspace(-4, np.log10(64.0), 16))
    out = {}
    for window in (0, 8, 16):
        dev.set_shift_window(window)
        xs = [dev.new_field(0) for _ in sigma]
        n, diff, rc = dev.shiftcg(xs, sigma, fb, 1e-22, 3000)
        assert rc == 0 and diff < 1e-9
        out[window] = (n, [dev.reverse(x) for x in xs])
    for window in (8, 16):
        assert abs(out[window][0] - out[0][0]) <= 1
        for i in range(len(sigma)):
            assert rel(out[window][1][i], out[0][1][i]) < 1e-10, (window, i)
    for bad in (-1, 17):
        with pytest.raises(b200dwf.B200Error):
            dev.set_shift_window(bad)


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


@pytest.mark.parametrize("alpha", [1.0, 1.3])
def test_solvers_with_nontrivial_prefactor(alpha):
    """Moebius kernel (b = 1.5, c = 0.5) and, with alpha = 1.3, a pre-factor
    that differs per chirality: the D_eo pre-factor is not the identity, so
    CG, multishift (per-iteration and windowed) and Richardson carry the
    M5pre p field that the Shamir runs above skip.  All against the oracle."""
    import b200dwf
    from oracle.oracle import OracleDWF
    lat, ls = [4, 4, 4, 8], 8
    u = synth.gauge_field(lat, 21, "near", eps=0.3)
    ora = OracleDWF(lat, ls, 0.02, 1.0, 1.5, 0.5, alpha)
    ora.set_links(u)
    dev = b200dwf.DomainWall(lat, ls, 0.02, 1.0, 1.5, 0.5, alpha)
    dev.set_config(u)
    b = synth.spinor_field(lat, ls, 22)
    fb, fx = dev.new_field(0), dev.new_field(0)
    dev.convert(fb, b)
    n, diff, rc = dev.cg(fx, fb, 1e-22, 3000)
    xr, nr, _, rcr = ora.cg(b, 1e-22, 3000)
    assert rc == 0 and rcr == 0 and abs(n - nr) <= 1
    assert rel(dev.reverse(fx), xr) < 1e-9
    sigma = [0.005, 0.05, 0.5, 5.0]
    xsr, nsr, _, _ = ora.shiftcg(b, sigma, 1e-22, 3000)
    for window in (0, 16):
        dev.set_shift_window(window)
        xs = [dev.new_field(0) for _ in sigma]
        n, diff, rc = dev.shiftcg(xs, sigma, fb, 1e-22, 3000)
        assert rc == 0 and abs(n - nsr) <= 1 and diff < 1e-9
        for i in range(len(sigma)):
            assert rel(dev.reverse(xs[i]), xsr[i]) < 1e-9, (window, i)
    fx2 = dev.new_field(0)
    nout, nin, diff, rc = dev.richardson(fx2, fb, 1, 1e-20, 60, 1e-8, 5000)
    assert rc == 0 and diff < 1e-10
    assert rel(dev.reverse(fx2), xr) < 1e-8
