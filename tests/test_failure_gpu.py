"""The failure path of the bulk-copy (TMA-fed) hop kernels, exercised without
any GPU fault.

A host-set hook (b200_dwf_inject_wait_failure) makes every TMA-fed hop treat
its wait for one hop direction as if the wait's bound had run out.  The
kernel then sets the plan's device error word, still waits for the copies it
has in flight, and returns without writing its outputs.  Nothing hangs and
no copy is abandoned: the copies complete normally.  Checked here:

* a synchronous mult (the default) reports B200_ECUDA and leaves its output
  untouched; the word is cleared, and the next call is correct again;
* with asynchronous calls the error surfaces at the next synchronising call
  (reverse, check_error) instead;
* the solvers and the force report it too.

The reference has no fault handling on this path (its OpenACC runtime aborts;
its solvers log a non-convergence and continue), so the oracle only checks
the recovered results."""
import numpy as np
import pytest

from b200dwf import synth

pytestmark = pytest.mark.gpu

CASE = ([4, 4, 4, 8], 8, 0.04, 1.8)
# (storage precision, a TMA-fed hop variant of it)
TMA = [(0, 1), (0, 3), (0, 7), (1, 6), (2, 7), (1, 8)]


def make(seed=3):
    import b200dwf
    from oracle.oracle import OracleDWF
    lat, ls, mq, m0 = CASE
    u = synth.gauge_field(lat, 200 + seed, "hot")
    ora = OracleDWF(lat, ls, mq, m0)
    ora.set_links(u)
    op = b200dwf.DomainWall(lat, ls, mq, m0)
    op.set_config(u)
    return ora, op


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("prec,variant", TMA)
@pytest.mark.parametrize("direction", [0, 5, 7])
def test_sync_mult_reports_and_leaves_output(prec, variant, direction, monkeypatch):
    import b200dwf
    monkeypatch.setenv("B200_HOP_VARIANT", str(variant))
    lat, ls = CASE[0], CASE[1]
    ora, op = make()
    w = synth.spinor_field(lat, ls, 5)
    sentinel = synth.spinor_field(lat, ls, 6)
    fw, fv = op.new_field(prec), op.new_field(prec)
    op.convert(fw, w)
    op.convert(fv, sentinel)
    before = op.reverse(fv)
    op.inject_wait_failure(direction)
    with pytest.raises(b200dwf.B200Error, match="gave up waiting"):
        op.mult(fv, fw, "Deo")
    assert np.array_equal(op.reverse(fv), before)      # output untouched, word cleared
    op.inject_wait_failure(-1)
    op.mult(fv, fw, "Deo")
    tol = {0: 1e-13, 1: 1e-5, 2: 1e-2}[prec]
    assert rel(op.reverse(fv), ora.mult("Deo", w)) < tol


def test_async_mult_reports_at_next_sync(monkeypatch):
    import b200dwf
    monkeypatch.setenv("B200_HOP_VARIANT", "3")
    lat, ls = CASE[0], CASE[1]
    ora, op = make()
    w = synth.spinor_field(lat, ls, 7)
    fw, fv = op.new_field(0), op.new_field(0)
    op.convert(fw, w)
    op.set_async(True)
    op.inject_wait_failure(2)
    op.mult_dag(fv, fw, "Deo")                  # queued: no report yet
    with pytest.raises(b200dwf.B200Error, match="gave up waiting"):
        op.check_error()
    op.check_error()                            # cleared by the report
    op.mult(fv, fw, "Deo")
    with pytest.raises(b200dwf.B200Error, match="gave up waiting"):
        op.reverse(fv)
    op.inject_wait_failure(-1)
    op.mult(fv, fw, "Deo")
    op.check_error()
    assert rel(op.reverse(fv), ora.mult("Deo", w)) < 1e-13
    op.set_async(False)


def test_solvers_and_force_report(monkeypatch):
    import b200dwf
    monkeypatch.setenv("B200_HOP_VARIANT", "3")
    lat, ls = CASE[0], CASE[1]
    ora, op = make()
    b = synth.spinor_field(lat, ls, 8)
    fb, fx = op.new_field(0), op.new_field(0)
    op.convert(fb, b)
    op.inject_wait_failure(4)
    with pytest.raises(b200dwf.B200Error, match="gave up waiting"):
        op.cg(fx, fb, 1e-20, 100)
    with pytest.raises(b200dwf.B200Error, match="gave up waiting"):
        op.shiftcg([op.new_field(0), op.new_field(0)], [0.01, 0.1], fb, 1e-20, 100)
    with pytest.raises(b200dwf.B200Error, match="gave up waiting"):
        op.force_udiv(fb)
    op.inject_wait_failure(-1)
    n, diff, rc = op.cg(fx, fb, 1e-20, 3000)
    assert rc == 0
    xr, _, _, _ = ora.cg(b, 1e-20, 3000)
    assert rel(op.reverse(fx), xr) < 1e-8
