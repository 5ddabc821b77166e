"""The allocation-free norm2 entry point (b200_field_norm2_noalloc).

It serves callers that cannot allocate device memory: code under a host
framework that owns all device memory through its own pool (an allocation
behind the pool's back can fail or exhaust what the pool planned for), or a
caller on a GPU already committed to resident fields.  Its scratch is a fixed
array inside the library instead of the operator plan's buffers.

Checked through the C ABI, on two calls in a row with different data, in every
storage layout (f64, f32, and f16/bf16 with their per-(site, s) scale column),
against the plan-based b200_field_norm2 on the same field and against numpy on
the field read back to the host.  Collected last so that a failure here never
hides the other tests in a run that stops at the first failure."""
import ctypes

import numpy as np
import pytest

from b200dwf import synth

pytestmark = pytest.mark.gpu

# (storage precision, tolerance against the plan's norm2, tolerance against
# numpy on the decoded field).  The two device paths run the same per-block
# arithmetic; numpy sums the decoded values in another order.
CASES = ((0, 1e-12, 1e-12), (1, 1e-6, 1e-6), (2, 1e-6, 1e-5), (3, 1e-6, 1e-5))


@pytest.mark.parametrize("prec,tol_plan,tol_np", CASES)
def test_norm2_noalloc_matches_plan_norm2_on_two_calls(prec, tol_plan, tol_np):
    import b200dwf
    lib = b200dwf.lib()
    lat, ls = [8, 8, 8, 8], 8
    op = b200dwf.DomainWall(lat, ls, 0.01, 1.8)
    vh = op.nvol
    fields = []
    for seed in (1, 2):
        f = op.new_field(prec)
        op.convert(f, synth.spinor_field(lat, ls, seed) * (1.0 + seed))
        fields.append(f)
    for f in fields:                      # two calls in a row, different data
        expected = op.norm2(f)
        decoded = op.reverse(f)
        ref_np = float(np.dot(decoded, decoded))
        got = ctypes.c_double(-1.0)
        rc = lib.b200_field_norm2_noalloc(prec, f.ptr, vh, ls, ctypes.byref(got), None)
        assert rc == 0, lib.b200_last_error()
        assert abs(got.value - expected) <= tol_plan * expected, (prec, got.value, expected)
        assert abs(got.value - ref_np) <= tol_np * ref_np, (prec, got.value, ref_np)


def test_norm2_noalloc_rejects_sizes_beyond_its_scratch():
    import b200dwf
    lib = b200dwf.lib()
    got = ctypes.c_double(0.0)
    dummy = ctypes.c_void_p(1)   # never dereferenced: the size check comes first
    rc = lib.b200_field_norm2_noalloc(0, dummy, 1 << 20, 16, ctypes.byref(got), None)
    assert rc == -1
    assert b"exceeds the fixed scratch maximum" in lib.b200_last_error()
