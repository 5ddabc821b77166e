"""The allocation-free norm2 entry point (b200_field_norm2_noalloc).

It serves callers that cannot allocate device memory (inside a graph capture,
under a framework that owns all device memory, on a fully committed GPU); its
scratch is a fixed array inside the library instead of the operator plan's
buffers.  Checked through the C ABI against the plan-based b200_field_norm2 on
two calls in a row.  Collected last so that a failure here never hides the
other tests in a run that stops at the first failure."""
import ctypes

import numpy as np
import pytest

from b200dwf import synth

pytestmark = pytest.mark.gpu


def test_norm2_noalloc_matches_plan_norm2_on_two_calls():
    import b200dwf
    lib = b200dwf.lib()
    lat, ls = [8, 8, 8, 8], 8
    op = b200dwf.DomainWall(lat, ls, 0.01, 1.8)
    vh = op.nvol
    for prec, tol in ((0, 1e-12), (1, 1e-6)):
        fields = []
        for seed in (1, 2):
            f = op.new_field(prec)
            op.convert(f, synth.spinor_field(lat, ls, seed))
            fields.append(f)
        for f in fields:                      # two calls in a row, different data
            expected = op.norm2(f)
            got = ctypes.c_double(-1.0)
            rc = lib.b200_field_norm2_noalloc(prec, f.ptr, vh, ls, ctypes.byref(got), None)
            assert rc == 0, lib.b200_last_error()
            assert abs(got.value - expected) <= tol * expected, (prec, got.value, expected)


def test_norm2_noalloc_rejects_sizes_beyond_its_scratch():
    import b200dwf
    lib = b200dwf.lib()
    got = ctypes.c_double(0.0)
    dummy = ctypes.c_void_p(1)   # never dereferenced: the size check comes first
    rc = lib.b200_field_norm2_noalloc(0, dummy, 1 << 20, 16, ctypes.byref(got), None)
    assert rc == -1
    assert b"exceeds the fixed scratch maximum" in lib.b200_last_error()
