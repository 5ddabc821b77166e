"""GPU stout smearing (levels) and the smeared-force Jacobian against the
reference corelib's own outputs (golden), plus mult_generator against a
direct restatement."""
import json
import os

import numpy as np
import pytest

from b200dwf import synth

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_stout_levels_and_jacobian_match_reference():
    import b200dwf
    z = np.load(os.path.join(GOLDEN, "smear_stout.npz"))
    m = json.loads(str(z["meta"]))
    lat = m["lattice"]
    u = synth.gauge_field(lat, m["gauge"][1], m["gauge"][0])
    sm = b200dwf.StoutSmear(lat, m["rho"], m["nsmear"])
    sm.set_config(u)
    assert np.array_equal(sm.config(0), u)
    for i in range(1, m["nsmear"] + 1):
        assert rel(sm.config(i), z["smear_%d" % i]) < 1e-14, i
    sigma = np.random.default_rng(m["sigma"]).standard_normal(18 * 4 * int(np.prod(lat)))
    assert rel(sm.jacobian(sigma), z["jacobian"]) < 1e-13


def test_stout_matches_numpy_restatement_on_larger_lattice():
    import b200dwf
    lat = [4, 4, 6, 8]
    u = synth.gauge_field(lat, 5, "near", eps=0.4)
    sm = b200dwf.StoutSmear(lat, 0.12, 3)
    sm.set_config(u)
    ref = u
    for i in range(1, 4):
        ref = synth.stout_smear(ref, lat, 0.12, 1)
        assert rel(sm.config(i), ref) < 1e-13


def _at(m):
    a = 0.5 * (m - np.conj(np.swapaxes(m, -1, -2)))
    tr = np.trace(a, axis1=-2, axis2=-1) / 3.0
    return a - tr[..., None, None] * np.eye(3)


def test_mult_generator():
    import b200dwf
    lat = [4, 4, 4, 4]
    n = 4 * int(np.prod(lat))
    u = synth.gauge_field(lat, 8, "hot")
    f = np.random.default_rng(9).standard_normal(18 * n)
    got = b200dwf.mult_generator(lat, f, u)
    uc = u.reshape(n, 3, 3, 2)
    fc = f.reshape(n, 3, 3, 2)
    um = uc[..., 0] + 1j * uc[..., 1]
    fm = fc[..., 0] + 1j * fc[..., 1]
    ref = -2.0 * _at(um @ fm)
    refr = np.stack([ref.real, ref.imag], -1).reshape(-1)
    assert rel(got, refr) < 1e-14
