"""The CPU oracle against golden vectors produced by the reference corelib
itself (tests/golden/make_golden.py runs oracle/_ref/ref_harness)."""
import json
import os

import numpy as np
import pytest

from b200dwf import synth
from oracle.oracle import OracleDWF

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load_case(name):
    z = np.load(os.path.join(GOLDEN, "dwf_%s.npz" % name))
    meta = json.loads(str(z["meta"]))
    u = synth.gauge_field(meta["lattice"], meta["gauge"][1], meta["gauge"][0])
    src = synth.spinor_field(meta["lattice"], meta["Ls"], meta["src"])
    op = OracleDWF(meta["lattice"], meta["Ls"], meta["mq"], meta["M0"], meta["b"], meta["c"],
                   meta["alpha"], meta["bc"])
    op.set_links(u)
    return z, meta, op, src


@pytest.mark.parametrize("name", ["shamir", "mobius_alpha"])
def test_operator_modes_match_reference(name):
    z, meta, op, src = load_case(name)
    for m in meta["modes"]:
        dag = m.startswith("dag_")
        out = op.mult(m[4:] if dag else m, src, dag)
        ref = z[m]
        rel = np.linalg.norm(out - ref) / np.linalg.norm(ref)
        assert rel < 1e-14, (m, rel)


def test_cg_and_multishift_match_reference():
    _, meta_c, op, src = load_case("shamir")
    z = np.load(os.path.join(GOLDEN, "solve_shamir.npz"))
    meta = json.loads(str(z["meta"]))
    x, nconv, diff, rc = op.cg(src, meta["tol"])
    assert rc == 0
    ref_nconv = int(meta["cg_info"].split()[1])
    assert nconv == ref_nconv
    assert np.linalg.norm(x - z["cg_x"]) / np.linalg.norm(z["cg_x"]) < 1e-11
    xs, nconv, diff, rc = op.shiftcg(src, meta["sigma"], meta["tol"])
    assert rc == 0
    # the reference counts multishift iterations from -1 (ashiftsolver_CG-tmpl.h:108)
    assert nconv - 1 == int(meta["shift_info"].split()[1])
    for i in range(len(meta["sigma"])):
        ref = z["shift_%d" % i]
        assert np.linalg.norm(xs[i] - ref) / np.linalg.norm(ref) < 1e-11


def test_plaquette_of_unit_and_random_links():
    lat = [4, 4, 4, 4]
    assert abs(synth.plaquette(synth.gauge_field(lat, 0, "unit"), lat) - 1.0) < 1e-15
    p = synth.plaquette(synth.gauge_field(lat, 1, "near", eps=0.05), lat)
    assert 0.9 < p < 1.0


def test_force_matches_reference():
    z = np.load(os.path.join(GOLDEN, "force_mobius.npz"))
    m = json.loads(str(z["meta"]))
    u = synth.gauge_field(m["lattice"], m["gauge"][1], m["gauge"][0])
    eta = synth.spinor_field(m["lattice"], m["Ls"], m["src"])
    zeta = synth.spinor_field(m["lattice"], m["Ls"], m["src2"])
    op = OracleDWF(m["lattice"], m["Ls"], m["mq"], m["M0"], m["b"], m["c"], m["alpha"], m["bc"])
    op.set_links(u)
    for mode, a, b, key in (("H", zeta, eta, "H"), ("Hdag", eta, zeta, "Hdag")):
        f = op.force_udiv1(mode, a, b)
        assert np.linalg.norm(f - z[key]) / np.linalg.norm(z[key]) < 1e-14
    f = op.force_udiv(eta)
    assert np.linalg.norm(f - z["udiv"]) / np.linalg.norm(z["udiv"]) < 1e-14
