"""GPU fermion force (Force_F_Domainwall_eo::force_udiv1 H/Hdag and
force_udiv) against the CPU oracle and the reference's golden vectors."""
import json
import os

import numpy as np
import pytest

from b200dwf import synth

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

CASES = [
    ([4, 4, 4, 4], 4, 0.02, 1.4, 1.5, 0.5, (1, 1, 1, -1), "near"),
    ([4, 4, 4, 8], 8, 0.01, 1.8, 1.0, 0.0, (1, -1, 1, -1), "hot"),
    ([8, 4, 4, 4], 12, 0.04, 1.0, 1.5, 0.5, (1, 1, 1, -1), "near"),
    ([4, 4, 8, 4], 16, 0.01, 1.8, 1.0, 0.0, (1, 1, 1, -1), "hot"),
]


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_force_matches_reference_golden():
    import b200dwf
    z = np.load(os.path.join(GOLDEN, "force_mobius.npz"))
    m = json.loads(str(z["meta"]))
    u = synth.gauge_field(m["lattice"], m["gauge"][1], m["gauge"][0])
    eta = synth.spinor_field(m["lattice"], m["Ls"], m["src"])
    zeta = synth.spinor_field(m["lattice"], m["Ls"], m["src2"])
    op = b200dwf.DomainWall(m["lattice"], m["Ls"], m["mq"], m["M0"], m["b"], m["c"], 1.0, m["bc"])
    op.set_config(u)
    fe, fz = op.new_field(0), op.new_field(0)
    op.convert(fe, eta)
    op.convert(fz, zeta)
    assert rel(op.force_udiv1("H", fz, fe), z["H"]) < 1e-13
    assert rel(op.force_udiv1("Hdag", fe, fz), z["Hdag"]) < 1e-13
    assert rel(op.force_udiv(fe), z["udiv"]) < 1e-13


@pytest.mark.parametrize("ci", range(len(CASES)))
def test_force_matches_oracle(ci):
    import b200dwf
    from oracle.oracle import OracleDWF
    lat, ls, mq, M0, b, c, bc, kind = CASES[ci]
    u = synth.gauge_field(lat, 40 + ci, kind)
    eta = synth.spinor_field(lat, ls, 50 + ci)
    zeta = synth.spinor_field(lat, ls, 60 + ci)
    ora = OracleDWF(lat, ls, mq, M0, b, c, 1.0, bc)
    ora.set_links(u)
    op = b200dwf.DomainWall(lat, ls, mq, M0, b, c, 1.0, bc)
    op.set_config(u)
    fe, fz = op.new_field(0), op.new_field(0)
    op.convert(fe, eta)
    op.convert(fz, zeta)
    assert rel(op.force_udiv1("H", fz, fe), ora.force_udiv1("H", zeta, eta)) < 1e-13
    assert rel(op.force_udiv1("Hdag", fe, fz), ora.force_udiv1("Hdag", eta, zeta)) < 1e-13
    assert rel(op.force_udiv(fe), ora.force_udiv(eta)) < 1e-13
