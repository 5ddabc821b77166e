"""GPU parity of the gauge side of the HMC step against the reference
corelib's own outputs (tests/golden/gauge_rect.npz, made by
tests/golden/make_golden.py from Force_G_Rectangle, Action_G_Rectangle and
mult_exp_Field_G): the Iwasaki rectangle force, the gauge Hamiltonian, the
link update exp(alpha iP) U, plus the momentum update and kinetic energy."""
import json
import os

import numpy as np
import pytest

from b200dwf import synth

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def golden():
    z = np.load(os.path.join(HERE, "golden", "gauge_rect.npz"))
    meta = json.loads(str(z["meta"]))
    kind, seed = meta["gauge"]
    u = synth.gauge_field(meta["lattice"], seed, kind)
    ip = synth.algebra_field(meta["lattice"], meta["mom"])
    return meta, u, ip, z


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_rectangle_force_matches_reference():
    import b200dwf
    meta, u, _, z = golden()
    g = b200dwf.GaugeRect(meta["lattice"], meta["beta"], meta["c_plaq"], meta["c_rect"])
    assert rel(g.force(u), z["gforce"]) < 1e-13


def test_gauge_hamiltonian_matches_reference():
    import b200dwf
    meta, u, _, z = golden()
    g = b200dwf.GaugeRect(meta["lattice"], meta["beta"], meta["c_plaq"], meta["c_rect"])
    h = g.action(u)
    assert abs(h - float(z["H"])) <= 1e-12 * abs(float(z["H"]))


def test_link_update_matches_reference():
    import b200dwf
    meta, u, ip, z = golden()
    g = b200dwf.GaugeRect(meta["lattice"], meta["beta"])
    w = g.link_update(u, ip, meta["step"], meta["nprec"])
    assert np.max(np.abs(w - z["update"])) < 1e-14


def test_momentum_update_and_energy():
    import b200dwf
    meta, u, ip, _ = golden()
    g = b200dwf.GaugeRect(meta["lattice"], meta["beta"])
    f = np.random.default_rng(3).standard_normal(ip.size)
    np.testing.assert_allclose(g.momentum_update(ip, f, 0.05), ip + 0.05 * f, rtol=0, atol=1e-15)
    assert g.momentum_energy(ip) == pytest.approx(0.5 * float(ip @ ip), rel=1e-13)


def test_force_is_minus_gradient_of_action():
    """Finite-difference check of the device force against the device action
    along one algebra direction X: dS/dt at t=0 for U -> exp(t X) U."""
    import b200dwf
    lat = [4, 4, 4, 4]
    u = synth.gauge_field(lat, 55, "near", 0.4)
    g = b200dwf.GaugeRect(lat, 2.13)
    X = synth.algebra_field(lat, 56, 1.0)
    h = 1e-5
    sp = g.action(g.link_update(u, X, h, 16))
    sm = g.action(g.link_update(u, X, -h, 16))
    dS = (sp - sm) / (2 * h)
    F = g.force(u)
    # F and X are anti-Hermitian traceless: Re tr(F^+ X) = the sum of products
    # of their reals, and dS/dt = -F.X (what makes H = |iP|^2/2 + S conserved
    # by the reference's UpdateP / UpdateU)
    proj = float(F @ X)
    assert abs(dS + proj) <= 1e-5 * max(1.0, abs(dS)), (dS, proj)


def test_leapfrog_energy_violation_falls_as_step_squared():
    """Pure-gauge molecular dynamics entirely on the device: |dH| of a
    leapfrog trajectory drops by ~4 when the step count doubles (O(eps^2)),
    and reversing the momenta brings the links back."""
    from b200dwf.hmc import GaugeMD
    lat = [4, 4, 4, 4]
    u = synth.gauge_field(lat, 61, "near", 0.3)
    ip = synth.algebra_field(lat, 62, 1.0)
    md = GaugeMD(lat, 2.13)
    dh = [abs(md.trajectory_dh(u, ip, 0.5, n)[0]) for n in (10, 20, 40)]
    r1, r2 = dh[0] / dh[1], dh[1] / dh[2]
    assert 3.3 < r1 < 4.7 and 3.3 < r2 < 4.7, dh
    # reversibility: run forward, flip iP, run back
    U = md.to_device(u)
    P = md.to_device(ip)
    md.leapfrog(P, U, 0.5, 20)
    P.mul_(-1.0)
    md.leapfrog(P, U, 0.5, 20)
    assert float((U.cpu().numpy() - u).__abs__().max()) < 1e-10


def _dwf_md(lat, ls, seed):
    import b200dwf
    from b200dwf.hmc import DwfMD
    u = synth.gauge_field(lat, seed, "near", 0.3)
    op = b200dwf.DomainWall(lat, ls, 0.1, 1.8)
    op.set_config(u)
    psi = op.new_field(b200dwf.F64)
    op.convert(psi, synth.spinor_field(lat, ls, seed + 1))
    return u, op, DwfMD(op, psi, lat, 2.13)


def test_fermion_force_is_minus_gradient_of_fermion_action():
    """The device fermion force mult_generator(force_udiv((DdagD)^-1 psi))
    against a finite difference of S_F = <psi, (DdagD)^-1 psi> along one
    algebra direction, both evaluated with the library's own kernels."""
    lat, ls = [4, 4, 4, 4], 4
    u, op, md = _dwf_md(lat, ls, 71)
    X = synth.algebra_field(lat, 72, 1.0)
    h = 1e-5
    up = md.to_device(u)
    md.update_u(md.to_device(X), up, h)
    um = md.to_device(u)
    md.update_u(md.to_device(X), um, -h)
    dS = (md.fermion_action(up) - md.fermion_action(um)) / (2 * h)
    F = md.fermion_force(md.to_device(u)).cpu().numpy()
    proj = float(F @ X)
    assert abs(dS + proj) <= 1e-5 * max(1.0, abs(dS)), (dS, proj)


def test_dwf_hmc_energy_violation_falls_as_step_squared():
    """Two-flavour domain-wall + Iwasaki molecular dynamics with every
    operator, solver, force and update on the device: |dH| of a leapfrog
    trajectory falls ~4x per doubling of the step count."""
    lat, ls = [4, 4, 4, 4], 4
    u, op, md = _dwf_md(lat, ls, 81)
    ip = synth.algebra_field(lat, 82, 1.0)
    dh = [abs(md.trajectory_dh(u, ip, 0.25, n)[0]) for n in (4, 8, 16)]
    r1, r2 = dh[0] / dh[1], dh[1] / dh[2]
    assert 3.0 < r1 < 5.0 and 3.0 < r2 < 5.0, dh


def test_trajectory_solvers_agree():
    """The same trajectory with FP64 CG, mixed-precision Richardson (f16
    inner) and the learned flexible CG as the fermion solver: |dH| agrees to
    the solver tolerance and the end links agree."""
    import b200dwf
    from b200dwf.hmc import DwfMD
    lat, ls = [4, 4, 4, 8], 8
    u = synth.gauge_field(lat, 91, "near", 0.3)
    ip = synth.algebra_field(lat, 92, 1.0)
    out = {}
    for solver in ("cg", "mixed", "learned"):
        op = b200dwf.DomainWall(lat, ls, 0.05, 1.8)
        op.set_config(u)
        psi = op.new_field(b200dwf.F64)
        op.convert(psi, synth.spinor_field(lat, ls, 93))
        lp = b200dwf.LearnedPrecond(op, hidden=8, seed=3) if solver == "learned" else None
        md = DwfMD(op, psi, lat, 2.13, tol2=1e-20, solver=solver, lp=lp)
        dh, uf = md.trajectory_dh(u, ip, 0.2, 4)
        out[solver] = (dh, uf.cpu().numpy())
    for s in ("mixed", "learned"):
        assert abs(out[s][0] - out["cg"][0]) < 1e-6 * max(1.0, abs(out["cg"][0])), (s, out[s][0], out["cg"][0])
        assert np.max(np.abs(out[s][1] - out["cg"][1])) < 1e-8, s


def _rhmc_md(lat, ls, seed, mass_l=0.1, mass_s=0.2):
    import b200dwf
    from b200dwf.hmc import GaugeMD, TwoFlavour, Rational
    from b200dwf.rational import inv_sqrt_partial_fractions
    u = synth.gauge_field(lat, seed, "near", 0.3)
    opl = b200dwf.DomainWall(lat, ls, mass_l, 1.8)
    ops = b200dwf.DomainWall(lat, ls, mass_s, 1.8)
    for op in (opl, ops):
        op.set_config(u)
    psi = opl.new_field(b200dwf.F64)
    opl.convert(psi, synth.spinor_field(lat, ls, seed + 1))
    phi = ops.new_field(b200dwf.F64)
    ops.convert(phi, synth.spinor_field(lat, ls, seed + 2))
    a0, b, c = inv_sqrt_partial_fractions(1e-4, 10.0, 16)
    rat = Rational(ops, phi, a0, b, c)
    md = GaugeMD(lat, 2.13, fermions=[TwoFlavour(opl, psi), rat])
    return u, md, rat


def test_rational_force_is_minus_gradient_of_rational_action():
    lat, ls = [4, 4, 4, 4], 4
    u, md, rat = _rhmc_md(lat, ls, 101)
    X = synth.algebra_field(lat, 102, 1.0)
    h = 1e-5
    up = md.to_device(u)
    md.update_u(md.to_device(X), up, h)
    um = md.to_device(u)
    md.update_u(md.to_device(X), um, -h)
    dS = (rat.action(md, up) - rat.action(md, um)) / (2 * h)
    F = md.fermion_force(md.to_device(u), rat).cpu().numpy()
    proj = float(F @ X)
    assert abs(dS + proj) <= 1e-5 * max(1.0, abs(dS)), (dS, proj)


def test_two_plus_one_flavour_energy_violation_falls_as_step_squared():
    """Iwasaki + two-flavour DWF (light) + RHMC one-flavour DWF (strange, 16
    poles, multishift CG) on the device: |dH| falls ~4x per step doubling."""
    lat, ls = [4, 4, 4, 4], 4
    u, md, _ = _rhmc_md(lat, ls, 111)
    ip = synth.algebra_field(lat, 112, 1.0)
    dh = [abs(md.trajectory_dh(u, ip, 0.25, n)[0]) for n in (4, 8, 16)]
    r1, r2 = dh[0] / dh[1], dh[1] / dh[2]
    assert 3.0 < r1 < 5.0 and 3.0 < r2 < 5.0, dh
