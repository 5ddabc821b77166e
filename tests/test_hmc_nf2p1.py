"""The reference's 2+1-flavour HMC (benchmark_hmc_dwf_corelib/hmc_dwf_eo.cpp:
rational-ratio strange quark over Pauli-Villars, two Hasenbusch ratios for the
light pair, rectangle gauge action, stout-smeared fermion links, nested
Omelyan [2,1,3]) on the device, against one trajectory of the reference
corelib itself (tests/golden/traj_nf2p1.npz: the momenta and pseudofermion
noise its M-series generator handed out, both Hamiltonians, the per-action
values, the end links and momenta).

CPU tests pin the golden's bookkeeping and the rational tables; GPU tests
run the device trajectory from the recorded noise and check every force
against a finite difference of its own action."""
import ctypes
import json
import os

import numpy as np
import pytest

from b200dwf import synth

HERE = os.path.dirname(os.path.abspath(__file__))


def golden():
    z = np.load(os.path.join(HERE, "golden", "traj_nf2p1.npz"))
    meta = json.loads(str(z["meta"]))
    kind, seed = meta["gauge"]
    u = synth.gauge_field(meta["lattice"], seed, kind)
    return meta, u, z


# ------------------------------------------------------------------ CPU

def test_golden_hamiltonian_bookkeeping():
    """H_total(init) of the reference = |iP|^2/2 + sum of the three
    pseudofermion heatbath values |xi_k|^2 + the gauge action at the start:
    the recorded fields are exactly what its langevin step consumed."""
    meta, u, z = golden()
    h0 = 0.5 * float(z["mom"] @ z["mom"])
    h0 += sum(float(z["xi_%d" % k] @ z["xi_%d" % k]) for k in range(3))
    h0 += float(z["h_start"][3])
    assert h0 == pytest.approx(float(z["H0"][0]), rel=1e-13)
    assert float(z["dH"][0]) == pytest.approx(float(z["H1"][0] - z["H0"][0]), abs=1e-9)
    # each pseudofermion action's calcH at the start reproduces its heatbath
    # value up to the rational and solver tolerances
    for k in range(3):
        xi2 = float(z["xi_%d" % k] @ z["xi_%d" % k])
        assert float(z["h_start"][k]) == pytest.approx(xi2, rel=1e-4)


def test_rational_tables_state_their_error():
    from b200dwf.rational import TABLE_DIR, max_rel_error, read_table
    names = sorted(os.listdir(TABLE_DIR))
    assert len(names) == 9
    for name in names:
        ne, de, lo, hi, err, a0, b, c = read_table(os.path.join(TABLE_DIR, name))
        assert err < 3e-6
        assert max_rel_error(a0, b, c, lo, hi, ne / de) <= 1.01 * err
        assert np.all(c > 0)


def test_rational_table_roundtrip(tmp_path):
    from b200dwf.rational import Rational, table_name, write_table, read_table
    r = Rational(16, -1, 2, 1e-2, 3.16227766)
    path = tmp_path / table_name(-1, 2, 16, r.lo, r.hi)
    assert path.name == "parameter_rational.1_2inv_16_0.00010000_010.000"
    write_table(str(path), -1, 2, r.lo, r.hi, r.a0, r.b, r.c, r.err)
    ne, de, lo, hi, err, a0, b, c = read_table(str(path))
    assert (ne, de) == (-1, 2) and a0 == r.a0
    np.testing.assert_array_equal(b, r.b)
    np.testing.assert_array_equal(c, r.c)
    x = np.array([1e-3, 0.1, 5.0])
    np.testing.assert_allclose(r(x), x ** -0.5, rtol=1e-9)


# ------------------------------------------------------------------ GPU

def _hmc_from_meta(meta, solvers=None):
    from b200dwf.hmc import build_dwf_nf2p1
    return build_dwf_nf2p1(
        meta["lattice"], meta["Ls"], meta["M0"],
        dict(l=meta["mq_l"], h=meta["mq_h"], s=meta["mq_s"], pv=meta["mq_pv"]),
        meta["beta"], meta["c_plaq"], meta["c_rect"], meta["rho"], meta["nsmear"],
        meta["nstep"], meta["level"], meta["tau"], meta["lambda_"], meta["nprec"],
        meta["np_md"], meta["np_h"], (meta["rat_lo"], meta["rat_hi"]),
        meta["tol_md"], meta["tol_h"], solvers=solvers, bc=meta["bc"],
        integrator=meta["integrator"])


@pytest.mark.gpu
def test_trajectory_matches_reference():
    """One device trajectory driven by the reference's recorded momenta and
    noise (solvers at |r|^2/|b|^2 < 1e-24 on both sides): H_total(init),
    every action's Hamiltonian and force at the start, H(diff) and the end
    links and momenta against what the reference produced.  Measured on a
    B200: H0 to 2e-15, actions to 2e-13, forces to 2e-10, |dH - dH_ref|
    8e-9 (dH = 44.5), end links to 4e-11, end momenta to 1.3e-10."""
    import torch
    from b200dwf.hmc import HostNoise
    meta, u, z = golden()
    hmc = _hmc_from_meta(meta)
    ud = torch.from_numpy(u.copy()).cuda()
    hmc.set_config(ud)
    ip = torch.zeros_like(ud)
    noise = HostNoise(z["mom"], [z["xi_0"], z["xi_1"], z["xi_2"]])
    h0, parts0 = hmc.langevin(ip, noise)
    assert h0 == pytest.approx(float(z["H0"][0]), rel=1e-13)
    hs = [a.calcH() for a in hmc.actions]
    np.testing.assert_allclose(hs, z["h_start"], rtol=1e-11)
    # every action's force at the start links (Action::force after
    # mult_generator, smeared-force Jacobian included)
    F = torch.zeros_like(ud)
    for i, a in enumerate(hmc.actions):
        hmc.level_force([a], ud, F)
        ref = z["force_%d" % i]
        err = np.linalg.norm(F.cpu().numpy() - ref) / np.linalg.norm(ref)
        assert err < 2e-9, (i, err)
    hmc.integrator.evolve(meta["tau"], ip, ud)
    h1, parts1 = hmc.calc_hamiltonian(ip)
    dh = h1 - h0
    np.testing.assert_allclose(parts1[1:], z["h_end"], rtol=1e-10)
    assert abs(dh - float(z["dH"][0])) < 1e-7, (dh, float(z["dH"][0]))
    assert np.max(np.abs(ud.cpu().numpy() - z["u_end"])) < 1e-9
    assert np.max(np.abs(ip.cpu().numpy() - z["mom_end"])) < 1e-8
    # the nested Omelyan [2,1,3] with cached forces evaluates 5 / 9 / 49
    # forces on levels 0 / 1 / 2
    assert hmc.force_evaluations == {0: 5, 1: 9, 2: 49}


def _small_hmc(seed, **kw):
    import torch
    from b200dwf.hmc import build_dwf_nf2p1, DeviceNoise
    lat, ls = [4, 4, 4, 4], 4
    u = synth.gauge_field(lat, seed, "near", 0.3)
    args = dict(np_md=16, np_h=16, tol2_md=1e-24, tol2_h=1e-24, tau=0.2)
    args.update(kw)
    hmc = build_dwf_nf2p1(lat, ls, 1.8, dict(l=0.1, h=0.3, s=0.2, pv=1.0), 2.13, **args)
    ud = torch.from_numpy(u).cuda()
    hmc.set_config(ud)
    ip = torch.zeros_like(ud)
    hmc.langevin(ip, DeviceNoise(seed + 1))
    return hmc, u, ud, ip


def _shifted(u, X, h):
    import torch
    from b200dwf import lib, check
    L = (ctypes.c_int * 4)(4, 4, 4, 4)
    w = torch.from_numpy(u.copy()).cuda()
    x = torch.from_numpy(X).cuda()
    check(lib().b200_link_update(L, h, ctypes.c_void_p(x.data_ptr()),
                                 ctypes.c_void_p(w.data_ptr()), 16, None))
    return w


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["nf1", "nf2", "nf2p"])
def test_smeared_fermion_force_is_minus_gradient(name):
    """Each fermion action's force (force_udiv on the smeared links, the
    stout Jacobian back to the thin links, mult_generator) against a finite
    difference of its own Hamiltonian along one algebra direction."""
    import torch
    hmc, u, ud, _ = _small_hmc(121)
    act = hmc.fermions[name]
    X = synth.algebra_field([4, 4, 4, 4], 122, 1.0)
    h = 1e-5
    s = []
    for sign in (1.0, -1.0):
        hmc.set_config(_shifted(u, X, sign * h))
        s.append(act.calcH())
    dS = (s[0] - s[1]) / (2 * h)
    hmc.set_config(ud)
    F = torch.zeros_like(ud)
    hmc.level_force([act], ud, F)
    proj = float(F.cpu().numpy() @ X)
    assert abs(dS + proj) <= 2e-5 * max(1.0, abs(dS)), (name, dS, proj)


@pytest.mark.gpu
def test_streamed_rational_force_matches_paired():
    """The rational ratio's force with one pool of np_md solution fields
    (numerator cross terms from the combined sources s*phi +- v/s) equals
    the paired form (eta1_i and zeta_i side by side, balanced per pole) to
    the multishift tolerance, and holds np_md fewer fields."""
    import torch
    F = {}
    for pool in ("paired", "streamed"):
        hmc, u, ud, _ = _small_hmc(151, rational_force_pool=pool)
        act = hmc.fermions["nf1"]
        out = torch.zeros_like(ud)
        hmc.level_force([act], ud, out)
        F[pool] = (out.cpu().numpy(), len(act.pool))
    err = np.linalg.norm(F["streamed"][0] - F["paired"][0]) / np.linalg.norm(F["paired"][0])
    assert err < 1e-9, err
    assert F["paired"][1] == 32 and F["streamed"][1] == 16


@pytest.mark.gpu
def test_nested_omelyan_energy_violation_falls_as_step_squared():
    """The full action set under the nested Omelyan integrator: |dH| falls
    ~4x per doubling of the outer step count (inner levels nested inside),
    and reversing the momenta retraces the trajectory."""
    import torch
    dh = []
    for n in (2, 4, 8):
        hmc, u, ud, ip = _small_hmc(131, nstep=(n, 1, 3), tau=0.5)
        h0, _ = hmc.calc_hamiltonian(ip)
        hmc.integrator.evolve(0.5, ip, ud)
        h1, _ = hmc.calc_hamiltonian(ip)
        dh.append(abs(h1 - h0))
    r1, r2 = dh[0] / dh[1], dh[1] / dh[2]
    assert 3.0 < r1 < 5.5 and 3.0 < r2 < 5.5, dh
    ip.mul_(-1.0)
    hmc.integrator.evolve(0.5, ip, ud)
    assert float((ud.cpu() - torch.from_numpy(u)).abs().max()) < 1e-9


@pytest.mark.gpu
def test_mixed_precision_solvers_reproduce_the_fp64_trajectory():
    """Light and Hasenbusch solves by mixed-precision Richardson (FP16
    inner) give the FP64 trajectory's dH and end links to the solver
    tolerance."""
    from b200dwf.hmc import Solver
    out = {}
    for kind in ("cg", "mixed"):
        sv = {k: Solver(kind, 1e-24) for k in ("l_md", "h_md", "l_h", "h_h", "pv_h")}
        hmc, u, ud, ip = _small_hmc(141, solvers=sv)
        h0, _ = hmc.calc_hamiltonian(ip)
        hmc.integrator.evolve(0.2, ip, ud)
        h1, _ = hmc.calc_hamiltonian(ip)
        out[kind] = (h1 - h0, ud.cpu().numpy())
    assert abs(out["mixed"][0] - out["cg"][0]) < 1e-8
    assert np.max(np.abs(out["mixed"][1] - out["cg"][1])) < 1e-10


@pytest.mark.gpu
def test_chronological_guess_keeps_the_trajectory_and_saves_iterations():
    """The MD solves of the ratio actions starting from the previous solution
    (use_initial_guess, CG and Richardson): the same dH and end links to the
    solver tolerance, and fewer solver iterations."""
    from b200dwf.hmc import Solver
    out = {}
    for chrono in (False, True):
        for kind in ("cg", "mixed"):
            sv = {k: Solver(kind, 1e-24, chrono=chrono) for k in ("l_md", "h_md", "l_h", "h_h", "pv_h")}
            hmc, u, ud, ip = _small_hmc(151, solvers=sv)
            h0, _ = hmc.calc_hamiltonian(ip)
            hmc.integrator.evolve(0.2, ip, ud)
            h1, _ = hmc.calc_hamiltonian(ip)
            its = sum(sv[k].iterations for k in ("l_md", "h_md"))
            out[(chrono, kind)] = (h1 - h0, ud.cpu().numpy(), its)
    for kind in ("cg", "mixed"):
        a, b = out[(False, kind)], out[(True, kind)]
        assert abs(a[0] - b[0]) < 1e-8, kind
        assert np.max(np.abs(a[1] - b[1])) < 1e-10, kind
        assert b[2] < a[2], (kind, a[2], b[2])


@pytest.mark.gpu
def test_minimal_residual_guess_keeps_the_trajectory():
    """MD solves starting from the minimal residual extrapolation of the last
    4 solutions (chrono_depth 4) against the previous solution alone
    (chrono_depth 1): the same dH and end links to the solver tolerance, and
    no more iterations (the extrapolation's error is minimal in the DdagD
    norm over a span that holds the previous solution)."""
    from b200dwf.hmc import Solver
    out = {}
    for depth in (1, 4):
        sv = {k: Solver("mixed", 1e-24, chrono=True, chrono_depth=depth)
              for k in ("l_md", "h_md", "l_h", "h_h", "pv_h")}
        hmc, u, ud, ip = _small_hmc(161, solvers=sv, nstep=(4, 1, 3))
        h0, _ = hmc.calc_hamiltonian(ip)
        hmc.integrator.evolve(0.2, ip, ud)
        h1, _ = hmc.calc_hamiltonian(ip)
        out[depth] = (h1 - h0, ud.cpu().numpy(), sum(sv[k].iterations for k in ("l_md", "h_md")))
    assert abs(out[4][0] - out[1][0]) < 1e-8
    assert np.max(np.abs(out[4][1] - out[1][1])) < 1e-10
    assert out[4][2] <= out[1][2], (out[1][2], out[4][2])


@pytest.mark.gpu
def test_minimal_residual_guess_reproduces_a_repeated_solve():
    """Two solutions of one system in the history: the extrapolation alone
    is the solution (the degenerate direction of the nearly singular 2x2
    system is dropped), so the third solve, from a zeroed x, needs only the
    iterations of the second."""
    import b200dwf
    from b200dwf.hmc import Solver
    lat, ls = [4, 4, 4, 8], 8
    op = b200dwf.DomainWall(lat, ls, 0.05, 1.8)
    op.set_config(synth.gauge_field(lat, 171, "near", 0.3))
    b = op.new_field()
    op.convert(b, synth.spinor_field(lat, ls, 172))
    x = op.new_field()
    s = Solver("cg", 1e-24, chrono=True, chrono_depth=3)
    n1 = s.solve(op, x, b)
    n2 = s.solve(op, x, b, guess=True)
    x.zero()                                   # the guess must come from the history
    n3 = s.solve(op, x, b, guess=True)
    # a solution to |r| < 1e-12 recursively can sit a little above it in the
    # true residual the restarted solve checks: a few iterations at most
    assert n1 > 50 and n2 <= 5 and n3 <= 5, (n1, n2, n3)
