"""CPU checks of the learned-preconditioner oracle: its gradient against
central finite differences, gauge covariance of the network, and the adjoint
layer used by back-propagation.  (The network has no reference counterpart;
these pin the oracle that the GPU kernels are compared with.)"""
import numpy as np
import pytest

from b200dwf import synth
from oracle import learned_oracle as lo

LAT = [4, 4, 4, 4]
LS = 4
H = 8


def ddagd(u):
    """DdagD of the operator oracle (pinned to the reference) on network fields."""
    from oracle.oracle import OracleDWF
    ora = OracleDWF(LAT, LS, 0.05, 1.8)
    ora.set_links(u)
    vh = int(np.prod(LAT)) // 2
    return lambda a: lo.spinor_to_act(ora.mult("DdagD", lo.act_to_spinor(a)), vh, LS)


def setup(seed=3, kind="hot"):
    u = synth.gauge_field(LAT, 200 + seed, kind)
    geo = lo.Geometry(LAT, u, bc=(1, 1, 1, -1))
    rng = np.random.default_rng(seed)
    shapes = [(11, H, 4), (11, H, H), (11, 4, H)]
    Ws = [0.3 * (rng.standard_normal(s) + 1j * rng.standard_normal(s)) for s in shapes]
    vh = geo.vh
    r = rng.standard_normal((vh, LS, 4, 3)) + 1j * rng.standard_normal((vh, LS, 4, 3))
    e = rng.standard_normal((vh, LS, 4, 3)) + 1j * rng.standard_normal((vh, LS, 4, 3))
    return u, geo, Ws, r, e


def test_gradient_matches_finite_differences():
    u, geo, Ws, r, e = setup()
    A = ddagd(u)
    loss, G, _ = lo.loss_and_grad(geo, Ws, r, e, A)
    rng = np.random.default_rng(11)
    h = 1e-6
    for layer in range(3):
        for _ in range(6):
            idx = tuple(rng.integers(0, n) for n in Ws[layer].shape)
            for part, unit in (("re", 1.0), ("im", 1j)):
                Wp = [w.copy() for w in Ws]
                Wm = [w.copy() for w in Ws]
                Wp[layer][idx] += h * unit
                Wm[layer][idx] -= h * unit
                lp_, _, _ = lo.loss_and_grad(geo, Wp, r, e, A)
                lm_, _, _ = lo.loss_and_grad(geo, Wm, r, e, A)
                fd = (lp_ - lm_) / (2 * h)
                an = G[layer][idx].real if part == "re" else G[layer][idx].imag
                assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (layer, idx, part, fd, an)


def test_network_is_gauge_covariant():
    u, geo, Ws, r, _ = setup(seed=5)
    V = int(np.prod(LAT))
    rng = np.random.default_rng(9)
    om = synth.random_su3_gram_schmidt(rng, V)         # Omega(x), lexical
    uc = u.reshape(4, V, 3, 3, 2)
    uc = uc[..., 0] + 1j * uc[..., 1]
    Nx, Ny, Nz, Nt = LAT
    lex = np.arange(V)
    x = lex % Nx
    y = (lex // Nx) % Ny
    z = (lex // (Nx * Ny)) % Nz
    t = lex // (Nx * Ny * Nz)
    ut = np.empty_like(uc)
    for mu in range(4):
        c = [x.copy(), y.copy(), z.copy(), t.copy()]
        c[mu] = (c[mu] + 1) % LAT[mu]
        fwd = c[0] + Nx * (c[1] + Ny * (c[2] + Nz * c[3]))
        ut[mu] = om @ uc[mu] @ np.conj(np.transpose(om[fwd], (0, 2, 1)))
    u2 = np.stack([ut.real, ut.imag], axis=-1).reshape(-1)
    geo2 = lo.Geometry(LAT, u2, bc=(1, 1, 1, -1))
    # Omega on the even sites of the residual
    nx2 = Nx // 2
    site = np.arange(geo.vh)
    yy = (site // nx2) % Ny
    zz = (site // (nx2 * Ny)) % Nz
    tt = site // (nx2 * Ny * Nz)
    xx = 2 * (site % nx2) + ((yy + zz + tt) & 1)
    om_e = om[xx + Nx * (yy + Ny * (zz + Nz * tt))]
    r2 = np.einsum('xij,xsbj->xsbi', om_e, r)
    y1, _ = lo.forward(geo, Ws, r)
    y2, _ = lo.forward(geo2, Ws, r2)
    expect = np.einsum('xij,xsbj->xsbi', om_e, y1)
    assert np.linalg.norm(y2 - expect) <= 1e-12 * np.linalg.norm(expect)


def test_adjoint_layer():
    _, geo, Ws, _, _ = setup(seed=7)
    rng = np.random.default_rng(1)
    W = Ws[1]
    vh = geo.vh

    def rnd():
        return rng.standard_normal((vh, LS, H, 3)) + 1j * rng.standard_normal((vh, LS, H, 3))

    ue, uo, ve, vo = rnd(), rnd(), rnd(), rnd()
    Le = lo.layer(geo, W, 0, ue, uo)
    Lo = lo.layer(geo, W, 1, uo, ue)
    A = lo.adjoint_weights(W)
    Ae = lo.layer(geo, A, 0, ve, vo)
    Ao = lo.layer(geo, A, 1, vo, ve)
    lhs = np.vdot(ve, Le) + np.vdot(vo, Lo)
    rhs = np.vdot(Ae, ue) + np.vdot(Ao, uo)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("seed", [0, 1])
def test_spinor_layout_round_trip(seed):
    vh = int(np.prod(LAT)) // 2
    f = synth.spinor_field(LAT, LS, seed)
    a = lo.spinor_to_act(f, vh, LS)
    assert a.shape == (vh, LS, 4, 3)
    np.testing.assert_array_equal(lo.act_to_spinor(a), f)
