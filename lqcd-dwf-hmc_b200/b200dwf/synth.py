"""Seeded synthetic lattice inputs: SU(3) gauge links and 5D spinor fields.

Layouts are the host layouts of the reference corelib (Bridge++):

* gauge links, lexical ``Field_G(Nvol, 4)``: index
  ``ri + 2*(col + 3*row) + 18*(site + Nvol*mu)`` with
  ``site = x + Nx*(y + Ny*(z + Nz*t))``
  (reference src/lib/Field/field.h:64-66, src/lib/Field/field_G.h).
* 5D half-lattice spinor ``Field(24, Nvol/2, Ls)``: index
  ``ri + 2*(color + 3*spin) + 24*(site_eo + Nvol2*s)`` with
  ``site_eo = x/2 + Nx/2*(y + Ny*(z + Nz*t))`` on the sites of one parity
  (reference src/lib/Field/index_eo.h:65-105).

All generators use ``numpy.random.default_rng(seed)`` so the same seed gives
the same field on every machine.
"""

import numpy as np


def random_su3_gram_schmidt(rng, n):
    """n Haar-like random SU(3) matrices: Gram-Schmidt on Gaussian complex
    3x3 rows, third row = conj(row1 x row2) so that det = 1 exactly (the
    hot-start recipe of the reference, src/lib/Field/Imp/field_G_imp.cpp:57-73
    "set_random = Gaussian then reunit")."""
    a = rng.standard_normal((n, 2, 3)) + 1j * rng.standard_normal((n, 2, 3))
    r1 = a[:, 0] / np.linalg.norm(a[:, 0], axis=1, keepdims=True)
    r2 = a[:, 1] - np.sum(np.conj(r1) * a[:, 1], axis=1, keepdims=True) * r1
    r2 /= np.linalg.norm(r2, axis=1, keepdims=True)
    r3 = np.conj(np.cross(r1, r2))
    return np.stack([r1, r2, r3], axis=1)


def near_unit_su3(rng, n, eps):
    """n matrices exp(i*eps*H), H Gaussian Hermitian traceless (unit-variance
    generator components)."""
    g = rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))
    h = 0.5 * (g + np.conj(np.swapaxes(g, 1, 2)))
    tr = np.trace(h, axis1=1, axis2=2) / 3.0
    h -= tr[:, None, None] * np.eye(3)
    w, v = np.linalg.eigh(h)
    ph = np.exp(1j * eps * w)
    u = np.einsum('nij,nj,nkj->nik', v, ph, np.conj(v))
    # remove the determinant phase left by rounding (exactly SU(3) up to 1 ulp)
    det = np.linalg.det(u)
    u /= (det ** (1.0 / 3.0))[:, None, None]
    # re-orthonormalise and rebuild the third row so the 12-real compressed
    # form reconstructs the stored matrix to machine precision
    r1 = u[:, 0] / np.linalg.norm(u[:, 0], axis=1, keepdims=True)
    r2 = u[:, 1] - np.sum(np.conj(r1) * u[:, 1], axis=1, keepdims=True) * r1
    r2 /= np.linalg.norm(r2, axis=1, keepdims=True)
    r3 = np.conj(np.cross(r1, r2))
    return np.stack([r1, r2, r3], axis=1)


def gauge_field(lattice, seed, kind="hot", eps=0.3):
    """Lexical links as float64 array in the reference Field_G layout.

    kind = "hot" (Gram-Schmidt SU(3)), "near" (exp(i eps H)) or "unit"."""
    nx, ny, nz, nt = lattice
    nvol = nx * ny * nz * nt
    rng = np.random.default_rng(seed)
    n = 4 * nvol
    if kind == "hot":
        u = random_su3_gram_schmidt(rng, n)
    elif kind == "near":
        u = near_unit_su3(rng, n, eps)
    elif kind == "unit":
        u = np.broadcast_to(np.eye(3, dtype=complex), (n, 3, 3)).copy()
    else:
        raise ValueError(kind)
    # u[mu*nvol + site] -> reals [mu][site][row][col][ri]
    out = np.empty((n, 3, 3, 2))
    out[..., 0] = u.real
    out[..., 1] = u.imag
    return out.reshape(-1)


def spinor_field(lattice, ls, seed):
    """5D half-lattice spinor, float64, Field(24, Nvol/2, Ls) layout, every
    real component N(0,1)."""
    nvol = int(np.prod(lattice))
    rng = np.random.default_rng(seed)
    return rng.standard_normal(24 * (nvol // 2) * ls)


def plaquette(links, lattice):
    """Average plaquette Re tr(U_mu U_nu U_mu^+ U_nu^+)/3 over all planes
    (the reference's normalisation, src/lib/Measurements/Gauge/staple_lex.cpp)."""
    nx, ny, nz, nt = lattice
    nvol = nx * ny * nz * nt
    r = links.reshape(4, nt, nz, ny, nx, 3, 3, 2)
    u = r[..., 0] + 1j * r[..., 1]
    tot = 0.0
    for mu in range(4):
        for nu in range(mu + 1, 4):
            amu = 3 - mu
            anu = 3 - nu
            umu = u[mu]
            unu = u[nu]
            unu_xmu = np.roll(unu, -1, axis=amu)
            umu_xnu = np.roll(umu, -1, axis=anu)
            p = np.einsum('...ij,...jk,...lk,...ml->...im', umu, unu_xmu,
                          np.conj(umu_xnu), np.conj(unu))
            tot += np.trace(p, axis1=-2, axis2=-1).real.sum()
    return tot / (6 * 3 * nvol)


def _as_complex(links, lattice):
    nx, ny, nz, nt = lattice
    r = links.reshape(4, nt, nz, ny, nx, 3, 3, 2)
    return r[..., 0] + 1j * r[..., 1]


def _as_real(u):
    out = np.empty(u.shape + (2,))
    out[..., 0] = u.real
    out[..., 1] = u.imag
    return out.reshape(-1)


def _dag(m):
    return np.conj(np.swapaxes(m, -1, -2))


def staples(u):
    """Sum over nu != mu of the two plaquette staples attached to U_mu(x):
    U_nu(x) U_mu(x+nu) U_nu(x+mu)^+ + U_nu(x-nu)^+ U_mu(x-nu) U_nu(x-nu+mu).
    u: complex [4, t, z, y, x, 3, 3]; array axis of direction mu is 3-mu."""
    c = np.zeros_like(u)
    for mu in range(4):
        amu = 4 - mu
        for nu in range(4):
            if nu == mu:
                continue
            anu = 4 - nu
            unu = u[nu]
            umu_xnu = np.roll(u[mu], -1, axis=anu - 1)
            unu_xmu = np.roll(unu, -1, axis=amu - 1)
            c[mu] += unu @ umu_xnu @ _dag(unu_xmu)
            unu_xmnu = np.roll(unu, 1, axis=anu - 1)
            umu_xmnu = np.roll(u[mu], 1, axis=anu - 1)
            unu_xmnu_pmu = np.roll(unu_xmnu, -1, axis=amu - 1)
            c[mu] += _dag(unu_xmnu) @ umu_xmnu @ unu_xmnu_pmu
    return c


def stout_smear(links, lattice, rho, nsteps):
    """Stout smearing U -> exp(iQ) U with Q = (i/2)(W^+ - W) - (i/6) tr(W^+ - W),
    W = rho C U^+ (Morningstar-Peardon), applied nsteps times to all four
    directions at once (the APE-type uniform-rho stout used by the reference
    Smear_APE + Projection_Stout_SU3).  Returns links in the same layout."""
    u = _as_complex(links, lattice).copy()
    for _ in range(nsteps):
        c = staples(u)
        w = rho * c @ _dag(u)
        a = _dag(w) - w
        tr = np.trace(a, axis1=-2, axis2=-1)[..., None, None] / 3.0
        q = 0.5j * (a - tr * np.eye(3))
        ev, vec = np.linalg.eigh(q)
        expq = vec @ (np.exp(1j * ev)[..., None] * _dag(vec))
        u = expq @ u
    return _as_real(u)


def algebra_field(lattice, seed, scale=1.0):
    """Momentum-like field iP (anti-Hermitian traceless 3x3 per link, the
    matrices Integrator_UpdateU exponentiates), scale * i * H with H Gaussian
    Hermitian traceless; float64 in the Field_G(Nvol, 4) layout."""
    nvol = int(np.prod(lattice))
    rng = np.random.default_rng(seed)
    n = 4 * nvol
    a = rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))
    h = 0.5 * (a + np.conj(np.transpose(a, (0, 2, 1))))
    tr = np.trace(h, axis1=1, axis2=2) / 3.0
    h = h - tr[:, None, None] * np.eye(3)[None]
    ip = 1j * scale * h
    out = np.empty((n, 3, 3, 2))
    out[..., 0] = ip.real
    out[..., 1] = ip.imag
    return out.reshape(-1)

