"""CPU oracle of the learned gauge-covariant preconditioner (numpy, float64).

TEST INFRASTRUCTURE ONLY: the product never imports this module.  The network
has no counterpart in the reference, so this is a plain restatement of its
definition, written independently of the CUDA kernels (lexical-coordinate
neighbour tables, einsum contractions), and its gradient is itself checked
against central finite differences in the CPU tests.

Definition (per parity p of the even/odd 5D half lattice, fields shaped
(Vh, Ls, C, 3) complex: site, s, channel, color):
  paths 0 identity, 1 s+1, 2 s-1 (zero beyond the walls),
        3 + 2*mu (+mu: ph U_mu(x) v(x+mu)), 4 + 2*mu (-mu: ph U_mu(x-mu)^+ v(x-mu)),
  ph = bc[mu] on the hop that crosses the lattice edge (the operator's
  boundary phases; src/lib_alt_Accel/BridgeOpenACC/src/
  mult_Domainwall_5din_eo_openacc-inc.h applies them the same way).
  layer(W, same, other)(x) = sum_path W[path] (T_path input)(x), W complex
  (11, Cout, Cin) acting on channels only.
  N(r): y1e = L1(r, -), y1o = L1(-, r), y2e = L2(y1e, y1o), y2o = L2(y1o, y1e),
        N(r) = y3e = L3(y2e, y2o).
  loss(r, e) = |A (N(r) - e)|^2 / |r|^2 for a pair with A e = r, A = DdagD
  (the error of N in the residual norm); gradient G = dL/dRe W + i dL/dIm W,
  with dL/dy = 2 A A (N(r) - e) / |r|^2 (A Hermitian).
Site order within a parity: x/2 + Nx/2*(y + Ny*(z + Nz*t)) (index_eo.h of
the reference); spinor fields in the reference host layout
Field(24, Vh, Ls): ri + 2*(color + 3*spin) + 24*(site + Vh*s).
"""
import numpy as np

NPATH = 11


def swap_path(p):
    if p == 0:
        return 0
    if p in (1, 2):
        return 3 - p
    return p + 1 if (p - 3) % 2 == 0 else p - 1


class Geometry:
    def __init__(self, lattice, u_lex, bc=(1, 1, 1, -1)):
        Nx, Ny, Nz, Nt = lattice
        self.L = list(lattice)
        self.vh = Nx * Ny * Nz * Nt // 2
        nx2 = Nx // 2
        site = np.arange(self.vh)
        V = Nx * Ny * Nz * Nt
        u = np.asarray(u_lex, np.float64).reshape(4, V, 3, 3, 2)
        u = u[..., 0] + 1j * u[..., 1]            # [mu][lex][row][col]
        self.nb = {}    # (p, mu, fwd) -> eo index in parity 1-p
        self.ph = {}
        self.U = {}     # (p, mu, fwd) -> link matrices used by the hop
        for p in (0, 1):
            ix2 = site % nx2
            iyzt = site // nx2
            y = iyzt % Ny
            z = (iyzt // Ny) % Nz
            t = iyzt // (Ny * Nz)
            x = 2 * ix2 + ((p + y + z + t) & 1)
            c = [x, y, z, t]
            for mu in range(4):
                for fwd in (True, False):
                    cc = [a.copy() for a in c]
                    step = 1 if fwd else -1
                    cc[mu] = (cc[mu] + step) % self.L[mu]
                    nb = cc[0] // 2 + nx2 * (cc[1] + Ny * (cc[2] + Nz * cc[3]))
                    edge = (c[mu] == self.L[mu] - 1) if fwd else (c[mu] == 0)
                    self.nb[(p, mu, fwd)] = nb
                    self.ph[(p, mu, fwd)] = np.where(edge, float(bc[mu]), 1.0)
                    if fwd:
                        lex = c[0] + Nx * (c[1] + Ny * (c[2] + Nz * c[3]))
                        self.U[(p, mu, fwd)] = u[mu][lex]
                    else:
                        lex = cc[0] + Nx * (cc[1] + Ny * (cc[2] + Nz * cc[3]))
                        self.U[(p, mu, fwd)] = np.conj(np.transpose(u[mu][lex], (0, 2, 1)))


def spinor_to_act(f, vh, ls):
    """Reference host layout Field(24, Vh, Ls) -> (Vh, Ls, 4, 3) complex."""
    a = np.asarray(f, np.float64).reshape(ls, vh, 4, 3, 2)
    return np.transpose(a[..., 0] + 1j * a[..., 1], (1, 0, 2, 3))


def act_to_spinor(a):
    vh, ls = a.shape[:2]
    b = np.transpose(a, (1, 0, 2, 3))
    out = np.stack([b.real, b.imag], axis=-1)
    return out.reshape(ls * vh * 24)


def path_input(geo, p_out, path, same, other):
    if path < 3:
        if same is None:
            return None
        if path == 0:
            return same
        v = np.zeros_like(same)
        if path == 1:
            v[:, :-1] = same[:, 1:]
        else:
            v[:, 1:] = same[:, :-1]
        return v
    if other is None:
        return None
    mu = (path - 3) // 2
    fwd = (path - 3) % 2 == 0
    key = (p_out, mu, fwd)
    v = other[geo.nb[key]]                       # (vh, ls, C, 3)
    t = np.einsum('xij,xsbj->xsbi', geo.U[key], v)
    return t * geo.ph[key][:, None, None, None]


def layer(geo, W, p_out, same, other):
    cout = W.shape[1]
    ref = same if same is not None else other
    out = np.zeros(ref.shape[:2] + (cout, 3), np.complex128)
    for path in range(NPATH):
        u = path_input(geo, p_out, path, same, other)
        if u is not None:
            out += np.einsum('ab,xsbc->xsac', W[path], u)
    return out


def adjoint_weights(W):
    Wa = np.empty((NPATH, W.shape[2], W.shape[1]), np.complex128)
    for path in range(NPATH):
        Wa[swap_path(path)] = np.conj(W[path]).T
    return Wa


def forward(geo, Ws, r):
    W1, W2, W3 = Ws
    y1e = layer(geo, W1, 0, r, None)
    y1o = layer(geo, W1, 1, None, r)
    y2e = layer(geo, W2, 0, y1e, y1o)
    y2o = layer(geo, W2, 1, y1o, y1e)
    y3 = layer(geo, W3, 0, y2e, y2o)
    return y3, (y1e, y1o, y2e, y2o)


def grad_w(geo, p_out, delta, same, other, cin):
    G = np.zeros((NPATH, delta.shape[2], cin), np.complex128)
    for path in range(NPATH):
        u = path_input(geo, p_out, path, same, other)
        if u is not None:
            G[path] = np.einsum('xsac,xsbc->ab', delta, np.conj(u))
    return G


def loss_and_grad(geo, Ws, r, e, A):
    """A: the Hermitian operator DdagD as a function on (Vh, Ls, 4, 3) fields."""
    W1, W2, W3 = Ws
    y3, (y1e, y1o, y2e, y2o) = forward(geo, Ws, r)
    rr = np.vdot(r, r).real
    d = A(y3 - e)
    loss = np.vdot(d, d).real / rr
    d3 = 2.0 * A(d) / rr
    G3 = grad_w(geo, 0, d3, y2e, y2o, W3.shape[2])
    A3 = adjoint_weights(W3)
    d2e = layer(geo, A3, 0, d3, None)
    d2o = layer(geo, A3, 1, None, d3)
    G2 = grad_w(geo, 0, d2e, y1e, y1o, W2.shape[2]) + grad_w(geo, 1, d2o, y1o, y1e, W2.shape[2])
    A2 = adjoint_weights(W2)
    d1e = layer(geo, A2, 0, d2e, d2o)
    d1o = layer(geo, A2, 1, d2o, d2e)
    G1 = grad_w(geo, 0, d1e, r, None, W1.shape[2]) + grad_w(geo, 1, d1o, None, r, W1.shape[2])
    return loss, (G1, G2, G3), y3


def split_weights(flat, hidden):
    """Flat [layer][path][out][in] complex vector -> (W1, W2, W3)."""
    shapes = [(NPATH, hidden, 4), (NPATH, hidden, hidden), (NPATH, 4, hidden)]
    out, o = [], 0
    for sh in shapes:
        n = int(np.prod(sh))
        out.append(np.asarray(flat[o:o + n]).reshape(sh))
        o += n
    return out


def join_weights(Ws):
    return np.concatenate([np.asarray(w).ravel() for w in Ws])
