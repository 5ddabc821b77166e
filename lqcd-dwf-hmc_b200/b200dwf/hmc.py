"""Molecular-dynamics integration on the device.

Host-side driver in the shape of the reference's HMC_Leapfrog / Integrator
chain (src/lib/HMC/hmc_Leapfrog.cpp, integrator_UpdateP.cpp:44-66,
integrator_UpdateU.cpp:79-86, hmc_General.cpp:305-346): every field stays on
the GPU; each step is the library's force, momentum-update and link-update
kernels, and the fermion actions' solves and forces.  Actions:

* the Iwasaki / rectangle gauge action (always present);
* TwoFlavour: S = Re <psi, (DdagD)^-1 psi> (Action_F_Standard_eo,
  src/lib/Action/Fermion/action_F_Standard_eo.cpp:47-150), force
  mult_generator(force_udiv(eta)), eta = (DdagD)^-1 psi (Force::force_core,
  src/lib/Force/Fermion/force_F.cpp:67-79);
* Rational: S = Re <phi, R(DdagD) phi>, R(x) = a0 + sum b_i/(x + c_i) ~ x^-1/2
  (Action_F_Rational, src/lib/Action/Fermion/action_F_Rational.cpp:76-130),
  force sum_i b_i force_udiv(x_i) with x_i = (DdagD + c_i)^-1 phi from one
  multishift solve (Force_F_Rational::force_udiv_impl,
  src/lib/Force/Fermion/force_F_Rational.cpp:142-178).

The leapfrog trajectory conserves H = |iP|^2/2 + sum S up to O(eps^2).
"""
import ctypes

import numpy as np

from . import check, lib


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


class TwoFlavour:
    """Two-flavour even/odd domain-wall pseudofermion action."""

    def __init__(self, op, psi, tol2=1e-20, solver="cg", inner_prec=None, lp=None):
        from . import Field, F64, F16
        self.op, self.psi, self.tol2 = op, psi, tol2
        self.eta = Field(op, F64)
        self.solver = solver                  # "cg", "mixed" (Richardson) or "learned" (flexible CG)
        self.inner_prec = F16 if inner_prec is None else inner_prec
        self.lp = lp
        self.iterations = 0

    def solve(self):
        """eta = (DdagD)^-1 psi with the chosen solver (Fprop 'DdagD_even')."""
        if self.solver == "cg":
            n, _, rc = self.op.cg(self.eta, self.psi, self.tol2, 100000)
        elif self.solver == "mixed":
            _, n, _, rc = self.op.richardson(self.eta, self.psi, self.inner_prec, self.tol2, 200,
                                             1e-4 if self.inner_prec != 1 else 1e-8, 100000)
        elif self.solver == "learned":
            n0, n1, _, rc = self.op.fcg(self.eta, self.psi, self.lp, self.tol2, 100000, 2)
            n = n0 + n1
        else:
            raise ValueError(self.solver)
        if rc != 0:
            raise RuntimeError("fermion solve did not converge (%s)" % self.solver)
        self.iterations += n

    def action(self, md, u):
        md.set_links(self.op, u)
        self.solve()
        return self.op.dot(self.psi, self.eta)

    def force_udiv(self, md, u, out):
        md.set_links(self.op, u)
        self.solve()
        check(lib().b200_dwf_force_udiv(self.op.handle, _p(out), self.eta.ptr, None))


class Rational:
    """One-flavour rational (RHMC) pseudofermion action R(DdagD) ~ DdagD^-1/2."""

    def __init__(self, op, phi, a0, b, c, tol2=1e-20):
        from . import Field, F64
        self.op, self.phi, self.tol2 = op, phi, tol2
        self.a0 = float(a0)
        self.b = [float(v) for v in b]
        self.c = [float(v) for v in c]
        self.xs = [Field(op, F64) for _ in self.c]
        self.iterations = 0

    def solve(self):
        n, _, rc = self.op.shiftcg(self.xs, self.c, self.phi, self.tol2, 100000)
        if rc != 0:
            raise RuntimeError("multishift solve did not converge")
        self.iterations += n

    def action(self, md, u):
        md.set_links(self.op, u)
        self.solve()
        s = self.a0 * self.op.norm2(self.phi)
        for bi, x in zip(self.b, self.xs):
            s += bi * self.op.dot(self.phi, x)
        return s

    def force_udiv(self, md, u, out):
        import torch
        md.set_links(self.op, u)
        self.solve()
        tmp = torch.empty_like(out)
        out.zero_()
        for bi, x in zip(self.b, self.xs):
            check(lib().b200_dwf_force_udiv(self.op.handle, _p(tmp), x.ptr, None))
            out.add_(tmp, alpha=bi)


class GaugeMD:
    """Leapfrog MD of the Iwasaki gauge action plus optional fermion actions."""

    def __init__(self, lattice, beta, c_plaq=3.648, c_rect=-0.331, nprec=8, fermions=()):
        import torch
        self.lattice = list(lattice)
        self.nvol = int(np.prod(lattice))
        self.beta, self.c_plaq, self.c_rect, self.nprec = beta, c_plaq, c_rect, nprec
        self._L = (ctypes.c_int * 4)(*lattice)
        self.fermions = list(fermions)
        n = 18 * 4 * self.nvol
        self.force_buf = torch.empty(n, dtype=torch.float64, device="cuda")
        self.fbuf = torch.empty(n, dtype=torch.float64, device="cuda")

    def to_device(self, a):
        import torch
        return torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()

    @staticmethod
    def set_links(op, u):
        check(lib().b200_dwf_set_config_device(op.handle, _p(u), None))

    def force(self, u):
        """Gauge force (Force_G_Rectangle) into force_buf."""
        check(lib().b200_gauge_force_rect(self._L, self.beta, self.c_plaq, self.c_rect,
                                          _p(self.force_buf), _p(u), None))
        return self.force_buf

    def fermion_force(self, u, action=None):
        """Sum of the fermion forces (or one action's), lexical Field_G layout."""
        import torch
        acts = self.fermions if action is None else [action]
        total = torch.zeros_like(self.fbuf)
        for a in acts:
            a.force_udiv(self, u, self.fbuf)
            total.add_(self.fbuf)
        # mult_generator is linear: applied once to the summed force_udiv
        check(lib().b200_force_mult_generator(self._L, _p(total), _p(u), None))
        return total

    def update_p(self, ip, u, eps):
        """Integrator_UpdateP: iP += eps * F(U) for every action."""
        fg = self.force(u)
        check(lib().b200_momentum_update(self._L, eps, _p(fg), _p(ip), None))
        if self.fermions:
            ff = self.fermion_force(u)
            check(lib().b200_momentum_update(self._L, eps, _p(ff), _p(ip), None))

    def update_u(self, ip, u, eps):
        """Integrator_UpdateU: U <- exp(eps iP) U."""
        check(lib().b200_link_update(self._L, eps, _p(ip), _p(u), self.nprec, None))

    def gauge_hamiltonian(self, ip, u):
        hp = ctypes.c_double()
        hu = ctypes.c_double()
        check(lib().b200_momentum_energy(self._L, _p(ip), ctypes.byref(hp), None))
        check(lib().b200_gauge_action_rect(self._L, self.beta, self.c_plaq, self.c_rect,
                                           _p(u), ctypes.byref(hu), None))
        return hp.value + hu.value

    def hamiltonian(self, ip, u):
        return self.gauge_hamiltonian(ip, u) + sum(a.action(self, u) for a in self.fermions)

    def leapfrog(self, ip, u, tau, nsteps):
        """Leapfrog trajectory of length tau in nsteps steps (in place)."""
        eps = tau / nsteps
        self.update_p(ip, u, 0.5 * eps)
        for k in range(nsteps):
            self.update_u(ip, u, eps)
            self.update_p(ip, u, eps if k < nsteps - 1 else 0.5 * eps)

    def trajectory_dh(self, u_lex, ip_lex, tau, nsteps):
        """H(end) - H(start) of one leapfrog trajectory from (u, iP)."""
        u = self.to_device(u_lex)
        ip = self.to_device(ip_lex)
        h0 = self.hamiltonian(ip, u)
        self.leapfrog(ip, u, tau, nsteps)
        return self.hamiltonian(ip, u) - h0, u

    @property
    def iterations(self):
        return sum(a.iterations for a in self.fermions)

    @iterations.setter
    def iterations(self, v):
        for a in self.fermions:
            a.iterations = v


class DwfMD(GaugeMD):
    """Iwasaki gauge action + one two-flavour domain-wall action."""

    def __init__(self, op, psi, lattice, beta, c_plaq=3.648, c_rect=-0.331, nprec=8, tol2=1e-24,
                 solver="cg", inner_prec=None, lp=None):
        self.two = TwoFlavour(op, psi, tol2, solver, inner_prec, lp)
        super().__init__(lattice, beta, c_plaq, c_rect, nprec, fermions=[self.two])
        self.op, self.psi = op, psi

    def fermion_action(self, u):
        return self.two.action(self, u)
