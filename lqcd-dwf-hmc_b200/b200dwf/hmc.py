"""Molecular-dynamics integration of the gauge field on the device.

Host-side driver in the shape of the reference's HMC_Leapfrog / Integrator
chain (src/lib/HMC/hmc_Leapfrog.cpp, integrator_UpdateP.cpp:44-66,
integrator_UpdateU.cpp:79-86, hmc_General.cpp:305-346): every field stays on
the GPU; each step is the library's force, momentum-update and link-update
kernels.  The action here is the Iwasaki / rectangle gauge action; the
leapfrog trajectory conserves H = |iP|^2/2 + S_G(U) up to O(eps^2), so the
energy violation |dH| falls by four when the step count doubles.
"""
import ctypes

import numpy as np

from . import check, lib


class GaugeMD:
    def __init__(self, lattice, beta, c_plaq=3.648, c_rect=-0.331, nprec=8):
        import torch
        self.lattice = list(lattice)
        self.nvol = int(np.prod(lattice))
        self.beta, self.c_plaq, self.c_rect, self.nprec = beta, c_plaq, c_rect, nprec
        self._L = (ctypes.c_int * 4)(*lattice)
        self.force_buf = torch.empty(18 * 4 * self.nvol, dtype=torch.float64, device="cuda")

    @staticmethod
    def _p(t):
        return ctypes.c_void_p(t.data_ptr())

    def to_device(self, a):
        import torch
        return torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()

    def force(self, u):
        check(lib().b200_gauge_force_rect(self._L, self.beta, self.c_plaq, self.c_rect,
                                          self._p(self.force_buf), self._p(u), None))
        return self.force_buf

    def update_p(self, ip, u, eps):
        """Integrator_UpdateP: iP += eps * F(U)."""
        f = self.force(u)
        check(lib().b200_momentum_update(self._L, eps, self._p(f), self._p(ip), None))

    def update_u(self, ip, u, eps):
        """Integrator_UpdateU: U <- exp(eps iP) U."""
        check(lib().b200_link_update(self._L, eps, self._p(ip), self._p(u), self.nprec, None))

    def hamiltonian(self, ip, u):
        hp = ctypes.c_double()
        hu = ctypes.c_double()
        check(lib().b200_momentum_energy(self._L, self._p(ip), ctypes.byref(hp), None))
        check(lib().b200_gauge_action_rect(self._L, self.beta, self.c_plaq, self.c_rect,
                                           self._p(u), ctypes.byref(hu), None))
        return hp.value + hu.value

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


class DwfMD(GaugeMD):
    """Gauge + two-flavour even/odd domain-wall fermion molecular dynamics on
    the device, in the shape of Action_F_Standard_eo (src/lib/Action/Fermion/
    action_F_Standard_eo.cpp:47-150): S_F = Re <psi, (DdagD)^-1 psi> on the
    even sites, force = mult_generator(force_udiv(eta)) with
    eta = (DdagD)^-1 psi (Force::force_core, src/lib/Force/Fermion/
    force_F.cpp:67-79), added to the gauge force."""

    def __init__(self, op, psi, lattice, beta, c_plaq=3.648, c_rect=-0.331, nprec=8, tol2=1e-24,
                 solver="cg", inner_prec=None, lp=None):
        super().__init__(lattice, beta, c_plaq, c_rect, nprec)
        from . import Field, F64, F16
        self.op = op
        self.psi = psi
        self.tol2 = tol2
        self.eta = Field(op, F64)
        self.solver = solver                  # "cg", "mixed" (Richardson) or "learned" (flexible CG)
        self.inner_prec = F16 if inner_prec is None else inner_prec
        self.lp = lp
        self.last_cg = 0
        self.iterations = 0                   # solver iterations summed over the calls

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
        self.last_cg = n
        self.iterations += n

    def _set(self, u):
        check(lib().b200_dwf_set_config_device(self.op.handle, self._p(u), None))

    def fermion_action(self, u):
        self._set(u)
        self.solve()
        return self.op.dot(self.psi, self.eta)

    def fermion_force(self, u):
        """F_F(U) in the lexical Field_G layout (device tensor)."""
        import torch
        self._set(u)
        self.solve()
        f = torch.empty(18 * 4 * self.nvol, dtype=torch.float64, device="cuda")
        check(lib().b200_dwf_force_udiv(self.op.handle, self._p(f), self.eta.ptr, None))
        check(lib().b200_force_mult_generator(self._L, self._p(f), self._p(u), None))
        return f

    def update_p(self, ip, u, eps):
        fg = self.force(u)
        check(lib().b200_momentum_update(self._L, eps, self._p(fg), self._p(ip), None))
        ff = self.fermion_force(u)
        check(lib().b200_momentum_update(self._L, eps, self._p(ff), self._p(ip), None))

    def hamiltonian(self, ip, u):
        return super().hamiltonian(ip, u) + self.fermion_action(u)
