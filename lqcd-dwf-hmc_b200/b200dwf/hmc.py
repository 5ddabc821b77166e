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
