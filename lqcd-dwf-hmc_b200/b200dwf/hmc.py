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
import time

import numpy as np

from . import check, lib


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


# |r|^2 / |b|^2 at which the mixed-precision Richardson's inner CG stops, per
# inner storage precision (1 f32, 2 f16, 3 bf16).  The half-precision values
# are the fastest of a sweep of one light solve to 1e-10 at 24^3x48 Ls=16,
# mass 0.01, on the tiled conf_04040408 with 2 stout steps: f16 1e-2 / 3e-3 /
# 1e-3 / 1e-4 / 1e-5 took 5.93 / 5.22 / 5.09 / 5.44 / 6.77 s, bf16 1e-2 /
# 3e-3 / 1e-3 / 1e-4 6.05 / 6.03 / 7.41 / 6.84 s (a looser inner solve
# restarts more often, a tighter one runs into the storage's rounding).
INNER_TOL2 = {1: 1e-8, 2: 1e-3, 3: 3e-3}


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
                                             INNER_TOL2[self.inner_prec], 100000)
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

    def force_udiv(self, md, u, out, accumulate=False):
        """out (+)= force_udiv(eta) (accumulate: add to out, else overwrite)."""
        md.set_links(self.op, u)
        self.solve()
        check(lib().b200_dwf_force_acc(self.op.handle, b"DdagD", _p(out), self.eta.ptr, None, 1.0,
                                       None) if accumulate else
              lib().b200_dwf_force_udiv(self.op.handle, _p(out), self.eta.ptr, None))


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

    def force_udiv(self, md, u, out, accumulate=False):
        """out (+)= sum_i b_i force_udiv(x_i), accumulated in place by the
        library's force kernels (the first pole overwrites unless
        accumulate)."""
        md.set_links(self.op, u)
        self.solve()
        L = lib()
        for i, (bi, x) in enumerate(zip(self.b, self.xs)):
            if i == 0 and not accumulate:
                check(L.b200_dwf_force_udiv(self.op.handle, _p(out), x.ptr, None))
                if bi != 1.0:       # out = bi * out (x = y = out, finite here)
                    check(L.b200_links_axpby(md._L, 0.0, _p(out), bi, _p(out), None))
            else:
                check(L.b200_dwf_force_acc(self.op.handle, b"DdagD", _p(out), x.ptr, None, bi, None))


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
        acts = self.fermions if action is None else [action]
        total = self.fbuf
        for k, a in enumerate(acts):
            a.force_udiv(self, u, total, accumulate=k > 0)
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


# ---------------------------------------------------------------------------
# The reference's 2+1-flavour HMC (benchmark_hmc_dwf_corelib/hmc_dwf_eo.cpp:
# 155-352) on the device: stout-smeared links under one director, the
# rational-ratio one-flavour action, two Hasenbusch ratio actions, the
# rectangle gauge action, the nested Omelyan integrator and HMC_General.
# ---------------------------------------------------------------------------

class DirectorSmear:
    """Director_Smear (src/lib/Smear/director_Smear.cpp): the stout levels of
    the current thin links, rebuilt lazily after notify_linkv()."""

    def __init__(self, lattice, rho, nsmear):
        from . import StoutSmear
        self.lattice, self.nsmear = list(lattice), nsmear
        self.sm = StoutSmear(lattice, rho, nsmear) if nsmear > 0 else None
        self.u = None
        self.version = 0
        self._smeared = -1

    def set_config(self, u):
        self.u = u
        self.notify_linkv()

    def notify_linkv(self):
        self.version += 1

    def config_ptr(self):
        """Device pointer of the fully smeared links."""
        if self.nsmear == 0:
            return self.u.data_ptr()
        if self._smeared != self.version:
            check(lib().b200_smear_set_config(self.sm.handle, _p(self.u), 1, None))
            self._smeared = self.version
        return self.sm.config_ptr(self.nsmear)

    def jacobian(self, sigma):
        """Force_F_Smeared::mult_jacobian, in place (src/lib/Force/Fermion/
        force_F_Smeared.cpp:77-88)."""
        if self.nsmear:
            self.config_ptr()
            check(lib().b200_smear_jacobian(self.sm.handle, _p(sigma), None))


class FoprSmeared:
    """Fopr_Smeared_eo: a DomainWall operator that sees the director's
    smeared links (src/lib/Fopr/fopr_Smeared_eo.cpp)."""

    def __init__(self, op, director):
        self.op, self.dr = op, director
        self._version = None

    def sync(self):
        if self._version != self.dr.version or self.dr.nsmear == 0:
            check(lib().b200_dwf_set_config_device(self.op.handle,
                                                   ctypes.c_void_p(self.dr.config_ptr()), None))
            self._version = self.dr.version
        return self.op


class Solver:
    """Fprop 'DdagD_even' with a chosen method: FP64 CG (the reference's
    Solver_CG), mixed-precision Richardson, or the learned flexible CG.
    chrono: the MD solves of an action start from that action's previous
    solution (the reference's use_initial_guess; CG and Richardson only).
    chrono_depth > 1: they start instead from the combination of the last
    chrono_depth solutions (since the action's pseudofermion was drawn) that
    minimises the DdagD-norm of the error, the minimal residual
    extrapolation of the chronological inversion method (Brower, Ivanenko,
    Levi and Orginos, Nucl. Phys. B 484 (1997) 353): k FP64 DdagD
    applications and k(k+1) inner products for k stored solutions, then the
    same solve to the same stopping rule.  No reference counterpart (its
    Fprop starts from the previous solution at most)."""

    def __init__(self, kind="cg", tol2=1e-20, maxiter=100000, inner_prec=None, lp=None,
                 chrono=False, chrono_depth=1):
        from . import F16
        self.kind, self.tol2, self.maxiter = kind, tol2, maxiter
        self.chrono = chrono
        self.chrono_depth = max(1, int(chrono_depth))
        self.inner_prec = F16 if inner_prec is None else inner_prec
        self.lp = lp
        self.iterations = 0
        self.seconds = 0.0
        self.calls = 0
        self._hist = []           # FP64 solutions since the last forget(), oldest first
        self._spare = []          # fields of forgotten solutions, reused
        self._hist_op = None
        self._tmp = None

    def forget(self):
        """The action drew a new pseudofermion: earlier solutions solve
        another system and no longer enter a guess."""
        self._spare.extend(self._hist)
        self._hist = []

    def solve(self, op, x, b, guess=False):
        """x = (DdagD)^-1 b; with guess (and chrono) x on entry is the start."""
        t0 = time.perf_counter()
        use = bool(guess and self.chrono and self.kind in ("cg", "mixed"))
        if self._hist_op is not op:
            self._hist, self._spare, self._tmp, self._hist_op = [], [], None, op
        if use:
            if self.chrono_depth > 1 and len(self._hist) >= 2:
                self._extrapolate(op, x, b)
            op.set_initial_guess(True)
        else:
            x.zero()
        try:
            n = self._solve(op, x, b)
        finally:
            if use:
                op.set_initial_guess(False)
        if self.chrono and self.chrono_depth > 1:
            self._remember(op, x)
        self.seconds += time.perf_counter() - t0   # the solvers end with a host read
        self.calls += 1
        return n

    def _remember(self, op, x):
        if len(self._hist) == self.chrono_depth:
            f = self._hist.pop(0)
        elif self._spare:
            f = self._spare.pop()
        else:
            f = op.new_field()
        op.axpby(f, 1.0, x, 0.0)
        self._hist.append(f)

    def _extrapolate(self, op, x, b):
        """x = sum_j c_j v_j minimising |x* - x|_A (A = DdagD) over real c:
        G c = f with G_ij = Re<v_i, A v_j>, f_i = Re<v_i, b>, solved on the
        eigenvectors of G above 1e-13 of its largest eigenvalue (successive
        solutions are nearly parallel)."""
        v = self._hist
        k = len(v)
        if self._tmp is None:
            self._tmp = op.new_field()
        t = self._tmp
        g = np.empty((k, k))
        f = np.empty(k)
        for j in range(k):
            op.mult(t, v[j], "DdagD")
            for i in range(k):
                g[i, j] = op.dot(v[i], t)
            f[j] = op.dot(v[j], b)
        g = 0.5 * (g + g.T)
        w, q = np.linalg.eigh(g)
        keep = w > w[-1] * 1e-13
        c = q[:, keep] @ ((q[:, keep].T @ f) / w[keep])
        op.axpby(x, float(c[0]), v[0], 0.0)
        for j in range(1, k):
            op.axpby(x, float(c[j]), v[j], 1.0)

    def _solve(self, op, x, b):
        if self.kind == "cg":
            n, _, rc = op.cg(x, b, self.tol2, self.maxiter)
        elif self.kind == "mixed":
            _, n, _, rc = op.richardson(x, b, self.inner_prec, self.tol2, 200,
                                        INNER_TOL2[self.inner_prec], self.maxiter)
        elif self.kind == "learned":
            n0, n1, _, rc = op.fcg(x, b, self.lp, self.tol2, self.maxiter, 2)
            n = n0 + n1
        else:
            raise ValueError(self.kind)
        if rc != 0:
            raise RuntimeError("fermion solve did not converge (%s)" % self.kind)
        self.iterations += n
        return n


class FoprRational:
    """Fopr_Rational (src/lib/Fopr/afopr_Rational-tmpl.h:181-219):
    v = a0 b + sum_i b_i (DdagD + c_i)^-1 b from one multishift solve."""

    def __init__(self, fopr, rational, tol2, maxiter=100000):
        self.fopr, self.r = fopr, rational
        self.tol2, self.maxiter = tol2, maxiter
        self.xs = None
        self.iterations = 0
        self.seconds = 0.0
        self.calls = 0

    def shifts(self, b):
        """x_i = (DdagD + c_i)^-1 b (kept in self.xs)."""
        from . import Field
        op = self.fopr.sync()
        if self.xs is None:
            self.xs = [Field(op) for _ in self.r.c]
        t0 = time.perf_counter()
        n, _, rc = op.shiftcg(self.xs, self.r.c, b, self.tol2, self.maxiter)
        self.seconds += time.perf_counter() - t0
        self.calls += 1
        if rc != 0:
            raise RuntimeError("multishift solve did not converge")
        self.iterations += n
        return self.xs

    def mult(self, v, b):
        xs = self.shifts(b)
        op = self.fopr.op
        op.axpby(v, self.r.a0, b, 0.0)
        for bi, x in zip(self.r.b, xs):
            op.axpby(v, bi, x, 1.0)
        return v


class ActionFRatio:
    """Action_F_Ratio_eo (src/lib/Action/Fermion/action_F_Ratio_eo.cpp):
    S = <psi, H_p (DdagD)^-1 H_p^dag psi> for det[DdagD / DdagD_p], the
    Hasenbusch ratio of a lighter (fopr) over a heavier (fopr_prec) operator.
    The three solves follow the reference's Fprop roles: solver_h_prec in the
    heatbath, solver_md in the force, solver_h in the Hamiltonian."""

    def __init__(self, fopr_prec, fopr, solver_md, solver_h, solver_h_prec, label=""):
        from . import Field
        self.fp, self.f = fopr_prec, fopr
        self.solver_md, self.solver_h, self.solver_h_prec = solver_md, solver_h, solver_h_prec
        self.label = label
        op = fopr.op
        self.psf, self.v1, self.v2 = Field(op), Field(op), Field(op)
        self.fermion = True
        self._guess = False       # v2 holds a solution of the current psf

    def langevin(self, xi):
        f, fp = self.f.sync(), self.fp.sync()
        f.mult_dag(self.v2, xi, "H")
        self.solver_h_prec.solve(fp, self.v1, self.v2)
        fp.mult(self.psf, self.v1, "H")
        self._guess = False
        self.solver_md.forget()
        self.solver_h.forget()
        return f.norm2(xi)

    def calcH(self):
        f, fp = self.f.sync(), self.fp.sync()
        fp.mult_dag(self.v1, self.psf, "H")
        self.solver_h.solve(f, self.v2, self.v1, self._guess)
        self._guess = True
        return f.dot(self.v1, self.v2)

    def force_udiv(self, acc):
        """acc += this action's force_udiv on the smeared links
        (action_F_Ratio_eo.cpp:171-205 before mult_generator)."""
        f, fp = self.f.sync(), self.fp.sync()
        fp.mult_dag(self.v1, self.psf, "H")
        self.solver_md.solve(f, self.v2, self.v1, self._guess)
        self._guess = True
        L = lib()
        check(L.b200_dwf_force_acc(f.handle, b"DdagD", _p(acc), self.v2.ptr, None, 1.0, None))
        check(L.b200_dwf_force_acc(fp.handle, b"Hdag", _p(acc), self.v2.ptr, self.psf.ptr, -1.0, None))
        check(L.b200_dwf_force_acc(fp.handle, b"H", _p(acc), self.psf.ptr, self.v2.ptr, -1.0, None))


class ActionFRationalRatio:
    """Action_F_Rational_Ratio_eo + Force_F_Rational_Ratio (src/lib/Action/
    Fermion/action_F_Rational_Ratio_eo.cpp:73-170, src/lib/Force/Fermion/
    force_F_Rational_Ratio.cpp:187-292): one flavour as
    det[(B^dag B)^(1/2) / (A^dag A)^(1/2)], A = fopr_numer (Pauli-Villars),
    B = fopr_denom.  rats: dict of Rational coefficient sets
    'md_numer' x^(1/4), 'md_denom' x^(-1/2), 'h_numer' x^(1/4),
    'h_denom' x^(-1/2), 'psf_denom' x^(1/4), 'psf_numer' x^(-1/4).

    force_pool: 'paired' keeps the numerator's two sets of shifted solutions
    (eta1_i, zeta_i) side by side, 2*np_md solution fields; 'streamed' takes
    the numerator's cross terms from two further multishift solves of the
    combined sources s*phi +- v/s (one balance factor s for all poles), one
    set of np_md solution fields at a time: np_md fewer fields (39 GB at
    32^3x64 Ls=12, FP64) for one more multishift per force evaluation."""

    def __init__(self, fopr_numer, fopr_denom, rats, tol2_md, tol2_h, label="",
                 force_pool="paired"):
        from . import Field
        if force_pool not in ("paired", "streamed"):
            raise ValueError("force_pool: 'paired' or 'streamed'")
        self.fa, self.fb = fopr_numer, fopr_denom
        self.label = label
        self.force_pool = force_pool
        self.md_numer = FoprRational(fopr_numer, rats["md_numer"], tol2_md)
        self.md_denom = FoprRational(fopr_denom, rats["md_denom"], tol2_md)
        self.md_numer2 = FoprRational(fopr_numer, rats["md_numer"], tol2_md)
        self.h_numer = FoprRational(fopr_numer, rats["h_numer"], tol2_h)
        self.h_denom = FoprRational(fopr_denom, rats["h_denom"], tol2_h)
        self.psf_denom = FoprRational(fopr_denom, rats["psf_denom"], tol2_h)
        self.psf_numer = FoprRational(fopr_numer, rats["psf_numer"], tol2_h)
        op = fopr_denom.op
        self.psf, self.v1, self.v2 = Field(op), Field(op), Field(op)
        # the combined source of the streamed force; the paired force's two
        # polarised vectors
        self.t1 = Field(op)
        self.t2 = Field(op) if force_pool == "paired" else None
        self.fermion = True
        # one pool of solution vectors: eta1_i in the first np_md slots, eta2_i
        # and later zeta_i in the next np_md (the denominator's forces are
        # taken before zeta overwrites eta2), and the heatbath / Hamiltonian
        # rationals, which only need their sums, in the first np_h slots
        nmd, nh = len(rats["md_numer"].c), len(rats["h_numer"].c)
        if len(rats["md_denom"].c) != nmd:
            raise ValueError("numerator and denominator MD rationals need equal pole counts")
        if force_pool == "paired":
            self.pool = [Field(op) for _ in range(max(2 * nmd, nh))]
            self.md_numer.xs = self.pool[:nmd]
            self.md_denom.xs = self.pool[nmd:2 * nmd]
            self.md_numer2.xs = self.pool[nmd:2 * nmd]
        else:
            # eta1_i only make v1, eta2_i only the denominator's forces, and
            # the combined sources' solutions are used one set at a time
            self.pool = [Field(op) for _ in range(max(nmd, nh))]
            for r in (self.md_numer, self.md_denom, self.md_numer2):
                r.xs = self.pool[:nmd]
        for r in (self.h_numer, self.h_denom, self.psf_denom, self.psf_numer):
            r.xs = self.pool[:len(r.r.c)]

    @property
    def rationals(self):
        return dict(md_numer=self.md_numer, md_denom=self.md_denom, md_numer2=self.md_numer2,
                    h_numer=self.h_numer, h_denom=self.h_denom, psf_denom=self.psf_denom,
                    psf_numer=self.psf_numer)

    @property
    def iterations(self):
        return sum(r.iterations for r in self.rationals.values())

    def langevin(self, xi):
        self.psf_denom.mult(self.v1, xi)          # (B^dag B)^(1/4) xi
        self.psf_numer.mult(self.psf, self.v1)    # (A^dag A)^(-1/4)
        return self.fb.op.norm2(xi)

    def calcH(self):
        self.h_numer.mult(self.v1, self.psf)      # (A^dag A)^(1/4) psf
        self.h_denom.mult(self.v2, self.v1)       # (B^dag B)^(-1/2)
        return self.fb.op.dot(self.v1, self.v2)

    def force_udiv(self, acc):
        """acc += force_udiv of the rational ratio on the smeared links.  The
        numerator's four mixed terms per pole (force_udiv1 in modes H and Hdag
        with eta1_i and zeta_i swapped) are the cross term of the quadratic
        force_udiv, taken by polarisation:
            sum = (force_udiv(s eta1 + zeta/s) - force_udiv(s eta1 - zeta/s)) / 2,
        s^2 = |zeta| / |eta1| balancing the two vectors."""
        L = lib()
        fa, fb = self.fa.sync(), self.fb.sync()
        rn, rd = self.md_numer.r, self.md_denom.r
        self.md_numer.mult(self.v1, self.psf)          # phi2, eta1_i in md_numer.xs
        self.md_denom.mult(self.v2, self.v1)           # xi, eta2_i in md_denom.xs
        for bi, e2 in zip(rd.b, self.md_denom.xs):
            check(L.b200_dwf_force_acc(fb.handle, b"DdagD", _p(acc), e2.ptr, None, bi, None))
        if self.force_pool == "streamed":
            # sum_i b_i cross(eta1_i, zeta_i) = sum_i b_i/4 [F(x+_i) - F(x-_i)],
            # x+-_i = (A^dag A + c_i)^-1 (s psf +- v2/s): F is quadratic and
            # the shifted solve linear in its source
            npsf, nv2 = fa.norm2(self.psf), fa.norm2(self.v2)
            if npsf == 0.0 or nv2 == 0.0:
                return
            s = (nv2 / npsf) ** 0.25
            for sign in (1.0, -1.0):
                fa.axpby(self.t1, s, self.psf, 0.0)
                fa.axpby(self.t1, sign / s, self.v2, 1.0)
                for bi, x in zip(rn.b, self.md_numer2.shifts(self.t1)):
                    check(L.b200_dwf_force_acc(fa.handle, b"DdagD", _p(acc), x.ptr, None,
                                               0.5 * sign * bi, None))
            return
        zetas = self.md_numer2.shifts(self.v2)         # zeta_i, over the eta2_i slots
        for bi, e1, z in zip(rn.b, self.md_numer.xs, zetas):
            ne, nz = fa.norm2(e1), fa.norm2(z)
            if ne == 0.0 or nz == 0.0:
                continue
            s = (nz / ne) ** 0.25
            fa.axpby(self.t1, s, e1, 0.0)
            fa.axpby(self.t1, 1.0 / s, z, 1.0)
            fa.axpby(self.t2, s, e1, 0.0)
            fa.axpby(self.t2, -1.0 / s, z, 1.0)
            check(L.b200_dwf_force_acc(fa.handle, b"DdagD", _p(acc), self.t1.ptr, None, 0.5 * bi, None))
            check(L.b200_dwf_force_acc(fa.handle, b"DdagD", _p(acc), self.t2.ptr, None, -0.5 * bi, None))


class ActionGRectangle:
    """Action_G_Rectangle with Force_G_Rectangle (src/lib/Action/Gauge/
    action_G_Rectangle.cpp:97-200, src/lib/Force/Gauge/force_G_Rectangle.cpp)."""

    def __init__(self, lattice, beta, c_plaq=3.648, c_rect=-0.331):
        self._L = (ctypes.c_int * 4)(*lattice)
        self.beta, self.c_plaq, self.c_rect = beta, c_plaq, c_rect
        self.fermion = False
        self.u = None
        self.label = "gauge"

    def langevin(self, _xi=None):
        return self.calcH()

    def calcH(self):
        h = ctypes.c_double()
        check(lib().b200_gauge_action_rect(self._L, self.beta, self.c_plaq, self.c_rect,
                                           _p(self.u), ctypes.byref(h), None))
        return h.value

    def force(self, out):
        check(lib().b200_gauge_force_rect(self._L, self.beta, self.c_plaq, self.c_rect,
                                          _p(out), _p(self.u), None))


class UpdateP:
    """Integrator_UpdateP (src/lib/HMC/integrator_UpdateP.cpp:44-66): the
    level's summed force, cached until the links change.  The fermion
    actions of a level share one smeared-force Jacobian and one
    mult_generator (both are linear)."""

    def __init__(self, hmc, actions):
        import torch
        self.hmc, self.actions = hmc, list(actions)
        n = 18 * 4 * hmc.nvol
        self.force = torch.zeros(n, dtype=torch.float64, device="cuda")
        self.valid = False
        self.evaluations = 0

    def evolve(self, step, ip, u):
        if not self.valid:
            self.hmc.level_force(self.actions, u, self.force)
            self.valid = True
            self.evaluations += 1
        check(lib().b200_momentum_update(self.hmc._L, step, _p(self.force), _p(ip), None))


class UpdateU:
    """Integrator_UpdateU (src/lib/HMC/integrator_UpdateU.cpp:79-98):
    U <- exp(step iP) U, then every force cache and the director are told."""

    def __init__(self, hmc, nprec):
        self.hmc, self.nprec = hmc, nprec
        self.clients = []

    def evolve(self, step, ip, u):
        check(lib().b200_link_update(self.hmc._L, step, _p(ip), _p(u), self.nprec, None))
        for c in self.clients:
            c.valid = False
        self.hmc.director.notify_linkv()


class Omelyan:
    """Integrator_Omelyan::evolve (src/lib/HMC/integrator_Omelyan.cpp:
    85-117): P(l e) [U(e/2) P((1-2l) e) U(e/2) P(2 l e)]... P(l e), the
    inner 'U' being the next level's integrator."""

    def __init__(self, update_p, inner, nstep, lam):
        self.p, self.u, self.nstep, self.lam = update_p, inner, nstep, lam

    def evolve(self, step, ip, u):
        if self.nstep <= 0:
            return
        e = step / self.nstep
        self.p.evolve(e * self.lam, ip, u)
        for k in range(1, self.nstep + 1):
            self.u.evolve(0.5 * e, ip, u)
            self.p.evolve(e * (1.0 - 2.0 * self.lam), ip, u)
            self.u.evolve(0.5 * e, ip, u)
            if k < self.nstep:
                self.p.evolve(2.0 * e * self.lam, ip, u)
        self.p.evolve(e * self.lam, ip, u)


class Leapfrog:
    """Integrator_Leapfrog::evolve (src/lib/HMC/integrator_Leapfrog.cpp)."""

    def __init__(self, update_p, inner, nstep):
        self.p, self.u, self.nstep = update_p, inner, nstep

    def evolve(self, step, ip, u):
        if self.nstep <= 0:
            return
        e = step / self.nstep
        self.p.evolve(0.5 * e, ip, u)
        for k in range(1, self.nstep + 1):
            self.u.evolve(e, ip, u)
            if k < self.nstep:
                self.p.evolve(e, ip, u)
        self.p.evolve(0.5 * e, ip, u)


def _momentum_from_gauss(h, ip, nvol):
    """iP = i sum_a h_a lambda_a on the 4*nvol links (b200_momentum_from_gauss);
    the kernel sees only the site count, so both buffers are checked here."""
    if ip.numel() != 72 * nvol or h.numel() != 32 * nvol:
        raise ValueError("momentum: %d and %d reals for %d sites (72 and 32 per site expected)"
                         % (ip.numel(), h.numel(), nvol))
    check(lib().b200_momentum_from_gauss((ctypes.c_int * 4)(nvol, 1, 1, 1), _p(h), _p(ip), None))


class DeviceNoise:
    """Gaussian heatbath fields drawn on the device (torch's Philox stream):
    momenta iP = i sum_a h_a lambda_a with <h_a^2> = 1/2, so that
    P(iP) ~ exp(-|iP|^2/2) as Langevin_Momentum::set_iP
    (src/lib/HMC/langevin_Momentum.cpp:86-140), and pseudofermion noise with
    variance 1/2 per real component (RandomNumbers::gauss,
    src/lib/Tools/randomNumbers.cpp:64-75).  Every component is iid, so the
    noise is drawn straight in the device field layout."""

    def __init__(self, seed):
        import torch
        self.g = torch.Generator(device="cuda")
        self.g.manual_seed(int(seed))

    def momentum(self, ip):
        import torch
        h = torch.empty(ip.numel() // 18, 8, dtype=torch.float64, device="cuda")
        h.normal_(0.0, 0.5 ** 0.5, generator=self.g)
        _momentum_from_gauss(h, ip, ip.numel() // 72)

    def fermion(self, field):
        field.buf.view(dtype=__import__("torch").float64).normal_(0.0, 0.5 ** 0.5, generator=self.g)


class MseriesNoise:
    """The benchmark driver's heatbath draws on the device: the parallel
    M-series generator (random_number_type Mseries_parallel, b200_rng_*)
    hands out, in the reference's order, Field(8, Nvol, 4) Gaussians for the
    momenta, turned into iP = i sum_a h_a lambda_a (Gell-Mann order) as
    Langevin_Momentum::set_iP_SU3 does
    (src/lib/HMC/langevin_Momentum.cpp:150-210), and for each fermion action a
    lexical Field(24, Nvol, Ls) whose even sites are the noise xi
    (Index_eo::convertField(xi, xi_lexical, 0),
    src/lib/Action/Fermion/action_F_Ratio_eo.cpp:70-78,
    action_F_Rational_Ratio_eo.cpp:95-99).  reset(seed) is the driver's
    rand->reset(i_conf + traj) before each trajectory
    (benchmark_hmc_dwf_corelib/hmc_dwf_eo.cpp:347)."""

    def __init__(self, lattice, seed):
        from . import MseriesParallel
        self.lattice = list(lattice)
        self.nvol = int(np.prod(lattice))
        self.rng = MseriesParallel(lattice, seed)

    def reset(self, seed):
        self.rng.reset(seed)

    def momentum(self, ip):
        _momentum_from_gauss(self.rng.gauss_lex_global(8, 4), ip, self.nvol)

    def fermion(self, field):
        op = field.op
        if 2 * op.nvol != self.nvol:
            raise ValueError("noise lattice (%d sites) differs from the operator's (%d)"
                             % (self.nvol, 2 * op.nvol))
        lex = self.rng.gauss_lex_global(24, op.Ls)
        check(lib().b200_field_convert_lex_device(op.handle, field.prec, field.ptr, _p(lex), 0, None))


class HostNoise:
    """Heatbath fields handed in from outside (for instance recorded from the
    reference's own random-number generator): momenta in the lexical
    Field_G layout, pseudofermion noise as even-site corelib spinors."""

    def __init__(self, ip_lex, xis):
        self.ip, self.xis = ip_lex, list(xis)
        self.k = 0

    def momentum(self, ip):
        import torch
        ip.copy_(torch.from_numpy(np.ascontiguousarray(self.ip, np.float64)))

    def fermion(self, field):
        field.op.convert(field, self.xis[self.k])
        self.k += 1


class HMCGeneral:
    """HMC_General (src/lib/HMC/hmc_General.cpp:166-356) over device fields:
    langevin (momenta + every action's heatbath), the nested integrator
    built as Builder_Integrator::build_omelyan does
    (src/lib/HMC/builder_Integrator.cpp:226-255), the Hamiltonian and the
    Metropolis test.  actions: list of (level, action) in the reference's
    registration order; nstep: steps per level (level 0 outermost)."""

    def __init__(self, lattice, actions, director, nstep, tau=1.0, lam=0.1931833275,
                 nprec=8, integrator="Omelyan"):
        import torch
        self.lattice = list(lattice)
        self.nvol = int(np.prod(lattice))
        self._L = (ctypes.c_int * 4)(*lattice)
        self.actions = [a for _, a in actions]
        self.director = director
        self.tau = tau
        n = 18 * 4 * self.nvol
        self.fbuf = torch.zeros(n, dtype=torch.float64, device="cuda")
        self.gbuf = torch.zeros(n, dtype=torch.float64, device="cuda")
        self.update_u = UpdateU(self, nprec)
        inner = self.update_u
        self.update_ps = []
        for lv in range(len(nstep) - 1, -1, -1):
            up = UpdateP(self, [a for l, a in actions if l == lv])
            self.update_u.clients.append(up)
            self.update_ps.append(up)
            inner = (Omelyan(up, inner, nstep[lv], lam) if integrator == "Omelyan"
                     else Leapfrog(up, inner, nstep[lv]))
        self.integrator = inner
        self.u = None

    def set_config(self, u):
        self.u = u
        self.director.set_config(u)
        for a in self.actions:
            if not a.fermion:
                a.u = u

    def level_force(self, actions, u, out):
        """Integrator_UpdateP's summed force of one level into out (library
        kernels: the first term overwrites out, the others add to it)."""
        L = lib()
        beta = 0.0
        ferm = [a for a in actions if a.fermion]
        if ferm:
            check(L.b200_links_axpby(self._L, 0.0, _p(self.fbuf), 0.0, _p(self.fbuf), None))
            for a in ferm:
                a.force_udiv(self.fbuf)
            self.director.jacobian(self.fbuf)
            check(L.b200_force_mult_generator(self._L, _p(self.fbuf), _p(u), None))
            check(L.b200_links_axpby(self._L, 1.0, _p(self.fbuf), beta, _p(out), None))
            beta = 1.0
        for a in actions:
            if not a.fermion:
                a.force(self.gbuf)
                check(L.b200_links_axpby(self._L, 1.0, _p(self.gbuf), beta, _p(out), None))
                beta = 1.0
        if beta == 0.0:
            check(L.b200_links_axpby(self._L, 0.0, _p(out), 0.0, _p(out), None))

    def momentum_energy(self, ip):
        h = ctypes.c_double()
        check(lib().b200_momentum_energy(self._L, _p(ip), ctypes.byref(h), None))
        return h.value

    def langevin(self, ip, noise):
        """HMC_General::langevin: returns (H_total, per-action values)."""
        from . import Field
        for up in self.update_ps:
            up.valid = False
        self.director.notify_linkv()
        noise.momentum(ip)
        parts = [self.momentum_energy(ip)]
        for a in self.actions:
            if a.fermion:
                # one noise field for every action: each consumes its xi in
                # its own langevin (all operators share the geometry)
                xi = getattr(self, "_xi", None)
                if xi is None:
                    xi = self._xi = Field(a.f.op if hasattr(a, "f") else a.fb.op)
                noise.fermion(xi)
                parts.append(a.langevin(xi))
            else:
                parts.append(a.langevin())
        return sum(parts), parts

    def calc_hamiltonian(self, ip):
        parts = [self.momentum_energy(ip)] + [a.calcH() for a in self.actions]
        return sum(parts), parts

    def trajectory(self, u, noise):
        """One trajectory from links u (device, modified in place): returns
        a dict with H0, H1, dH and the per-action parts."""
        import torch
        self.set_config(u)
        ip = torch.zeros_like(u)
        h0, p0 = self.langevin(ip, noise)
        self.integrator.evolve(self.tau, ip, u)
        h1, p1 = self.calc_hamiltonian(ip)
        return dict(H0=h0, H1=h1, dH=h1 - h0, parts0=p0, parts1=p1, ip=ip)

    def update(self, u, noise, rng):
        """HMC_General::update: trajectory + Metropolis (FP64, host uniform
        number from rng); u keeps the accepted links."""
        u_old = u.clone()
        r = self.trajectory(u, noise)
        accept = rng.random() <= np.exp(-r["dH"])
        if not accept:
            u.copy_(u_old)
        r["accepted"] = bool(accept)
        return r

    @property
    def force_evaluations(self):
        return {len(self.update_ps) - 1 - i: up.evaluations for i, up in enumerate(self.update_ps)}

    def stats(self):
        """Iterations, calls and host-side seconds of every solver and
        multishift of the action set (the solvers end with a host read, so
        their wall times are device times plus launch overhead)."""
        out = {}
        for name, sv in getattr(self, "solvers", {}).items():
            out["solver_" + name] = dict(kind=sv.kind, iterations=sv.iterations, calls=sv.calls,
                                         seconds=sv.seconds)
        nf1 = getattr(self, "fermions", {}).get("nf1")
        if nf1 is not None:
            for name, r in nf1.rationals.items():
                out["multishift_" + name] = dict(poles=len(r.r.c), iterations=r.iterations,
                                                 calls=r.calls, seconds=r.seconds)
        out["force_evaluations"] = self.force_evaluations
        return out

    def warmup(self):
        """Untimed first use of every operator, solver, multishift pole set
        and force path (autotuning, work buffers, multishift graph capture)."""
        import torch
        from . import Field
        ops = {}
        for a in self.actions:
            for fo in (getattr(a, "fp", None), getattr(a, "f", None), getattr(a, "fa", None),
                       getattr(a, "fb", None)):
                if fo is not None:
                    ops[id(fo)] = fo
        scratch = torch.zeros_like(self.fbuf)
        for fo in ops.values():
            op = fo.sync()
            b = Field(op)
            DeviceNoise(1).fermion(b)
            x = Field(op)
            op.cg(x, b, 1e-30, 5)
            for sv in getattr(self, "solvers", {}).values():
                if sv.kind == "mixed":
                    op.richardson(x, b, sv.inner_prec, 1e-30, 1, 1e-4, 5)
                elif sv.kind == "learned" and sv.lp is not None and sv.lp.op is op:
                    op.fcg(x, b, sv.lp, 1.0, 5, 2)
            check(lib().b200_dwf_force_acc(op.handle, b"DdagD", _p(scratch), b.ptr, None, 0.0, None))
            check(lib().b200_dwf_force_acc(op.handle, b"H", _p(scratch), b.ptr, x.ptr, 0.0, None))
        nf1 = getattr(self, "fermions", {}).get("nf1")
        if nf1 is not None:
            for r in nf1.rationals.values():
                op = r.fopr.sync()
                if r.xs is None:
                    r.xs = [Field(op) for _ in r.r.c]
                b = Field(op)
                DeviceNoise(2).fermion(b)
                op.shiftcg(r.xs, r.r.c, b, 1e-30, 40)
        self.director.jacobian(scratch)
        torch.cuda.synchronize()


def build_dwf_nf2p1(lattice, Ls, M0, masses, beta, c_plaq=3.648, c_rect=-0.331, rho=0.1,
                    nsmear=2, nstep=(2, 1, 3), level=(0, 0, 1, 2), tau=1.0,
                    lam=0.1931833275, nprec=8, np_md=16, np_h=24, rat_bounds=(1e-2, 3.16227766),
                    tol2_md=1e-20, tol2_h=1e-20, solvers=None, b=1.0, c=0.0,
                    bc=(1, 1, 1, -1), integrator="Omelyan", shift_window=None,
                    rational_dir=None, tol2_rat_md=None, tol2_rat_h=None,
                    rational_force_pool="paired"):
    """The benchmark driver's action set (hmc_dwf_eo.cpp:155-352) on the
    device.  masses: dict l (light), h (Hasenbusch), s (strange), pv.
    solvers: dict of Solver objects 'l_md', 'l_h', 'h_md', 'h_h', 'pv_h'
    (default FP64 CG at tol2_md / tol2_h).  shift_window: residual window of
    the multishift solves (None keeps the library default, 0 updates every
    shift every iteration).  rational_dir: directory of the coefficient files
    (Math_Rational's format and names; default: this package's tables), as
    the reference reads them from its run directory.  tol2_rat_md /
    tol2_rat_h: the multishift tolerances of the rational operators
    (Fopr_Nf1_Rational_MD / _calcH convergence_criterion_squared; default
    tol2_md / tol2_h).  rational_force_pool: ActionFRationalRatio's
    force_pool ('streamed' for lattices whose 2*np_md solution fields do not
    fit beside the rest)."""
    from . import DomainWall
    from .rational import Rational, TABLE_DIR
    tdir = rational_dir or TABLE_DIR
    tol2_rat_md = tol2_md if tol2_rat_md is None else tol2_rat_md
    tol2_rat_h = tol2_h if tol2_rat_h is None else tol2_rat_h
    dr = DirectorSmear(lattice, rho, nsmear)

    def fopr(m):
        op = DomainWall(lattice, Ls, m, M0, b=b, c=c, bc=bc)
        if shift_window is not None:
            op.set_shift_window(shift_window)
        return FoprSmeared(op, dr)

    lo, hi = rat_bounds
    rats = dict(md_numer=Rational(np_md, 1, 4, lo, hi, tdir),
                md_denom=Rational(np_md, -1, 2, lo, hi, tdir),
                h_numer=Rational(np_h, 1, 4, lo, hi, tdir), h_denom=Rational(np_h, -1, 2, lo, hi, tdir),
                psf_denom=Rational(np_h, 1, 4, lo, hi, tdir),
                psf_numer=Rational(np_h, -1, 4, lo, hi, tdir))
    # one operator per distinct mass: the Pauli-Villars operator serves the
    # rational ratio and the outer Hasenbusch ratio alike
    f_s, f_l, f_h, f_pv = (fopr(masses[k]) for k in ("s", "l", "h", "pv"))
    f_pv1 = f_pv
    sv = dict(solvers or {})
    for k, t in (("l_md", tol2_md), ("h_md", tol2_md), ("l_h", tol2_h), ("h_h", tol2_h),
                 ("pv_h", tol2_h)):
        sv.setdefault(k, Solver("cg", t))
    nf1 = ActionFRationalRatio(f_pv1, f_s, rats, tol2_rat_md, tol2_rat_h, "Nf1",
                               force_pool=rational_force_pool)
    nf2 = ActionFRatio(f_h, f_l, sv["l_md"], sv["l_h"], sv["h_h"], "Nf2")
    nf2p = ActionFRatio(f_pv, f_h, sv["h_md"], sv["h_h"], sv["pv_h"], "Nf2_prec")
    gauge = ActionGRectangle(lattice, beta, c_plaq, c_rect)
    acts = list(zip(level, (nf1, nf2, nf2p, gauge)))
    hmc = HMCGeneral(lattice, acts, dr, list(nstep), tau, lam, nprec, integrator)
    hmc.solvers = sv
    hmc.fermions = dict(nf1=nf1, nf2=nf2, nf2p=nf2p)
    return hmc
