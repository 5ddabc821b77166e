"""Python binding of the B200 domain-wall library (libb200dwf.so, C ABI in
include/b200dwf.h).

The host-side mirror of the reference operator interface
``AFopr_Domainwall_5din_eo`` (src/lib_alt_Accel/Fopr/afopr_Domainwall_5din_eo.h):
``set_config``, ``set_mode``, ``mult``/``mult_dag`` (with and without an
explicit mode), ``convert``/``reverse``, ``field_nin/nvol/nex``.  Device fields
are ``torch`` uint8 buffers on the current CUDA device; PyTorch is only the
allocator here, every operation runs in the library's own sm_100a kernels.

The library is loaded from this package directory; importing the operator on a
machine without the built library raises instead of falling back to anything.
"""
import ctypes
import os

import numpy as np

from . import synth  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(os.path.dirname(HERE), "libb200dwf.so")

F64, F32, F16, BF16 = 0, 1, 2, 3
PREC_NAMES = {"f64": F64, "f32": F32, "f16": F16, "bf16": BF16}

_lib = None


class B200Error(RuntimeError):
    pass


# int (*b200_halo_fn)(void* ctx, void* field, int prec, void* stream)
HALO_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                           ctypes.c_void_p)


def lib():
    """Load libb200dwf.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise B200Error("libb200dwf.so not built (run `make -C lqcd-dwf-hmc_b200`)")
    L = ctypes.CDLL(LIBPATH)
    vp = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    L.b200_last_error.restype = ctypes.c_char_p
    L.b200_init.argtypes = [ctypes.c_int, ctypes.c_int]
    L.b200_dwf_create.argtypes = [ctypes.POINTER(vp), ip, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_double, dp, dp, ctypes.c_double, ip]
    L.b200_dwf_destroy.argtypes = [vp]
    L.b200_dwf_set_config.argtypes = [vp, dp, vp]
    L.b200_dwf_set_config_device.argtypes = [vp, vp, vp]
    L.b200_dwf_field_bytes.argtypes = [vp, ctypes.c_int]
    L.b200_dwf_field_bytes.restype = ctypes.c_size_t
    L.b200_dwf_field_nreal.argtypes = [vp]
    L.b200_dwf_field_nreal.restype = ctypes.c_size_t
    L.b200_field_convert.argtypes = [vp, ctypes.c_int, vp, dp, vp]
    L.b200_field_reverse.argtypes = [vp, ctypes.c_int, dp, vp, vp]
    L.b200_field_convert_device.argtypes = [vp, ctypes.c_int, vp, vp, vp]
    L.b200_field_convert_async.argtypes = [vp, ctypes.c_int, vp, vp, vp]
    L.b200_field_reverse_async.argtypes = [vp, ctypes.c_int, vp, vp, vp]
    L.b200_dwf_mult.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_char_p, ctypes.c_int, vp]
    L.b200_dwf_set_async.argtypes = [vp, ctypes.c_int]
    L.b200_dwf_check_error.argtypes = [vp, vp]
    L.b200_dwf_inject_wait_failure.argtypes = [vp, ctypes.c_int]
    L.b200_dwf_set_halo_exchange.argtypes = [vp, HALO_FN, vp]
    L.b200_dwf_set_halo_exchange_split.argtypes = [vp, HALO_FN, HALO_FN, vp]
    L.b200_field_axpby.argtypes = [vp, ctypes.c_int, vp, ctypes.c_double, vp, ctypes.c_double, vp]
    L.b200_field_norm2.argtypes = [vp, ctypes.c_int, vp, dp, vp]
    L.b200_field_dot.argtypes = [vp, ctypes.c_int, vp, vp, dp, vp]
    L.b200_field_copy_convert.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, vp, vp]
    L.b200_shiftcg_solve.argtypes = [vp, ctypes.POINTER(vp), dp, ctypes.c_int, vp, ctypes.c_int,
                                     ctypes.c_double, ip, dp, vp]
    L.b200_richardson_solve.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_int, ctypes.c_double, ip, ip, dp, vp]
    L.b200_dwf_force_udiv1.argtypes = [vp, ctypes.c_char_p, vp, vp, vp, vp]
    L.b200_dwf_force_udiv.argtypes = [vp, vp, vp, vp]
    L.b200_shiftcg_set_window.argtypes = [vp, ctypes.c_int]
    L.b200_solver_set_initial_guess.argtypes = [vp, ctypes.c_int]
    L.b200_dwf_force_acc.argtypes = [vp, ctypes.c_char_p, vp, vp, vp, ctypes.c_double, vp]
    L.b200_smear_create.argtypes = [ctypes.POINTER(vp), ip, ctypes.c_double, ctypes.c_int]
    L.b200_smear_destroy.argtypes = [vp]
    L.b200_smear_set_config.argtypes = [vp, vp, ctypes.c_int, vp]
    L.b200_smear_config.argtypes = [vp, ctypes.c_int]
    L.b200_smear_config.restype = ctypes.c_void_p
    L.b200_smear_jacobian.argtypes = [vp, vp, vp]
    L.b200_smear_get_config.argtypes = [vp, ctypes.c_int, dp, vp]
    L.b200_force_mult_generator.argtypes = [ip, vp, vp, vp]
    L.b200_field_norm2_noalloc.argtypes = [ctypes.c_int, vp, ctypes.c_long, ctypes.c_int, dp, vp]
    L.b200_rng_create.argtypes = [ctypes.POINTER(vp), ip, ctypes.c_ulong]
    L.b200_rng_reset.argtypes = [vp, ctypes.c_ulong]
    L.b200_rng_gauss_lex.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, vp]
    L.b200_rng_uniform_lex.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, vp]
    L.b200_rng_destroy.argtypes = [vp]
    L.b200_tuning_table.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    L.b200_cg_solve.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_double,
                                ip, dp, vp]
    d_ = ctypes.c_double
    L.b200_gauge_force_rect.argtypes = [ip, d_, d_, d_, vp, vp, vp]
    L.b200_gauge_action_rect.argtypes = [ip, d_, d_, d_, vp, dp, vp]
    L.b200_link_update.argtypes = [ip, d_, vp, vp, ctypes.c_int, vp]
    L.b200_momentum_update.argtypes = [ip, d_, vp, vp, vp]
    L.b200_momentum_energy.argtypes = [ip, vp, dp, vp]
    L.b200_momentum_from_gauss.argtypes = [ip, vp, vp, vp]
    L.b200_links_axpby.argtypes = [ip, d_, vp, d_, vp, vp]
    L.b200_blas_fill.argtypes = [ctypes.c_int, ctypes.c_size_t, d_, vp, vp]
    L.b200_blas_axpby.argtypes = [ctypes.c_int, ctypes.c_size_t, d_, vp, d_, vp, vp]
    L.b200_blas_dot.argtypes = [ctypes.c_int, ctypes.c_size_t, vp, vp, dp, vp]
    L.b200_field_convert_lex_device.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, vp]
    fp = ctypes.POINTER(ctypes.c_float)
    L.b200_lp_create.argtypes = [ctypes.POINTER(vp), vp, ctypes.c_int, ctypes.c_ulonglong,
                                 ctypes.c_double]
    L.b200_lp_destroy.argtypes = [vp]
    L.b200_lp_nparams.argtypes = [vp]
    L.b200_lp_set_weights.argtypes = [vp, fp, ctypes.c_int]
    L.b200_lp_get_weights.argtypes = [vp, fp, ctypes.c_int, ctypes.c_int]
    L.b200_lp_apply.argtypes = [vp, vp, vp, vp]
    L.b200_lp_loss_grad.argtypes = [vp, vp, vp, dp, vp]
    L.b200_lp_get_grad.argtypes = [vp, fp, ctypes.c_int]
    L.b200_lp_adam_step.argtypes = [vp, ctypes.c_double, vp]
    L.b200_lp_train.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                ctypes.c_int, ctypes.c_double, ctypes.c_ulonglong, dp, dp, vp]
    L.b200_cg_snapshots.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_double,
                                    ctypes.c_int, ip, ctypes.POINTER(vp), ip, vp]
    L.b200_fcg_solve.argtypes = [vp, vp, vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                 ip, ip, dp, vp]
    _lib = L
    return L


def check(rc):
    if rc != 0:
        raise B200Error("b200 error %d: %s" % (rc, lib().b200_last_error().decode()))
    return rc


def tuning_table():
    """The autotuner's choices so far, one text line per kernel configuration."""
    buf = ctypes.create_string_buffer(16384)
    check(lib().b200_tuning_table(buf, len(buf)))
    return buf.value.decode()


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _stream(s):
    """ctypes handle of a torch.cuda.Stream (None: the legacy default stream)."""
    return None if s is None else ctypes.c_void_p(s.cuda_stream)


class Field:
    """One device 5D half-lattice spinor of a DomainWall operator."""

    def __init__(self, op, prec=F64):
        import torch
        self.op = op
        self.prec = prec
        nbytes = lib().b200_dwf_field_bytes(op.handle, prec)
        self.buf = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")

    @property
    def ptr(self):
        return ctypes.c_void_p(self.buf.data_ptr())

    def zero(self):
        """Every value 0, by the library's fill kernel (zero bits are a zero
        value in every storage precision, scales included)."""
        check(lib().b200_blas_fill(1, self.buf.numel() // 4, 0.0, self.ptr, None))


class DomainWall:
    """Mirror of AFopr_Domainwall_5din_eo<AField<REAL, B200>> over the C ABI."""

    def __init__(self, lattice, Ls, mq, M0, b=1.0, c=0.0, alpha=1.0, bc=(1, 1, 1, -1)):
        L = lib()
        self.lattice = list(lattice)
        self.Ls = Ls
        bb = np.full(Ls, b, np.float64) if np.isscalar(b) else np.ascontiguousarray(b, np.float64)
        cc = np.full(Ls, c, np.float64) if np.isscalar(c) else np.ascontiguousarray(c, np.float64)
        h = ctypes.c_void_p()
        check(L.b200_dwf_create(ctypes.byref(h), (ctypes.c_int * 4)(*lattice), Ls, mq, M0,
                                _dp(bb), _dp(cc), alpha, (ctypes.c_int * 4)(*bc)))
        self.handle = h
        self.mode = "D"
        self.nvol = int(np.prod(lattice)) // 2
        self.nreal = 24 * self.nvol * Ls

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and _lib is not None:
            _lib.b200_dwf_destroy(h)
            self.handle = None

    # AFopr interface ---------------------------------------------------
    def field_nin(self):
        return 24 * self.Ls

    def field_nvol(self):
        return self.nvol

    def field_nex(self):
        return 1

    def needs_convert(self):
        return True

    def set_config(self, u_lex):
        u = np.ascontiguousarray(u_lex, np.float64)
        check(lib().b200_dwf_set_config(self.handle, _dp(u), None))

    def set_mode(self, mode):
        self.mode = mode

    def new_field(self, prec=F64):
        return Field(self, prec)

    def convert(self, v, w_host):
        w = np.ascontiguousarray(w_host, np.float64)
        check(lib().b200_field_convert(self.handle, v.prec, v.ptr, _dp(w), None))

    def convert_device(self, v, w_dev):
        """convert() from a float64 CUDA tensor in the reference layout."""
        import torch
        if w_dev.numel() != self.nreal or w_dev.dtype != torch.float64 or not w_dev.is_cuda:
            raise B200Error("convert_device needs a float64 CUDA tensor of %d elements" % self.nreal)
        w_dev = w_dev.contiguous()
        check(lib().b200_field_convert_device(self.handle, v.prec, v.ptr,
                                              ctypes.c_void_p(w_dev.data_ptr()),
                                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))

    def reverse(self, w, out=None):
        if out is None:
            out = np.empty(self.nreal)
        check(lib().b200_field_reverse(self.handle, w.prec, _dp(out), w.ptr, None))
        return out

    def mult(self, v, w, mode=None, stream=None):
        check(lib().b200_dwf_mult(self.handle, w.prec, v.ptr, w.ptr,
                                  (mode or self.mode).encode(), 0, _stream(stream)))

    def mult_dag(self, v, w, mode=None, stream=None):
        check(lib().b200_dwf_mult(self.handle, w.prec, v.ptr, w.ptr,
                                  (mode or self.mode).encode(), 1, _stream(stream)))

    def convert_async(self, v, w_pinned, stream=None):
        """convert() from a page-locked host array (numpy view of a pinned
        torch tensor), queued on `stream` (torch.cuda.Stream or None)."""
        if w_pinned.size != self.nreal or w_pinned.dtype != np.float64:
            raise B200Error("convert_async needs %d float64 values" % self.nreal)
        check(lib().b200_field_convert_async(self.handle, v.prec, v.ptr,
                                             ctypes.c_void_p(w_pinned.ctypes.data), _stream(stream)))

    def reverse_async(self, w, out_pinned, stream=None):
        """reverse() into a page-locked host array, queued on `stream`."""
        if out_pinned.size != self.nreal or out_pinned.dtype != np.float64:
            raise B200Error("reverse_async needs %d float64 values" % self.nreal)
        check(lib().b200_field_reverse_async(self.handle, w.prec, ctypes.c_void_p(out_pinned.ctypes.data),
                                             w.ptr, _stream(stream)))

    def set_async(self, flag):
        """Asynchronous mult/force calls (errors surface at the next
        synchronising call or check_error); default synchronous."""
        check(lib().b200_dwf_set_async(self.handle, int(bool(flag))))

    def check_error(self):
        """Wait for the work queued so far and raise if a hop kernel gave up
        waiting for its bulk copies."""
        check(lib().b200_dwf_check_error(self.handle, None))

    def inject_wait_failure(self, direction):
        """Test hook: TMA-fed hops treat their wait for hop direction
        `direction` (0..7) as timed out; -1 switches it off."""
        check(lib().b200_dwf_inject_wait_failure(self.handle, int(direction)))

    # AField BLAS -------------------------------------------------------
    def axpby(self, y, a, x, b):
        check(lib().b200_field_axpby(self.handle, y.prec, y.ptr, a, x.ptr if x else None, b, None))

    def norm2(self, x):
        r = ctypes.c_double()
        check(lib().b200_field_norm2(self.handle, x.prec, x.ptr, ctypes.byref(r), None))
        return r.value

    def dot(self, x, y):
        r = ctypes.c_double()
        check(lib().b200_field_dot(self.handle, x.prec, x.ptr, y.ptr, ctypes.byref(r), None))
        return r.value

    def copy_convert(self, out, inp):
        check(lib().b200_field_copy_convert(self.handle, out.prec, out.ptr, inp.prec, inp.ptr, None))

    # force (Force_F_Domainwall_eo) --------------------------------------
    def _force_buf(self):
        import torch
        return torch.empty(18 * 2 * self.nvol * 4, dtype=torch.float64, device="cuda")

    def force_udiv1(self, mode, a, b):
        """force_udiv1 in mode H (a=zeta, b=eta) or Hdag (a=eta, b=zeta);
        returns the lexical Field_G(Nvol, 4) force as a numpy array."""
        f = self._force_buf()
        check(lib().b200_dwf_force_udiv1(self.handle, mode.encode(), ctypes.c_void_p(f.data_ptr()),
                                         a.ptr, b.ptr, None))
        return f.cpu().numpy()

    def force_udiv(self, eta):
        f = self._force_buf()
        check(lib().b200_dwf_force_udiv(self.handle, ctypes.c_void_p(f.data_ptr()), eta.ptr, None))
        return f.cpu().numpy()

    # solvers -----------------------------------------------------------
    def shiftcg(self, xs, sigma, b, tol2, maxiter=10000):
        """Multishift CG on DdagD + sigma_i (FP64 fields)."""
        arr = (ctypes.c_void_p * len(xs))(*[f.buf.data_ptr() for f in xs])
        sig = np.ascontiguousarray(sigma, np.float64)
        n = ctypes.c_int()
        d = ctypes.c_double()
        rc = lib().b200_shiftcg_solve(self.handle, arr, _dp(sig), len(xs), b.ptr, maxiter, tol2,
                                      ctypes.byref(n), ctypes.byref(d), None)
        if rc not in (0, -4):
            check(rc)
        return n.value, d.value, rc

    def set_initial_guess(self, use):
        """use_initial_guess for cg / richardson: start from the x passed in."""
        check(lib().b200_solver_set_initial_guess(self.handle, int(bool(use))))

    def set_shift_window(self, window):
        """Residual window of the multishift solver (0: per-iteration updates)."""
        check(lib().b200_shiftcg_set_window(self.handle, int(window)))

    def richardson(self, x, b, inner_prec, tol2, maxiter=100, tol2_inner=1e-8, maxiter_inner=10000):
        """Mixed-precision Richardson (FP64 outer, inner CG in inner_prec)."""
        n = ctypes.c_int()
        ni = ctypes.c_int()
        d = ctypes.c_double()
        rc = lib().b200_richardson_solve(self.handle, inner_prec, x.ptr, b.ptr, maxiter, tol2,
                                         maxiter_inner, tol2_inner, ctypes.byref(n),
                                         ctypes.byref(ni), ctypes.byref(d), None)
        if rc not in (0, -4):
            check(rc)
        return n.value, ni.value, d.value, rc

    def cg(self, x, b, tol2, maxiter=10000):
        n = ctypes.c_int()
        d = ctypes.c_double()
        rc = lib().b200_cg_solve(self.handle, b.prec, x.ptr, b.ptr, maxiter, tol2,
                                 ctypes.byref(n), ctypes.byref(d), None)
        if rc not in (0, -4):
            check(rc)
        return n.value, d.value, rc

    def cg_snapshots(self, x, b, tol2, iters, snaps, maxiter=10000):
        """Plain CG copying x after each iteration in `iters` into `snaps`."""
        it = (ctypes.c_int * len(iters))(*iters)
        arr = (ctypes.c_void_p * len(snaps))(*[f.buf.data_ptr() for f in snaps])
        n = ctypes.c_int()
        rc = lib().b200_cg_snapshots(self.handle, b.prec, x.ptr, b.ptr, maxiter, tol2, len(iters),
                                     it, arr, ctypes.byref(n), None)
        if rc not in (0, -4):
            check(rc)
        return n.value, rc

    def fcg(self, x, b, lp, tol2, maxiter=10000, mtrunc=1):
        """Flexible CG preconditioned by a LearnedPrecond; returns
        (iterations, fallback CG iterations, true relative residual, rc)."""
        n = ctypes.c_int()
        nf = ctypes.c_int()
        d = ctypes.c_double()
        rc = lib().b200_fcg_solve(self.handle, lp.handle, x.ptr, b.ptr, maxiter, tol2, mtrunc,
                                  ctypes.byref(n), ctypes.byref(nf), ctypes.byref(d), None)
        if rc not in (0, -4):
            check(rc)
        return n.value, nf.value, d.value, rc


class GaugeRect:
    """Iwasaki / rectangle gauge action (Force_G_Rectangle, Action_G_Rectangle)
    and the HMC link/momentum updates (Integrator_UpdateU/UpdateP,
    HMC_General::calcH_P) on device copies of lexical Field_G arrays."""

    def __init__(self, lattice, beta, c_plaq=3.648, c_rect=-0.331):
        self.lattice = list(lattice)
        self.beta, self.c_plaq, self.c_rect = beta, c_plaq, c_rect
        self._L = (ctypes.c_int * 4)(*lattice)

    @staticmethod
    def _dev(a):
        import torch
        return torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()

    def force(self, u_lex):
        u = self._dev(u_lex)
        f = u.new_empty(u.shape)
        check(lib().b200_gauge_force_rect(self._L, self.beta, self.c_plaq, self.c_rect,
                                          ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(u.data_ptr()), None))
        return f.cpu().numpy()

    def action(self, u_lex):
        u = self._dev(u_lex)
        h = ctypes.c_double()
        check(lib().b200_gauge_action_rect(self._L, self.beta, self.c_plaq, self.c_rect,
                                           ctypes.c_void_p(u.data_ptr()), ctypes.byref(h), None))
        return h.value

    def link_update(self, u_lex, ip_lex, alpha, nprec=8):
        u = self._dev(u_lex)
        ipd = self._dev(ip_lex)
        check(lib().b200_link_update(self._L, alpha, ctypes.c_void_p(ipd.data_ptr()),
                                     ctypes.c_void_p(u.data_ptr()), nprec, None))
        return u.cpu().numpy()

    def momentum_update(self, ip_lex, force_lex, eps):
        ipd = self._dev(ip_lex)
        f = self._dev(force_lex)
        check(lib().b200_momentum_update(self._L, eps, ctypes.c_void_p(f.data_ptr()),
                                         ctypes.c_void_p(ipd.data_ptr()), None))
        return ipd.cpu().numpy()

    def momentum_energy(self, ip_lex):
        ipd = self._dev(ip_lex)
        h = ctypes.c_double()
        check(lib().b200_momentum_energy(self._L, ctypes.c_void_p(ipd.data_ptr()), ctypes.byref(h), None))
        return h.value


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class LearnedPrecond:
    """Gauge-covariant 3-layer convolution network N ~ (DdagD)^-1 of a
    DomainWall operator (the preconditioner slot of APrecond<AFIELD>,
    src/lib_alt/Solver/aprecond.h).  Fields are FP32 `Field`s of the operator;
    weights are complex numpy arrays of b200_lp_nparams() entries laid out
    [layer][path][out][in]."""

    def __init__(self, op, hidden=8, seed=1, init_noise=0.01):
        self.op = op
        self.hidden = hidden
        h = ctypes.c_void_p()
        check(lib().b200_lp_create(ctypes.byref(h), op.handle, hidden, seed, init_noise))
        self.handle = h
        self.nparams = lib().b200_lp_nparams(h)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and _lib is not None:
            _lib.b200_lp_destroy(h)
            self.handle = None

    def weights(self, deployed=True):
        w = np.empty(2 * self.nparams, np.float32)
        check(lib().b200_lp_get_weights(self.handle, _fp(w), len(w), 1 if deployed else 0))
        return w.view(np.complex64).astype(np.complex128)

    def set_weights(self, w):
        a = np.ascontiguousarray(np.asarray(w, np.complex64)).view(np.float32)
        check(lib().b200_lp_set_weights(self.handle, _fp(a), len(a)))

    def apply(self, z, r):
        check(lib().b200_lp_apply(self.handle, z.ptr, r.ptr, None))

    def loss_grad(self, r, e):
        loss = ctypes.c_double()
        check(lib().b200_lp_loss_grad(self.handle, r.ptr, e.ptr, ctypes.byref(loss), None))
        return loss.value

    def grad(self):
        g = np.empty(2 * self.nparams, np.float32)
        check(lib().b200_lp_get_grad(self.handle, _fp(g), len(g)))
        return g.view(np.complex64).astype(np.complex128)

    def adam_step(self, lr):
        check(lib().b200_lp_adam_step(self.handle, lr, None))

    def train(self, rs, es, epochs, lr, seed=7):
        ra = (ctypes.c_void_p * len(rs))(*[f.buf.data_ptr() for f in rs])
        ea = (ctypes.c_void_p * len(es))(*[f.buf.data_ptr() for f in es])
        l0 = ctypes.c_double()
        l1 = ctypes.c_double()
        check(lib().b200_lp_train(self.handle, len(rs), ra, ea, epochs, lr, seed, ctypes.byref(l0),
                                  ctypes.byref(l1), None))
        return l0.value, l1.value


def cg_training_pairs(op, b, iters, tol2_star=1e-24, maxiter=100000):
    """(residual, error) pairs of plain CG on DdagD x = b for the learned
    preconditioner: the iterate x_k after each iteration in `iters`, the error
    e_k = x* - x_k against a tightly converged x*, and r_k = DdagD e_k (so each
    pair satisfies DdagD e = r exactly).  Returns FP32 fields (rs, es)."""
    xs = Field(op, F64)
    n, _, _ = op.cg(xs, b, tol2_star, maxiter)
    iters = [k for k in iters if k <= n]
    snaps = [Field(op, F64) for _ in iters]
    x = Field(op, F64)
    op.cg_snapshots(x, b, tol2_star, iters, snaps, maxiter)
    rs, es = [], []
    tmp = Field(op, F64)
    for sf in snaps:
        op.axpby(sf, 1.0, xs, -1.0)        # e = x* - x_k
        op.mult(tmp, sf, "DdagD")          # r = DdagD e
        r32 = Field(op, F32)
        e32 = Field(op, F32)
        op.copy_convert(r32, tmp)
        op.copy_convert(e32, sf)
        rs.append(r32)
        es.append(e32)
    return rs, es


class StoutSmear:
    """Mirror of Director_alt_Smear with APE/stout smearing (rho, nsmear) over
    the C ABI: smearing levels on the device and the smeared-force Jacobian."""

    def __init__(self, lattice, rho, nsmear):
        self.lattice = list(lattice)
        self.nsmear = nsmear
        self.nvol = int(np.prod(lattice))
        h = ctypes.c_void_p()
        check(lib().b200_smear_create(ctypes.byref(h), (ctypes.c_int * 4)(*lattice), rho, nsmear))
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and _lib is not None:
            _lib.b200_smear_destroy(h)
            self.handle = None

    def set_config(self, u_lex):
        u = np.ascontiguousarray(u_lex, np.float64)
        check(lib().b200_smear_set_config(self.handle, u.ctypes.data_as(ctypes.c_void_p), 0, None))

    def config_ptr(self, level):
        p = lib().b200_smear_config(self.handle, level)
        if not p:
            raise B200Error("no smearing level %d" % level)
        return p

    def config(self, level):
        out = np.empty(18 * 4 * self.nvol)
        check(lib().b200_smear_get_config(self.handle, level, _dp(out), None))
        return out

    def jacobian(self, sigma_lex):
        import torch
        t = torch.from_numpy(np.ascontiguousarray(sigma_lex, np.float64)).cuda()
        check(lib().b200_smear_jacobian(self.handle, ctypes.c_void_p(t.data_ptr()), None))
        return t.cpu().numpy()


def mult_generator(lattice, force_lex, u_lex):
    """AForce_F::mult_generator on the device: -2 at(U F) per link."""
    import torch
    f = torch.from_numpy(np.ascontiguousarray(force_lex, np.float64)).cuda()
    u = torch.from_numpy(np.ascontiguousarray(u_lex, np.float64)).cuda()
    check(lib().b200_force_mult_generator((ctypes.c_int * 4)(*lattice), ctypes.c_void_p(f.data_ptr()),
                                          ctypes.c_void_p(u.data_ptr()), None))
    return f.cpu().numpy()


class MseriesParallel:
    """RandomNumbers_parallel<RandomNumbers_Mseries> on the device (the
    benchmark driver's random_number_type Mseries_parallel): one M-series
    stream per (z, t) plane, advancing across calls as in the reference
    (src/lib/Tools/randomNumbers_parallel-tmpl.h:160-300).  Draws fill torch
    float64 CUDA tensors in the corelib Field(nin, Nvol, nex) layout."""

    def __init__(self, lattice, seed):
        self.lattice = list(lattice)
        self.nvol = int(np.prod(lattice))
        h = ctypes.c_void_p()
        check(lib().b200_rng_create(ctypes.byref(h), (ctypes.c_int * 4)(*lattice), int(seed)))
        self.handle = h

    def reset(self, seed):
        check(lib().b200_rng_reset(self.handle, int(seed)))

    def _draw(self, fn, nin, nex, out):
        import torch
        n = nin * self.nvol * nex
        if out is None:
            out = torch.empty(n, dtype=torch.float64, device="cuda")
        if out.numel() != n or out.dtype != torch.float64 or not out.is_cuda or not out.is_contiguous():
            raise B200Error("output must be a contiguous float64 CUDA tensor of %d elements" % n)
        check(fn(self.handle, ctypes.c_void_p(out.data_ptr()), int(nin), int(nex),
                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        return out

    def gauss_lex_global(self, nin, nex, out=None):
        """Field(nin, Nvol, nex) of Gaussians with variance 1/2 (nin even)."""
        return self._draw(lib().b200_rng_gauss_lex, nin, nex, out)

    def uniform_lex_global(self, nin, nex, out=None):
        """One uniform number per site in component 0 (the others 0)."""
        return self._draw(lib().b200_rng_uniform_lex, nin, nex, out)

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.b200_rng_destroy(self.handle)
            self.handle = None
