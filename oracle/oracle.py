"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the CPU
baseline leg of bench.py, never by the product path.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        lib = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        lib.oracle_dwf_create.restype = ctypes.c_void_p
        lib.oracle_dwf_create.argtypes = [ip, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double, dp, dp, ctypes.c_double, ip]
        lib.oracle_dwf_destroy.argtypes = [ctypes.c_void_p]
        lib.oracle_dwf_set_links.argtypes = [ctypes.c_void_p, dp]
        lib.oracle_dwf_mult.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, dp, dp]
        lib.oracle_dwf_mult.restype = ctypes.c_int
        lib.oracle_cg.argtypes = [ctypes.c_void_p, dp, dp, ctypes.c_double, ctypes.c_int, ip, dp]
        lib.oracle_cg.restype = ctypes.c_int
        lib.oracle_shiftcg.argtypes = [ctypes.c_void_p, dp, dp, ctypes.c_int, dp,
                                       ctypes.c_double, ctypes.c_int, ip, dp]
        lib.oracle_shiftcg.restype = ctypes.c_int
        lib.oracle_dwf_force_udiv1.argtypes = [ctypes.c_void_p, ctypes.c_char_p, dp, dp, dp]
        lib.oracle_dwf_force_udiv1.restype = ctypes.c_int
        lib.oracle_dwf_force_udiv.argtypes = [ctypes.c_void_p, dp, dp]
        lib.oracle_dwf_force_udiv.restype = ctypes.c_int
        _LIB = lib
    return _LIB


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class OracleDWF:
    """Even-odd 5D domain-wall operator of the reference corelib, on the CPU."""

    def __init__(self, lattice, Ls, mq, M0, b=1.0, c=0.0, alpha=1.0, bc=(1, 1, 1, -1)):
        lib = _lib()
        self.lattice = list(lattice)
        self.Ls = Ls
        L = (ctypes.c_int * 4)(*lattice)
        bcv = (ctypes.c_int * 4)(*bc)
        bb = np.full(Ls, b, dtype=np.float64) if np.isscalar(b) else np.asarray(b, np.float64)
        cc = np.full(Ls, c, dtype=np.float64) if np.isscalar(c) else np.asarray(c, np.float64)
        self._h = lib.oracle_dwf_create(L, Ls, mq, M0, _dp(bb), _dp(cc), alpha, bcv)
        if not self._h:
            raise ValueError("invalid oracle parameters")
        self.n = 24 * (int(np.prod(lattice)) // 2) * Ls

    def __del__(self):
        if getattr(self, "_h", None):
            _lib().oracle_dwf_destroy(self._h)
            self._h = None

    def set_links(self, u_lex):
        u = np.ascontiguousarray(u_lex, dtype=np.float64)
        _lib().oracle_dwf_set_links(self._h, _dp(u))

    def mult(self, mode, w, dag=False):
        w = np.ascontiguousarray(w, dtype=np.float64)
        out = np.empty(self.n)
        rc = _lib().oracle_dwf_mult(self._h, mode.encode(), int(dag), _dp(out), _dp(w))
        if rc != 0:
            raise ValueError("unknown mode " + mode)
        return out

    def cg(self, b, tol2, maxiter=10000):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty(self.n)
        nconv = ctypes.c_int(0)
        diff = ctypes.c_double(0)
        rc = _lib().oracle_cg(self._h, _dp(x), _dp(b), tol2, maxiter,
                              ctypes.byref(nconv), ctypes.byref(diff))
        return x, nconv.value, diff.value, rc

    def force_udiv1(self, mode, a, b):
        """Force_F_Domainwall_eo::force_udiv1 in mode H (a=zeta, b=eta) or
        Hdag (a=eta, b=zeta); lexical Field_G(Nvol, 4) result."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        f = np.empty(18 * int(np.prod(self.lattice)) * 4)
        rc = _lib().oracle_dwf_force_udiv1(self._h, mode.encode(), _dp(f), _dp(a), _dp(b))
        if rc != 0:
            raise ValueError(mode)
        return f

    def force_udiv(self, eta):
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        f = np.empty(18 * int(np.prod(self.lattice)) * 4)
        _lib().oracle_dwf_force_udiv(self._h, _dp(f), _dp(eta))
        return f

    def shiftcg(self, b, sigma, tol2, maxiter=10000):
        b = np.ascontiguousarray(b, dtype=np.float64)
        sig = np.ascontiguousarray(sigma, dtype=np.float64)
        x = np.empty(self.n * len(sig))
        nconv = ctypes.c_int(0)
        diff = ctypes.c_double(0)
        rc = _lib().oracle_shiftcg(self._h, _dp(x), _dp(sig), len(sig), _dp(b), tol2,
                                   maxiter, ctypes.byref(nconv), ctypes.byref(diff))
        return x.reshape(len(sig), self.n), nconv.value, diff.value, rc
