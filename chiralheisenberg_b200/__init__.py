"""chiralheisenberg_b200 -- B200 (sm_100a) implementation of the RHMC fermion
path of j-ostmeyer/chiralHeisenberg (rhmc/cheisdwf.f).

The product is the C-ABI shared library ``libchdwf.so`` (declared in
include/chdwf.h).  This module loads it with ctypes and exposes the
reference's routines under their own names and argument meanings:

    dslash(Phi, R, chi, am, hpin, imass)         rhmc/cheisdwf.f:2634
    dslashd(Phi, R, chi, am, hpin, imass)        rhmc/cheisdwf.f:3071
    qmrherm(Phi, res, am, hpin, imass, anum, aden, ndiag, iflag, chi, dSdchi)
                                                 rhmc/cheisdwf.f:599
    derivs(R, X2, anum, imass, dSdchi)           rhmc/cheisdwf.f:747
    congrad(Phi, res, am, hpin, imass, chi, x)   rhmc/cheisdwf.f:1064
    force(...), hamilton(...)                    rhmc/cheisdwf.f:470, :522

Arrays follow the reference layout: a spinor is complex128 with shape
(2, 4, ksizet, ksize, ksize, kthird) in C order (== Fortran
R(kthird, ksize, ksize, ksizet, 4, 2)); chi is float64 (3, kvol); pp and
dSdchi are float32 (3, kvol).  There is no CPU fallback: if the library is
missing or no GPU is present the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libchdwf.so")

CHDWF_OK, CHDWF_ITER_CAP, CHDWF_NONFINITE, CHDWF_CUDA_ERROR, CHDWF_BAD_ARG = 0, 1, 2, 3, 4

# every symbol include/chdwf.h declares (checked by the CPU test suite)
EXPORTS = (
    "chdwf_create", "chdwf_destroy", "chdwf_set_para", "chdwf_last_error", "chdwf_version",
    "chdwf_dslash", "chdwf_dslashd", "chdwf_qmrherm", "chdwf_derivs", "chdwf_congrad",
    "chdwf_force", "chdwf_hamilton", "chdwf_dslash_dev", "chdwf_qmrherm_dev",
    "chdwf_congrad_dev",
)

_lib = None


class ChdwfError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"chdwf status {code}: {msg}")
        self.code = code


class IterationCapError(ChdwfError):
    pass


def load_library(path: str = LIB_PATH):
    """Load libchdwf.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"{path} not built; run python -m chiralheisenberg_b200.build")
    L = C.CDLL(path)
    P, I, F, D = C.c_void_p, C.c_int, C.c_float, C.c_double
    PI = C.POINTER(C.c_int)
    L.chdwf_create.argtypes = [C.POINTER(P), I, I, I, I]
    L.chdwf_destroy.argtypes = [P]
    L.chdwf_destroy.restype = None
    L.chdwf_set_para.argtypes = [P, F, F, I]
    L.chdwf_last_error.argtypes = [P]
    L.chdwf_last_error.restype = C.c_char_p
    L.chdwf_version.restype = C.c_char_p
    L.chdwf_dslash.argtypes = [P, P, P, P, F, F, I]
    L.chdwf_dslashd.argtypes = [P, P, P, P, F, F, I]
    L.chdwf_qmrherm.argtypes = [P, P, F, PI, F, F, I, P, P, I, I, P, P, P]
    L.chdwf_derivs.argtypes = [P, P, P, D, I, P]
    L.chdwf_congrad.argtypes = [P, P, F, PI, F, F, I, P, P]
    L.chdwf_force.argtypes = [P, P, F, F, F, I, P, P, P, P, P, I, P, P, PI, PI]
    L.chdwf_hamilton.argtypes = [P, P, F, F, F, I, P, P, P, P, I, P, P, PI]
    L.chdwf_dslash_dev.argtypes = [P, P, P, P, F, I, I, P]
    L.chdwf_qmrherm_dev.argtypes = [P, P, F, PI, F, I, P, P, I, I, P, P, P]
    L.chdwf_congrad_dev.argtypes = [P, P, F, PI, F, I, P, P]
    _lib = L
    return L


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _c128(a, shape):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    if a.size != int(np.prod(shape)):
        raise ValueError(f"spinor has {a.size} entries, expected shape {shape}")
    return a


class Lattice:
    """A device context for one lattice size (ksize, ksizet, kthird) and the
    /para/ common block (beta, am3, ibound)."""

    def __init__(self, ksize, ksizet, kthird, beta=0.475, am3=1.0, ibound=-1, device=0):
        self.lib = load_library()
        self.L, self.Lt, self.Ls = ksize, ksizet, kthird
        self.kvol = ksize * ksize * ksizet
        self.kferm = 8 * self.kvol * kthird
        self.shape = (2, 4, ksizet, ksize, ksize, kthird)
        h = C.c_void_p()
        rc = self.lib.chdwf_create(C.byref(h), ksize, ksizet, kthird, device)
        if rc != CHDWF_OK:
            raise ChdwfError(rc, self.lib.chdwf_last_error(None).decode())
        self.h = h
        self.set_para(beta, am3, ibound)

    def set_para(self, beta, am3, ibound=-1):
        self.beta, self.am3, self.ibound = beta, am3, ibound
        self._check(self.lib.chdwf_set_para(self.h, beta, am3, ibound))

    def close(self):
        if getattr(self, "h", None):
            self.lib.chdwf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc == CHDWF_OK:
            return
        msg = self.lib.chdwf_last_error(self.h).decode()
        if rc == CHDWF_ITER_CAP:
            raise IterationCapError(rc, msg)
        raise ChdwfError(rc, msg)

    def _chi(self, chi):
        chi = np.ascontiguousarray(chi, dtype=np.float64)
        if chi.size != 3 * self.kvol:
            raise ValueError("chi must hold 3*kvol values")
        return chi

    # ---- reference routines ------------------------------------------------
    def dslash(self, R, chi, am=0.0, hpin=0.0, imass=1):
        """Phi = M R (rhmc/cheisdwf.f:2634)."""
        R = _c128(R, self.shape)
        out = np.empty(self.shape, dtype=np.complex128)
        self._check(self.lib.chdwf_dslash(self.h, _ptr(out), _ptr(R), _ptr(self._chi(chi)),
                                          am, hpin, imass))
        return out

    def dslashd(self, R, chi, am=0.0, hpin=0.0, imass=1):
        """Phi = M^dagger R (rhmc/cheisdwf.f:3071)."""
        R = _c128(R, self.shape)
        out = np.empty(self.shape, dtype=np.complex128)
        self._check(self.lib.chdwf_dslashd(self.h, _ptr(out), _ptr(R), _ptr(self._chi(chi)),
                                           am, hpin, imass))
        return out

    def qmrherm(self, Phi, res, anum, aden, iflag, chi, am=0.0, hpin=0.0, imass=1, dSdchi=None):
        """Multi-shift solve (rhmc/cheisdwf.f:599).  Returns (x, itercg, dSdchi)."""
        Phi = _c128(Phi, self.shape)
        anum = np.ascontiguousarray(anum, dtype=np.float64)
        aden = np.ascontiguousarray(aden, dtype=np.float64)
        if len(anum) != len(aden) + 1:
            raise ValueError("anum must hold a0..a_n and aden sigma_1..sigma_n")
        x = np.empty(self.shape, dtype=np.complex128)
        if dSdchi is None:
            dSdchi = np.zeros((3, self.kvol), dtype=np.float32)
        it = C.c_int(0)
        self._check(self.lib.chdwf_qmrherm(self.h, _ptr(Phi), res, C.byref(it), am, hpin, imass,
                                           _ptr(anum), _ptr(aden), len(aden), iflag,
                                           _ptr(self._chi(chi)), _ptr(x), _ptr(dSdchi)))
        return x, it.value, dSdchi

    def derivs(self, R, X2, anum, imass, dSdchi):
        """dSdchi += one pole's force term (rhmc/cheisdwf.f:747)."""
        assert dSdchi.dtype == np.float32 and dSdchi.flags.c_contiguous
        self._check(self.lib.chdwf_derivs(self.h, _ptr(_c128(R, self.shape)),
                                          _ptr(_c128(X2, self.shape)), float(anum), imass,
                                          _ptr(dSdchi)))
        return dSdchi

    def congrad(self, Phi, res, chi, x0, am=0.0, hpin=0.0, imass=1):
        """CGNE from initial guess x0 (rhmc/cheisdwf.f:1064).  Returns (x, itercg)."""
        x = _c128(x0, self.shape).copy()
        it = C.c_int(0)
        self._check(self.lib.chdwf_congrad(self.h, _ptr(_c128(Phi, self.shape)), res,
                                           C.byref(it), am, hpin, imass, _ptr(self._chi(chi)),
                                           _ptr(x)))
        return x, it.value

    def force(self, Phi, res1, chi, remez2g, am=0.0, hpin=0.0, imass=1):
        """dSdchi (rhmc/cheisdwf.f:470).  remez2g = (anum, aden, bnum, bden)."""
        an, ad, bn, bd = [np.ascontiguousarray(v, dtype=np.float64) for v in remez2g]
        dS = np.empty((3, self.kvol), dtype=np.float32)
        x = np.empty(self.shape, dtype=np.complex128)
        itg, itf = C.c_int(0), C.c_int(0)
        self._check(self.lib.chdwf_force(self.h, _ptr(_c128(Phi, self.shape)), res1, am, hpin,
                                         imass, _ptr(self._chi(chi)), _ptr(an), _ptr(ad),
                                         _ptr(bn), _ptr(bd), len(ad), _ptr(dS), _ptr(x),
                                         C.byref(itg), C.byref(itf)))
        return dS, x, itg.value, itf.value

    def hamilton(self, Phi, res2, chi, pp, bnum, bden, am=0.0, hpin=0.0, imass=1):
        """(h, hg, hp, s, hf), x, itercg (rhmc/cheisdwf.f:522)."""
        bn = np.ascontiguousarray(bnum, dtype=np.float64)
        bd = np.ascontiguousarray(bden, dtype=np.float64)
        pp = np.ascontiguousarray(pp, dtype=np.float32)
        out = np.zeros(5, dtype=np.float64)
        x = np.empty(self.shape, dtype=np.complex128)
        it = C.c_int(0)
        self._check(self.lib.chdwf_hamilton(self.h, _ptr(_c128(Phi, self.shape)), res2, am, hpin,
                                            imass, _ptr(self._chi(chi)), _ptr(pp), _ptr(bn),
                                            _ptr(bd), len(bd), _ptr(out), _ptr(x), C.byref(it)))
        return tuple(out), x, it.value


def version() -> str:
    return load_library().chdwf_version().decode()
