"""ctypes bindings to the CPU oracle (oracle/_build/liboracle.so).

Test infrastructure only: imported by tests/, by ``__graft_entry__.smoke`` and
by the CPU-baseline legs of ``bench.py``.  The product package never imports
this module.  Array layouts are those of the reference (rhmc/cheisdwf.f):
spinors complex128 of shape (2, 4, Lt, L, L, Ls) in C order == Fortran
R(Ls, L, L, Lt, 4, 2); chi float64 (3, Lt, L, L) == chi(kvol, 3).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (gcc, no fused multiply-add)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class Lat(C.Structure):
    _fields_ = [("L", C.c_int), ("Lt", C.c_int), ("Ls", C.c_int),
                ("beta", C.c_float), ("am3", C.c_float), ("ibound", C.c_int),
                ("threads", C.c_int)]


class Rng(C.Structure):
    _fields_ = [("ds", C.c_double * 2), ("v", C.c_float * 97), ("yran", C.c_float),
                ("yrun", C.c_float), ("idum", C.c_int)]


class Remez(C.Structure):
    _fields_ = [("n", C.c_int), ("anum", C.c_double * 32), ("aden", C.c_double * 32),
                ("bnum", C.c_double * 32), ("bden", C.c_double * 32)]


class TrajRec(C.Structure):
    _fields_ = [("H0", C.c_double), ("H1", C.c_double), ("dH", C.c_double), ("dS", C.c_double),
                ("S0", C.c_double), ("S1", C.c_double), ("hg", C.c_double), ("hp", C.c_double),
                ("y", C.c_float), ("x", C.c_float), ("accepted", C.c_int), ("nsteps", C.c_int),
                ("it_pf", C.c_int), ("it_h0", C.c_int), ("it_h1", C.c_int),
                ("it_guid", C.c_double), ("it_force", C.c_double), ("nforce", C.c_int),
                ("action", C.c_float), ("gaction", C.c_float), ("paction", C.c_float),
                ("vel2", C.c_float), ("measured", C.c_int), ("cond", C.c_float * 3),
                ("susc", C.c_float * 3), ("condmod", C.c_float), ("susctot", C.c_float),
                ("ancgm", C.c_float)]


class State(C.Structure):
    _fields_ = [("lat", Lat), ("rng", Rng), ("r2", Remez), ("r4", Remez), ("r2g", Remez),
                ("dt", C.c_float), ("am", C.c_float), ("hpin", C.c_float),
                ("imass", C.c_int), ("iterl", C.c_int), ("iprint", C.c_int), ("measure", C.c_int),
                ("rescga", C.c_float), ("rescgg", C.c_float), ("rescgm", C.c_float),
                ("chi", C.POINTER(C.c_double)), ("chit", C.POINTER(C.c_double)),
                ("pp", C.POINTER(C.c_float)), ("dSdchi", C.POINTER(C.c_float)),
                ("Phi", C.POINTER(C.c_double)), ("X1", C.POINTER(C.c_double)),
                ("R", C.POINTER(C.c_double)), ("ps", C.POINTER(C.c_float)),
                ("cferm", C.POINTER(C.c_float)), ("isweep", C.c_int),
                ("gaction", C.c_float)]


class HmcRec(C.Structure):
    _fields_ = [("H0", C.c_double), ("H1", C.c_double), ("dH", C.c_double), ("dS", C.c_double),
                ("S0", C.c_double), ("S1", C.c_double), ("hg", C.c_double), ("hp", C.c_double),
                ("y", C.c_float), ("x", C.c_float), ("drew_x", C.c_int), ("accepted", C.c_int),
                ("nsteps", C.c_int), ("it_h0", C.c_int), ("it_h1", C.c_int),
                ("it_force", C.c_int), ("nforce", C.c_int), ("action", C.c_float),
                ("gaction", C.c_float), ("paction", C.c_float), ("vel2", C.c_float),
                ("measured", C.c_int), ("cond", C.c_float * 3), ("susc", C.c_float * 3),
                ("condmod", C.c_float), ("susctot", C.c_float)]


class HmcState(C.Structure):
    _fields_ = [("lat", Lat), ("rng", Rng), ("dt", C.c_float), ("am", C.c_float),
                ("imass", C.c_int), ("iterl", C.c_int), ("iprint", C.c_int),
                ("rescga", C.c_float), ("rescgg", C.c_float),
                ("chi", C.POINTER(C.c_float)), ("chit", C.POINTER(C.c_float)),
                ("pp", C.POINTER(C.c_float)), ("dSdchi", C.POINTER(C.c_float)),
                ("Phi", C.POINTER(C.c_float)), ("X0", C.POINTER(C.c_float)),
                ("X1", C.POINTER(C.c_float)), ("R", C.POINTER(C.c_float)),
                ("ps", C.POINTER(C.c_float)), ("isweep", C.c_int), ("itot", C.c_int),
                ("naccp", C.c_int), ("action", C.c_float), ("gaction", C.c_float),
                ("paction", C.c_float), ("actiona", C.c_float), ("vel2a", C.c_float),
                ("yav", C.c_float), ("yyav", C.c_float)]


class ThrRec(C.Structure):
    _fields_ = [("H0", C.c_double), ("H1", C.c_double), ("dH", C.c_double), ("dS", C.c_double),
                ("S0", C.c_double), ("S1", C.c_double), ("hg", C.c_double), ("hp", C.c_double),
                ("y", C.c_float), ("x", C.c_float), ("drew_x", C.c_int), ("accepted", C.c_int),
                ("nsteps", C.c_int), ("it_pf", C.c_int), ("it_pfpv", C.c_int),
                ("it_h0", C.c_int), ("it_h0pv", C.c_int), ("it_h1", C.c_int),
                ("it_h1pv", C.c_int), ("it_force", C.c_int * 4), ("nforce", C.c_int),
                ("action", C.c_float), ("gaction", C.c_float), ("paction", C.c_float),
                ("vel2", C.c_float), ("measured", C.c_int), ("pbp", C.c_float),
                ("ancgm", C.c_float)]


class ThrState(C.Structure):
    _fields_ = [("lat", Lat), ("rng", Rng), ("r2", Remez), ("r4", Remez), ("r2g", Remez),
                ("r4g", Remez), ("dt", C.c_float), ("am", C.c_float), ("imass", C.c_int),
                ("iterl", C.c_int), ("iprint", C.c_int), ("rescga", C.c_float),
                ("rescgg", C.c_float), ("theta", C.POINTER(C.c_float)),
                ("thetat", C.POINTER(C.c_float)), ("pp", C.POINTER(C.c_float)),
                ("dSdpi", C.POINTER(C.c_float)), ("ut", C.POINTER(C.c_double)),
                ("Phi", C.POINTER(C.c_double)), ("X1", C.POINTER(C.c_double)),
                ("R", C.POINTER(C.c_double)), ("Phi0", C.POINTER(C.c_double)),
                ("ps", C.POINTER(C.c_float)), ("isweep", C.c_int), ("itot", C.c_int),
                ("naccp", C.c_int), ("action", C.c_float), ("gaction", C.c_float),
                ("paction", C.c_float), ("actiona", C.c_float), ("vel2a", C.c_float),
                ("yav", C.c_float), ("yyav", C.c_float)]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or (
                os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "chdwf_oracle.c"))):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.c_void_p
        L.orc_rranf.restype = C.c_float
        L.orc_rano.restype = C.c_float
        L.orc_rranget.restype = C.c_double
        L.orc_rranset.argtypes = [P, C.c_double]
        L.orc_rng_startup.argtypes = [P, C.c_double]
        L.orc_gauss0.argtypes = [P, C.c_int64, P]
        L.orc_gaussp.argtypes = [P, C.c_int64, P]
        for f in (L.orc_dslash, L.orc_dslashd, L.orc_dslash_v1):
            f.argtypes = [P, P, P, P, C.c_float, C.c_float, C.c_int]
        L.orc_qmrherm.argtypes = [P, P, C.c_float, P, C.c_float, C.c_float, C.c_int, P, P,
                                  C.c_int, C.c_int, P, P, P, C.c_int]
        L.orc_derivs.argtypes = [P, P, P, C.c_double, C.c_int, P]
        L.orc_congrad.argtypes = [P, P, C.c_float, P, C.c_float, C.c_float, C.c_int, P, P]
        L.orc_force.argtypes = [P, P, C.c_float, C.c_float, C.c_float, C.c_int, P, P, P, P, P, P]
        L.orc_hamilton.argtypes = [P, P, C.c_float, C.c_float, C.c_float, C.c_int, P, P, P, P,
                                   P, P]
        L.orc_fermion.argtypes = [P, P, C.c_float, C.c_float, C.c_float, C.c_int, P, P, P, P]
        L.orc_fermion.restype = C.c_float
        L.orc_measure.argtypes = [P, P, C.c_float, C.c_float, C.c_float, C.c_int, P, P,
                                  C.POINTER(C.c_float), C.POINTER(C.c_float),
                                  C.POINTER(C.c_float), P]
        L.orc_state_new.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                    C.c_float, C.c_float, C.c_int, C.c_int]
        L.orc_state_new.restype = C.POINTER(State)
        L.orc_state_free.argtypes = [C.POINTER(State)]
        L.orc_state_set_remez.argtypes = [C.POINTER(State), C.c_int, P]
        L.orc_sweep.argtypes = [C.POINTER(State), P]
        L.orc_read_remez.argtypes = [C.c_char_p, C.c_int, P]
        L.orc_hmc_dslash.argtypes = [P, P, P, P, C.c_int, C.c_int]
        L.orc_hmc_congrad.argtypes = [P, P, C.c_float, P, C.c_int, P, P]
        L.orc_hmc_derivs.argtypes = [P, P, P, C.c_int, P]
        L.orc_hmc_force.argtypes = [P, P, P, P, P, C.c_float, C.c_int, P, P]
        L.orc_hmc_hamilton.argtypes = [P, P, P, P, P, C.c_float, C.c_int, P, P]
        L.orc_hmc_new.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                  C.c_float, C.c_int, C.c_int]
        L.orc_hmc_new.restype = C.POINTER(HmcState)
        L.orc_hmc_free.argtypes = [C.POINTER(HmcState)]
        L.orc_hmc_sweep.argtypes = [C.POINTER(HmcState), P]
        L.orc_thr_set_alphatild_fp64.argtypes = [C.c_int]
        L.orc_thr_set_alphatild_fp64.restype = None
        L.orc_thr_coef.argtypes = [P, P, P]
        L.orc_thr_dslash.argtypes = [P, P, P, P, C.c_float, C.c_int, C.c_int]
        L.orc_thr_derivs.argtypes = [P, P, P, C.c_double, C.c_int, P]
        L.orc_thr_qmrherm.argtypes = [P, P, C.c_float, P, C.c_float, C.c_int, P, P, C.c_int,
                                      C.c_int, P, P, P, P]
        L.orc_thr_new.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                  C.c_float, C.c_int, C.c_int]
        L.orc_thr_new.restype = C.POINTER(ThrState)
        L.orc_thr_free.argtypes = [C.POINTER(ThrState)]
        L.orc_thr_set_remez.argtypes = [C.POINTER(ThrState), C.c_int, P]
        L.orc_thr_force.argtypes = [C.POINTER(ThrState), C.c_float, P]
        L.orc_thr_hamilton.argtypes = [C.POINTER(ThrState), C.c_float, P, P]
        L.orc_thr_sweep.argtypes = [C.POINTER(ThrState), P]
        L.orc_thr_congrad.argtypes = [P, P, C.c_float, P, C.c_float, C.c_int, P, P]
        L.orc_thr_measure.argtypes = [P, P, C.c_float, C.c_float, C.c_int, P,
                                      C.POINTER(C.c_float), C.POINTER(C.c_float),
                                      C.POINTER(C.c_float), P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def make_lat(L, Lt, Ls, beta=0.475, am3=1.0, ibound=-1, threads=1) -> Lat:
    return Lat(L, Lt, Ls, beta, am3, ibound, threads)


def spinor_shape(lat: Lat):
    return (2, 4, lat.Lt, lat.L, lat.L, lat.Ls)


def kvol(lat: Lat) -> int:
    return lat.L * lat.L * lat.Lt


def dslash(lat, R, chi, hpin=0.0, imass=1, dag=False, am=0.0, v1=False):
    R = np.ascontiguousarray(R, dtype=np.complex128)
    chi = np.ascontiguousarray(chi, dtype=np.float64)
    out = np.empty_like(R)
    f = lib().orc_dslashd if dag else (lib().orc_dslash_v1 if v1 else lib().orc_dslash)
    f(C.byref(lat), _p(out), _p(R), _p(chi), am, hpin, imass)
    return out


def qmrherm(lat, Phi, chi, anum, aden, res, iflag=0, hpin=0.0, imass=1, dSdchi=None,
            niterc=5000, am=0.0):
    Phi = np.ascontiguousarray(Phi, dtype=np.complex128)
    chi = np.ascontiguousarray(chi, dtype=np.float64)
    anum = np.ascontiguousarray(anum, dtype=np.float64)
    aden = np.ascontiguousarray(aden, dtype=np.float64)
    x = np.empty_like(Phi)
    if dSdchi is None:
        dSdchi = np.zeros((3, kvol(lat)), dtype=np.float32)
    it = C.c_int(0)
    st = lib().orc_qmrherm(C.byref(lat), _p(Phi), res, C.byref(it), am, hpin, imass, _p(anum),
                           _p(aden), len(aden), iflag, _p(chi), _p(x), _p(dSdchi), niterc)
    return x, it.value, st, dSdchi


def derivs(lat, R, X2, anum, imass, dSdchi):
    lib().orc_derivs(C.byref(lat), _p(np.ascontiguousarray(R)), _p(np.ascontiguousarray(X2)),
                     float(anum), imass, _p(dSdchi))
    return dSdchi


def congrad(lat, Phi, chi, x0, res, hpin=0.0, imass=1, am=0.0):
    x = np.ascontiguousarray(x0, dtype=np.complex128).copy()
    it = C.c_int(0)
    capped = lib().orc_congrad(C.byref(lat), _p(np.ascontiguousarray(Phi)), res, C.byref(it), am,
                               hpin, imass, _p(np.ascontiguousarray(chi)), _p(x))
    return x, it.value, capped


# ---- the HMC predecessor (mh/cheisdwf_hmc.f), single precision ----------
def hmc_dslash(lat, R, chi, imass=1, dag=False):
    R = np.ascontiguousarray(R, dtype=np.complex64)
    chi = np.ascontiguousarray(chi, dtype=np.float32)
    out = np.empty_like(R)
    lib().orc_hmc_dslash(C.byref(lat), _p(out), _p(R), _p(chi), imass, 1 if dag else 0)
    return out


def hmc_congrad(lat, Phi, chi, x0, res, imass=1):
    x = np.ascontiguousarray(x0, dtype=np.complex64).copy()
    it = C.c_int(0)
    capped = lib().orc_hmc_congrad(C.byref(lat), _p(np.ascontiguousarray(Phi, dtype=np.complex64)),
                                   res, C.byref(it), imass,
                                   _p(np.ascontiguousarray(chi, dtype=np.float32)), _p(x))
    return x, it.value, capped


def hmc_derivs(lat, X1, chi, imass=1):
    dS = np.empty((3, kvol(lat)), dtype=np.float32)
    lib().orc_hmc_derivs(C.byref(lat), _p(np.ascontiguousarray(X1, dtype=np.complex64)),
                         _p(np.ascontiguousarray(chi, dtype=np.float32)), imass, _p(dS))
    return dS


class HmcSweeper:
    """The main loop of mh/cheisdwf_hmc.f (:140-320) over the oracle."""

    def __init__(self, L, Lt, Ls, beta, am3, dt, am, imass, iterl, chi=None, seed=None,
                 iprint=5):
        self.lib = lib()
        self.st = self.lib.orc_hmc_new(L, Lt, Ls, beta, am3, dt, am, imass, iterl)
        self.st.contents.iprint = iprint
        self.kvol = L * L * Lt
        if chi is not None:
            self.chi[:] = np.asarray(chi, dtype=np.float32).reshape(-1)
        if seed is not None:
            self.lib.orc_rng_startup(C.byref(self.st.contents.rng), float(seed))

    @property
    def chi(self):
        return np.ctypeslib.as_array(self.st.contents.chi, shape=(3 * self.kvol,))

    def seed(self):
        return self.lib.orc_rranget(C.byref(self.st.contents.rng))

    def sweep(self) -> HmcRec:
        rec = HmcRec()
        self.lib.orc_hmc_sweep(self.st, C.byref(rec))
        return rec

    def close(self):
        if self.st:
            self.lib.orc_hmc_free(self.st)
            self.st = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- the bulk Thirring RHMC (bulk_rhmc.f) ---------------------------------
def thr_alphatild_fp64(on: bool):
    """Thirring qmrherm's alphatild: False (default) sums in REAL*4 element by
    element as bulk_rhmc.f:691-694; True sums in REAL*8 and rounds once, the
    grouping the GPU's parallel reduction follows."""
    lib().orc_thr_set_alphatild_fp64(1 if on else 0)


def thr_shape(lat):
    return (4, lat.Lt, lat.L, lat.L, lat.Ls)


def thr_coef(lat, theta):
    u = np.empty((3, kvol(lat)), dtype=np.complex128)
    lib().orc_thr_coef(C.byref(lat), _p(np.ascontiguousarray(theta, dtype=np.float32)), _p(u))
    return u


def thr_dslash(lat, R, u, am, imass=1, dag=False):
    R = np.ascontiguousarray(R, dtype=np.complex128)
    out = np.empty_like(R)
    lib().orc_thr_dslash(C.byref(lat), _p(out), _p(R), _p(np.ascontiguousarray(u)), am, imass,
                         1 if dag else 0)
    return out


def thr_derivs(lat, R, X2, anum, iflag, dSdpi=None):
    dS = np.zeros((3, kvol(lat)), dtype=np.float32) if dSdpi is None else dSdpi
    lib().orc_thr_derivs(C.byref(lat), _p(np.ascontiguousarray(R)), _p(np.ascontiguousarray(X2)),
                         float(anum), iflag, _p(dS))
    return dS


def thr_qmrherm(lat, Phi, u, res, am, imass, anum, aden, iflag=0, Phi0=None, dSdpi=None):
    """Returns (x, itercg, capped, Phi0, dSdpi)."""
    n = len(aden)
    sh = thr_shape(lat)
    x = np.empty(sh, dtype=np.complex128)
    P0 = np.zeros((n,) + sh, dtype=np.complex128) if Phi0 is None else Phi0
    dS = np.zeros((3, kvol(lat)), dtype=np.float32) if dSdpi is None else dSdpi
    it = C.c_int(0)
    capped = lib().orc_thr_qmrherm(
        C.byref(lat), _p(np.ascontiguousarray(Phi, dtype=np.complex128)), res, C.byref(it), am,
        imass, _p(np.ascontiguousarray(anum, dtype=np.float64)),
        _p(np.ascontiguousarray(aden, dtype=np.float64)), n, iflag, _p(np.ascontiguousarray(u)),
        _p(x), _p(P0), _p(dS))
    return x, it.value, capped, P0, dS


def thr_congrad(lat, Phi, u, x0, res, am, imass=1):
    x = np.ascontiguousarray(x0, dtype=np.complex128).copy()
    it = C.c_int(0)
    capped = lib().orc_thr_congrad(C.byref(lat), _p(np.ascontiguousarray(Phi, dtype=np.complex128)),
                                   res, C.byref(it), am, imass, _p(np.ascontiguousarray(u)), _p(x))
    return x, it.value, capped


def thr_measure(lat, rand, u, res, am, imass):
    """measure of bulk_rhmc.f on the generator of a Rand:
    (psibarpsi, susclsing, aviter, parts[10, 4])."""
    parts = np.empty((10, 4), dtype=np.float64)
    pb, su, av = C.c_float(), C.c_float(), C.c_float()
    lib().orc_thr_measure(C.byref(lat), C.byref(rand.g), res, am, imass,
                          _p(np.ascontiguousarray(u)), C.byref(pb), C.byref(su), C.byref(av),
                          _p(parts))
    return pb.value, su.value, av.value, parts


class ThrSweeper:
    """The main loop of bulk_rhmc.f (:201-400) over the oracle, with measure
    on every iprint-th sweep."""

    def __init__(self, L, Lt, Ls, beta, am3, dt, am, imass, iterl, r2, r4, r2g, r4g,
                 theta=None, seed=None, iprint=5):
        self.lib = lib()
        self.st = self.lib.orc_thr_new(L, Lt, Ls, beta, am3, dt, am, imass, iterl)
        self.st.contents.iprint = iprint
        for which, r in ((2, r2), (4, r4), (22, r2g), (44, r4g)):
            self.lib.orc_thr_set_remez(self.st, which, C.byref(r))
        self.kvol = L * L * Lt
        if theta is not None:
            self.theta[:] = np.asarray(theta, dtype=np.float32).reshape(-1)
        if seed is not None:
            self.lib.orc_rng_startup(C.byref(self.st.contents.rng), float(seed))

    @property
    def theta(self):
        return np.ctypeslib.as_array(self.st.contents.theta, shape=(3 * self.kvol,))

    def seed(self):
        return self.lib.orc_rranget(C.byref(self.st.contents.rng))

    def sweep(self) -> ThrRec:
        rec = ThrRec()
        self.lib.orc_thr_sweep(self.st, C.byref(rec))
        return rec

    def close(self):
        if self.st:
            self.lib.orc_thr_free(self.st)
            self.st = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def remez_struct(a0, anum, aden, b0, bnum, bden) -> Remez:
    r = Remez()
    r.n = len(aden)
    r.anum[0] = a0
    r.bnum[0] = b0
    for k in range(r.n):
        r.anum[k + 1] = anum[k]
        r.aden[k] = aden[k]
        r.bnum[k + 1] = bnum[k]
        r.bden[k] = bden[k]
    return r


def read_remez(path, n) -> Remez:
    r = Remez()
    rc = lib().orc_read_remez(path.encode(), n, C.byref(r))
    if rc != 0:
        raise IOError(f"cannot read remez file {path}: {rc}")
    return r


class Sweeper:
    """The main loop of program dwf3d (cheisdwf.f:207-399) over the oracle."""

    def __init__(self, L, Lt, Ls, beta, am3, dt, am, hpin, imass, iterl, remez2, remez4,
                 remez2g, chi=None, seed=None, measure=True, threads=1):
        self.lib = lib()
        self.st = self.lib.orc_state_new(L, Lt, Ls, beta, am3, dt, am, hpin, imass, iterl)
        self.st.contents.lat.threads = threads
        self.st.contents.measure = 1 if measure else 0
        for which, r in ((2, remez2), (4, remez4), (22, remez2g)):
            self.lib.orc_state_set_remez(self.st, which, C.byref(r))
        self.kvol = L * L * Lt
        if chi is not None:
            self.chi[:] = np.asarray(chi, dtype=np.float64).reshape(-1)
        if seed is not None:
            self.lib.orc_rng_startup(C.byref(self.st.contents.rng), float(seed))

    @property
    def chi(self):
        return np.ctypeslib.as_array(self.st.contents.chi, shape=(3 * self.kvol,))

    @property
    def cferm(self):
        Lt = self.st.contents.lat.Lt
        return np.ctypeslib.as_array(self.st.contents.cferm, shape=(2, 2, Lt, 2)).copy()

    def sweep(self) -> TrajRec:
        rec = TrajRec()
        self.lib.orc_sweep(self.st, C.byref(rec))
        return rec

    def measure(self, res=1e-9):
        """measure() (cheisdwf.f:1164-1453) on chi with the state's am, hpin,
        imass and generator: (psibarpsi, susclsing, aviter, parts[10, 4])."""
        st = self.st.contents
        xi = np.empty(2 * 8 * self.kvol * st.lat.Ls, dtype=np.float64)
        parts = np.empty((10, 4), dtype=np.float64)
        pb, su, av = C.c_float(), C.c_float(), C.c_float()
        self.lib.orc_measure(C.byref(st.lat), C.byref(st.rng), res, st.am, st.hpin, st.imass,
                             C.cast(st.chi, C.c_void_p), _p(xi), C.byref(pb), C.byref(su),
                             C.byref(av), _p(parts))
        return pb.value, su.value, av.value, parts

    def close(self):
        if self.st:
            self.lib.orc_state_free(self.st)
            self.st = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Rand:
    """The reference RNG (RRANF + rano) on the oracle."""

    def __init__(self, seed):
        self.g = Rng()
        lib().orc_rng_startup(C.byref(self.g), float(seed))

    def seed(self) -> float:
        return lib().orc_rranget(C.byref(self.g))

    def rano(self, which="yran") -> float:
        y = C.c_float(getattr(self.g, which))
        v = lib().orc_rano(C.byref(self.g), C.byref(y))
        setattr(self.g, which, y.value)
        return v

    def gauss0(self, kvol):
        ps = np.empty((2, kvol), dtype=np.float32)
        lib().orc_gauss0(C.byref(self.g), kvol, _p(ps))
        return ps

    def gaussp(self, kvol):
        ps = np.empty((2, kvol), dtype=np.float32)
        lib().orc_gaussp(C.byref(self.g), kvol, _p(ps))
        return ps
