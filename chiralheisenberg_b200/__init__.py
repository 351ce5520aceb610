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
CHDWF_NOT_FOUND = 5

# every symbol include/*.h declares (checked by the CPU test suite)
EXPORTS = (
    "chdwf_create", "chdwf_destroy", "chdwf_set_para", "chdwf_last_error", "chdwf_version",
    "chdwf_dslash", "chdwf_dslashd", "chdwf_qmrherm", "chdwf_derivs", "chdwf_congrad",
    "chdwf_force", "chdwf_hamilton", "chdwf_dslash_dev", "chdwf_qmrherm_dev",
    "chdwf_congrad_dev",
    "chdwf_traj_set_remez", "chdwf_traj_set_chi", "chdwf_traj_get_chi", "chdwf_traj_begin",
    "chdwf_traj_heatbath", "chdwf_traj_heatbath_dev", "chdwf_traj_set_momenta",
    "chdwf_traj_get_momenta", "chdwf_traj_hamilton", "chdwf_traj_force", "chdwf_traj_get_force",
    "chdwf_traj_get_phi", "chdwf_traj_update_momenta", "chdwf_traj_update_chi",
    "chdwf_traj_accept", "chdwf_traj_sync", "chdwf_traj_propagator",
    "chdwf_traj_set_momenta_dev", "chdwf_timing", "chdwf_timing_read", "chdwf_prog_stage",
    "chdwf_timing_read_chunks",
    "chdwf_get_stream", "chdwf_kernel_launches", "chdwf_set_precision", "chdwf_dslash_dev_lp",
    "chdwf_prog_state_size", "chdwf_prog_get_state", "chdwf_prog_set_state",
    "chdwf_congrad_static", "chdwf_congrad_batch", "chdwf_set_basis_store",
    "chdwf_prog_create", "chdwf_prog_destroy", "chdwf_prog_context", "chdwf_prog_set_remez",
    "chdwf_prog_set_chi", "chdwf_prog_get_chi", "chdwf_prog_startup", "chdwf_prog_seed",
    "chdwf_prog_set_measure", "chdwf_prog_set_residuals", "chdwf_prog_sweep",
    "chdwf_prog_correlators", "chdwf_prog_last_error", "chdwf_prog_measure",
    "chdwf_traj_noise_solve",
    "chdwf_hmc_create", "chdwf_hmc_destroy", "chdwf_hmc_last_error", "chdwf_hmc_dslash",
    "chdwf_hmc_dslashd", "chdwf_hmc_congrad", "chdwf_hmc_derivs", "chdwf_hmc_set_chi",
    "chdwf_hmc_get_chi", "chdwf_hmc_startup", "chdwf_hmc_seed", "chdwf_hmc_set_measure",
    "chdwf_hmc_set_residuals", "chdwf_hmc_sweep",
    "chdwf_thr_create", "chdwf_thr_destroy", "chdwf_thr_last_error", "chdwf_thr_set_remez",
    "chdwf_thr_coef", "chdwf_thr_dslash", "chdwf_thr_dslashd", "chdwf_thr_derivs",
    "chdwf_thr_qmrherm", "chdwf_thr_set_theta", "chdwf_thr_get_theta", "chdwf_thr_startup",
    "chdwf_thr_seed", "chdwf_thr_sweep", "chdwf_thr_congrad", "chdwf_thr_measure",
    "chdwf_thr_set_measure",
    "chdwf_prog_sums", "chdwf_prog_reset_sums", "chdwf_prog_averages", "chdwf_prog_take_cg_caps",
    "chdwf_con_read", "chdwf_con_write", "chdwf_prog_read_con", "chdwf_prog_write_con",
    "chdwf_format_list", "chdwf_format_edit", "chdwf_run_dir",
    "chdwf_ext_set_remez", "chdwf_ext_select_pf", "chdwf_ext_heatbath_dev", "chdwf_ext_action",
    "chdwf_ext_force", "chdwf_ext_bosonic", "chdwf_prog_set_ext", "chdwf_multishift_dev",
    "chdwf_autotune_report", "chdwf_traj_propagators", "chdwf_stencil_launches",
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
    L.chdwf_traj_set_remez.argtypes = [P, I, P, P, P, P, I]
    L.chdwf_traj_set_chi.argtypes = [P, P]
    L.chdwf_traj_get_chi.argtypes = [P, P, I]
    L.chdwf_traj_begin.argtypes = [P]
    L.chdwf_traj_heatbath.argtypes = [P, P, F, F, F, I, PI]
    L.chdwf_traj_heatbath_dev.argtypes = [P, P, F, F, F, I, PI]
    L.chdwf_traj_set_momenta.argtypes = [P, P]
    L.chdwf_traj_get_momenta.argtypes = [P, P]
    L.chdwf_traj_hamilton.argtypes = [P, F, F, F, I, P, PI]
    L.chdwf_traj_force.argtypes = [P, F, F, F, I, PI, PI]
    L.chdwf_traj_get_force.argtypes = [P, P]
    L.chdwf_traj_get_phi.argtypes = [P, P]
    L.chdwf_traj_update_momenta.argtypes = [P, F]
    L.chdwf_traj_update_chi.argtypes = [P, F]
    L.chdwf_traj_accept.argtypes = [P]
    L.chdwf_traj_sync.argtypes = [P]
    L.chdwf_traj_propagator.argtypes = [P, I, I, F, F, F, I, P, PI]
    L.chdwf_prog_create.argtypes = [C.POINTER(P), I, I, I, F, F, F, F, F, I, I, I]
    L.chdwf_prog_destroy.argtypes = [P]
    L.chdwf_prog_destroy.restype = None
    L.chdwf_prog_context.argtypes = [P]
    L.chdwf_prog_context.restype = P
    L.chdwf_prog_set_remez.argtypes = [P, I, P, P, P, P, I]
    L.chdwf_prog_set_chi.argtypes = [P, P]
    L.chdwf_prog_get_chi.argtypes = [P, P]
    L.chdwf_prog_startup.argtypes = [P, D]
    L.chdwf_prog_seed.argtypes = [P]
    L.chdwf_prog_seed.restype = D
    L.chdwf_prog_set_measure.argtypes = [P, I, I]
    L.chdwf_prog_set_residuals.argtypes = [P, F, F, F]
    L.chdwf_prog_sweep.argtypes = [P, P]
    L.chdwf_prog_correlators.argtypes = [P, P]
    L.chdwf_prog_measure.argtypes = [P, F, C.POINTER(F), C.POINTER(F), C.POINTER(F), P]
    L.chdwf_traj_noise_solve.argtypes = [P, P, I, I, F, F, F, I, P, PI]
    L.chdwf_hmc_create.argtypes = [C.POINTER(P), I, I, I, F, F, F, F, I, I, I]
    L.chdwf_hmc_destroy.argtypes = [P]
    L.chdwf_hmc_destroy.restype = None
    L.chdwf_hmc_last_error.argtypes = [P]
    L.chdwf_hmc_last_error.restype = C.c_char_p
    L.chdwf_hmc_dslash.argtypes = [P, P, P, P, I]
    L.chdwf_hmc_dslashd.argtypes = [P, P, P, P, I]
    L.chdwf_hmc_congrad.argtypes = [P, P, F, PI, I, P, P]
    L.chdwf_hmc_derivs.argtypes = [P, P, P, I, P]
    L.chdwf_hmc_set_chi.argtypes = [P, P]
    L.chdwf_hmc_get_chi.argtypes = [P, P]
    L.chdwf_hmc_startup.argtypes = [P, D]
    L.chdwf_hmc_seed.argtypes = [P]
    L.chdwf_hmc_seed.restype = D
    L.chdwf_hmc_set_measure.argtypes = [P, I]
    L.chdwf_hmc_set_residuals.argtypes = [P, F, F]
    L.chdwf_hmc_sweep.argtypes = [P, P]
    L.chdwf_thr_create.argtypes = [C.POINTER(P), I, I, I, F, F, F, F, I, I, I]
    L.chdwf_thr_destroy.argtypes = [P]
    L.chdwf_thr_destroy.restype = None
    L.chdwf_thr_last_error.argtypes = [P]
    L.chdwf_thr_last_error.restype = C.c_char_p
    L.chdwf_thr_set_remez.argtypes = [P, I, P, P, P, P, I]
    L.chdwf_thr_coef.argtypes = [P, P, P]
    L.chdwf_thr_dslash.argtypes = [P, P, P, P, F, I]
    L.chdwf_thr_dslashd.argtypes = [P, P, P, P, F, I]
    L.chdwf_thr_derivs.argtypes = [P, P, P, D, I, P]
    L.chdwf_thr_qmrherm.argtypes = [P, P, F, PI, F, I, P, P, I, I, P, P, P, P]
    L.chdwf_thr_set_theta.argtypes = [P, P]
    L.chdwf_thr_get_theta.argtypes = [P, P]
    L.chdwf_thr_startup.argtypes = [P, D]
    L.chdwf_thr_seed.argtypes = [P]
    L.chdwf_thr_seed.restype = D
    L.chdwf_thr_sweep.argtypes = [P, P]
    L.chdwf_thr_congrad.argtypes = [P, P, F, PI, F, I, P, P]
    L.chdwf_thr_measure.argtypes = [P, F, P, C.POINTER(F), C.POINTER(F), C.POINTER(F), P]
    L.chdwf_thr_set_measure.argtypes = [P, I]
    L.chdwf_prog_last_error.argtypes = [P]
    L.chdwf_prog_last_error.restype = C.c_char_p
    L.chdwf_prog_stage.argtypes = [P, I]
    L.chdwf_traj_set_momenta_dev.argtypes = [P, P]
    L.chdwf_timing.argtypes = [P, I]
    L.chdwf_timing_read.argtypes = [P, P, P, P, P]
    L.chdwf_timing_read_chunks.argtypes = [P, P, P]
    L.chdwf_get_stream.argtypes = [P]
    L.chdwf_get_stream.restype = P
    L.chdwf_kernel_launches.restype = C.c_longlong
    L.chdwf_set_precision.argtypes = [P, I, I]
    L.chdwf_dslash_dev_lp.argtypes = [P, P, P, P, F, I, I, I, P]
    L.chdwf_congrad_static.argtypes = [P, P, P, I, I, I, F, I, F, F, I, PI, P]
    L.chdwf_congrad_batch.argtypes = [P, P, I, F, P, P]
    L.chdwf_set_basis_store.argtypes = [P, D]
    L.chdwf_prog_get_state.argtypes = [P, P, I]
    L.chdwf_prog_set_state.argtypes = [P, P, I]
    L.chdwf_prog_sums.argtypes = [P, P]
    L.chdwf_prog_reset_sums.argtypes = [P]
    L.chdwf_prog_averages.argtypes = [P, P]
    L.chdwf_prog_take_cg_caps.argtypes = [P]
    L.chdwf_con_read.argtypes = [C.c_char_p, I, P, C.POINTER(D), PI]
    L.chdwf_con_write.argtypes = [C.c_char_p, I, P, D]
    L.chdwf_prog_read_con.argtypes = [P, C.c_char_p, C.POINTER(D)]
    L.chdwf_prog_write_con.argtypes = [P, C.c_char_p]
    L.chdwf_format_list.argtypes = [C.c_char_p, I, C.c_char_p, P]
    L.chdwf_format_edit.argtypes = [C.c_char_p, I, C.c_char, I, I, D]
    L.chdwf_run_dir.argtypes = [C.c_char_p, I, I, I, I]
    L.chdwf_ext_set_remez.argtypes = [P, I, P, P, I]
    L.chdwf_ext_select_pf.argtypes = [P, I]
    L.chdwf_ext_heatbath_dev.argtypes = [P, P, F, F, I, PI]
    L.chdwf_ext_action.argtypes = [P, F, F, I, C.POINTER(D), PI]
    L.chdwf_ext_force.argtypes = [P, F, F, I, I, PI]
    L.chdwf_ext_bosonic.argtypes = [P, P]
    L.chdwf_prog_set_ext.argtypes = [P, I, I, I, F]
    L.chdwf_multishift_dev.argtypes = [P, P, F, P, F, I, I, P, P, P, I, PI, PI]
    L.chdwf_autotune_report.argtypes = [C.c_char_p, I]
    L.chdwf_stencil_launches.argtypes = [P]
    L.chdwf_traj_propagators.argtypes = [P, I, P, P, F, F, F, I, P, P]
    _lib = L
    return L


class CgSystem(C.Structure):
    """chdwf_cg_system (include/chdwf.h): one propagator solve of a batch."""
    _fields_ = [("ksize", C.c_int), ("ksizet", C.c_int), ("kthird", C.c_int),
                ("imass", C.c_int), ("hpin", C.c_float), ("am3", C.c_float),
                ("ibound", C.c_int), ("Phi", C.c_void_p), ("x", C.c_void_p), ("chi", C.c_void_p)]


def congrad_batch(lattice, systems, res):
    """Solve every CgSystem of the list in one set of launches (device
    pointers inside); returns (itercg, status) arrays.  lattice: any Lattice
    (its context supplies the stream and the workspace)."""
    n = len(systems)
    arr = (CgSystem * n)(*systems)
    it = np.zeros(n, dtype=np.int32)
    st = np.zeros(n, dtype=np.int32)
    rc = lattice.lib.chdwf_congrad_batch(lattice.h, C.cast(arr, C.c_void_p), n, res, _ptr(it),
                                         _ptr(st))
    if rc not in (CHDWF_OK, CHDWF_ITER_CAP, CHDWF_NONFINITE):
        raise ChdwfError(rc, lattice.lib.chdwf_last_error(lattice.h).decode())
    return it, st


class SweepRecord(C.Structure):
    """chdwf_sweep_record (include/chdwf_program.h)."""
    _fields_ = [("H0", C.c_double), ("H1", C.c_double), ("dH", C.c_double), ("dS", C.c_double),
                ("S0", C.c_double), ("S1", C.c_double), ("hg", C.c_double), ("hp", C.c_double),
                ("y", C.c_float), ("x", C.c_float), ("accepted", C.c_int), ("nsteps", C.c_int),
                ("it_pf", C.c_int), ("it_h0", C.c_int), ("it_h1", C.c_int),
                ("it_guid", C.c_double), ("it_force", C.c_double), ("nforce", C.c_int),
                ("action", C.c_float), ("gaction", C.c_float), ("paction", C.c_float),
                ("vel2", C.c_float), ("measured", C.c_int), ("cond", C.c_float * 3),
                ("susc", C.c_float * 3), ("condmod", C.c_float), ("susctot", C.c_float),
                ("ancgm", C.c_float), ("ended", C.c_int)]

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class RunSums(C.Structure):
    """chdwf_run_sums (include/chdwf_program.h): the main program's running sums."""
    _fields_ = [(n, C.c_float) for n in ("actiona", "vel2a", "condmoda", "susca")] + \
        [("conda", C.c_float * 3), ("pbpa", C.c_float)] + \
        [(n, C.c_float) for n in ("ancg", "ancgh", "ancgf", "ancgpf", "ancgma", "yav", "yyav")] + \
        [(n, C.c_int) for n in ("naccp", "ipbp", "itot", "nsweep")] + [("gaction", C.c_float)]


class RunAverages(C.Structure):
    """chdwf_run_averages: the averages of 'output' (rhmc/cheisdwf.f:413-443)."""
    _fields_ = [("iter2", C.c_int), ("naccp", C.c_int)] + \
        [(n, C.c_float) for n in ("atraj", "yav", "yyav", "ancg", "ancgh", "ancgf", "ancgpf",
                                  "ancgma", "condmoda", "susca")] + \
        [("conda", C.c_float * 3), ("pbpa", C.c_float), ("vel2a", C.c_float),
         ("actiona", C.c_float)]


def autotune_report():
    """The stencil autotuner's choices in this process (chdwf_autotune_report)."""
    import json
    lib = load_library()
    n = lib.chdwf_autotune_report(None, 0)
    buf = C.create_string_buffer(n)
    lib.chdwf_autotune_report(buf, n)
    return json.loads(buf.value.decode())


def con_read(path, kvol):
    """'con' (sread): returns (chi[3, kvol] float64, seed, single), where
    single tells that the file held a REAL*4 configuration."""
    lib = load_library()
    chi = np.empty((3, kvol), dtype=np.float64)
    seed, single = C.c_double(), C.c_int()
    rc = lib.chdwf_con_read(os.fsencode(path), kvol, _ptr(chi), C.byref(seed), C.byref(single))
    if rc == CHDWF_NOT_FOUND:
        raise FileNotFoundError(path)
    if rc != CHDWF_OK:
        raise ChdwfError(rc, f"not a {kvol}-site configuration: {path}")
    return chi, seed.value, bool(single.value)


def con_write(path, chi, seed):
    """'con' as swrite writes it: one unformatted record of chi (REAL*8) and seed."""
    lib = load_library()
    chi = np.ascontiguousarray(chi, dtype=np.float64)
    rc = lib.chdwf_con_write(os.fsencode(path), chi.size // 3, _ptr(chi), float(seed))
    if rc != CHDWF_OK:
        raise ChdwfError(rc, f"cannot write {path}")


def format_list(kinds: str, values) -> str:
    """One list-directed output record in gfortran's layout; kinds holds 'i'
    (INTEGER), 'f' (REAL*4) or 'd' (REAL*8) per value."""
    lib = load_library()
    vals = np.ascontiguousarray(values, dtype=np.float64)
    buf = C.create_string_buffer(64 * (len(kinds) + 1))
    n = lib.chdwf_format_list(buf, len(buf), kinds.encode(), _ptr(vals))
    if n < 0:
        raise ValueError(kinds)
    return buf.value.decode()


def format_edit(kind: str, w: int, d: int, value) -> str:
    """One explicit edit descriptor: 'I' (Iw), 'F' (Fw.d) or 'E' (Ew.d)."""
    lib = load_library()
    buf = C.create_string_buffer(w + 64)
    n = lib.chdwf_format_edit(buf, len(buf), kind.encode(), w, d, float(value))
    if n < 0:
        raise ValueError(kind)
    return buf.value.decode()


def run_dir(path, ksize, ksizet, kthird, device=0):
    """Run program dwf3d in directory path with the reference's input files
    (midout, con, remez2, remez4, remez2g) and output streams."""
    lib = load_library()
    rc = lib.chdwf_run_dir(os.fsencode(path), ksize, ksizet, kthird, device)
    if rc == CHDWF_NOT_FOUND:
        raise FileNotFoundError(path)
    if rc != CHDWF_OK:
        raise (IterationCapError if rc == CHDWF_ITER_CAP else ChdwfError)(
            rc, lib.chdwf_last_error(None).decode())


class Program:
    """The main loop of program dwf3d (rhmc/cheisdwf.f:207-399) on the GPU:
    host random numbers and control flow, resident fields (see
    include/chdwf_program.h).  Parameters are those of the 'midout' file."""

    def __init__(self, ksize, ksizet, kthird, dt, beta, am3, am, hpin, imass, iterl, remez2,
                 remez4, remez2g, device=0):
        self.lib = load_library()
        self.kvol = ksize * ksize * ksizet
        self.Lt = ksizet
        h = C.c_void_p()
        rc = self.lib.chdwf_prog_create(C.byref(h), ksize, ksizet, kthird, dt, beta, am3, am,
                                        hpin, imass, iterl, device)
        if rc != CHDWF_OK:
            raise ChdwfError(rc, self.lib.chdwf_last_error(None).decode())
        self.h = h
        self._rescgm = 0.000000001                    # rhmc/cheisdwf.f:33
        for which, r in ((2, remez2), (4, remez4), (22, remez2g)):
            arrs = [np.ascontiguousarray(r[k], dtype=np.float64)
                    for k in ("anum", "aden", "bnum", "bden")]
            self._check(self.lib.chdwf_prog_set_remez(self.h, which, *[_ptr(a) for a in arrs],
                                                      len(arrs[1])))
            setattr(self, f"_keep{which}", arrs)

    def _check(self, rc):
        if rc != CHDWF_OK:
            msg = self.lib.chdwf_prog_last_error(self.h).decode()
            raise (IterationCapError if rc == CHDWF_ITER_CAP else ChdwfError)(rc, msg)

    def startup(self, seed):
        self._check(self.lib.chdwf_prog_startup(self.h, float(seed)))

    def seed(self):
        return self.lib.chdwf_prog_seed(self.h)

    def set_chi(self, chi):
        chi = np.ascontiguousarray(chi, dtype=np.float64)
        self._check(self.lib.chdwf_prog_set_chi(self.h, _ptr(chi)))

    def get_chi(self):
        chi = np.empty((3, self.kvol), dtype=np.float64)
        self._check(self.lib.chdwf_prog_get_chi(self.h, _ptr(chi)))
        return chi

    def set_measure(self, iprint=5, measure=True):
        self._check(self.lib.chdwf_prog_set_measure(self.h, iprint, 1 if measure else 0))

    def set_residuals(self, rescga, rescgg, rescgm):
        self._check(self.lib.chdwf_prog_set_residuals(self.h, rescga, rescgg, rescgm))
        self._rescgm = rescgm

    def sweep(self) -> SweepRecord:
        rec = SweepRecord()
        self._check(self.lib.chdwf_prog_sweep(self.h, C.byref(rec)))
        return rec

    def correlators(self):
        cf = np.empty((2, 2, self.Lt, 2), dtype=np.float32)
        self._check(self.lib.chdwf_prog_correlators(self.h, _ptr(cf)))
        return cf

    def measure(self, res=None):
        """measure() of rhmc/cheisdwf.f:1164-1453 on the current chi: returns
        (psibarpsi, susclsing, aviter, parts) with parts[inoise] = (re p1,
        im p1, re p2, im p2), the unit-100 record of each noise vector.
        res defaults to the measurement residual rescgm."""
        pb, su, av = C.c_float(), C.c_float(), C.c_float()
        parts = np.empty((10, 4), dtype=np.float64)
        r = self._rescgm if res is None else res
        self._check(self.lib.chdwf_prog_measure(self.h, r, C.byref(pb), C.byref(su), C.byref(av),
                                                _ptr(parts)))
        return pb.value, su.value, av.value, parts

    def sums(self) -> RunSums:
        out = RunSums()
        self._check(self.lib.chdwf_prog_sums(self.h, C.byref(out)))
        return out

    def reset_sums(self):
        self._check(self.lib.chdwf_prog_reset_sums(self.h))

    def averages(self) -> RunAverages:
        out = RunAverages()
        self._check(self.lib.chdwf_prog_averages(self.h, C.byref(out)))
        return out

    def read_con(self, path) -> float:
        """sread: chi from 'con' (or the cold default); returns the seed."""
        seed = C.c_double()
        self._check(self.lib.chdwf_prog_read_con(self.h, os.fsencode(path), C.byref(seed)))
        return seed.value

    def write_con(self, path):
        """swrite with the generator's current seed."""
        self._check(self.lib.chdwf_prog_write_con(self.h, os.fsencode(path)))

    def get_state(self) -> bytes:
        """Generator state + sweep counter (exact resume; see chdwf_prog_get_state)."""
        n = self.lib.chdwf_prog_state_size()
        buf = C.create_string_buffer(n)
        self._check(self.lib.chdwf_prog_get_state(self.h, buf, n))
        return buf.raw

    def set_state(self, blob: bytes):
        buf = C.create_string_buffer(blob, len(blob))
        self._check(self.lib.chdwf_prog_set_state(self.h, buf, len(blob)))

    def stage(self, ntraj):
        """Draw the next ntraj trajectories' random inputs and place them in HBM."""
        self._check(self.lib.chdwf_prog_stage(self.h, ntraj))

    @property
    def context(self):
        return self.lib.chdwf_prog_context(self.h)

    @property
    def stream(self) -> int:
        """cudaStream_t of the program's context, as an integer handle."""
        return self.lib.chdwf_get_stream(self.context) or 0

    def timing(self, enable=True, chunks=False):
        """Solver-kernel timing: per launch (chunks=False), or per graph-replayed
        chunk of pass-1 iterations (chunks=True, read with timing_chunks)."""
        self._check(self.lib.chdwf_timing(self.context, (2 if chunks else 1) if enable else 0))

    def timing_chunks(self):
        """Pass-1 microseconds per iteration from graph-replayed chunks and the
        iterations timed, per Krylov-vector precision: ([FP64, FP32], [FP64, FP32])."""
        us = np.zeros(2, dtype=np.float64)
        its = np.zeros(2, dtype=np.int64)
        self._check(self.lib.chdwf_timing_read_chunks(self.context, _ptr(us), _ptr(its)))
        return us, its

    def set_basis_store(self, max_bytes):
        """HBM budget of the stored Lanczos basis (bytes; 0 disables, <0 default)."""
        self._check(self.lib.chdwf_set_basis_store(self.context, float(max_bytes)))

    def set_precision(self, md="f64", accept="f64"):
        """Krylov-vector precision of the force solves (md) and of the
        heatbath/hamilton solves (accept): "f64" (drop-in) or "f32"."""
        code = {"f64": 0, "f32": 1}
        self._check(self.lib.chdwf_set_precision(self.context, code[md], code[accept]))

    def set_ext(self, npf, nsteps, hb, act, integrator="omelyan",
                lam=0.1931833275037836):
        """The multi-pseudofermion variant (include/chdwf_program.h,
        chdwf_prog_set_ext): npf fields, nsteps integrator steps of dt.
        hb, act: (num[0..n], den[0..n-1]) of the heatbath function
        x^(1/(4 npf)) and of the action/force function x^(-1/(2 npf)),
        e.g. from chiralheisenberg_b200.remez.  npf=0 returns to the
        reference's sweep."""
        ctx = self.context
        if npf > 0:
            keep = []
            for which, (num, den) in ((0, hb), (1, act)):
                num = np.ascontiguousarray(num, dtype=np.float64)
                den = np.ascontiguousarray(den, dtype=np.float64)
                keep.append((num, den))
                self._check(self.lib.chdwf_ext_set_remez(ctx, which, _ptr(num), _ptr(den),
                                                         len(den)))
        code = {"leapfrog": 0, "omelyan": 1}[integrator]
        self._check(self.lib.chdwf_prog_set_ext(self.h, npf, nsteps, code, lam))

    def timing_read(self):
        """Per solver-kernel class (0-3 FP64 vectors, 4-7 FP32): (ms, timed
        launches, launches, bytes)."""
        ms = np.zeros(8, dtype=np.float64)
        timed = np.zeros(8, dtype=np.int64)
        launched = np.zeros(8, dtype=np.int64)
        nbytes = np.zeros(8, dtype=np.float64)
        self._check(self.lib.chdwf_timing_read(self.context, _ptr(ms), _ptr(timed),
                                               _ptr(launched), _ptr(nbytes)))
        return ms, timed, launched, nbytes

    def close(self):
        if getattr(self, "h", None):
            self.lib.chdwf_prog_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


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
        self.device = device
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

    def set_basis_store(self, max_bytes):
        """HBM budget of the stored Lanczos basis (bytes; 0 disables, <0 default)."""
        self._check(self.lib.chdwf_set_basis_store(self.h, float(max_bytes)))

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

    def multishift(self, Phi, res, chi, sigma, prec="f64", hpin=0.0, imass=1):
        """Per-shift solutions (M^dag M + sigma_k)^-1 Phi and their FP64 true
        relative residuals (chdwf_multishift_dev).  prec "f64", or "f32":
        FP32 Krylov vectors with FP64 defect correction.  Returns
        (x[n, ...] complex128, true_res[n], iters, refine_iters)."""
        import torch
        sigma = np.ascontiguousarray(sigma, dtype=np.float64)
        n = len(sigma)
        dev = torch.device("cuda", self.device)
        Phi_t = torch.from_numpy(np.ascontiguousarray(_c128(Phi, self.shape))).to(dev)
        chi_t = torch.from_numpy(self._chi(chi)).to(dev)
        xs = [torch.empty_like(Phi_t) for _ in range(n)]
        ptrs = (C.c_void_p * n)(*[x.data_ptr() for x in xs])
        tr = np.zeros(n, dtype=np.float64)
        it, rit = C.c_int(0), C.c_int(0)
        code = {"f64": 0, "f32": 1}[prec]
        self._check(self.lib.chdwf_multishift_dev(self.h, C.c_void_p(Phi_t.data_ptr()), res,
                                                  C.c_void_p(chi_t.data_ptr()), hpin, imass, n,
                                                  _ptr(sigma), ptrs, _ptr(tr), code,
                                                  C.byref(it), C.byref(rit)))
        torch.cuda.synchronize(dev)
        return np.stack([x.cpu().numpy() for x in xs]), tr, it.value, rit.value

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


def kernel_launches() -> int:
    """Kernels libchdwf has launched in this process."""
    return int(load_library().chdwf_kernel_launches())


def stencil_launches() -> dict:
    """Operator and pass-1 stencil launches in this process by kernel shape
    (chdwf_stencil_launches): {"gather3": n, "rows": n, "gather4": n}."""
    buf = (C.c_longlong * 3)()
    rc = load_library().chdwf_stencil_launches(buf)
    if rc != CHDWF_OK:
        raise ChdwfError(rc, "stencil_launches")
    return {"gather3": int(buf[0]), "rows": int(buf[1]), "gather4": int(buf[2])}


DATA_DIR = os.path.join(_HERE, "data")


def read_remez(name: str, n: int, path: str = None) -> dict:
    """Read a Remez data file in the reference's format (rhmc/remez*, read at
    rhmc/cheisdwf.f:140-159): a0; n lines "a_k, sigma_k"; b0; n lines
    "b_k, sigma_k".  Returns anum (a0..a_n), aden, bnum (b0..b_n), bden."""
    vals = []
    for line in open(path or os.path.join(DATA_DIR, name)):
        line = line.replace(",", " ").replace("d", "e").replace("D", "e").strip()
        if line:
            vals.append([float(t) for t in line.split()])
    if len(vals) < 2 * n + 2:
        raise ValueError(f"{name}: expected {2 * n + 2} lines, found {len(vals)}")
    a0 = vals[0][0]
    b0 = vals[n + 1][0]
    return {"anum": np.array([a0] + [v[0] for v in vals[1:n + 1]]),
            "aden": np.array([v[1] for v in vals[1:n + 1]]),
            "bnum": np.array([b0] + [v[0] for v in vals[n + 2:2 * n + 2]]),
            "bden": np.array([v[1] for v in vals[n + 2:2 * n + 2]])}


def reference_remez() -> dict:
    """The three rational approximations the reference ships: remez2 and
    remez4 (25 poles), remez2g (12 poles)."""
    return {"remez2": read_remez("remez2", 25), "remez4": read_remez("remez4", 25),
            "remez2g": read_remez("remez2g", 12)}


class HmcRecord(C.Structure):
    """chdwf_hmc_record (include/chdwf_hmc.h)."""
    _fields_ = [("H0", C.c_double), ("H1", C.c_double), ("dH", C.c_double), ("dS", C.c_double),
                ("S0", C.c_double), ("S1", C.c_double), ("hg", C.c_double), ("hp", C.c_double),
                ("y", C.c_float), ("x", C.c_float), ("drew_x", C.c_int), ("accepted", C.c_int),
                ("nsteps", C.c_int), ("it_h0", C.c_int), ("it_h1", C.c_int),
                ("it_force", C.c_int), ("nforce", C.c_int), ("action", C.c_float),
                ("gaction", C.c_float), ("paction", C.c_float), ("vel2", C.c_float),
                ("measured", C.c_int), ("cond", C.c_float * 3), ("susc", C.c_float * 3),
                ("condmod", C.c_float), ("susctot", C.c_float)]


class Hmc:
    """The HMC predecessor mh/cheisdwf_hmc.f on the GPU (include/chdwf_hmc.h):
    single-precision operator, congrad, chi force and main loop.  Spinors are
    complex64 of shape (2, 4, ksizet, ksize, ksize, kthird), chi float32
    (3, kvol)."""

    def __init__(self, ksize, ksizet, kthird, dt, beta, am3, am, imass, iterl, device=0):
        self.lib = load_library()
        self.kvol = ksize * ksize * ksizet
        self.shape = (2, 4, ksizet, ksize, ksize, kthird)
        self.imass = imass
        h = C.c_void_p()
        rc = self.lib.chdwf_hmc_create(C.byref(h), ksize, ksizet, kthird, dt, beta, am3, am,
                                       imass, iterl, device)
        if rc != CHDWF_OK:
            raise ChdwfError(rc, self.lib.chdwf_hmc_last_error(None).decode())
        self.h = h

    def _check(self, rc):
        if rc != CHDWF_OK:
            msg = self.lib.chdwf_hmc_last_error(self.h).decode()
            raise (IterationCapError if rc == CHDWF_ITER_CAP else ChdwfError)(rc, msg)

    def _spinor(self, a):
        a = np.ascontiguousarray(a, dtype=np.complex64)
        if a.size != int(np.prod(self.shape)):
            raise ValueError(f"spinor has {a.size} entries, expected shape {self.shape}")
        return a

    def _chi(self, chi):
        chi = np.ascontiguousarray(chi, dtype=np.float32)
        if chi.size != 3 * self.kvol:
            raise ValueError(f"chi has {chi.size} entries, expected {3 * self.kvol}")
        return chi

    def dslash(self, R, chi, imass=None, dag=False):
        R, chi = self._spinor(R), self._chi(chi)
        out = np.empty(self.shape, dtype=np.complex64)
        f = self.lib.chdwf_hmc_dslashd if dag else self.lib.chdwf_hmc_dslash
        self._check(f(self.h, _ptr(out), _ptr(R), _ptr(chi), self.imass if imass is None else imass))
        return out

    def congrad(self, Phi, chi, x0, res, imass=None):
        """x with M^dag M x = Phi from the guess x0; returns (x, itercg, capped)."""
        Phi, chi = self._spinor(Phi), self._chi(chi)
        x = self._spinor(x0).copy()
        it = C.c_int(0)
        rc = self.lib.chdwf_hmc_congrad(self.h, _ptr(Phi), res, C.byref(it),
                                        self.imass if imass is None else imass, _ptr(chi), _ptr(x))
        if rc not in (CHDWF_OK, CHDWF_ITER_CAP):
            self._check(rc)
        return x.reshape(self.shape), it.value, rc == CHDWF_ITER_CAP

    def derivs(self, X1, chi, imass=None):
        X1, chi = self._spinor(X1), self._chi(chi)
        dS = np.empty((3, self.kvol), dtype=np.float32)
        self._check(self.lib.chdwf_hmc_derivs(self.h, _ptr(X1), _ptr(chi),
                                              self.imass if imass is None else imass, _ptr(dS)))
        return dS

    def set_chi(self, chi):
        self._check(self.lib.chdwf_hmc_set_chi(self.h, _ptr(self._chi(chi))))

    def get_chi(self):
        chi = np.empty((3, self.kvol), dtype=np.float32)
        self._check(self.lib.chdwf_hmc_get_chi(self.h, _ptr(chi)))
        return chi

    def startup(self, seed):
        self._check(self.lib.chdwf_hmc_startup(self.h, float(seed)))

    def seed(self):
        return self.lib.chdwf_hmc_seed(self.h)

    def set_measure(self, iprint):
        self._check(self.lib.chdwf_hmc_set_measure(self.h, iprint))

    def set_residuals(self, rescga, rescgg):
        self._check(self.lib.chdwf_hmc_set_residuals(self.h, rescga, rescgg))

    def sweep(self) -> HmcRecord:
        rec = HmcRecord()
        self._check(self.lib.chdwf_hmc_sweep(self.h, C.byref(rec)))
        return rec

    def close(self):
        if getattr(self, "h", None):
            self.lib.chdwf_hmc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ThirringRecord(C.Structure):
    """chdwf_thr_record (include/chdwf_thirring.h)."""
    _fields_ = [("H0", C.c_double), ("H1", C.c_double), ("dH", C.c_double), ("dS", C.c_double),
                ("S0", C.c_double), ("S1", C.c_double), ("hg", C.c_double), ("hp", C.c_double),
                ("y", C.c_float), ("x", C.c_float), ("drew_x", C.c_int), ("accepted", C.c_int),
                ("nsteps", C.c_int), ("it_pf", C.c_int), ("it_pfpv", C.c_int),
                ("it_h0", C.c_int), ("it_h0pv", C.c_int), ("it_h1", C.c_int),
                ("it_h1pv", C.c_int), ("it_force", C.c_int * 4), ("nforce", C.c_int),
                ("action", C.c_float), ("gaction", C.c_float), ("paction", C.c_float),
                ("vel2", C.c_float), ("measured", C.c_int), ("pbp", C.c_float),
                ("ancgm", C.c_float)]


class Thirring:
    """The bulk Thirring RHMC of bulk_rhmc.f on the GPU
    (include/chdwf_thirring.h).  Spinors are complex128 of shape
    (4, ksizet, ksize, ksize, kthird), links u complex128 (3, kvol), link
    angles theta and the force float32 (3, kvol)."""

    def __init__(self, ksize, ksizet, kthird, dt, beta, am3, am, imass, iterl, device=0):
        self.lib = load_library()
        self.kvol = ksize * ksize * ksizet
        self.shape = (4, ksizet, ksize, ksize, kthird)
        h = C.c_void_p()
        rc = self.lib.chdwf_thr_create(C.byref(h), ksize, ksizet, kthird, dt, beta, am3, am,
                                       imass, iterl, device)
        if rc != CHDWF_OK:
            raise ChdwfError(rc, self.lib.chdwf_thr_last_error(None).decode())
        self.h = h
        self._keep = {}

    def _check(self, rc):
        if rc != CHDWF_OK:
            msg = self.lib.chdwf_thr_last_error(self.h).decode()
            raise (IterationCapError if rc == CHDWF_ITER_CAP else ChdwfError)(rc, msg)

    def _spinor(self, a):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        if a.size != int(np.prod(self.shape)):
            raise ValueError(f"spinor has {a.size} entries, expected shape {self.shape}")
        return a

    def set_remez(self, which, r):
        """which: 2, 4 (remez2, remez4) or 22, 44 (remez2g, remez4g); r a dict
        with anum, aden, bnum, bden as read from the file."""
        arrs = [np.ascontiguousarray(r[k], dtype=np.float64) for k in ("anum", "aden", "bnum", "bden")]
        self._check(self.lib.chdwf_thr_set_remez(self.h, which, *[_ptr(a) for a in arrs],
                                                 len(arrs[1])))
        self._keep[which] = arrs

    def coef(self, theta):
        u = np.empty((3, self.kvol), dtype=np.complex128)
        self._check(self.lib.chdwf_thr_coef(self.h, _ptr(np.ascontiguousarray(theta, dtype=np.float32)),
                                            _ptr(u)))
        return u

    def dslash(self, R, u, am, imass, dag=False):
        R = self._spinor(R)
        u = np.ascontiguousarray(u, dtype=np.complex128)
        out = np.empty(self.shape, dtype=np.complex128)
        f = self.lib.chdwf_thr_dslashd if dag else self.lib.chdwf_thr_dslash
        self._check(f(self.h, _ptr(out), _ptr(R), _ptr(u), am, imass))
        return out

    def derivs(self, R, X2, anum, iflag, dSdpi=None):
        dS = np.zeros((3, self.kvol), dtype=np.float32) if dSdpi is None else dSdpi
        self._check(self.lib.chdwf_thr_derivs(self.h, _ptr(self._spinor(R)), _ptr(self._spinor(X2)),
                                              float(anum), iflag, _ptr(dS)))
        return dS

    def qmrherm(self, Phi, u, res, am, imass, anum, aden, iflag=0, Phi0=None, dSdpi=None):
        """Returns (x, itercg, capped, Phi0, dSdpi)."""
        n = len(aden)
        x = np.empty(self.shape, dtype=np.complex128)
        P0 = np.zeros((n,) + self.shape, dtype=np.complex128) if Phi0 is None else Phi0
        dS = np.zeros((3, self.kvol), dtype=np.float32) if dSdpi is None else dSdpi
        it = C.c_int(0)
        rc = self.lib.chdwf_thr_qmrherm(
            self.h, _ptr(self._spinor(Phi)), res, C.byref(it), am, imass,
            _ptr(np.ascontiguousarray(anum, dtype=np.float64)),
            _ptr(np.ascontiguousarray(aden, dtype=np.float64)), n, iflag,
            _ptr(np.ascontiguousarray(u, dtype=np.complex128)), _ptr(x), _ptr(P0), _ptr(dS))
        if rc not in (CHDWF_OK, CHDWF_ITER_CAP):
            self._check(rc)
        return x, it.value, rc == CHDWF_ITER_CAP, P0, dS

    def congrad(self, Phi, u, x0, res, am, imass):
        """congrad: x with M^dag M x = Phi from x0; returns (x, itercg, capped)."""
        x = self._spinor(x0).copy()
        it = C.c_int(0)
        rc = self.lib.chdwf_thr_congrad(self.h, _ptr(self._spinor(Phi)), res, C.byref(it), am,
                                        imass, _ptr(np.ascontiguousarray(u, dtype=np.complex128)),
                                        _ptr(x))
        if rc not in (CHDWF_OK, CHDWF_ITER_CAP):
            self._check(rc)
        return x.reshape(self.shape), it.value, rc == CHDWF_ITER_CAP

    def measure(self, u, res=1e-6):
        """measure with links u: (psibarpsi, susclsing, aviter, parts[10, 4])."""
        pb, su, av = C.c_float(), C.c_float(), C.c_float()
        parts = np.empty((10, 4), dtype=np.float64)
        self._check(self.lib.chdwf_thr_measure(
            self.h, res, _ptr(np.ascontiguousarray(u, dtype=np.complex128)), C.byref(pb),
            C.byref(su), C.byref(av), _ptr(parts)))
        return pb.value, su.value, av.value, parts

    def set_measure(self, iprint):
        self._check(self.lib.chdwf_thr_set_measure(self.h, iprint))

    def set_theta(self, theta):
        self._check(self.lib.chdwf_thr_set_theta(self.h, _ptr(np.ascontiguousarray(theta, dtype=np.float32))))

    def get_theta(self):
        th = np.empty((3, self.kvol), dtype=np.float32)
        self._check(self.lib.chdwf_thr_get_theta(self.h, _ptr(th)))
        return th

    def startup(self, seed):
        self._check(self.lib.chdwf_thr_startup(self.h, float(seed)))

    def seed(self):
        return self.lib.chdwf_thr_seed(self.h)

    def sweep(self) -> ThirringRecord:
        rec = ThirringRecord()
        self._check(self.lib.chdwf_thr_sweep(self.h, C.byref(rec)))
        return rec

    def close(self):
        if getattr(self, "h", None):
            self.lib.chdwf_thr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
