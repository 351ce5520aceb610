"""CPU checks of the C-ABI library: it builds, loads without a GPU, and
exports every function include/chdwf.h declares (no compute calls here)."""
import ctypes as C
import os
import re

import pytest

import chiralheisenberg_b200 as chb
from chiralheisenberg_b200 import build as chbuild
from conftest import ROOT


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for h in sorted(os.listdir(inc)):
        if h.endswith(".h"):
            text = open(os.path.join(inc, h)).read()
            names |= set(re.findall(r"\b(chdwf_\w+)\s*\(", text))
    return sorted(names)


def test_header_matches_python_export_list():
    assert set(declared_symbols()) == set(chb.EXPORTS)


def test_library_builds_and_exports_all_symbols():
    lib_path = chbuild.build()
    assert os.path.exists(lib_path)
    lib = C.CDLL(lib_path)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_version_string():
    chbuild.build()
    assert "sm_100a" in chb.version()


def test_create_rejects_bad_sizes():
    chbuild.build()
    lib = chb.load_library()
    h = C.c_void_p()
    assert lib.chdwf_create(C.byref(h), 1, 4, 4, 0) == chb.CHDWF_BAD_ARG
    assert lib.chdwf_create(None, 4, 4, 4, 0) == chb.CHDWF_BAD_ARG


def test_null_context_is_rejected():
    chbuild.build()
    lib = chb.load_library()
    assert lib.chdwf_set_para(None, 0.5, 1.0, -1) == chb.CHDWF_BAD_ARG
    assert lib.chdwf_dslash(None, None, None, None, 0.0, 0.0, 1) == chb.CHDWF_BAD_ARG


def test_hmc_and_thirring_reject_bad_arguments():
    """The single-precision HMC and the Thirring contexts validate their
    arguments before touching a device: bad lattices, mass terms and
    trajectory lengths are refused, and every entry point refuses a NULL
    context."""
    chbuild.build()
    lib = chb.load_library()
    h = C.c_void_p()
    assert lib.chdwf_hmc_create(C.byref(h), 1, 4, 4, 0.1, 0.5, 1.0, 0.0, 1, 5, 0) == chb.CHDWF_BAD_ARG
    assert lib.chdwf_hmc_create(C.byref(h), 4, 4, 4, 0.1, 0.5, 1.0, 0.0, 5, 5, 0) == chb.CHDWF_BAD_ARG
    assert lib.chdwf_hmc_create(C.byref(h), 4, 4, 4, 0.1, 0.5, 1.0, 0.0, 1, 0, 0) == chb.CHDWF_BAD_ARG
    assert b"bad lattice" in lib.chdwf_hmc_last_error(None)
    assert lib.chdwf_thr_create(C.byref(h), 4, 1, 4, 0.1, 0.5, 1.0, 0.2, 1, 5, 0) == chb.CHDWF_BAD_ARG
    assert lib.chdwf_thr_create(C.byref(h), 4, 4, 4, 0.1, 0.5, 1.0, 0.2, 2, 5, 0) == chb.CHDWF_BAD_ARG
    assert lib.chdwf_thr_create(None, 4, 4, 4, 0.1, 0.5, 1.0, 0.2, 1, 5, 0) == chb.CHDWF_BAD_ARG
    assert lib.chdwf_hmc_dslash(None, None, None, None, 1) == chb.CHDWF_BAD_ARG
    assert lib.chdwf_hmc_sweep(None, None) == chb.CHDWF_BAD_ARG
    assert lib.chdwf_hmc_set_measure(None, 2) == chb.CHDWF_BAD_ARG
    assert lib.chdwf_thr_dslash(None, None, None, None, 0.2, 1) == chb.CHDWF_BAD_ARG
    assert lib.chdwf_thr_sweep(None, None) == chb.CHDWF_BAD_ARG
    z = (C.c_double * 26)()
    assert lib.chdwf_thr_set_remez(None, 2, z, z, z, z, 25) == chb.CHDWF_BAD_ARG
    assert lib.chdwf_thr_set_measure(None, 2) == chb.CHDWF_BAD_ARG
