"""The allocation-free congrad entry point (chdwf_congrad_static).

It serves callers that cannot allocate GPU memory themselves: a host program
whose device memory is owned by another runtime's pool or reserved in full at
start-up, or code that must not allocate.  Such callers cannot create a
context (creating one allocates), so this entry point takes every argument
explicitly and keeps its scratch in a static device array of the library.

Checked here through the C ABI: two calls in a row give the same solution as
the context-based chdwf_congrad_dev on the same inputs, within the congrad
tolerance of the other tests (relative 1e-6), with the same iteration count.
The second call also shows that nothing left in the shared static array from
the first call leaks into the next solve.  The file is named to be collected
last, so a run that stops at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import chiralheisenberg_b200 as chb
from conftest import random_fields

pytestmark = pytest.mark.gpu


def _solve_static(lib, Phi, x0, chi, L, Lt, Ls):
    import torch
    x = x0.clone()
    it = C.c_int(0)
    rc = lib.chdwf_congrad_static(C.c_void_p(Phi.data_ptr()), C.c_void_p(x.data_ptr()),
                                  C.c_void_p(chi.data_ptr()), L, Lt, Ls, 1.0, -1, 1e-9, 0.2, 1,
                                  C.byref(it), None)
    torch.cuda.synchronize()
    assert rc == 0, rc
    return x, it.value


def test_congrad_static_matches_context_entry_point():
    import torch
    L, Lt, Ls = 6, 6, 6
    lib = chb.load_library()
    cases = [random_fields(L, Lt, Ls, seed=41, chi_scale=0.4),
             random_fields(L, Lt, Ls, seed=42, chi_scale=0.4)]
    gl = chb.Lattice(L, Lt, Ls, beta=0.475, am3=1.0)
    inputs, refs = [], []
    for Phi_h, chi_h in cases:
        Phi = torch.from_numpy(Phi_h).cuda()
        chi = torch.from_numpy(chi_h).cuda()
        # the existing entry point (context, same kernels)
        xr = Phi.clone()
        itr = C.c_int(0)
        rc = lib.chdwf_congrad_dev(gl.h, C.c_void_p(Phi.data_ptr()), 1e-9, C.byref(itr), 0.2, 1,
                                   C.c_void_p(chi.data_ptr()), C.c_void_p(xr.data_ptr()))
        torch.cuda.synchronize()
        assert rc == 0
        inputs.append((Phi, chi))
        refs.append((xr, itr.value))
    gl.close()
    # two calls of the allocation-free entry point in a row
    outs = [_solve_static(lib, Phi, Phi.clone(), chi, L, Lt, Ls) for Phi, chi in inputs]
    for (xs, its), (xr, itr) in zip(outs, refs):
        assert its == itr
        err = (torch.linalg.norm(xs - xr) / torch.linalg.norm(xr)).item()
        assert err <= 1e-6, err


def test_congrad_static_rejects_oversize():
    """Lattices beyond the static scratch are refused before any GPU work."""
    lib = chb.load_library()
    it = C.c_int(0)
    dummy = C.c_void_p(1)
    rc = lib.chdwf_congrad_static(dummy, dummy, dummy, 32, 32, 16, 1.0, -1, 1e-9, 0.0, 1,
                                  C.byref(it), None)
    assert rc == chb.CHDWF_BAD_ARG
