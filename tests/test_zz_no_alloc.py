"""The allocation-free congrad entry point (chdwf_congrad_static).

It serves callers that cannot allocate GPU memory themselves: a host program
whose device memory is owned by another runtime's pool or reserved in full at
start-up, or code that must not allocate.  Such callers cannot create a
context (creating one allocates), so this entry point takes every argument
explicitly and keeps its scratch in a static device array of the library.

Checked here through the C ABI:
  * two calls in a row give the same solution as the context-based
    chdwf_congrad_dev on the same inputs, within the congrad tolerance of the
    other tests (relative 1e-6), with the same iteration count, for imass 1
    and 3.  The second call also shows that nothing left in the shared
    static array from the first call leaks into the next solve;
  * the same solutions against the CPU oracle's congrad (rhmc/cheisdwf.f:
    1064-1157), with the tolerances of the context-based congrad test;
  * a NaN in chi returns CHDWF_NONFINITE, and a clean solve afterwards still
    agrees, so a failed call leaves nothing behind in the array.
The file is named to be collected last, so a run that stops at the first
failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import chiralheisenberg_b200 as chb
import pyoracle as po
from conftest import random_fields

pytestmark = pytest.mark.gpu

L, LT, LS = 6, 6, 6
RES = 1e-9


def _solve_static(lib, Phi, x0, chi, imass):
    import torch
    x = x0.clone()
    it = C.c_int(0)
    rc = lib.chdwf_congrad_static(C.c_void_p(Phi.data_ptr()), C.c_void_p(x.data_ptr()),
                                  C.c_void_p(chi.data_ptr()), L, LT, LS, 1.0, -1, RES, 0.2,
                                  imass, C.byref(it), None)
    torch.cuda.synchronize()
    return rc, x, it.value


def _solve_context(lib, gl, Phi, chi, imass):
    import torch
    xr = Phi.clone()
    itr = C.c_int(0)
    rc = lib.chdwf_congrad_dev(gl.h, C.c_void_p(Phi.data_ptr()), RES, C.byref(itr), 0.2, imass,
                               C.c_void_p(chi.data_ptr()), C.c_void_p(xr.data_ptr()))
    torch.cuda.synchronize()
    assert rc == 0
    return xr, itr.value


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("imass", [1, 3])
def test_congrad_static_matches_context_entry_point(imass):
    import torch
    lib = chb.load_library()
    cases = [random_fields(L, LT, LS, seed=41, chi_scale=0.4),
             random_fields(L, LT, LS, seed=42, chi_scale=0.4)]
    gl = chb.Lattice(L, LT, LS, beta=0.475, am3=1.0)
    inputs, refs = [], []
    for Phi_h, chi_h in cases:
        Phi = torch.from_numpy(Phi_h).cuda()
        chi = torch.from_numpy(chi_h).cuda()
        inputs.append((Phi, chi))
        refs.append(_solve_context(lib, gl, Phi, chi, imass))
    gl.close()
    # two calls of the allocation-free entry point in a row
    outs = [_solve_static(lib, Phi, Phi.clone(), chi, imass) for Phi, chi in inputs]
    lat = po.make_lat(L, LT, LS)
    for (rc, xs, its), (xr, itr), (Phi_h, chi_h) in zip(outs, refs, cases):
        assert rc == chb.CHDWF_OK, rc
        assert its == itr
        err = (torch.linalg.norm(xs - xr) / torch.linalg.norm(xr)).item()
        assert err <= 1e-6, err
        # the oracle: REAL*4 scalars summed sequentially there, in FP64 and
        # rounded once here, so iterations within 2 and x to the solver
        # tolerance (as the context-based congrad test)
        xo, ito, capped = po.congrad(lat, Phi_h, chi_h, Phi_h, RES, hpin=0.2, imass=imass)
        assert not capped
        assert abs(its - ito) <= 2, (its, ito)
        assert _rel(xs.cpu().numpy(), xo) < 1e-6


def test_congrad_static_reports_nonfinite_and_recovers():
    """A NaN in chi stops the solve with CHDWF_NONFINITE; the next call on
    clean inputs starts from a cleared control block and agrees with the
    context entry point."""
    import torch
    lib = chb.load_library()
    Phi_h, chi_h = random_fields(L, LT, LS, seed=43, chi_scale=0.4)
    Phi = torch.from_numpy(Phi_h).cuda()
    chi = torch.from_numpy(chi_h).cuda()
    bad = chi.clone()
    bad[1, 7] = float("nan")
    rc, _, _ = _solve_static(lib, Phi, Phi.clone(), bad, 1)
    assert rc == chb.CHDWF_NONFINITE, rc
    rc, xs, its = _solve_static(lib, Phi, Phi.clone(), chi, 1)
    assert rc == chb.CHDWF_OK, rc
    gl = chb.Lattice(L, LT, LS, beta=0.475, am3=1.0)
    xr, itr = _solve_context(lib, gl, Phi, chi, 1)
    gl.close()
    assert its == itr
    assert (torch.linalg.norm(xs - xr) / torch.linalg.norm(xr)).item() <= 1e-6


def test_congrad_static_rejects_oversize():
    """Lattices beyond the static scratch, and sizes whose 32-bit volume
    would wrap, are refused before any GPU work."""
    lib = chb.load_library()
    it = C.c_int(0)
    dummy = C.c_void_p(1)
    for dims in [(32, 32, 16), (65536, 65536, 4), (2048, 2048, 2048)]:
        rc = lib.chdwf_congrad_static(dummy, dummy, dummy, *dims, 1.0, -1, 1e-9, 0.0, 1,
                                      C.byref(it), None)
        assert rc == chb.CHDWF_BAD_ARG, dims
