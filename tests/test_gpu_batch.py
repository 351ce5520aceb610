"""Batched propagator solves (chdwf_congrad_batch) against the same solves one
at a time (chdwf_congrad_dev), on lattices of uneven size with their own chi,
imass and hpin.  Both run the same kernels per system with the same
reduction partition, so solutions and iteration counts agree exactly; the
test allows rounding-level differences (relative 1e-12)."""
import ctypes as C

import numpy as np
import pytest

import chiralheisenberg_b200 as chb
from conftest import random_fields

pytestmark = pytest.mark.gpu


def test_batch_matches_one_at_a_time():
    import torch
    sizes = [(4, 4, 4, 1, 0.0), (6, 4, 8, 3, 0.0), (8, 8, 4, 1, 0.5), (4, 6, 6, 1, 0.2),
             (8, 8, 8, 3, 0.0), (6, 6, 2, 1, 0.0)]
    keep, systems, refs = [], [], []
    for k, (L, Lt, Ls, imass, hpin) in enumerate(sizes):
        Phi_h, chi_h = random_fields(L, Lt, Ls, seed=50 + k, chi_scale=0.5)
        Phi = torch.from_numpy(Phi_h).cuda()
        chi = torch.from_numpy(chi_h).cuda()
        x = Phi.clone()
        gl = chb.Lattice(L, Lt, Ls, am3=1.0)
        xr = Phi.clone()
        it = C.c_int()
        rc = gl.lib.chdwf_congrad_dev(gl.h, C.c_void_p(Phi.data_ptr()), 1e-8, C.byref(it), hpin,
                                      imass, C.c_void_p(chi.data_ptr()), C.c_void_p(xr.data_ptr()))
        torch.cuda.synchronize()
        assert rc == 0
        gl.close()
        refs.append((xr, it.value))
        keep += [Phi, chi, x]
        systems.append(chb.CgSystem(L, Lt, Ls, imass, hpin, 1.0, -1, Phi.data_ptr(),
                                    x.data_ptr(), chi.data_ptr()))
    host = chb.Lattice(4, 4, 4)
    its, sts = chb.congrad_batch(host, systems, 1e-8)
    torch.cuda.synchronize()
    host.close()
    assert (sts == 0).all()
    for k, (xr, itr) in enumerate(refs):
        x = keep[3 * k + 2]
        assert its[k] == itr
        err = (torch.linalg.norm(x - xr) / torch.linalg.norm(xr)).item()
        assert err <= 1e-12, (k, err)


def test_batched_propagators_equal_sequential(remez):
    """chdwf_traj_propagators (the sources of fermion() as one batched,
    multi-right-hand-side solve) gives the same walls, bit for bit, and the
    same iterations as chdwf_traj_propagator source by source
    (rhmc/cheisdwf.f:937-1012)."""
    import ctypes as C
    L, Lt, Ls = 6, 8, 6
    beta = 0.475
    prog = chb.Program(L, Lt, Ls, 0.1, beta, 1.0, 0.01, 0.2, 1, 10, remez["remez2"],
                       remez["remez4"], remez["remez2g"])
    chi = np.random.default_rng(5).standard_normal((3, L * L * Lt)) / np.sqrt(beta)
    prog.set_chi(chi)
    lib, ctx = prog.lib, prog.context
    assert lib.chdwf_traj_begin(ctx) == 0
    kvol = L * L * Lt
    srcs = [(2, 3), (2, 4), (5, 3), (5, 4), (8, 3), (8, 4)]
    seq_w, seq_it = [], []
    for t, d in srcs:
        w = np.empty(16 * kvol)
        it = C.c_int()
        assert lib.chdwf_traj_propagator(ctx, t, d, 1e-9, 0.0, 0.2, 1,
                                         w.ctypes.data_as(C.c_void_p), C.byref(it)) == 0
        seq_w.append(w)
        seq_it.append(it.value)
    tt = (C.c_int * len(srcs))(*[t for t, _ in srcs])
    dd = (C.c_int * len(srcs))(*[d for _, d in srcs])
    its = (C.c_int * len(srcs))()
    wb = np.empty(16 * kvol * len(srcs))
    assert lib.chdwf_traj_propagators(ctx, len(srcs), tt, dd, 1e-9, 0.0, 0.2, 1,
                                      wb.ctypes.data_as(C.c_void_p), its) == 0
    prog.close()
    assert list(its) == seq_it
    for i, w in enumerate(seq_w):
        assert np.array_equal(wb[16 * kvol * i:16 * kvol * (i + 1)], w), i
