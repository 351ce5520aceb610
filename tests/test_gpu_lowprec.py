"""Reduced-precision paths (no reference counterpart: the reference is FP64
throughout), checked against the FP64 oracle and the FP64 GPU path.

  operator, FP32 storage + arithmetic      relative L2 error <= 1e-6
  operator, FP16 storage, FP32 arithmetic  relative L2 error <= 2e-3
  mixed trajectory (FP32 force solves)     same accept/reject decisions and
                                           MD steps; |dH_mixed - dH_fp64| <= 1e-8 * |H0|
"""
import ctypes as C

import numpy as np
import pytest

import pyoracle as po
import chiralheisenberg_b200 as chb
from conftest import random_fields

pytestmark = pytest.mark.gpu


def _lp_apply(gl, R, chi, prec, dag, hpin=0.3):
    import torch
    dt = torch.complex64 if prec == 1 else torch.float16
    Rt = torch.from_numpy(R.astype(np.complex64)).cuda()
    if prec == 2:
        Rt = torch.view_as_real(Rt).to(torch.float16).contiguous()
    out = torch.empty_like(Rt)
    chit = torch.from_numpy(np.ascontiguousarray(chi)).cuda()
    rc = gl.lib.chdwf_dslash_dev_lp(gl.h, C.c_void_p(out.data_ptr()), C.c_void_p(Rt.data_ptr()),
                                    C.c_void_p(chit.data_ptr()), hpin, 1, int(dag), prec, None)
    assert rc == 0
    gl.lib.chdwf_traj_sync(gl.h)
    torch.cuda.synchronize()
    if prec == 2:
        o = out.float().cpu().numpy()
        return o[..., 0] + 1j * o[..., 1]
    return out.cpu().numpy().astype(np.complex128)


@pytest.mark.parametrize("prec,tol", [(1, 1e-6), (2, 2e-3)])
@pytest.mark.parametrize("dag", [False, True])
@pytest.mark.parametrize("Ls", [8, 5])
def test_operator_reduced_precision(prec, tol, dag, Ls):
    """FP32 storage takes the two-point kernel when Ls is even and the
    one-point kernel when it is odd; FP16 always the one-point kernel."""
    L, Lt = 8, 8
    R, chi = random_fields(L, Lt, Ls, seed=31)
    lat = po.make_lat(L, Lt, Ls)
    ref = po.dslash(lat, R, chi, hpin=0.3, imass=1, dag=dag)
    gl = chb.Lattice(L, Lt, Ls)
    out = _lp_apply(gl, R, chi, prec, dag)
    err = np.linalg.norm(out.reshape(-1) - ref.reshape(-1)) / np.linalg.norm(ref)
    assert err <= tol, err


def test_mixed_precision_trajectory(remez):
    """FP32 Krylov vectors in the force solves, FP64 heatbath/hamilton: the
    same Markov chain decisions and dH within 1e-8 of H."""
    L, Lt, Ls = 8, 8, 8
    beta = 0.475
    chi = np.random.default_rng(12345).standard_normal((3, L * L * Lt)) / np.sqrt(beta)
    recs = {}
    for mode in ("f64", "f32"):
        prog = chb.Program(L, Lt, Ls, 0.1, beta, 1.0, 0.01, 0.0, 1, 10, remez["remez2"],
                           remez["remez4"], remez["remez2g"])
        prog.set_chi(chi)
        prog.startup(693764523745.0)
        prog.set_measure(5, False)
        prog.set_precision(md=mode, accept="f64")
        recs[mode] = [prog.sweep() for _ in range(2)]
        prog.close()
    for a, b in zip(recs["f64"], recs["f32"]):
        assert a.nsteps == b.nsteps and a.accepted == b.accepted
        assert abs(a.dH - b.dH) <= 1e-8 * abs(a.H0), (a.dH, b.dH)


def test_chunk_timing_keeps_the_trajectory(remez):
    """Timing mode 2 (events around each graph-replayed chunk of pass 1) runs
    the same trajectory bit for bit as an untimed sweep, times whole chunks
    of both vector precisions, and per iteration comes out no slower than
    the sum of the per-launch event times (mode 1) of the same trajectory."""
    L, Lt, Ls = 8, 8, 8
    beta = 0.475
    chi = np.random.default_rng(4242).standard_normal((3, L * L * Lt)) / np.sqrt(beta)
    prog = chb.Program(L, Lt, Ls, 0.1, beta, 1.0, 0.01, 0.0, 1, 10, remez["remez2"],
                       remez["remez4"], remez["remez2g"])
    prog.set_chi(chi)
    prog.startup(693764523745.0)
    prog.set_measure(5, False)
    prog.set_precision(md="f32", accept="f64")
    chi0, st0 = prog.get_chi(), prog.get_state()
    plain = prog.sweep()
    prog.set_chi(chi0)
    prog.set_state(st0)
    prog.timing(True, chunks=True)
    timed = prog.sweep()
    us, its = prog.timing_chunks()
    prog.timing(False)
    assert (timed.dH, timed.H0, timed.accepted) == (plain.dH, plain.H0, plain.accepted)
    assert np.all(its > 0) and np.all(its % 16 == 0) and np.all(us > 0), (us, its)
    prog.set_chi(chi0)
    prog.set_state(st0)
    prog.timing(True)
    prog.sweep()
    ms, timed_n, _, _ = prog.timing_read()
    prog.timing(False)
    prog.close()
    for prec in (0, 1):
        per_launch = 1e3 * sum(ms[4 * prec + c] / max(timed_n[4 * prec + c], 1) for c in (0, 1))
        assert us[prec] <= 1.05 * per_launch, (prec, us[prec], per_launch)


@pytest.mark.parametrize("Ls", [5, 6])
@pytest.mark.parametrize("store", [-1.0, 0.0])
def test_mixed_force_thread_shapes(remez, Ls, store):
    """The FP32 force solves on both of their thread shapes -- two adjacent
    points per thread (Ls even) and one point with both flavours (Ls odd) --
    with pass 2 from the stored basis (store < 0) and by regenerating the
    vectors (store 0): the FP64 chain's decisions, dH within 1e-8 of H."""
    L, Lt = 6, 6
    beta = 0.475
    chi = np.random.default_rng(99).standard_normal((3, L * L * Lt)) / np.sqrt(beta)
    recs = {}
    for mode in ("f64", "f32"):
        prog = chb.Program(L, Lt, Ls, 0.1, beta, 1.0, 0.01, 0.0, 1, 5, remez["remez2"],
                           remez["remez4"], remez["remez2g"])
        prog.set_basis_store(store)
        prog.set_chi(chi)
        prog.startup(693764523745.0)
        prog.set_measure(5, False)
        prog.set_precision(md=mode, accept="f64")
        recs[mode] = [prog.sweep() for _ in range(2)]
        prog.close()
    for a, b in zip(recs["f64"], recs["f32"]):
        assert a.nsteps == b.nsteps and a.accepted == b.accepted
        assert abs(a.dH - b.dH) <= 1e-8 * abs(a.H0), (a.dH, b.dH)


# FP32 and FP16 storage at the operator sweep's sizes, against the FP64
# oracle: relative L2 error <= 1e-6 (FP32) and <= 2e-3 (FP16 storage, the
# half-precision rounding of inputs and outputs).
@pytest.mark.parametrize("L,Ls", [(16, 16), (24, 24), (32, 16)])
@pytest.mark.parametrize("prec,tol", [(1, 1e-6), (2, 2e-3)])
def test_operator_reduced_precision_sweep_sizes(L, Ls, prec, tol):
    R, chi = random_fields(L, L, Ls, seed=3100 + L + Ls)
    lat = po.make_lat(L, L, Ls)
    gl = chb.Lattice(L, L, Ls)
    for dag in (False, True):
        ref = po.dslash(lat, R, chi, hpin=0.3, imass=1, dag=dag)
        out = _lp_apply(gl, R, chi, prec, dag)
        err = np.linalg.norm(out.reshape(-1) - ref.reshape(-1)) / np.linalg.norm(ref)
        print(f"L={L} Ls={Ls} prec={prec} dag={dag}: relative error {err:.3e}")
        assert err <= tol, err
    gl.close()
