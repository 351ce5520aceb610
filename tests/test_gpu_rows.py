"""The row-staged stencil kernels (csrc/row_stage.cuh) against the oracle and
against the point-gather kernels.

By default the row kernels run only where every block gets at least three
rows (L=24 and up); CHDWF_STENCIL=rows makes them run wherever their shared
memory fits, so they are exercised here on small lattices too, and
CHDWF_STENCIL=legacy selects the point-gather kernels for the comparison.

  FP64 operator M, M^dagger       bit-exact against the oracle (same per-element
                                  operation sequence as the point-gather kernel)
  FP32 / FP16 storage             relative 1e-6 / 2e-3 against the oracle
  multi-shift solve (iflag 0, 1)  against the oracle as in test_gpu_solvers
                                  (x to 1e-10, force to 2 REAL*4 ulps,
                                  iterations +-5); against the point-gather
                                  kernels: iterations +-2, x to 1e-12
  large rows (24^3x24 FP32, 16^3x16 FP64: the shapes the autotuner weighs
  for the trajectory)             bit-identical to the point-gather kernels
Every test checks, through chdwf_stencil_launches, that the row kernels did
run (a shape that cannot launch falls back to the point-gather kernels).
"""
import numpy as np
import pytest

import pyoracle as po
import chiralheisenberg_b200 as chb
from conftest import random_fields

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b))


@pytest.fixture(autouse=True)
def rows_ran():
    n0 = chb.stencil_launches()["rows"]
    yield
    assert chb.stencil_launches()["rows"] > n0, "the row kernels did not run"


@pytest.mark.parametrize("L,Lt,Ls", [(8, 8, 8), (6, 4, 6), (12, 12, 8), (16, 16, 16),
                                     (4, 6, 4)])
@pytest.mark.parametrize("imass", [1, 3])
def test_rows_operator_bit_exact(monkeypatch, L, Lt, Ls, imass):
    monkeypatch.setenv("CHDWF_STENCIL", "rows")
    R, chi = random_fields(L, Lt, Ls, seed=500 + L * 10 + Ls)
    hpin = 0.37 if imass == 1 else 0.0
    lat = po.make_lat(L, Lt, Ls, beta=0.475, am3=1.0)
    gl = chb.Lattice(L, Lt, Ls, beta=0.475, am3=1.0)
    for dag in (False, True):
        ref = po.dslash(lat, R, chi, hpin=hpin, imass=imass, dag=dag)
        out = (gl.dslashd if dag else gl.dslash)(R, chi, hpin=hpin, imass=imass)
        assert np.array_equal(out.view(np.float64), ref.view(np.float64)), dag
    gl.close()


def test_rows_operator_boundary_and_height(monkeypatch):
    monkeypatch.setenv("CHDWF_STENCIL", "rows")
    L, Lt, Ls = 4, 6, 4
    R, chi = random_fields(L, Lt, Ls, seed=11)
    for ibound, am3 in ((1, 1.0), (-1, 0.7)):
        lat = po.make_lat(L, Lt, Ls, am3=am3, ibound=ibound)
        gl = chb.Lattice(L, Lt, Ls, am3=am3, ibound=ibound)
        for dag in (False, True):
            ref = po.dslash(lat, R, chi, imass=1, dag=dag)
            out = (gl.dslashd if dag else gl.dslash)(R, chi, imass=1)
            assert np.array_equal(out.view(np.float64), ref.view(np.float64))
        gl.close()


@pytest.mark.parametrize("prec,tol", [(1, 1e-6), (2, 2e-3)])
def test_rows_operator_reduced_precision(monkeypatch, prec, tol):
    from test_gpu_lowprec import _lp_apply
    monkeypatch.setenv("CHDWF_STENCIL", "rows")
    L, Lt, Ls = 8, 8, 8
    R, chi = random_fields(L, Lt, Ls, seed=31)
    lat = po.make_lat(L, Lt, Ls)
    gl = chb.Lattice(L, Lt, Ls)
    for dag in (False, True):
        ref = po.dslash(lat, R, chi, hpin=0.3, imass=1, dag=dag)
        out = _lp_apply(gl, R, chi, prec, dag)
        assert rel(out, ref) <= tol
    gl.close()


@pytest.mark.parametrize("imass", [1, 3])
def test_rows_qmrherm_against_oracle_and_legacy(monkeypatch, remez, imass):
    L, Lt, Ls = 8, 8, 8
    r = remez["remez4"]
    Phi, chi = random_fields(L, Lt, Ls, seed=21, chi_scale=0.4)
    lat = po.make_lat(L, Lt, Ls, beta=0.475)
    xr, itr, st, _ = po.qmrherm(lat, Phi, chi, r["anum"], r["aden"], 1e-9, imass=imass)
    out = {}
    for mode in ("rows", "legacy"):
        monkeypatch.setenv("CHDWF_STENCIL", mode)
        gl = chb.Lattice(L, Lt, Ls, beta=0.475)
        for store in (-1.0, 0.0):
            gl.set_basis_store(store)
            out[(mode, store)] = gl.qmrherm(Phi, 1e-9, r["anum"], r["aden"], 0, chi, imass=imass)
        gl.close()
    for (mode, store), (xg, itg, _) in out.items():
        assert abs(itg - itr) <= 5, (mode, store, itg, itr)
        assert rel(xg, xr) < 1e-10, (mode, store)
    xa, ita, _ = out[("rows", -1.0)]
    xb, itb, _ = out[("legacy", -1.0)]
    assert abs(ita - itb) <= 2
    assert rel(xa, xb) < 1e-12


def test_rows_force_against_oracle(monkeypatch, remez):
    """iflag 1 (the wall store) on the row kernels."""
    monkeypatch.setenv("CHDWF_STENCIL", "rows")
    L, Lt, Ls = 6, 6, 6
    r = remez["remez2g"]
    Phi, chi = random_fields(L, Lt, Ls, seed=22, chi_scale=0.4)
    lat = po.make_lat(L, Lt, Ls, beta=0.475)
    dS0 = np.random.default_rng(1).standard_normal((3, L * L * Lt)).astype(np.float32)
    _, itr, _, dSr = po.qmrherm(lat, Phi, chi, r["anum"], r["aden"], 1e-6, iflag=1, imass=1,
                                hpin=0.0, dSdchi=dS0.copy())
    gl = chb.Lattice(L, Lt, Ls, beta=0.475)
    for store in (-1.0, 0.0):
        gl.set_basis_store(store)
        _, itg, dSg = gl.qmrherm(Phi, 1e-6, r["anum"], r["aden"], 1, chi, dSdchi=dS0.copy())
        assert abs(itg - itr) <= 5
        assert np.abs(dSg - dSr).max() <= 2 * np.spacing(np.float32(np.abs(dSr).max()))
    gl.close()


@pytest.mark.parametrize("Ls", [6, 5])
def test_rows_mixed_precision_trajectory(monkeypatch, remez, Ls):
    """Mixed precision with the row kernels forced: the FP64 heatbath and
    action solves run on rows in both cases; the FP32 force solves run on
    rows for Ls 5 (rows of 30 points), while for Ls 6 their vectors are in
    the split layout, which only the point-gather kernels read.  The FP64
    chain's decisions and dH within 1e-8 of H."""
    monkeypatch.setenv("CHDWF_STENCIL", "rows")
    L, Lt = 6, 6
    beta = 0.475
    chi = np.random.default_rng(99).standard_normal((3, L * L * Lt)) / np.sqrt(beta)
    recs = {}
    for mode in ("f64", "f32"):
        prog = chb.Program(L, Lt, Ls, 0.1, beta, 1.0, 0.01, 0.0, 1, 5, remez["remez2"],
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


@pytest.mark.parametrize("L,Ls,prec", [(24, 24, 1), (16, 16, 0)])
def test_rows_large_bit_identical_to_gather(monkeypatch, L, Ls, prec):
    """The row kernels at the sizes the autotuner weighs them: the same bits
    as the point-gather kernels (both keep dwf_apply_flavour's per-element
    operation sequence, FP32 without contraction)."""
    from test_gpu_lowprec import _lp_apply
    R, chi = random_fields(L, L, Ls, seed=41)
    outs = {}
    for mode in ("rows", "legacy"):
        monkeypatch.setenv("CHDWF_STENCIL", mode)
        gl = chb.Lattice(L, L, Ls, beta=0.475)
        for dag in (False, True):
            if prec == 0:
                outs[(mode, dag)] = (gl.dslashd if dag else gl.dslash)(R, chi, hpin=0.3, imass=1)
            else:
                outs[(mode, dag)] = _lp_apply(gl, R, chi, prec, dag)
        gl.close()
    for dag in (False, True):
        a, b = outs[("rows", dag)], outs[("legacy", dag)]
        assert np.array_equal(a, b), dag
