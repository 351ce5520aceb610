"""CPU tests of the oracle's restatement of the HMC predecessor,
mh/cheisdwf_hmc.f (single precision, oracle/chdwf_oracle_hmc.c).

Pins: its operator against the two FP64 restatements of the RHMC operator
(the live v2 routines and the table-driven v1 routines of rhmc/cheisdwf.f,
which mh/cheisdwf_hmc.f:1334-2028 repeats in single precision without the
pinning term); the adjoint identity; the chi-force against the exact
gradient of the action; the solver's stopping rule; the random stream of a
sweep replayed draw by draw.
"""
import numpy as np
import pytest

import pyoracle as po
from conftest import random_fields
from test_oracle import _dense

SEED = 693764523745.0


@pytest.mark.parametrize("imass", [1, 3])
def test_hmc_operator_matches_fp64_operators(imass):
    lat = po.make_lat(4, 4, 4)
    R, chi = random_fields(4, 4, 4, seed=3, chi_scale=0.5)
    R32, chi32 = R.astype(np.complex64), chi.astype(np.float32)
    sp = po.hmc_dslash(lat, R32, chi32, imass=imass)
    for v1 in (True, False):
        dp = po.dslash(lat, R32.astype(np.complex128), chi32.astype(np.float64), imass=imass,
                       v1=v1)
        assert np.abs(sp - dp).max() <= 5e-7 * np.abs(dp).max()


@pytest.mark.parametrize("imass", [1, 3])
def test_hmc_operator_adjoint(imass):
    lat = po.make_lat(4, 4, 6)
    R, chi = random_fields(4, 4, 6, seed=4, chi_scale=0.5)
    y = random_fields(4, 4, 6, seed=9)[0].astype(np.complex64)
    R32, chi32 = R.astype(np.complex64), chi.astype(np.float32)
    lhs = np.vdot(y.astype(complex), po.hmc_dslash(lat, R32, chi32, imass).astype(complex))
    rhs = np.vdot(po.hmc_dslash(lat, y, chi32, imass, dag=True).astype(complex),
                  R32.astype(complex))
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)


@pytest.mark.parametrize("imass", [1, 3])
def test_hmc_force_is_gradient(imass):
    """dSdchi of force (mh/cheisdwf_hmc.f:416-555) for X1 = (M^dag M)^-1 Phi
    equals the gradient of S = 2 beta chi^2 + Phi^dag (M^dag M)^-1 Phi,
    4 beta chi - 2 Re (M X1)^dag (dM/dchi) X1, evaluated densely in FP64.
    M is linear in chi, so dM/dchi is M(chi + e) - M(chi) exactly (a small
    finite-difference step would be rounded by the operator's REAL*4 wall
    coupling)."""
    L, Lt, Ls, beta = 2, 4, 4, 0.475
    kv = L * L * Lt
    lat = po.make_lat(L, Lt, Ls, beta=beta)
    R, chi = random_fields(L, Lt, Ls, seed=5, chi_scale=0.5)
    chi = chi.astype(np.float32).astype(np.float64)
    Phi = R.reshape(-1)
    M = _dense(lat, chi, imass=imass)
    X = np.linalg.solve(M.conj().T @ M, Phi)
    MX = M @ X
    grad = np.zeros((3, kv))
    for a in range(3):
        for i in range(kv):
            c = chi.copy()
            c[a, i] += 1.0
            dM = _dense(lat, c, imass=imass) - M
            grad[a, i] = 4 * beta * chi[a, i] - 2 * np.vdot(MX, dM @ X).real
    dS = po.hmc_derivs(lat, X.reshape(po.spinor_shape(lat)).astype(np.complex64),
                       chi.astype(np.float32), imass=imass)
    assert np.abs(dS - grad).max() <= 1e-6 * np.abs(grad).max()


def test_hmc_congrad_stopping_rule():
    lat = po.make_lat(4, 4, 8)
    Phi, chi = random_fields(4, 4, 8, seed=7)
    Phi32, chi32 = Phi.astype(np.complex64), chi.astype(np.float32)
    x, it, capped = po.hmc_congrad(lat, Phi32, chi32, Phi32, 1e-6)
    assert not capped and 2 <= it < 4 * 4 * 4 * 8
    r = Phi32.astype(complex) - po.dslash(lat, po.dslash(lat, x.astype(complex),
                                                          chi32.astype(float)),
                                          chi32.astype(float), dag=True)
    # stopping rule |r|^2 < kferm res^2 on the recursive REAL*4 residual; the
    # true residual of the single-precision iterate sits near it
    assert np.vdot(r, r).real < 100 * Phi.size * 1e-12


@pytest.mark.parametrize("imass", [1, 3])
def test_hmc_sweep_stream_and_energy(imass):
    """Two sweeps: the generator advances by exactly the draws of the main
    loop (8*kthird gauss0, 2 gaussp, one rano(yrun) per MD step, one more
    only when dH < 0: mh/cheisdwf_hmc.f:154-187, :228, :259-260), the trajectory
    ends at the first ytest below 1/iterl, and at the start of a trajectory
    hf = Phi^dag (M^dag M)^-1 Phi = |R|^2."""
    L, Lt, Ls, dt, iterl = 4, 4, 4, 0.1, 5
    kv = L * L * Lt
    chi = (np.random.default_rng(2).standard_normal((3, kv)) / np.sqrt(0.475)).astype(np.float32)
    sw = po.HmcSweeper(L, Lt, Ls, 0.475, 1.0, dt, 0.01, imass, iterl, chi=chi, seed=SEED,
                       iprint=2)
    rand = po.Rand(SEED)
    proby = np.float32(1.0) / np.float32(iterl)
    for k in range(2):
        c = sw.chi.copy()
        hg0 = float(np.float32(2.0) * np.float32(0.475)) * float(np.sum((c * c).astype(np.float64)))
        rec = sw.sweep()
        R2 = 0.0
        for _ in range(8 * Ls):
            ps = rand.gauss0(kv)
            R2 += float(np.sum(ps.astype(np.float64) ** 2))
        rand.gaussp(kv)
        rand.gaussp(kv)
        n = 0
        while True:
            n += 1
            if rand.rano("yrun") < proby or n == 1000:
                break
        assert rec.nsteps == n and rec.nforce == n + 1
        assert rec.drew_x == (rec.dH < 0)
        if rec.drew_x:
            assert rec.x == np.float32(rand.rano("yrun"))
        assert sw.seed() == rand.seed()
        assert rec.measured == ((k + 1) % 2 == 0)
        # S0 = hg + hf on the starting chi, hf = |R|^2 to single precision
        assert abs((rec.S0 - hg0) - R2) <= 1e-5 * R2, (rec.S0 - hg0, R2)
        assert np.isfinite(rec.H1) and abs(rec.dH) < 0.1 * R2
    sw.close()
