"""The HMC predecessor mh/cheisdwf_hmc.f on the GPU (include/chdwf_hmc.h)
against the oracle's single-precision restatement (oracle/chdwf_oracle_hmc.c).

Tolerances:
  operator M, M^dagger, chi force      bit-exact (REAL*4 arithmetic, same
                                       per-element operation order, no FMA)
  congrad x                            |x - x_oracle| <= 1e-5 max|x_oracle|;
                                       true residual within 1.5x the oracle's;
                                       iterations within 10% (+-3).
      The reference sums alphad and betan element by element in REAL*4;
      the GPU sums in FP64 and rounds once.  A CPU model of the GPU's sums
      gives the same solution to 1.6e-6 relative (the single-precision
      floor) and iterations equal or within 1 at res 1e-6, within 13 of 165
      at res 1e-9 (4^3 x 4 and 6^3 x 8, both mass terms).
  sweeps: H0, S0, H1, dH               within 1e-5 |H0|: hf = Phi^dag X1 carries
                                       the solver's 1.6e-6 relative error.
      Accept/reject, the Metropolis draw and the trajectory length are
      compared while the oracle's decision margins (|dH| for the draw,
      |x - y| for the acceptance) exceed that tolerance.
"""
import numpy as np
import pytest

import pyoracle as po
import chiralheisenberg_b200 as chb

pytestmark = pytest.mark.gpu

SEED = 693764523745.0


def _fields(L, Lt, Ls, seed):
    rng = np.random.default_rng(seed)
    sh = (2, 4, Lt, L, L, Ls)
    R = (rng.standard_normal(sh) + 1j * rng.standard_normal(sh)).astype(np.complex64)
    chi = (0.7 * rng.standard_normal((3, L * L * Lt))).astype(np.float32)
    return R, chi


@pytest.mark.parametrize("shape", [(4, 4, 4), (3, 2, 5), (6, 4, 8), (8, 8, 16)])
@pytest.mark.parametrize("imass", [1, 3])
def test_hmc_operator_and_force_bit_exact(shape, imass):
    L, Lt, Ls = shape
    R, chi = _fields(L, Lt, Ls, seed=L * 100 + Lt * 10 + Ls)
    lat = po.make_lat(L, Lt, Ls, beta=0.475)
    h = chb.Hmc(L, Lt, Ls, 0.1, 0.475, 1.0, 0.0, imass, 5)
    try:
        assert np.array_equal(h.dslash(R, chi), po.hmc_dslash(lat, R, chi, imass))
        assert np.array_equal(h.dslash(R, chi, dag=True),
                              po.hmc_dslash(lat, R, chi, imass, dag=True))
        assert np.array_equal(h.derivs(R, chi), po.hmc_derivs(lat, R, chi, imass))
    finally:
        h.close()


@pytest.mark.parametrize("imass", [1, 3])
@pytest.mark.parametrize("res", [1e-6, 1e-9])
def test_hmc_congrad(imass, res):
    L, Lt, Ls = 6, 6, 8
    Phi, chi = _fields(L, Lt, Ls, seed=7)
    lat = po.make_lat(L, Lt, Ls, beta=0.475)
    xo, ito, capo = po.hmc_congrad(lat, Phi, chi, Phi, res, imass)
    h = chb.Hmc(L, Lt, Ls, 0.1, 0.475, 1.0, 0.0, imass, 5)
    try:
        xg, itg, capg = h.congrad(Phi, chi, Phi, res)
    finally:
        h.close()
    assert not capo and not capg
    assert np.abs(xg - xo).max() <= 1e-5 * np.abs(xo).max()

    def true_res(x):
        A = po.dslash(lat, po.dslash(lat, x.astype(complex), chi.astype(float), imass=imass),
                      chi.astype(float), imass=imass, dag=True)
        return np.linalg.norm(Phi.astype(complex) - A) / np.linalg.norm(Phi)

    assert true_res(xg) <= 1.5 * true_res(xo)
    assert abs(itg - ito) <= max(3, 0.1 * ito), (itg, ito)


@pytest.mark.parametrize("imass", [1, 3])
def test_hmc_sweeps_against_oracle(imass):
    L, Lt, Ls, dt, iterl = 4, 4, 4, 0.1, 5
    kv = L * L * Lt
    chi = (np.random.default_rng(2).standard_normal((3, kv)) / np.sqrt(0.475)).astype(np.float32)
    sw = po.HmcSweeper(L, Lt, Ls, 0.475, 1.0, dt, 0.01, imass, iterl, chi=chi, seed=SEED,
                       iprint=2)
    h = chb.Hmc(L, Lt, Ls, dt, 0.475, 1.0, 0.01, imass, iterl)
    h.set_chi(chi)
    h.startup(SEED)
    h.set_measure(2)
    compared = 0
    try:
        for k in range(3):
            ro, rg = sw.sweep(), h.sweep()
            tol = 1e-5 * abs(ro.H0)
            for f in ("H0", "S0", "H1", "S1"):
                assert abs(getattr(rg, f) - getattr(ro, f)) <= tol, (f, getattr(rg, f),
                                                                      getattr(ro, f))
            assert abs(rg.dH - ro.dH) <= tol, (rg.dH, ro.dH)
            assert rg.nsteps == ro.nsteps and rg.nforce == ro.nforce
            assert rg.measured == ro.measured
            compared += 1
            if abs(ro.dH) <= 2 * tol:
                break                      # whether x is drawn is within the envelope
            assert rg.drew_x == ro.drew_x
            if ro.drew_x:
                assert rg.x == ro.x
                if abs(ro.x - ro.y) <= 2 * tol * abs(ro.y):
                    break                  # the acceptance is within the envelope
            assert rg.accepted == ro.accepted
            assert h.seed() == sw.seed()
            assert abs(rg.vel2 - ro.vel2) <= 1e-4 * abs(ro.vel2)
            if ro.measured:
                assert np.allclose(np.array(rg.cond[:]), np.array(ro.cond[:]), rtol=0,
                                   atol=1e-5 * max(1.0, np.abs(chi).max()))
            chi_g, chi_o = h.get_chi(), sw.chi.reshape(3, -1)
            assert np.abs(chi_g - chi_o).max() <= 1e-4 * np.abs(chi_o).max()
    finally:
        h.close()
        sw.close()
    assert compared >= 1
