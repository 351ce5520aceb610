/*
 * chdwf_hmc.h -- C ABI of the HMC predecessor of the RHMC code,
 * mh/cheisdwf_hmc.f (j-ostmeyer/chiralHeisenberg), on the GPU.
 *
 * mh/cheisdwf_hmc.f is the single-precision Hybrid Monte Carlo version of
 * the same model: COMPLEX (complex64) spinors, REAL*4 chi, one CGNE solve
 * (congrad) per force evaluation with an extrapolated initial guess, and the
 * operator of rhmc/cheisdwf.f without the pinning term.  The entry points
 * replace its routines with their argument meaning:
 *
 *   chdwf_hmc_dslash / _dslashd   dslash, dslashd   (mh/cheisdwf_hmc.f:1334, :1683)
 *   chdwf_hmc_congrad             congrad           (:625-716)
 *   chdwf_hmc_derivs              force, after its congrad call (:416-420, :445-555)
 *   chdwf_hmc_sweep               one pass of the main loop (:140-320)
 *
 * Layouts are the reference's: spinors Phi(kthird,ksize,ksize,ksizet,4,2) as
 * complex64 (re, im float pairs), s fastest; chi(kvol,3) and dSdchi(kvol,3)
 * REAL*4.  The arithmetic is the reference's REAL*4 arithmetic without fused
 * multiply-add: the operator and the force agree bit for bit with a
 * sequential evaluation; the solver's two REAL*4 sums are formed in FP64 and
 * rounded once (the reference adds element by element in REAL*4).
 * Return values are the CHDWF_* codes of chdwf.h.
 */
#ifndef CHDWF_HMC_H
#define CHDWF_HMC_H

#include "chdwf.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct chdwf_hmc chdwf_hmc;

/* One trajectory of the main loop.  Iteration counts are congrad's itercg:
 * it_h0/it_h1 of the two hamilton calls (:191, :251), it_force summed over
 * the nforce force calls (ancg, :433).  drew_x: dH < 0, so the Metropolis
 * draw x was taken (:259-263).  action/gaction/paction are the main
 * program's variables after the sweep (kept from the last sweep that set
 * them, :193-197, :271-274); measured, cond, susc, condmod, susctot as
 * written to units 12-14 (:288-315). */
typedef struct {
    double H0, H1, dH, dS, S0, S1, hg, hp;
    float y, x;
    int drew_x, accepted, nsteps;
    int it_h0, it_h1, it_force, nforce;
    float action, gaction, paction, vel2;
    int measured;
    float cond[3], susc[3], condmod, susctot;
} chdwf_hmc_record;

/* Lattice and 'midout' parameters (dt, beta, am3, am, imass, iterl;
 * mh/cheisdwf_hmc.f:78).  ibound = -1, iprint = 5, and the residuals
 * rescga = 1e-9, rescgg = 1e-6 (:35) as in the reference.  imass 1 or 3. */
int chdwf_hmc_create(chdwf_hmc** out, int ksize, int ksizet, int kthird, float dt, float beta,
                     float am3, float am, int imass, int iterl, int device);
void chdwf_hmc_destroy(chdwf_hmc* h);
const char* chdwf_hmc_last_error(chdwf_hmc* h);

/* Phi = M R and Phi = M^dagger R on host arrays (kferm complex64). */
int chdwf_hmc_dslash(chdwf_hmc* h, float* Phi, const float* R, const float* chi, int imass);
int chdwf_hmc_dslashd(chdwf_hmc* h, float* Phi, const float* R, const float* chi, int imass);
/* congrad: x (in: initial guess, out: solution) of M^dagger M x = Phi.
 * CHDWF_ITER_CAP when kthird*kvol iterations did not converge. */
int chdwf_hmc_congrad(chdwf_hmc* h, const float* Phi, float res, int* itercg, int imass,
                      const float* chi, float* x);
/* dSdchi of force for the solution X1: 2*(2*beta*chi - the wall products of
 * X1 with M X1).  beta is the context's. */
int chdwf_hmc_derivs(chdwf_hmc* h, const float* X1, const float* chi, int imass, float* dSdchi);

/* The main loop: chi (REAL*4 (kvol,3)), the generator (the reference's
 * RRANF + rano, started as the reference starts it), the measurement
 * interval, the two residuals, one sweep. */
int chdwf_hmc_set_chi(chdwf_hmc* h, const float* chi);
int chdwf_hmc_get_chi(chdwf_hmc* h, float* chi);
int chdwf_hmc_startup(chdwf_hmc* h, double seed);
double chdwf_hmc_seed(chdwf_hmc* h);
int chdwf_hmc_set_measure(chdwf_hmc* h, int iprint);
int chdwf_hmc_set_residuals(chdwf_hmc* h, float rescga, float rescgg);
int chdwf_hmc_sweep(chdwf_hmc* h, chdwf_hmc_record* rec);

#ifdef __cplusplus
}
#endif
#endif
