/*
 * chdwf_thirring.h -- C ABI of the bulk Thirring RHMC, bulk_rhmc.f
 * (j-ostmeyer/chiralHeisenberg), on the GPU.
 *
 * bulk_rhmc.f simulates the Thirring model with domain-wall fermions: one
 * flavour of 4-component spinors R(kthird,kvol,4) (complex*16), link angles
 * theta(kvol,3) (REAL*4) entering the hops as u = 1 + i*theta (the
 * antiperiodic sign folded into the last time slice), a wall mass term am
 * (imass 1, 3 or 5), and a Pauli-Villars determinant at mass 1.  The entry
 * points replace its routines with their argument meaning:
 *
 *   chdwf_thr_coef             coef               (bulk_rhmc.f:1799-1827)
 *   chdwf_thr_dslash / _dslashd dslash, dslashd   (:1946-2069, :2071-2188)
 *   chdwf_thr_derivs           derivs             (:820-878)
 *   chdwf_thr_qmrherm          qmrherm, iflag 0-3 with the Phi0 register (:630-818)
 *   chdwf_thr_congrad, _measure congrad, measure  (:931-1025, :1027-1285)
 *   chdwf_thr_sweep            one pass of the main loop (:201-400)
 *
 * Layouts are the reference's: spinors R(kthird,kvol,4) complex128, s
 * fastest; links u(kvol,3) complex128; theta, pp, dSdpi (kvol,3) REAL*4;
 * Phi0(kferm,ndiag) complex128.  The operator and derivs agree bit for bit
 * with a sequential evaluation.  The solver keeps the reference's scalar
 * types (alphatild, beta0, phimod, rhomax REAL*4; the shifted recurrences
 * REAL*8); its sums are formed in FP64 and rounded once.  Return values
 * are the CHDWF_* codes of chdwf.h.
 */
#ifndef CHDWF_THIRRING_H
#define CHDWF_THIRRING_H

#include "chdwf.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct chdwf_thr chdwf_thr;

/* One trajectory.  it_pf/it_pfpv: the two heatbath solves (:226, :236);
 * it_h0/it_h0pv and it_h1/it_h1pv: the mass-m and Pauli-Villars solves of
 * the two hamilton calls; it_force[4] summed over the nforce force calls:
 * PV (iflag 1), mass m (iflag 0), the DWF force (iflag 2), the PV force
 * (iflag 3) (:493-514).  drew_x: dH < 0, so x was drawn (:333-336). */
typedef struct {
    double H0, H1, dH, dS, S0, S1, hg, hp;
    float y, x;
    int drew_x, accepted, nsteps;
    int it_pf, it_pfpv, it_h0, it_h0pv, it_h1, it_h1pv;
    int it_force[4];
    int nforce;
    float action, gaction, paction, vel2;
    int measured;          /* isweep a multiple of iprint: measure ran */
    float pbp, ancgm;      /* its psibarpsi and aviter (:367-370) */
} chdwf_thr_record;

/* Lattice and 'midout' parameters (dt, beta, am3, am, imass, iterl;
 * bulk_rhmc.f:104).  ibound = -1; residuals rescga = 1e-9, rescgg = 1e-6
 * (:39).  imass 1, 3 or 5. */
int chdwf_thr_create(chdwf_thr** out, int ksize, int ksizet, int kthird, float dt, float beta,
                     float am3, float am, int imass, int iterl, int device);
void chdwf_thr_destroy(chdwf_thr* h);
const char* chdwf_thr_last_error(chdwf_thr* h);
/* The rational sets read from remez2, remez4 (which 2, 4) and remez2g,
 * remez4g (which 22, 44): a0 = anum[0], (anum[k], aden[k-1]) k = 1..ndiag,
 * likewise bnum/bden (:123-146).  ndiag <= 25. */
int chdwf_thr_set_remez(chdwf_thr* h, int which, const double* anum, const double* aden,
                        const double* bnum, const double* bden, int ndiag);

/* coef: u from theta (host arrays). */
int chdwf_thr_coef(chdwf_thr* h, const float* theta, double* u);
/* Phi = M R, Phi = M^dagger R with links u and mass (am, imass). */
int chdwf_thr_dslash(chdwf_thr* h, double* Phi, const double* R, const double* u, float am,
                     int imass);
int chdwf_thr_dslashd(chdwf_thr* h, double* Phi, const double* R, const double* u, float am,
                      int imass);
/* derivs: adds to dSdpi (in/out, REAL*4 (kvol,3)) 2*anum times
 * Re(R^dag dM^dag/dtheta X2) (iflag 0) or Re(R^dag dM/dtheta X2) (iflag 1),
 * with the t links of the last time slice taken without their antiperiodic
 * sign (force applies it, :520-525); summed term by term in REAL*4 as the
 * reference does. */
int chdwf_thr_derivs(chdwf_thr* h, const double* R, const double* X2, double anum, int iflag,
                     float* dSdpi);
/* qmrherm: iflag 0 x = anum0 Phi + sum_k anum_k (M^dag M + aden_k)^-1 Phi;
 * 1 also Phi0 (out); 2 adds the DWF force of the poles to dSdpi (in/out);
 * 3 adds the Pauli-Villars force from Phi0 (in).  CHDWF_ITER_CAP when
 * 7500 iterations did not converge (the reference then goes on). */
int chdwf_thr_qmrherm(chdwf_thr* h, const double* Phi, float res, int* itercg, float am,
                      int imass, const double* anum, const double* aden, int ndiag, int iflag,
                      const double* u, double* x, double* Phi0, float* dSdpi);

/* congrad (:931-1025): x (in: initial guess, out: solution) of
 * M^dagger M x = Phi at mass (am, imass); CHDWF_ITER_CAP at kthird*kvol. */
int chdwf_thr_congrad(chdwf_thr* h, const double* Phi, float res, int* itercg, float am,
                      int imass, const double* u, double* x);
/* measure (:1027-1285) with links u at the context's am and imass: the noisy
 * psibar psi estimator over 10 noise vectors from the context's generator;
 * parts (40 doubles or NULL) receives re/im of psibarpsi1 and psibarpsi2 per
 * noise (the unit-100 records). */
int chdwf_thr_measure(chdwf_thr* h, float res, const double* u, float* psibarpsi,
                      float* susclsing, float* aviter, double* parts);
/* Measure every iprint-th sweep (default 5, as the reference). */
int chdwf_thr_set_measure(chdwf_thr* h, int iprint);

/* The main loop: theta (REAL*4 (kvol,3)), the generator, one sweep. */
int chdwf_thr_set_theta(chdwf_thr* h, const float* theta);
int chdwf_thr_get_theta(chdwf_thr* h, float* theta);
int chdwf_thr_startup(chdwf_thr* h, double seed);
double chdwf_thr_seed(chdwf_thr* h);
int chdwf_thr_sweep(chdwf_thr* h, chdwf_thr_record* rec);

#ifdef __cplusplus
}
#endif
#endif
