/*
 * chdwf_oracle.h -- CPU oracle for the RHMC fermion path of the 2+1D chiral
 * Heisenberg domain-wall code (j-ostmeyer/chiralHeisenberg, rhmc/cheisdwf.f).
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * Fortran, used as the checker for the CUDA path and as the timed CPU
 * baseline.  Nothing in the product library links, loads or calls it.
 *
 * Parity status: the reference cannot be compiled in this environment (no
 * Fortran compiler), so the numerical routines are "parity unpinned" against
 * the reference binary.  Pinned: the random-number generator against the
 * seed pairs printed in rhmc/Ls_8/<run>/out_1 (196 draws of RRANF at start-up,
 * cheisdwf.f:125-130), and the Remez coefficient files against x^(+-1/4),
 * x^(+-1/2).  Everything else is a line-by-line restatement with the
 * reference's implicit REAL*4 / REAL*8 typing, loop order and
 * single-threaded reduction order (cheisdwf.f compiled without FMA
 * contraction), cited per function in chdwf_oracle.c.
 *
 * Layouts are the reference's Fortran column-major layouts, 0-based:
 *   spinor  R(s, x, y, t, d, f)  -> s + Ls*(site + kvol*(d + 4*f)),
 *           site = x + L*(y + L*t), complex128 as (re, im) pairs;
 *   chi     chi(site, a)         -> site + kvol*a, a = 0..2 (real*8);
 *   pp, dSdchi (site, a)         -> site + kvol*a (REAL*4).
 */
#ifndef CHDWF_ORACLE_H
#define CHDWF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Lattice and /para/ common block (cheisdwf.f:31,40). */
typedef struct {
    int L, Lt, Ls;          /* ksize, ksizet, kthird */
    float beta, am3;        /* /para/ beta, am3 (implicit REAL*4) */
    int ibound;             /* /para/ ibound (-1: antiperiodic in t) */
    int threads;            /* 1: reference single-thread order; >1 OpenMP */
} orc_lat;

/* RNG state: RRANF's DS(2), rano's v(97), the two "last output" variables
 * yran (/ranseed/) and yrun (main-program local), idum (cheisdwf.f:1722-1801). */
typedef struct {
    double ds[2];
    float v[97];
    float yran, yrun;
    int idum;
} orc_rng;

/* Remez sets as read by cheisdwf.f:140-159: a0, (a_k, sigma_k), b0, (b_k, sigma_k). */
typedef struct {
    int n;
    double anum[32], aden[32], bnum[32], bden[32];  /* anum[0], bnum[0] = a0, b0 */
} orc_remez;

int64_t orc_kvol(const orc_lat* lat);
int64_t orc_kferm(const orc_lat* lat);

/* --- random numbers (cheisdwf.f:1678-1801) ------------------------------ */
void   orc_rranset(orc_rng* g, double seed);
double orc_rranget(const orc_rng* g);
float  orc_rranf(orc_rng* g);
float  orc_rano(orc_rng* g, float* y);              /* y: &g->yran or &g->yrun */
void   orc_rng_startup(orc_rng* g, double seed);    /* cheisdwf.f:125-130 */
void   orc_gauss0(orc_rng* g, int64_t kvol, float* ps);  /* ps(kvol,2) */
void   orc_gaussp(orc_rng* g, int64_t kvol, float* ps);

/* --- operator (cheisdwf.f:2634-3501, the live v2 routines) -------------- */
void orc_dslash (const orc_lat* lat, double* Phi, const double* R,
                 const double* chi, float am, float hpin, int imass);
void orc_dslashd(const orc_lat* lat, double* Phi, const double* R,
                 const double* chi, float am, float hpin, int imass);
/* The dead table-driven "v1" M (cheisdwf.f:1804-2217), a second formulation. */
void orc_dslash_v1(const orc_lat* lat, double* Phi, const double* R,
                   const double* chi, float am, float hpin, int imass);

/* --- solvers ------------------------------------------------------------- */
/* qmrherm (cheisdwf.f:599-745).  x: /vector/x output (kferm complex).
 * dSdchi: /sforce/, accumulated into when iflag == 1.
 * niterc: iteration cap (5000 in the reference). */
int orc_qmrherm(const orc_lat* lat, const double* Phi, float res, int* itercg,
                float am, float hpin, int imass, const double* anum,
                const double* aden, int ndiag, int iflag, const double* chi,
                double* x, float* dSdchi, int niterc);
/* derivs (cheisdwf.f:747-849). */
void orc_derivs(const orc_lat* lat, const double* R, const double* X2,
                double anum, int imass, float* dSdchi);
/* congrad (cheisdwf.f:1064-1157). x: in = initial guess, out = solution.
 * Returns 1 when the iteration cap niterc (= kthird*kvol) was hit. */
int orc_congrad(const orc_lat* lat, const double* Phi, float res, int* itercg,
                float am, float hpin, int imass, const double* chi, double* x);

/* force (cheisdwf.f:470-518): dSdchi = 2 beta chi + fermion force; x: /vector/. */
void orc_force(const orc_lat* lat, const double* Phi, float res1, float am,
               float hpin, int imass, const double* chi, const orc_remez* r2g,
               float* dSdchi, double* x, int* itg, int* itf);
/* hamilton (cheisdwf.f:522-589).  out[0..4] = h, hg, hp, s, hf. */
void orc_hamilton(const orc_lat* lat, const double* Phi, float res2, float am,
                  float hpin, int imass, const double* chi, const float* pp,
                  const orc_remez* r2, double* out, double* x, int* itercg);

/* fermion (cheisdwf.f:897-1058): returns aviter; cferm1/cferm2 receive the
 * averaged correlators as complex64 pairs [(it, flavour)] = 2*(it + Lt*f). */
/* measure (cheisdwf.f:1164-1453): the noisy psibar psi estimator; imass 1 or 3. */
void orc_measure(const orc_lat* lat, orc_rng* g, float res, float am, float hpin, int imass,
                 const double* chi, double* xi, float* psibarpsi, float* susclsing,
                 float* aviter, double* parts);
float orc_fermion(const orc_lat* lat, orc_rng* g, float res, float am,
                  float hpin, int imass, const double* chi, double* x,
                  float* cferm1, float* cferm2);

/* --- trajectory (program dwf3d, cheisdwf.f:207-399) --------------------- */
typedef struct {
    double H0, H1, dH, dS, S0, S1, hg, hp;
    float y, x;
    int accepted, nsteps;
    int it_pf, it_h0, it_h1;
    double it_guid, it_force;      /* summed over force calls */
    int nforce;
    float action, gaction, paction, vel2;
    int measured;
    float cond[3], susc[3], condmod, susctot;
    float ancgm;
} orc_traj_rec;

typedef struct {
    orc_lat lat;
    orc_rng rng;
    orc_remez r2, r4, r2g;
    float dt, am, hpin;
    int imass, iterl, iprint, measure;
    float rescga, rescgg, rescgm;
    double* chi;       /* /chi/ chi(kvol,3)  */
    double* chit;      /* /trial/ chit       */
    float* pp;         /* /trial/ pp (REAL*4) */
    float* dSdchi;     /* /sforce/          */
    double* Phi;       /* pseudofermion     */
    double* X1;        /* /vector/          */
    double* R;         /* /dum1/ R          */
    float* ps;         /* /dum1/ ps(kvol,2) */
    float* cferm;      /* 4*Lt*2 floats: cferm1, cferm2 (last measurement) */
    int isweep;
    float gaction;     /* main-program variable, kept across sweeps (:264, :342) */
} orc_state;

orc_state* orc_state_new(int L, int Lt, int Ls, float beta, float am3,
                         float dt, float am, float hpin, int imass, int iterl);
void orc_state_free(orc_state* st);
void orc_state_set_remez(orc_state* st, int which, const orc_remez* r);
/* One sweep of the main loop (cheisdwf.f:207-399). */
void orc_sweep(orc_state* st, orc_traj_rec* rec);

/* --- the HMC predecessor, mh/cheisdwf_hmc.f (chdwf_oracle_hmc.c) --------
 * single precision: spinors complex64 (re, im float pairs), chi REAL*4. */
void orc_hmc_dslash(const orc_lat* lat, float* Phi, const float* R, const float* chi,
                    int imass, int dag);
int orc_hmc_congrad(const orc_lat* lat, const float* Phi, float res, int* itercg, int imass,
                    const float* chi, float* x);
void orc_hmc_derivs(const orc_lat* lat, const float* X1, const float* chi, int imass,
                    float* dSdchi);
int orc_hmc_force(const orc_lat* lat, const float* Phi, float* X0, float* X1, const float* chi,
                  float res1, int imass, float* dSdchi, int* itercg);
int orc_hmc_hamilton(const orc_lat* lat, const float* Phi, float* X0, const float* chi,
                     const float* pp, float res2, int imass, double* out, int* itercg);

typedef struct {
    double H0, H1, dH, dS, S0, S1, hg, hp;
    float y, x;
    int drew_x, accepted, nsteps;
    int it_h0, it_h1, it_force, nforce;
    float action, gaction, paction, vel2;
    int measured;
    float cond[3], susc[3], condmod, susctot;
} orc_hmc_rec;

typedef struct {
    orc_lat lat;
    orc_rng rng;
    float dt, am;
    int imass, iterl, iprint;
    float rescga, rescgg;
    float* chi;        /* /chi/ chi(kvol,3), REAL*4 */
    float* chit;       /* /trial/ chit      */
    float* pp;         /* /trial/ pp        */
    float* dSdchi;
    float* Phi;        /* pseudofermion     */
    float* X0;         /* solver guess, extrapolated by force */
    float* X1;         /* /vector/          */
    float* R;          /* /dum1/ R          */
    float* ps;         /* /dum1/ ps(kvol,2) */
    int isweep, itot, naccp;
    float action, gaction, paction;   /* main-program variables kept across sweeps */
    float actiona, vel2a, yav, yyav;
} orc_hmc_state;

orc_hmc_state* orc_hmc_new(int L, int Lt, int Ls, float beta, float am3, float dt, float am,
                           int imass, int iterl);
void orc_hmc_free(orc_hmc_state* st);
/* One sweep of the main loop of mh/cheisdwf_hmc.f (:140-320). */
void orc_hmc_sweep(orc_hmc_state* st, orc_hmc_rec* rec);

/* --- the bulk Thirring RHMC, bulk_rhmc.f (chdwf_oracle_thirring.c) ------
 * spinors R(s, site, d) complex128 (4 Dirac components, one flavour); link
 * angles theta(kvol,3) REAL*4; links u(kvol,3) complex128. */
void orc_thr_coef(const orc_lat* lat, const float* theta, double* u);
void orc_thr_dslash(const orc_lat* lat, double* Phi, const double* R, const double* u, float am,
                    int imass, int dag);
void orc_thr_derivs(const orc_lat* lat, const double* R, const double* X2, double anum,
                    int iflag, float* dSdpi);
void orc_thr_set_alphatild_fp64(int on);
int orc_thr_qmrherm(const orc_lat* lat, const double* Phi, float res, int* itercg, float am,
                    int imass, const double* anum, const double* aden, int ndiag, int iflag,
                    const double* u, double* x, double* Phi0, float* dSdpi);

typedef struct {
    double H0, H1, dH, dS, S0, S1, hg, hp;
    float y, x;
    int drew_x, accepted, nsteps;
    int it_pf, it_pfpv, it_h0, it_h0pv, it_h1, it_h1pv;
    int it_force[4];   /* summed per force solve: PV (iflag 1), m, DWF force, PV force */
    int nforce;
    float action, gaction, paction, vel2;
    int measured;
    float pbp, ancgm;  /* measure's psibarpsi and aviter (measurement sweeps) */
} orc_thr_rec;

typedef struct {
    orc_lat lat;
    orc_rng rng;
    orc_remez r2, r4, r2g, r4g;
    float dt, am;
    int imass, iterl, iprint;
    float rescga, rescgg;
    float* theta;      /* /gauge/ theta(kvol,3) */
    float* thetat;     /* /trial/ thetat     */
    float* pp;         /* /trial/ pp         */
    float* dSdpi;      /* /gforce/           */
    double* ut;        /* /trial/ ut         */
    double* Phi;       /* pseudofermion      */
    double* X1;        /* /vector/           */
    double* R;         /* /dum1/ R           */
    double* Phi0;      /* /phi0/ Phi0(kferm,25) */
    float* ps;         /* /dum1/ ps(kvol,2)  */
    int isweep, itot, naccp;
    float action, gaction, paction;
    float actiona, vel2a, yav, yyav;
} orc_thr_state;

orc_thr_state* orc_thr_new(int L, int Lt, int Ls, float beta, float am3, float dt, float am,
                           int imass, int iterl);
void orc_thr_free(orc_thr_state* st);
/* which: 2, 4 (remez2, remez4), 22, 44 (remez2g, remez4g) */
void orc_thr_set_remez(orc_thr_state* st, int which, const orc_remez* r);
void orc_thr_force(orc_thr_state* st, float res1, int* its);
void orc_thr_hamilton(orc_thr_state* st, float res2, double* out, int* its);
int orc_thr_congrad(const orc_lat* lat, const double* Phi, float res, int* itercg, float am,
                    int imass, const double* u, double* x);
void orc_thr_measure(const orc_lat* lat, orc_rng* g, float res, float am, int imass,
                     const double* u, float* psibarpsi, float* susclsing, float* aviter,
                     double* parts);
/* One sweep of the main loop of bulk_rhmc.f (:201-400), with measure on
 * every iprint-th sweep. */
void orc_thr_sweep(orc_thr_state* st, orc_thr_rec* rec);

/* Remez file reader (format of rhmc/remez*): returns 0 on success. */
int orc_read_remez(const char* path, int n, orc_remez* r);

#ifdef __cplusplus
}
#endif
#endif
