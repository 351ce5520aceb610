/*
 * chdwf_program.h -- host driver of libchdwf: the main loop of program dwf3d
 * (rhmc/cheisdwf.f:1-466) in C, over the resident C ABI of chdwf.h.
 *
 * It is the host side a user runs in place of the Fortran program when no
 * Fortran compiler is at hand, and the reference for how a Fortran driver
 * calls the resident ABI: the random numbers (the reference's RRANF + rano
 * generator) and the control flow stay on the host; every field operation
 * runs on the GPU.
 */
#ifndef CHDWF_PROGRAM_H
#define CHDWF_PROGRAM_H

#include "chdwf.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct chdwf_prog chdwf_prog;

/* What one sweep of the main loop produced (the values the reference
 * writes to 'control', fort.11-14 and the averages in 'output'). */
typedef struct {
    double H0, H1, dH, dS, S0, S1, hg, hp;
    float y, x;                      /* exp(dH) and the Metropolis draw (REAL*4) */
    int accepted, nsteps;
    int it_pf, it_h0, it_h1;         /* solver iterations: heatbath, H0, H1 */
    double it_guid, it_force;        /* summed over the force calls */
    int nforce;
    float action, gaction, paction, vel2;
    int measured;
    float cond[3], susc[3], condmod, susctot;
    float ancgm;                     /* fermion(): average CG iterations */
} chdwf_sweep_record;

/* Create a driver for ksize^2 x ksizet x kthird with the midout parameters
 * (rhmc/cheisdwf.f:117: dt beta am3 am hpin imass iterl).  chi starts at
 * 0.1/beta and the generator at the reference's default seed, as sread does
 * without a 'con' file (:1467-1468). */
int chdwf_prog_create(chdwf_prog** p, int ksize, int ksizet, int kthird, float dt, float beta,
                      float am3, float am, float hpin, int imass, int iterl, int device);
void chdwf_prog_destroy(chdwf_prog* p);
chdwf_ctx* chdwf_prog_context(chdwf_prog* p);
int chdwf_prog_set_remez(chdwf_prog* p, int which, const double* anum, const double* aden,
                         const double* bnum, const double* bden, int ndiag);
int chdwf_prog_set_chi(chdwf_prog* p, const double* chi);
int chdwf_prog_get_chi(chdwf_prog* p, double* chi);
/* rranset(seed); idum=-1; rano(yran) (rhmc/cheisdwf.f:125-130) */
int chdwf_prog_startup(chdwf_prog* p, double seed);
/* rranget (rhmc/cheisdwf.f:1755) as of the end of the last completed sweep */
double chdwf_prog_seed(chdwf_prog* p);
/* Full generator state (LCG, shuffle table, yran, yrun) and sweep counter as
 * an opaque blob of chdwf_prog_state_size() bytes.  The reference's 'con'
 * keeps only the LCG seed, so its resumed runs re-shuffle (rhmc/cheisdwf.f:
 * 129-130); restoring this blob (with chi) resumes the Markov chain exactly. */
int chdwf_prog_state_size(void);
int chdwf_prog_get_state(chdwf_prog* p, void* buf, int nbytes);
int chdwf_prog_set_state(chdwf_prog* p, const void* buf, int nbytes);
/* measurement every iprint sweeps (default 5); measure=0 disables it */
int chdwf_prog_set_measure(chdwf_prog* p, int iprint, int measure);
/* stopping residuals rescga, rescgg, rescgm (default 1e-9, 1e-6, 1e-9, :32-33) */
int chdwf_prog_set_residuals(chdwf_prog* p, float rescga, float rescgg, float rescgm);
/* one sweep (rhmc/cheisdwf.f:207-399) */
int chdwf_prog_sweep(chdwf_prog* p, chdwf_sweep_record* rec);
/* Draw the random inputs (heatbath Gaussians, momenta, trajectory-end and
 * Metropolis draws) of the next ntraj sweeps now and place the field-sized
 * ones in HBM; those sweeps then start with every input resident.  The
 * random stream is the same as without staging. */
int chdwf_prog_stage(chdwf_prog* p, int ntraj);
/* correlators of the last measurement: cferm1(0:Lt-1,2) then cferm2, each a
 * complex64 (re, im) pair at [it + Lt*flavour] (written by the reference to
 * fort.5001/5002 and 5011/5012, :1036-1047) */
int chdwf_prog_correlators(chdwf_prog* p, float* cferm);
const char* chdwf_prog_last_error(chdwf_prog* p);

#ifdef __cplusplus
}
#endif
#endif
