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
    int ended;                       /* 1: the trajectory ended by its end-of-trajectory draw,
                                        0: it ran the full itermax = 1000 steps */
} chdwf_sweep_record;

/* Running sums the main program keeps over a run (rhmc/cheisdwf.f:185-203,
 * updated at :235, :264, :305, :326-348, :356, :382-396 and in force and
 * hamilton through COMMON /param/, :507, :515, :575), in REAL*4 as there.
 * gaction persists from the last sweep that set it (sweep 1 or an
 * acceptance), as the reference's variable does. */
typedef struct {
    float actiona, vel2a, condmoda, susca, conda[3], pbpa;
    float ancg, ancgh, ancgf, ancgpf, ancgma, yav, yyav;
    int naccp, ipbp, itot, nsweep;
    float gaction;
} chdwf_run_sums;

/* The averages written at the end of a run (rhmc/cheisdwf.f:413-443). */
typedef struct {
    int iter2, naccp;
    float atraj, yav, yyav, ancg, ancgh, ancgf, ancgpf, ancgma;
    float condmoda, susca, conda[3], pbpa, vel2a, actiona;
} chdwf_run_averages;

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
/* The multi-pseudofermion variant (no reference counterpart; the reference
 * has one pseudofermion and a leapfrog of random length, rhmc/cheisdwf.f:
 * 218-345).  npf > 0 makes every following sweep one trajectory with npf
 * pseudofermion fields (rational sets by chdwf_ext_set_remez on the
 * program's context), nsteps integrator steps of size dt, integrator 1 =
 * Omelyan's second-order minimum-norm scheme with parameter lambda
 * (0.1931833275037836 is its optimum), 0 = leapfrog; the same H0/H1,
 * Metropolis draw and record.  Its random stream: npf blocks of 2*4*kthird
 * gauss0 calls, the momenta, the Metropolis draw.  No measurement.
 * npf = 0 returns to the reference's sweep. */
int chdwf_prog_set_ext(chdwf_prog* p, int npf, int nsteps, int integrator, float lambda);
/* Draw the random inputs (heatbath Gaussians, momenta, trajectory-end and
 * Metropolis draws) of the next ntraj sweeps now and place the field-sized
 * ones in HBM; those sweeps then start with every input resident.  The
 * random stream is the same as without staging. */
int chdwf_prog_stage(chdwf_prog* p, int ntraj);
/* correlators of the last measurement: cferm1(0:Lt-1,2) then cferm2, each a
 * complex64 (re, im) pair at [it + Lt*flavour] (written by the reference to
 * fort.5001/5002 and 5011/5012, :1036-1047) */
int chdwf_prog_correlators(chdwf_prog* p, float* cferm);
/* measure(psibarpsi, res, aviter, am, hpin, imass) (rhmc/cheisdwf.f:1164-1453)
 * on the current chi with the program's am, hpin and imass (1 or 3): the
 * noisy psibar psi estimator over knoise = 10 Gaussian noise vectors drawn
 * from the program's generator (two gauss0 calls per noise), four CGNE
 * solves per noise at residual res.  psibarpsi and susclsing are the
 * values the reference writes to unit 200; aviter = iterations / 40.
 * parts (40 doubles, or NULL) receives re/im of psibarpsi1 and psibarpsi2
 * per noise, the unit-100 records.  The main program of the reference does
 * not call it (:392); this entry point leaves the running sums alone. */
int chdwf_prog_measure(chdwf_prog* p, float res, float* psibarpsi, float* susclsing,
                       float* aviter, double* parts);
const char* chdwf_prog_last_error(chdwf_prog* p);

/* The running sums since creation (or the last reset); they are part of
 * the state blob, so an exact resume continues them. */
int chdwf_prog_sums(chdwf_prog* p, chdwf_run_sums* out);
int chdwf_prog_reset_sums(chdwf_prog* p);
/* Averages over the sweeps summed so far (rhmc/cheisdwf.f:413-431). */
int chdwf_prog_averages(chdwf_prog* p, chdwf_run_averages* out);
/* Number of congrad iteration caps met since the last call (the reference
 * writes one line for each to units 6 and 7, :1151-1153). */
int chdwf_prog_take_cg_caps(chdwf_prog* p);

/* ---- on-disk formats of the reference program ---------------------------
 * 'con' is one Fortran unformatted sequential record (4-byte length markers)
 * holding chi(kvol,3) and seed, written by swrite (rhmc/cheisdwf.f:1480-1489)
 * and read by sread (:1455-1478).  chdwf_con_read accepts a REAL*8 chi and
 * the REAL*4 chi of the older configurations (the conversion
 * rhmc/sp_to_dp.f makes); *single tells which it found.  Returns CHDWF_OK,
 * CHDWF_NOT_FOUND when the file is missing, CHDWF_BAD_ARG when its record
 * does not hold a kvol-site configuration. */
int chdwf_con_read(const char* path, int kvol, double* chi, double* seed, int* single);
int chdwf_con_write(const char* path, int kvol, const double* chi, double seed);
/* sread: chi and seed from 'path', or chi = 0.1/beta and the default seed
 * when the file is missing (:1462-1470).  Sets the driver's chi and returns
 * the seed (not yet applied: chdwf_prog_startup does that, as :127-130). */
int chdwf_prog_read_con(chdwf_prog* p, const char* path, double* seed);
/* swrite with the seed rranget returns after the last completed sweep. */
int chdwf_prog_write_con(chdwf_prog* p, const char* path);

/* One record of list-directed output in gfortran's layout: kinds[i] is 'i'
 * (INTEGER), 'f' (REAL*4) or 'd' (REAL*8) for values[i]; the line (with its
 * newline) goes to out.  Returns its length, or -1 if cap is too small. */
int chdwf_format_list(char* out, int cap, const char* kinds, const double* values);
/* One explicit edit descriptor: kind 'I' (Iw), 'F' (Fw.d) or 'E' (Ew.d). */
int chdwf_format_edit(char* out, int cap, char kind, int w, int d, double value);

/* Runs program dwf3d in directory dir as the reference does in its working
 * directory (rhmc/cheisdwf.f:1-466): reads 'midout' (dt beta am3 am hpin
 * imass iterl iter2), 'con' (sread) and 'remez2', 'remez4', 'remez2g'
 * (ndiag = 25, ndiagg = 12 poles); appends to 'control', fort.11-14 and
 * fort.5001/5011/5002/5012; writes 'output' and checkpoints 'con' every
 * iprint = 5 sweeps and at the end.  ksize, ksizet and kthird are the
 * reference's compile-time lattice parameters. */
int chdwf_run_dir(const char* dir, int ksize, int ksizet, int kthird, int device);

#ifdef __cplusplus
}
#endif
#endif
