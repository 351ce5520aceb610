/*
 * chdwf.h -- C ABI of libchdwf: the RHMC fermion hot path of the 2+1D chiral
 * Heisenberg domain-wall code (j-ostmeyer/chiralHeisenberg, rhmc/cheisdwf.f)
 * on NVIDIA B200 (sm_100a).
 *
 * Two levels:
 *  1. Routine level: one entry point per reference subroutine on the path,
 *     same arguments, same meaning, host arrays in the reference layout and
 *     types.  The reference's subroutines take implicit-interface, by-reference
 *     arguments and read/write COMMON blocks; here the COMMON inputs
 *     (/para/ beta, am3, ibound) are set once per context
 *     (chdwf_set_para) and the COMMON outputs (/vector/ x, /sforce/ dSdchi)
 *     are explicit output arrays.  Each call copies its inputs to HBM and its
 *     outputs back.
 *  2. Resident level (chdwf_traj_*): the blocks of the trajectory that call
 *     those subroutines (heatbath, hamilton, force, leapfrog updates,
 *     Metropolis bookkeeping) with every field kept in HBM; only REAL*4
 *     momenta/forces or scalars cross when the caller asks for them.
 *
 * Layouts (reference, Fortran column-major, shown 0-based):
 *   spinor   complex*16 R(kthird, ksize, ksize, ksizet, 4, 2): s fastest.
 *            Passed as double* pointing at (re, im) pairs.
 *   chi      real*8 chi(ksize*ksize*ksizet, 3)
 *   pp, dSdchi  REAL*4 (kvol, 3)
 *
 * Every function returns a status: CHDWF_OK, CHDWF_ITER_CAP (solver hit its
 * iteration cap: the reference's qmrherm stops silently at 5000, congrad
 * prints "# iterations of congrad exceeds niterc"), CHDWF_NONFINITE,
 * CHDWF_CUDA_ERROR, CHDWF_BAD_ARG, CHDWF_NOT_FOUND (a file the host driver
 * reads is missing).  chdwf_last_error() describes the last
 * failure of a context.  A context is single-threaded: one CUDA stream,
 * calls must not overlap.
 */
#ifndef CHDWF_H
#define CHDWF_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CHDWF_OK 0
#define CHDWF_ITER_CAP 1
#define CHDWF_NONFINITE 2
#define CHDWF_CUDA_ERROR 3
#define CHDWF_BAD_ARG 4
#define CHDWF_NOT_FOUND 5

typedef struct chdwf_ctx chdwf_ctx;

/* ---- context ------------------------------------------------------------ */
/* Lattice sizes are the reference's compile-time parameters ksize, ksizet,
 * kthird (rhmc/cheisdwf.f:31).  device: CUDA ordinal. */
int chdwf_create(chdwf_ctx** ctx, int ksize, int ksizet, int kthird, int device);
void chdwf_destroy(chdwf_ctx* ctx);
/* /para/ beta, am3, ibound (rhmc/cheisdwf.f:40, :85) */
int chdwf_set_para(chdwf_ctx* ctx, float beta, float am3, int ibound);
const char* chdwf_last_error(const chdwf_ctx* ctx);
/* version string of the library build */
const char* chdwf_version(void);
/* CUDA-event timing of the multi-shift solver's kernels (no reference
 * counterpart; instrumentation).  enable=1 turns it on (every solver launch
 * is then bracketed by events and issued one by one) and resets the totals.
 * chdwf_timing_read fills, per kernel class (0: pass-1 M, 1: pass-1
 * M^dagger + update, 2: pass-2 accumulation from the stored basis, 3: pass-2
 * regeneration; 4-7: the same classes with FP32 Krylov vectors), the summed
 * milliseconds, the number of timed launches, the number of launches and
 * the algorithmic bytes of the timed launches (arrays of 8).  enable=2
 * instead keeps the multi-shift pass 1 on its CUDA-graph replays (as in an
 * untimed solve) and brackets each replayed chunk of 16 iterations with
 * events; chdwf_timing_read_chunks then gives, per Krylov-vector precision
 * (0: FP64, 1: FP32), the microseconds per pass-1 iteration (M, the scalar
 * step and M^dagger) over the chunks that ended at or before their solve's
 * last iteration, and the number of iterations timed (arrays of 2). */
int chdwf_timing(chdwf_ctx* ctx, int enable);
int chdwf_timing_read_chunks(chdwf_ctx* ctx, double* us_per_iter, long long* iters);
/* Precision of the Krylov vectors in the resident trajectory solves (no
 * reference counterpart: the reference is FP64 throughout).  md: the two
 * multi-shift solves of every force evaluation; accept: the heatbath and
 * hamilton solves that enter the Metropolis test.  CHDWF_PREC_F64 (default,
 * the drop-in) or CHDWF_PREC_F32 (FP32 vectors and stencil, FP64
 * reductions, recurrences and solution accumulation). */
#define CHDWF_PREC_F64 0
#define CHDWF_PREC_F32 1
int chdwf_set_precision(chdwf_ctx* ctx, int md, int accept);
/* HBM for the stored Lanczos basis of the multi-shift solver, per vector
 * precision (no reference counterpart).  A solve whose iterations fit keeps
 * every Lanczos vector and forms its solution in one pass over them; longer
 * solves regenerate the vectors instead (same results, twice the operator
 * applications).  max_bytes: the FP64 store; the FP32 store keeps as many
 * vectors in half the bytes.  max_bytes < 0: 40% of the free HBM at the
 * first solve of each precision (default); 0: no store. */
int chdwf_set_basis_store(chdwf_ctx* ctx, double max_bytes);
/* the context's CUDA stream (a cudaStream_t), for callers that time or order
 * their own work against the library's */
void* chdwf_get_stream(chdwf_ctx* ctx);
/* number of CUDA kernels the library has launched in this process */
long long chdwf_kernel_launches(void);
/* operator and multi-shift pass-1 stencil launches in this process by kernel
 * shape: counts[0] point-gather at 3 blocks a SM, counts[1] row-staged,
 * counts[2] point-gather at 4 blocks a SM (the shapes chdwf_autotune_report
 * names).  No counterpart in the reference. */
int chdwf_stencil_launches(long long* counts);
int chdwf_timing_read(chdwf_ctx* ctx, double* ms, long long* timed, long long* launched,
                      double* bytes);

/* ---- routine level (host arrays) -------------------------------------- */
/* Phi = M R.  Replaces dslash(Phi,R,chi,am,hpin,imass), rhmc/cheisdwf.f:2634.
 * am is accepted and unused, as in the reference (":26 not currently
 * implemented"). */
int chdwf_dslash(chdwf_ctx* ctx, double* Phi, const double* R, const double* chi, float am,
                 float hpin, int imass);
/* Phi = M^dagger R.  Replaces dslashd(...), rhmc/cheisdwf.f:3071. */
int chdwf_dslashd(chdwf_ctx* ctx, double* Phi, const double* R, const double* chi, float am,
                  float hpin, int imass);
/* Multi-shift solve over ndiag poles.  Replaces
 * qmrherm(Phi,res,itercg,am,hpin,imass,anum,aden,ndiag,iflag),
 * rhmc/cheisdwf.f:599.  anum[0..ndiag], aden[0..ndiag-1].  x receives
 * /vector/x: iflag 0: a0*Phi + sum_k a_k (M^dagger M + aden_k)^-1 Phi;
 * iflag 1: a0*Phi, and the force of every pole is added to dSdchi (in/out,
 * the /sforce/ block) exactly as the reference's derivs calls do.
 * chi is the /trial/ field the operator reads. */
int chdwf_qmrherm(chdwf_ctx* ctx, const double* Phi, float res, int* itercg, float am,
                  float hpin, int imass, const double* anum, const double* aden, int ndiag,
                  int iflag, const double* chi, double* x, float* dSdchi);
/* dSdchi += force term of one pole.  Replaces derivs(R,X2,anum,imass),
 * rhmc/cheisdwf.f:747. */
int chdwf_derivs(chdwf_ctx* ctx, const double* R, const double* X2, double anum, int imass,
                 float* dSdchi);
/* CGNE on M^dagger M with x as initial guess (in/out, the /vector/ block).
 * Replaces congrad(Phi,res,itercg,am,hpin,imass), rhmc/cheisdwf.f:1064. */
int chdwf_congrad(chdwf_ctx* ctx, const double* Phi, float res, int* itercg, float am,
                  float hpin, int imass, const double* chi, double* x);
/* dSdchi = 2 beta chi + fermion force via two solves over the guidance set
 * (b then a coefficients).  Replaces force(Phi,res1,am,hpin,imass),
 * rhmc/cheisdwf.f:470, with the remez2g common block passed explicitly. */
int chdwf_force(chdwf_ctx* ctx, const double* Phi, float res1, float am, float hpin, int imass,
                const double* chi, const double* anum, const double* aden, const double* bnum,
                const double* bden, int ndiag, float* dSdchi, double* x, int* itg, int* itf);
/* h = hg + hp + hf, s = hg + hf.  Replaces
 * hamilton(Phi,h,hg,hp,s,res2,isweep,am,hpin,imass), rhmc/cheisdwf.f:522,
 * with /trial/ (chi, pp) and the remez2 b-coefficients passed explicitly.
 * out[0..4] = h, hg, hp, s, hf. */
int chdwf_hamilton(chdwf_ctx* ctx, const double* Phi, float res2, float am, float hpin, int imass,
                   const double* chi, const float* pp, const double* bnum, const double* bden,
                   int ndiag, double* out, double* x, int* itercg);

/* ---- device-pointer variants (arrays already in HBM, same layouts) ------ */
/* stream: a cudaStream_t or NULL for the context's own stream. */
int chdwf_dslash_dev(chdwf_ctx* ctx, void* Phi, const void* R, const void* chi, float hpin,
                     int imass, int dagger, void* stream);
/* The operator on reduced-precision storage (no reference counterpart; the
 * reference is FP64): prec = CHDWF_PREC_F32 (complex64 spinors) or
 * CHDWF_PREC_F16 (two IEEE halves per complex); arithmetic in FP32. */
#define CHDWF_PREC_F16 2
int chdwf_dslash_dev_lp(chdwf_ctx* ctx, void* Phi, const void* R, const void* chi, float hpin,
                        int imass, int dagger, int prec, void* stream);
int chdwf_qmrherm_dev(chdwf_ctx* ctx, const void* Phi, float res, int* itercg, float hpin,
                      int imass, const double* anum, const double* aden, int ndiag, int iflag,
                      const void* chi, void* x, void* dSdchi);
int chdwf_congrad_dev(chdwf_ctx* ctx, const void* Phi, float res, int* itercg, float hpin,
                      int imass, const void* chi, void* x);
/* congrad that allocates nothing (no counterpart in the reference).  For
 * callers that cannot allocate device memory -- e.g. a host program whose GPU
 * memory belongs to another runtime's pool or is reserved in full up front,
 * or a code path where allocating is not allowed -- and so cannot create a
 * context either.  Same solve as chdwf_congrad_dev; every argument is
 * explicit and Phi, x (initial guess in, solution out) and chi (real*8
 * (kvol,3)) are device pointers on the current device; stream may be NULL.
 * Scratch lives in one static device array of the library, sized for
 * 8*ksize^2*ksizet*kthird <= 262144 (about 13 MB, held by every GPU that
 * loads the library until the process exits); larger lattices return
 * CHDWF_BAD_ARG.  The first call on a device looks up the array's device
 * address (make it before any stream capture).  All calls share the array:
 * calls whose GPU work overlaps race.  Returns the CHDWF_* statuses. */
int chdwf_congrad_static(const void* Phi, void* x, const void* chi, int ksize, int ksizet,
                         int kthird, float am3, int ibound, float res, float hpin, int imass,
                         int* itercg, void* stream);

/* ---- batched propagator solves ------------------------------------------
 * fermion() (rhmc/cheisdwf.f:897-1058) runs congrad once per source.  This
 * solves nsys independent CGNE systems M^dag M x = Phi in one set of
 * launches per CG stage; every system has its own lattice size, chi, imass,
 * hpin, am3, ibound, REAL*4 scalars and stopping test (congrad's rule with
 * residual res).  Pointers are device memory; x is the initial guess on
 * input.  itercg[i], status[i] per system; the return value is the worst
 * status. */
typedef struct {
    int ksize, ksizet, kthird;
    int imass;
    float hpin, am3;
    int ibound;
    const void* Phi;   /* complex128, reference layout */
    void* x;           /* complex128, in: initial guess, out: solution */
    const void* chi;   /* real*8 chi(kvol,3) */
} chdwf_cg_system;
int chdwf_congrad_batch(chdwf_ctx* ctx, const chdwf_cg_system* sys, int nsys, float res,
                        int* itercg, int* status);

/* ---- resident trajectory level ------------------------------------------
 * The blocks of the main loop of program dwf3d (rhmc/cheisdwf.f:207-399)
 * that call the routines above, with chi, chit, pp, dSdchi and Phi resident
 * in HBM.  The caller keeps the control flow and the random numbers. */
/* Remez set: which = 2 (remez2, hamilton), 4 (remez4, heatbath),
 * 22 (remez2g, force); the common blocks /remez2/, /remez4/, /remez2g/
 * filled at rhmc/cheisdwf.f:140-159. */
int chdwf_traj_set_remez(chdwf_ctx* ctx, int which, const double* anum, const double* aden,
                         const double* bnum, const double* bden, int ndiag);
/* /chi/ chi(kvol,3) in and out; trial=1 reads /trial/ chit instead. */
int chdwf_traj_set_chi(chdwf_ctx* ctx, const double* chi);
int chdwf_traj_get_chi(chdwf_ctx* ctx, double* chi, int trial);
/* chit = chi (rhmc/cheisdwf.f:213-216) */
int chdwf_traj_begin(chdwf_ctx* ctx);
/* Pseudofermion heatbath (rhmc/cheisdwf.f:218-245): ps holds the outputs of
 * the 2*4*kthird gauss0 calls in call order (flavour, Dirac, s; s fastest),
 * each ps(kvol,2) REAL*4; R = cmplx(ps(:,1), ps(:,2)); Phi = (M^dag M)^(1/4) R
 * with the remez4 a-coefficients, kept resident. */
int chdwf_traj_heatbath(chdwf_ctx* ctx, const float* ps, float res, float am, float hpin,
                        int imass, int* itercg);
int chdwf_traj_heatbath_dev(chdwf_ctx* ctx, const void* ps_dev, float res, float am, float hpin,
                            int imass, int* itercg);
/* /trial/ pp(kvol,3) REAL*4 in and out */
int chdwf_traj_set_momenta(chdwf_ctx* ctx, const float* pp);
int chdwf_traj_set_momenta_dev(chdwf_ctx* ctx, const void* pp_dev);
int chdwf_traj_get_momenta(chdwf_ctx* ctx, float* pp);
/* hamilton on the resident fields (rhmc/cheisdwf.f:522-589):
 * out[0..4] = h, hg, hp, s, hf */
int chdwf_traj_hamilton(chdwf_ctx* ctx, float res2, float am, float hpin, int imass, double* out,
                        int* itercg);
/* force on the resident fields (rhmc/cheisdwf.f:470-518) into a resident
 * dSdchi; chdwf_traj_get_force copies it out. */
int chdwf_traj_force(chdwf_ctx* ctx, float res1, float am, float hpin, int imass, int* itg,
                     int* itf);
int chdwf_traj_get_force(chdwf_ctx* ctx, float* dSdchi);
int chdwf_traj_get_phi(chdwf_ctx* ctx, double* Phi);
/* pp = pp - dSdchi*d (REAL*4; rhmc/cheisdwf.f:273-277, :300-311) */
int chdwf_traj_update_momenta(chdwf_ctx* ctx, float d);
/* chit = chit + d*pp (rhmc/cheisdwf.f:285-289) */
int chdwf_traj_update_chi(chdwf_ctx* ctx, float d);
/* chi = chit (rhmc/cheisdwf.f:337-341) */
int chdwf_traj_accept(chdwf_ctx* ctx);
int chdwf_traj_sync(chdwf_ctx* ctx);
/* One wall-source propagator of fermion() (rhmc/cheisdwf.f:937-1012):
 * source 1/ksize^2 on timeslice ittt (1-based), s=1, Dirac idsource,
 * flavour 1; Phi = M^dag xi; CGNE from x0 = Phi.  walls receives the
 * solution on s=1 Dirac 1,2 and s=kthird Dirac 3,4, both flavours, as
 * complex128 [(w*2 + dd)*2 + f][kvol] (w=0: s=1, dd: Dirac pair index). */
int chdwf_traj_propagator(chdwf_ctx* ctx, int ittt, int idsource, float res, float am, float hpin,
                          int imass, double* walls, int* itercg);
/* nsrc wall-source propagators of fermion() in one batched solve (the
 * reference runs them one after the other, rhmc/cheisdwf.f:937-1012): source
 * i on timeslice ittt[i], Dirac idsource[i], as chdwf_traj_propagator; all
 * share chit, so chdwf_congrad_batch runs them as multi-right-hand-side
 * groups.  Each solve's arithmetic is that of chdwf_traj_propagator.  walls
 * receives nsrc blocks of 8*kvol complex128 in chdwf_traj_propagator's
 * layout, itercg[i] the iterations of source i. */
int chdwf_traj_propagators(chdwf_ctx* ctx, int nsrc, const int* ittt, const int* idsource,
                           float res, float am, float hpin, int imass, double* walls,
                           int* itercg);
/* One noise-source solve of measure() (rhmc/cheisdwf.f:1192-1403; the
 * reference routine replaced is the body of its idsource loop):
 * source cmplx(eta(i,1), eta(i,2)) (eta: REAL*4 (kvol,2), as gauss0 fills
 * ps and pt) on wall s=swall (1 or kthird), Dirac idirac, both flavours;
 * Phi = M^dag xi; CGNE from x0 = Phi on the current chit.  slice receives
 * the solution on the opposite wall (s=kthird for swall=1, s=1 for
 * swall=kthird), Dirac idirac, both flavours, as complex128 [f][kvol].
 * imass 1 or 3. */
int chdwf_traj_noise_solve(chdwf_ctx* ctx, const float* eta, int swall, int idirac, float res,
                           float am, float hpin, int imass, double* slice, int* itercg);

/* The stencil autotuner's choices so far in this process (no reference
 * counterpart): a JSON array with one entry per (lattice, element size) of
 * the median microseconds of the operator in each kernel shape (the
 * point-gather kernels at 3 or 4 blocks a SM, the row-staged kernels; 0 when
 * a shape does not apply) and the shape chosen.  Writes at most cap bytes
 * (NUL-terminated) and returns the length the full text needs, including
 * the NUL. */
int chdwf_autotune_report(char* buf, int cap);

/* ---- per-shift multi-shift solutions --------------------------------------
 * x_k = (M^dag M + sigma_k)^-1 Phi for k = 0..n-1 (n <= 32), each into the
 * device buffer x[k] (complex128, reference layout), with its true relative
 * residual |Phi - (M^dag M + sigma_k) x_k| / |Phi| computed in FP64 into
 * true_res[k].  The reference's qmrherm keeps these x_k only internally
 * (rhmc/cheisdwf.f:614, :689-695) and its testinv (:854-890) checks the same
 * per-pole residuals.  prec = CHDWF_PREC_F64: the FP64 multi-shift solve
 * (the reference's stopping rule at res).  CHDWF_PREC_F32: the multi-shift
 * solve with FP32 Krylov vectors to max(res, 1e-6), the x_k accumulated in
 * FP64, then per shift FP64 defect correction (FP32 CG on the FP64 true
 * residual, added in FP64) until the true residual is below res.
 * iters: multi-shift iterations; refine_iters: inner CG iterations summed.
 * Phi, chi (real*8 (kvol,3)) are device pointers; the stored Lanczos basis
 * must hold the solve (chdwf_set_basis_store).  Allocates its work space. */
int chdwf_multishift_dev(chdwf_ctx* ctx, const void* Phi, float res, const void* chi, float hpin,
                         int imass, int n, const double* sigma, void* const* x, double* true_res,
                         int prec, int* iters, int* refine_iters);

/* ---- multi-pseudofermion variant (no reference counterpart) ---------------
 * The reference samples det(M^dag M)^(1/2) with one pseudofermion
 * (rhmc/cheisdwf.f:218-345).  These blocks split it over npf fields, each
 * carrying det(M^dag M)^(1/(2 npf)): heatbath Phi_i = r_hb(M^dag M) R_i with
 * r_hb ~ x^(1/(4 npf)); action Re Phi_i^dag r_act(M^dag M) Phi_i with
 * r_act ~ x^(-1/(2 npf)); force from one multi-shift solve over r_act's poles
 * (the per-pole derivs term of rhmc/cheisdwf.f:729-742).  Rational sets in
 * the reference's partial-fraction form: num[0..n] = a0, a_k; den = sigma_k. */
/* which = 0: r_hb, 1: r_act */
int chdwf_ext_set_remez(chdwf_ctx* ctx, int which, const double* num, const double* den, int n);
/* make field k (0..3) the one the resident blocks act on (field 0 is the
 * reference's Phi) */
int chdwf_ext_select_pf(chdwf_ctx* ctx, int k);
/* Phi_k = r_hb(M^dag M) R, R from 2*4*kthird gauss0 outputs on the device
 * (the layout of chdwf_traj_heatbath's ps), on chit */
int chdwf_ext_heatbath_dev(chdwf_ctx* ctx, const void* ps_dev, float res, float hpin, int imass,
                           int* itercg);
/* hf = Re Phi_k^dag r_act(M^dag M) Phi_k on chit */
int chdwf_ext_action(chdwf_ctx* ctx, float res, float hpin, int imass, double* hf, int* itercg);
/* init = 1: dSdchi = 2 beta chit first (rhmc/cheisdwf.f:494-498); then
 * dSdchi += d/dchi (Phi_k^dag r_act(M^dag M) Phi_k), REAL*4, resident */
int chdwf_ext_force(chdwf_ctx* ctx, float res, float hpin, int imass, int init, int* itercg);
/* hp_hg[0] = 0.5 sum pp^2, hp_hg[1] = beta sum chit^2 (rhmc/cheisdwf.f:546-559) */
int chdwf_ext_bosonic(chdwf_ctx* ctx, double* hp_hg);

#ifdef __cplusplus
}
#endif
#endif
