/*
 * chdwf_oracle.c -- CPU oracle (test infrastructure, never linked into the
 * product).  A plain-C restatement of the RHMC fermion path of
 * j-ostmeyer/chiralHeisenberg, rhmc/cheisdwf.f; every function cites the
 * lines it follows.  Parity unpinned against a compiled reference (none can
 * be built here); pinned pieces are listed in chdwf_oracle.h.
 *
 * Typing rules reproduced from the Fortran (implicit typing, i-n integer,
 * everything else REAL*4 unless declared):
 *   REAL*4 : pp, dSdchi, beta, am3, dt, hpin, d, y, x, ytest, proby, tpi,
 *            resid, arelax, diag, every scalar of congrad, cond/susc/condmod.
 *   REAL*8 : chi, chit, H0/H1/dH/dS/hg/hp/hf, Remez coefficients, every
 *            scalar recurrence of qmrherm.
 *   cmplx(a, b) without KIND is DEFAULT complex, so chi entering the wall
 *   coupling of the live operator is rounded to REAL*4 (cheisdwf.f:2914,2962).
 * Compiled with -ffp-contract=off: no fused multiply-add anywhere.
 */
#include "chdwf_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double re, im; } cx;

static inline cx ld(const double* p, int64_t j) { cx r = {p[2 * j], p[2 * j + 1]}; return r; }
static inline void st(double* p, int64_t j, cx v) { p[2 * j] = v.re; p[2 * j + 1] = v.im; }
static inline cx cadd(cx a, cx b) { cx r = {a.re + b.re, a.im + b.im}; return r; }
static inline cx csub(cx a, cx b) { cx r = {a.re - b.re, a.im - b.im}; return r; }
static inline cx cmuli(cx a) { cx r = {-a.im, a.re}; return r; }          /* zi*a */
static inline cx cmul(cx a, cx b) {
    cx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}
static inline cx cscal(double s, cx a) { cx r = {s * a.re, s * a.im}; return r; }
static inline cx cconj(cx a) { cx r = {a.re, -a.im}; return r; }

int64_t orc_kvol(const orc_lat* l) { return (int64_t)l->L * l->L * l->Lt; }
int64_t orc_kferm(const orc_lat* l) { return 8 * orc_kvol(l) * l->Ls; }

/* ======================================================================
 * Random numbers: RRANF / G900GT / G900ST (cheisdwf.f:1755-1801) and the
 * Numerical-Recipes shuffle rano (cheisdwf.f:1722-1751).
 * ==================================================================== */
static const double DM1 = 15184245.0, DM2 = 2651554.0;
static const double DX24 = 16777216.0, DX48 = 281474976710656.0;

void orc_rranset(orc_rng* g, double seed) {           /* G900ST, :1797-1800 */
    g->ds[1] = trunc(seed / DX24);
    g->ds[0] = seed - g->ds[1] * DX24;
}
double orc_rranget(const orc_rng* g) { return g->ds[1] * DX24 + g->ds[0]; } /* :1794 */

float orc_rranf(orc_rng* g) {                          /* :1785-1792 */
    double dl = g->ds[0] * DM1;
    double dc = trunc(dl / DX24);
    dl = dl - dc * DX24;
    double du = g->ds[0] * DM2 + g->ds[1] * DM1 + dc;
    g->ds[1] = du - trunc(du / DX24) * DX24;
    g->ds[0] = dl;
    double dr = (g->ds[1] * DX24 + g->ds[0]) / DX48;
    return (float)dr;                                  /* SNGL */
}

float orc_rano(orc_rng* g, float* y) {                 /* :1722-1751 */
    if (g->idum < 0) {
        g->idum = 1;
        for (int j = 0; j < 97; j++) (void)orc_rranf(g);
        for (int j = 0; j < 97; j++) g->v[j] = orc_rranf(g);
        *y = orc_rranf(g);
    }
    int j = 1 + (int)(97.0f * *y);
    if (j > 97) j = 97;
    if (j < 1) j = 1;
    *y = g->v[j - 1];
    float r = *y;
    g->v[j - 1] = orc_rranf(g);
    return r;
}

/* Start-up sequence of program dwf3d (cheisdwf.f:125-130): rranset(seed),
 * idum=-1, one rano(yran) call that fills the shuffle table.  yrun, the
 * undeclared main-program local used for the trajectory-end and Metropolis
 * draws (:298,:329), starts at 0.0. */
void orc_rng_startup(orc_rng* g, double seed) {
    memset(g, 0, sizeof(*g));
    orc_rranset(g, seed);
    g->idum = -1;
    g->yrun = 0.0f;
    (void)orc_rano(g, &g->yran);
}

static const float TPI_F = 2.0f * 3.14159265358979323846f;  /* tpi=2.0*acos(-1.0), :93 */

void orc_gauss0(orc_rng* g, int64_t kvol, float* ps) {        /* :1701-1718 */
    for (int64_t i = 0; i < kvol; i++) ps[kvol + i] = sqrtf(-logf(orc_rano(g, &g->yran)));
    for (int64_t i = 0; i < kvol; i++) {
        float theta = TPI_F * orc_rano(g, &g->yran);
        ps[i] = ps[kvol + i] * sinf(theta);
        ps[kvol + i] = ps[kvol + i] * cosf(theta);
    }
}

void orc_gaussp(orc_rng* g, int64_t kvol, float* ps) {        /* :1678-1695 */
    for (int64_t i = 0; i < kvol; i++)
        ps[kvol + i] = sqrtf(-2.0f * logf(orc_rano(g, &g->yran)));
    for (int64_t i = 0; i < kvol; i++) {
        float theta = TPI_F * orc_rano(g, &g->yran);
        ps[i] = ps[kvol + i] * sinf(theta);
        ps[kvol + i] = ps[kvol + i] * cosf(theta);
    }
}

/* ======================================================================
 * Operator M and M^dagger, live "v2" routines (cheisdwf.f:2634-3501),
 * restated sweep by sweep so each output element sees the reference's
 * sequence of floating-point operations.
 * ==================================================================== */
#define SIDX(s, site, d, f) ((int64_t)(s) + Ls * ((int64_t)(site) + kvol * ((int64_t)(d) + 4 * (int64_t)(f))))

/* One Wilson+Dirac hop sweep.  mu: 0=x,1=y,2=t.  sig=+1 is the pattern the
 * reference uses for M with the forward neighbour (cheisdwf.f:2672-2693,
 * 2719-2739, 2766-2787); sig=-1 the backward-neighbour pattern (:2695-2717,
 * 2741-2763, 2789-2812).  M^dagger swaps the two (:3107-3246).  neg=1 gives
 * the antiperiodic boundary correction, which adds the same combinations
 * with all signs reversed (:2831-2876, :3265-3310). */
typedef struct { int pa, pb, ia, ib, sa, sb, x3, x4, i3, i4, s3, s4; } hop_pat;

static hop_pat pattern(int mu, int sig) {
    hop_pat p;
    if (mu == 0) {        /* a=R1+zi*R4 b=R2+zi*R3 ; Phi3+=zi*b Phi4+=zi*a */
        p.pa = 3; p.pb = 2; p.ia = 1; p.ib = 1; p.sa = 1; p.sb = 1;
        p.x3 = 1; p.x4 = 0; p.i3 = 1; p.i4 = 1; p.s3 = 1; p.s4 = 1;
    } else if (mu == 1) { /* a=R1+R4 b=R2-R3 ; Phi3+=b Phi4-=a */
        p.pa = 3; p.pb = 2; p.ia = 0; p.ib = 0; p.sa = 1; p.sb = -1;
        p.x3 = 1; p.x4 = 0; p.i3 = 0; p.i4 = 0; p.s3 = 1; p.s4 = -1;
    } else {              /* a=R1+zi*R3 b=R2-zi*R4 ; Phi3+=zi*a Phi4-=zi*b */
        p.pa = 2; p.pb = 3; p.ia = 1; p.ib = 1; p.sa = 1; p.sb = -1;
        p.x3 = 0; p.x4 = 1; p.i3 = 1; p.i4 = 1; p.s3 = 1; p.s4 = -1;
    }
    p.sa *= sig; p.sb *= sig; p.s3 *= sig; p.s4 *= sig;
    return p;
}

static inline cx comb(cx x, cx y, int use_i, int sgn) {
    cx t = use_i ? cmuli(y) : y;
    return sgn > 0 ? cadd(x, t) : csub(x, t);
}

/* Apply pattern p to output point j with source neighbour n. */
static inline void hop_apply(double* Phi, const double* R, int64_t o0, int64_t n0,
                             int64_t cstride, hop_pat p, int neg) {
    cx r1 = ld(R, n0), r2 = ld(R, n0 + cstride);
    cx rpa = ld(R, n0 + p.pa * cstride), rpb = ld(R, n0 + p.pb * cstride);
    cx a = comb(r1, rpa, p.ia, p.sa);
    cx b = comb(r2, rpb, p.ib, p.sb);
    int m = neg ? -1 : 1;
    st(Phi, o0, comb(ld(Phi, o0), a, 0, -m));
    st(Phi, o0 + cstride, comb(ld(Phi, o0 + cstride), b, 0, -m));
    cx x3 = p.x3 ? b : a, x4 = p.x4 ? b : a;
    st(Phi, o0 + 2 * cstride, comb(ld(Phi, o0 + 2 * cstride), x3, p.i3, m * p.s3));
    st(Phi, o0 + 3 * cstride, comb(ld(Phi, o0 + 3 * cstride), x4, p.i4, m * p.s4));
}

static void hop_sweep(const orc_lat* lat, double* Phi, const double* R, int f,
                      int mu, int dir, int sig) {
    const int L = lat->L, Lt = lat->Lt;
    const int64_t Ls = lat->Ls, kvol = orc_kvol(lat);
    const int64_t cs = Ls * kvol;                 /* Dirac stride */
#pragma omp parallel for if (lat->threads > 1) num_threads(lat->threads > 1 ? lat->threads : 1)
    for (int it = 0; it < Lt; it++)
        for (int iy = 0; iy < L; iy++)
            for (int ix = 0; ix < L; ix++) {
                int nx = ix, ny = iy, nt = it;
                if (mu == 0) nx = (ix + dir + L) % L;
                if (mu == 1) ny = (iy + dir + L) % L;
                if (mu == 2) nt = (it + dir + Lt) % Lt;
                int64_t site = ix + (int64_t)L * (iy + (int64_t)L * it);
                int64_t nsite = nx + (int64_t)L * (ny + (int64_t)L * nt);
                hop_pat p = pattern(mu, sig);
                for (int64_t s = 0; s < Ls; s++)
                    hop_apply(Phi, R, SIDX(s, site, 0, f), SIDX(s, nsite, 0, f), cs, p, 0);
            }
}

static void s_and_walls(const orc_lat* lat, double* Phi, const double* R, const double* chi,
                        float hpin, int imass, int dag);

static void dslash_common(const orc_lat* lat, double* Phi, const double* R,
                          const double* chi, float hpin, int imass, int dag) {
    const int L = lat->L, Lt = lat->Lt;
    const int64_t Ls = lat->Ls, kvol = orc_kvol(lat), kferm = orc_kferm(lat);
    const int64_t cs = Ls * kvol;
    const int nth = lat->threads > 1 ? lat->threads : 1;
    (void)nth;
    /* diagonal term, scaled by two (:2651-2667 / :3088-3104) */
    const float diag = 2.0f * ((3.0f - lat->am3) + 1.0f);
#pragma omp parallel for if (lat->threads > 1) num_threads(nth)
    for (int64_t j = 0; j < kferm; j++) st(Phi, j, cscal((double)diag, ld(R, j)));
    /* Wilson + Dirac hops per flavour: +x, -x, +y, -y, +t, -t */
    const int sf = dag ? -1 : 1;
    for (int f = 0; f < 2; f++)
        for (int mu = 0; mu < 3; mu++) {
            hop_sweep(lat, Phi, R, f, mu, +1, sf);
            hop_sweep(lat, Phi, R, f, mu, -1, -sf);
        }
    /* kappa = 0.5 normalisation (:2815-2829 / :3249-3263) */
#pragma omp parallel for if (lat->threads > 1) num_threads(nth)
    for (int64_t j = 0; j < kferm; j++) st(Phi, j, cscal(0.5, ld(Phi, j)));
    /* antiperiodic t boundary (:2831-2876 / :3265-3310) */
    if (lat->ibound == -1) {
        for (int f = 0; f < 2; f++) {
            for (int iy = 0; iy < L; iy++)
                for (int ix = 0; ix < L; ix++) {
                    int64_t s_last = ix + (int64_t)L * (iy + (int64_t)L * (Lt - 1));
                    int64_t s_first = ix + (int64_t)L * iy;
                    for (int64_t s = 0; s < Ls; s++)
                        hop_apply(Phi, R, SIDX(s, s_last, 0, f), SIDX(s, s_first, 0, f), cs,
                                  pattern(2, sf), 1);
                }
            for (int iy = 0; iy < L; iy++)
                for (int ix = 0; ix < L; ix++) {
                    int64_t s_last = ix + (int64_t)L * (iy + (int64_t)L * (Lt - 1));
                    int64_t s_first = ix + (int64_t)L * iy;
                    for (int64_t s = 0; s < Ls; s++)
                        hop_apply(Phi, R, SIDX(s, s_first, 0, f), SIDX(s, s_last, 0, f), cs,
                                  pattern(2, -sf), 1);
                }
        }
    }
    s_and_walls(lat, Phi, R, chi, hpin, imass, dag);
}

static void s_and_walls(const orc_lat* lat, double* Phi, const double* R, const double* chi,
                        float hpin, int imass, int dag) {
    const int64_t Ls = lat->Ls, kvol = orc_kvol(lat);
    /* s hops exploiting the chiral projection (:2879-2908 / :3313-3342).
     * M: Dirac 3,4 from s+1 then Dirac 1,2 from s-1; M^dagger the reverse roles. */
    const int up0 = dag ? 0 : 2;   /* Dirac pair taking s+1 */
    const int dn0 = dag ? 2 : 0;   /* Dirac pair taking s-1 */
    for (int f = 0; f < 2; f++) {
        for (int d = up0; d < up0 + 2; d++)
            for (int64_t site = 0; site < kvol; site++)
                for (int64_t s = 0; s < Ls - 1; s++) {
                    int64_t o = SIDX(s, site, d, f);
                    st(Phi, o, csub(ld(Phi, o), ld(R, SIDX(s + 1, site, d, f))));
                }
        for (int d = dn0; d < dn0 + 2; d++)
            for (int64_t site = 0; site < kvol; site++)
                for (int64_t s = 0; s < Ls - 1; s++) {
                    int64_t o = SIDX(s + 1, site, d, f);
                    st(Phi, o, csub(ld(Phi, o), ld(R, SIDX(s, site, d, f))));
                }
    }
    /* chi coupling between the walls.  M: Dirac 3,4 at s=Ls read s=1 and
     * Dirac 1,2 at s=1 read s=Ls; M^dagger swaps the Dirac pairs. */
    const int wA = dag ? 0 : 2;    /* pair written at s=Ls */
    const int wB = dag ? 2 : 0;    /* pair written at s=1  */
    const int64_t sL = Ls - 1;
    if (imass == 1) {
        /* spm = cmplx(chi3, 0.0): REAL*4-rounded (:2912-2946 / :3345-3379) */
        for (int d = wA; d < wA + 2; d++)
            for (int64_t i = 0; i < kvol; i++) {
                cx spm = {(double)(float)chi[i + 2 * kvol], 0.0};
                int64_t o1 = SIDX(sL, i, d, 0), o2 = SIDX(sL, i, d, 1);
                st(Phi, o1, cadd(ld(Phi, o1), cmul(spm, ld(R, SIDX(0, i, d, 0)))));
                st(Phi, o2, csub(ld(Phi, o2), cmul(spm, ld(R, SIDX(0, i, d, 1)))));
            }
        for (int d = wB; d < wB + 2; d++)
            for (int64_t i = 0; i < kvol; i++) {
                cx spm = {(double)(float)chi[i + 2 * kvol], 0.0};
                int64_t o1 = SIDX(0, i, d, 0), o2 = SIDX(0, i, d, 1);
                st(Phi, o1, cadd(ld(Phi, o1), cmul(spm, ld(R, SIDX(sL, i, d, 0)))));
                st(Phi, o2, csub(ld(Phi, o2), cmul(spm, ld(R, SIDX(sL, i, d, 1)))));
            }
        /* pinning at site (1,1,1) (:2948-2959 / :3381-3392) */
        for (int d = wA; d < wA + 2; d++) {
            int64_t o1 = SIDX(sL, 0, d, 0), o2 = SIDX(sL, 0, d, 1);
            st(Phi, o1, cadd(ld(Phi, o1), cscal((double)hpin, ld(R, SIDX(0, 0, d, 0)))));
            st(Phi, o2, csub(ld(Phi, o2), cscal((double)hpin, ld(R, SIDX(0, 0, d, 1)))));
        }
        for (int d = wB; d < wB + 2; d++) {
            int64_t o1 = SIDX(0, 0, d, 0), o2 = SIDX(0, 0, d, 1);
            st(Phi, o1, cadd(ld(Phi, o1), cscal((double)hpin, ld(R, SIDX(sL, 0, d, 0)))));
            st(Phi, o2, csub(ld(Phi, o2), cscal((double)hpin, ld(R, SIDX(sL, 0, d, 1)))));
        }
        /* spm = cmplx(chi1, -chi2) (:2962-2995 / :3395-3428) */
        for (int d = wA; d < wA + 2; d++)
            for (int64_t i = 0; i < kvol; i++) {
                cx spm = {(double)(float)chi[i], (double)(float)(-chi[i + kvol])};
                int64_t o1 = SIDX(sL, i, d, 0), o2 = SIDX(sL, i, d, 1);
                st(Phi, o1, cadd(ld(Phi, o1), cmul(spm, ld(R, SIDX(0, i, d, 1)))));
                st(Phi, o2, cadd(ld(Phi, o2), cmul(cconj(spm), ld(R, SIDX(0, i, d, 0)))));
            }
        for (int d = wB; d < wB + 2; d++)
            for (int64_t i = 0; i < kvol; i++) {
                cx spm = {(double)(float)chi[i], (double)(float)(-chi[i + kvol])};
                int64_t o1 = SIDX(0, i, d, 0), o2 = SIDX(0, i, d, 1);
                st(Phi, o1, cadd(ld(Phi, o1), cmul(spm, ld(R, SIDX(sL, i, d, 1)))));
                st(Phi, o2, cadd(ld(Phi, o2), cmul(cconj(spm), ld(R, SIDX(sL, i, d, 0)))));
            }
    } else if (imass == 3) {
        /* M:  spm = cmplx(0,+chi3) (:2996-3030); M^dagger: cmplx(0,-chi3) (:3429-3463) */
        for (int d = wA; d < wA + 2; d++)
            for (int64_t i = 0; i < kvol; i++) {
                float c3 = dag ? (float)(-chi[i + 2 * kvol]) : (float)chi[i + 2 * kvol];
                cx spm = {0.0, (double)c3};
                int64_t o1 = SIDX(sL, i, d, 0), o2 = SIDX(sL, i, d, 1);
                cx t1 = cmul(spm, ld(R, SIDX(0, i, d, 0))), t2 = cmul(spm, ld(R, SIDX(0, i, d, 1)));
                if (!dag) { st(Phi, o1, csub(ld(Phi, o1), t1)); st(Phi, o2, cadd(ld(Phi, o2), t2)); }
                else      { st(Phi, o1, cadd(ld(Phi, o1), t1)); st(Phi, o2, csub(ld(Phi, o2), t2)); }
            }
        for (int d = wB; d < wB + 2; d++)
            for (int64_t i = 0; i < kvol; i++) {
                float c3 = dag ? (float)(-chi[i + 2 * kvol]) : (float)chi[i + 2 * kvol];
                cx spm = {0.0, (double)c3};
                int64_t o1 = SIDX(0, i, d, 0), o2 = SIDX(0, i, d, 1);
                cx t1 = cmul(spm, ld(R, SIDX(sL, i, d, 0))), t2 = cmul(spm, ld(R, SIDX(sL, i, d, 1)));
                if (!dag) { st(Phi, o1, cadd(ld(Phi, o1), t1)); st(Phi, o2, csub(ld(Phi, o2), t2)); }
                else      { st(Phi, o1, csub(ld(Phi, o1), t1)); st(Phi, o2, cadd(ld(Phi, o2), t2)); }
            }
        /* M: spm = cmplx(chi2, chi1) (:3032-3065); M^dagger: cmplx(-chi2,-chi1) (:3465-3497) */
        for (int d = wA; d < wA + 2; d++)
            for (int64_t i = 0; i < kvol; i++) {
                cx spm;
                if (!dag) { spm.re = (double)(float)chi[i + kvol]; spm.im = (double)(float)chi[i]; }
                else { spm.re = (double)(float)(-chi[i + kvol]); spm.im = (double)(float)(-chi[i]); }
                int64_t o1 = SIDX(sL, i, d, 0), o2 = SIDX(sL, i, d, 1);
                cx t1 = cmul(spm, ld(R, SIDX(0, i, d, 1))), t2 = cmul(cconj(spm), ld(R, SIDX(0, i, d, 0)));
                if (!dag) { st(Phi, o1, csub(ld(Phi, o1), t1)); st(Phi, o2, cadd(ld(Phi, o2), t2)); }
                else      { st(Phi, o1, cadd(ld(Phi, o1), t1)); st(Phi, o2, csub(ld(Phi, o2), t2)); }
            }
        for (int d = wB; d < wB + 2; d++)
            for (int64_t i = 0; i < kvol; i++) {
                cx spm;
                if (!dag) { spm.re = (double)(float)chi[i + kvol]; spm.im = (double)(float)chi[i]; }
                else { spm.re = (double)(float)(-chi[i + kvol]); spm.im = (double)(float)(-chi[i]); }
                int64_t o1 = SIDX(0, i, d, 0), o2 = SIDX(0, i, d, 1);
                cx t1 = cmul(spm, ld(R, SIDX(sL, i, d, 1))), t2 = cmul(cconj(spm), ld(R, SIDX(sL, i, d, 0)));
                if (!dag) { st(Phi, o1, cadd(ld(Phi, o1), t1)); st(Phi, o2, csub(ld(Phi, o2), t2)); }
                else      { st(Phi, o1, csub(ld(Phi, o1), t1)); st(Phi, o2, cadd(ld(Phi, o2), t2)); }
            }
    }
}

void orc_dslash(const orc_lat* lat, double* Phi, const double* R, const double* chi,
                float am, float hpin, int imass) {
    (void)am;                       /* "not currently implemented", :26 */
    dslash_common(lat, Phi, R, chi, hpin, imass, 0);
}
void orc_dslashd(const orc_lat* lat, double* Phi, const double* R, const double* chi,
                 float am, float hpin, int imass) {
    (void)am;
    dslash_common(lat, Phi, R, chi, hpin, imass, 1);
}

/* ======================================================================
 * The dead "v1" operator (cheisdwf.f:1804-2217): separate Wilson and Dirac
 * sweeps driven by the gamma tables of init (:1521-1597).  Restated only
 * as a second, independent formulation of M to check the v2 restatement.
 * ==================================================================== */
void orc_dslash_v1(const orc_lat* lat, double* Phi, const double* R, const double* chi,
                   float am, float hpin, int imass) {
    (void)am;
    const int L = lat->L, Lt = lat->Lt;
    const int64_t Ls = lat->Ls, kvol = orc_kvol(lat), kferm = orc_kferm(lat);
    const double ak = 0.5;
    /* gamval(mu,idirac)*akappa and gamin(mu,idirac), mu = 1,2,3 (:1524-1561) */
    const cx gv[3][4] = {{{0, -ak}, {0, -ak}, {0, ak}, {0, ak}},
                         {{-ak, 0}, {ak, 0}, {ak, 0}, {-ak, 0}},
                         {{0, -ak}, {0, ak}, {0, ak}, {0, -ak}}};
    const int gi[3][4] = {{3, 2, 1, 0}, {3, 2, 1, 0}, {2, 3, 0, 1}};
    const float diag = (3.0f - lat->am3) + 1.0f;                      /* :1823 */
    for (int64_t j = 0; j < kferm; j++) st(Phi, j, cscal((double)diag, ld(R, j)));
#define NB(ix, iy, it) ((int64_t)(ix) + (int64_t)L * ((iy) + (int64_t)L * (it)))
    /* Wilson term (:1841-1888) */
    for (int f = 0; f < 2; f++)
        for (int d = 0; d < 4; d++)
            for (int mu = 0; mu < 3; mu++)
                for (int it = 0; it < Lt; it++)
                    for (int iy = 0; iy < L; iy++)
                        for (int ix = 0; ix < L; ix++) {
                            int xp = ix, xm = ix, yp = iy, ym = iy, tp = it, tm = it;
                            if (mu == 0) { xp = (ix + 1) % L; xm = (ix + L - 1) % L; }
                            if (mu == 1) { yp = (iy + 1) % L; ym = (iy + L - 1) % L; }
                            if (mu == 2) { tp = (it + 1) % Lt; tm = (it + Lt - 1) % Lt; }
                            for (int64_t s = 0; s < Ls; s++) {
                                int64_t o = SIDX(s, NB(ix, iy, it), d, f);
                                cx sum = cadd(ld(R, SIDX(s, NB(xp, yp, tp), d, f)),
                                              ld(R, SIDX(s, NB(xm, ym, tm), d, f)));
                                st(Phi, o, csub(ld(Phi, o), cscal(ak, sum)));
                            }
                        }
    if (lat->ibound == -1)                                            /* :1891-1919 */
        for (int f = 0; f < 2; f++)
            for (int d = 0; d < 4; d++) {
                for (int iy = 0; iy < L; iy++)
                    for (int ix = 0; ix < L; ix++)
                        for (int64_t s = 0; s < Ls; s++) {
                            int64_t o = SIDX(s, NB(ix, iy, Lt - 1), d, f);
                            st(Phi, o, cadd(ld(Phi, o), ld(R, SIDX(s, NB(ix, iy, 0), d, f))));
                        }
                for (int iy = 0; iy < L; iy++)
                    for (int ix = 0; ix < L; ix++)
                        for (int64_t s = 0; s < Ls; s++) {
                            int64_t o = SIDX(s, NB(ix, iy, 0), d, f);
                            st(Phi, o, cadd(ld(Phi, o), ld(R, SIDX(s, NB(ix, iy, Lt - 1), d, f))));
                        }
            }
    /* Dirac term (:1921-1979) */
    for (int f = 0; f < 2; f++)
        for (int d = 0; d < 4; d++)
            for (int mu = 0; mu < 3; mu++) {
                const int ig = gi[mu][d];
                for (int it = 0; it < Lt; it++)
                    for (int iy = 0; iy < L; iy++)
                        for (int ix = 0; ix < L; ix++) {
                            int xp = ix, xm = ix, yp = iy, ym = iy, tp = it, tm = it;
                            if (mu == 0) { xp = (ix + 1) % L; xm = (ix + L - 1) % L; }
                            if (mu == 1) { yp = (iy + 1) % L; ym = (iy + L - 1) % L; }
                            if (mu == 2) { tp = (it + 1) % Lt; tm = (it + Lt - 1) % Lt; }
                            for (int64_t s = 0; s < Ls; s++) {
                                int64_t o = SIDX(s, NB(ix, iy, it), d, f);
                                cx dif = csub(ld(R, SIDX(s, NB(xp, yp, tp), ig, f)),
                                              ld(R, SIDX(s, NB(xm, ym, tm), ig, f)));
                                st(Phi, o, cadd(ld(Phi, o), cmul(gv[mu][d], dif)));
                            }
                        }
            }
    if (lat->ibound == -1)                                            /* :1981-2011 */
        for (int f = 0; f < 2; f++)
            for (int d = 0; d < 4; d++) {
                const int ig = gi[2][d];
                const cx g2 = cscal(2.0, gv[2][d]);
                for (int iy = 0; iy < L; iy++)
                    for (int ix = 0; ix < L; ix++)
                        for (int64_t s = 0; s < Ls; s++) {
                            int64_t o = SIDX(s, NB(ix, iy, Lt - 1), d, f);
                            st(Phi, o, csub(ld(Phi, o), cmul(g2, ld(R, SIDX(s, NB(ix, iy, 0), ig, f)))));
                        }
                for (int iy = 0; iy < L; iy++)
                    for (int ix = 0; ix < L; ix++)
                        for (int64_t s = 0; s < Ls; s++) {
                            int64_t o = SIDX(s, NB(ix, iy, 0), d, f);
                            st(Phi, o, cadd(ld(Phi, o), cmul(g2, ld(R, SIDX(s, NB(ix, iy, Lt - 1), ig, f)))));
                        }
            }
#undef NB
    /* s hops and wall coupling: the same statements as v2 (:2013-2217) */
    s_and_walls(lat, Phi, R, chi, hpin, imass, 0);
}

/* ======================================================================
 * qmrherm: multi-shift Lanczos (cheisdwf.f:599-745)
 * ==================================================================== */
int orc_qmrherm(const orc_lat* lat, const double* Phi, float res, int* itercg,
                float am, float hpin, int imass, const double* anum,
                const double* aden, int ndiag, int iflag, const double* chi,
                double* x, float* dSdchi, int niterc) {
    const int64_t kferm = orc_kferm(lat);
    const int nth = lat->threads > 1 ? lat->threads : 1;
    (void)nth;
    double* vtild = malloc(sizeof(double) * 2 * kferm);
    double* q = malloc(sizeof(double) * 2 * kferm);
    double* qm1 = calloc(2 * kferm, sizeof(double));
    double* x3 = malloc(sizeof(double) * 2 * kferm);
    double* r = malloc(sizeof(double) * 2 * kferm);
    double* p = malloc(sizeof(double) * 2 * kferm * ndiag);   /* p(ndiag,kferm) */
    double* x1 = malloc(sizeof(double) * 2 * kferm * ndiag);  /* x1(ndiag,kferm) */
    double alpha[64], amu[64], d[64], dm1[64], rho[64];
    int status = 0;

    const float resid = sqrtf((float)kferm * res * res);     /* :621 */
    *itercg = 0;
    memcpy(r, Phi, sizeof(double) * 2 * kferm);
    for (int64_t i = 0; i < kferm; i++) st(x, i, cscal(anum[0], ld(Phi, i)));  /* :628 */
    double beta = 0.0;
    for (int64_t i = 0; i < 2 * kferm; i++) beta = beta + r[i] * r[i];
    beta = sqrt(beta);
    const double phimod = beta;

    int iter;
    for (iter = 1; iter <= niterc; iter++) {
        (*itercg)++;
        for (int64_t i = 0; i < kferm; i++) {                 /* q=r/beta, :644 */
            cx v = ld(r, i);
            cx w = {v.re / beta, v.im / beta};
            st(q, i, w);
        }
        orc_dslash(lat, vtild, q, chi, am, hpin, imass);
        orc_dslashd(lat, x3, vtild, chi, am, hpin, imass);
        double alphatild = 0.0;                                /* :649-653 */
        if (lat->threads > 1) {
#pragma omp parallel for reduction(+ : alphatild) num_threads(nth)
            for (int64_t i = 0; i < kferm; i++) {
                cx t = cmul(cconj(ld(q, i)), ld(x3, i));
                alphatild = alphatild + t.re;
            }
        } else {
            for (int64_t i = 0; i < kferm; i++) {
                cx t = cmul(cconj(ld(q, i)), ld(x3, i));
                alphatild = alphatild + t.re;
            }
        }
        for (int64_t i = 0; i < kferm; i++) {                 /* :655 */
            cx v = csub(csub(ld(x3, i), cscal(alphatild, ld(q, i))), cscal(beta, ld(qm1, i)));
            st(r, i, v);
        }
        memcpy(qm1, q, sizeof(double) * 2 * kferm);
        const double beta0 = beta;
        beta = 0.0;                                            /* :659-664 */
        if (lat->threads > 1) {
#pragma omp parallel for reduction(+ : beta) num_threads(nth)
            for (int64_t i = 0; i < kferm; i++) beta = beta + r[2 * i] * r[2 * i] + r[2 * i + 1] * r[2 * i + 1];
        } else {
            for (int64_t i = 0; i < kferm; i++) beta = beta + r[2 * i] * r[2 * i] + r[2 * i + 1] * r[2 * i + 1];
        }
        beta = sqrt(beta);
        for (int k = 0; k < ndiag; k++) alpha[k] = alphatild + aden[k];  /* :666-668 */

        if (iter == 1) {                                       /* :670-681 */
            for (int k = 0; k < ndiag; k++) { d[k] = alpha[k]; rho[k] = beta0 / alpha[k]; }
#pragma omp parallel for if (lat->threads > 1) num_threads(nth)
            for (int64_t i = 0; i < kferm; i++) {
                cx qi = ld(q, i);
                for (int k = 0; k < ndiag; k++) {
                    st(p, i * ndiag + k, qi);
                    st(x1, i * ndiag + k, cscal(rho[k], qi));
                }
            }
        } else {                                               /* :682-715 */
            for (int k = 0; k < ndiag; k++) {
                amu[k] = beta0 / d[k];
                dm1[k] = d[k];
                d[k] = alpha[k] - beta0 * amu[k];
                rho[k] = -amu[k] * dm1[k] * rho[k] / d[k];
            }
#pragma omp parallel for if (lat->threads > 1) num_threads(nth)
            for (int64_t i = 0; i < kferm; i++) {
                cx qi = ld(q, i);
                for (int k = 0; k < ndiag; k++) {
                    cx pn = csub(qi, cscal(amu[k], ld(p, i * ndiag + k)));
                    st(p, i * ndiag + k, pn);
                    st(x1, i * ndiag + k, cadd(ld(x1, i * ndiag + k), cscal(rho[k], pn)));
                }
            }
            double rhomax = 0.0;
            for (int k = 0; k < ndiag; k++) {
                double v = fabs(phimod * rho[k]);
                if (k == 0) rhomax = v;
                else if (v > rhomax) rhomax = v;
            }
            const float arelax = 2.0f;
            if (rhomax < (double)(arelax * resid)) break;
        }
    }
    if (iter > niterc) status = 1;     /* cap reached: silent in the reference */

    if (iflag == 0) {                                          /* :722-727 */
        for (int k = 1; k <= ndiag; k++)
            for (int64_t i = 0; i < kferm; i++)
                st(x, i, cadd(ld(x, i), cscal(anum[k], ld(x1, i * ndiag + (k - 1)))));
    } else {                                                   /* :729-740 */
        double* R = malloc(sizeof(double) * 2 * kferm);
        double* X2 = malloc(sizeof(double) * 2 * kferm);
        for (int k = 1; k <= ndiag; k++) {
            for (int64_t i = 0; i < kferm; i++) st(R, i, ld(x1, i * ndiag + (k - 1)));
            orc_dslash(lat, X2, R, chi, am, hpin, imass);
            orc_derivs(lat, R, X2, anum[k], imass, dSdchi);
        }
        free(R); free(X2);
    }
    free(vtild); free(q); free(qm1); free(x3); free(r); free(p); free(x1);
    return status;
}

/* ======================================================================
 * derivs (cheisdwf.f:747-849): REAL*8 products, REAL*4 accumulation.
 * ==================================================================== */
void orc_derivs(const orc_lat* lat, const double* R, const double* X2, double anum,
                int imass, float* dSdchi) {
    const int64_t Ls = lat->Ls, kvol = orc_kvol(lat);
    const int64_t sL = Ls - 1;
    const double tzi = -2 * anum;
    /* Dirac 1,2: R at s=Ls against X2 at s=1; Dirac 3,4: R at s=1 against X2 at s=Ls */
    for (int half = 0; half < 2; half++) {
        const int64_t sr = half == 0 ? sL : 0, sx = half == 0 ? 0 : sL;
        const double sg = half == 0 ? 1.0 : -1.0;  /* imass=3 flips sign between halves */
        for (int d = 2 * half; d < 2 * half + 2; d++)
            for (int64_t i = 0; i < kvol; i++) {
                cx r1 = cconj(ld(R, SIDX(sr, i, d, 0))), r2 = cconj(ld(R, SIDX(sr, i, d, 1)));
                cx y1 = ld(X2, SIDX(sx, i, d, 0)), y2 = ld(X2, SIDX(sx, i, d, 1));
                cx c1 = cscal(tzi, cadd(cmul(r1, y2), cmul(r2, y1)));
                cx c2 = cscal(tzi, csub(cmul(r1, y2), cmul(r2, y1)));
                cx c3 = cscal(tzi, csub(cmul(r1, y1), cmul(r2, y2)));
                float* f1 = &dSdchi[i];
                float* f2 = &dSdchi[i + kvol];
                float* f3 = &dSdchi[i + 2 * kvol];
                if (imass == 1) {                               /* :762-802 */
                    *f1 = (float)((double)*f1 - c1.re);
                    *f2 = (float)((double)*f2 - c2.im);
                    *f3 = (float)((double)*f3 - c3.re);
                } else if (imass == 3) {                        /* :804-845 */
                    if (sg > 0) {
                        *f1 = (float)((double)*f1 - c1.im);
                        *f2 = (float)((double)*f2 + c2.re);
                        *f3 = (float)((double)*f3 - c3.im);
                    } else {
                        *f1 = (float)((double)*f1 + c1.im);
                        *f2 = (float)((double)*f2 - c2.re);
                        *f3 = (float)((double)*f3 + c3.im);
                    }
                }
            }
    }
}

/* REAL*4 sum of |v_i|^2 over n complex entries, as congrad's
 * !$OMP PARALLEL DO REDUCTION(+:alphad) / (+:betan) forms it (cheisdwf.f:1105-1108,
 * :1133-1136): each term is added in REAL*8 and the sum rounded to REAL*4 at
 * every step.  With nth > 1 the loop is split as OpenMP's static schedule
 * splits it (the first n % nth threads take one entry more), each thread
 * sums its contiguous chunk from zero, and the partials are added to the
 * shared REAL*4 sum in thread order (one of the orders the runtime may
 * take).  nth = 1 is the sequential loop. */
static float r4_norm2(const double* v, int64_t n, int nth) {
    if (nth < 1) nth = 1;
    const int64_t q0 = n / nth, rem = n % nth;
    float s = 0.0f;
    for (int t = 0; t < nth; t++) {
        const int64_t q = q0 + (t < rem ? 1 : 0), s0 = q0 * t + (t < rem ? t : rem);
        float part = 0.0f;
        for (int64_t i = s0; i < s0 + q; i++)
            part = (float)((double)part + v[2 * i] * v[2 * i] + v[2 * i + 1] * v[2 * i + 1]);
        s = s + part;
    }
    return s;
}

/* ======================================================================
 * congrad: CGNE on M^dagger M with REAL*4 scalars (cheisdwf.f:1064-1157)
 * ==================================================================== */
int orc_congrad(const orc_lat* lat, const double* Phi, float res, int* itercg,
                float am, float hpin, int imass, const double* chi, double* x) {
    const int64_t kferm = orc_kferm(lat), kvol = orc_kvol(lat);
    const int64_t niterc = lat->Ls * kvol;
    double* x1 = malloc(sizeof(double) * 2 * kferm);
    double* x2 = malloc(sizeof(double) * 2 * kferm);
    double* p = malloc(sizeof(double) * 2 * kferm);
    double* r = malloc(sizeof(double) * 2 * kferm);
    const float resid = (float)kferm * res * res;
    float betad = 1.0f, alpha = 1.0f, alphad = 0.0f, alphan = 0.0f, betan, beta;
    int capped = 1;
    *itercg = 0;
    for (int64_t nx = 1; nx <= niterc; nx++) {
        (*itercg)++;
        if (nx == 1) {
            memcpy(p, x, sizeof(double) * 2 * kferm);
            memcpy(r, Phi, sizeof(double) * 2 * kferm);
            betad = 1.0f;
            alpha = 1.0f;
        }
        alphad = 0.0f;
        orc_dslash(lat, x1, p, chi, am, hpin, imass);
        if (nx != 1) {
            alphad = r4_norm2(x1, kferm, lat->threads);
            alpha = alphan / alphad;
            for (int64_t i = 0; i < kferm; i++) st(x, i, cadd(ld(x, i), cscal((double)alpha, ld(p, i))));
        }
        orc_dslashd(lat, x2, x1, chi, am, hpin, imass);
        for (int64_t i = 0; i < kferm; i++) st(r, i, csub(ld(r, i), cscal((double)alpha, ld(x2, i))));
        betan = r4_norm2(r, kferm, lat->threads);
        beta = betan / betad;
        betad = betan;
        alphan = betan;
        if (nx == 1) beta = 0.0f;
        for (int64_t i = 0; i < kferm; i++) st(p, i, cadd(ld(r, i), cscal((double)beta, ld(p, i))));
        if (betan < resid) { capped = 0; break; }
    }
    free(x1); free(x2); free(p); free(r);
    return capped;
}

/* ======================================================================
 * measure (cheisdwf.f:1164-1453): noisy estimator of psibar psi and its
 * disconnected susceptibility, knoise = 10 noise vectors, each with sources
 * on the s=1 and s=Ls walls for Dirac indices 1, 2.  imass 1 or 3 (the
 * operator of this code has no imass 5 term).  xi: /vector/ scratch.
 * parts (4*knoise doubles, or NULL): re/im of psibarpsi1 and psibarpsi2 of
 * each noise, the record written to fort.100 (:1433-1434).
 * ==================================================================== */
void orc_measure(const orc_lat* lat, orc_rng* g, float res, float am, float hpin, int imass,
                 const double* chi, double* xi, float* psibarpsi, float* susclsing,
                 float* aviter, double* parts) {
    const int64_t Ls = lat->Ls, kvol = orc_kvol(lat), kferm = orc_kferm(lat);
    enum { knoise = 10 };
    float* ps = malloc(sizeof(float) * 2 * kvol);
    float* pt = malloc(sizeof(float) * 2 * kvol);
    double* Phi = malloc(sizeof(double) * 2 * kferm);
    float pbp[knoise];
    int iter = 0;
    for (int inoise = 0; inoise < knoise; inoise++) {
        orc_gauss0(g, kvol, ps);                                               /* :1187 */
        cx p1 = {0.0, 0.0};
        orc_gauss0(g, kvol, pt);                                               /* :1189 */
        cx p2 = {0.0, 0.0};
        for (int idsource = 1; idsource <= 2; idsource++) {
            for (int wall = 0; wall < 2; wall++) {
                /* wall 0: source x = cmplx(ps) on s=1 for Dirac idsource
                 * (:1194-1235); wall 1: x = cmplx(pt) on s=Ls for idsource+2
                 * (:1303-1346) */
                const float* nz = wall == 0 ? ps : pt;
                const int d = wall == 0 ? idsource - 1 : idsource + 1;
                const int64_t s_src = wall == 0 ? 0 : Ls - 1;
                const int64_t s_read = wall == 0 ? Ls - 1 : 0;
                memset(xi, 0, sizeof(double) * 2 * kferm);
                for (int f = 0; f < 2; f++)
                    for (int64_t i = 0; i < kvol; i++) {
                        cx x = {(double)nz[i], (double)nz[kvol + i]};
                        st(xi, SIDX(s_src, i, d, f), x);
                    }
                orc_dslashd(lat, Phi, xi, chi, am, hpin, imass);               /* :1273, :1372 */
                memcpy(xi, Phi, sizeof(double) * 2 * kferm);
                int itercg = 0;
                orc_congrad(lat, Phi, res, &itercg, am, hpin, imass, chi, xi);  /* :1284, :1383 */
                iter += itercg;
                cx acc = wall == 0 ? p1 : p2;
                for (int f = 0; f < 2; f++)                                    /* :1289-1294, :1388-1393 */
                    for (int64_t i = 0; i < kvol; i++) {
                        cx x = {(double)nz[i], (double)nz[kvol + i]};
                        acc = cadd(acc, cmul(cconj(x), ld(xi, SIDX(s_read, i, d, f))));
                    }
                if (wall == 0) p1 = acc;
                else p2 = acc;
            }
        }
        const double kv = (double)kvol;
        if (imass == 1) {                                                      /* :1418-1421 */
            p1.re /= kv; p1.im /= kv;
            p2.re /= kv; p2.im /= kv;
        } else {                                                               /* :1422-1425 */
            const cx mi = {0.0, -1.0}, pi = {0.0, 1.0};
            p1 = cmul(mi, p1); p1.re /= kv; p1.im /= kv;
            p2 = cmul(pi, p2); p2.re /= kv; p2.im /= kv;
        }
        pbp[inoise] = (float)(p1.re + p2.re);
        if (parts) {
            parts[4 * inoise] = p1.re; parts[4 * inoise + 1] = p1.im;
            parts[4 * inoise + 2] = p2.re; parts[4 * inoise + 3] = p2.im;
        }
    }
    float pb = 0.0f, sus = 0.0f;                                               /* :1440-1449 */
    for (int inoise = 0; inoise < knoise; inoise++) {
        pb = pb + pbp[inoise];
        for (int jnoise = knoise - 1; jnoise >= inoise + 1; jnoise--) sus = sus + pbp[inoise] * pbp[jnoise];
    }
    pb = pb / (float)knoise;
    sus = (float)(2 * kvol) * sus / (float)(knoise * (knoise - 1));
    *psibarpsi = pb;
    *susclsing = sus;
    *aviter = (float)iter / (float)(4 * knoise);                               /* :1451 */
    free(ps); free(pt); free(Phi);
}

/* ======================================================================
 * force (cheisdwf.f:470-518) and hamilton (cheisdwf.f:522-589)
 * ==================================================================== */
void orc_force(const orc_lat* lat, const double* Phi, float res1, float am, float hpin,
               int imass, const double* chi, const orc_remez* r2g, float* dSdchi,
               double* x, int* itg, int* itf) {
    const int64_t kvol = orc_kvol(lat), kferm = orc_kferm(lat);
    const float twob = 2 * lat->beta;
    for (int a = 0; a < 3; a++)
        for (int64_t i = 0; i < kvol; i++)
            dSdchi[i + kvol * a] = (float)((double)twob * chi[i + kvol * a]);
    double* X2 = malloc(sizeof(double) * 2 * kferm);
    memcpy(X2, Phi, sizeof(double) * 2 * kferm);
    orc_qmrherm(lat, X2, res1, itg, am, hpin, imass, r2g->bnum, r2g->bden + 0, r2g->n, 0,
                chi, x, dSdchi, 5000);
    memcpy(X2, x, sizeof(double) * 2 * kferm);
    orc_qmrherm(lat, X2, res1, itf, am, hpin, imass, r2g->anum, r2g->aden, r2g->n, 1,
                chi, x, dSdchi, 5000);
    free(X2);
}

void orc_hamilton(const orc_lat* lat, const double* Phi, float res2, float am, float hpin,
                  int imass, const double* chi, const float* pp, const orc_remez* r2,
                  double* out, double* x, int* itercg) {
    const int64_t kvol = orc_kvol(lat), kferm = orc_kferm(lat);
    double hp = 0.0, hg = 0.0, hf = 0.0;
    for (int a = 0; a < 3; a++)
        for (int64_t i = 0; i < kvol; i++) hp = hp + (double)(pp[i + kvol * a] * pp[i + kvol * a]);
    hp = hp * 0.5;
    for (int a = 0; a < 3; a++)
        for (int64_t i = 0; i < kvol; i++) hg = hg + chi[i + kvol * a] * chi[i + kvol * a];
    hg = (double)lat->beta * hg;
    orc_qmrherm(lat, Phi, res2, itercg, am, hpin, imass, r2->bnum, r2->bden, r2->n, 0, chi, x,
                NULL, 5000);
    for (int64_t i = 0; i < kferm; i++) hf = hf + cmul(cconj(ld(Phi, i)), ld(x, i)).re;
    out[0] = hg + hp + hf;
    out[1] = hg;
    out[2] = hp;
    out[3] = hg + hf;
    out[4] = hf;
}

/* ======================================================================
 * fermion: wall-source propagator and correlators (cheisdwf.f:897-1058)
 * ==================================================================== */
float orc_fermion(const orc_lat* lat, orc_rng* g, float res, float am, float hpin, int imass,
                  const double* chi, double* xi, float* cferm1, float* cferm2) {
    const int L = lat->L, Lt = lat->Lt;
    const int64_t Ls = lat->Ls, kvol = orc_kvol(lat), kferm = orc_kferm(lat);
    const int64_t ksize2 = (int64_t)L * L;
    const int nsource = 5;
    const float akappa = 0.5f;
    /* gamval(3,idd)*akappa for idd=3,4 is (0,+0.5),(0,-0.5); gamin(3,3..4)=1,2 (:1549-1557,:1596) */
    const cx gam3[2] = {{0.0, 0.5}, {0.0, -0.5}};
    const int gin3[2] = {0, 1};
    float* prop00 = calloc((size_t)kvol * 2 * 2 * 2 * 2, sizeof(float)); /* (kvol,3:4,1:2,2) complex */
    float* prop0L = calloc((size_t)kvol * 2 * 2 * 2 * 2, sizeof(float)); /* (kvol,3:4,3:4,2) complex */
    double* Phi = malloc(sizeof(double) * 2 * kferm);
    int iter = 0;
    for (int i = 0; i < 4 * Lt; i++) { cferm1[i] = 0.0f; cferm2[i] = 0.0f; }
#define PIDX(i, a, b, f) (2 * ((i) + kvol * ((a) + 2 * ((b) + 2 * (int64_t)(f)))))
    const int ittt0 = (int)((float)Lt * orc_rano(g, &g->yran)) + 1;           /* :929 */
    for (int ksource = 1; ksource <= nsource; ksource++) {
        const int ittt = (ittt0 + ksource * (Lt / nsource)) % Lt + 1;          /* :937 */
        for (int idsource = 3; idsource <= 4; idsource++) {
            memset(xi, 0, sizeof(double) * 2 * kferm);
            const int64_t ioff = (int64_t)(ittt - 1) * ksize2;
            const double wall = (double)(1.0f / (float)ksize2);               /* (1.0,0.0)/ksize2 */
            for (int64_t i = 0; i < ksize2; i++) {
                cx w = {wall, 0.0};
                st(xi, SIDX(0, i + ioff, idsource - 1, 0), w);
            }
            orc_dslashd(lat, Phi, xi, chi, am, hpin, imass);                 /* :979 */
            memcpy(xi, Phi, sizeof(double) * 2 * kferm);
            int itercg;
            orc_congrad(lat, Phi, res, &itercg, am, hpin, imass, chi, xi);  /* :996 */
            iter += itercg;
            for (int f = 0; f < 2; f++)
                for (int idsink = 1; idsink <= 2; idsink++) {
                    const int idsink2 = idsink + 2;
                    for (int64_t i = 0; i < kvol; i++) {
                        cx a = ld(xi, SIDX(0, i, idsink - 1, f));
                        cx b = ld(xi, SIDX(Ls - 1, i, idsink2 - 1, f));
                        int64_t pa = PIDX(i, idsource - 3, idsink - 1, f);
                        int64_t pb = PIDX(i, idsource - 3, idsink2 - 3, f);
                        prop00[pa] = (float)a.re; prop00[pa + 1] = (float)a.im;
                        prop0L[pb] = (float)b.re; prop0L[pb + 1] = (float)b.im;
                    }
                }
        }
        for (int idd = 3; idd <= 4; idd++)                                    /* :1014-1034 */
            for (int it = 0; it < Lt; it++) {
                const int itt = (ittt + it - 1) % Lt + 1;
                const int isign = itt >= ittt ? 1 : lat->ibound;
                const int64_t ioff = (int64_t)(itt - 1) * ksize2;
                for (int f = 0; f < 2; f++)
                    for (int64_t i = 0; i < ksize2; i++) {
                        const float sk = (float)isign * akappa;
                        int64_t pl = PIDX(i + ioff, idd - 3, idd - 3, f);
                        float* c1 = &cferm1[2 * (it + Lt * f)];
                        c1[0] = c1[0] + sk * prop0L[pl];
                        c1[1] = c1[1] + sk * prop0L[pl + 1];
                        cx gv = cscal((double)isign, gam3[idd - 3]);
                        int64_t p0 = PIDX(i + ioff, idd - 3, gin3[idd - 3], f);
                        cx pv = {(double)prop00[p0], (double)prop00[p0 + 1]};
                        cx t = cmul(gv, pv);
                        float* c2 = &cferm2[2 * (it + Lt * f)];
                        c2[0] = (float)((double)c2[0] + t.re);
                        c2[1] = (float)((double)c2[1] + t.im);
                    }
            }
    }
    for (int i = 0; i < 4 * Lt; i++) {
        cferm1[i] = cferm1[i] / (float)nsource;
        cferm2[i] = cferm2[i] / (float)nsource;
    }
#undef PIDX
    free(prop00); free(prop0L); free(Phi);
    return (float)iter / (float)(2 * nsource);
}

/* ======================================================================
 * program dwf3d main loop (cheisdwf.f:207-399)
 * ==================================================================== */
orc_state* orc_state_new(int L, int Lt, int Ls, float beta, float am3, float dt, float am,
                         float hpin, int imass, int iterl) {
    orc_state* s = calloc(1, sizeof(orc_state));
    s->lat.L = L; s->lat.Lt = Lt; s->lat.Ls = Ls;
    s->lat.beta = beta; s->lat.am3 = am3; s->lat.ibound = -1; s->lat.threads = 1;
    s->dt = dt; s->am = am; s->hpin = hpin; s->imass = imass; s->iterl = iterl;
    s->iprint = 5; s->measure = 1;
    s->rescga = 0.000000001f; s->rescgg = 0.000001f; s->rescgm = 0.000000001f;  /* :32-33 */
    const int64_t kvol = orc_kvol(&s->lat), kferm = orc_kferm(&s->lat);
    s->chi = malloc(sizeof(double) * 3 * kvol);
    s->chit = malloc(sizeof(double) * 3 * kvol);
    s->pp = calloc(3 * kvol, sizeof(float));
    s->dSdchi = calloc(3 * kvol, sizeof(float));
    s->Phi = calloc(2 * kferm, sizeof(double));
    s->X1 = calloc(2 * kferm, sizeof(double));
    s->R = calloc(2 * kferm, sizeof(double));
    s->ps = calloc(2 * kvol, sizeof(float));
    s->cferm = calloc(4 * Lt * 2, sizeof(float));
    for (int64_t i = 0; i < 3 * kvol; i++) s->chi[i] = (double)(0.1f / beta);  /* sread, :1467 */
    orc_rng_startup(&s->rng, (double)693764523745.0f);                          /* :1468 */
    return s;
}

void orc_state_free(orc_state* s) {
    if (!s) return;
    free(s->chi); free(s->chit); free(s->pp); free(s->dSdchi); free(s->Phi);
    free(s->X1); free(s->R); free(s->ps); free(s->cferm); free(s);
}

void orc_state_set_remez(orc_state* s, int which, const orc_remez* r) {
    if (which == 2) s->r2 = *r;
    else if (which == 4) s->r4 = *r;
    else s->r2g = *r;
}

void orc_sweep(orc_state* st_, orc_traj_rec* rec) {
    orc_state* S = st_;
    const orc_lat* lat = &S->lat;
    const int64_t kvol = orc_kvol(lat), kferm = orc_kferm(lat);
    const int64_t Ls = lat->Ls;
    const int itermax = 1000;
    memset(rec, 0, sizeof(*rec));
    S->isweep++;
    const float proby = 1.0f / (float)S->iterl;                                 /* :164 */
    memcpy(S->chit, S->chi, sizeof(double) * 3 * kvol);                          /* :213-216 */
    /* pseudofermion heatbath (:221-245) */
    for (int f = 0; f < 2; f++)
        for (int d = 0; d < 4; d++)
            for (int64_t s = 0; s < Ls; s++) {
                orc_gauss0(&S->rng, kvol, S->ps);
                for (int64_t i = 0; i < kvol; i++) {
                    cx v = {(double)S->ps[i], (double)S->ps[kvol + i]};
                    st(S->R, SIDX(s, i, d, f), v);
                }
            }
    orc_qmrherm(lat, S->R, S->rescga, &rec->it_pf, S->am, S->hpin, S->imass, S->r4.anum,
                S->r4.aden, S->r4.n, 0, S->chit, S->X1, S->dSdchi, 5000);
    memcpy(S->Phi, S->X1, sizeof(double) * 2 * kferm);
    /* momentum heatbath (:249-257) */
    orc_gaussp(&S->rng, kvol, S->ps);
    for (int64_t i = 0; i < kvol; i++) { S->pp[i] = S->ps[i]; S->pp[i + kvol] = S->ps[kvol + i]; }
    orc_gaussp(&S->rng, kvol, S->ps);
    for (int64_t i = 0; i < kvol; i++) S->pp[i + 2 * kvol] = S->ps[i];
    /* H0 (:261-268) */
    double h[5];
    orc_hamilton(lat, S->Phi, S->rescga, S->am, S->hpin, S->imass, S->chit, S->pp, &S->r2, h,
                 S->X1, &rec->it_h0);
    rec->H0 = h[0]; rec->S0 = h[3];
    if (S->isweep == 1) S->gaction = (float)(h[1] / (double)kvol);
    rec->action = (float)(h[3] / (double)kvol);
    rec->paction = (float)(h[2] / (double)kvol);
    /* half step for p (:272-277) */
    int itg, itf;
    orc_force(lat, S->Phi, S->rescgg, S->am, S->hpin, S->imass, S->chit, &S->r2g, S->dSdchi,
              S->X1, &itg, &itf);
    rec->it_guid += itg; rec->it_force += itf; rec->nforce++;
    float d = S->dt * 0.5f;
    for (int64_t i = 0; i < 3 * kvol; i++) S->pp[i] = S->pp[i] - S->dSdchi[i] * d;
    /* MD loop (:281-315) */
    for (int iter = 1; iter <= itermax; iter++) {
        d = S->dt;
        for (int64_t i = 0; i < 3 * kvol; i++) S->chit[i] = S->chit[i] + (double)(d * S->pp[i]);
        orc_force(lat, S->Phi, S->rescgg, S->am, S->hpin, S->imass, S->chit, &S->r2g, S->dSdchi,
                  S->X1, &itg, &itf);
        rec->it_guid += itg; rec->it_force += itf; rec->nforce++;
        float ytest = orc_rano(&S->rng, &S->rng.yrun);
        rec->nsteps = iter;
        if (ytest < proby) {
            d = S->dt * 0.5f;
            for (int64_t i = 0; i < 3 * kvol; i++) S->pp[i] = S->pp[i] - d * S->dSdchi[i];
            break;
        } else {
            d = S->dt;
            for (int64_t i = 0; i < 3 * kvol; i++) S->pp[i] = S->pp[i] - d * S->dSdchi[i];
        }
    }
    /* Metropolis (:320-345) */
    orc_hamilton(lat, S->Phi, S->rescga, S->am, S->hpin, S->imass, S->chit, S->pp, &S->r2, h,
                 S->X1, &rec->it_h1);
    rec->H1 = h[0]; rec->S1 = h[3]; rec->hg = h[1]; rec->hp = h[2];
    rec->dH = rec->H0 - rec->H1;
    rec->dS = rec->S0 - rec->S1;
    rec->y = (float)exp(rec->dH);
    rec->x = orc_rano(&S->rng, &S->rng.yrun);
    rec->accepted = 0;
    if (rec->x < rec->y) {
        rec->accepted = 1;
        memcpy(S->chi, S->chit, sizeof(double) * 3 * kvol);
        rec->action = (float)(h[3] / (double)kvol);
        S->gaction = (float)(h[1] / (double)kvol);
        rec->paction = (float)(h[2] / (double)kvol);
    }
    rec->gaction = S->gaction;
    float vel2 = 0.0f;                                                           /* :349-355 */
    for (int64_t i = 0; i < 3 * kvol; i++) vel2 = vel2 + S->pp[i] * S->pp[i];
    rec->vel2 = vel2 / (float)kvol;
    /* measurements every iprint sweeps (:359-399) */
    if (S->measure && (S->isweep / S->iprint) * S->iprint == S->isweep) {
        rec->measured = 1;
        memcpy(S->chit, S->chi, sizeof(double) * 3 * kvol);
        float susctot = 0.0f, condmod = 0.0f;
        for (int a = 0; a < 3; a++) {
            float c = 0.0f;
            for (int64_t i = 0; i < kvol; i++) c = (float)((double)c + S->chi[i + kvol * a]);
            float su = c * c;
            c = c / (float)kvol;
            condmod = condmod + c * c;
            su = su / (float)kvol;
            susctot = susctot + su;
            rec->cond[a] = c; rec->susc[a] = su;
        }
        rec->condmod = sqrtf(condmod);
        rec->susctot = susctot;
        rec->ancgm = orc_fermion(lat, &S->rng, S->rescgm, S->am, S->hpin, S->imass, S->chit,
                                 S->X1, S->cferm, S->cferm + 2 * 2 * lat->Lt);
    }
}

int orc_read_remez(const char* path, int n, orc_remez* r) {
    FILE* fp = fopen(path, "r");
    if (!fp) return -1;
    char line[512];
    double v[2 * 64 + 2][2];
    int cnt = 0;
    while (fgets(line, sizeof line, fp) && cnt < 2 * 64 + 2) {
        char* c = line;
        for (char* q = c; *q; q++) if (*q == ',' || *q == 'd' || *q == 'D') *q = (*q == ',') ? ' ' : 'e';
        double a = 0, b = 0;
        int k = sscanf(c, "%lf %lf", &a, &b);
        if (k <= 0) continue;
        v[cnt][0] = a; v[cnt][1] = b;
        cnt++;
    }
    fclose(fp);
    if (cnt < 2 * n + 2) return -2;
    r->n = n;
    r->anum[0] = v[0][0];
    for (int k = 1; k <= n; k++) { r->anum[k] = v[k][0]; r->aden[k - 1] = v[k][1]; }
    r->bnum[0] = v[n + 1][0];
    for (int k = 1; k <= n; k++) { r->bnum[k] = v[n + 1 + k][0]; r->bden[k - 1] = v[n + 1 + k][1]; }
    return 0;
}
