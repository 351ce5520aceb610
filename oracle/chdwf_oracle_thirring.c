/*
 * chdwf_oracle_thirring.c -- CPU oracle for the bulk Thirring RHMC code,
 * bulk_rhmc.f (j-ostmeyer/chiralHeisenberg).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path in
 * chiralheisenberg_b200/csrc/thirring.cu; nothing in the product library
 * links, loads or calls it.
 *
 * bulk_rhmc.f is the domain-wall RHMC for the Thirring model: one flavour of
 * 4-component spinors R(kthird,kvol,4) (complex*16), non-compact U(1) link
 * angles theta(kvol,3) (REAL*4) entering the hops through u = 1 + i*theta
 * with the antiperiodic sign folded into the last time slice (coef), a mass
 * term am on the walls, and a Pauli-Villars determinant at mass 1.  The
 * file has no OpenMP, so every sum runs in loop order.  Undeclared
 * variables are REAL*4 by implicit typing: in qmrherm alphatild, beta0,
 * phimod, rhomax, resid; in derivs the force dSdpi; and tzi =
 * cmplx(0.0, 2*anum) is default-kind, so 2*anum is rounded to REAL*4.
 * Compiled with -ffp-contract=off like the reference (gfortran without
 * -march, no fused multiply-add).
 *
 * Layouts, 0-based: spinor R(s, site, d) -> s + Ls*(site + kvol*d),
 * site = x + L*(y + L*t), complex128 (re, im) pairs; theta, pp, dSdpi
 * (site, mu) -> site + kvol*mu (REAL*4); u(site, mu) complex128.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "chdwf_oracle.h"

typedef struct { double re, im; } zc;

static inline zc zld(const double* v, int64_t j) { zc r = {v[2 * j], v[2 * j + 1]}; return r; }
static inline void zst(double* v, int64_t j, zc a) { v[2 * j] = a.re; v[2 * j + 1] = a.im; }
static inline zc zadd(zc a, zc b) { zc r = {a.re + b.re, a.im + b.im}; return r; }
static inline zc zsub(zc a, zc b) { zc r = {a.re - b.re, a.im - b.im}; return r; }
static inline zc zmul(zc a, zc b) {
    zc r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}
static inline zc zscal(double s, zc a) { zc r = {s * a.re, s * a.im}; return r; }
static inline zc zconj(zc a) { zc r = {a.re, -a.im}; return r; }

#define TIDX(s, site, d) ((int64_t)(s) + Ls * ((int64_t)(site) + kvol * (int64_t)(d)))

/* gamval(mu,idirac)*akappa, gamin(mu,idirac) - 1 (bulk_rhmc.f:1646-1722, scaled by akappa at :1720) */
static const double kTGv[3][4][2] = {{{0., -0.5}, {0., -0.5}, {0., 0.5}, {0., 0.5}},
                                     {{-0.5, 0.}, {0.5, 0.}, {0.5, 0.}, {-0.5, 0.}},
                                     {{0., -0.5}, {0., 0.5}, {0., 0.5}, {0., -0.5}}};
static const int kTGi[3][4] = {{3, 2, 1, 0}, {3, 2, 1, 0}, {2, 3, 0, 1}};

/* iu(i,mu), id(i,mu) of addrc (:1746-1797): periodic neighbours */
static int64_t nbr(const orc_lat* lat, int64_t i, int mu, int up) {
    const int L = lat->L, Lt = lat->Lt;
    int x = (int)(i % L), y = (int)((i / L) % L), t = (int)(i / ((int64_t)L * L));
    const int dlt = up ? 1 : -1;
    if (mu == 0) x = (x + dlt + L) % L;
    else if (mu == 1) y = (y + dlt + L) % L;
    else t = (t + dlt + Lt) % Lt;
    return x + (int64_t)L * (y + (int64_t)L * t);
}

/* coef (:1799-1827): u = 1 + i*theta, the last time slice of u(.,3) negated */
void orc_thr_coef(const orc_lat* lat, const float* theta, double* u) {
    const int64_t kvol = orc_kvol(lat), kvol2 = (int64_t)lat->L * lat->L;
    for (int64_t j = 0; j < 3 * kvol; j++) {
        u[2 * j] = 1.0;
        u[2 * j + 1] = (double)theta[j];
    }
    if (lat->ibound == -1)
        for (int64_t i = (int64_t)(lat->Lt - 1) * kvol2; i < kvol; i++) {
            u[2 * (i + 2 * kvol)] = -u[2 * (i + 2 * kvol)];
            u[2 * (i + 2 * kvol) + 1] = -u[2 * (i + 2 * kvol) + 1];
        }
}

/* Phi = M R (dag 0, :1946-2069) or M^dagger R (dag 1, :2071-2188) */
void orc_thr_dslash(const orc_lat* lat, double* Phi, const double* R, const double* u, float am,
                    int imass, int dag) {
    const int64_t Ls = lat->Ls, kvol = orc_kvol(lat), kferm = 4 * kvol * Ls;
    const float akappa = 0.5f;
    const float diag = (3.0f - lat->am3) + 1.0f;                              /* :1967, :2092 */
    for (int64_t j = 0; j < kferm; j++) zst(Phi, j, zscal((double)diag, zld(R, j)));
    /* Wilson term (:1976-1987, :2101-2112) */
    for (int mu = 0; mu < 3; mu++)
        for (int d = 0; d < 4; d++)
            for (int64_t i = 0; i < kvol; i++) {
                const int64_t up = nbr(lat, i, mu, 1), dn = nbr(lat, i, mu, 0);
                const zc uu = zld(u, i + kvol * mu), ud = zconj(zld(u, dn + kvol * mu));
                for (int64_t s = 0; s < Ls; s++) {
                    const int64_t o = TIDX(s, i, d);
                    zc w = zadd(zmul(uu, zld(R, TIDX(s, up, d))), zmul(ud, zld(R, TIDX(s, dn, d))));
                    zst(Phi, o, zsub(zld(Phi, o), zscal((double)akappa, w)));
                }
            }
    /* Dirac term: M adds gamval*(...), M^dagger subtracts it (:1989-2002, :2114-2127) */
    for (int mu = 0; mu < 3; mu++)
        for (int d = 0; d < 4; d++) {
            const int dg = kTGi[mu][d];
            const zc g = {kTGv[mu][d][0], kTGv[mu][d][1]};
            for (int64_t i = 0; i < kvol; i++) {
                const int64_t up = nbr(lat, i, mu, 1), dn = nbr(lat, i, mu, 0);
                const zc uu = zld(u, i + kvol * mu), ud = zconj(zld(u, dn + kvol * mu));
                for (int64_t s = 0; s < Ls; s++) {
                    const int64_t o = TIDX(s, i, d);
                    zc t = zmul(g, zsub(zmul(uu, zld(R, TIDX(s, up, dg))),
                                        zmul(ud, zld(R, TIDX(s, dn, dg)))));
                    zst(Phi, o, dag ? zsub(zld(Phi, o), t) : zadd(zld(Phi, o), t));
                }
            }
        }
    /* s hops: M takes Dirac 3,4 from s+1, Dirac 1,2 from s-1 (:2004-2020);
     * M^dagger the reverse (:2129-2145) */
    const int up0 = dag ? 0 : 2, dn0 = dag ? 2 : 0;
    for (int d = up0; d < up0 + 2; d++)
        for (int64_t i = 0; i < kvol; i++)
            for (int64_t s = 0; s < Ls - 1; s++) {
                const int64_t o = TIDX(s, i, d);
                zst(Phi, o, zsub(zld(Phi, o), zld(R, TIDX(s + 1, i, d))));
            }
    for (int d = dn0; d < dn0 + 2; d++)
        for (int64_t s = 0; s < Ls - 1; s++)
            for (int64_t i = 0; i < kvol; i++) {
                const int64_t o = TIDX(s + 1, i, d);
                zst(Phi, o, zsub(zld(Phi, o), zld(R, TIDX(s, i, d))));
            }
    /* mass term (:2022-2067, :2147-2186); zkappa = cmplx(am,0) for imass 1,
     * cmplx(0,-am) (M) or cmplx(0,am) (M^dagger) for imass 3 and 5.  Group A
     * is written at s=kthird (M: Dirac 3,4; M^dagger: Dirac 1,2), group B at
     * s=1 (the other pair). */
    const int64_t sL = Ls - 1;
    zc zk;
    if (imass == 1) { zk.re = (double)am; zk.im = 0.0; }
    else { zk.re = 0.0; zk.im = dag ? (double)am : (double)(-am); }
    for (int grp = 0; grp < 2; grp++) {
        const int d0 = (grp == 0) == (dag == 0) ? 2 : 0;
        const int64_t sw = grp == 0 ? sL : 0;
        for (int d = d0; d < d0 + 2; d++)
            for (int64_t i = 0; i < kvol; i++) {
                const int64_t o = TIDX(sw, i, d);
                int sg;
                int64_t src;
                if (imass == 5) {
                    /* the other Dirac pair on the same wall, always subtracted */
                    src = TIDX(sw, i, d >= 2 ? d - 2 : d + 2);
                    sg = -1;
                } else {
                    src = TIDX(grp == 0 ? 0 : sL, i, d);
                    if (imass == 1) sg = 1;
                    else sg = (grp == 0) == (dag == 0) ? -1 : 1;   /* M: A -, B + ; M^dag: A +, B - */
                }
                const zc t = zmul(zk, zld(R, src));
                zst(Phi, o, sg > 0 ? zadd(zld(Phi, o), t) : zsub(zld(Phi, o), t));
            }
    }
}

/* derivs (:820-878): dSdpi -= akappa*Re(tzi*(R^dag(x) X2(x+mu) - R^dag(x+mu) X2(x)))
 * and -/+ Re(tzi*gamval*(R^dag(x) X2(x+mu,gamin) + R^dag(x+mu) X2(x,gamin)))
 * for iflag 0/1, tzi = cmplx(0, 2*anum) in REAL*4, dSdpi REAL*4. */
void orc_thr_derivs(const orc_lat* lat, const double* R, const double* X2, double anum,
                    int iflag, float* dSdpi) {
    const int64_t Ls = lat->Ls, kvol = orc_kvol(lat);
    const double akappa = (double)0.5f;
    const zc tzi = {0.0, (double)(float)(2.0 * anum)};                       /* :839 */
    for (int mu = 0; mu < 3; mu++)
        for (int d = 0; d < 4; d++)
            for (int64_t s = 0; s < Ls; s++) {
                for (int64_t i = 0; i < kvol; i++) {                            /* :843-850 */
                    const int64_t up = nbr(lat, i, mu, 1);
                    const zc a = zmul(zconj(zld(R, TIDX(s, i, d))), zld(X2, TIDX(s, up, d)));
                    const zc b = zmul(zconj(zld(R, TIDX(s, up, d))), zld(X2, TIDX(s, i, d)));
                    const zc t = zmul(tzi, zsub(a, b));
                    float* f = &dSdpi[i + kvol * mu];
                    *f = (float)((double)*f - akappa * t.re);
                }
                const int dg = kTGi[mu][d];
                const zc g = {kTGv[mu][d][0], kTGv[mu][d][1]};
                const zc tg = zmul(tzi, g);
                for (int64_t i = 0; i < kvol; i++) {                            /* :851-868 */
                    const int64_t up = nbr(lat, i, mu, 1);
                    const zc a = zmul(zconj(zld(R, TIDX(s, i, d))), zld(X2, TIDX(s, up, dg)));
                    const zc b = zmul(zconj(zld(R, TIDX(s, up, d))), zld(X2, TIDX(s, i, dg)));
                    const zc t = zmul(tg, zadd(a, b));
                    float* f = &dSdpi[i + kvol * mu];
                    *f = iflag == 0 ? (float)((double)*f - t.re) : (float)((double)*f + t.re);
                }
            }
}

/* qmrherm (:630-818): multi-shift Lanczos for (M^dag M + aden_k) x_k = Phi
 * on the operator of mass (am, imass).  iflag 0: x = anum0 Phi + sum anum_k
 * x_k; 1: also Phi0_k = x_k; 2: the DWF force, derivs(x_k, M x_k, anum_k, 0)
 * per pole; 3: the PV force, with coeff = -anum_k, derivs(Phi0_k, M x_k, 0)
 * then derivs(M Phi0_k, x_k, 1).  Phi0: ndiag*kferm complex, dSdpi: the force
 * accumulated into.  Returns 1 at the cap niterc = 7500. */
/* How qmrherm forms alphatild, a REAL*4 variable by implicit typing
 * (bulk_rhmc.f:691-694).  0 (default): as the reference, element by element
 * with the REAL*4 sum rounded after every addition.  1: the sum in REAL*8,
 * rounded to REAL*4 once -- the grouping a parallel reduction (the GPU's)
 * can follow, so the GPU is compared with the same arithmetic; the
 * difference between the two is the reference's own REAL*4 accumulation
 * error, tested on the CPU. */
static int g_alphatild_fp64 = 0;
void orc_thr_set_alphatild_fp64(int on) { g_alphatild_fp64 = on != 0; }

int orc_thr_qmrherm(const orc_lat* lat, const double* Phi, float res, int* itercg, float am,
                    int imass, const double* anum, const double* aden, int ndiag, int iflag,
                    const double* u, double* x, double* Phi0, float* dSdpi) {
    const int64_t kvol = orc_kvol(lat), kferm = 4 * kvol * lat->Ls;
    const int niterc = 7500;                                                 /* :635 */
    const size_t vb = sizeof(double) * 2 * kferm;
    double* R = malloc(vb);
    double* qm1 = calloc(2 * kferm, sizeof(double));
    double* q = malloc(vb);
    double* vt = malloc(vb);
    double* x3 = malloc(vb);
    double* p = malloc(vb * ndiag);
    double* pm1 = malloc(vb * ndiag);
    double* x1 = malloc(vb * ndiag);
    double alpha[32], amu[32], d[32], dm1[32], rho[32], rhom1[32];
    const float resid = sqrtf((float)kferm * res * res);                    /* :660 */
    *itercg = 0;
    memcpy(R, Phi, vb);                                                      /* :662-667 */
    for (int64_t i = 0; i < kferm; i++) zst(x, i, zscal(anum[0], zld(Phi, i)));
    double beta = 0.0;
    for (int64_t i = 0; i < kferm; i++) beta = beta + zmul(zconj(zld(R, i)), zld(R, i)).re;
    beta = sqrt(beta);
    const float phimod = (float)beta;
    int capped = 1;
    for (int niter = 1; niter <= niterc; niter++) {                          /* :679 */
        (*itercg)++;
        for (int64_t i = 0; i < kferm; i++) {                                /* q = R/beta, :684-686 */
            q[2 * i] = R[2 * i] / beta;
            q[2 * i + 1] = R[2 * i + 1] / beta;
        }
        orc_thr_dslash(lat, vt, q, u, am, imass, 0);
        orc_thr_dslash(lat, x3, vt, u, am, imass, 1);
        float alphatild = 0.0f;                                              /* :691-694 */
        if (g_alphatild_fp64) {
            /* the GPU's grouping: the sum in REAL*8, rounded to REAL*4 once */
            double a8 = 0.0;
            for (int64_t i = 0; i < kferm; i++) a8 += zmul(zconj(zld(q, i)), zld(x3, i)).re;
            alphatild = (float)a8;
        } else {
            for (int64_t i = 0; i < kferm; i++)
                alphatild = (float)((double)alphatild + zmul(zconj(zld(q, i)), zld(x3, i)).re);
        }
        for (int64_t i = 0; i < kferm; i++) {                                /* :696-699 */
            zst(R, i, zsub(zsub(zld(x3, i), zscal((double)alphatild, zld(q, i))),
                           zscal(beta, zld(qm1, i))));
            zst(qm1, i, zld(q, i));
        }
        const float beta0 = (float)beta;
        beta = 0.0;
        for (int64_t i = 0; i < kferm; i++) beta = beta + zmul(zconj(zld(R, i)), zld(R, i)).re;
        beta = sqrt(beta);
        for (int k = 0; k < ndiag; k++) alpha[k] = (double)alphatild + aden[k];
        if (niter == 1) {                                                    /* :712-724 */
            for (int k = 0; k < ndiag; k++) {
                d[k] = alpha[k];
                memcpy(p + 2 * kferm * k, q, vb);
                memcpy(pm1 + 2 * kferm * k, q, vb);
                rho[k] = (double)beta0 / alpha[k];
                rhom1[k] = rho[k];
                for (int64_t i = 0; i < kferm; i++)
                    zst(x1 + 2 * kferm * k, i, zscal(rho[k], zld(q, i)));
            }
        } else {                                                             /* :725-747 */
            float rhomax = 0.0f;
            for (int k = 0; k < ndiag; k++) {
                double* pk = p + 2 * kferm * k;
                double* pmk = pm1 + 2 * kferm * k;
                double* xk = x1 + 2 * kferm * k;
                amu[k] = (double)beta0 / d[k];
                dm1[k] = d[k];
                d[k] = alpha[k] - (double)beta0 * amu[k];
                for (int64_t i = 0; i < kferm; i++) {
                    zst(pk, i, zsub(zld(q, i), zscal(amu[k], zld(pmk, i))));
                    zst(pmk, i, zld(pk, i));
                }
                rho[k] = -(amu[k] * dm1[k] * rhom1[k] / d[k]);
                const double rm = fabs((double)phimod * rho[k]);
                if (k == 0) rhomax = (float)rm;
                else if (rm > (double)rhomax) rhomax = (float)rm;
                rhom1[k] = rho[k];
                for (int64_t i = 0; i < kferm; i++)
                    zst(xk, i, zadd(zld(xk, i), zscal(rho[k], zld(pk, i))));
            }
            const float arelax = 2.0f;                                       /* :750-757 */
            if (rhomax < arelax * resid) { capped = 0; break; }
        }
    }
    if (iflag < 2) {                                                         /* :766-780 */
        for (int k = 0; k < ndiag; k++)
            for (int64_t i = 0; i < kferm; i++)
                zst(x, i, zadd(zld(x, i), zscal(anum[k + 1], zld(x1 + 2 * kferm * k, i))));
        if (iflag == 1) memcpy(Phi0, x1, vb * ndiag);
    } else {                                                                 /* :781-806 */
        double* X2 = vt;
        for (int k = 0; k < ndiag; k++) {
            const double* xk = x1 + 2 * kferm * k;
            orc_thr_dslash(lat, X2, xk, u, am, imass, 0);
            if (iflag == 2) {
                orc_thr_derivs(lat, xk, X2, anum[k + 1], 0, dSdpi);
            } else {
                const double coeff = -anum[k + 1];
                const double* p0 = Phi0 + 2 * kferm * k;
                orc_thr_derivs(lat, p0, X2, coeff, 0, dSdpi);
                orc_thr_dslash(lat, X2, p0, u, am, imass, 0);
                orc_thr_derivs(lat, X2, xk, coeff, 1, dSdpi);
            }
        }
    }
    free(R); free(qm1); free(q); free(vt); free(x3); free(p); free(pm1); free(x1);
    return capped;
}

/* force (:449-535): dSdpi of the pseudofermion action
 * Phi^dag {M^dag M(1)}^1/4 {M^dag M(m)}^-1/2 {M^dag M(1)}^1/4 Phi with the
 * guidance sets r2g (mass m) and r4g (Pauli-Villars, mass 1), then the
 * antiperiodic sign on the t links of the last slice and beta*theta. */
void orc_thr_force(orc_thr_state* st, float res1, int* its) {
    const orc_lat* lat = &st->lat;
    const int64_t kvol = orc_kvol(lat), kferm = 4 * kvol * lat->Ls;
    const int64_t kvol2 = (int64_t)lat->L * lat->L;
    const size_t vb = sizeof(double) * 2 * kferm;
    double* X2 = malloc(vb);
    memset(st->dSdpi, 0, sizeof(float) * 3 * kvol);                          /* :477-481 */
    const orc_remez* a4 = &st->r4g;
    const orc_remez* r2 = &st->r2g;
    orc_thr_qmrherm(lat, st->Phi, res1, &its[0], 1.0f, 1, a4->anum, a4->aden, a4->n, 1, st->ut,
                    st->X1, st->Phi0, st->dSdpi);                             /* :493 */
    memcpy(X2, st->X1, vb);
    orc_thr_qmrherm(lat, X2, res1, &its[1], st->am, st->imass, r2->bnum, r2->bden, r2->n, 0,
                    st->ut, st->X1, st->Phi0, st->dSdpi);                     /* :500 */
    memcpy(X2, st->X1, vb);
    orc_thr_qmrherm(lat, X2, res1, &its[2], st->am, st->imass, r2->anum, r2->aden, r2->n, 2,
                    st->ut, st->X1, st->Phi0, st->dSdpi);                     /* :509 */
    orc_thr_qmrherm(lat, X2, res1, &its[3], 1.0f, 1, a4->anum, a4->aden, a4->n, 3, st->ut,
                    st->X1, st->Phi0, st->dSdpi);                             /* :514 */
    if (lat->ibound == -1)                                                   /* :520-525 */
        for (int64_t i = (int64_t)(lat->Lt - 1) * kvol2; i < kvol; i++)
            st->dSdpi[i + 2 * kvol] = -st->dSdpi[i + 2 * kvol];
    const float b = lat->beta * 1.0f;                                        /* b = beta*Nf, :527-532 */
    for (int64_t j = 0; j < 3 * kvol; j++) st->dSdpi[j] = st->dSdpi[j] + b * st->thetat[j];
    free(X2);
}

/* hamilton (:539-628): h = hg + hp + hf, hp = 0.5 sum pp^2, hg = 0.5*beta
 * sum theta^2, hf = Re Phi'^dag X1 from the PV solve (r4, mass 1) then the
 * r2 b-set solve at mass m.  out: h, hg, hp, s = hg + hf. */
void orc_thr_hamilton(orc_thr_state* st, float res2, double* out, int* its) {
    const orc_lat* lat = &st->lat;
    const int64_t kvol = orc_kvol(lat), kferm = 4 * kvol * lat->Ls;
    const size_t vb = sizeof(double) * 2 * kferm;
    double hp = 0.0, hg = 0.0, hf = 0.0;
    for (int64_t j = 0; j < 3 * kvol; j++) hp = hp + (double)(st->pp[j] * st->pp[j]);   /* :571-574 */
    hp = hp * 0.5;
    for (int64_t j = 0; j < 3 * kvol; j++) hg = hg + (double)(st->thetat[j] * st->thetat[j]);
    hg = (double)(0.5f * 1.0f * lat->beta) * hg;                            /* :581 */
    double* R = malloc(vb);
    memcpy(R, st->Phi, vb);                                                  /* :593-596 */
    orc_thr_qmrherm(lat, R, res2, &its[0], 1.0f, 1, st->r4.anum, st->r4.aden, st->r4.n, 0, st->ut,
                    st->X1, st->Phi0, st->dSdpi);
    memcpy(R, st->X1, vb);
    orc_thr_qmrherm(lat, R, res2, &its[1], st->am, st->imass, st->r2.bnum, st->r2.bden, st->r2.n,
                    0, st->ut, st->X1, st->Phi0, st->dSdpi);                 /* :603 */
    for (int64_t j = 0; j < kferm; j++)                                      /* :607-609 */
        hf = hf + zmul(zconj(zld(R, j)), zld(st->X1, j)).re;
    free(R);
    out[0] = hg + hp + hf;
    out[1] = hg;
    out[2] = hp;
    out[3] = hg + hf;
}

/* congrad (:931-1025): CGNE on M^dagger M, FP64 vectors with REAL*4 scalars;
 * alphad and betan take each complex*16 term and round to REAL*4.  x: in =
 * initial guess (/vector/), out = solution.  Returns 1 at the cap
 * niterc = kthird*kvol. */
int orc_thr_congrad(const orc_lat* lat, const double* Phi, float res, int* itercg, float am,
                    int imass, const double* u, double* x) {
    const int64_t kvol = orc_kvol(lat), kferm = 4 * kvol * lat->Ls;
    const int64_t niterc = lat->Ls * kvol;                                  /* :934 */
    const size_t vb = sizeof(double) * 2 * kferm;
    double* x1 = malloc(vb);
    double* x2 = malloc(vb);
    double* p = malloc(vb);
    double* r = malloc(vb);
    const float resid = (float)kferm * res * res;                           /* :947 */
    float betad = 1.0f, alpha = 1.0f, alphan = 0.0f;
    int capped = 1;
    *itercg = 0;
    for (int64_t nx = 1; nx <= niterc; nx++) {
        (*itercg)++;
        if (nx == 1) {                                                       /* :951-962 */
            memcpy(p, x, vb);
            memcpy(r, Phi, vb);
            betad = 1.0f;
            alpha = 1.0f;
        }
        orc_thr_dslash(lat, x1, p, u, am, imass, 0);                         /* :966 */
        if (nx != 1) {                                                       /* :970-983 */
            float alphad = 0.0f;
            for (int64_t i = 0; i < kferm; i++)
                alphad = (float)((double)alphad + zmul(zconj(zld(x1, i)), zld(x1, i)).re);
            alpha = alphan / alphad;
            for (int64_t i = 0; i < kferm; i++)
                zst(x, i, zadd(zld(x, i), zscal((double)alpha, zld(p, i))));
        }
        orc_thr_dslash(lat, x2, x1, u, am, imass, 1);                        /* :987 */
        for (int64_t i = 0; i < kferm; i++) zst(r, i, zsub(zld(r, i), zscal((double)alpha, zld(x2, i))));
        float betan = 0.0f;                                                  /* :996-1001 */
        for (int64_t i = 0; i < kferm; i++)
            betan = (float)((double)betan + zmul(zconj(zld(r, i)), zld(r, i)).re);
        float beta = betan / betad;
        betad = betan;
        alphan = betan;
        if (nx == 1) beta = 0.0f;
        for (int64_t i = 0; i < kferm; i++) zst(p, i, zadd(zld(r, i), zscal((double)beta, zld(p, i))));
        if (betan < resid) { capped = 0; break; }
    }
    free(x1); free(x2); free(p); free(r);
    return capped;
}

/* measure (:1027-1285): the noisy psibar psi estimator, knoise = 10 noise
 * vectors (two gauss0 calls each); per noise and Dirac source 1, 2 a
 * source on the s=1 wall and one on the s=kthird wall (imass 5: the other
 * chirality, negated), Phi = M^dagger xi, congrad from the source itself as
 * initial guess, and the overlap with the opposite wall.  pbp is REAL*8;
 * psibarpsi and susclsing REAL*4.  parts (40 doubles or NULL): re/im of
 * psibarpsi1 and psibarpsi2 per noise (the unit-100 records). */
void orc_thr_measure(const orc_lat* lat, orc_rng* g, float res, float am, int imass,
                     const double* u, float* psibarpsi, float* susclsing, float* aviter,
                     double* parts) {
    const int64_t Ls = lat->Ls, kvol = orc_kvol(lat), kferm = 4 * kvol * Ls;
    enum { knoise = 10 };
    float* ps = malloc(sizeof(float) * 2 * kvol);
    float* pt = malloc(sizeof(float) * 2 * kvol);
    double* xi = malloc(sizeof(double) * 2 * kferm);
    double* Phi = malloc(sizeof(double) * 2 * kferm);
    double pbp[knoise];
    int iter = 0;
    for (int inoise = 0; inoise < knoise; inoise++) {
        orc_gauss0(g, kvol, ps);                                             /* :1061 */
        orc_gauss0(g, kvol, pt);                                             /* :1063 */
        zc p1 = {0.0, 0.0}, p2 = {0.0, 0.0};
        for (int idsource = 1; idsource <= 2; idsource++) {
            for (int w = 0; w < 2; w++) {
                /* w=0: ps on s=1 (:1066-1156); w=1: pt on s=kthird (:1157-1241).
                 * dn: Dirac index of the noise x; dsrc: component of xi set;
                 * sgn: -1 for the gamma_5 sources of imass 5. */
                const float* nz = w == 0 ? ps : pt;
                int dn, dsrc;
                double sgn = 1.0;
                if (imass != 5) {
                    dn = w == 0 ? idsource : idsource + 2;
                    dsrc = dn;
                } else {
                    dn = w == 0 ? idsource + 2 : idsource;
                    dsrc = w == 0 ? dn - 2 : dn + 2;
                    sgn = -1.0;
                }
                const int64_t s_src = w == 0 ? 0 : Ls - 1;
                memset(xi, 0, sizeof(double) * 2 * kferm);
                for (int64_t i = 0; i < kvol; i++) {
                    zc x = {(double)nz[i], (double)nz[kvol + i]};
                    if (sgn < 0) { x.re = -x.re; x.im = -x.im; }
                    zst(xi, TIDX(s_src, i, dsrc - 1), x);
                }
                orc_thr_dslash(lat, Phi, xi, u, am, imass, 1);              /* :1136, :1220 */
                int it = 0;
                orc_thr_congrad(lat, Phi, res, &it, am, imass, u, xi);      /* :1138, :1225 */
                iter += it;
                /* read: imass != 5 the noise component on the opposite wall;
                 * imass 5 the noise component on the same wall */
                const int64_t s_rd = imass != 5 ? (w == 0 ? Ls - 1 : 0) : s_src;
                zc acc = w == 0 ? p1 : p2;
                for (int64_t i = 0; i < kvol; i++) {
                    const zc x = {(double)nz[i], (double)nz[kvol + i]};
                    acc = zadd(acc, zmul(zconj(x), zld(xi, TIDX(s_rd, i, dn - 1))));
                }
                if (w == 0) p1 = acc; else p2 = acc;
            }
        }
        const double kv = (double)kvol;
        if (imass == 1) {                                                    /* :1245-1257 */
            p1.re /= kv; p1.im /= kv; p2.re /= kv; p2.im /= kv;
        } else {
            const zc m1 = {0.0, -1.0}, s2 = {0.0, imass == 3 ? 1.0 : -1.0};
            p1 = zmul(m1, p1); p1.re /= kv; p1.im /= kv;
            p2 = zmul(s2, p2); p2.re /= kv; p2.im /= kv;
        }
        pbp[inoise] = p1.re + p2.re;
        if (parts) {
            parts[4 * inoise] = p1.re; parts[4 * inoise + 1] = p1.im;
            parts[4 * inoise + 2] = p2.re; parts[4 * inoise + 3] = p2.im;
        }
    }
    float pb = 0.0f, sus = 0.0f;                                             /* :1266-1276 */
    for (int i = 0; i < knoise; i++) {
        pb = (float)((double)pb + pbp[i]);
        for (int j = knoise - 1; j >= i + 1; j--) sus = (float)((double)sus + pbp[i] * pbp[j]);
    }
    *psibarpsi = pb / (float)knoise;
    *susclsing = (float)(2 * kvol) * sus / (float)(knoise * (knoise - 1));
    *aviter = (float)iter / (float)(4 * knoise);                             /* :1278 */
    free(ps); free(pt); free(xi); free(Phi);
}

/* ---- program dwf3d of bulk_rhmc.f (:201-400) ----------------------------- */
orc_thr_state* orc_thr_new(int L, int Lt, int Ls, float beta, float am3, float dt, float am,
                           int imass, int iterl) {
    orc_thr_state* s = calloc(1, sizeof(*s));
    s->lat.L = L; s->lat.Lt = Lt; s->lat.Ls = Ls;
    s->lat.beta = beta; s->lat.am3 = am3; s->lat.ibound = -1; s->lat.threads = 1;
    s->dt = dt; s->am = am; s->imass = imass; s->iterl = iterl; s->iprint = 5;
    s->rescga = 0.000000001f; s->rescgg = 0.000001f;                         /* :39 */
    const int64_t kvol = (int64_t)L * L * Lt, kferm = 4 * kvol * Ls;
    s->theta = calloc(3 * kvol, sizeof(float));
    s->thetat = calloc(3 * kvol, sizeof(float));
    s->pp = calloc(3 * kvol, sizeof(float));
    s->dSdpi = calloc(3 * kvol, sizeof(float));
    s->ut = calloc(6 * kvol, sizeof(double));
    s->Phi = calloc(2 * kferm, sizeof(double));
    s->X1 = calloc(2 * kferm, sizeof(double));
    s->R = calloc(2 * kferm, sizeof(double));
    s->Phi0 = calloc(2 * kferm * 25, sizeof(double));
    s->ps = calloc(2 * kvol, sizeof(float));
    orc_rng_startup(&s->rng, 693764523745.0);
    return s;
}

void orc_thr_free(orc_thr_state* s) {
    if (!s) return;
    free(s->theta); free(s->thetat); free(s->pp); free(s->dSdpi); free(s->ut);
    free(s->Phi); free(s->X1); free(s->R); free(s->Phi0); free(s->ps);
    free(s);
}

void orc_thr_set_remez(orc_thr_state* st, int which, const orc_remez* r) {
    if (which == 2) st->r2 = *r;
    else if (which == 4) st->r4 = *r;
    else if (which == 22) st->r2g = *r;
    else if (which == 44) st->r4g = *r;
}

/* One sweep, with measure on every iprint-th sweep (:360-374). */
void orc_thr_sweep(orc_thr_state* st, orc_thr_rec* rec) {
    const orc_lat* lat = &st->lat;
    const int64_t Ls = lat->Ls, kvol = orc_kvol(lat), kferm = 4 * kvol * Ls;
    const size_t vb = sizeof(double) * 2 * kferm;
    memset(rec, 0, sizeof(*rec));
    st->isweep++;
    memcpy(st->thetat, st->theta, sizeof(float) * 3 * kvol);                /* :203-208 */
    orc_thr_coef(lat, st->thetat, st->ut);
    for (int d = 0; d < 4; d++)                                              /* :213-222 */
        for (int64_t s = 0; s < Ls; s++) {
            orc_gauss0(&st->rng, kvol, st->ps);
            for (int64_t i = 0; i < kvol; i++) {
                zc v = {(double)st->ps[i], (double)st->ps[kvol + i]};
                zst(st->R, TIDX(s, i, d), v);
            }
        }
    int it = 0;
    orc_thr_qmrherm(lat, st->R, st->rescga, &it, st->am, st->imass, st->r4.anum, st->r4.aden,
                    st->r4.n, 0, st->ut, st->X1, st->Phi0, st->dSdpi);       /* :226 */
    rec->it_pf = it;
    memcpy(st->R, st->X1, vb);
    orc_thr_qmrherm(lat, st->R, st->rescga, &it, 1.0f, 1, st->r4.bnum, st->r4.bden, st->r4.n, 0,
                    st->ut, st->X1, st->Phi0, st->dSdpi);                     /* :236 */
    rec->it_pfpv = it;
    memcpy(st->Phi, st->X1, vb);
    for (int mu = 0; mu < 3; mu++) {                                         /* :255-260 */
        orc_gaussp(&st->rng, kvol, st->ps);
        memcpy(st->pp + kvol * mu, st->ps, sizeof(float) * kvol);
    }
    double h[4];
    int ih[2], fi[4];
    orc_thr_hamilton(st, st->rescga, h, ih);                                /* :265 */
    rec->it_h0 = ih[1];
    rec->it_h0pv = ih[0];
    rec->H0 = h[0];
    rec->S0 = h[3];
    if (st->isweep == 1) {                                                   /* :267-271 */
        st->action = (float)(h[3] / (double)kvol);
        st->gaction = (float)(h[1] / (double)kvol);
        st->paction = (float)(h[2] / (double)kvol);
    }
    orc_thr_force(st, st->rescgg, fi);                                      /* :276 */
    for (int k = 0; k < 4; k++) rec->it_force[k] += fi[k];
    rec->nforce++;
    float dd = st->dt * 0.5f;
    for (int64_t j = 0; j < 3 * kvol; j++) st->pp[j] = st->pp[j] - st->dSdpi[j] * dd;
    const float proby = 1.0f / (float)st->iterl;                             /* :151 */
    for (int iter = 1; iter <= 1000; iter++) {                               /* :285-320 */
        dd = st->dt;
        for (int64_t j = 0; j < 3 * kvol; j++) st->thetat[j] = st->thetat[j] + dd * st->pp[j];
        orc_thr_coef(lat, st->thetat, st->ut);
        orc_thr_force(st, st->rescgg, fi);
        for (int k = 0; k < 4; k++) rec->it_force[k] += fi[k];
        rec->nforce++;
        rec->nsteps = iter;
        const float ytest = orc_rano(&st->rng, &st->rng.yran);              /* :302 */
        if (ytest < proby) {
            dd = st->dt * 0.5f;
            for (int64_t j = 0; j < 3 * kvol; j++) st->pp[j] = st->pp[j] - dd * st->dSdpi[j];
            st->itot = st->itot + iter;
            break;
        }
        dd = st->dt;
        for (int64_t j = 0; j < 3 * kvol; j++) st->pp[j] = st->pp[j] - dd * st->dSdpi[j];
    }
    orc_thr_hamilton(st, st->rescga, h, ih);                                /* :325 */
    rec->it_h1 = ih[1];
    rec->it_h1pv = ih[0];
    rec->H1 = h[0];
    rec->S1 = h[3];
    rec->hg = h[1];
    rec->hp = h[2];
    rec->dH = rec->H0 - rec->H1;
    rec->dS = rec->S0 - rec->S1;
    rec->y = (float)exp(rec->dH);                                            /* :330 */
    st->yav = st->yav + rec->y;
    st->yyav = st->yyav + rec->y * rec->y;
    int accept = 1;
    if (rec->dH < 0.0) {                                                     /* :333-336 */
        rec->x = orc_rano(&st->rng, &st->rng.yran);
        rec->drew_x = 1;
        if (rec->x > rec->y) accept = 0;
    }
    if (accept) {                                                            /* :338-348 */
        memcpy(st->theta, st->thetat, sizeof(float) * 3 * kvol);
        st->naccp = st->naccp + 1;
        st->action = (float)(rec->S1 / (double)kvol);
        st->gaction = (float)(rec->hg / (double)kvol);
        st->paction = (float)(rec->hp / (double)kvol);
    }
    rec->accepted = accept;
    rec->action = st->action;
    rec->gaction = st->gaction;
    rec->paction = st->paction;
    st->actiona = st->actiona + st->action;                                  /* :350 */
    float vel2 = 0.0f;                                                       /* :351-357 */
    for (int64_t j = 0; j < 3 * kvol; j++) vel2 = vel2 + st->pp[j] * st->pp[j];
    rec->vel2 = vel2 / (float)(3 * kvol);
    st->vel2a = st->vel2a + rec->vel2;
    if ((st->isweep / st->iprint) * st->iprint == st->isweep) {              /* :361-371 */
        memcpy(st->thetat, st->theta, sizeof(float) * 3 * kvol);
        orc_thr_coef(lat, st->thetat, st->ut);
        float sus = 0.0f;
        orc_thr_measure(lat, &st->rng, 0.000001f, st->am, st->imass, st->ut, &rec->pbp, &sus,
                        &rec->ancgm, NULL);                                  /* respbp, :39 */
        rec->measured = 1;
    }
}
