/*
 * chdwf_oracle_hmc.c -- CPU oracle for the HMC predecessor of the RHMC code,
 * mh/cheisdwf_hmc.f (j-ostmeyer/chiralHeisenberg).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path in
 * chiralheisenberg_b200/csrc/hmc.cu; nothing in the product library links,
 * loads or calls it.
 *
 * mh/cheisdwf_hmc.f is single precision throughout: spinors COMPLEX (8
 * bytes), chi, chit, pp, dSdchi REAL*4, and every scalar REAL*4 except the
 * Hamiltonian pieces (REAL*8).  Its Makefile (mh/Makefile) builds it with
 * gfortran -O3 and neither OpenMP nor -march, so every sum runs in loop
 * order in the declared precision and nothing is contracted; this file keeps
 * both (compiled with -ffp-contract=off, float arithmetic in float).  The
 * operator is restated as the reference's separate sweeps (diagonal, Wilson,
 * antiperiodic correction, Dirac, its correction, s hops, wall coupling), in
 * the reference's order.  It has no pinning term.
 *
 * Layouts: as in chdwf_oracle.h, with complex64 spinors (re, im float pairs)
 * and REAL*4 chi(site, a) -> site + kvol*a.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "chdwf_oracle.h"

typedef struct { float re, im; } cf;

static inline cf cfld(const float* v, int64_t j) { cf r = {v[2 * j], v[2 * j + 1]}; return r; }
static inline void cfst(float* v, int64_t j, cf a) { v[2 * j] = a.re; v[2 * j + 1] = a.im; }
static inline cf cfadd(cf a, cf b) { cf r = {a.re + b.re, a.im + b.im}; return r; }
static inline cf cfsub(cf a, cf b) { cf r = {a.re - b.re, a.im - b.im}; return r; }
static inline cf cfmul(cf a, cf b) {
    cf r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}
static inline cf cfscal(float s, cf a) { cf r = {s * a.re, s * a.im}; return r; }
static inline cf cfconj(cf a) { cf r = {a.re, -a.im}; return r; }

#define HIDX(s, site, d, f) \
    ((int64_t)(s) + Ls * ((int64_t)(site) + kvol * ((int64_t)(d) + 4 * (int64_t)(f))))
#define SITE(ix, iy, it) ((int64_t)(ix) + (int64_t)L * ((iy) + (int64_t)L * (it)))

/* gamval(mu,idirac)*akappa and gamin(mu,idirac) of init, mu = 1,2,3
 * (mh/cheisdwf_hmc.f:1060-1094, scaled by akappa at :1132-1136) */
static const float kGv[3][4][2] = {{{0.f, -0.5f}, {0.f, -0.5f}, {0.f, 0.5f}, {0.f, 0.5f}},
                                   {{-0.5f, 0.f}, {0.5f, 0.f}, {0.5f, 0.f}, {-0.5f, 0.f}},
                                   {{0.f, -0.5f}, {0.f, 0.5f}, {0.f, 0.5f}, {0.f, -0.5f}}};
static const int kGi[3][4] = {{3, 2, 1, 0}, {3, 2, 1, 0}, {2, 3, 0, 1}};

/* neighbour sites of (ix, iy, it) in direction mu = x, y, t */
static void hops(int L, int Lt, int mu, int ix, int iy, int it, int64_t* up, int64_t* dn) {
    if (mu == 0) { *up = SITE((ix + 1) % L, iy, it); *dn = SITE((ix + L - 1) % L, iy, it); }
    else if (mu == 1) { *up = SITE(ix, (iy + 1) % L, it); *dn = SITE(ix, (iy + L - 1) % L, it); }
    else { *up = SITE(ix, iy, (it + 1) % Lt); *dn = SITE(ix, iy, (it + Lt - 1) % Lt); }
}

/* Phi = M R (dag = 0, mh/cheisdwf_hmc.f:1334-1681) or M^dagger R (dag = 1,
 * :1683-2028).  chi: REAL*4 (kvol, 3). */
void orc_hmc_dslash(const orc_lat* lat, float* Phi, const float* R, const float* chi,
                    int imass, int dag) {
    const int L = lat->L, Lt = lat->Lt;
    const int64_t Ls = lat->Ls, kvol = orc_kvol(lat), kferm = orc_kferm(lat);
    const float akappa = 0.5f;
    const float diag = (3.0f - lat->am3) + 1.0f;                              /* :1351, :1700 */
    for (int64_t j = 0; j < kferm; j++) cfst(Phi, j, cfscal(diag, cfld(R, j)));
    /* Wilson term, mu = 1, 2, 0 (:1367-1411, :1716-1760) */
    for (int f = 0; f < 2; f++)
        for (int d = 0; d < 4; d++)
            for (int mu = 0; mu < 3; mu++)
                for (int it = 0; it < Lt; it++)
                    for (int iy = 0; iy < L; iy++)
                        for (int ix = 0; ix < L; ix++) {
                            int64_t up, dn;
                            hops(L, Lt, mu, ix, iy, it, &up, &dn);
                            const int64_t site = SITE(ix, iy, it);
                            for (int64_t s = 0; s < Ls; s++) {
                                const int64_t o = HIDX(s, site, d, f);
                                cf w = cfadd(cfld(R, HIDX(s, up, d, f)), cfld(R, HIDX(s, dn, d, f)));
                                cfst(Phi, o, cfsub(cfld(Phi, o), cfscal(akappa, w)));
                            }
                        }
    /* antiperiodic correction of the Wilson term (:1412-1437, :1761-1786) */
    if (lat->ibound == -1)
        for (int f = 0; f < 2; f++)
            for (int d = 0; d < 4; d++) {
                for (int iy = 0; iy < L; iy++)
                    for (int ix = 0; ix < L; ix++)
                        for (int64_t s = 0; s < Ls; s++) {
                            const int64_t o = HIDX(s, SITE(ix, iy, Lt - 1), d, f);
                            cfst(Phi, o, cfadd(cfld(Phi, o), cfld(R, HIDX(s, SITE(ix, iy, 0), d, f))));
                        }
                for (int iy = 0; iy < L; iy++)
                    for (int ix = 0; ix < L; ix++)
                        for (int64_t s = 0; s < Ls; s++) {
                            const int64_t o = HIDX(s, SITE(ix, iy, 0), d, f);
                            cfst(Phi, o, cfadd(cfld(Phi, o), cfld(R, HIDX(s, SITE(ix, iy, Lt - 1), d, f))));
                        }
            }
    /* Dirac term, mu = 1, 2, 3: M adds gamval*(R(+) - R(-)) of component
     * gamin, M^dagger subtracts it (:1438-1490, :1787-1839) */
    for (int f = 0; f < 2; f++)
        for (int d = 0; d < 4; d++)
            for (int mu = 0; mu < 3; mu++) {
                const int dg = kGi[mu][d];
                const cf g = {kGv[mu][d][0], kGv[mu][d][1]};
                for (int it = 0; it < Lt; it++)
                    for (int iy = 0; iy < L; iy++)
                        for (int ix = 0; ix < L; ix++) {
                            int64_t up, dn;
                            hops(L, Lt, mu, ix, iy, it, &up, &dn);
                            const int64_t site = SITE(ix, iy, it);
                            for (int64_t s = 0; s < Ls; s++) {
                                const int64_t o = HIDX(s, site, d, f);
                                cf t = cfmul(g, cfsub(cfld(R, HIDX(s, up, dg, f)), cfld(R, HIDX(s, dn, dg, f))));
                                cfst(Phi, o, dag ? cfsub(cfld(Phi, o), t) : cfadd(cfld(Phi, o), t));
                            }
                        }
            }
    /* antiperiodic correction of the Dirac term: M subtracts
     * 2*gamval(3)*R(t=1) at t=ksizet and adds 2*gamval(3)*R(t=ksizet) at t=1
     * (:1491-1516); M^dagger the opposite signs (:1840-1865) */
    if (lat->ibound == -1)
        for (int f = 0; f < 2; f++)
            for (int d = 0; d < 4; d++) {
                const int dg = kGi[2][d];
                const cf g2 = {2.0f * kGv[2][d][0], 2.0f * kGv[2][d][1]};
                for (int iy = 0; iy < L; iy++)
                    for (int ix = 0; ix < L; ix++)
                        for (int64_t s = 0; s < Ls; s++) {
                            const int64_t o = HIDX(s, SITE(ix, iy, Lt - 1), d, f);
                            cf t = cfmul(g2, cfld(R, HIDX(s, SITE(ix, iy, 0), dg, f)));
                            cfst(Phi, o, dag ? cfadd(cfld(Phi, o), t) : cfsub(cfld(Phi, o), t));
                        }
                for (int iy = 0; iy < L; iy++)
                    for (int ix = 0; ix < L; ix++)
                        for (int64_t s = 0; s < Ls; s++) {
                            const int64_t o = HIDX(s, SITE(ix, iy, 0), d, f);
                            cf t = cfmul(g2, cfld(R, HIDX(s, SITE(ix, iy, Lt - 1), dg, f)));
                            cfst(Phi, o, dag ? cfsub(cfld(Phi, o), t) : cfadd(cfld(Phi, o), t));
                        }
            }
    /* s hops exploiting the projection: M takes Dirac 3,4 from s+1 and Dirac
     * 1,2 from s-1 (:1518-1546); M^dagger the reverse (:1867-1895) */
    const int up0 = dag ? 0 : 2, dn0 = dag ? 2 : 0;
    for (int f = 0; f < 2; f++) {
        for (int d = up0; d < up0 + 2; d++)
            for (int64_t site = 0; site < kvol; site++)
                for (int64_t s = 0; s < Ls - 1; s++) {
                    const int64_t o = HIDX(s, site, d, f);
                    cfst(Phi, o, cfsub(cfld(Phi, o), cfld(R, HIDX(s + 1, site, d, f))));
                }
        for (int d = dn0; d < dn0 + 2; d++)
            for (int64_t site = 0; site < kvol; site++)
                for (int64_t s = 0; s < Ls - 1; s++) {
                    const int64_t o = HIDX(s + 1, site, d, f);
                    cfst(Phi, o, cfsub(cfld(Phi, o), cfld(R, HIDX(s, site, d, f))));
                }
    }
    /* chi coupling of the walls (:1549-1679, :1897-2026), two stages with
     * spm1 and spm2.  Group A is written at s=kthird from s=1 (M: Dirac 3,4;
     * M^dagger: Dirac 1,2), group B at s=1 from s=kthird (the other pair).
     * Stage 1: flavour f gets sgn1 * spm1 * R(f); stage 2: flavour 1 gets
     * sgn2 * spm2 * R(2), flavour 2 gets sgn2 * conjg(spm2) * R(1). */
    const int64_t sL = Ls - 1;
    for (int stage = 0; stage < 2; stage++)
        for (int grp = 0; grp < 2; grp++) {
            const int d0 = (grp == 0) == (dag == 0) ? 2 : 0;
            const int64_t sw = grp == 0 ? sL : 0, sr = grp == 0 ? 0 : sL;
            for (int d = d0; d < d0 + 2; d++)
                for (int64_t i = 0; i < kvol; i++) {
                    const float c1 = chi[i], c2 = chi[i + kvol], c3 = chi[i + 2 * kvol];
                    cf spm;
                    int s1, s2;   /* signs for flavour 1 and 2 */
                    if (imass == 1) {
                        if (stage == 0) { spm.re = c3; spm.im = 0.0f; }
                        else { spm.re = c1; spm.im = -c2; }
                        s1 = 1;
                        s2 = stage == 0 ? -1 : 1;
                    } else {
                        if (stage == 0) { spm.re = 0.0f; spm.im = dag ? -c3 : c3; }
                        else if (!dag) { spm.re = c2; spm.im = c1; }
                        else { spm.re = -c2; spm.im = -c1; }
                        /* M: group A -,+ ; group B +,- ; M^dagger: A +,- ; B -,+ */
                        const int a_first = (grp == 0) == (dag == 0) ? -1 : 1;
                        s1 = a_first;
                        s2 = -a_first;
                    }
                    const int64_t o1 = HIDX(sw, i, d, 0), o2 = HIDX(sw, i, d, 1);
                    cf t1, t2;
                    if (stage == 0) {
                        t1 = cfmul(spm, cfld(R, HIDX(sr, i, d, 0)));
                        t2 = cfmul(spm, cfld(R, HIDX(sr, i, d, 1)));
                    } else {
                        t1 = cfmul(spm, cfld(R, HIDX(sr, i, d, 1)));
                        t2 = cfmul(cfconj(spm), cfld(R, HIDX(sr, i, d, 0)));
                    }
                    cfst(Phi, o1, s1 > 0 ? cfadd(cfld(Phi, o1), t1) : cfsub(cfld(Phi, o1), t1));
                    cfst(Phi, o2, s2 > 0 ? cfadd(cfld(Phi, o2), t2) : cfsub(cfld(Phi, o2), t2));
                }
        }
}

/* congrad (mh/cheisdwf_hmc.f:625-716): CGNE on M^dagger M, all REAL*4.
 * x: in = initial guess (/vector/), out = solution.  Returns 1 at the cap. */
int orc_hmc_congrad(const orc_lat* lat, const float* Phi, float res, int* itercg, int imass,
                    const float* chi, float* x) {
    const int64_t kferm = orc_kferm(lat), kvol = orc_kvol(lat);
    const int64_t niterc = lat->Ls * kvol;
    float* x1 = malloc(sizeof(float) * 2 * kferm);
    float* x2 = malloc(sizeof(float) * 2 * kferm);
    float* p = malloc(sizeof(float) * 2 * kferm);
    float* r = malloc(sizeof(float) * 2 * kferm);
    const float resid = (float)kferm * res * res;                           /* :638 */
    float betad = 1.0f, alpha = 1.0f, alphad, alphan = 0.0f, betan, beta;
    int capped = 1;
    *itercg = 0;
    for (int64_t nx = 1; nx <= niterc; nx++) {
        (*itercg)++;
        if (nx == 1) {                                                       /* :645-652 */
            memcpy(p, x, sizeof(float) * 2 * kferm);
            memcpy(r, Phi, sizeof(float) * 2 * kferm);
            betad = 1.0f;
            alpha = 1.0f;
        }
        orc_hmc_dslash(lat, x1, p, chi, imass, 0);                           /* :657 */
        if (nx != 1) {
            alphad = 0.0f;                                                   /* :663-667 */
            for (int64_t i = 0; i < kferm; i++)
                alphad = alphad + x1[2 * i] * x1[2 * i] + x1[2 * i + 1] * x1[2 * i + 1];
            alpha = alphan / alphad;
            for (int64_t i = 0; i < kferm; i++) cfst(x, i, cfadd(cfld(x, i), cfscal(alpha, cfld(p, i))));
        }
        orc_hmc_dslash(lat, x2, x1, chi, imass, 1);                          /* :678 */
        for (int64_t i = 0; i < kferm; i++) cfst(r, i, cfsub(cfld(r, i), cfscal(alpha, cfld(x2, i))));
        betan = 0.0f;                                                        /* :688-691 */
        for (int64_t i = 0; i < kferm; i++)
            betan = betan + r[2 * i] * r[2 * i] + r[2 * i + 1] * r[2 * i + 1];
        beta = betan / betad;
        betad = betan;
        alphan = betan;
        if (nx == 1) beta = 0.0f;
        for (int64_t i = 0; i < kferm; i++) cfst(p, i, cfadd(cfld(r, i), cfscal(beta, cfld(p, i))));
        if (betan < resid) { capped = 0; break; }
    }
    free(x1); free(x2); free(p); free(r);
    return capped;
}

/* The chi-force of force() given X1 = (M^dagger M)^-1 Phi
 * (mh/cheisdwf_hmc.f:416-420, :445-555): dSdchi = 2*beta*chi, then the wall
 * products of X1 with X2 = M X1 in the reference's order, then doubled. */
void orc_hmc_derivs(const orc_lat* lat, const float* X1, const float* chi, int imass,
                    float* dSdchi) {
    const int64_t Ls = lat->Ls, kvol = orc_kvol(lat), kferm = orc_kferm(lat);
    float* X2 = malloc(sizeof(float) * 2 * kferm);
    const float b2 = 2.0f * lat->beta;
    for (int64_t j = 0; j < 3 * kvol; j++) dSdchi[j] = b2 * chi[j];
    orc_hmc_dslash(lat, X2, X1, chi, imass, 0);                              /* :445 */
    float* d1 = dSdchi;
    float* d2 = dSdchi + kvol;
    float* d3 = dSdchi + 2 * kvol;
    const int64_t sL = Ls - 1;
    /* group 1: X1 at s=kthird, X2 at s=1, Dirac 1,2; group 2: X1 at s=1,
     * X2 at s=kthird, Dirac 3,4 */
    for (int grp = 0; grp < 2; grp++) {
        const int d0 = grp == 0 ? 0 : 2;
        const int64_t s1 = grp == 0 ? sL : 0, s2 = grp == 0 ? 0 : sL;
        for (int d = d0; d < d0 + 2; d++)
            for (int64_t i = 0; i < kvol; i++) {
                const cf a1 = cfconj(cfld(X1, HIDX(s1, i, d, 0)));
                const cf a2 = cfconj(cfld(X1, HIDX(s1, i, d, 1)));
                const cf b1 = cfld(X2, HIDX(s2, i, d, 0)), b2v = cfld(X2, HIDX(s2, i, d, 1));
                const cf p12 = cfmul(a1, b2v), p21 = cfmul(a2, b1);
                const cf p11 = cfmul(a1, b1), p22 = cfmul(a2, b2v);
                if (imass == 1) {            /* the same signs on both walls, :453-500 */
                    d1[i] = d1[i] - p12.re; d1[i] = d1[i] - p21.re;
                    d2[i] = d2[i] - p12.im; d2[i] = d2[i] + p21.im;
                    d3[i] = d3[i] - p11.re; d3[i] = d3[i] + p22.re;
                } else if (grp == 0) {                                       /* :501-526 */
                    d1[i] = d1[i] - p12.im; d1[i] = d1[i] - p21.im;
                    d2[i] = d2[i] + p12.re; d2[i] = d2[i] - p21.re;
                    d3[i] = d3[i] - p11.im; d3[i] = d3[i] + p22.im;
                } else {                                                     /* :527-549 */
                    d1[i] = d1[i] + p12.im; d1[i] = d1[i] + p21.im;
                    d2[i] = d2[i] - p12.re; d2[i] = d2[i] + p21.re;
                    d3[i] = d3[i] + p11.im; d3[i] = d3[i] - p22.im;
                }
            }
    }
    for (int64_t j = 0; j < 3 * kvol; j++) dSdchi[j] = 2.0f * dSdchi[j];        /* :550-554 */
    free(X2);
}

/* force (mh/cheisdwf_hmc.f:393-557): X1 = X0, X1 = (M^dagger M)^-1 Phi from
 * that guess, X0 = 2*X1 - X0 (the extrapolated next guess), then the chi
 * force of X1.  X1 (kferm complex) receives the solution. */
int orc_hmc_force(const orc_lat* lat, const float* Phi, float* X0, float* X1, const float* chi,
                  float res1, int imass, float* dSdchi, int* itercg) {
    const int64_t kferm = orc_kferm(lat);
    memcpy(X1, X0, sizeof(float) * 2 * kferm);                               /* :425-430 */
    const int capped = orc_hmc_congrad(lat, Phi, res1, itercg, imass, chi, X1);  /* :432 */
    for (int64_t j = 0; j < kferm; j++)                                      /* :434-439 */
        cfst(X0, j, cfsub(cfscal(2.0f, cfld(X1, j)), cfld(X0, j)));
    orc_hmc_derivs(lat, X1, chi, imass, dSdchi);
    return capped;
}

/* hamilton (mh/cheisdwf_hmc.f:561-623): h = hg + hp + hf with
 * hp = 0.5 sum pp^2, hg = 2 beta sum chi^2, hf = Re Phi^dagger X1 where
 * X1 = (M^dagger M)^-1 Phi from the guess X0; X0 then holds X1.  The
 * REAL*4 products are summed in REAL*8.  out: h, hg, hp, s = hg + hf. */
int orc_hmc_hamilton(const orc_lat* lat, const float* Phi, float* X0, const float* chi,
                     const float* pp, float res2, int imass, double* out, int* itercg) {
    const int64_t kferm = orc_kferm(lat), kvol = orc_kvol(lat);
    double hp = 0.0, hg = 0.0, hf = 0.0;
    for (int64_t j = 0; j < 3 * kvol; j++) hp = hp + (double)(pp[j] * pp[j]);     /* :582-587 */
    hp = hp * 0.5;
    for (int64_t j = 0; j < 3 * kvol; j++) hg = hg + (double)(chi[j] * chi[j]);   /* :589-594 */
    hg = (double)(2.0f * lat->beta) * hg;
    float* X1 = malloc(sizeof(float) * 2 * kferm);
    memcpy(X1, X0, sizeof(float) * 2 * kferm);                               /* :601-603 */
    const int capped = orc_hmc_congrad(lat, Phi, res2, itercg, imass, chi, X1);
    for (int64_t j = 0; j < kferm; j++) {                                    /* :606-611 */
        cfst(X0, j, cfld(X1, j));
        hf = hf + (double)cfmul(cfconj(cfld(Phi, j)), cfld(X1, j)).re;
    }
    free(X1);
    out[0] = hg + hp + hf;
    out[1] = hg;
    out[2] = hp;
    out[3] = hg + hf;
    return capped;
}

/* ---- program dwf3d of mh/cheisdwf_hmc.f (:140-320) ---------------------- */
orc_hmc_state* orc_hmc_new(int L, int Lt, int Ls, float beta, float am3, float dt, float am,
                           int imass, int iterl) {
    orc_hmc_state* s = calloc(1, sizeof(*s));
    s->lat.L = L; s->lat.Lt = Lt; s->lat.Ls = Ls;
    s->lat.beta = beta; s->lat.am3 = am3; s->lat.ibound = -1; s->lat.threads = 1;
    s->dt = dt; s->am = am; s->imass = imass; s->iterl = iterl; s->iprint = 5;
    s->rescga = 0.000000001f; s->rescgg = 0.000001f;                         /* :35 */
    const int64_t kvol = (int64_t)L * L * Lt, kferm = 8 * kvol * Ls;
    s->chi = calloc(3 * kvol, sizeof(float));
    s->chit = calloc(3 * kvol, sizeof(float));
    s->pp = calloc(3 * kvol, sizeof(float));
    s->dSdchi = calloc(3 * kvol, sizeof(float));
    s->Phi = calloc(2 * kferm, sizeof(float));
    s->X0 = calloc(2 * kferm, sizeof(float));
    s->X1 = calloc(2 * kferm, sizeof(float));
    s->R = calloc(2 * kferm, sizeof(float));
    s->ps = calloc(2 * kvol, sizeof(float));
    orc_rng_startup(&s->rng, 693764523745.0);
    return s;
}

void orc_hmc_free(orc_hmc_state* s) {
    if (!s) return;
    free(s->chi); free(s->chit); free(s->pp); free(s->dSdchi);
    free(s->Phi); free(s->X0); free(s->X1); free(s->R); free(s->ps);
    free(s);
}

void orc_hmc_sweep(orc_hmc_state* st, orc_hmc_rec* rec) {
    const orc_lat* lat = &st->lat;
    const int64_t Ls = lat->Ls, kvol = orc_kvol(lat), kferm = orc_kferm(lat);
    memset(rec, 0, sizeof(*rec));
    st->isweep++;
    const int isweep = st->isweep;
    memcpy(st->chit, st->chi, sizeof(float) * 3 * kvol);                    /* :146-149 */
    for (int f = 0; f < 2; f++)                                              /* :154-162 */
        for (int d = 0; d < 4; d++)
            for (int64_t s = 0; s < Ls; s++) {
                orc_gauss0(&st->rng, kvol, st->ps);
                for (int64_t i = 0; i < kvol; i++) {
                    cf v = {st->ps[i], st->ps[kvol + i]};
                    cfst(st->R, HIDX(s, i, d, f), v);
                }
            }
    orc_hmc_dslash(lat, st->Phi, st->R, st->chit, st->imass, 1);            /* :165 */
    memcpy(st->X0, st->Phi, sizeof(float) * 2 * kferm);                      /* :167-175 */
    orc_gaussp(&st->rng, kvol, st->ps);                                      /* :179-187 */
    memcpy(st->pp, st->ps, sizeof(float) * 2 * kvol);
    orc_gaussp(&st->rng, kvol, st->ps);
    memcpy(st->pp + 2 * kvol, st->ps, sizeof(float) * kvol);
    double h[4];
    int it = 0;
    orc_hmc_hamilton(lat, st->Phi, st->X0, st->chit, st->pp, st->rescga, st->imass, h, &it);  /* :191 */
    rec->it_h0 = it;
    rec->H0 = h[0];
    rec->S0 = h[3];
    if (isweep == 1) {                                                       /* :193-197 */
        st->action = (float)(h[3] / (double)kvol);
        st->gaction = (float)(h[1] / (double)kvol);
        st->paction = (float)(h[2] / (double)kvol);
    }
    orc_hmc_force(lat, st->Phi, st->X0, st->X1, st->chit, st->rescgg, st->imass, st->dSdchi, &it);  /* :202 */
    rec->it_force += it;
    rec->nforce++;
    float dd = st->dt * 0.5f;                                                /* :203-207 */
    for (int64_t j = 0; j < 3 * kvol; j++) st->pp[j] = st->pp[j] - st->dSdchi[j] * dd;
    const float proby = 1.0f / (float)st->iterl;                             /* :100 */
    for (int iter = 1; iter <= 1000; iter++) {                               /* :211-248 */
        dd = st->dt;
        for (int64_t j = 0; j < 3 * kvol; j++) st->chit[j] = st->chit[j] + dd * st->pp[j];
        orc_hmc_force(lat, st->Phi, st->X0, st->X1, st->chit, st->rescgg, st->imass, st->dSdchi, &it);
        rec->it_force += it;
        rec->nforce++;
        rec->nsteps = iter;
        const float ytest = orc_rano(&st->rng, &st->rng.yrun);              /* :228 */
        if (ytest < proby) {
            dd = st->dt * 0.5f;
            for (int64_t j = 0; j < 3 * kvol; j++) st->pp[j] = st->pp[j] - dd * st->dSdchi[j];
            st->itot = st->itot + iter;
            break;
        }
        dd = st->dt;
        for (int64_t j = 0; j < 3 * kvol; j++) st->pp[j] = st->pp[j] - dd * st->dSdchi[j];
    }
    orc_hmc_hamilton(lat, st->Phi, st->X0, st->chit, st->pp, st->rescga, st->imass, h, &it);  /* :251 */
    rec->it_h1 = it;
    rec->H1 = h[0];
    rec->S1 = h[3];
    rec->hg = h[1];
    rec->hp = h[2];
    rec->dH = rec->H0 - rec->H1;
    rec->dS = rec->S0 - rec->S1;
    rec->y = (float)exp(rec->dH);                                            /* :256 */
    st->yav = st->yav + rec->y;
    st->yyav = st->yyav + rec->y * rec->y;
    int accept = 1;
    if (rec->dH < 0.0) {                                                     /* :259-263 */
        rec->x = orc_rano(&st->rng, &st->rng.yrun);
        rec->drew_x = 1;
        if (rec->x > rec->y) accept = 0;
    }
    if (accept) {                                                            /* :264-274 */
        memcpy(st->chi, st->chit, sizeof(float) * 3 * kvol);
        st->naccp = st->naccp + 1;
        st->action = (float)(rec->S1 / (double)kvol);
        st->gaction = (float)(rec->hg / (double)kvol);
        st->paction = (float)(rec->hp / (double)kvol);
    }
    rec->accepted = accept;
    rec->action = st->action;
    rec->gaction = st->gaction;
    rec->paction = st->paction;
    st->actiona = st->actiona + st->action;                                  /* :277 */
    float vel2 = 0.0f;                                                       /* :278-283 */
    for (int64_t j = 0; j < 3 * kvol; j++) vel2 = vel2 + st->pp[j] * st->pp[j];
    rec->vel2 = vel2 / (float)kvol;
    st->vel2a = st->vel2a + rec->vel2;
    if ((isweep / st->iprint) * st->iprint == isweep) {                      /* :288-315 */
        rec->measured = 1;
        memcpy(st->chit, st->chi, sizeof(float) * 3 * kvol);
        float susctot = 0.0f, condmod = 0.0f;
        for (int a = 0; a < 3; a++) {
            float cnd = 0.0f;
            for (int64_t i = 0; i < kvol; i++) cnd = cnd + st->chi[i + kvol * a];
            float su = cnd * cnd;
            cnd = cnd / (float)kvol;
            condmod = condmod + cnd * cnd;
            su = su / (float)kvol;
            susctot = susctot + su;
            rec->cond[a] = cnd;
            rec->susc[a] = su;
        }
        rec->condmod = sqrtf(condmod);
        rec->susctot = susctot;
    }
}
