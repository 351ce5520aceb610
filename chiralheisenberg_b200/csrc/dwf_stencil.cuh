// dwf_stencil.cuh -- the domain-wall operator M (and M^dagger) for one lattice
// point, fused into a single gather.
//
// The reference applies M in about twelve read-modify-write sweeps over the
// whole 5D field (rhmc/cheisdwf.f:2651-3066 for M, :3088-3498 for
// M^dagger).  Here one thread computes all eight complex components of one
// output point in registers, performing for each element the same sequence of
// operations as those sweeps:
//   diag*R; hops +x,-x,+y,-y,+t,-t; *kappa; antiperiodic t correction;
//   s hop; chi3 wall term; pinning term; chi1/chi2 wall term.
// With the exact (non-contracted) FP64 helpers the result is bit-identical to
// the sweep-by-sweep evaluation.
#pragma once
#include "common.cuh"

namespace chdwf {

// Hop pattern of direction MU (0=x, 1=y, 2=t).  SIG=+1 is the combination
// the reference uses in M with the forward neighbour (cheisdwf.f:2675-2693,
// :2722-2739, :2769-2787), SIG=-1 the backward one (:2698-2716, :2744-2762,
// :2791-2811); M^dagger uses them the other way round (:3110-3246).
// NEG reverses every sign: the antiperiodic boundary correction
// (:2833-2875, :3267-3309).
template <int MU, int SIG, bool NEG, class T>
__device__ __forceinline__ void hop(T* acc, const T* r) {
    constexpr int pa = (MU == 2) ? 2 : 3;          // partner of Dirac 1 in a
    constexpr int pb = (MU == 2) ? 3 : 2;          // partner of Dirac 2 in b
    constexpr bool ii = (MU != 1);                 // combinations carry i
    constexpr int sa = SIG;
    constexpr int sb = ((MU == 0) ? 1 : -1) * SIG;
    constexpr int s3 = SIG;
    constexpr int s4 = ((MU == 0) ? 1 : -1) * SIG;
    constexpr bool x3b = (MU != 2);                // Phi3 takes b (x,y) or a (t)
    constexpr bool x4b = (MU == 2);
    constexpr int m = NEG ? -1 : 1;
    const T a = zcomb(r[0], r[pa], ii, sa);
    const T b = zcomb(r[1], r[pb], ii, sb);
    acc[0] = zcomb(acc[0], a, false, -m);
    acc[1] = zcomb(acc[1], b, false, -m);
    acc[2] = zcomb(acc[2], x3b ? b : a, ii, m * s3);
    acc[3] = zcomb(acc[3], x4b ? b : a, ii, m * s4);
}

struct PointIdx {
    int s, site, ix, iy, it;
    int64_t p;   // s + Ls*site
};

__device__ __forceinline__ PointIdx point_of(const Geom& g, int64_t p) {
    PointIdx q;
    q.p = p;
    const int site = (int)(p / g.Ls);
    q.s = (int)(p - (int64_t)site * g.Ls);
    q.site = site;
    const int LL = g.L * g.L;
    q.it = site / LL;
    const int rem = site - q.it * LL;
    q.iy = rem / g.L;
    q.ix = rem - q.iy * g.L;
    return q;
}

// Loads the four Dirac components of flavour f at point index n.
template <class Ld, class T>
__device__ __forceinline__ void load4(T* r, const Ld& ld, const Geom& g, int64_t n, int f) {
#pragma unroll
    for (int d = 0; d < 4; d++) r[d] = ld(n + g.cs * (d + 4 * f));
}

// chi is passed pre-rounded to REAL*4: the reference builds the wall
// coupling with cmplx(chi, ...) without a KIND, i.e. in default (single)
// precision (cheisdwf.f:2914, :2962, :2998, :3034).  chif holds (chi1, chi2,
// chi3) as three planes of kvol floats.
template <bool DAG, int IMASS, class T, class Ld>
__device__ __forceinline__ void dwf_apply_point(T acc[2][4], const Ld& ld, const Geom& g,
                                                const PointIdx& q, const float* __restrict__ chif,
                                                typename real_of<T>::type diag,
                                                typename real_of<T>::type hpin, bool apbc) {
    typedef typename real_of<T>::type R;
    constexpr int SF = DAG ? -1 : 1;               // pattern sign of the forward hop
    const int L = g.L, Lt = g.Lt, Ls = g.Ls;
    const int64_t LsI = Ls;
    // diagonal term (:2651-2667)
#pragma unroll
    for (int f = 0; f < 2; f++)
#pragma unroll
        for (int d = 0; d < 4; d++) acc[f][d] = zscal(diag, ld(q.p + g.cs * (d + 4 * f)));
    // neighbour sites
    const int xp = q.ix + 1 == L ? 0 : q.ix + 1, xm = q.ix == 0 ? L - 1 : q.ix - 1;
    const int yp = q.iy + 1 == L ? 0 : q.iy + 1, ym = q.iy == 0 ? L - 1 : q.iy - 1;
    const int tp = q.it + 1 == Lt ? 0 : q.it + 1, tm = q.it == 0 ? Lt - 1 : q.it - 1;
    const int64_t rowb = (int64_t)L * (q.iy + (int64_t)L * q.it);
    const int64_t n_xp = q.s + LsI * (xp + rowb), n_xm = q.s + LsI * (xm + rowb);
    const int64_t colb = q.ix + (int64_t)L * L * q.it;
    const int64_t n_yp = q.s + LsI * (colb + (int64_t)L * yp), n_ym = q.s + LsI * (colb + (int64_t)L * ym);
    const int64_t plb = q.ix + (int64_t)L * q.iy;
    const int64_t n_tp = q.s + LsI * (plb + (int64_t)L * L * tp), n_tm = q.s + LsI * (plb + (int64_t)L * L * tm);
#pragma unroll
    for (int f = 0; f < 2; f++) {
        T r[4];
        load4(r, ld, g, n_xp, f); hop<0, SF, false>(acc[f], r);
        load4(r, ld, g, n_xm, f); hop<0, -SF, false>(acc[f], r);
        load4(r, ld, g, n_yp, f); hop<1, SF, false>(acc[f], r);
        load4(r, ld, g, n_ym, f); hop<1, -SF, false>(acc[f], r);
        load4(r, ld, g, n_tp, f); hop<2, SF, false>(acc[f], r);
        load4(r, ld, g, n_tm, f); hop<2, -SF, false>(acc[f], r);
    }
    // kappa = 1/2 (:2815-2829)
#pragma unroll
    for (int f = 0; f < 2; f++)
#pragma unroll
        for (int d = 0; d < 4; d++) acc[f][d] = zscal((R)0.5, acc[f][d]);
    // antiperiodic boundary in t (:2831-2876): reverse the wrapped hop
    if (apbc) {
        if (q.it == Lt - 1) {
#pragma unroll
            for (int f = 0; f < 2; f++) { T r[4]; load4(r, ld, g, n_tp, f); hop<2, SF, true>(acc[f], r); }
        }
        if (q.it == 0) {
#pragma unroll
            for (int f = 0; f < 2; f++) { T r[4]; load4(r, ld, g, n_tm, f); hop<2, -SF, true>(acc[f], r); }
        }
    }
    // s hops with chiral projection (:2879-2908; M^dagger :3313-3342)
    constexpr int UP = DAG ? 0 : 2;    // Dirac pair fed from s+1
    constexpr int DN = DAG ? 2 : 0;    // Dirac pair fed from s-1
    if (q.s < Ls - 1) {
#pragma unroll
        for (int f = 0; f < 2; f++)
#pragma unroll
            for (int d = UP; d < UP + 2; d++) acc[f][d] = zsub(acc[f][d], ld(q.p + 1 + g.cs * (d + 4 * f)));
    }
    if (q.s > 0) {
#pragma unroll
        for (int f = 0; f < 2; f++)
#pragma unroll
            for (int d = DN; d < DN + 2; d++) acc[f][d] = zsub(acc[f][d], ld(q.p - 1 + g.cs * (d + 4 * f)));
    }
    // wall coupling: pair WA at s=Ls reads s=1, pair WB at s=1 reads s=Ls
    constexpr int WA = DAG ? 0 : 2;
    constexpr int WB = DAG ? 2 : 0;
    const bool atL = (q.s == Ls - 1), at0 = (q.s == 0);
    if (!(atL || at0)) return;
    const float c1f = __ldg(chif + q.site), c2f = __ldg(chif + g.kvol + q.site),
                c3f = __ldg(chif + 2 * g.kvol + q.site);
    const int64_t other = atL ? (int64_t)LsI * q.site : (int64_t)LsI * q.site + Ls - 1;
    const bool pin = (q.site == 0);
#pragma unroll
    for (int side = 0; side < 2; side++) {
        const bool active = side == 0 ? atL : at0;
        if (!active) continue;
        const int d0 = side == 0 ? WA : WB;
        // Sign of the terms: M/imass=1 adds on both walls; see the oracle.
#pragma unroll
        for (int d = d0; d < d0 + 2; d++) {
            const T r1 = ld(other + g.cs * (d + 0)), r2 = ld(other + g.cs * (d + 4));
            if (IMASS == 1) {
                // spm = cmplx(chi3, 0) (:2912-2946 / :3345-3379)
                const T spm = zmake<T>((R)c3f, (R)0);
                acc[0][d] = zadd(acc[0][d], zmul(spm, r1));
                acc[1][d] = zsub(acc[1][d], zmul(spm, r2));
                if (pin) {  // (:2948-2959 / :3381-3392)
                    acc[0][d] = zadd(acc[0][d], zscal(hpin, r1));
                    acc[1][d] = zsub(acc[1][d], zscal(hpin, r2));
                }
                // spm = cmplx(chi1, -chi2) (:2962-2995 / :3395-3428)
                const T sp = zmake<T>((R)c1f, (R)(-c2f));
                acc[0][d] = zadd(acc[0][d], zmul(sp, r2));
                acc[1][d] = zadd(acc[1][d], zmul(zconj(sp), r1));
            } else if (IMASS == 3) {
                // M: spm = cmplx(0, chi3) (:2996-3030); M^dagger cmplx(0,-chi3) (:3429-3463)
                const T spm = zmake<T>((R)0, (R)(DAG ? -c3f : c3f));
                const T t1 = zmul(spm, r1), t2 = zmul(spm, r2);
                // sign of the flavour-1 term: M: -,+ at s=Ls / +,- at s=1;
                // M^dagger: +,- at s=Ls / -,+ at s=1
                const bool minus_first = (!DAG && side == 0) || (DAG && side == 1);
                if (minus_first) { acc[0][d] = zsub(acc[0][d], t1); acc[1][d] = zadd(acc[1][d], t2); }
                else             { acc[0][d] = zadd(acc[0][d], t1); acc[1][d] = zsub(acc[1][d], t2); }
                // M: spm = cmplx(chi2, chi1) (:3032-3065); M^dagger cmplx(-chi2,-chi1) (:3465-3497)
                const T sp = DAG ? zmake<T>((R)(-c2f), (R)(-c1f)) : zmake<T>((R)c2f, (R)c1f);
                const T u1 = zmul(sp, r2), u2 = zmul(zconj(sp), r1);
                if (minus_first) { acc[0][d] = zsub(acc[0][d], u1); acc[1][d] = zadd(acc[1][d], u2); }
                else             { acc[0][d] = zadd(acc[0][d], u1); acc[1][d] = zsub(acc[1][d], u2); }
            }
        }
    }
}

}  // namespace chdwf
