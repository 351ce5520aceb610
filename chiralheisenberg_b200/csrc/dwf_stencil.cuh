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

// Coordinates of point p (p < 2^31: see kMaxPoints), in 32-bit arithmetic
// with the geometry's precomputed divisions.
__device__ __forceinline__ PointIdx point_of(const Geom& g, int64_t p) {
    PointIdx q;
    q.p = p;
    const unsigned up = (unsigned)p, Ls = (unsigned)g.Ls, L = (unsigned)g.L;
    const unsigned site = fdiv(up, g.dLs);
    q.s = (int)(up - site * Ls);
    q.site = (int)site;
    const unsigned it = fdiv(site, g.dLL);
    const unsigned rem = site - it * (L * L);
    const unsigned iy = fdiv(rem, g.dL);
    q.it = (int)it;
    q.iy = (int)iy;
    q.ix = (int)(rem - iy * L);
    return q;
}

// Loads the four Dirac components of flavour f at point index n.
template <class Ld, class T>
__device__ __forceinline__ void load4(T* r, const Ld& ld, const Geom& g, int64_t n, int f) {
#pragma unroll
    for (int d = 0; d < 4; d++) r[d] = ld(n + g.cs * (d + 4 * f));
}

// One element of the wall coupling: a of flavour f takes r1 (flavour 0) and
// r2 (flavour 1), the other wall's components of the same Dirac index.
template <bool DAG, int IMASS, int SIDE, class T>
__device__ __forceinline__ void wall_elem(T& a, T r1, T r2, int f, float c1f, float c2f,
                                          float c3f, bool pin, typename real_of<T>::type hpin) {
    typedef typename real_of<T>::type R;
    if (IMASS == 1) {
        // spm = cmplx(chi3, 0) (:2912-2946 / :3345-3379), pinning
        // (:2948-2959 / :3381-3392), spm = cmplx(chi1, -chi2)
        // (:2962-2995 / :3395-3428)
        const T spm = zmake<T>((R)c3f, (R)0);
        const T sp = zmake<T>((R)c1f, (R)(-c2f));
        if (f == 0) {
            a = zadd(a, zmul(spm, r1));
            if (pin) a = zadd(a, zscal(hpin, r1));
            a = zadd(a, zmul(sp, r2));
        } else {
            a = zsub(a, zmul(spm, r2));
            if (pin) a = zsub(a, zscal(hpin, r2));
            a = zadd(a, zmul(zconj(sp), r1));
        }
    } else if (IMASS == 3) {
        // M: spm = cmplx(0, chi3) (:2996-3030); M^dagger cmplx(0,-chi3)
        // (:3429-3463).  Sign of the flavour-1 term: M: -,+ at s=Ls and
        // +,- at s=1; M^dagger: +,- at s=Ls and -,+ at s=1.
        const T spm = zmake<T>((R)0, (R)(DAG ? -c3f : c3f));
        constexpr bool minus_first = (!DAG && SIDE == 0) || (DAG && SIDE == 1);
        // M: spm = cmplx(chi2, chi1) (:3032-3065); M^dagger
        // cmplx(-chi2,-chi1) (:3465-3497)
        const T sp = DAG ? zmake<T>((R)(-c2f), (R)(-c1f)) : zmake<T>((R)c2f, (R)c1f);
        if (f == 0) {
            const T t1 = zmul(spm, r1), u1 = zmul(sp, r2);
            a = minus_first ? zsub(a, t1) : zadd(a, t1);
            a = minus_first ? zsub(a, u1) : zadd(a, u1);
        } else {
            const T t2 = zmul(spm, r2), u2 = zmul(zconj(sp), r1);
            a = minus_first ? zadd(a, t2) : zsub(a, t2);
            a = minus_first ? zadd(a, u2) : zsub(a, u2);
        }
    }
}

// wall_elem with the wall known only at run time (side1: the s = 1 wall), so
// a thread evaluates either wall with one code path instead of a warp
// running both branches.  a - b is formed as a + (-b), the same IEEE result.
template <class T> __device__ __forceinline__ T zneg_if(bool n, T v) {
    return n ? zmake<T>(-v.x, -v.y) : v;
}
template <bool DAG, int IMASS, class T>
__device__ __forceinline__ void wall_elem_rt(T& a, T r1, T r2, int f, bool side1, float c1f,
                                             float c2f, float c3f, bool pin,
                                             typename real_of<T>::type hpin) {
    typedef typename real_of<T>::type R;
    if (IMASS == 1) {
        wall_elem<DAG, 1, 0>(a, r1, r2, f, c1f, c2f, c3f, pin, hpin);   // no side dependence
    } else if (IMASS == 3) {
        const T spm = zmake<T>((R)0, (R)(DAG ? -c3f : c3f));
        const bool minus_first = DAG ? side1 : !side1;
        const T sp = DAG ? zmake<T>((R)(-c2f), (R)(-c1f)) : zmake<T>((R)c2f, (R)c1f);
        if (f == 0) {
            const T t1 = zmul(spm, r1), u1 = zmul(sp, r2);
            a = zadd(a, zneg_if(minus_first, t1));
            a = zadd(a, zneg_if(minus_first, u1));
        } else {
            const T t2 = zmul(spm, r2), u2 = zmul(zconj(sp), r1);
            a = zadd(a, zneg_if(!minus_first, t2));
            a = zadd(a, zneg_if(!minus_first, u2));
        }
    }
}

// The wall update of one point at either wall (atL: s = Ls, else s = 1):
// Dirac pair WA or WB takes the other wall's components of both flavours.
template <bool DAG, int IMASS, class T, class Ld>
__device__ __forceinline__ void wall_terms_rt(T acc[4], const Ld& ld, int64_t cs, int64_t other,
                                              bool atL, int f, float c1f, float c2f, float c3f,
                                              bool pin, typename real_of<T>::type hpin) {
    constexpr int WA = DAG ? 0 : 2;
    constexpr int WB = DAG ? 2 : 0;
    const int d0 = atL ? WA : WB;
    T a0 = atL ? acc[WA] : acc[WB], a1 = atL ? acc[WA + 1] : acc[WB + 1];
    wall_elem_rt<DAG, IMASS>(a0, ld(other + cs * d0), ld(other + cs * (d0 + 4)), f, !atL, c1f,
                             c2f, c3f, pin, hpin);
    wall_elem_rt<DAG, IMASS>(a1, ld(other + cs * (d0 + 1)), ld(other + cs * (d0 + 5)), f, !atL,
                             c1f, c2f, c3f, pin, hpin);
    if (atL) {
        acc[WA] = a0;
        acc[WA + 1] = a1;
    } else {
        acc[WB] = a0;
        acc[WB + 1] = a1;
    }
}

// Wall coupling of one flavour at a wall point (s = Ls for SIDE 0, s = 1 for
// SIDE 1): Dirac pair D0, D0+1 of flavour f takes the other wall's components
// of both flavours.  Per element the operation sequence is that of the
// reference's wall sweeps.
template <bool DAG, int IMASS, int D0, int SIDE, class T, class Ld>
__device__ __forceinline__ void wall_terms(T acc[4], const Ld& ld, int64_t cs, int64_t other,
                                           int f, float c1f, float c2f, float c3f, bool pin,
                                           typename real_of<T>::type hpin) {
#pragma unroll
    for (int d = D0; d < D0 + 2; d++)
        wall_elem<DAG, IMASS, SIDE>(acc[d], ld(other + cs * d), ld(other + cs * (d + 4)), f, c1f,
                                    c2f, c3f, pin, hpin);
}

// The four Dirac components of flavour f at one output point.  The flavours
// couple only through the wall terms, which read both flavours' inputs on
// the other wall, so two threads can share a point (one per flavour) and
// each needs half the accumulator registers.
//
// chi is passed pre-rounded to REAL*4: the reference builds the wall
// coupling with cmplx(chi, ...) without a KIND, i.e. in default (single)
// precision (cheisdwf.f:2914, :2962, :2998, :3034).  chif holds (chi1, chi2,
// chi3) as three planes of kvol floats.
template <bool DAG, int IMASS, class T, class Ld>
__device__ __forceinline__ void dwf_apply_flavour(T acc[4], const Ld& ld, const Geom& g,
                                                  const PointIdx& q, int f,
                                                  const float* __restrict__ chif,
                                                  typename real_of<T>::type diag,
                                                  typename real_of<T>::type hpin, bool apbc) {
    typedef typename real_of<T>::type R;
    constexpr int SF = DAG ? -1 : 1;               // pattern sign of the forward hop
    const int L = g.L, Lt = g.Lt, Ls = g.Ls;
    const int64_t LsI = Ls, cs = g.cs, fo = g.cs * (4 * f);
    // diagonal term (:2651-2667)
#pragma unroll
    for (int d = 0; d < 4; d++) acc[d] = zscal(diag, ld(q.p + fo + cs * d));
    // neighbour sites
    const int xp = q.ix + 1 == L ? 0 : q.ix + 1, xm = q.ix == 0 ? L - 1 : q.ix - 1;
    const int yp = q.iy + 1 == L ? 0 : q.iy + 1, ym = q.iy == 0 ? L - 1 : q.iy - 1;
    const int tp = q.it + 1 == Lt ? 0 : q.it + 1, tm = q.it == 0 ? Lt - 1 : q.it - 1;
    const int64_t sb = q.s + fo;
    const int64_t rowb = (int64_t)L * (q.iy + (int64_t)L * q.it);
    const int64_t n_xp = sb + LsI * (xp + rowb), n_xm = sb + LsI * (xm + rowb);
    const int64_t colb = q.ix + (int64_t)L * L * q.it;
    const int64_t n_yp = sb + LsI * (colb + (int64_t)L * yp), n_ym = sb + LsI * (colb + (int64_t)L * ym);
    const int64_t plb = q.ix + (int64_t)L * q.iy;
    const int64_t n_tp = sb + LsI * (plb + (int64_t)L * L * tp), n_tm = sb + LsI * (plb + (int64_t)L * L * tm);
    T r[4];
    load4(r, ld, g, n_xp, 0); hop<0, SF, false>(acc, r);
    load4(r, ld, g, n_xm, 0); hop<0, -SF, false>(acc, r);
    load4(r, ld, g, n_yp, 0); hop<1, SF, false>(acc, r);
    load4(r, ld, g, n_ym, 0); hop<1, -SF, false>(acc, r);
    load4(r, ld, g, n_tp, 0); hop<2, SF, false>(acc, r);
    load4(r, ld, g, n_tm, 0); hop<2, -SF, false>(acc, r);
    // kappa = 1/2 (:2815-2829)
#pragma unroll
    for (int d = 0; d < 4; d++) acc[d] = zscal((R)0.5, acc[d]);
    // antiperiodic boundary in t (:2831-2876): reverse the wrapped hop
    if (apbc) {
        if (q.it == Lt - 1) { load4(r, ld, g, n_tp, 0); hop<2, SF, true>(acc, r); }
        if (q.it == 0) { load4(r, ld, g, n_tm, 0); hop<2, -SF, true>(acc, r); }
    }
    // s hops with chiral projection (:2879-2908; M^dagger :3313-3342)
    constexpr int UP = DAG ? 0 : 2;    // Dirac pair fed from s+1
    constexpr int DN = DAG ? 2 : 0;    // Dirac pair fed from s-1
    if (q.s < Ls - 1) {
#pragma unroll
        for (int d = UP; d < UP + 2; d++) acc[d] = zsub(acc[d], ld(q.p + 1 + fo + cs * d));
    }
    if (q.s > 0) {
#pragma unroll
        for (int d = DN; d < DN + 2; d++) acc[d] = zsub(acc[d], ld(q.p - 1 + fo + cs * d));
    }
    // wall coupling: the pair at s=Ls reads s=1, the pair at s=1 reads s=Ls
    const bool atL = (q.s == Ls - 1), at0 = (q.s == 0);
    if (!(atL || at0)) return;
    const float c1f = __ldg(chif + q.site), c2f = __ldg(chif + g.kvol + q.site),
                c3f = __ldg(chif + 2 * g.kvol + q.site);
    const int64_t other = atL ? LsI * q.site : LsI * q.site + Ls - 1;
    const bool pin = (q.site == 0);
    wall_terms_rt<DAG, IMASS>(acc, ld, cs, other, atL, f, c1f, c2f, c3f, pin, hpin);
}

// All eight components of one output point (one thread per point).
template <bool DAG, int IMASS, class T, class Ld>
__device__ __forceinline__ void dwf_apply_point(T acc[2][4], const Ld& ld, const Geom& g,
                                                const PointIdx& q, const float* __restrict__ chif,
                                                typename real_of<T>::type diag,
                                                typename real_of<T>::type hpin, bool apbc) {
    dwf_apply_flavour<DAG, IMASS>(acc[0], ld, g, q, 0, chif, diag, hpin, apbc);
    dwf_apply_flavour<DAG, IMASS>(acc[1], ld, g, q, 1, chif, diag, hpin, apbc);
}

struct LdF2 {
    const float2* __restrict__ p;
    __device__ __forceinline__ float2 operator()(int64_t j) const { return __ldg(p + j); }
};

// Two adjacent points (s, s+1), s even, of flavour f on FP32 storage.  Each
// load is one 16-byte float4 holding both points' components (the spinor
// layout has s innermost, so an even point and its successor are adjacent),
// which doubles the bytes per load instruction; each point's elements go
// through the same operation sequence as dwf_apply_flavour.  Needs Ls even
// and kferm < 2^31: element indices are 32-bit (pair_ok), which halves the
// address arithmetic of its 34 loads.
inline bool pair_ok(const Geom& g) { return g.Ls % 2 == 0 && g.kferm < (int64_t(1) << 31); }

template <bool DAG, int IMASS>
__device__ __forceinline__ void dwf_apply_flavour_pair(float2 acc[2][4],
                                                       const float2* __restrict__ in,
                                                       const Geom& g, const PointIdx& q, int f,
                                                       const float* __restrict__ chif, float diag,
                                                       float hpin, bool apbc) {
    constexpr int SF = DAG ? -1 : 1;
    const int L = g.L, Lt = g.Lt, Ls = g.Ls;
    const uint32_t LsI = (uint32_t)Ls, cs = (uint32_t)g.cs, fo = cs * (uint32_t)(4 * f);
    const uint32_t qp = (uint32_t)q.p;
    auto ld2 = [&](uint32_t n, float2& r0, float2& r1) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(in + n));
        r0 = make_float2(v.x, v.y);
        r1 = make_float2(v.z, v.w);
    };
    // diagonal term (:2651-2667)
#pragma unroll
    for (int d = 0; d < 4; d++) {
        float2 r0, r1;
        ld2(qp + fo + cs * d, r0, r1);
        acc[0][d] = zscal(diag, r0);
        acc[1][d] = zscal(diag, r1);
    }
    const uint32_t uL = (uint32_t)L;
    const uint32_t xp = q.ix + 1 == L ? 0 : q.ix + 1, xm = q.ix == 0 ? L - 1 : q.ix - 1;
    const uint32_t yp = q.iy + 1 == L ? 0 : q.iy + 1, ym = q.iy == 0 ? L - 1 : q.iy - 1;
    const uint32_t tp = q.it + 1 == Lt ? 0 : q.it + 1, tm = q.it == 0 ? Lt - 1 : q.it - 1;
    const uint32_t sb = (uint32_t)q.s + fo;
    const uint32_t rowb = uL * ((uint32_t)q.iy + uL * (uint32_t)q.it);
    const uint32_t n_xp = sb + LsI * (xp + rowb), n_xm = sb + LsI * (xm + rowb);
    const uint32_t colb = (uint32_t)q.ix + uL * uL * (uint32_t)q.it;
    const uint32_t n_yp = sb + LsI * (colb + uL * yp), n_ym = sb + LsI * (colb + uL * ym);
    const uint32_t plb = (uint32_t)q.ix + uL * (uint32_t)q.iy;
    const uint32_t n_tp = sb + LsI * (plb + uL * uL * tp), n_tm = sb + LsI * (plb + uL * uL * tm);
    float2 r0[4], r1[4];
#define CHDWF_PAIR_HOP(N, MU, SIG, NEG)                                         \
    {                                                                          \
        _Pragma("unroll") for (int d = 0; d < 4; d++) ld2((N) + cs * d, r0[d], r1[d]); \
        hop<MU, SIG, NEG>(acc[0], r0);                                         \
        hop<MU, SIG, NEG>(acc[1], r1);                                         \
    }
    CHDWF_PAIR_HOP(n_xp, 0, SF, false)
    CHDWF_PAIR_HOP(n_xm, 0, -SF, false)
    CHDWF_PAIR_HOP(n_yp, 1, SF, false)
    CHDWF_PAIR_HOP(n_ym, 1, -SF, false)
    CHDWF_PAIR_HOP(n_tp, 2, SF, false)
    CHDWF_PAIR_HOP(n_tm, 2, -SF, false)
    // kappa = 1/2 (:2815-2829)
#pragma unroll
    for (int d = 0; d < 4; d++) {
        acc[0][d] = zscal(0.5f, acc[0][d]);
        acc[1][d] = zscal(0.5f, acc[1][d]);
    }
    // antiperiodic boundary in t (:2831-2876)
    if (apbc) {
        if (q.it == Lt - 1) CHDWF_PAIR_HOP(n_tp, 2, SF, true)
        if (q.it == 0) CHDWF_PAIR_HOP(n_tm, 2, -SF, true)
    }
#undef CHDWF_PAIR_HOP
    // s hops (:2879-2908; M^dagger :3313-3342).  Point 0 is s, point 1 is s+1:
    // the pair fed from s+1 takes point 0's value from this pair and point 1's
    // from the next pair; the pair fed from s-1 takes point 0's value from the
    // previous pair and point 1's from this pair.
    constexpr int UP = DAG ? 0 : 2;
    constexpr int DN = DAG ? 2 : 0;
#pragma unroll
    for (int d = UP; d < UP + 2; d++) {
        float2 c0, c1;
        ld2(qp + fo + cs * d, c0, c1);
        acc[0][d] = zsub(acc[0][d], c1);
        if (q.s + 2 < Ls) {
            float2 n0, n1;
            ld2(qp + 2 + fo + cs * d, n0, n1);
            acc[1][d] = zsub(acc[1][d], n0);
        }
    }
#pragma unroll
    for (int d = DN; d < DN + 2; d++) {
        float2 c0, c1;
        ld2(qp + fo + cs * d, c0, c1);
        if (q.s > 0) {
            float2 p0, p1;
            ld2(qp - 2 + fo + cs * d, p0, p1);
            acc[0][d] = zsub(acc[0][d], p1);
        }
        acc[1][d] = zsub(acc[1][d], c0);
    }
    // wall coupling: point 1 at s=Ls (pair WA, reads s=1), point 0 at s=1
    // (pair WB, reads s=Ls)
    constexpr int WA = DAG ? 0 : 2;
    constexpr int WB = DAG ? 2 : 0;
    const bool atL = (q.s + 2 == Ls), at0 = (q.s == 0);
    if (!(atL || at0)) return;
    const float c1f = __ldg(chif + q.site), c2f = __ldg(chif + g.kvol + q.site),
                c3f = __ldg(chif + 2 * g.kvol + q.site);
    const bool pin = (q.site == 0);
    if (atL && at0) {   // Ls = 2: one pair holds both walls
        wall_terms<DAG, IMASS, WA, 0>(acc[1], LdF2{in}, cs, LsI * q.site, f, c1f, c2f, c3f, pin, hpin);
        wall_terms<DAG, IMASS, WB, 1>(acc[0], LdF2{in}, cs, LsI * q.site + Ls - 1, f, c1f, c2f, c3f,
                                      pin, hpin);
        return;
    }
    // one wall point: point 1 at s=Ls or point 0 at s=1, through one code path
    float2 w[4];
#pragma unroll
    for (int d = 0; d < 4; d++) w[d] = atL ? acc[1][d] : acc[0][d];
    wall_terms_rt<DAG, IMASS>(w, LdF2{in}, (int64_t)cs,
                              atL ? (int64_t)LsI * q.site : (int64_t)LsI * q.site + Ls - 1, atL, f,
                              c1f, c2f, c3f, pin, hpin);
#pragma unroll
    for (int d = 0; d < 4; d++) {
        if (atL) acc[1][d] = w[d];
        else acc[0][d] = w[d];
    }
}

// Element loader of a split-layout FP32 vector (the wall operands).
struct LdSp {
    const float2* __restrict__ p;
    __device__ __forceinline__ float2 operator()(int64_t j) const { return sp_get(p, j); }
};

// dwf_apply_flavour_pair on a split-layout vector (see cpair): the same two
// points, loads and per-element operation sequence, with every hop, scaling
// and three-term step done as packed FP32x2 operations on both points at
// once.  The s hops and the wall terms act on one point of the pair and stay
// per point.  Needs pair_ok(g).
template <bool DAG, int IMASS>
__device__ __forceinline__ void dwf_apply_flavour_pair_sp(cpair acc[4],
                                                          const float2* __restrict__ in,
                                                          const Geom& g, const PointIdx& q, int f,
                                                          const float* __restrict__ chif,
                                                          float diag, float hpin, bool apbc) {
    constexpr int SF = DAG ? -1 : 1;
    const int L = g.L, Lt = g.Lt, Ls = g.Ls;
    const uint32_t LsI = (uint32_t)Ls, cs = (uint32_t)g.cs, fo = cs * (uint32_t)(4 * f);
    const uint32_t qp = (uint32_t)q.p;
    // diagonal term (:2651-2667)
#pragma unroll
    for (int d = 0; d < 4; d++) acc[d] = zscal(diag, ld_cpair(in, qp + fo + cs * d));
    const uint32_t uL = (uint32_t)L;
    const uint32_t xp = q.ix + 1 == L ? 0 : q.ix + 1, xm = q.ix == 0 ? L - 1 : q.ix - 1;
    const uint32_t yp = q.iy + 1 == L ? 0 : q.iy + 1, ym = q.iy == 0 ? L - 1 : q.iy - 1;
    const uint32_t tp = q.it + 1 == Lt ? 0 : q.it + 1, tm = q.it == 0 ? Lt - 1 : q.it - 1;
    const uint32_t sb = (uint32_t)q.s + fo;
    const uint32_t rowb = uL * ((uint32_t)q.iy + uL * (uint32_t)q.it);
    const uint32_t n_xp = sb + LsI * (xp + rowb), n_xm = sb + LsI * (xm + rowb);
    const uint32_t colb = (uint32_t)q.ix + uL * uL * (uint32_t)q.it;
    const uint32_t n_yp = sb + LsI * (colb + uL * yp), n_ym = sb + LsI * (colb + uL * ym);
    const uint32_t plb = (uint32_t)q.ix + uL * (uint32_t)q.iy;
    const uint32_t n_tp = sb + LsI * (plb + uL * uL * tp), n_tm = sb + LsI * (plb + uL * uL * tm);
    cpair r[4];
#define CHDWF_SP_HOP(N, MU, SIG, NEG)                                                  \
    {                                                                                 \
        _Pragma("unroll") for (int d = 0; d < 4; d++) r[d] = ld_cpair(in, (N) + cs * d); \
        hop<MU, SIG, NEG>(acc, r);                                                    \
    }
    CHDWF_SP_HOP(n_xp, 0, SF, false)
    CHDWF_SP_HOP(n_xm, 0, -SF, false)
    CHDWF_SP_HOP(n_yp, 1, SF, false)
    CHDWF_SP_HOP(n_ym, 1, -SF, false)
    CHDWF_SP_HOP(n_tp, 2, SF, false)
    CHDWF_SP_HOP(n_tm, 2, -SF, false)
    // kappa = 1/2 (:2815-2829)
#pragma unroll
    for (int d = 0; d < 4; d++) acc[d] = zscal(0.5f, acc[d]);
    // antiperiodic boundary in t (:2831-2876)
    if (apbc) {
        if (q.it == Lt - 1) CHDWF_SP_HOP(n_tp, 2, SF, true)
        if (q.it == 0) CHDWF_SP_HOP(n_tm, 2, -SF, true)
    }
#undef CHDWF_SP_HOP
    // s hops (:2879-2908; M^dagger :3313-3342): point 0 is s, point 1 is s+1
    constexpr int UP = DAG ? 0 : 2;
    constexpr int DN = DAG ? 2 : 0;
#pragma unroll
    for (int d = UP; d < UP + 2; d++) {
        const cpair c = ld_cpair(in, qp + fo + cs * d);
        acc[d].re.x = __fsub_rn(acc[d].re.x, c.re.y);
        acc[d].im.x = __fsub_rn(acc[d].im.x, c.im.y);
        if (q.s + 2 < Ls) {
            const cpair n = ld_cpair(in, qp + 2 + fo + cs * d);
            acc[d].re.y = __fsub_rn(acc[d].re.y, n.re.x);
            acc[d].im.y = __fsub_rn(acc[d].im.y, n.im.x);
        }
    }
#pragma unroll
    for (int d = DN; d < DN + 2; d++) {
        const cpair c = ld_cpair(in, qp + fo + cs * d);
        if (q.s > 0) {
            const cpair pv = ld_cpair(in, qp - 2 + fo + cs * d);
            acc[d].re.x = __fsub_rn(acc[d].re.x, pv.re.y);
            acc[d].im.x = __fsub_rn(acc[d].im.x, pv.im.y);
        }
        acc[d].re.y = __fsub_rn(acc[d].re.y, c.re.x);
        acc[d].im.y = __fsub_rn(acc[d].im.y, c.im.x);
    }
    // wall coupling: point 1 at s=Ls (pair WA, reads s=1), point 0 at s=1
    // (pair WB, reads s=Ls)
    constexpr int WA = DAG ? 0 : 2;
    constexpr int WB = DAG ? 2 : 0;
    const bool atL = (q.s + 2 == Ls), at0 = (q.s == 0);
    if (!(atL || at0)) return;
    const float c1f = __ldg(chif + q.site), c2f = __ldg(chif + g.kvol + q.site),
                c3f = __ldg(chif + 2 * g.kvol + q.site);
    const bool pin = (q.site == 0);
    if (atL && at0) {   // Ls = 2: one pair holds both walls
        float2 w0[4], w1[4];
#pragma unroll
        for (int d = 0; d < 4; d++) {
            w0[d] = cpair_pt(acc[d], 0);
            w1[d] = cpair_pt(acc[d], 1);
        }
        wall_terms<DAG, IMASS, WA, 0>(w1, LdSp{in}, cs, LsI * q.site, f, c1f, c2f, c3f, pin, hpin);
        wall_terms<DAG, IMASS, WB, 1>(w0, LdSp{in}, cs, LsI * q.site + Ls - 1, f, c1f, c2f, c3f,
                                      pin, hpin);
#pragma unroll
        for (int d = 0; d < 4; d++) {
            acc[d].re = make_float2(w0[d].x, w1[d].x);
            acc[d].im = make_float2(w0[d].y, w1[d].y);
        }
        return;
    }
    // one wall point: point 1 at s=Ls or point 0 at s=1, one code path
    float2 w[4];
#pragma unroll
    for (int d = 0; d < 4; d++) w[d] = cpair_pt(acc[d], atL ? 1 : 0);
    wall_terms_rt<DAG, IMASS>(w, LdSp{in}, (int64_t)cs,
                              atL ? (int64_t)LsI * q.site : (int64_t)LsI * q.site + Ls - 1, atL,
                              f, c1f, c2f, c3f, pin, hpin);
#pragma unroll
    for (int d = 0; d < 4; d++) {
        if (atL) {
            acc[d].re.y = w[d].x;
            acc[d].im.y = w[d].y;
        } else {
            acc[d].re.x = w[d].x;
            acc[d].im.x = w[d].y;
        }
    }
}

// Thread -> (point, flavour) map of the flavour-split kernels: a block of
// kSplitThreads threads covers kSplitThreads/2 consecutive points, the first
// half of its threads flavour 0 and the second half flavour 1, so every warp
// reads contiguous runs of one component plane.
constexpr int kSplitThreads = 256;
constexpr int kSplitPoints = kSplitThreads / 2;
__device__ __forceinline__ int split_flavour() { return threadIdx.x >= kSplitPoints; }
__device__ __forceinline__ int64_t split_point() {
    return (int64_t)blockIdx.x * kSplitPoints + (threadIdx.x & (kSplitPoints - 1));
}
inline unsigned split_blocks(int64_t npts) {
    return (unsigned)((npts + kSplitPoints - 1) / kSplitPoints);
}

}  // namespace chdwf
