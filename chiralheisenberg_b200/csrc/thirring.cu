// thirring.cu -- the bulk Thirring RHMC, bulk_rhmc.f, on the GPU: its link
// operator, multi-shift solver with the Phi0 register, link force, force and
// Hamiltonian with the Pauli-Villars terms, and main loop
// (include/chdwf_thirring.h).
//
// The operator is a chain of sweeps in the reference (diagonal, Wilson and
// Dirac hops through the links, s hops, wall mass term).  One thread per
// spinor element replays the chain for its element in FP64 with
// round-to-nearest intrinsics, so the result equals the sequential
// evaluation bit for bit.  derivs gives one thread to each link (site, mu)
// and adds its 8*kthird terms in the reference's order into a REAL*4
// register, also bit for bit.  The multi-shift solver and congrad run
// their scalar recurrences on the device, in the last block of each
// reduction, with the reference's implicit REAL*4 / REAL*8 types; the sums
// are FP64 block partials added in block order, and the host polls a stop
// flag once every 16 iterations instead of reading every scalar.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "chdwf_thirring.h"
#include "common.cuh"
#include "internal.h"
#include "rng.h"

namespace chdwf {
namespace {

constexpr int kThrMaxPoles = 25;
constexpr int kRedBlocks = 592;           // 4 per SM, fixed: partials summed in block order

struct TGeom {
    int L, Lt, Ls, kvol;
    int64_t kferm;                        // 4*kvol*Ls
};

// gamval(mu,idirac)*akappa, gamin(mu,idirac) - 1 (bulk_rhmc.f:1646-1722)
__constant__ double2 c_tgv[3][4] = {{{0., -0.5}, {0., -0.5}, {0., 0.5}, {0., 0.5}},
                                    {{-0.5, 0.}, {0.5, 0.}, {0.5, 0.}, {-0.5, 0.}},
                                    {{0., -0.5}, {0., 0.5}, {0., 0.5}, {0., -0.5}}};
__constant__ int c_tgi[3][4] = {{3, 2, 1, 0}, {3, 2, 1, 0}, {2, 3, 0, 1}};

__device__ __forceinline__ int64_t tsite(int L, int x, int y, int t) {
    return x + (int64_t)L * (y + (int64_t)L * t);
}

// the periodic neighbours up/down of site (x, y, t) in direction mu (addrc, :1746-1797)
__device__ __forceinline__ void tnbr(const TGeom& g, int x, int y, int t, int mu, int64_t* up,
                                     int64_t* dn) {
    if (mu == 0) {
        *up = tsite(g.L, x + 1 == g.L ? 0 : x + 1, y, t);
        *dn = tsite(g.L, x == 0 ? g.L - 1 : x - 1, y, t);
    } else if (mu == 1) {
        *up = tsite(g.L, x, y + 1 == g.L ? 0 : y + 1, t);
        *dn = tsite(g.L, x, y == 0 ? g.L - 1 : y - 1, t);
    } else {
        *up = tsite(g.L, x, y, t + 1 == g.Lt ? 0 : t + 1);
        *dn = tsite(g.L, x, y, t == 0 ? g.Lt - 1 : t - 1);
    }
}

// Site coordinates (site < kvol < 2^31): 32-bit divisions.
__device__ __forceinline__ void tsite_xyt(int L, int64_t site, int* x, int* y, int* t) {
    const uint32_t uL = (uint32_t)L, st = (uint32_t)site, xy = st / uL;
    *x = (int)(st - xy * uL);
    const uint32_t tt = xy / uL;
    *y = (int)(xy - tt * uL);
    *t = (int)tt;
}

// One element (s, site, d) of Phi = M R (DAG false, :1946-2069) or
// Phi = M^dagger R (DAG true, :2071-2188).
template <bool DAG, int IMASS>
__device__ double2 thr_element(const double2* __restrict__ R, const double2* __restrict__ u,
                               const TGeom& g, int s, int64_t i, int d, double diag, double2 zk) {
    const int L = g.L, Ls = g.Ls;
    const int64_t kvol = g.kvol;
    auto at = [&](int ss, int64_t st, int dd) -> double2 {
        return __ldg(R + ss + (int64_t)Ls * (st + kvol * dd));
    };
    int x, y, t;
    tsite_xyt(L, i, &x, &y, &t);
    int64_t up[3], dn[3];
#pragma unroll
    for (int mu = 0; mu < 3; mu++) tnbr(g, x, y, t, mu, &up[mu], &dn[mu]);
    double2 phi = zscal(diag, at(s, i, d));                                 // :1967-1974
#pragma unroll
    for (int mu = 0; mu < 3; mu++) {                                         // Wilson, :1976-1987
        const double2 uu = __ldg(u + i + kvol * mu), ud = zconj(__ldg(u + dn[mu] + kvol * mu));
        const double2 w = zadd(zmul(uu, at(s, up[mu], d)), zmul(ud, at(s, dn[mu], d)));
        phi = zsub(phi, zscal(0.5, w));
    }
#pragma unroll
    for (int mu = 0; mu < 3; mu++) {                                         // Dirac, :1989-2002
        const int dg = c_tgi[mu][d];
        const double2 uu = __ldg(u + i + kvol * mu), ud = zconj(__ldg(u + dn[mu] + kvol * mu));
        const double2 tt = zmul(c_tgv[mu][d], zsub(zmul(uu, at(s, up[mu], dg)),
                                                   zmul(ud, at(s, dn[mu], dg))));
        phi = DAG ? zsub(phi, tt) : zadd(phi, tt);
    }
    // s hops (:2004-2020): M takes Dirac 3,4 from s+1, Dirac 1,2 from s-1;
    // M^dagger the reverse (:2129-2145)
    const bool from_up = DAG ? d < 2 : d >= 2;
    if (from_up) {
        if (s < Ls - 1) phi = zsub(phi, at(s + 1, i, d));
    } else if (s > 0) {
        phi = zsub(phi, at(s - 1, i, d));
    }
    // mass term (:2022-2067, :2147-2186): group A at s=kthird (the pair that
    // takes s+1), group B at s=1 (the other pair)
    const bool grpA = s == Ls - 1 && from_up, grpB = s == 0 && !from_up;
    if (grpA || grpB) {
        double2 src;
        int sg;
        if (IMASS == 5) {
            src = at(s, i, d >= 2 ? d - 2 : d + 2);
            sg = -1;
        } else {
            src = at(grpA ? 0 : Ls - 1, i, d);
            sg = IMASS == 1 ? 1 : (grpA == !DAG ? -1 : 1);
        }
        const double2 tt = zmul(zk, src);
        phi = sg > 0 ? zadd(phi, tt) : zsub(phi, tt);
    }
    return phi;
}

// Stop state of a solve whose scalar recurrences run on the device: once
// done is set at iteration iters, the kernels queued for later iterations
// return at once (the host polls the flag only every few iterations).
struct ThrRun {
    int done, iters;   // done: 0 running, 1 converged, 2 at the iteration cap
};
__device__ __forceinline__ bool thr_skip(const ThrRun* run, int it) {
    return run != nullptr && run->done && it > run->iters;
}

template <bool DAG, int IMASS>
__global__ void __launch_bounds__(kThreads) k_thr_dslash(double2* __restrict__ out,
                                                         const double2* __restrict__ in,
                                                         const double2* __restrict__ u, TGeom g,
                                                         double diag, double2 zk,
                                                         const ThrRun* run, int it) {
    if (thr_skip(run, it)) return;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= g.kferm) return;
    if (g.kferm <= (int64_t)0xffffffffLL) {   // 32-bit divisions when every index fits
        const uint32_t uj = (uint32_t)j, Ls = (uint32_t)g.Ls, kv = (uint32_t)g.kvol;
        const uint32_t r = uj / Ls, d = r / kv;
        out[j] = thr_element<DAG, IMASS>(in, u, g, (int)(uj - r * Ls), (int64_t)(r - d * kv),
                                         (int)d, diag, zk);
        return;
    }
    const int s = (int)(j % g.Ls);
    const int64_t r = j / g.Ls;
    out[j] = thr_element<DAG, IMASS>(in, u, g, s, r % g.kvol, (int)(r / g.kvol), diag, zk);
}

// derivs (:820-878), one thread per link (i, mu): for Dirac d and s in the
// reference's order, the Wilson term then the Dirac term, each rounded to
// REAL*4 as it is added.
__global__ void __launch_bounds__(kThreads) k_thr_derivs(const double2* __restrict__ R,
                                                         const double2* __restrict__ X2, TGeom g,
                                                         double tz, int iflag,
                                                         float* __restrict__ dS) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= 3 * (int64_t)g.kvol) return;
    const int64_t kvol = g.kvol;
    const int mu = (int)((uint32_t)j / (uint32_t)kvol);    // j < 3 kvol < 2^32
    const int64_t i = j - (int64_t)mu * kvol;
    const int Ls = g.Ls;
    int x, y, t;
    tsite_xyt(g.L, i, &x, &y, &t);
    int64_t up, dn;
    tnbr(g, x, y, t, mu, &up, &dn);
    const double2 tzi = make_double2(0.0, tz);
    float f = dS[j];
    for (int d = 0; d < 4; d++) {
        const int dg = c_tgi[mu][d];
        const double2 tg = zmul(tzi, c_tgv[mu][d]);
        for (int s = 0; s < Ls; s++) {
            const double2 ri = zconj(R[s + (int64_t)Ls * (i + kvol * d)]);
            const double2 ru = zconj(R[s + (int64_t)Ls * (up + kvol * d)]);
            const double2 a = zmul(ri, X2[s + (int64_t)Ls * (up + kvol * d)]);
            const double2 b = zmul(ru, X2[s + (int64_t)Ls * (i + kvol * d)]);
            const double2 w = zmul(tzi, zsub(a, b));
            f = __double2float_rn(__dsub_rn((double)f, __dmul_rn(0.5, w.x)));     // :843-850
            const double2 a2 = zmul(ri, X2[s + (int64_t)Ls * (up + kvol * dg)]);
            const double2 b2 = zmul(ru, X2[s + (int64_t)Ls * (i + kvol * dg)]);
            const double2 w2 = zmul(tg, zadd(a2, b2));
            f = __double2float_rn(iflag == 0 ? __dsub_rn((double)f, w2.x)             // :851-868
                                             : __dadd_rn((double)f, w2.x));
        }
    }
    dS[j] = f;
}

// coef (:1799-1827)
__global__ void k_thr_coef(const float* __restrict__ theta, double2* __restrict__ u, TGeom g) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= 3 * (int64_t)g.kvol) return;
    double2 v = make_double2(1.0, (double)theta[j]);
    const int64_t i = j % g.kvol;
    if (j / g.kvol == 2 && i >= (int64_t)(g.Lt - 1) * g.L * g.L) v = make_double2(-v.x, -v.y);
    u[j] = v;
}

// ---- multi-shift solver kernels (qmrherm, :630-818) ------------------------
struct PoleCoef {
    double rho[kThrMaxPoles], amu[kThrMaxPoles];
};

// The solver's scalar recurrences run on the device, in thread 0 of the
// block that finishes a reduction last, with the reference's implicit types
// and the same operation order as a sequential host evaluation (no fused
// multiply-adds), so the iterates do not depend on where the scalars are
// formed.  The host only polls the stop flag every few iterations.
struct ThrQCtl {
    ThrRun run;
    int niterc, ndiag;
    float phimod, resid, alphatild, pad_;
    double beta;                                   // REAL*8 beta of :684-704
    double aden[kThrMaxPoles], d[kThrMaxPoles], rhom1[kThrMaxPoles];
    double rho[kThrMaxPoles], amu[kThrMaxPoles];
    unsigned count1, count2;
};

// Grid sum of one double per thread with the block partials added in block
// order by one thread (the order of a host loop over the partials).  The
// block that arrives last returns true with the total in *total (thread 0)
// and resets the counter.  NB is the fixed grid size of the reductions.
template <int NT, int NB>
__device__ __forceinline__ bool last_block_seq(double v, double* part, unsigned* count,
                                               double* total) {
    __shared__ double sh[NT / 32];
    __shared__ double all[NB];
    __shared__ bool is_last;
    v = block_sum<NT>(v, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = v;
        __threadfence();
        is_last = (atomicAdd(count, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    for (int i = threadIdx.x; i < NB; i += blockDim.x) all[i] = ((volatile double*)part)[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < NB; b++) s = __dadd_rn(s, all[b]);
        *total = s;
        *count = 0;
    }
    return true;
}

// q = R/beta (:684-686)
__global__ void k_thr_q(double2* __restrict__ q, const double2* __restrict__ R,
                        const ThrQCtl* __restrict__ c, int it, int64_t n) {
    if (thr_skip(&c->run, it)) return;
    const double beta = c->beta;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j < n) q[j] = make_double2(__ddiv_rn(R[j].x, beta), __ddiv_rn(R[j].y, beta));
}

// block partials of sum Re(conjg(a)*b); the host adds them in block order
__global__ void __launch_bounds__(kThreads) k_thr_dot(const double2* __restrict__ a,
                                                      const double2* __restrict__ b, int64_t n,
                                                      double* __restrict__ part) {
    __shared__ double sh[kThreads / 32];
    double loc = 0.0;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x)
        loc += zmul(zconj(a[j]), b[j]).x;
    loc = block_sum<kThreads>(loc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = loc;
}

// alphatild = sum Re(conjg(q)*x3), rounded once to REAL*4 (:688-694)
__global__ void __launch_bounds__(kThreads) k_thr_alpha(const double2* __restrict__ q,
                                                        const double2* __restrict__ x3, int64_t n,
                                                        double* __restrict__ part,
                                                        ThrQCtl* __restrict__ c, int it) {
    if (thr_skip(&c->run, it)) return;
    double loc = 0.0;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x)
        loc += zmul(zconj(q[j]), x3[j]).x;
    double tot;
    if (!last_block_seq<kThreads, kRedBlocks>(loc, part, &c->count1, &tot)) return;
    if (threadIdx.x == 0) c->alphatild = (float)tot;
}

// R = x3 - alphatild q - beta qm1 ; qm1 = q ; beta = |R| (:696-704), then
// the pole recurrences and the stopping test (:712-757) in the last block
__global__ void __launch_bounds__(kThreads) k_thr_lanczos(double2* __restrict__ R,
                                                          double2* __restrict__ qm1,
                                                          const double2* __restrict__ q,
                                                          const double2* __restrict__ x3, int64_t n,
                                                          double* __restrict__ part,
                                                          ThrQCtl* __restrict__ c, int it) {
    if (thr_skip(&c->run, it)) return;
    const double alphat = (double)c->alphatild, beta = c->beta;
    double loc = 0.0;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x) {
        const double2 qj = q[j];
        const double2 r = zsub(zsub(x3[j], zscal(alphat, qj)), zscal(beta, qm1[j]));
        R[j] = r;
        qm1[j] = qj;
        loc += zmul(zconj(r), r).x;
    }
    double b2;
    if (!last_block_seq<kThreads, kRedBlocks>(loc, part, &c->count2, &b2)) return;
    if (threadIdx.x != 0) return;
    const float beta0 = (float)beta;
    c->beta = __dsqrt_rn(b2);
    const int nd = c->ndiag;
    float rhomax = 0.0f;
    for (int k = 0; k < nd; k++) {
        const double alpha = __dadd_rn((double)c->alphatild, c->aden[k]);
        if (it == 1) {                                                     // :712-724
            c->d[k] = alpha;
            c->rho[k] = __ddiv_rn((double)beta0, alpha);
            c->rhom1[k] = c->rho[k];
        } else {                                                           // :725-747
            const double amu = __ddiv_rn((double)beta0, c->d[k]);
            const double dm1 = c->d[k];
            const double dk = __dsub_rn(alpha, __dmul_rn((double)beta0, amu));
            const double rho = -__ddiv_rn(__dmul_rn(__dmul_rn(amu, dm1), c->rhom1[k]), dk);
            c->amu[k] = amu;
            c->d[k] = dk;
            c->rho[k] = rho;
            const double rm = fabs(__dmul_rn((double)c->phimod, rho));
            if (k == 0) rhomax = (float)rm;
            else if (rm > (double)rhomax) rhomax = (float)rm;
            c->rhom1[k] = rho;
        }
    }
    const float arelax = 2.0f;                                             // :750-757
    if (it > 1 && rhomax < __fmul_rn(arelax, c->resid)) {
        c->run.iters = it;
        c->run.done = 1;
    } else if (it >= c->niterc) {
        c->run.iters = it;
        c->run.done = 2;
    }
}

// all poles at once: first iteration p_k = q, x_k = rho_k q; later
// p_k = q - amu_k p_k, x_k += rho_k p_k (:712-747; pm1 equals p).  Runs in
// the iteration that stopped the solve too.
__global__ void k_thr_poles(double2* __restrict__ p, double2* __restrict__ x1,
                            const double2* __restrict__ q, const ThrQCtl* __restrict__ c,
                            int it, int64_t n, int* hflag) {
    if (thr_skip(&c->run, it)) return;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j == 0 && c->run.done && hflag) {
        *(volatile int*)hflag = c->run.done;
        __threadfence_system();
    }
    if (j >= n) return;
    const double2 qj = q[j];
    const int nd = c->ndiag;
    for (int k = 0; k < nd; k++) {
        const int64_t e = j + n * k;
        const double rho = c->rho[k];
        if (it == 1) {
            p[e] = qj;
            x1[e] = zscal(rho, qj);
        } else {
            const double2 pk = zsub(qj, zscal(c->amu[k], p[e]));
            p[e] = pk;
            x1[e] = zadd(x1[e], zscal(rho, pk));
        }
    }
}

// x = anum0 Phi, then x += anum_k x_k in pole order (:666, :766-772)
__global__ void k_thr_combine(double2* __restrict__ x, const double2* __restrict__ Phi,
                              const double2* __restrict__ x1, PoleCoef c, double a0, int npole,
                              int64_t n) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n) return;
    double2 v = zscal(a0, Phi[j]);
    for (int k = 0; k < npole; k++) v = zadd(v, zscal(c.rho[k], x1[j + n * k]));
    x[j] = v;
}

// R = x3 - ... helpers for the leapfrog: pp -= dS*d ; theta += d*pp
__global__ void k_thr_update_p(float* __restrict__ pp, const float* __restrict__ dS, float d,
                               int64_t n) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j < n) pp[j] = __fsub_rn(pp[j], __fmul_rn(dS[j], d));
}
__global__ void k_thr_update_theta(float* __restrict__ th, const float* __restrict__ pp,
                                   float d, int64_t n) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j < n) th[j] = __fadd_rn(th[j], __fmul_rn(d, pp[j]));
}

// end of force (:520-532): the antiperiodic sign on the t links of the last
// slice, then dSdpi + beta*Nf*theta
__global__ void k_thr_force_end(float* __restrict__ dS, const float* __restrict__ theta,
                                float b, TGeom g) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= 3 * (int64_t)g.kvol) return;
    float v = dS[j];
    if (j / g.kvol == 2 && j % g.kvol >= (int64_t)(g.Lt - 1) * g.L * g.L) v = -v;
    dS[j] = __fadd_rn(v, __fmul_rn(b, theta[j]));
}

// R(s, i, d) = cmplx(ps(i,1), ps(i,2)) of gauss0 call d*kthird + s (:213-222)
__global__ void k_thr_noise(double2* __restrict__ R, const float* __restrict__ gauss, TGeom g) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= g.kferm) return;
    const int s = (int)(j % g.Ls);
    const int64_t r = j / g.Ls;
    const int64_t site = r % g.kvol;
    const int64_t c = (r / g.kvol) * g.Ls + s;
    const float* ps = gauss + c * 2 * g.kvol;
    R[j] = make_double2((double)ps[site], (double)ps[g.kvol + site]);
}

// ---- congrad (:931-1025) and measure (:1027-1285) -------------------------
// The REAL*4 scalars of congrad, formed on the device like those of qmrherm.
struct ThrCgCtl {
    ThrRun run;
    int64_t niterc;
    float alpha, alphan, betad, beta, resid, pad_;
    unsigned count1, count2;
};

// alphad = |x1|^2 ; alpha = alphan/alphad (:970-977)
__global__ void __launch_bounds__(kThreads) k_thr_cg_alpha(const double2* __restrict__ x1,
                                                           int64_t n, double* __restrict__ part,
                                                           ThrCgCtl* __restrict__ c, int it) {
    if (thr_skip(&c->run, it)) return;
    double loc = 0.0;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x)
        loc += zmul(zconj(x1[j]), x1[j]).x;
    double tot;
    if (!last_block_seq<kThreads, kRedBlocks>(loc, part, &c->count1, &tot)) return;
    if (threadIdx.x == 0) c->alpha = __fdiv_rn(c->alphan, (float)tot);
}

// x += alpha p (:979-983)
__global__ void k_thr_axpy(double2* __restrict__ x, const double2* __restrict__ p,
                           const ThrCgCtl* __restrict__ c, int it, int64_t n) {
    if (thr_skip(&c->run, it)) return;
    const double a = (double)c->alpha;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j < n) x[j] = zadd(x[j], zscal(a, p[j]));
}

// r -= alpha x2 ; betan = |r|^2, beta and the stopping test (:989-1001) in
// the last block
__global__ void __launch_bounds__(kThreads) k_thr_cg_r(double2* __restrict__ r,
                                                       const double2* __restrict__ x2, int64_t n,
                                                       double* __restrict__ part,
                                                       ThrCgCtl* __restrict__ c, int it,
                                                       int* hflag) {
    if (thr_skip(&c->run, it)) return;
    const double a = (double)c->alpha;
    double loc = 0.0;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x) {
        const double2 v = zsub(r[j], zscal(a, x2[j]));
        r[j] = v;
        loc += zmul(zconj(v), v).x;
    }
    double bn;
    if (!last_block_seq<kThreads, kRedBlocks>(loc, part, &c->count2, &bn)) return;
    if (threadIdx.x != 0) return;
    const float betan = (float)bn;
    float beta = __fdiv_rn(betan, c->betad);
    c->betad = betan;
    c->alphan = betan;
    if (it == 1) beta = 0.0f;
    c->beta = beta;
    if (betan < c->resid) {
        c->run.iters = it;
        c->run.done = 1;
    } else if (it >= c->niterc) {
        c->run.iters = it;
        c->run.done = 2;
    }
    if (c->run.done && hflag) {
        *(volatile int*)hflag = c->run.done;
        __threadfence_system();
    }
}

// p = r + beta p (:1003-1005); runs in the iteration that stopped the solve
__global__ void k_thr_xpay(double2* __restrict__ p, const double2* __restrict__ r,
                           const ThrCgCtl* __restrict__ c, int it, int64_t n) {
    if (thr_skip(&c->run, it)) return;
    const double b = (double)c->beta;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j < n) p[j] = zadd(r[j], zscal(b, p[j]));
}

// xi = 0 except component d at wall s: sgn*cmplx(eta(i,1), eta(i,2))
__global__ void k_thr_wall_source(double2* __restrict__ xi, const float* __restrict__ eta,
                                  int s, int d, double sgn, TGeom g) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= g.kferm) return;
    const int sj = (int)(j % g.Ls);
    const int64_t r = j / g.Ls;
    const int64_t i = r % g.kvol;
    const int dj = (int)(r / g.kvol);
    double2 v = make_double2(0.0, 0.0);
    if (sj == s && dj == d) v = make_double2(sgn * (double)eta[i], sgn * (double)eta[g.kvol + i]);
    xi[j] = v;
}

// out[i] = x(s, i, d)
__global__ void k_thr_slice(const double2* __restrict__ x, int s, int d, TGeom g,
                            double2* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < g.kvol) out[i] = x[s + (int64_t)g.Ls * (i + (int64_t)g.kvol * d)];
}

unsigned tblk(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

}  // namespace
}  // namespace chdwf

using chdwf::TGeom;

struct ThrRemez {
    std::vector<double> anum, aden, bnum, bden;
    int n = 0;
};

struct chdwf_thr {
    int device = 0;
    TGeom g{};
    float dt = 0.1f, beta = 0.5f, am3 = 1.0f, am = 0.0f;
    int imass = 1, iterl = 1, iprint = 5;
    float rescga = 0.000000001f, rescgg = 0.000001f;                   // :39
    float respbp = 0.000001f;                                            // :39
    ThrRemez r2, r4, r2g, r4g;
    cudaStream_t st = nullptr;
    float *theta = nullptr, *thetat = nullptr, *pp = nullptr, *dS = nullptr, *gauss = nullptr;
    double2 *ut = nullptr, *uio = nullptr;
    double2 *Phi = nullptr, *X1 = nullptr, *R = nullptr, *X2 = nullptr, *Phi0 = nullptr;
    double2 *q = nullptr, *qm1 = nullptr, *vt = nullptr, *x3 = nullptr, *rr = nullptr;
    double2 *p = nullptr, *x1 = nullptr;
    double* part = nullptr;
    std::vector<double> hpart;
    chdwf::ThrQCtl* qctl = nullptr;       // device scalars of qmrherm
    chdwf::ThrCgCtl* cgctl = nullptr;     // device scalars of congrad
    int* hflag_host = nullptr;            // stop flag, mapped pinned memory
    int* hflag_dev = nullptr;
    chdwf::Rng rng;
    int isweep = 0, itot = 0, naccp = 0;
    float action = 0.0f, gaction = 0.0f, paction = 0.0f;
    float actiona = 0.0f, vel2a = 0.0f, yav = 0.0f, yyav = 0.0f;
    std::string err;

    double diag() const { return (double)((3.0f - am3) + 1.0f); }       // :1967
    int fail(cudaError_t e, const char* where) {
        err = std::string(where) + ": " + cudaGetErrorString(e);
        return CHDWF_CUDA_ERROR;
    }
};

namespace {

thread_local std::string g_thr_create_err;

template <class T>
cudaError_t talloc(T** p, size_t n) { return cudaMalloc((void**)p, sizeof(T) * n); }

void thr_dslash(chdwf_thr* h, bool dag, float am, int imass, double2* out, const double2* in,
                const double2* u, const chdwf::ThrRun* run = nullptr, int it = 0) {
    const unsigned nb = chdwf::tblk(h->g.kferm);
    double2 zk = imass == 1 ? make_double2((double)am, 0.0)
                            : make_double2(0.0, dag ? (double)am : (double)(-am));
    const double dg = h->diag();
#define THR_LAUNCH(D, I) chdwf::k_thr_dslash<D, I><<<nb, chdwf::kThreads, 0, h->st>>>(out, in, u, h->g, dg, zk, run, it)
    if (dag) {
        if (imass == 1) THR_LAUNCH(true, 1); else if (imass == 3) THR_LAUNCH(true, 3); else THR_LAUNCH(true, 5);
    } else {
        if (imass == 1) THR_LAUNCH(false, 1); else if (imass == 3) THR_LAUNCH(false, 3); else THR_LAUNCH(false, 5);
    }
#undef THR_LAUNCH
    chdwf::count_launches(1);
}

void thr_derivs(chdwf_thr* h, const double2* R, const double2* X2, double anum, int iflag) {
    const double tz = (double)(float)(2.0 * anum);                         // tzi, :839
    chdwf::k_thr_derivs<<<chdwf::tblk(3 * (int64_t)h->g.kvol), chdwf::kThreads, 0, h->st>>>(
        R, X2, h->g, tz, iflag, h->dS);
    chdwf::count_launches(1);
}

// sum of the block partials in block order
cudaError_t thr_sum(chdwf_thr* h, double* out) {
    cudaMemcpyAsync(h->hpart.data(), h->part, sizeof(double) * chdwf::kRedBlocks,
                    cudaMemcpyDeviceToHost, h->st);
    const cudaError_t e = cudaStreamSynchronize(h->st);
    double s = 0.0;
    for (int b = 0; b < chdwf::kRedBlocks; b++) s = s + h->hpart[b];
    *out = s;
    return e;
}

// Launches iterations 1, 2, ... of a solve in chunks of 16 until the
// device raises the stop flag or cap iterations are queued.  The flag is
// read one chunk behind, so up to two chunks are in flight; the kernels of
// iterations past the stopping one return at once.
template <class F>
cudaError_t thr_run_chunks(chdwf_thr* h, int64_t cap, F&& launch_iteration) {
    const int chunk = 16;
    cudaEvent_t ev[2];
    cudaError_t e = cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
    if (e) return e;
    if ((e = cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming))) {
        cudaEventDestroy(ev[0]);
        return e;
    }
    int64_t launched = 0;
    int nchunk = 0;
    while (launched < cap) {
        for (int c = 0; c < chunk && launched < cap; c++) launch_iteration((int)++launched);
        if ((e = cudaGetLastError())) break;
        cudaEventRecord(ev[nchunk & 1], h->st);
        if (nchunk >= 1) {
            if ((e = cudaEventSynchronize(ev[(nchunk - 1) & 1]))) break;
            if (*(volatile int*)h->hflag_host) break;
        }
        nchunk++;
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    return e;
}

// qmrherm on device vectors (:630-818): Phi in, x out, Phi0 and dS of the
// context; the scalars follow the reference's implicit typing.
int thr_qmrherm(chdwf_thr* h, const double2* Phi, float res, int* itercg, float am, int imass,
                const double* anum, const double* aden, int ndiag, int iflag, const double2* u,
                double2* x) {
    const int64_t n = h->g.kferm;
    const unsigned nb = chdwf::tblk(n);
    const int niterc = 7500;                                             // :635
    const float resid = std::sqrt((float)n * res * res);                // :660
    cudaError_t e;
    cudaMemcpyAsync(h->rr, Phi, sizeof(double2) * n, cudaMemcpyDeviceToDevice, h->st);   // :662-667
    cudaMemsetAsync(h->qm1, 0, sizeof(double2) * n, h->st);
    chdwf::k_thr_dot<<<chdwf::kRedBlocks, chdwf::kThreads, 0, h->st>>>(h->rr, h->rr, n, h->part);
    chdwf::count_launches(1);
    double b0;
    if ((e = thr_sum(h, &b0))) return h->fail(e, "thr_qmrherm");
    chdwf::ThrQCtl hc;
    memset(&hc, 0, sizeof(hc));
    hc.beta = std::sqrt(b0);
    hc.phimod = (float)hc.beta;
    hc.resid = resid;
    hc.niterc = niterc;
    hc.ndiag = ndiag;
    for (int k = 0; k < ndiag; k++) hc.aden[k] = aden[k];
    if ((e = cudaMemcpyAsync(h->qctl, &hc, sizeof(hc), cudaMemcpyHostToDevice, h->st)))
        return h->fail(e, "thr_qmrherm");
    *h->hflag_host = 0;
    chdwf::ThrQCtl* c = h->qctl;
    const chdwf::ThrRun* run = &c->run;
    e = thr_run_chunks(h, niterc, [&](int it) {
        chdwf::k_thr_q<<<nb, chdwf::kThreads, 0, h->st>>>(h->q, h->rr, c, it, n);
        thr_dslash(h, false, am, imass, h->vt, h->q, u, run, it);
        thr_dslash(h, true, am, imass, h->x3, h->vt, u, run, it);
        chdwf::k_thr_alpha<<<chdwf::kRedBlocks, chdwf::kThreads, 0, h->st>>>(h->q, h->x3, n,
                                                                            h->part, c, it);
        chdwf::k_thr_lanczos<<<chdwf::kRedBlocks, chdwf::kThreads, 0, h->st>>>(
            h->rr, h->qm1, h->q, h->x3, n, h->part, c, it);
        chdwf::k_thr_poles<<<nb, chdwf::kThreads, 0, h->st>>>(h->p, h->x1, h->q, c, it, n,
                                                               h->hflag_dev);
        chdwf::count_launches(4);
    });
    if (e) return h->fail(e, "thr_qmrherm");
    chdwf::ThrRun hr;
    if ((e = cudaMemcpyAsync(&hr, run, sizeof(hr), cudaMemcpyDeviceToHost, h->st)) ||
        (e = cudaStreamSynchronize(h->st)))
        return h->fail(e, "thr_qmrherm");
    *itercg = hr.iters;
    const int capped = hr.done != 1;
    chdwf::PoleCoef c0;
    memset(&c0, 0, sizeof(c0));
    if (iflag < 2) {                                                       // :766-780
        chdwf::PoleCoef a;
        for (int k = 0; k < ndiag; k++) a.rho[k] = anum[k + 1];
        chdwf::k_thr_combine<<<nb, chdwf::kThreads, 0, h->st>>>(x, Phi, h->x1, a, anum[0], ndiag, n);
        chdwf::count_launches(1);
        if (iflag == 1)
            cudaMemcpyAsync(h->Phi0, h->x1, sizeof(double2) * n * ndiag, cudaMemcpyDeviceToDevice,
                            h->st);
    } else {                                                               // :781-806
        chdwf::k_thr_combine<<<nb, chdwf::kThreads, 0, h->st>>>(x, Phi, h->x1, c0, anum[0], 0, n);
        chdwf::count_launches(1);
        for (int k = 0; k < ndiag; k++) {
            const double2* xk = h->x1 + n * k;
            thr_dslash(h, false, am, imass, h->X2, xk, u);
            if (iflag == 2) {
                thr_derivs(h, xk, h->X2, anum[k + 1], 0);
            } else {
                const double coeff = -anum[k + 1];
                const double2* p0 = h->Phi0 + n * k;
                thr_derivs(h, p0, h->X2, coeff, 0);
                thr_dslash(h, false, am, imass, h->X2, p0, u);
                thr_derivs(h, h->X2, xk, coeff, 1);
            }
        }
    }
    if ((e = cudaGetLastError())) return h->fail(e, "thr_qmrherm");
    return capped ? CHDWF_ITER_CAP : CHDWF_OK;
}

// force (:449-535) on thetat/ut; its[4] receives the four solves' iterations
int thr_force(chdwf_thr* h, float res1, int* its) {
    const int64_t n = h->g.kferm;
    cudaMemsetAsync(h->dS, 0, sizeof(float) * 3 * h->g.kvol, h->st);   // :477-481
    int rc;
    const ThrRemez& a4 = h->r4g;
    const ThrRemez& r2 = h->r2g;
    rc = thr_qmrherm(h, h->Phi, res1, &its[0], 1.0f, 1, a4.anum.data(), a4.aden.data(), a4.n, 1,
                     h->ut, h->X1);                                       // :493
    if (rc != CHDWF_OK && rc != CHDWF_ITER_CAP) return rc;
    cudaMemcpyAsync(h->R, h->X1, sizeof(double2) * n, cudaMemcpyDeviceToDevice, h->st);
    rc = thr_qmrherm(h, h->R, res1, &its[1], h->am, h->imass, r2.bnum.data(), r2.bden.data(), r2.n,
                     0, h->ut, h->X1);                                    // :500
    if (rc != CHDWF_OK && rc != CHDWF_ITER_CAP) return rc;
    cudaMemcpyAsync(h->R, h->X1, sizeof(double2) * n, cudaMemcpyDeviceToDevice, h->st);
    rc = thr_qmrherm(h, h->R, res1, &its[2], h->am, h->imass, r2.anum.data(), r2.aden.data(), r2.n,
                     2, h->ut, h->X1);                                    // :509
    if (rc != CHDWF_OK && rc != CHDWF_ITER_CAP) return rc;
    rc = thr_qmrherm(h, h->R, res1, &its[3], 1.0f, 1, a4.anum.data(), a4.aden.data(), a4.n, 3,
                     h->ut, h->X1);                                       // :514
    if (rc != CHDWF_OK && rc != CHDWF_ITER_CAP) return rc;
    const float b = h->beta * 1.0f;                                       // b = beta*Nf, :527
    chdwf::k_thr_force_end<<<chdwf::tblk(3 * (int64_t)h->g.kvol), chdwf::kThreads, 0, h->st>>>(
        h->dS, h->thetat, b, h->g);
    chdwf::count_launches(1);
    const cudaError_t e = cudaGetLastError();
    return e ? h->fail(e, "thr_force") : CHDWF_OK;
}

// hamilton (:539-628): out = h, hg, hp, s; its = {mass m, PV}
int thr_hamilton(chdwf_thr* h, float res2, double* out, int* its) {
    const int64_t n = h->g.kferm, n3 = 3 * (int64_t)h->g.kvol;
    std::vector<float> pp(n3), th(n3);
    cudaMemcpyAsync(pp.data(), h->pp, sizeof(float) * n3, cudaMemcpyDeviceToHost, h->st);
    cudaMemcpyAsync(th.data(), h->thetat, sizeof(float) * n3, cudaMemcpyDeviceToHost, h->st);
    int rc = thr_qmrherm(h, h->Phi, res2, &its[1], 1.0f, 1, h->r4.anum.data(), h->r4.aden.data(),
                         h->r4.n, 0, h->ut, h->X1);                       // :596
    if (rc != CHDWF_OK && rc != CHDWF_ITER_CAP) return rc;
    cudaMemcpyAsync(h->R, h->X1, sizeof(double2) * n, cudaMemcpyDeviceToDevice, h->st);
    rc = thr_qmrherm(h, h->R, res2, &its[0], h->am, h->imass, h->r2.bnum.data(), h->r2.bden.data(),
                     h->r2.n, 0, h->ut, h->X1);                           // :603
    if (rc != CHDWF_OK && rc != CHDWF_ITER_CAP) return rc;
    chdwf::k_thr_dot<<<chdwf::kRedBlocks, chdwf::kThreads, 0, h->st>>>(h->R, h->X1, n, h->part);
    chdwf::count_launches(1);
    double hf;
    const cudaError_t e = thr_sum(h, &hf);                                 // :607-609
    if (e) return h->fail(e, "thr_hamilton");
    double hp = 0.0, hg = 0.0;
    for (int64_t j = 0; j < n3; j++) hp = hp + (double)(pp[j] * pp[j]);         // :571-575
    hp = hp * 0.5;
    for (int64_t j = 0; j < n3; j++) hg = hg + (double)(th[j] * th[j]);
    hg = (double)(0.5f * 1.0f * h->beta) * hg;                          // :581
    out[0] = hg + hp + hf;
    out[1] = hg;
    out[2] = hp;
    out[3] = hg + hf;
    return CHDWF_OK;
}

// congrad (:931-1025) on device vectors: x in = guess, out = solution;
// REAL*4 scalars, FP64 sums rounded once.  Returns CHDWF_ITER_CAP at the cap.
int thr_congrad(chdwf_thr* h, const double2* Phi, float res, int* itercg, float am, int imass,
                const double2* u, double2* x) {
    const int64_t n = h->g.kferm;
    const unsigned nb = chdwf::tblk(n);
    const int64_t niterc = h->g.Ls * (int64_t)h->g.kvol;                 // :934
    const float resid = (float)n * res * res;                            // :947
    double2 *p = h->q, *r = h->rr, *x1 = h->vt, *x2 = h->x3;
    cudaMemcpyAsync(p, x, sizeof(double2) * n, cudaMemcpyDeviceToDevice, h->st);   // :956-959
    cudaMemcpyAsync(r, Phi, sizeof(double2) * n, cudaMemcpyDeviceToDevice, h->st);
    chdwf::ThrCgCtl hc;
    memset(&hc, 0, sizeof(hc));
    hc.betad = 1.0f;                                                      // :951-952
    hc.alpha = 1.0f;
    hc.alphan = 0.0f;
    hc.resid = resid;
    hc.niterc = niterc;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(h->cgctl, &hc, sizeof(hc), cudaMemcpyHostToDevice, h->st)))
        return h->fail(e, "thr_congrad");
    *h->hflag_host = 0;
    chdwf::ThrCgCtl* c = h->cgctl;
    const chdwf::ThrRun* run = &c->run;
    e = thr_run_chunks(h, niterc, [&](int it) {
        thr_dslash(h, false, am, imass, x1, p, u, run, it);               // :966
        if (it != 1) {                                                    // :970-983
            chdwf::k_thr_cg_alpha<<<chdwf::kRedBlocks, chdwf::kThreads, 0, h->st>>>(x1, n, h->part,
                                                                                   c, it);
            chdwf::k_thr_axpy<<<nb, chdwf::kThreads, 0, h->st>>>(x, p, c, it, n);
            chdwf::count_launches(2);
        }
        thr_dslash(h, true, am, imass, x2, x1, u, run, it);               // :987
        chdwf::k_thr_cg_r<<<chdwf::kRedBlocks, chdwf::kThreads, 0, h->st>>>(r, x2, n, h->part, c,
                                                                          it, h->hflag_dev);
        chdwf::k_thr_xpay<<<nb, chdwf::kThreads, 0, h->st>>>(p, r, c, it, n);
        chdwf::count_launches(2);
    });
    if (e) return h->fail(e, "thr_congrad");
    chdwf::ThrRun hr;
    if ((e = cudaMemcpyAsync(&hr, run, sizeof(hr), cudaMemcpyDeviceToHost, h->st)) ||
        (e = cudaStreamSynchronize(h->st)))
        return h->fail(e, "thr_congrad");
    *itercg = hr.iters;
    return hr.done == 1 ? CHDWF_OK : CHDWF_ITER_CAP;
}

// measure (:1027-1285) with links u: psibarpsi, susclsing, aviter and the
// unit-100 records (parts, 40 doubles, or NULL).  Noise from the context's
// generator (two gauss0 calls per noise vector); the overlaps are summed on
// the host in the reference's order.
int thr_measure(chdwf_thr* h, float res, float am, int imass, const double2* u, float* psibarpsi,
                float* susclsing, float* aviter, double* parts) {
    const TGeom& g = h->g;
    const int64_t kvol = g.kvol, n = g.kferm;
    const int Ls = g.Ls;
    constexpr int knoise = 10;
    std::vector<float> ps(2 * kvol), pt(2 * kvol);
    std::vector<double2> slice(kvol);
    double pbp[knoise];
    int iter = 0;
    double2* xi = h->X2;
    double2* Phi = h->R;
    for (int inoise = 0; inoise < knoise; inoise++) {
        h->rng.gauss0(kvol, ps.data());                                   // :1061
        h->rng.gauss0(kvol, pt.data());                                   // :1063
        double p1r = 0.0, p1i = 0.0, p2r = 0.0, p2i = 0.0;
        for (int idsource = 1; idsource <= 2; idsource++) {
            for (int w = 0; w < 2; w++) {
                const float* nz = w == 0 ? ps.data() : pt.data();
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
                const int s_src = w == 0 ? 0 : Ls - 1;
                cudaMemcpyAsync(h->gauss, nz, sizeof(float) * 2 * kvol, cudaMemcpyHostToDevice, h->st);
                chdwf::k_thr_wall_source<<<chdwf::tblk(n), chdwf::kThreads, 0, h->st>>>(
                    xi, h->gauss, s_src, dsrc - 1, sgn, g);
                chdwf::count_launches(1);
                thr_dslash(h, true, am, imass, Phi, xi, u);               // :1136, :1220
                int it = 0;
                const int rc = thr_congrad(h, Phi, res, &it, am, imass, u, xi);   // :1138, :1225
                if (rc != CHDWF_OK && rc != CHDWF_ITER_CAP) return rc;
                iter += it;
                const int s_rd = imass != 5 ? (w == 0 ? Ls - 1 : 0) : s_src;
                chdwf::k_thr_slice<<<chdwf::tblk(kvol), chdwf::kThreads, 0, h->st>>>(xi, s_rd, dn - 1,
                                                                                 g, h->X1);
                chdwf::count_launches(1);
                cudaMemcpyAsync(slice.data(), h->X1, sizeof(double2) * kvol, cudaMemcpyDeviceToHost,
                                h->st);
                const cudaError_t e = cudaStreamSynchronize(h->st);
                if (e) return h->fail(e, "thr_measure");
                double ar = w == 0 ? p1r : p2r, ai = w == 0 ? p1i : p2i;
                for (int64_t i = 0; i < kvol; i++) {                      // conjg(x)*xi, in order
                    const double xr = (double)nz[i], xim = (double)nz[kvol + i];
                    const double yr = slice[i].x, yi = slice[i].y;
                    ar = ar + (xr * yr - (-xim) * yi);
                    ai = ai + (xr * yi + (-xim) * yr);
                }
                if (w == 0) { p1r = ar; p1i = ai; } else { p2r = ar; p2i = ai; }
            }
        }
        const double kv = (double)kvol;
        if (imass == 1) {                                                 // :1245-1257
            p1r = p1r / kv; p1i = p1i / kv; p2r = p2r / kv; p2i = p2i / kv;
        } else {
            // (0,-1)*p1 ; (0,+1)*p2 (imass 3) or (0,-1)*p2 (imass 5), as complex products
            const double s2 = imass == 3 ? 1.0 : -1.0;
            const double a1 = 0.0 * p1r - (-1.0) * p1i, b1 = 0.0 * p1i + (-1.0) * p1r;
            const double a2 = 0.0 * p2r - s2 * p2i, b2 = 0.0 * p2i + s2 * p2r;
            p1r = a1 / kv; p1i = b1 / kv; p2r = a2 / kv; p2i = b2 / kv;
        }
        pbp[inoise] = p1r + p2r;
        if (parts) {
            parts[4 * inoise] = p1r; parts[4 * inoise + 1] = p1i;
            parts[4 * inoise + 2] = p2r; parts[4 * inoise + 3] = p2i;
        }
    }
    float pb = 0.0f, sus = 0.0f;                                          // :1266-1276
    for (int i = 0; i < knoise; i++) {
        pb = (float)((double)pb + pbp[i]);
        for (int j = knoise - 1; j >= i + 1; j--) sus = (float)((double)sus + pbp[i] * pbp[j]);
    }
    *psibarpsi = pb / (float)knoise;
    *susclsing = (float)(2 * kvol) * sus / (float)(knoise * (knoise - 1));
    *aviter = (float)iter / (float)(4 * knoise);                          // :1278
    return CHDWF_OK;
}

chdwf_thr* thr_ok(chdwf_thr* h) {
    if (h) cudaSetDevice(h->device);
    return h;
}

int thr_apply(chdwf_thr* h, bool dag, double* Phi, const double* R, const double* u, float am,
              int imass) {
    if (!thr_ok(h) || !Phi || !R || !u || (imass != 1 && imass != 3 && imass != 5))
        return CHDWF_BAD_ARG;
    const int64_t n = h->g.kferm;
    cudaMemcpyAsync(h->R, R, sizeof(double2) * n, cudaMemcpyHostToDevice, h->st);
    cudaMemcpyAsync(h->uio, u, sizeof(double2) * 3 * h->g.kvol, cudaMemcpyHostToDevice, h->st);
    thr_dslash(h, dag, am, imass, h->X2, h->R, h->uio);
    cudaMemcpyAsync(Phi, h->X2, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->st);
    const cudaError_t e = cudaStreamSynchronize(h->st);
    return e ? h->fail(e, "thr_dslash") : CHDWF_OK;
}

}  // namespace

extern "C" {

int chdwf_thr_create(chdwf_thr** out, int ksize, int ksizet, int kthird, float dt, float beta,
                     float am3, float am, int imass, int iterl, int device) {
    if (!out) return CHDWF_BAD_ARG;
    *out = nullptr;
    if (!chdwf::geom_ok(ksize, ksizet, kthird) || (imass != 1 && imass != 3 && imass != 5) ||
        iterl < 1) {
        g_thr_create_err = "chdwf_thr_create: bad lattice, imass or iterl";
        return CHDWF_BAD_ARG;
    }
    chdwf_thr* h = new chdwf_thr;
    h->device = device;
    h->g.L = ksize; h->g.Lt = ksizet; h->g.Ls = kthird;
    h->g.kvol = ksize * ksize * ksizet;
    h->g.kferm = 4 * (int64_t)h->g.kvol * kthird;
    h->dt = dt; h->beta = beta; h->am3 = am3; h->am = am; h->imass = imass; h->iterl = iterl;
    const int64_t n3 = 3 * (int64_t)h->g.kvol, n = h->g.kferm;
    const int np = chdwf::kThrMaxPoles;
    cudaError_t e = cudaSetDevice(device);
    if (!e) e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
    if (!e) e = talloc(&h->theta, n3);
    if (!e) e = talloc(&h->thetat, n3);
    if (!e) e = talloc(&h->pp, n3);
    if (!e) e = talloc(&h->dS, n3);
    if (!e) e = talloc(&h->gauss, 8 * (size_t)h->g.kvol * kthird);
    if (!e) e = talloc(&h->ut, n3);
    if (!e) e = talloc(&h->uio, n3);
    for (double2** v : {&h->Phi, &h->X1, &h->R, &h->X2, &h->q, &h->qm1, &h->vt, &h->x3, &h->rr})
        if (!e) e = talloc(v, n);
    if (!e) e = talloc(&h->Phi0, n * np);
    if (!e) e = talloc(&h->p, n * np);
    if (!e) e = talloc(&h->x1, n * np);
    if (!e) e = talloc(&h->part, chdwf::kRedBlocks);
    if (!e) e = talloc(&h->qctl, 1);
    if (!e) e = talloc(&h->cgctl, 1);
    if (!e) e = cudaHostAlloc((void**)&h->hflag_host, sizeof(int), cudaHostAllocMapped);
    if (!e) e = cudaHostGetDevicePointer((void**)&h->hflag_dev, h->hflag_host, 0);
    if (!e) e = cudaMemsetAsync(h->theta, 0, sizeof(float) * n3, h->st);
    if (!e) e = cudaMemsetAsync(h->Phi0, 0, sizeof(double2) * n * np, h->st);
    if (!e) e = cudaStreamSynchronize(h->st);
    if (e) {
        g_thr_create_err = std::string("chdwf_thr_create: ") + cudaGetErrorString(e);
        chdwf_thr_destroy(h);
        return CHDWF_CUDA_ERROR;
    }
    h->hpart.resize(chdwf::kRedBlocks);
    h->rng.startup((double)693764523745.0f);
    *out = h;
    return CHDWF_OK;
}

void chdwf_thr_destroy(chdwf_thr* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->st) cudaStreamSynchronize(h->st);
    for (float* v : {h->theta, h->thetat, h->pp, h->dS, h->gauss}) if (v) cudaFree(v);
    for (double2* v : {h->ut, h->uio, h->Phi, h->X1, h->R, h->X2, h->Phi0, h->q, h->qm1, h->vt,
                       h->x3, h->rr, h->p, h->x1})
        if (v) cudaFree(v);
    if (h->part) cudaFree(h->part);
    if (h->qctl) cudaFree(h->qctl);
    if (h->cgctl) cudaFree(h->cgctl);
    if (h->hflag_host) cudaFreeHost(h->hflag_host);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

const char* chdwf_thr_last_error(chdwf_thr* h) {
    return h ? h->err.c_str() : g_thr_create_err.c_str();
}

int chdwf_thr_set_remez(chdwf_thr* h, int which, const double* anum, const double* aden,
                        const double* bnum, const double* bden, int ndiag) {
    if (!h || !anum || !aden || !bnum || !bden || ndiag < 1 || ndiag > chdwf::kThrMaxPoles)
        return CHDWF_BAD_ARG;
    ThrRemez* r = which == 2 ? &h->r2 : which == 4 ? &h->r4 : which == 22 ? &h->r2g
                : which == 44 ? &h->r4g : nullptr;
    if (!r) return CHDWF_BAD_ARG;
    r->anum.assign(anum, anum + ndiag + 1);
    r->aden.assign(aden, aden + ndiag);
    r->bnum.assign(bnum, bnum + ndiag + 1);
    r->bden.assign(bden, bden + ndiag);
    r->n = ndiag;
    return CHDWF_OK;
}

int chdwf_thr_coef(chdwf_thr* h, const float* theta, double* u) {
    if (!thr_ok(h) || !theta || !u) return CHDWF_BAD_ARG;
    const int64_t n3 = 3 * (int64_t)h->g.kvol;
    cudaMemcpyAsync(h->dS, theta, sizeof(float) * n3, cudaMemcpyHostToDevice, h->st);
    chdwf::k_thr_coef<<<chdwf::tblk(n3), chdwf::kThreads, 0, h->st>>>(h->dS, h->uio, h->g);
    chdwf::count_launches(1);
    cudaMemcpyAsync(u, h->uio, sizeof(double2) * n3, cudaMemcpyDeviceToHost, h->st);
    const cudaError_t e = cudaStreamSynchronize(h->st);
    return e ? h->fail(e, "thr_coef") : CHDWF_OK;
}

int chdwf_thr_dslash(chdwf_thr* h, double* Phi, const double* R, const double* u, float am,
                     int imass) {
    return thr_apply(h, false, Phi, R, u, am, imass);
}

int chdwf_thr_dslashd(chdwf_thr* h, double* Phi, const double* R, const double* u, float am,
                      int imass) {
    return thr_apply(h, true, Phi, R, u, am, imass);
}

int chdwf_thr_derivs(chdwf_thr* h, const double* R, const double* X2, double anum, int iflag,
                     float* dSdpi) {
    if (!thr_ok(h) || !R || !X2 || !dSdpi || (iflag != 0 && iflag != 1)) return CHDWF_BAD_ARG;
    const int64_t n = h->g.kferm, n3 = 3 * (int64_t)h->g.kvol;
    cudaMemcpyAsync(h->R, R, sizeof(double2) * n, cudaMemcpyHostToDevice, h->st);
    cudaMemcpyAsync(h->X1, X2, sizeof(double2) * n, cudaMemcpyHostToDevice, h->st);
    cudaMemcpyAsync(h->dS, dSdpi, sizeof(float) * n3, cudaMemcpyHostToDevice, h->st);
    thr_derivs(h, h->R, h->X1, anum, iflag);
    cudaMemcpyAsync(dSdpi, h->dS, sizeof(float) * n3, cudaMemcpyDeviceToHost, h->st);
    const cudaError_t e = cudaStreamSynchronize(h->st);
    return e ? h->fail(e, "thr_derivs") : CHDWF_OK;
}

int chdwf_thr_qmrherm(chdwf_thr* h, const double* Phi, float res, int* itercg, float am,
                      int imass, const double* anum, const double* aden, int ndiag, int iflag,
                      const double* u, double* x, double* Phi0, float* dSdpi) {
    if (!thr_ok(h) || !Phi || !itercg || !anum || !aden || !u || !x ||
        ndiag < 1 || ndiag > chdwf::kThrMaxPoles || iflag < 0 || iflag > 3 ||
        (imass != 1 && imass != 3 && imass != 5) || (iflag >= 1 && !Phi0) ||
        (iflag >= 2 && !dSdpi))
        return CHDWF_BAD_ARG;
    const int64_t n = h->g.kferm, n3 = 3 * (int64_t)h->g.kvol;
    cudaMemcpyAsync(h->Phi, Phi, sizeof(double2) * n, cudaMemcpyHostToDevice, h->st);
    cudaMemcpyAsync(h->uio, u, sizeof(double2) * n3, cudaMemcpyHostToDevice, h->st);
    if (iflag == 3)
        cudaMemcpyAsync(h->Phi0, Phi0, sizeof(double2) * n * ndiag, cudaMemcpyHostToDevice, h->st);
    if (iflag >= 2) cudaMemcpyAsync(h->dS, dSdpi, sizeof(float) * n3, cudaMemcpyHostToDevice, h->st);
    const int rc = thr_qmrherm(h, h->Phi, res, itercg, am, imass, anum, aden, ndiag, iflag, h->uio,
                               h->X1);
    if (rc != CHDWF_OK && rc != CHDWF_ITER_CAP) return rc;
    cudaMemcpyAsync(x, h->X1, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->st);
    if (iflag == 1)
        cudaMemcpyAsync(Phi0, h->Phi0, sizeof(double2) * n * ndiag, cudaMemcpyDeviceToHost, h->st);
    if (iflag >= 2) cudaMemcpyAsync(dSdpi, h->dS, sizeof(float) * n3, cudaMemcpyDeviceToHost, h->st);
    const cudaError_t e = cudaStreamSynchronize(h->st);
    if (e) return h->fail(e, "thr_qmrherm");
    return rc;
}

int chdwf_thr_congrad(chdwf_thr* h, const double* Phi, float res, int* itercg, float am,
                      int imass, const double* u, double* x) {
    if (!thr_ok(h) || !Phi || !itercg || !u || !x || (imass != 1 && imass != 3 && imass != 5))
        return CHDWF_BAD_ARG;
    const int64_t n = h->g.kferm;
    cudaMemcpyAsync(h->R, Phi, sizeof(double2) * n, cudaMemcpyHostToDevice, h->st);
    cudaMemcpyAsync(h->X2, x, sizeof(double2) * n, cudaMemcpyHostToDevice, h->st);
    cudaMemcpyAsync(h->uio, u, sizeof(double2) * 3 * h->g.kvol, cudaMemcpyHostToDevice, h->st);
    const int rc = thr_congrad(h, h->R, res, itercg, am, imass, h->uio, h->X2);
    if (rc != CHDWF_OK && rc != CHDWF_ITER_CAP) return rc;
    cudaMemcpyAsync(x, h->X2, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->st);
    const cudaError_t e = cudaStreamSynchronize(h->st);
    return e ? h->fail(e, "thr_congrad") : rc;
}

int chdwf_thr_measure(chdwf_thr* h, float res, const double* u, float* psibarpsi,
                      float* susclsing, float* aviter, double* parts) {
    if (!thr_ok(h) || !u || !psibarpsi || !susclsing || !aviter) return CHDWF_BAD_ARG;
    cudaMemcpyAsync(h->uio, u, sizeof(double2) * 3 * h->g.kvol, cudaMemcpyHostToDevice, h->st);
    return thr_measure(h, res, h->am, h->imass, h->uio, psibarpsi, susclsing, aviter, parts);
}

int chdwf_thr_set_measure(chdwf_thr* h, int iprint) {
    if (!h || iprint < 1) return CHDWF_BAD_ARG;
    h->iprint = iprint;
    return CHDWF_OK;
}

int chdwf_thr_set_theta(chdwf_thr* h, const float* theta) {
    if (!thr_ok(h) || !theta) return CHDWF_BAD_ARG;
    cudaMemcpyAsync(h->theta, theta, sizeof(float) * 3 * h->g.kvol, cudaMemcpyHostToDevice, h->st);
    const cudaError_t e = cudaStreamSynchronize(h->st);
    return e ? h->fail(e, "thr_set_theta") : CHDWF_OK;
}

int chdwf_thr_get_theta(chdwf_thr* h, float* theta) {
    if (!thr_ok(h) || !theta) return CHDWF_BAD_ARG;
    cudaMemcpyAsync(theta, h->theta, sizeof(float) * 3 * h->g.kvol, cudaMemcpyDeviceToHost, h->st);
    const cudaError_t e = cudaStreamSynchronize(h->st);
    return e ? h->fail(e, "thr_get_theta") : CHDWF_OK;
}

int chdwf_thr_startup(chdwf_thr* h, double seed) {
    if (!h) return CHDWF_BAD_ARG;
    h->rng.startup(seed);
    return CHDWF_OK;
}

double chdwf_thr_seed(chdwf_thr* h) { return h ? h->rng.seed() : 0.0; }

int chdwf_thr_sweep(chdwf_thr* h, chdwf_thr_record* rec) {
    if (!thr_ok(h) || !rec) return CHDWF_BAD_ARG;
    if (h->r2.n < 1 || h->r4.n < 1 || h->r2g.n < 1 || h->r4g.n < 1) {
        h->err = "thr_sweep: set remez2, remez4, remez2g and remez4g first";
        return CHDWF_BAD_ARG;
    }
    memset(rec, 0, sizeof(*rec));
    const TGeom& g = h->g;
    const int64_t kvol = g.kvol, n = g.kferm, n3 = 3 * kvol;
    const unsigned nb3 = chdwf::tblk(n3);
    int rc;
#define CK(x) do { rc = (x); if (rc != CHDWF_OK && rc != CHDWF_ITER_CAP) return rc; } while (0)
#define CKC(x, w) do { cudaError_t e_ = (x); if (e_) return h->fail(e_, w); } while (0)
    h->isweep++;
    cudaMemcpyAsync(h->thetat, h->theta, sizeof(float) * n3, cudaMemcpyDeviceToDevice, h->st);  // :203-208
    chdwf::k_thr_coef<<<nb3, chdwf::kThreads, 0, h->st>>>(h->thetat, h->ut, g);
    chdwf::count_launches(1);
    std::vector<float> gauss(8 * (size_t)kvol * g.Ls);                    // :213-222
    for (int c = 0; c < 4 * g.Ls; c++) h->rng.gauss0(kvol, gauss.data() + (size_t)c * 2 * kvol);
    CKC(cudaMemcpyAsync(h->gauss, gauss.data(), sizeof(float) * gauss.size(),
                        cudaMemcpyHostToDevice, h->st), "thr_sweep");
    chdwf::k_thr_noise<<<chdwf::tblk(n), chdwf::kThreads, 0, h->st>>>(h->R, h->gauss, g);
    chdwf::count_launches(1);
    CK(thr_qmrherm(h, h->R, h->rescga, &rec->it_pf, h->am, h->imass, h->r4.anum.data(),
                   h->r4.aden.data(), h->r4.n, 0, h->ut, h->X1));          // :226
    cudaMemcpyAsync(h->R, h->X1, sizeof(double2) * n, cudaMemcpyDeviceToDevice, h->st);
    CK(thr_qmrherm(h, h->R, h->rescga, &rec->it_pfpv, 1.0f, 1, h->r4.bnum.data(),
                   h->r4.bden.data(), h->r4.n, 0, h->ut, h->X1));          // :236
    cudaMemcpyAsync(h->Phi, h->X1, sizeof(double2) * n, cudaMemcpyDeviceToDevice, h->st);
    std::vector<float> ps(2 * kvol), pp(n3);                               // :255-260
    for (int mu = 0; mu < 3; mu++) {
        h->rng.gaussp(kvol, ps.data());
        memcpy(pp.data() + kvol * mu, ps.data(), sizeof(float) * kvol);
    }
    CKC(cudaMemcpyAsync(h->pp, pp.data(), sizeof(float) * n3, cudaMemcpyHostToDevice, h->st),
        "thr_sweep");
    double hh[4];
    int ih[2];
    CK(thr_hamilton(h, h->rescga, hh, ih));                               // :265
    rec->it_h0 = ih[0];
    rec->it_h0pv = ih[1];
    rec->H0 = hh[0];
    rec->S0 = hh[3];
    if (h->isweep == 1) {                                                  // :267-271
        h->action = (float)(hh[3] / (double)kvol);
        h->gaction = (float)(hh[1] / (double)kvol);
        h->paction = (float)(hh[2] / (double)kvol);
    }
    int fi[4];
    CK(thr_force(h, h->rescgg, fi));                                      // :276
    for (int k = 0; k < 4; k++) rec->it_force[k] += fi[k];
    rec->nforce++;
    float d = h->dt * 0.5f;
    chdwf::k_thr_update_p<<<nb3, chdwf::kThreads, 0, h->st>>>(h->pp, h->dS, d, n3);
    chdwf::count_launches(1);
    const float proby = 1.0f / (float)h->iterl;                           // :151
    for (int iter = 1; iter <= 1000; iter++) {                            // :285-320
        d = h->dt;
        chdwf::k_thr_update_theta<<<nb3, chdwf::kThreads, 0, h->st>>>(h->thetat, h->pp, d, n3);
        chdwf::k_thr_coef<<<nb3, chdwf::kThreads, 0, h->st>>>(h->thetat, h->ut, g);
        chdwf::count_launches(2);
        CK(thr_force(h, h->rescgg, fi));
        for (int k = 0; k < 4; k++) rec->it_force[k] += fi[k];
        rec->nforce++;
        rec->nsteps = iter;
        const float ytest = h->rng.rano_yran();                            // :302
        if (ytest < proby) {
            d = h->dt * 0.5f;
            chdwf::k_thr_update_p<<<nb3, chdwf::kThreads, 0, h->st>>>(h->pp, h->dS, d, n3);
            chdwf::count_launches(1);
            h->itot = h->itot + iter;
            break;
        }
        d = h->dt;
        chdwf::k_thr_update_p<<<nb3, chdwf::kThreads, 0, h->st>>>(h->pp, h->dS, d, n3);
        chdwf::count_launches(1);
    }
    CK(thr_hamilton(h, h->rescga, hh, ih));                               // :325
    rec->it_h1 = ih[0];
    rec->it_h1pv = ih[1];
    rec->H1 = hh[0];
    rec->S1 = hh[3];
    rec->hg = hh[1];
    rec->hp = hh[2];
    rec->dH = rec->H0 - rec->H1;
    rec->dS = rec->S0 - rec->S1;
    rec->y = (float)std::exp(rec->dH);                                    // :330
    h->yav = h->yav + rec->y;
    h->yyav = h->yyav + rec->y * rec->y;
    int accept = 1;
    if (rec->dH < 0.0) {                                                  // :333-336
        rec->x = h->rng.rano_yran();
        rec->drew_x = 1;
        if (rec->x > rec->y) accept = 0;
    }
    if (accept) {                                                         // :338-348
        cudaMemcpyAsync(h->theta, h->thetat, sizeof(float) * n3, cudaMemcpyDeviceToDevice, h->st);
        h->naccp = h->naccp + 1;
        h->action = (float)(rec->S1 / (double)kvol);
        h->gaction = (float)(rec->hg / (double)kvol);
        h->paction = (float)(rec->hp / (double)kvol);
    }
    rec->accepted = accept;
    rec->action = h->action;
    rec->gaction = h->gaction;
    rec->paction = h->paction;
    h->actiona = h->actiona + h->action;                                  // :350
    CKC(cudaMemcpyAsync(pp.data(), h->pp, sizeof(float) * n3, cudaMemcpyDeviceToHost, h->st),
        "thr_sweep");
    CKC(cudaStreamSynchronize(h->st), "thr_sweep");
    float vel2 = 0.0f;                                                    // :351-357
    for (int64_t j = 0; j < n3; j++) vel2 = vel2 + pp[j] * pp[j];
    rec->vel2 = vel2 / (float)(3 * kvol);
    h->vel2a = h->vel2a + rec->vel2;
    if ((h->isweep / h->iprint) * h->iprint == h->isweep) {               // :361-371
        cudaMemcpyAsync(h->thetat, h->theta, sizeof(float) * n3, cudaMemcpyDeviceToDevice, h->st);
        chdwf::k_thr_coef<<<nb3, chdwf::kThreads, 0, h->st>>>(h->thetat, h->ut, g);
        chdwf::count_launches(1);
        float sus = 0.0f;
        CK(thr_measure(h, h->respbp, h->am, h->imass, h->ut, &rec->pbp, &sus, &rec->ancgm,
                       nullptr));
        rec->measured = 1;
    }
    CKC(cudaGetLastError(), "thr_sweep");
#undef CK
#undef CKC
    return CHDWF_OK;
}

}  // extern "C"
