// hmc.cu -- the HMC predecessor of the RHMC code, mh/cheisdwf_hmc.f, on the
// GPU: its single-precision operator, CGNE solver, chi force and main loop
// (include/chdwf_hmc.h).
//
// The reference applies the operator as a chain of sweeps over the whole
// field (diagonal, Wilson hops, antiperiodic correction, Dirac hops, their
// correction, s hops, wall coupling).  Each output element receives its
// updates in that fixed order, so one thread per element replays the chain
// in registers and the result is bit-identical, as long as every REAL*4
// operation is rounded the same way: all complex arithmetic here uses
// round-to-nearest intrinsics, never fused multiply-add.
//
// The solver keeps the reference's REAL*4 scalars; its two sums of squares
// are accumulated in FP64 over a fixed reduction tree and rounded once (the
// reference adds element by element in REAL*4, an order no parallel sum can
// follow).  The random numbers are drawn on the host by the reference's
// generator in the reference's order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cg.h"
#include "chdwf_hmc.h"
#include "common.cuh"
#include "internal.h"
#include "rng.h"

namespace chdwf {
namespace {

// ---- REAL*4 complex arithmetic, rounded per operation --------------------
__device__ __forceinline__ float2 fc_add(float2 a, float2 b) {
    return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}
__device__ __forceinline__ float2 fc_sub(float2 a, float2 b) {
    return make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y));
}
__device__ __forceinline__ float2 fc_scal(float s, float2 a) {
    return make_float2(__fmul_rn(s, a.x), __fmul_rn(s, a.y));
}
__device__ __forceinline__ float2 fc_mul(float2 a, float2 b) {
    return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                       __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float2 fc_conj(float2 a) { return make_float2(a.x, -a.y); }

// gamval(mu,idirac)*akappa and gamin(mu,idirac) - 1 for mu = 1, 2, 3
// (mh/cheisdwf_hmc.f:1060-1094, scaled by akappa at :1132-1136)
__constant__ float2 c_gv[3][4] = {{{0.f, -0.5f}, {0.f, -0.5f}, {0.f, 0.5f}, {0.f, 0.5f}},
                                  {{-0.5f, 0.f}, {0.5f, 0.f}, {0.5f, 0.f}, {-0.5f, 0.f}},
                                  {{0.f, -0.5f}, {0.f, 0.5f}, {0.f, 0.5f}, {0.f, -0.5f}}};
__constant__ int c_gi[3][4] = {{3, 2, 1, 0}, {3, 2, 1, 0}, {2, 3, 0, 1}};

struct Elem {
    int s, x, y, t, d, f;
    int64_t site;
};

// Site coordinates (site < kvol < 2^31): 32-bit divisions.
__device__ __forceinline__ void site_xyt(const Geom& g, uint32_t site, int* x, int* y, int* t) {
    const uint32_t L = (uint32_t)g.L, xy = site / L;
    *x = (int)(site - xy * L);
    const uint32_t tt = xy / L;
    *y = (int)(xy - tt * L);
    *t = (int)tt;
}

// Element j -> (s, site, d, f): in 32-bit arithmetic when every element
// index fits (the 64-bit divisions it replaces are software routines).
__device__ __forceinline__ Elem elem_of(const Geom& g, int64_t j) {
    Elem e;
    int c;
    if (g.kferm <= (int64_t)0xffffffffLL) {
        const uint32_t u = (uint32_t)j, Ls = (uint32_t)g.Ls, kv = (uint32_t)g.kvol;
        const uint32_t r = u / Ls;
        e.s = (int)(u - r * Ls);
        const uint32_t cc = r / kv;
        e.site = (int64_t)(r - cc * kv);
        c = (int)cc;
    } else {
        e.s = (int)(j % g.Ls);
        const int64_t r = j / g.Ls;
        e.site = r % g.kvol;
        c = (int)(r / g.kvol);
    }
    e.d = c & 3;
    e.f = c >> 2;
    site_xyt(g, (uint32_t)e.site, &e.x, &e.y, &e.t);
    return e;
}

// One element (s, site, d, f) of Phi = M R (DAG false: mh/cheisdwf_hmc.f:1334-1681)
// or Phi = M^dagger R (DAG true: :1683-2028), updates applied in the order of
// the reference's sweeps.
template <bool DAG, int IMASS>
__device__ float2 hmc_element(const float2* __restrict__ R, const Geom& g, int s, int ix, int iy,
                              int it, int d, int f, const float* __restrict__ chi, float diag,
                              bool apbc) {
    const int L = g.L, Lt = g.Lt, Ls = g.Ls;
    const int64_t kvol = g.kvol;
    auto site = [L](int x, int y, int t) -> int64_t { return x + (int64_t)L * (y + (int64_t)L * t); };
    auto at = [&](int ss, int64_t st, int dd, int ff) -> float2 {
        return __ldg(R + ss + (int64_t)Ls * (st + kvol * (dd + 4 * ff)));
    };
    const int xp = ix + 1 == L ? 0 : ix + 1, xm = ix == 0 ? L - 1 : ix - 1;
    const int yp = iy + 1 == L ? 0 : iy + 1, ym = iy == 0 ? L - 1 : iy - 1;
    const int tp = it + 1 == Lt ? 0 : it + 1, tm = it == 0 ? Lt - 1 : it - 1;
    const int64_t i0 = site(ix, iy, it);
    const int64_t nb[3][2] = {{site(xp, iy, it), site(xm, iy, it)},
                              {site(ix, yp, it), site(ix, ym, it)},
                              {site(ix, iy, tp), site(ix, iy, tm)}};
    float2 phi = fc_scal(diag, at(s, i0, d, f));                        // :1351-1365
#pragma unroll
    for (int mu = 0; mu < 3; mu++)                                         // Wilson, :1367-1411
        phi = fc_sub(phi, fc_scal(0.5f, fc_add(at(s, nb[mu][0], d, f), at(s, nb[mu][1], d, f))));
    if (apbc) {                                                            // :1412-1437
        if (it == Lt - 1) phi = fc_add(phi, at(s, site(ix, iy, 0), d, f));
        if (it == 0) phi = fc_add(phi, at(s, site(ix, iy, Lt - 1), d, f));
    }
#pragma unroll
    for (int mu = 0; mu < 3; mu++) {                                       // Dirac, :1438-1490
        const int dg = c_gi[mu][d];
        const float2 t = fc_mul(c_gv[mu][d], fc_sub(at(s, nb[mu][0], dg, f), at(s, nb[mu][1], dg, f)));
        phi = DAG ? fc_sub(phi, t) : fc_add(phi, t);
    }
    if (apbc) {                                                            // :1491-1516
        const int dg = c_gi[2][d];
        const float2 g2 = make_float2(__fmul_rn(2.0f, c_gv[2][d].x), __fmul_rn(2.0f, c_gv[2][d].y));
        if (it == Lt - 1) {
            const float2 t = fc_mul(g2, at(s, site(ix, iy, 0), dg, f));
            phi = DAG ? fc_add(phi, t) : fc_sub(phi, t);
        }
        if (it == 0) {
            const float2 t = fc_mul(g2, at(s, site(ix, iy, Lt - 1), dg, f));
            phi = DAG ? fc_sub(phi, t) : fc_add(phi, t);
        }
    }
    // s hops (:1518-1546): M takes Dirac 3,4 from s+1 and Dirac 1,2 from
    // s-1; M^dagger the reverse (:1867-1895)
    const bool upper = d >= 2;
    const bool from_up = DAG ? !upper : upper;
    if (from_up) {
        if (s < Ls - 1) phi = fc_sub(phi, at(s + 1, i0, d, f));
    } else if (s > 0) {
        phi = fc_sub(phi, at(s - 1, i0, d, f));
    }
    // wall coupling (:1549-1679, :1897-2026).  Group A: s=kthird, the pair
    // that takes s+1 (M: Dirac 3,4), reading s=1; group B: s=1, the other
    // pair, reading s=kthird.  Stage 1 couples equal flavours through spm1,
    // stage 2 the other flavour through spm2 (flavour 2: conjg(spm2)).
    int sr = -1;
    if (s == Ls - 1 && from_up) sr = 0;
    else if (s == 0 && !from_up) sr = Ls - 1;
    if (sr >= 0) {
        const bool grpA = sr == 0;
        const float c1 = chi[i0], c2 = chi[kvol + i0], c3 = chi[2 * kvol + i0];
#pragma unroll
        for (int stage = 0; stage < 2; stage++) {
            float2 spm;
            int sg;
            if (IMASS == 1) {
                spm = stage == 0 ? make_float2(c3, 0.0f) : make_float2(c1, -c2);
                sg = (stage == 0 && f == 1) ? -1 : 1;
            } else {
                if (stage == 0) spm = make_float2(0.0f, DAG ? -c3 : c3);
                else spm = DAG ? make_float2(-c2, -c1) : make_float2(c2, c1);
                const int first = (grpA == !DAG) ? -1 : 1;    // sign for flavour 1
                sg = f == 0 ? first : -first;
            }
            float2 t;
            if (stage == 0) t = fc_mul(spm, at(sr, i0, d, f));
            else if (f == 0) t = fc_mul(spm, at(sr, i0, d, 1));
            else t = fc_mul(fc_conj(spm), at(sr, i0, d, 0));
            phi = sg > 0 ? fc_add(phi, t) : fc_sub(phi, t);
        }
    }
    return phi;
}

template <bool DAG, int IMASS>
__global__ void __launch_bounds__(kThreads) k_hmc_dslash(float2* __restrict__ out,
                                                         const float2* __restrict__ in,
                                                         const float* __restrict__ chi, Geom g,
                                                         float diag, int apbc) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= g.kferm) return;
    const Elem e = elem_of(g, j);
    out[j] = hmc_element<DAG, IMASS>(in, g, e.s, e.x, e.y, e.t, e.d, e.f, chi, diag, apbc != 0);
}

// ---- congrad (mh/cheisdwf_hmc.f:625-716) ----------------------------------
struct HcgArgs {
    Geom g;
    float2 *x, *p, *r, *x1;
    const float* chi;
    float diag;
    int apbc;
    CgCtl* ctl;
    double* part;
    int* hflag;
};

// x1 = M p ; alphad = |x1|^2 ; alpha = alphan/alphad  (:657-667)
template <int IMASS>
__global__ void __launch_bounds__(kThreads) k_hcg1(HcgArgs a) {
    CgCtl* c = a.ctl;
    if (c->done) return;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double loc = 0.0;
    if (j < a.g.kferm) {
        const Elem e = elem_of(a.g, j);
        const float2 v = hmc_element<false, IMASS>(a.p, a.g, e.s, e.x, e.y, e.t, e.d, e.f, a.chi,
                                                   a.diag, a.apbc != 0);
        a.x1[j] = v;
        loc = (double)__fmul_rn(v.x, v.x) + (double)__fmul_rn(v.y, v.y);
    }
    double tot;
    if (!last_block_total<kThreads>(loc, a.part, &c->count1, &tot)) return;
    if (threadIdx.x == 0 && c->nx > 1) c->alpha = c->alphan / (float)tot;
}

// x2 = M^dagger x1 ; x += alpha p (nx > 1) ; r -= alpha x2 ; betan = |r|^2,
// beta, stopping test  (:671-704)
template <int IMASS>
__global__ void __launch_bounds__(kThreads) k_hcg2(HcgArgs a) {
    CgCtl* c = a.ctl;
    if (c->done) return;
    const int nx = c->nx;
    const float alpha = c->alpha;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double loc = 0.0;
    if (j < a.g.kferm) {
        const Elem e = elem_of(a.g, j);
        const float2 v = hmc_element<true, IMASS>(a.x1, a.g, e.s, e.x, e.y, e.t, e.d, e.f, a.chi,
                                                  a.diag, a.apbc != 0);
        if (nx > 1) a.x[j] = fc_add(a.x[j], fc_scal(alpha, a.p[j]));
        const float2 r = fc_sub(a.r[j], fc_scal(alpha, v));
        a.r[j] = r;
        loc = (double)__fmul_rn(r.x, r.x) + (double)__fmul_rn(r.y, r.y);
    }
    double tot;
    if (!last_block_total<kThreads>(loc, a.part, &c->count2, &tot)) return;
    if (threadIdx.x == 0) {
        const float betan = (float)tot;
        float beta = betan / c->betad;
        c->betad = betan;
        c->alphan = betan;
        if (nx == 1) beta = 0.0f;
        c->beta = beta;
        if (betan < c->resid) {
            c->done = 1;
            c->iters = nx;
        } else if (nx >= c->niterc) {
            c->done = 2;
            c->iters = nx;
        }
        if (!(betan == betan)) { c->done = 3; c->iters = nx; }
        if (c->done && a.hflag) {
            *(volatile int*)a.hflag = c->done;
            __threadfence_system();
        }
        if (!c->done) c->nx = nx + 1;
    }
}

// p = r + beta p  (:700-702)
__global__ void __launch_bounds__(kThreads) k_hcg3(HcgArgs a) {
    CgCtl* c = a.ctl;
    if (c->done) return;
    const float beta = c->beta;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j < a.g.kferm) a.p[j] = fc_add(a.r[j], fc_scal(beta, a.p[j]));
}

// ---- force, Hamiltonian and the leapfrog updates ---------------------------
// dSdchi of force for X1 (:416-420, :445-555), one thread per site: the wall
// elements of X2 = M X1 are formed in-thread, then the products are added
// in the reference's order (Dirac 1, 2 on X1(kthird) x X2(1), then Dirac 3,
// 4 on X1(1) x X2(kthird)) and the sum is doubled.
template <int IMASS>
__global__ void __launch_bounds__(kThreads) k_hmc_derivs(const float2* __restrict__ X1,
                                                         const float* __restrict__ chi, Geom g,
                                                         float b2, float diag, int apbc,
                                                         float* __restrict__ dS) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= g.kvol) return;
    const int64_t kvol = g.kvol;
    const int Ls = g.Ls;
    int ix, iy, it;
    site_xyt(g, (uint32_t)i, &ix, &iy, &it);
    float d1 = __fmul_rn(b2, chi[i]), d2 = __fmul_rn(b2, chi[kvol + i]);
    float d3 = __fmul_rn(b2, chi[2 * kvol + i]);
    for (int grp = 0; grp < 2; grp++) {
        const int d0 = grp == 0 ? 0 : 2;
        const int s1 = grp == 0 ? Ls - 1 : 0, s2 = grp == 0 ? 0 : Ls - 1;
        for (int d = d0; d < d0 + 2; d++) {
            const float2 a1 = fc_conj(X1[s1 + (int64_t)Ls * (i + kvol * d)]);
            const float2 a2 = fc_conj(X1[s1 + (int64_t)Ls * (i + kvol * (d + 4))]);
            const float2 y1 = hmc_element<false, IMASS>(X1, g, s2, ix, iy, it, d, 0, chi, diag,
                                                        apbc != 0);
            const float2 y2 = hmc_element<false, IMASS>(X1, g, s2, ix, iy, it, d, 1, chi, diag,
                                                        apbc != 0);
            const float2 p12 = fc_mul(a1, y2), p21 = fc_mul(a2, y1);
            const float2 p11 = fc_mul(a1, y1), p22 = fc_mul(a2, y2);
            if (IMASS == 1) {                                              // :453-500
                d1 = __fsub_rn(d1, p12.x); d1 = __fsub_rn(d1, p21.x);
                d2 = __fsub_rn(d2, p12.y); d2 = __fadd_rn(d2, p21.y);
                d3 = __fsub_rn(d3, p11.x); d3 = __fadd_rn(d3, p22.x);
            } else if (grp == 0) {                                         // :501-526
                d1 = __fsub_rn(d1, p12.y); d1 = __fsub_rn(d1, p21.y);
                d2 = __fadd_rn(d2, p12.x); d2 = __fsub_rn(d2, p21.x);
                d3 = __fsub_rn(d3, p11.y); d3 = __fadd_rn(d3, p22.y);
            } else {                                                       // :527-549
                d1 = __fadd_rn(d1, p12.y); d1 = __fadd_rn(d1, p21.y);
                d2 = __fsub_rn(d2, p12.x); d2 = __fadd_rn(d2, p21.x);
                d3 = __fadd_rn(d3, p11.y); d3 = __fsub_rn(d3, p22.y);
            }
        }
    }
    dS[i] = __fmul_rn(2.0f, d1);                                           // :550-554
    dS[kvol + i] = __fmul_rn(2.0f, d2);
    dS[2 * kvol + i] = __fmul_rn(2.0f, d3);
}

// R(s, i, d, f) = cmplx(ps(i,1), ps(i,2)) of gauss0 call (f*4 + d)*kthird + s
// (:154-162); gauss holds the calls' ps arrays back to back
__global__ void k_hmc_noise(float2* __restrict__ R, const float* __restrict__ gauss, Geom g) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= g.kferm) return;
    const int s = (int)(j % g.Ls);
    const int64_t r = j / g.Ls;
    const int64_t site = r % g.kvol;
    const int64_t c = (r / g.kvol) * g.Ls + s;
    const float* ps = gauss + c * 2 * g.kvol;
    R[j] = make_float2(ps[site], ps[g.kvol + site]);
}

// X0 = 2*X1 - X0  (:434-439)
__global__ void k_hmc_extrap(float2* __restrict__ X0, const float2* __restrict__ X1, int64_t n) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j < n) X0[j] = fc_sub(fc_scal(2.0f, X1[j]), X0[j]);
}

// pp = pp - dSdchi*d  (:204-207, :231-234, :239-242)
__global__ void k_hmc_update_p(float* __restrict__ pp, const float* __restrict__ dS, float d,
                               int64_t n) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j < n) pp[j] = __fsub_rn(pp[j], __fmul_rn(dS[j], d));
}

// chit = chit + d*pp  (:216-219)
__global__ void k_hmc_update_chi(float* __restrict__ chit, const float* __restrict__ pp, float d,
                                 int64_t n) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j < n) chit[j] = __fadd_rn(chit[j], __fmul_rn(d, pp[j]));
}

// block partials of hf = sum Re(conjg(Phi)*X1), each product in REAL*4
// (:606-611); the host adds the partials in block order
__global__ void __launch_bounds__(kThreads) k_hmc_hf(const float2* __restrict__ Phi,
                                                     const float2* __restrict__ X1, int64_t n,
                                                     double* __restrict__ part) {
    __shared__ double sh[kThreads / 32];
    double loc = 0.0;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x) {
        const float2 a = fc_conj(Phi[j]), b = X1[j];
        loc += (double)__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
    }
    loc = block_sum<kThreads>(loc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = loc;
}

constexpr int kHfBlocks = 592;    // 4 per SM

unsigned nblk(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

}  // namespace
}  // namespace chdwf

using chdwf::Geom;

struct chdwf_hmc {
    int device = 0;
    Geom g{};
    float dt = 0.1f, beta = 0.5f, am3 = 1.0f, am = 0.0f;
    int imass = 1, iterl = 1, iprint = 5;
    float rescga = 0.000000001f, rescgg = 0.000001f;                   // :35
    cudaStream_t st = nullptr;
    float *chi = nullptr, *chit = nullptr, *pp = nullptr, *dS = nullptr, *chi_io = nullptr;
    float2 *Phi = nullptr, *X0 = nullptr, *X1 = nullptr, *R = nullptr;
    float2 *cp = nullptr, *cr = nullptr, *cx1 = nullptr;
    float* gauss = nullptr;
    double* part = nullptr;
    chdwf::CgCtl* ctl = nullptr;
    int* hflag_host = nullptr;
    int* hflag_dev = nullptr;
    chdwf::Rng rng;
    int isweep = 0, itot = 0, naccp = 0;
    float action = 0.0f, gaction = 0.0f, paction = 0.0f;
    float actiona = 0.0f, vel2a = 0.0f, yav = 0.0f, yyav = 0.0f;
    std::string err;

    float diag() const { return (3.0f - am3) + 1.0f; }                  // :1351
    int fail(cudaError_t e, const char* where) {
        err = std::string(where) + ": " + cudaGetErrorString(e);
        return CHDWF_CUDA_ERROR;
    }
};

namespace {

thread_local std::string g_hmc_create_err;

template <class T>
cudaError_t dalloc(T** p, size_t n) { return cudaMalloc((void**)p, sizeof(T) * n); }

void launch_dslash(chdwf_hmc* h, bool dag, int imass, float2* out, const float2* in,
                   const float* chi) {
    const unsigned nb = chdwf::nblk(h->g.kferm);
    const float dg = h->diag();
    if (dag) {
        if (imass == 3) chdwf::k_hmc_dslash<true, 3><<<nb, chdwf::kThreads, 0, h->st>>>(out, in, chi, h->g, dg, 1);
        else chdwf::k_hmc_dslash<true, 1><<<nb, chdwf::kThreads, 0, h->st>>>(out, in, chi, h->g, dg, 1);
    } else {
        if (imass == 3) chdwf::k_hmc_dslash<false, 3><<<nb, chdwf::kThreads, 0, h->st>>>(out, in, chi, h->g, dg, 1);
        else chdwf::k_hmc_dslash<false, 1><<<nb, chdwf::kThreads, 0, h->st>>>(out, in, chi, h->g, dg, 1);
    }
    chdwf::count_launches(1);
}

// congrad on device vectors: x in = guess, out = solution.  status 0
// converged, 1 at the cap kthird*kvol, 2 non-finite.
cudaError_t hcg_solve(chdwf_hmc* h, const float2* phi, float res, int imass, const float* chi,
                      float2* x, int* itercg, int* status) {
    const Geom& g = h->g;
    chdwf::CgCtl hc;
    memset(&hc, 0, sizeof(hc));
    hc.nx = 1;
    hc.alpha = 1.0f;                                                    // :651-652
    hc.betad = 1.0f;
    hc.resid = (float)g.kferm * res * res;                              // :638
    hc.niterc = (int)(g.Ls * (int64_t)g.kvol);
    cudaError_t e;
    if ((e = cudaMemcpyAsync(h->ctl, &hc, sizeof(hc), cudaMemcpyHostToDevice, h->st))) return e;
    *h->hflag_host = 0;
    cudaMemcpyAsync(h->cp, x, sizeof(float2) * g.kferm, cudaMemcpyDeviceToDevice, h->st);   // :647-650
    cudaMemcpyAsync(h->cr, phi, sizeof(float2) * g.kferm, cudaMemcpyDeviceToDevice, h->st);
    chdwf::HcgArgs a;
    memset(&a, 0, sizeof(a));
    a.g = g;
    a.x = x; a.p = h->cp; a.r = h->cr; a.x1 = h->cx1;
    a.chi = chi;
    a.diag = h->diag();
    a.apbc = 1;
    a.ctl = h->ctl;
    a.part = h->part;
    a.hflag = h->hflag_dev;
    const unsigned nb = chdwf::nblk(g.kferm);
    const int chunk = 16;
    cudaEvent_t ev[2];
    cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
    int64_t launched = 0;
    int nchunk = 0;
    const int64_t cap = hc.niterc;
    while (launched < cap) {
        for (int c = 0; c < chunk && launched < cap; c++, launched++) {
            if (imass == 3) {
                chdwf::k_hcg1<3><<<nb, chdwf::kThreads, 0, h->st>>>(a);
                chdwf::k_hcg2<3><<<nb, chdwf::kThreads, 0, h->st>>>(a);
            } else {
                chdwf::k_hcg1<1><<<nb, chdwf::kThreads, 0, h->st>>>(a);
                chdwf::k_hcg2<1><<<nb, chdwf::kThreads, 0, h->st>>>(a);
            }
            chdwf::k_hcg3<<<nb, chdwf::kThreads, 0, h->st>>>(a);
            chdwf::count_launches(3);
        }
        cudaEventRecord(ev[nchunk & 1], h->st);
        if (nchunk >= 1) {
            cudaEventSynchronize(ev[(nchunk - 1) & 1]);
            if (*(volatile int*)h->hflag_host) break;
        }
        nchunk++;
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if ((e = cudaGetLastError())) return e;
    chdwf::CgCtl hr;
    if ((e = cudaMemcpyAsync(&hr, h->ctl, sizeof(hr), cudaMemcpyDeviceToHost, h->st))) return e;
    if ((e = cudaStreamSynchronize(h->st))) return e;
    *itercg = hr.iters;
    *status = hr.done == 1 ? 0 : (hr.done == 2 ? 1 : 2);
    return cudaSuccess;
}

void launch_derivs(chdwf_hmc* h, int imass, const float2* X1, const float* chi, float* dS) {
    const unsigned nb = chdwf::nblk(h->g.kvol);
    const float b2 = 2.0f * h->beta;                                    // :418
    if (imass == 3) chdwf::k_hmc_derivs<3><<<nb, chdwf::kThreads, 0, h->st>>>(X1, chi, h->g, b2, h->diag(), 1, dS);
    else chdwf::k_hmc_derivs<1><<<nb, chdwf::kThreads, 0, h->st>>>(X1, chi, h->g, b2, h->diag(), 1, dS);
    chdwf::count_launches(1);
}

// force (mh/cheisdwf_hmc.f:393-557) on chit: X1 = X0 ; congrad ; X0 = 2 X1 - X0 ;
// dSdchi from X1
int hmc_force(chdwf_hmc* h, float res1, int* itercg) {
    const Geom& g = h->g;
    cudaMemcpyAsync(h->X1, h->X0, sizeof(float2) * g.kferm, cudaMemcpyDeviceToDevice, h->st);
    int stt = 0;
    cudaError_t e = hcg_solve(h, h->Phi, res1, h->imass, h->chit, h->X1, itercg, &stt);
    if (e) return h->fail(e, "force");
    if (stt == 2) { h->err = "force: non-finite solver residual"; return CHDWF_NONFINITE; }
    chdwf::k_hmc_extrap<<<chdwf::nblk(g.kferm), chdwf::kThreads, 0, h->st>>>(h->X0, h->X1, g.kferm);
    chdwf::count_launches(1);
    launch_derivs(h, h->imass, h->X1, h->chit, h->dS);
    if ((e = cudaGetLastError())) return h->fail(e, "force");
    return CHDWF_OK;
}

// hamilton (mh/cheisdwf_hmc.f:561-623) on chit and pp: out = h, hg, hp, s
int hmc_hamilton(chdwf_hmc* h, float res2, double* out, int* itercg) {
    const Geom& g = h->g;
    const int64_t n3 = 3 * (int64_t)g.kvol;
    std::vector<float> pp(n3), chi(n3);
    cudaMemcpyAsync(pp.data(), h->pp, sizeof(float) * n3, cudaMemcpyDeviceToHost, h->st);
    cudaMemcpyAsync(chi.data(), h->chit, sizeof(float) * n3, cudaMemcpyDeviceToHost, h->st);
    cudaMemcpyAsync(h->X1, h->X0, sizeof(float2) * g.kferm, cudaMemcpyDeviceToDevice, h->st);  // :601-603
    int stt = 0;
    cudaError_t e = hcg_solve(h, h->Phi, res2, h->imass, h->chit, h->X1, itercg, &stt);        // :605
    if (e) return h->fail(e, "hamilton");
    if (stt == 2) { h->err = "hamilton: non-finite solver residual"; return CHDWF_NONFINITE; }
    cudaMemcpyAsync(h->X0, h->X1, sizeof(float2) * g.kferm, cudaMemcpyDeviceToDevice, h->st);  // :608
    chdwf::k_hmc_hf<<<chdwf::kHfBlocks, chdwf::kThreads, 0, h->st>>>(h->Phi, h->X1, g.kferm, h->part);
    chdwf::count_launches(1);
    std::vector<double> part(chdwf::kHfBlocks);
    cudaMemcpyAsync(part.data(), h->part, sizeof(double) * chdwf::kHfBlocks, cudaMemcpyDeviceToHost,
                    h->st);
    if ((e = cudaStreamSynchronize(h->st))) return h->fail(e, "hamilton");
    double hp = 0.0, hg = 0.0, hf = 0.0;
    for (int64_t j = 0; j < n3; j++) hp = hp + (double)(pp[j] * pp[j]);         // :582-587
    hp = hp * 0.5;
    for (int64_t j = 0; j < n3; j++) hg = hg + (double)(chi[j] * chi[j]);       // :589-594
    hg = (double)(2.0f * h->beta) * hg;
    for (int b = 0; b < chdwf::kHfBlocks; b++) hf = hf + part[b];
    out[0] = hg + hp + hf;
    out[1] = hg;
    out[2] = hp;
    out[3] = hg + hf;
    return CHDWF_OK;
}

chdwf_hmc* as_ok(chdwf_hmc* h) {
    if (h) cudaSetDevice(h->device);
    return h;
}

int hmc_apply(chdwf_hmc* h, bool dag, float* Phi, const float* R, const float* chi, int imass) {
    if (!as_ok(h) || !Phi || !R || !chi || (imass != 1 && imass != 3)) return CHDWF_BAD_ARG;
    const Geom& g = h->g;
    cudaMemcpyAsync(h->R, R, sizeof(float2) * g.kferm, cudaMemcpyHostToDevice, h->st);
    cudaMemcpyAsync(h->chi_io, chi, sizeof(float) * 3 * g.kvol, cudaMemcpyHostToDevice, h->st);
    launch_dslash(h, dag, imass, h->X1, h->R, h->chi_io);
    cudaMemcpyAsync(Phi, h->X1, sizeof(float2) * g.kferm, cudaMemcpyDeviceToHost, h->st);
    const cudaError_t e = cudaStreamSynchronize(h->st);
    return e ? h->fail(e, dag ? "hmc_dslashd" : "hmc_dslash") : CHDWF_OK;
}

}  // namespace

extern "C" {

int chdwf_hmc_create(chdwf_hmc** out, int ksize, int ksizet, int kthird, float dt, float beta,
                     float am3, float am, int imass, int iterl, int device) {
    if (!out) return CHDWF_BAD_ARG;
    *out = nullptr;
    if (!chdwf::geom_ok(ksize, ksizet, kthird) || (imass != 1 && imass != 3) || iterl < 1) {
        g_hmc_create_err = "chdwf_hmc_create: bad lattice, imass or iterl";
        return CHDWF_BAD_ARG;
    }
    chdwf_hmc* h = new chdwf_hmc;
    h->device = device;
    h->g = chdwf::make_geom(ksize, ksizet, kthird);
    h->dt = dt; h->beta = beta; h->am3 = am3; h->am = am; h->imass = imass; h->iterl = iterl;
    cudaError_t e = cudaSetDevice(device);
    const int64_t n3 = 3 * (int64_t)h->g.kvol, nf = h->g.kferm;
    if (!e) e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
    if (!e) e = dalloc(&h->chi, n3);
    if (!e) e = dalloc(&h->chit, n3);
    if (!e) e = dalloc(&h->pp, n3);
    if (!e) e = dalloc(&h->dS, n3);
    if (!e) e = dalloc(&h->chi_io, n3);
    if (!e) e = dalloc(&h->Phi, nf);
    if (!e) e = dalloc(&h->X0, nf);
    if (!e) e = dalloc(&h->X1, nf);
    if (!e) e = dalloc(&h->R, nf);
    if (!e) e = dalloc(&h->cp, nf);
    if (!e) e = dalloc(&h->cr, nf);
    if (!e) e = dalloc(&h->cx1, nf);
    if (!e) e = dalloc(&h->gauss, 16 * (size_t)h->g.kvol * kthird);
    const int64_t nbmax = std::max<int64_t>(chdwf::nblk(nf), chdwf::kHfBlocks);
    if (!e) e = dalloc(&h->part, nbmax + 64);
    if (!e) e = dalloc(&h->ctl, 1);
    if (!e) e = cudaHostAlloc((void**)&h->hflag_host, sizeof(int), cudaHostAllocMapped);
    if (!e) e = cudaHostGetDevicePointer((void**)&h->hflag_dev, h->hflag_host, 0);
    if (!e) e = cudaMemsetAsync(h->chi, 0, sizeof(float) * n3, h->st);
    if (!e) e = cudaMemsetAsync(h->ctl, 0, sizeof(chdwf::CgCtl), h->st);
    if (!e) e = cudaStreamSynchronize(h->st);
    if (e) {
        g_hmc_create_err = std::string("chdwf_hmc_create: ") + cudaGetErrorString(e);
        chdwf_hmc_destroy(h);
        return CHDWF_CUDA_ERROR;
    }
    h->rng.startup((double)693764523745.0f);
    *out = h;
    return CHDWF_OK;
}

void chdwf_hmc_destroy(chdwf_hmc* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->st) cudaStreamSynchronize(h->st);
    for (float* p : {h->chi, h->chit, h->pp, h->dS, h->chi_io, h->gauss}) if (p) cudaFree(p);
    for (float2* p : {h->Phi, h->X0, h->X1, h->R, h->cp, h->cr, h->cx1}) if (p) cudaFree(p);
    if (h->part) cudaFree(h->part);
    if (h->ctl) cudaFree(h->ctl);
    if (h->hflag_host) cudaFreeHost(h->hflag_host);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

const char* chdwf_hmc_last_error(chdwf_hmc* h) {
    return h ? h->err.c_str() : g_hmc_create_err.c_str();
}

int chdwf_hmc_dslash(chdwf_hmc* h, float* Phi, const float* R, const float* chi, int imass) {
    return hmc_apply(h, false, Phi, R, chi, imass);
}

int chdwf_hmc_dslashd(chdwf_hmc* h, float* Phi, const float* R, const float* chi, int imass) {
    return hmc_apply(h, true, Phi, R, chi, imass);
}

int chdwf_hmc_congrad(chdwf_hmc* h, const float* Phi, float res, int* itercg, int imass,
                      const float* chi, float* x) {
    if (!as_ok(h) || !Phi || !itercg || !chi || !x || (imass != 1 && imass != 3))
        return CHDWF_BAD_ARG;
    const Geom& g = h->g;
    cudaMemcpyAsync(h->R, Phi, sizeof(float2) * g.kferm, cudaMemcpyHostToDevice, h->st);
    cudaMemcpyAsync(h->X1, x, sizeof(float2) * g.kferm, cudaMemcpyHostToDevice, h->st);
    cudaMemcpyAsync(h->chi_io, chi, sizeof(float) * 3 * g.kvol, cudaMemcpyHostToDevice, h->st);
    int stt = 0;
    cudaError_t e = hcg_solve(h, h->R, res, imass, h->chi_io, h->X1, itercg, &stt);
    if (e) return h->fail(e, "hmc_congrad");
    cudaMemcpyAsync(x, h->X1, sizeof(float2) * g.kferm, cudaMemcpyDeviceToHost, h->st);
    if ((e = cudaStreamSynchronize(h->st))) return h->fail(e, "hmc_congrad");
    if (stt == 2) { h->err = "hmc_congrad: non-finite residual"; return CHDWF_NONFINITE; }
    return stt == 1 ? CHDWF_ITER_CAP : CHDWF_OK;
}

int chdwf_hmc_derivs(chdwf_hmc* h, const float* X1, const float* chi, int imass, float* dSdchi) {
    if (!as_ok(h) || !X1 || !chi || !dSdchi || (imass != 1 && imass != 3)) return CHDWF_BAD_ARG;
    const Geom& g = h->g;
    cudaMemcpyAsync(h->X1, X1, sizeof(float2) * g.kferm, cudaMemcpyHostToDevice, h->st);
    cudaMemcpyAsync(h->chi_io, chi, sizeof(float) * 3 * g.kvol, cudaMemcpyHostToDevice, h->st);
    launch_derivs(h, imass, h->X1, h->chi_io, h->dS);
    cudaMemcpyAsync(dSdchi, h->dS, sizeof(float) * 3 * g.kvol, cudaMemcpyDeviceToHost, h->st);
    const cudaError_t e = cudaStreamSynchronize(h->st);
    return e ? h->fail(e, "hmc_derivs") : CHDWF_OK;
}

int chdwf_hmc_set_chi(chdwf_hmc* h, const float* chi) {
    if (!as_ok(h) || !chi) return CHDWF_BAD_ARG;
    cudaMemcpyAsync(h->chi, chi, sizeof(float) * 3 * h->g.kvol, cudaMemcpyHostToDevice, h->st);
    const cudaError_t e = cudaStreamSynchronize(h->st);
    return e ? h->fail(e, "hmc_set_chi") : CHDWF_OK;
}

int chdwf_hmc_get_chi(chdwf_hmc* h, float* chi) {
    if (!as_ok(h) || !chi) return CHDWF_BAD_ARG;
    cudaMemcpyAsync(chi, h->chi, sizeof(float) * 3 * h->g.kvol, cudaMemcpyDeviceToHost, h->st);
    const cudaError_t e = cudaStreamSynchronize(h->st);
    return e ? h->fail(e, "hmc_get_chi") : CHDWF_OK;
}

int chdwf_hmc_startup(chdwf_hmc* h, double seed) {
    if (!h) return CHDWF_BAD_ARG;
    h->rng.startup(seed);
    return CHDWF_OK;
}

double chdwf_hmc_seed(chdwf_hmc* h) { return h ? h->rng.seed() : 0.0; }

int chdwf_hmc_set_measure(chdwf_hmc* h, int iprint) {
    if (!h || iprint < 1) return CHDWF_BAD_ARG;
    h->iprint = iprint;
    return CHDWF_OK;
}

int chdwf_hmc_set_residuals(chdwf_hmc* h, float rescga, float rescgg) {
    if (!h) return CHDWF_BAD_ARG;
    h->rescga = rescga;
    h->rescgg = rescgg;
    return CHDWF_OK;
}

int chdwf_hmc_sweep(chdwf_hmc* h, chdwf_hmc_record* rec) {
    if (!as_ok(h) || !rec) return CHDWF_BAD_ARG;
    memset(rec, 0, sizeof(*rec));
    const Geom& g = h->g;
    const int64_t kvol = g.kvol, n3 = 3 * kvol;
    const unsigned nb3 = chdwf::nblk(n3);
    int rc;
#define CK(x) do { rc = (x); if (rc != CHDWF_OK) return rc; } while (0)
#define CKC(x, w) do { cudaError_t e_ = (x); if (e_) return h->fail(e_, w); } while (0)
    h->isweep++;
    const int isweep = h->isweep;
    cudaMemcpyAsync(h->chit, h->chi, sizeof(float) * n3, cudaMemcpyDeviceToDevice, h->st);  // :146-149
    // pseudofermion heatbath: 8*kthird gauss0 calls, Phi = M^dagger R (:154-165)
    std::vector<float> gauss(16 * (size_t)kvol * g.Ls);
    for (int c = 0; c < 8 * g.Ls; c++) h->rng.gauss0(kvol, gauss.data() + (size_t)c * 2 * kvol);
    CKC(cudaMemcpyAsync(h->gauss, gauss.data(), sizeof(float) * gauss.size(),
                        cudaMemcpyHostToDevice, h->st), "hmc_sweep");
    chdwf::k_hmc_noise<<<chdwf::nblk(g.kferm), chdwf::kThreads, 0, h->st>>>(h->R, h->gauss, g);
    chdwf::count_launches(1);
    launch_dslash(h, true, h->imass, h->Phi, h->R, h->chit);
    cudaMemcpyAsync(h->X0, h->Phi, sizeof(float2) * g.kferm, cudaMemcpyDeviceToDevice, h->st);  // :167-175
    // momenta (:179-187)
    std::vector<float> ps(2 * kvol), pp(n3);
    h->rng.gaussp(kvol, ps.data());
    memcpy(pp.data(), ps.data(), sizeof(float) * 2 * kvol);
    h->rng.gaussp(kvol, ps.data());
    memcpy(pp.data() + 2 * kvol, ps.data(), sizeof(float) * kvol);
    CKC(cudaMemcpyAsync(h->pp, pp.data(), sizeof(float) * n3, cudaMemcpyHostToDevice, h->st),
        "hmc_sweep");
    double hh[4];
    CK(hmc_hamilton(h, h->rescga, hh, &rec->it_h0));                    // :191
    rec->H0 = hh[0];
    rec->S0 = hh[3];
    if (isweep == 1) {                                                   // :193-197
        h->action = (float)(hh[3] / (double)kvol);
        h->gaction = (float)(hh[1] / (double)kvol);
        h->paction = (float)(hh[2] / (double)kvol);
    }
    int itf = 0;
    CK(hmc_force(h, h->rescgg, &itf));                                   // :202
    rec->it_force += itf;
    rec->nforce++;
    float d = h->dt * 0.5f;                                              // :203-207
    chdwf::k_hmc_update_p<<<nb3, chdwf::kThreads, 0, h->st>>>(h->pp, h->dS, d, n3);
    chdwf::count_launches(1);
    const float proby = 1.0f / (float)h->iterl;                          // :100
    for (int iter = 1; iter <= 1000; iter++) {                           // :211-248
        d = h->dt;
        chdwf::k_hmc_update_chi<<<nb3, chdwf::kThreads, 0, h->st>>>(h->chit, h->pp, d, n3);
        chdwf::count_launches(1);
        CK(hmc_force(h, h->rescgg, &itf));
        rec->it_force += itf;
        rec->nforce++;
        rec->nsteps = iter;
        const float ytest = h->rng.rano_yrun();                           // :228
        if (ytest < proby) {
            d = h->dt * 0.5f;
            chdwf::k_hmc_update_p<<<nb3, chdwf::kThreads, 0, h->st>>>(h->pp, h->dS, d, n3);
            chdwf::count_launches(1);
            h->itot = h->itot + iter;
            break;
        }
        d = h->dt;
        chdwf::k_hmc_update_p<<<nb3, chdwf::kThreads, 0, h->st>>>(h->pp, h->dS, d, n3);
        chdwf::count_launches(1);
    }
    CK(hmc_hamilton(h, h->rescga, hh, &rec->it_h1));                    // :251
    rec->H1 = hh[0];
    rec->S1 = hh[3];
    rec->hg = hh[1];
    rec->hp = hh[2];
    rec->dH = rec->H0 - rec->H1;
    rec->dS = rec->S0 - rec->S1;
    rec->y = (float)std::exp(rec->dH);                                   // :256
    h->yav = h->yav + rec->y;
    h->yyav = h->yyav + rec->y * rec->y;
    int accept = 1;
    if (rec->dH < 0.0) {                                                 // :259-263
        rec->x = h->rng.rano_yrun();
        rec->drew_x = 1;
        if (rec->x > rec->y) accept = 0;
    }
    if (accept) {                                                        // :264-274
        cudaMemcpyAsync(h->chi, h->chit, sizeof(float) * n3, cudaMemcpyDeviceToDevice, h->st);
        h->naccp = h->naccp + 1;
        h->action = (float)(rec->S1 / (double)kvol);
        h->gaction = (float)(rec->hg / (double)kvol);
        h->paction = (float)(rec->hp / (double)kvol);
    }
    rec->accepted = accept;
    rec->action = h->action;
    rec->gaction = h->gaction;
    rec->paction = h->paction;
    h->actiona = h->actiona + h->action;                                 // :277
    CKC(cudaMemcpyAsync(pp.data(), h->pp, sizeof(float) * n3, cudaMemcpyDeviceToHost, h->st),
        "hmc_sweep");
    CKC(cudaStreamSynchronize(h->st), "hmc_sweep");
    float vel2 = 0.0f;                                                   // :278-283
    for (int64_t j = 0; j < n3; j++) vel2 = vel2 + pp[j] * pp[j];
    rec->vel2 = vel2 / (float)kvol;
    h->vel2a = h->vel2a + rec->vel2;
    if ((isweep / h->iprint) * h->iprint == isweep) {                    // :288-315
        rec->measured = 1;
        cudaMemcpyAsync(h->chit, h->chi, sizeof(float) * n3, cudaMemcpyDeviceToDevice, h->st);
        std::vector<float> chi(n3);
        CKC(cudaMemcpyAsync(chi.data(), h->chi, sizeof(float) * n3, cudaMemcpyDeviceToHost, h->st),
            "hmc_sweep");
        CKC(cudaStreamSynchronize(h->st), "hmc_sweep");
        float susctot = 0.0f, condmod = 0.0f;
        for (int a = 0; a < 3; a++) {
            float cnd = 0.0f;
            for (int64_t i = 0; i < kvol; i++) cnd = cnd + chi[i + kvol * a];
            float su = cnd * cnd;
            cnd = cnd / (float)kvol;
            condmod = condmod + cnd * cnd;
            su = su / (float)kvol;
            susctot = susctot + su;
            rec->cond[a] = cnd;
            rec->susc[a] = su;
        }
        rec->condmod = std::sqrt(condmod);
        rec->susctot = susctot;
    }
    CKC(cudaGetLastError(), "hmc_sweep");
#undef CK
#undef CKC
    return CHDWF_OK;
}

}  // extern "C"
