// lanczos.cu -- multi-shift solver for (M^dagger M + sigma_k) x_k = Phi over
// the Remez poles: the reference's qmrherm (rhmc/cheisdwf.f:599-745).
//
// The reference runs the Lanczos-based multi-shift recurrence and keeps two
// ndiag x kferm arrays (p_k, x_k), so every iteration streams (10 + 4n)
// spinors.  This implementation runs the SAME Lanczos process and the SAME
// scalar recurrences (d_k, mu_k, rho_k and the stopping rule, :670-715) but
// in two passes:
//   pass 1  Lanczos vectors + scalar recurrences only; 6 spinor streams per
//           iteration (M with a fused |Mq|^2, M^dagger with the fused
//           three-term update and |r|^2);
//   pass 2  regenerate the identical Lanczos vectors (same kernels, same
//           stored scalars, bit-identical) and accumulate the solution
//           x = a0 Phi + sum_j c_j q_j, where c_j = sum_k a_k y_kj and y_kj is
//           the coefficient of q_j in x_k, obtained from rho and mu by the
//           backward recurrence y_km = rho_km, y_ki = rho_ki - mu_k,i+1 y_k,i+1
//           (x_k = sum_j rho_kj p_kj, p_kj = q_j - mu_kj p_k,j-1).
// For iflag=1 only the two wall slices of each x_k are accumulated: the force
// (derivs) reads x_k and M x_k on s=1 and s=Ls only, and M x_k there depends
// on x_k on those two slices alone.
// alpha~_j = q_j^dagger M^dagger M q_j is evaluated as |M q_j|^2, which lets
// the three-term update be fused into the M^dagger kernel.
#include <cmath>
#include <cstddef>
#include <cstring>
#include <type_traits>
#include <utility>

#include "dwf_stencil.cuh"
#include "lanczos.h"

namespace chdwf {

template <class T> struct LdPlainT {
    const T* __restrict__ p;
    __device__ __forceinline__ T operator()(int64_t j) const { return __ldg(p + j); }
};

__device__ __forceinline__ double2 widen(double2 v) { return v; }
__device__ __forceinline__ double2 widen(float2 v) { return make_double2((double)v.x, (double)v.y); }

template <class T>
__device__ __forceinline__ T* ring(const LzArgsT<T>& a, int j) {
    if (j < a.hcap) return a.basis + (int64_t)j * a.g.kferm;
    const int r = j % 3;
    return r == 0 ? a.rb0 : (r == 1 ? a.rb1 : a.rb2);
}

// Element e of a Krylov vector: FP32 vectors with Ls even are in the split
// layout (cpair), FP64 vectors and odd-Ls FP32 vectors plain.
__device__ __forceinline__ double2 vget(const LzArgsT<double2>&, const double2* v, int64_t e) {
    return __ldg(v + e);
}
__device__ __forceinline__ float2 vget(const LzArgsT<float2>& a, const float2* v, int64_t e) {
    return a.pl ? sp_get(v, e) : __ldg(v + e);
}

static_assert(kSplitThreads == kThreads, "the reductions assume kThreads-wide blocks");

// KernelTimer class of a launch: c for FP64 Krylov vectors, c + 4 for FP32.
template <class T>
static inline int timer_class(int c) {
    return c + (std::is_same<T, float2>::value ? 4 : 0);
}

// Sum of the n chunk partials part[0..n) in a fixed order; every block that
// calls it gets the same value.  Valid in all threads.
__device__ __forceinline__ double sum_partials(const double* part, int n) {
    __shared__ double sh[kThreads / 32];
    __shared__ double total;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += kThreads) s += __ldcg(part + i);
    s = block_sum<kThreads>(s, sh);
    if (threadIdx.x == 0) total = s;
    __syncthreads();
    return total;
}

// The stop flag, read once per block: every thread of a block takes the same
// branch (the scalar step may set it while an M^dagger block starts).
__device__ __forceinline__ bool block_stopped(const LzCtl* ctl) {
    __shared__ int s_done;
    if (threadIdx.x == 0) s_done = *(const volatile int*)&ctl->done;
    __syncthreads();
    return s_done != 0;
}

// ---- thread mapping ----------------------------------------------------------
// FP64 vectors: two threads per point, one per flavour (split_point /
// split_flavour), which halves the accumulator registers and doubles the
// warps in flight.  FP32 vectors with Ls even (PAIR): a thread takes two
// adjacent points of one flavour, loading both with one 16-byte float4.
// FP32 otherwise: one thread per point and both flavours.
template <class T, bool PAIR = false> struct LzShape;
template <> struct LzShape<double2, false> {
    static constexpr bool split = true;
    static constexpr int min_blocks = 3;          // <= 85 registers: no spills
    static constexpr int unit = kSplitPoints;     // points per block pass
};
template <> struct LzShape<float2, false> {
    static constexpr bool split = false;
    static constexpr int min_blocks = 3;          // <= 85 registers a thread
    static constexpr int unit = kThreads;
};
template <> struct LzShape<float2, true> {
    static constexpr bool split = true;
    static constexpr int min_blocks = 3;
    static constexpr int unit = 2 * kSplitPoints; // 128 point pairs per flavour
};

// Pass 1 runs on a persistent grid (a whole number of blocks per SM); block b
// owns the contiguous, warp-aligned point range below, so every SM gets the
// same amount of work and none idles through a partial last wave.  Each
// block leaves its |.|^2 partial in part[b]; the kernel that needs the sum
// adds the partials itself, in block order, so no block waits on another.
struct PtRange { int64_t begin, end; };
__device__ __forceinline__ PtRange block_range(int64_t npts) {
    const int64_t nb = gridDim.x, b = blockIdx.x;
    PtRange r;
    r.begin = (b * npts / nb) & ~(int64_t)31;
    r.end = b + 1 == nb ? npts : (((b + 1) * npts / nb) & ~(int64_t)31);
    return r;
}

// One block pass over points [base, base + unit) of flavour(s) f0..f0+NF-1
// (PAIR: p is the even point of the thread's pair).
template <class T, bool PAIR = false>
__device__ __forceinline__ void lz_lane(int64_t base, int64_t* p, int* f0) {
    if (PAIR) {
        *p = base + 2 * (threadIdx.x & (kSplitPoints - 1));
        *f0 = split_flavour();
    } else if (LzShape<T>::split) {
        *p = base + (threadIdx.x & (kSplitPoints - 1));
        *f0 = split_flavour();
    } else {
        *p = base + threadIdx.x;
        *f0 = 0;
    }
}

// vt = M q_j with q_j = r_j / beta_j, formed as (1/beta_j) (M r_j): one
// scaling per output element instead of one per stencil load.  The pass-1
// kernel and the regenerating pass 2 use this same sequence.
template <bool DAG, int IMASS, class T>
__device__ __forceinline__ void apply_scaled(T acc[4], const T* r, typename real_of<T>::type ib,
                                             const LzArgsT<T>& a, const PointIdx& q, int f) {
    dwf_apply_flavour<DAG, IMASS>(acc, LdPlainT<T>{r}, a.g, q, f, a.chif, a.diag, a.hpin,
                                  a.apbc != 0);
#pragma unroll
    for (int d = 0; d < 4; d++) acc[d] = zscal(ib, acc[d]);
}

// ---- pass 1, kernel 1: vt = M q_j and the block partials of |vt|^2 ---------
// beta_j is the sum of the previous M^dagger launch's partials (beta_1 comes
// from the source), formed by every block.  The partial buffers: part[0..nb)
// for this kernel, part[nb..2nb) for M^dagger.
template <class T, int IMASS, bool PAIR, int OCC>
__global__ void __launch_bounds__(kThreads, OCC) k_lz1_M(LzArgsT<T> a) {
    typedef typename real_of<T>::type Real;
    typedef LzShape<T, PAIR> S;
    constexpr int NF = S::split ? 1 : 2;
    // One flavour a thread: beta_j is first needed to scale the block's
    // first outputs, so its sum over the previous launch's partials (an L2
    // round trip and two block barriers) is formed after the first pass's
    // stencil loads are issued.  Every thread of the block reaches it (the
    // loop's trip count is the same for the whole block).
    constexpr bool LATE = NF == 1;
    LzCtl* ctl = a.ctl;
    if (block_stopped(ctl)) return;
    const int j = ctl->it_m;
    const int nb = gridDim.x;
    bool have = j == 1 || !LATE;
    double bj = j == 1 ? a.h.beta[1] : (LATE ? 0.0 : sqrt(sum_partials(a.part + nb, nb)));
    double ibj = j == 1 ? a.h.invbeta[1] : (LATE ? 0.0 : 1.0 / bj);
    const T* rj = ring(a, j);
    const PtRange R = block_range(a.g.npts);
    double loc = 0.0;
#pragma unroll 1
    for (int64_t base = R.begin; base < R.end; base += S::unit) {
        int64_t p;
        int f0;
        lz_lane<T, PAIR>(base, &p, &f0);
        const bool act = p < R.end;
        const PointIdx q = point_of(a.g, act ? p : R.begin);
        if constexpr (PAIR) {
            cpair acc[4];
            if (act)
                dwf_apply_flavour_pair_sp<false, IMASS>(acc, rj, a.g, q, f0, a.chif, a.diag,
                                                        a.hpin, a.apbc != 0);
            if (!have) {
                bj = sqrt(sum_partials(a.part + nb, nb));
                ibj = 1.0 / bj;
                have = true;
            }
            if (!act) continue;
            const Real ib = (Real)ibj;
            // |vt|^2 is summed in FP64 from the first term: a pair's partial
            // sum in FP32 made the FP32 force solves 7% longer (alpha~ and
            // beta steer the recurrences)
#pragma unroll
            for (int d = 0; d < 4; d++) {
                const cpair v = zscal(ib, acc[d]);
                st_cpair(a.vt, (uint32_t)p + (uint32_t)a.g.cs * (uint32_t)(d + 4 * f0), v);
                const double2 w0 = widen(cpair_pt(v, 0)), w1 = widen(cpair_pt(v, 1));
                loc += w0.x * w0.x + w0.y * w0.y;
                loc += w1.x * w1.x + w1.y * w1.y;
            }
        } else if constexpr (LATE) {
            T acc[4];
            if (act)
                dwf_apply_flavour<false, IMASS>(acc, LdPlainT<T>{rj}, a.g, q, f0, a.chif, a.diag,
                                                a.hpin, a.apbc != 0);
            if (!have) {
                bj = sqrt(sum_partials(a.part + nb, nb));
                ibj = 1.0 / bj;
                have = true;
            }
            if (!act) continue;
            const Real ib = (Real)ibj;
#pragma unroll
            for (int d = 0; d < 4; d++) {
                const T v = zscal(ib, acc[d]);   // apply_scaled's scaling
                a.vt[p + a.g.cs * (d + 4 * f0)] = v;
                const double2 w = widen(v);
                loc += w.x * w.x + w.y * w.y;
            }
        } else {
            if (!act) continue;
            const Real ib = (Real)ibj;
#pragma unroll
            for (int f = f0; f < f0 + NF; f++) {
                T acc[4];
                apply_scaled<false, IMASS>(acc, rj, ib, a, q, f);
#pragma unroll
                for (int d = 0; d < 4; d++) {
                    a.vt[p + a.g.cs * (d + 4 * f)] = acc[d];
                    const double2 w = widen(acc[d]);
                    loc += w.x * w.x + w.y * w.y;
                }
            }
        }
    }
    if (!have) {   // a block whose range is empty
        bj = sqrt(sum_partials(a.part + nb, nb));
        ibj = 1.0 / bj;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->it_md = j;
        if (j > 1) {
            a.h.beta[j] = bj;
            a.h.invbeta[j] = ibj;
        }
    }
    __shared__ double sh[kThreads / 32];
    loc = block_sum<kThreads>(loc, sh);
    if (threadIdx.x == 0) a.part[blockIdx.x] = loc;
}

// Scalar recurrences of qmrherm for iteration j (cheisdwf.f:666-715), one
// lane per pole (the poles are independent), and the stopping test.
template <class T>
__device__ __forceinline__ void pole_step(const LzArgsT<T>& a, int j, double at) {
    LzCtl* ctl = a.ctl;
    const int k = threadIdx.x;
    const double beta0 = a.h.beta[j];
    if (k == 0) a.h.alphat[j] = at;
    const int n = ctl->npole;
    const int64_t H = kMaxIter + 2;
    double v = -1.0;
    if (k < n) {
        const double alpha = __dadd_rn(at, ctl->sigma[k]);
        double rho, mu = 0.0;
        if (j == 1) {
            ctl->d[k] = alpha;
            rho = __ddiv_rn(beta0, alpha);
        } else {
            const double dm1 = ctl->d[k];
            mu = __ddiv_rn(beta0, dm1);
            const double dn = __dsub_rn(alpha, __dmul_rn(beta0, mu));
            ctl->d[k] = dn;
            rho = -__ddiv_rn(__dmul_rn(__dmul_rn(mu, dm1), ctl->rho[k]), dn);
        }
        ctl->rho[k] = rho;
        a.h.rho[k * H + j] = rho;
        a.h.mu[k * H + j] = mu;
        v = fabs(__dmul_rn(ctl->phimod, rho));
    }
    // rhomax as the sequential scan over the poles forms it: start from pole
    // 0 and take any larger value (a NaN in pole 0 stays, NaNs of the other
    // poles are skipped)
    const double v0 = __shfl_sync(0xffffffffu, v, 0);
    double m1 = k >= 1 ? v : -1.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
    if (k != 0) return;
    const double rhomax = (v0 != v0) ? v0 : fmax(v0, m1);
    int done = 0;
    if (j >= 2 && rhomax < ctl->thresh) done = 1;
    else if (j >= ctl->niter_cap) done = 2;
    if (!(rhomax == rhomax)) done = 3;   // NaN: stop, reported as non-finite
    if (done) {
        ctl->done = done;
        ctl->m = j;
        if (a.hflag) {
            *(volatile int*)a.hflag = done;
            __threadfence_system();
        }
    }
}

// alpha~_j from M(j)'s partials (the same sum, in the same order, as the
// M^dagger blocks form), the pole recurrences and the stopping test.  One
// block, launched on a side stream next to M^dagger(j): it overlaps that
// kernel instead of lengthening either pass-1 kernel.  A converged solve
// stops before M(j+1).
template <class T>
__global__ void __launch_bounds__(kThreads) k_lz_pole(LzArgsT<T> a, int nb) {
    LzCtl* ctl = a.ctl;
    if (block_stopped(ctl)) return;
    const int j = ctl->it_md;
    const double at = sum_partials(a.part, nb);
    if (threadIdx.x == 0) ctl->it_m = j + 1;
    if (threadIdx.x < 32) pole_step(a, j, at);
}

// r_{j+1} = x3 - alpha~ q_j - beta_j q_{j-1} at one point (cheisdwf.f:655)
template <class T>
__device__ __forceinline__ T three_term(const LzArgsT<T>& a, T x3, int64_t e, int j,
                                        double alphat) {
    typedef typename real_of<T>::type Real;
    const T* rj = ring(a, j);
    const T* rjm = ring(a, j - 1);
    const Real ib = (Real)a.h.invbeta[j], at = (Real)alphat, bj = (Real)a.h.beta[j];
    const T qj = zscal(ib, rj[e]);
    T v = zsub(x3, zscal(at, qj));
    if (j > 1) v = zsub(v, zscal(bj, zscal((Real)a.h.invbeta[j - 1], rjm[e])));
    return v;
}

// The same update for the two points of an FP32 pair (elements e, e+1) of
// split-layout vectors, both points at once.
__device__ __forceinline__ cpair three_term_sp(const LzArgsT<float2>& a, cpair x, uint32_t e,
                                               int j, double alphat) {
    const float2* rj = ring(a, j);
    const float2* rjm = ring(a, j - 1);
    const float ib = (float)a.h.invbeta[j], at = (float)alphat, bj = (float)a.h.beta[j];
    cpair v = zsub(x, zscal(at, zscal(ib, ld_cpair(rj, e))));
    if (j > 1) {
        const float ibm = (float)a.h.invbeta[j - 1];
        v = zsub(v, zscal(bj, zscal(ibm, ld_cpair(rjm, e))));
    }
    return v;
}

// Force solves with a wall store: element e of r_{j+1} at point (s, site),
// component c, also goes to the wall store when s is a wall.
template <class T>
__device__ __forceinline__ void wall_put(const LzArgsT<T>& a, int j1, int s, int site, int c,
                                         T v) {
    if (a.wcap == 0 || j1 >= a.wcap) return;
    const int Ls = a.g.Ls;
    if (s != 0 && s != Ls - 1) return;
    const int64_t cs2 = 2 * (int64_t)a.g.kvol;
    a.wbasis[(int64_t)j1 * 8 * cs2 + (s == 0 ? 0 : 1) + 2 * (int64_t)site + cs2 * c] = v;
}

// ---- pass 1, kernel 2: r_{j+1} = M^dagger vt - alpha~ q_j - beta_j q_{j-1} ---
// alpha~_j is the sum of M(j)'s partials, formed by every block.
template <class T, int IMASS, bool PAIR, bool WALLS, int OCC>
__global__ void __launch_bounds__(kThreads, OCC) k_lz1_Md(LzArgsT<T> a) {
    typedef LzShape<T, PAIR> S;
    constexpr int NF = S::split ? 1 : 2;
    // alpha~_j, as beta_j in k_lz1_M, is summed after the first pass's
    // stencil (one flavour a thread)
    constexpr bool LATE = NF == 1;
    LzCtl* ctl = a.ctl;
    if (block_stopped(ctl)) return;
    const int j = ctl->it_md;
    const int nb = gridDim.x;
    bool have = !LATE;
    double at = LATE ? 0.0 : sum_partials(a.part, nb);
    T* rn = ring(a, j + 1);
    const PtRange R = block_range(a.g.npts);
    double loc = 0.0;
#pragma unroll 1
    for (int64_t base = R.begin; base < R.end; base += S::unit) {
        int64_t p;
        int f0;
        lz_lane<T, PAIR>(base, &p, &f0);
        const bool act = p < R.end;
        const PointIdx q = point_of(a.g, act ? p : R.begin);
        if constexpr (PAIR) {
            cpair acc[4];
            if (act)
                dwf_apply_flavour_pair_sp<true, IMASS>(acc, a.vt, a.g, q, f0, a.chif, a.diag,
                                                       a.hpin, a.apbc != 0);
            if (!have) {
                at = sum_partials(a.part, nb);
                have = true;
            }
            if (!act) continue;
#pragma unroll
            for (int d = 0; d < 4; d++) {
                const uint32_t e = (uint32_t)p + (uint32_t)a.g.cs * (uint32_t)(d + 4 * f0);
                const cpair v = three_term_sp(a, acc[d], e, j, at);
                st_cpair(rn, e, v);
                const float2 v0 = cpair_pt(v, 0), v1 = cpair_pt(v, 1);
                if (WALLS) {
                    wall_put(a, j + 1, q.s, q.site, d + 4 * f0, v0);
                    wall_put(a, j + 1, q.s + 1, q.site, d + 4 * f0, v1);
                }
                const double2 w0 = widen(v0), w1 = widen(v1);
                loc += w0.x * w0.x + w0.y * w0.y;
                loc += w1.x * w1.x + w1.y * w1.y;
            }
        } else {
            T acc[NF][4];
            if (LATE && act)
                dwf_apply_flavour<true, IMASS>(acc[0], LdPlainT<T>{a.vt}, a.g, q, f0, a.chif,
                                               a.diag, a.hpin, a.apbc != 0);
            if (!have) {
                at = sum_partials(a.part, nb);
                have = true;
            }
            if (!act) continue;
#pragma unroll
            for (int f = f0; f < f0 + NF; f++) {
                if (!LATE)
                    dwf_apply_flavour<true, IMASS>(acc[f - f0], LdPlainT<T>{a.vt}, a.g, q, f,
                                                   a.chif, a.diag, a.hpin, a.apbc != 0);
#pragma unroll
                for (int d = 0; d < 4; d++) {
                    const int64_t e = p + a.g.cs * (d + 4 * f);
                    const T v = three_term(a, acc[f - f0][d], e, j, at);
                    rn[e] = v;
                    if (WALLS) wall_put(a, j + 1, q.s, q.site, d + 4 * f, v);
                    const double2 w = widen(v);
                    loc += w.x * w.x + w.y * w.y;
                }
            }
        }
    }
    __shared__ double sh[kThreads / 32];
    loc = block_sum<kThreads>(loc, sh);
    if (threadIdx.x == 0) a.part[nb + blockIdx.x] = loc;
}

// ---- pass 1 on staged rows ---------------------------------------------------
// The same two kernels with the stencil's input rows staged in shared memory
// (row_stage.cuh): a persistent grid of the blocks that fit on all SMs at
// once, each walking a contiguous range of output rows of one flavour at a
// time.  Per element the operation sequence is that of k_lz1_M / k_lz1_Md,
// so the vectors are the same bits and the regenerating pass 2 reproduces
// them.  A copy that does not arrive within the bounded wait stops the solve
// with done = 4 (reported as a CUDA error).
__device__ __forceinline__ void row_fail(LzCtl* ctl, int* hflag) {
    ctl->done = 4;
    ctl->m = ctl->it_m;
    if (hflag) {
        *(volatile int*)hflag = 4;
        __threadfence_system();
    }
}

// PPT adjacent elements of a global vector
template <class T, int PPT> struct LzLd;
template <class T> struct LzLd<T, 1> {
    __device__ __forceinline__ static void get(const T* p, T* v) { v[0] = *p; }
    __device__ __forceinline__ static void put(T* p, const T* v) { *p = v[0]; }
};

template <class T, int IMASS, int PPT>
struct LzRowsM {
    typedef typename real_of<T>::type Real;
    const LzArgsT<T>& a;
    const T* rj;
    Real ib;
    double loc;
    RowWall<T, PPT> rw;
    __device__ __forceinline__ void pre(int f, int t, int y, int x, int s) {
        row_wall_prefetch<false, PPT>(rw, rj, a.g, f, t, y, x, s, a.chif);
    }
    __device__ __forceinline__ void compute(const T* c, const T* yp, const T* ym, const T* tps,
                                            const T* tms, int f, int t, int y, int x, int s,
                                            int i, int ixp, int ixm) {
        const Geom& g = a.g;
        const int site = x + g.L * (y + g.L * t);
        T acc[PPT][4];
        dwf_apply_rows<false, IMASS, PPT>(acc, c, yp, ym, tps, tms, a.rp.Lrow, i, ixp, ixm, s,
                                          site, t, rw, g, f, a.diag, a.hpin, a.apbc != 0);
        const int64_t p0 = s + (int64_t)g.Ls * site;
#pragma unroll
        for (int d = 0; d < 4; d++) {
            T v[PPT];
#pragma unroll
            for (int p = 0; p < PPT; p++) {
                v[p] = zscal(ib, acc[p][d]);
                const double2 w = widen(v[p]);
                loc += w.x * w.x + w.y * w.y;
            }
            LzLd<T, PPT>::put(a.vt + p0 + g.cs * (d + 4 * f), v);
        }
    }
};

template <class T, int IMASS, int PPT>
__global__ void __maxnreg__(kRowRegs) k_lz1_M_rows(LzArgsT<T> a) {
    extern __shared__ __align__(128) unsigned char row_smem[];
    LzCtl* ctl = a.ctl;
    if (block_stopped(ctl)) return;
    const int j = ctl->it_m;
    const int nb = gridDim.x;
    const double bj = j == 1 ? a.h.beta[1] : sqrt(sum_partials_any(a.part + nb, nb));
    const double ibj = j == 1 ? a.h.invbeta[1] : 1.0 / bj;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->it_md = j;
        if (j > 1) {
            a.h.beta[j] = bj;
            a.h.invbeta[j] = ibj;
        }
    }
    LzRowsM<T, IMASS, PPT> body{a, ring(a, j), (typename real_of<T>::type)ibj, 0.0};
    const bool ok = row_sweep<T, PPT>(a.g, a.rp, row_smem, body.rj, body);
    __shared__ double sh[32];
    const double loc = block_sum_any(body.loc, sh);
    if (threadIdx.x == 0) {
        a.part[blockIdx.x] = loc;
        if (!ok) row_fail(ctl, a.hflag);
    }
}

template <class T, int IMASS, bool WALLS, int PPT>
struct LzRowsMd {
    typedef typename real_of<T>::type Real;
    const LzArgsT<T>& a;
    const T* rj;
    const T* rjm;
    T* rn;
    int j;
    Real ib, at, bj, ibm;
    double loc;
    T cj[4][PPT], cm[4][PPT];
    RowWall<T, PPT> rw;
    // q_j and q_{j-1} at the thread's points (streamed, not staged) and the
    // wall operands
    __device__ __forceinline__ void pre(int f, int t, int y, int x, int s) {
        const Geom& g = a.g;
        const int64_t e0 = (int64_t)x * g.Ls + s + (int64_t)g.L * g.Ls * (y + (int64_t)g.L * t);
#pragma unroll
        for (int d = 0; d < 4; d++) {
            const int64_t po = g.cs * (d + 4 * f);
            LzLd<T, PPT>::get(rj + e0 + po, cj[d]);
            if (j > 1) LzLd<T, PPT>::get(rjm + e0 + po, cm[d]);
        }
        row_wall_prefetch<true, PPT>(rw, a.vt, g, f, t, y, x, s, a.chif);
    }
    __device__ __forceinline__ void compute(const T* c, const T* yp, const T* ym, const T* tps,
                                            const T* tms, int f, int t, int y, int x, int s,
                                            int i, int ixp, int ixm) {
        const Geom& g = a.g;
        const int site = x + g.L * (y + g.L * t);
        T acc[PPT][4];
        dwf_apply_rows<true, IMASS, PPT>(acc, c, yp, ym, tps, tms, a.rp.Lrow, i, ixp, ixm, s,
                                         site, t, rw, g, f, a.diag, a.hpin, a.apbc != 0);
        const int64_t p0 = s + (int64_t)g.Ls * site;
#pragma unroll
        for (int d = 0; d < 4; d++) {
            T v[PPT];
#pragma unroll
            for (int p = 0; p < PPT; p++) {
                // r_{j+1} = x3 - alpha~ q_j - beta_j q_{j-1}, as three_term (:655)
                const T qj = zscal(ib, cj[d][p]);
                v[p] = zsub(acc[p][d], zscal(at, qj));
                if (j > 1) v[p] = zsub(v[p], zscal(bj, zscal(ibm, cm[d][p])));
                if (WALLS) wall_put(a, j + 1, s + p, site, d + 4 * f, v[p]);
                const double2 w = widen(v[p]);
                loc += w.x * w.x + w.y * w.y;
            }
            LzLd<T, PPT>::put(rn + p0 + g.cs * (d + 4 * f), v);
        }
    }
};

template <class T, int IMASS, bool WALLS, int PPT>
__global__ void __maxnreg__(kRowRegs) k_lz1_Md_rows(LzArgsT<T> a) {
    typedef typename real_of<T>::type Real;
    extern __shared__ __align__(128) unsigned char row_smem[];
    LzCtl* ctl = a.ctl;
    if (block_stopped(ctl)) return;
    const int j = ctl->it_md;
    const int nb = gridDim.x;
    const double at = sum_partials_any(a.part, nb);
    LzRowsMd<T, IMASS, WALLS, PPT> body{a, ring(a, j), ring(a, j - 1), ring(a, j + 1), j,
                                        (Real)a.h.invbeta[j], (Real)at, (Real)a.h.beta[j],
                                        (Real)(j > 1 ? a.h.invbeta[j - 1] : 0.0), 0.0};
    const bool ok = row_sweep<T, PPT>(a.g, a.rp, row_smem, a.vt, body);
    __shared__ double sh[32];
    const double loc = block_sum_any(body.loc, sh);
    if (threadIdx.x == 0) {
        a.part[nb + blockIdx.x] = loc;
        if (!ok) row_fail(ctl, a.hflag);
    }
}

// ---- pass 2: regenerate q_j and accumulate --------------------------------
// One block pass per block (grid lz_direct_blocks).  The solution update of
// one element of x (iflag 0) or of the wall fields (iflag 1).
template <class T, int IFLAG>
__device__ __forceinline__ void lz2_accumulate(const LzArgsT<T>& a, int j, const T* rj,
                                               typename real_of<T>::type ib, int64_t p,
                                               const PointIdx& q, int c0, int nc) {
    if (IFLAG == 0) {
        const double cj = a.h.c[j];
        for (int c = c0; c < c0 + nc; c++) {
            const int64_t e = p + a.g.cs * c;
            const double2 qj = widen(zscal(ib, vget(a, rj, e)));
            double2 xv = a.x[e];
            xv.x += cj * qj.x;
            xv.y += cj * qj.y;
            a.x[e] = xv;
        }
    } else {
        const int Ls = a.g.Ls;
        if (q.s != 0 && q.s != Ls - 1) return;
        const int sw = (q.s == 0) ? 0 : 1;
        const int64_t cs2 = 2 * (int64_t)a.g.kvol, kf2 = 8 * cs2;
        const int64_t H = kMaxIter + 2;
        const int n = a.npole;
        double2 qv[8];
#pragma unroll
        for (int c = 0; c < 8; c++)
            if (c < nc) qv[c] = widen(zscal(ib, vget(a, rj, p + a.g.cs * (c + c0))));
        const int64_t base = sw + 2 * (int64_t)q.site + cs2 * c0;
        for (int k = 0; k < n; k++) {
            const double y = a.h.y[k * H + j];
            double2* xk = a.xw + k * kf2 + base;
#pragma unroll
            for (int c = 0; c < 8; c++) {
                if (c >= nc) break;
                double2 xv = xk[cs2 * c];
                xv.x += y * qv[c].x;
                xv.y += y * qv[c].y;
                xk[cs2 * c] = xv;
            }
        }
    }
}

template <class T, int IMASS, int IFLAG, bool PAIR>
__global__ void __launch_bounds__(kThreads, (LzShape<T, PAIR>::min_blocks))
    k_lz2_M(LzArgsT<T> a, int j, int apply) {
    typedef typename real_of<T>::type Real;
    typedef LzShape<T, PAIR> S;
    constexpr int NF = S::split ? 1 : 2;
    int64_t p;
    int f0;
    lz_lane<T, PAIR>((int64_t)blockIdx.x * S::unit, &p, &f0);
    if (p >= a.g.npts) return;
    const PointIdx q = point_of(a.g, p);
    const Real ib = (Real)a.h.invbeta[j];
    const T* rj = ring(a, j);
    if constexpr (PAIR) {
        if (apply) {
            cpair acc[4];
            dwf_apply_flavour_pair_sp<false, IMASS>(acc, rj, a.g, q, f0, a.chif, a.diag, a.hpin,
                                                    a.apbc != 0);
#pragma unroll
            for (int d = 0; d < 4; d++)
                st_cpair(a.vt, (uint32_t)(p + a.g.cs * (d + 4 * f0)), zscal(ib, acc[d]));
        }
        lz2_accumulate<T, IFLAG>(a, j, rj, ib, p, q, 4 * f0, 4);
        const PointIdx q1 = point_of(a.g, p + 1);
        lz2_accumulate<T, IFLAG>(a, j, rj, ib, p + 1, q1, 4 * f0, 4);
    } else {
        if (apply) {
#pragma unroll
            for (int f = f0; f < f0 + NF; f++) {
                T acc[4];
                apply_scaled<false, IMASS>(acc, rj, ib, a, q, f);
#pragma unroll
                for (int d = 0; d < 4; d++) a.vt[p + a.g.cs * (d + 4 * f)] = acc[d];
            }
        }
        lz2_accumulate<T, IFLAG>(a, j, rj, ib, p, q, 4 * f0, 4 * NF);
    }
}

template <class T, int IMASS, bool PAIR>
__global__ void __launch_bounds__(kThreads, (LzShape<T, PAIR>::min_blocks))
    k_lz2_Md(LzArgsT<T> a, int j) {
    typedef LzShape<T, PAIR> S;
    constexpr int NF = S::split ? 1 : 2;
    int64_t p;
    int f0;
    lz_lane<T, PAIR>((int64_t)blockIdx.x * S::unit, &p, &f0);
    if (p >= a.g.npts) return;
    const PointIdx q = point_of(a.g, p);
    T* rn = ring(a, j + 1);
    if constexpr (PAIR) {
        cpair acc[4];
        dwf_apply_flavour_pair_sp<true, IMASS>(acc, a.vt, a.g, q, f0, a.chif, a.diag, a.hpin,
                                               a.apbc != 0);
#pragma unroll
        for (int d = 0; d < 4; d++) {
            const uint32_t e = (uint32_t)(p + a.g.cs * (d + 4 * f0));
            st_cpair(rn, e, three_term_sp(a, acc[d], e, j, a.h.alphat[j]));
        }
    } else {
#pragma unroll
        for (int f = f0; f < f0 + NF; f++) {
            T acc[4];
            dwf_apply_flavour<true, IMASS>(acc, LdPlainT<T>{a.vt}, a.g, q, f, a.chif, a.diag,
                                           a.hpin, a.apbc != 0);
#pragma unroll
            for (int d = 0; d < 4; d++) {
                const int64_t e = p + a.g.cs * (d + 4 * f);
                rn[e] = three_term(a, acc[d], e, j, a.h.alphat[j]);
            }
        }
    }
}

template <class T, bool PAIR = false>
static unsigned lz_direct_blocks(int64_t npts) {
    return (unsigned)((npts + LzShape<T, PAIR>::unit - 1) / LzShape<T, PAIR>::unit);
}

// Persistent pass-1 grid: the resident blocks of both pass-1 kernels on all
// SMs, at most one block pass per block.
template <class T, int IMASS, bool PAIR, int OCC>
static unsigned lz_pass1_blocks(int64_t npts) {
    int dev = 0, nsm = 0, b1 = 0, b2 = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_lz1_M<T, IMASS, PAIR, OCC>, kThreads, 0);
    int b3 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, k_lz1_Md<T, IMASS, PAIR, false, OCC>,
                                                  kThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b3, k_lz1_Md<T, IMASS, PAIR, true, OCC>,
                                                  kThreads, 0);
    if (b3 < b2) b2 = b3;
    int64_t nb = (int64_t)nsm * (b1 < b2 ? b1 : b2);
    const int64_t direct = lz_direct_blocks<T, PAIR>(npts);
    if (nb < 1 || nb > direct) nb = direct;
    return (unsigned)nb;
}

// ---- between the passes: y_kj and c_j -------------------------------------
// The backward recurrence is sequential in i for each pole: the block stages
// rho and mu in shared memory a chunk of iterations at a time, so each pole's
// lane runs its chain from shared memory; c_j of the chunk follows in
// parallel, summed over the poles in order.
__global__ void __launch_bounds__(kThreads) k_lz_coeffs(LzCtl* ctl, LzHist h, int iflag) {
    constexpr int CH = 48;
    __shared__ double s_rho[kMaxPoles][CH], s_mu[kMaxPoles][CH], s_y[kMaxPoles][CH];
    __shared__ double s_anum[kMaxPoles];
    const int m = ctl->m, n = ctl->npole;
    const int64_t H = kMaxIter + 2;
    const int k = threadIdx.x;
    if (k < n) s_anum[k] = ctl->anum[k];
    double y = 0.0;
    for (int hi = m; hi >= 1; hi -= CH) {
        const int lo = hi - CH + 1 > 1 ? hi - CH + 1 : 1;
        const int len = hi - lo + 1;
        for (int t = threadIdx.x; t < n * len; t += blockDim.x) {
            const int kk = t / len, o = t - kk * len;
            s_rho[kk][o] = h.rho[kk * H + lo + o];
            s_mu[kk][o] = h.mu[kk * H + lo + o + 1];
        }
        __syncthreads();
        if (k < n) {
            for (int o = len - 1; o >= 0; o--) {
                const int i = lo + o;
                y = i == m ? s_rho[k][o] : __dsub_rn(s_rho[k][o], __dmul_rn(s_mu[k][o], y));
                s_y[k][o] = y;
                h.y[k * H + i] = y;
            }
        }
        __syncthreads();
        if (iflag == 0) {
            for (int o = threadIdx.x; o < len; o += blockDim.x) {
                double c = 0.0;
                for (int kk = 0; kk < n; kk++) c = __dadd_rn(c, __dmul_rn(s_anum[kk], s_y[kk][o]));
                h.c[lo + o] = c;
            }
        }
        __syncthreads();
    }
}

// r_1 = Phi in the vector precision; partial sums of |r_1|^2
template <class T>
__global__ void k_lz_source(T* __restrict__ r1, const double2* __restrict__ phi, int64_t n,
                            double* __restrict__ part, int pl) {
    __shared__ double sh[kThreads / 32];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double2 v = phi[i];
        T t;
        t.x = (typename real_of<T>::type)v.x;
        t.y = (typename real_of<T>::type)v.y;
        if constexpr (std::is_same<T, float2>::value) {
            if (pl) sp_put(r1, i, t);
            else r1[i] = t;
        } else {
            r1[i] = t;
        }
        const double2 w = widen(t);
        s += w.x * w.x + w.y * w.y;
    }
    s = block_sum<kThreads>(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_lz_init(LzCtl* ctl, LzHist h, const double* part, int nb) {
    __shared__ double sh[kThreads / 32];
    double s = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) s += part[i];
    s = block_sum<kThreads>(s, sh);
    if (threadIdx.x == 0) {
        const double b = sqrt(s);
        h.beta[1] = b;
        h.invbeta[1] = 1.0 / b;
        ctl->phimod = b;
    }
}

template <class T, int IMASS, bool PAIR, int OCC>
static void launch_pass1_occ(const LzArgsT<T>& a, unsigned nb, cudaStream_t st,
                             const LzSide& side, KernelTimer* tm) {
    // algorithmic bytes: M reads q, writes vt; M^dagger reads vt, r_j, r_{j-1}
    // and writes r_{j+1}; both read chi as REAL*4
    const double V = (double)a.g.kferm * sizeof(T), chi = 12.0 * a.g.kvol;
    if (tm) tm->begin(timer_class<T>(0), st, 2 * V + chi);
    k_lz1_M<T, IMASS, PAIR, OCC><<<nb, kThreads, 0, st>>>(a);
    if (tm) tm->end(st);
    // the scalar step of iteration j on the side stream, beside M^dagger(j)
    cudaEventRecord(side.fork, st);
    cudaStreamWaitEvent(side.stream, side.fork, 0);
    k_lz_pole<T><<<1, kThreads, 0, side.stream>>>(a, (int)nb);
    cudaEventRecord(side.join, side.stream);
    if (tm) tm->begin(timer_class<T>(1), st, 4 * V + chi);
    if (a.wcap > 0) k_lz1_Md<T, IMASS, PAIR, true, OCC><<<nb, kThreads, 0, st>>>(a);
    else k_lz1_Md<T, IMASS, PAIR, false, OCC><<<nb, kThreads, 0, st>>>(a);
    if (tm) tm->end(st);
    cudaStreamWaitEvent(st, side.join, 0);
}

// The point-gather pass 1 at the register budget the autotuner chose: 3
// blocks of 256 a SM (80 registers a thread) or 4 (64 registers).
template <class T, int IMASS, bool PAIR>
static void launch_pass1(const LzArgsT<T>& a, unsigned nb, cudaStream_t st, const LzSide& side,
                         KernelTimer* tm) {
    if (a.occ == 4) launch_pass1_occ<T, IMASS, PAIR, 4>(a, nb, st, side, tm);
    else launch_pass1_occ<T, IMASS, PAIR, 3>(a, nb, st, side, tm);
}

// Row-staged pass 1 (same protocol: M, the scalar step on the side stream,
// M^dagger).  Grid: the blocks that fit on all SMs at once.
template <class T, int IMASS, int PPT>
static void launch_pass1_rows_ppt(const LzArgsT<T>& a, unsigned nb, cudaStream_t st,
                                  const LzSide& side, KernelTimer* tm) {
    const double V = (double)a.g.kferm * sizeof(T), chi = 12.0 * a.g.kvol;
    const unsigned nt = (unsigned)a.rp.nthreads, sm = a.rp.smem;
    if (tm) tm->begin(timer_class<T>(0), st, 2 * V + chi);
    k_lz1_M_rows<T, IMASS, PPT><<<nb, nt, sm, st>>>(a);
    if (tm) tm->end(st);
    cudaEventRecord(side.fork, st);
    cudaStreamWaitEvent(side.stream, side.fork, 0);
    k_lz_pole<T><<<1, kThreads, 0, side.stream>>>(a, (int)nb);
    cudaEventRecord(side.join, side.stream);
    if (tm) tm->begin(timer_class<T>(1), st, 4 * V + chi);
    if (a.wcap > 0) k_lz1_Md_rows<T, IMASS, true, PPT><<<nb, nt, sm, st>>>(a);
    else k_lz1_Md_rows<T, IMASS, false, PPT><<<nb, nt, sm, st>>>(a);
    if (tm) tm->end(st);
    cudaStreamWaitEvent(st, side.join, 0);
}

// One point a thread: the FP64 solves and odd-Ls FP32 solves (even-Ls FP32
// vectors are in the split layout, which only the point-gather kernels read).
template <class T, int IMASS>
static void launch_pass1_rows(const LzArgsT<T>& a, unsigned nb, cudaStream_t st,
                              const LzSide& side, KernelTimer* tm) {
    launch_pass1_rows_ppt<T, IMASS, 1>(a, nb, st, side, tm);
}

// The six pass-1 row kernels of one precision and thread shape.
template <class T, int PPT>
static void lz_rows_kernels(const void* kern[6]) {
    kern[0] = (const void*)k_lz1_M_rows<T, 1, PPT>;
    kern[1] = (const void*)k_lz1_M_rows<T, 3, PPT>;
    kern[2] = (const void*)k_lz1_Md_rows<T, 1, false, PPT>;
    kern[3] = (const void*)k_lz1_Md_rows<T, 1, true, PPT>;
    kern[4] = (const void*)k_lz1_Md_rows<T, 3, false, PPT>;
    kern[5] = (const void*)k_lz1_Md_rows<T, 3, true, PPT>;
}

// Whether pass 1 runs on the row-staged kernels (the autotuner's choice),
// and their plan and grid.
template <class T>
static bool lz_rows_setup(const Geom& g, RowPlan* rp, unsigned* nb, cudaStream_t st) {
    if (stencil_choice(g, (int)sizeof(T), st) != kStencilRows) return false;
    if (!row_plan(g, sizeof(T), rp) || rp->ppt != 1) return false;
    const void* kern[6];
    lz_rows_kernels<T, 1>(kern);
    int dev = 0, nsm = 0, per_sm = 1 << 20;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    for (const void* k : kern) {
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rp->smem) !=
            cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, rp->nthreads, rp->smem) !=
                cudaSuccess || b < 1) {
            cudaGetLastError();
            return false;
        }
        if (b < per_sm) per_sm = b;
    }
    int64_t n = (int64_t)nsm * per_sm;
    if (n > rp->nrows) n = rp->nrows;
    if (n < 1) return false;
    *nb = (unsigned)n;
    return true;
}

// L2 residency of vt = M q_j: k_lz1_M writes it and k_lz1_Md reads it right
// back, so its address range is marked persisting in L2 for the pass-1
// launches instead of taking a DRAM round trip.  The persisting carve-out is
// a limit of this process's context.  Returns the window (num_bytes 0 when
// the device offers none).
static constexpr bool kVtL2Window = true;

static cudaAccessPolicyWindow vt_window(const void* vt, size_t bytes) {
    cudaAccessPolicyWindow w{};
    if (!kVtL2Window) return w;
    int dev = 0, max_win = 0, max_persist = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_win, cudaDevAttrMaxAccessPolicyWindowSize, dev);
    cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev);
    if (max_win <= 0 || max_persist <= 0) return w;
    const size_t win = bytes < (size_t)max_win ? bytes : (size_t)max_win;
    size_t cur = 0;
    cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize);
    const size_t want = win < (size_t)max_persist ? win : (size_t)max_persist;
    if (cur < want && cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) == cudaSuccess)
        cur = want;
    cudaGetLastError();
    if (cur == 0) return w;
    w.base_ptr = const_cast<void*>(vt);
    w.num_bytes = win;
    w.hitRatio = cur >= win ? 1.0f : (float)((double)cur / (double)win);
    w.hitProp = cudaAccessPropertyPersisting;
    w.missProp = cudaAccessPropertyStreaming;
    return w;
}

static void set_stream_window(cudaStream_t st, const cudaAccessPolicyWindow& w) {
    cudaStreamAttrValue v{};
    v.accessPolicyWindow = w;
    cudaStreamSetAttribute(st, cudaStreamAttributeAccessPolicyWindow, &v);
    cudaGetLastError();
}

// Pass 1 is a sequence of identical launch pairs (the iteration index and the
// residual ring live in device memory), so a chunk of them is captured once
// as a CUDA graph and replayed; the graph is rebuilt when any argument
// changes.
template <class T>
static void launch_pass1_any(const LzArgsT<T>& a, unsigned nb, cudaStream_t st, const LzSide& side,
                             KernelTimer* tm, int imass);

template <class T>
static cudaGraphExec_t pass1_graph(LzWork& w, const LzArgsT<T>& a_in, unsigned nb, int imass,
                                   int chunk, cudaStream_t st, const cudaAccessPolicyWindow& win) {
    // pass-1 kernels never touch the pass-2 fields: clear them so one graph
    // serves every solve of this precision (heatbath, hamilton, force)
    LzArgsT<T> a = a_in;
    a.x = nullptr;
    a.xw = nullptr;
    a.npole = 0;
    LzGraph& G = w.graph[sizeof(T) == sizeof(float2) ? 1 : 0][a.wcap > 0 ? 1 : 0];
    const unsigned char* key = reinterpret_cast<const unsigned char*>(&a);
    if (G.exec && G.nb == nb && G.imass == imass && G.chunk == chunk &&
        G.key.size() == sizeof(a) && memcmp(G.key.data(), key, sizeof(a)) == 0)
        return G.exec;
    if (G.exec) cudaGraphExecDestroy(G.exec);
    G.exec = nullptr;
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    for (int c = 0; c < chunk; c++) {
        launch_pass1_any<T>(a, nb, st, w.side, nullptr, imass);
    }
    if (cudaStreamEndCapture(st, &graph) != cudaSuccess || !graph) {
        cudaGetLastError();
        return nullptr;
    }
    if (win.num_bytes) {                 // the L2 window on every captured launch
        size_t nn = 0;
        cudaGraphGetNodes(graph, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        if (nn && cudaGraphGetNodes(graph, nodes.data(), &nn) == cudaSuccess) {
            cudaKernelNodeAttrValue v{};
            v.accessPolicyWindow = win;
            for (cudaGraphNode_t nd : nodes) {
                cudaGraphNodeType t;
                if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
                    cudaGraphKernelNodeSetAttribute(nd, cudaKernelNodeAttributeAccessPolicyWindow, &v);
            }
        }
        cudaGetLastError();
    }
    cudaGraphExec_t exec = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    G.exec = exec;
    G.nb = nb;
    G.imass = imass;
    G.chunk = chunk;
    G.key.assign(key, key + sizeof(a));
    return exec;
}

template <class T, int IMASS, bool PAIR>
static void launch_pass2(const LzArgsT<T>& a, int j, int m, int iflag, cudaStream_t st,
                         KernelTimer& tm) {
    const unsigned nb = lz_direct_blocks<T, PAIR>(a.g.npts);
    const int apply = j < m;
    const double V = (double)a.g.kferm * sizeof(T), chi = 12.0 * a.g.kvol;
    const double acc = iflag == 0 ? 2.0 * a.g.kferm * sizeof(double2) + V : 0.0;
    if (apply) tm.begin(timer_class<T>(3), st, 2 * V + chi + acc);
    if (iflag == 0) k_lz2_M<T, IMASS, 0, PAIR><<<nb, kThreads, 0, st>>>(a, j, apply);
    else k_lz2_M<T, IMASS, 1, PAIR><<<nb, kThreads, 0, st>>>(a, j, apply);
    count_launches(1);
    if (apply) {
        tm.end(st);
        tm.begin(timer_class<T>(3), st, 4 * V + chi);
        k_lz2_Md<T, IMASS, PAIR><<<nb, kThreads, 0, st>>>(a, j);
        tm.end(st);
        count_launches(1);
    }
}

template <class T>
static int pass1_shape(const LzArgsT<T>& a) {
    return a.rows ? kStencilRows : (a.occ == 4 ? kStencilGather4 : kStencilGather3);
}

// Shape dispatch: FP32 vectors with Ls even take the two-point kernels.
template <class T>
static bool lz_pair(const Geom& g) {
    return std::is_same<T, float2>::value && pair_ok(g);
}

template <class T>
static void launch_pass1_any(const LzArgsT<T>& a, unsigned nb, cudaStream_t st, const LzSide& side,
                             KernelTimer* tm, int imass) {
    if (a.rows) {
        if (imass == 3) launch_pass1_rows<T, 3>(a, nb, st, side, tm);
        else launch_pass1_rows<T, 1>(a, nb, st, side, tm);
        return;
    }
    if constexpr (std::is_same<T, float2>::value) {
        if (lz_pair<T>(a.g)) {
            if (imass == 3) launch_pass1<T, 3, true>(a, nb, st, side, tm);
            else launch_pass1<T, 1, true>(a, nb, st, side, tm);
            return;
        }
    }
    if (imass == 3) launch_pass1<T, 3, false>(a, nb, st, side, tm);
    else launch_pass1<T, 1, false>(a, nb, st, side, tm);
}

template <class T>
static void launch_pass2_any(const LzArgsT<T>& a, int j, int m, int iflag, cudaStream_t st,
                             KernelTimer& tm, int imass) {
    if constexpr (std::is_same<T, float2>::value) {
        if (lz_pair<T>(a.g)) {
            if (imass == 3) launch_pass2<T, 3, true>(a, j, m, iflag, st, tm);
            else launch_pass2<T, 1, true>(a, j, m, iflag, st, tm);
            return;
        }
    }
    if (imass == 3) launch_pass2<T, 3, false>(a, j, m, iflag, st, tm);
    else launch_pass2<T, 1, false>(a, j, m, iflag, st, tm);
}

template <class T, bool PAIR>
static unsigned lz_pass1_blocks_occ(const Geom& g, int imass, int occ) {
    if (occ == 4)
        return imass == 3 ? lz_pass1_blocks<T, 3, PAIR, 4>(g.npts)
                          : lz_pass1_blocks<T, 1, PAIR, 4>(g.npts);
    return imass == 3 ? lz_pass1_blocks<T, 3, PAIR, 3>(g.npts)
                      : lz_pass1_blocks<T, 1, PAIR, 3>(g.npts);
}

template <class T>
static unsigned lz_pass1_blocks_any(const Geom& g, int imass, int occ) {
    if constexpr (std::is_same<T, float2>::value) {
        if (lz_pair<T>(g)) return lz_pass1_blocks_occ<T, true>(g, imass, occ);
    }
    return lz_pass1_blocks_occ<T, false>(g, imass, occ);
}

// ---- kernel timer ----------------------------------------------------------
void KernelTimer::enable() {
    if (enabled) return;
    for (int i = 0; i < 2 * kPool; i++) cudaEventCreate(&ev[i]);
    for (int i = 0; i < 2 * kChunkPool; i++) cudaEventCreate(&cev[i]);
    enabled = true;
    reset();
}

void KernelTimer::release() {
    if (!enabled) return;
    for (int i = 0; i < 2 * kPool; i++) cudaEventDestroy(ev[i]);
    for (int i = 0; i < 2 * kChunkPool; i++) cudaEventDestroy(cev[i]);
    enabled = false;
    chunks = false;
}

void KernelTimer::chunk_begin(cudaStream_t st, int first) {
    if (!enabled || cused >= kChunkPool) return;
    cfirst[cused] = first;
    cudaEventRecord(cev[2 * cused], st);
}

void KernelTimer::chunk_end(cudaStream_t st) {
    if (!enabled || cused >= kChunkPool) return;
    cudaEventRecord(cev[2 * cused + 1], st);
    cused++;
}

void KernelTimer::collect_chunks(int m, int chunk, int prec) {
    if (!enabled) return;
    for (int i = 0; i < cused; i++) {
        float ms = 0.0f;
        if (cfirst[i] + chunk - 1 <= m &&
            cudaEventElapsedTime(&ms, cev[2 * i], cev[2 * i + 1]) == cudaSuccess) {
            chunk_ms[prec] += ms;
            chunk_iters[prec] += chunk;
        }
    }
    cused = 0;
}

void KernelTimer::reset() {
    used = 0;
    for (int c = 0; c < kClasses; c++) {
        total_ms[c] = 0;
        total_bytes[c] = 0;
        count[c] = 0;
        launches[c] = 0;
    }
    cused = 0;
    chunk_ms[0] = chunk_ms[1] = 0.0;
    chunk_iters[0] = chunk_iters[1] = 0;
}

void KernelTimer::begin(int c, cudaStream_t st, double nbytes) {
    if (!enabled) return;
    launches[c]++;
    if (used >= kPool) return;          // pool full: the launch is counted, not timed
    cls[used] = c;
    bytes[used] = nbytes;
    cudaEventRecord(ev[2 * used], st);
}

void KernelTimer::end(cudaStream_t st) {
    if (!enabled || used >= kPool) return;
    cudaEventRecord(ev[2 * used + 1], st);
    used++;
}

void KernelTimer::collect() {
    if (!enabled) return;
    for (int i = 0; i < used; i++) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]) == cudaSuccess) {
            total_ms[cls[i]] += ms;
            total_bytes[cls[i]] += bytes[i];
            count[cls[i]]++;
        }
    }
    used = 0;
}

LzWork::~LzWork() {
    release();
    timer.release();
}

void LzWork::release() {
    for (auto& row : graph)
        for (LzGraph& gr : row) {
            if (gr.exec) cudaGraphExecDestroy(gr.exec);
            gr = LzGraph();
        }
    if (side.fork) cudaEventDestroy(side.fork);
    if (side.join) cudaEventDestroy(side.join);
    if (side.stream) cudaStreamDestroy(side.stream);
    side = LzSide();
    if (ctl) cudaFree(ctl);
    if (hist_mem) cudaFree(hist_mem);
    if (part) cudaFree(part);
    if (hflag_host) cudaFreeHost(hflag_host);
    for (int i = 0; i < 3; i++) {
        if (rb[i]) cudaFree(rb[i]);
        if (rb32[i]) cudaFree(rb32[i]);
    }
    if (vt) cudaFree(vt);
    if (vt32) cudaFree(vt32);
    if (basis) cudaFree(basis);
    if (basis32) cudaFree(basis32);
    if (wall) cudaFree(wall);
    if (wall32) cudaFree(wall32);
    basis = nullptr;
    basis32 = nullptr;
    wall = nullptr;
    wall32 = nullptr;
    hcap = hcap32 = 0;
    wcap = wcap32 = 0;
    if (xw) cudaFree(xw);
    if (x2w) cudaFree(x2w);
    ctl = nullptr; hist_mem = nullptr; part = nullptr; hflag_host = nullptr;
    rb[0] = rb[1] = rb[2] = vt = xw = x2w = nullptr;
    rb32[0] = rb32[1] = rb32[2] = vt32 = nullptr;
    xw_poles = 0;
}

cudaError_t LzWork::ensure(const Geom& g, int npole_max, int prec, bool walls) {
    cudaError_t e;
    const bool same = ctl && g.kferm == geom.kferm && g.L == geom.L && g.Lt == geom.Lt;
    if (!same) {
        release();
        geom = g;
        if ((e = cudaMalloc(&ctl, sizeof(LzCtl)))) return e;
        const int64_t H = kMaxIter + 2;
        const size_t nh = 4 * H + 3 * (size_t)kMaxPoles * H;
        if ((e = cudaMalloc(&hist_mem, nh * sizeof(double)))) return e;
        hist.alphat = hist_mem;
        hist.beta = hist_mem + H;
        hist.invbeta = hist_mem + 2 * H;
        hist.c = hist_mem + 3 * H;
        hist.rho = hist_mem + 4 * H;
        hist.mu = hist.rho + kMaxPoles * H;
        hist.y = hist.mu + kMaxPoles * H;
        // block partials of the two pass-1 kernels (at most split_blocks
        // blocks each), and the source norm's block partials
        const int64_t nb = 2 * (int64_t)split_blocks(g.npts);
        if ((e = cudaMalloc(&part, sizeof(double) * (nb + 2048)))) return e;
        if ((e = cudaHostAlloc(&hflag_host, sizeof(int), cudaHostAllocMapped))) return e;
        if ((e = cudaStreamCreateWithFlags(&side.stream, cudaStreamNonBlocking))) return e;
        if ((e = cudaEventCreateWithFlags(&side.fork, cudaEventDisableTiming))) return e;
        if ((e = cudaEventCreateWithFlags(&side.join, cudaEventDisableTiming))) return e;
        if ((e = cudaHostGetDevicePointer((void**)&hflag_dev, hflag_host, 0))) return e;
    }
    if (prec == kPrecF64 && !rb[0]) {
        for (int i = 0; i < 3; i++)
            if ((e = cudaMalloc(&rb[i], sizeof(double2) * g.kferm))) return e;
        if ((e = cudaMalloc(&vt, sizeof(double2) * g.kferm))) return e;
    }
    if (prec == kPrecF32 && !rb32[0]) {
        for (int i = 0; i < 3; i++)
            if ((e = cudaMalloc(&rb32[i], sizeof(float2) * g.kferm))) return e;
        if ((e = cudaMalloc(&vt32, sizeof(float2) * g.kferm))) return e;
    }
    // Basis store: up to kMaxIter+2 vectors, at most 40% of the free HBM per
    // precision.  Solves longer than the store regenerate their vectors.
    if (basis_enabled && ((prec == kPrecF64 && !basis) || (prec == kPrecF32 && !basis32))) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        const size_t vb = (prec == kPrecF64 ? sizeof(double2) : sizeof(float2)) * (size_t)g.kferm;
        // an explicit budget names the FP64 store; the FP32 store keeps the
        // same number of vectors in half the bytes
        const double budget = basis_max_bytes >= 0.0
                                  ? basis_max_bytes * (prec == kPrecF64 ? 1.0 : 0.5)
                                  : 0.4 * (double)fr;
        int64_t cap = (int64_t)(budget / (double)vb);
        if (cap > kMaxIter + 2) cap = kMaxIter + 2;
        if (cap >= 8) {
            void* ptr = nullptr;
            if (cudaMalloc(&ptr, vb * (size_t)cap) == cudaSuccess) {
                if (prec == kPrecF64) { basis = (double2*)ptr; hcap = (int)cap; }
                else { basis32 = (float2*)ptr; hcap32 = (int)cap; }
            } else {
                cudaGetLastError();   // not enough memory: regenerate instead
            }
        }
    }
    // Wall store: up to kMaxIter+2 two-slice vectors within 15% of the free
    // HBM; force solves that outgrow it regenerate their vectors.
    if (walls && basis_enabled && ((prec == kPrecF64 && !wall) || (prec == kPrecF32 && !wall32))) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        const size_t vb = (prec == kPrecF64 ? sizeof(double2) : sizeof(float2)) * 16 * (size_t)g.kvol;
        int64_t cap = (int64_t)(0.15 * (double)fr / (double)vb);
        if (cap > kMaxIter + 2) cap = kMaxIter + 2;
        if (cap >= 8) {
            void* ptr = nullptr;
            if (cudaMalloc(&ptr, vb * (size_t)cap) == cudaSuccess) {
                if (prec == kPrecF64) { wall = (double2*)ptr; wcap = (int)cap; }
                else { wall32 = (float2*)ptr; wcap32 = (int)cap; }
            } else {
                cudaGetLastError();
            }
        }
    }
    if (npole_max > xw_poles) {
        if (xw) cudaFree(xw);
        if (x2w) cudaFree(x2w);
        xw_poles = npole_max;
        const size_t nw = (size_t)xw_poles * 16 * g.kvol;
        if ((e = cudaMalloc(&xw, sizeof(double2) * nw))) return e;
        if ((e = cudaMalloc(&x2w, sizeof(double2) * nw))) return e;
    }
    return cudaSuccess;
}

template <class T>
static void set_ring(LzArgsT<T>& a, LzWork& w);
template <>
void set_ring<double2>(LzArgsT<double2>& a, LzWork& w) {
    a.rb0 = w.rb[0]; a.rb1 = w.rb[1]; a.rb2 = w.rb[2]; a.vt = w.vt;
    a.basis = w.basis_enabled ? w.basis : nullptr;
    a.hcap = a.basis ? w.hcap : 0;
}
template <>
void set_ring<float2>(LzArgsT<float2>& a, LzWork& w) {
    a.rb0 = w.rb32[0]; a.rb1 = w.rb32[1]; a.rb2 = w.rb32[2]; a.vt = w.vt32;
    a.basis = w.basis_enabled ? w.basis32 : nullptr;
    a.hcap = a.basis ? w.hcap32 : 0;
}

// Force solves with a wall store keep only the ring and the wall slices.
template <class T>
static void set_walls(LzArgsT<T>& a, LzWork& w) {
    T* ws;
    int cap;
    if constexpr (std::is_same<T, double2>::value) { ws = w.wall; cap = w.wcap; }
    else { ws = w.wall32; cap = w.wcap32; }
    if (!w.basis_enabled || !ws) return;
    a.wbasis = ws;
    a.wcap = cap;
    a.basis = nullptr;
    a.hcap = 0;
}

// The two wall slices of r (s = 1 and s = Ls) into wall-store vector j, laid
// out as the wall fields: element (slice sw, component c, site) at
// sw + 2 site + 2 kvol c.
template <class T>
__global__ void __launch_bounds__(kThreads) k_lz_walls_of(LzArgsT<T> a, const T* __restrict__ r,
                                                         int j) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t cs2 = 2 * (int64_t)a.g.kvol;
    if (t >= 8 * cs2) return;
    const int c = (int)(t / cs2);
    const int64_t rr = t - c * cs2;
    const int sw = (int)(rr & 1);
    const int64_t site = rr >> 1;
    a.wbasis[(int64_t)j * 8 * cs2 + t] =
        vget(a, r, (sw ? a.g.Ls - 1 : 0) + (int64_t)a.g.Ls * site + a.g.cs * c);
}

// q_j's wall slices (j = 1..m) into every pole's two-slice x_k: the same
// sums, in the same order, as from the full stored vectors.  One thread per
// wall element (slice, component, site) and NC poles per pass (one pass for
// up to 24 poles), so the store is read once or twice; the pass's y_kj and 1/beta_j
// are staged in shared memory kYChunk iterations at a time.  STORE: the q_j
// come from the wall store (coalesced), else from the stored basis.
constexpr int kYChunk = 32;
template <class T, int NC, bool STORE>
__global__ void __launch_bounds__(kThreads, 2) k_lz_accum_walls(LzArgsT<T> a, int m, int k0) {
    typedef typename real_of<T>::type Real;
    __shared__ double ys[NC][kYChunk];
    __shared__ Real ibs[kYChunk];
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t cs2 = 2 * (int64_t)a.g.kvol, kf2 = 8 * cs2;
    const bool act = t < kf2;
    int64_t e = t, stride = kf2;
    const T* src = a.wbasis;
    if (!STORE) {
        const int c = act ? (int)(t / cs2) : 0;             // component
        const int64_t r = act ? t - c * cs2 : 0;           // s' + 2 site
        e = ((r & 1) ? a.g.Ls - 1 : 0) + (int64_t)a.g.Ls * (r >> 1) + a.g.cs * c;
        stride = a.g.kferm;
        src = a.basis;
    }
    const int64_t H = kMaxIter + 2;
    const int n = a.npole;
    double2 acc[NC];
#pragma unroll
    for (int k = 0; k < NC; k++) acc[k] = make_double2(0.0, 0.0);
    for (int j0 = 1; j0 <= m; j0 += kYChunk) {
        const int jn = m - j0 + 1 < kYChunk ? m - j0 + 1 : kYChunk;
        __syncthreads();
        for (int i = threadIdx.x; i < NC * kYChunk; i += blockDim.x) {
            const int k = i / kYChunk, jj = i - k * kYChunk;
            ys[k][jj] = (k0 + k < n && jj < jn) ? a.h.y[(k0 + k) * H + j0 + jj] : 0.0;
        }
        for (int i = threadIdx.x; i < kYChunk; i += blockDim.x)
            ibs[i] = i < jn ? (Real)a.h.invbeta[j0 + i] : (Real)0;
        __syncthreads();
        if (act) {
            // q_{j+1} is loaded while q_j is accumulated
            const int64_t b = e + j0 * stride;
            T qn = STORE ? __ldg(src + b) : vget(a, src, b);
#pragma unroll 1
            for (int jj = 0; jj < jn; jj++) {
                const T q = qn;
                if (jj + 1 < jn) {
                    const int64_t bn = b + (jj + 1) * stride;
                    qn = STORE ? __ldg(src + bn) : vget(a, src, bn);
                }
                const double2 qj = widen(zscal(ibs[jj], q));
#pragma unroll
                for (int k = 0; k < NC; k++) {
                    const double y = ys[k][jj];
                    acc[k].x += y * qj.x;
                    acc[k].y += y * qj.y;
                }
            }
        }
    }
    if (!act) return;
#pragma unroll
    for (int k = 0; k < NC; k++)
        if (k0 + k < n) a.xw[(k0 + k) * kf2 + t] = acc[k];
}

template <class T, bool STORE>
static void launch_accum_walls(const LzArgsT<T>& a, int m, int n, int64_t kvol, cudaStream_t st) {
    const unsigned nb = (unsigned)((16 * kvol + kThreads - 1) / kThreads);
    for (int k0 = 0; k0 < n; k0 += 24) {
        const int left = n - k0;
        if (left <= 8) k_lz_accum_walls<T, 8, STORE><<<nb, kThreads, 0, st>>>(a, m, k0);
        else if (left <= 16) k_lz_accum_walls<T, 16, STORE><<<nb, kThreads, 0, st>>>(a, m, k0);
        else k_lz_accum_walls<T, 24, STORE><<<nb, kThreads, 0, st>>>(a, m, k0);
        count_launches(1);
    }
}

// ---- pass 2 from the stored basis ---------------------------------------
// x += sum_j c_j q_j, q_j = r_j / beta_j, j = 1..m, in j order per element
// (the same sequence of operations as the regenerating pass 2).
template <class T>
__global__ void __launch_bounds__(kThreads) k_lz_accum_x(LzArgsT<T> a, int j0, int j1) {
    typedef typename real_of<T>::type Real;
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= a.g.kferm) return;
    double2 xv = a.x[e];
    const int64_t stride = a.g.kferm;
#pragma unroll 4
    for (int j = j0; j <= j1; j++) {
        const double2 qj = widen(zscal((Real)a.h.invbeta[j], vget(a, a.basis, e + j * stride)));
        const double cj = a.h.c[j];
        xv.x += cj * qj.x;
        xv.y += cj * qj.y;
    }
    a.x[e] = xv;
}

static constexpr int kAccumChunk = 64;

// Per-shift solutions (iflag 2): x_k = sum_j y_kj q_j for poles k0..k0+7,
// every element summing j = 1..m in order; xk[k] are device pointers.
template <class T>
__global__ void __launch_bounds__(kThreads) k_lz_accum_poles(LzArgsT<T> a, int m, int k0,
                                                             double2* const* xk) {
    typedef typename real_of<T>::type Real;
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= a.g.kferm) return;
    const int64_t H = kMaxIter + 2, stride = a.g.kferm;
    const int n = a.npole;
    double2 acc[8];
#pragma unroll
    for (int k = 0; k < 8; k++) acc[k] = make_double2(0.0, 0.0);
    for (int j = 1; j <= m; j++) {
        const double2 qj = widen(zscal((Real)a.h.invbeta[j], vget(a, a.basis, j * stride + e)));
#pragma unroll
        for (int k = 0; k < 8; k++) {
            if (k0 + k < n) {
                const double y = a.h.y[(k0 + k) * H + j];
                acc[k].x += y * qj.x;
                acc[k].y += y * qj.y;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 8; k++)
        if (k0 + k < n) xk[k0 + k][e] = acc[k];
}


template <class T>
static cudaError_t lz_solve_t(LzWork& w, const Geom& g, const double2* phi, float res, int ndiag,
                              const double* anum, const double* aden, int iflag,
                              const float* chif, float am3, float hpin, int imass, int ibound,
                              double2* x, float* dSdchi, int* itercg, int* status,
                              LzStats* stats, cudaStream_t st) {
    typedef typename real_of<T>::type Real;
    cudaError_t e;
    LzCtl hc;
    memset(&hc, 0, sizeof(hc));
    hc.it_m = 1;
    hc.npole = ndiag;
    hc.niter_cap = kMaxIter;
    const float resid = sqrtf((float)g.kferm * res * res);   // :621
    const float arelax = 2.0f;                                // :711
    hc.thresh = (double)(arelax * resid);
    for (int k = 0; k < ndiag; k++) {
        hc.sigma[k] = aden[k];
        hc.anum[k] = anum[k + 1];
    }
    if ((e = cudaMemcpyAsync(w.ctl, &hc, sizeof(hc), cudaMemcpyHostToDevice, st))) return e;
    *w.hflag_host = 0;

    LzArgsT<T> a;
    memset(&a, 0, sizeof(a));
    a.g = g;
    set_ring(a, w);
    if (iflag == 1) set_walls(a, w);
    a.chif = chif;
    a.diag = (Real)(2.0f * ((3.0f - am3) + 1.0f));
    a.hpin = (Real)hpin;
    a.apbc = ibound == -1;
    a.ctl = w.ctl;
    a.h = w.hist;
    a.part = w.part;
    a.hflag = w.hflag_dev;
    a.x = x;
    a.xw = w.xw;
    a.npole = ndiag;
    unsigned nb = 0;
    // FP32 vectors with Ls even live in the split layout, which only the
    // point-gather kernels read (the row-staged shape serves the FP64 solves
    // and odd Ls)
    a.pl = lz_pair<T>(g) ? 1 : 0;
    a.rows = !a.pl && lz_rows_setup<T>(g, &a.rp, &nb, st) ? 1 : 0;
    a.occ = (a.pl ? stencil_choice_split(g, st) : stencil_choice(g, (int)sizeof(T), st)) ==
                    kStencilGather4
                ? 4
                : 3;
    if (!a.rows) nb = lz_pass1_blocks_any<T>(g, imass, a.occ);
    const int nbr = reduce_blocks(g.kferm);
    // r_1 lives where ring(a, 1) looks for it: the basis store when present
    T* r1 = a.hcap > 1 ? a.basis + g.kferm : a.rb1;

    // r_1 = Phi, beta_1 = |r_1|
    k_lz_source<T><<<nbr, kThreads, 0, st>>>(r1, phi, g.kferm, w.part, a.pl);
    k_lz_init<<<1, kThreads, 0, st>>>(w.ctl, w.hist, w.part, nbr);
    count_launches(2);
    if (a.wcap > 1) {                    // r_1's wall slices (pass 1 adds r_2, r_3, ...)
        k_lz_walls_of<T><<<(unsigned)((16 * (int64_t)g.kvol + kThreads - 1) / kThreads), kThreads,
                           0, st>>>(a, r1, 1);
        count_launches(1);
    }

    // pass 1: launch chunks of iterations and poll the mapped flag with
    // kAhead chunks queued beyond the one being checked, so a host thread
    // that wakes late still finds the GPU busy
    const int chunk = 16;
    constexpr int kAhead = 2;
    cudaEvent_t ev[kAhead + 1];
    for (cudaEvent_t& e : ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    int launched = 0, nchunk = 0;
    // the per-launch path when kernels are being timed, else graph replays
    const cudaAccessPolicyWindow win = vt_window(a.vt, sizeof(T) * (size_t)g.kferm);
    if (win.num_bytes) set_stream_window(st, win);
    // per-launch timing issues pass 1 launch by launch; chunk timing keeps
    // the graph replays and brackets each one
    const bool chunked = w.timer.enabled && w.timer.chunks;
    cudaGraphExec_t gexec = w.timer.enabled && !chunked
                                ? nullptr
                                : pass1_graph<T>(w, a, nb, imass, chunk, st, win);
    while (launched < kMaxIter) {
        if (gexec) {
            if (chunked) w.timer.chunk_begin(st, launched + 1);
            cudaGraphLaunch(gexec, st);
            if (chunked) w.timer.chunk_end(st);
            launched += chunk;
            count_launches(3 * chunk);
            note_stencil(pass1_shape(a), 2 * chunk);
        } else {
            for (int c = 0; c < chunk && launched < kMaxIter; c++, launched++) {
                launch_pass1_any<T>(a, nb, st, w.side, &w.timer, imass);
                count_launches(3);
                note_stencil(pass1_shape(a), 2);
            }
        }
        cudaEventRecord(ev[nchunk % (kAhead + 1)], st);
        if (nchunk >= kAhead) {
            cudaEventSynchronize(ev[(nchunk - kAhead) % (kAhead + 1)]);
            if (*(volatile int*)w.hflag_host) break;
        }
        nchunk++;
    }
    if (chunked) {
        cudaStreamSynchronize(st);
        LzCtl hm;
        cudaMemcpy(&hm, w.ctl, sizeof(hm), cudaMemcpyDeviceToHost);
        w.timer.collect_chunks(hm.m, chunk, std::is_same<T, float2>::value ? 1 : 0);
    } else if (w.timer.enabled) {
        // launches after convergence returned at once: drop them
        cudaStreamSynchronize(st);
        LzCtl hm;
        cudaMemcpy(&hm, w.ctl, sizeof(hm), cudaMemcpyDeviceToHost);
        int keep = 0;
        for (int i = 0, it = 0; i < w.timer.used; i++) {
            if (w.timer.cls[i] == timer_class<T>(0)) it++;
            const bool real = it <= hm.m;      // M^dagger(m) completes too
            if (real) {
                w.timer.cls[keep] = w.timer.cls[i];
                w.timer.bytes[keep] = w.timer.bytes[i];
                std::swap(w.timer.ev[2 * keep], w.timer.ev[2 * i]);
                std::swap(w.timer.ev[2 * keep + 1], w.timer.ev[2 * i + 1]);
                keep++;
            }
        }
        w.timer.launches[timer_class<T>(0)] -= launched - hm.m;
        w.timer.launches[timer_class<T>(1)] -= launched - hm.m;
        w.timer.used = keep;
        w.timer.collect();
    }
    for (cudaEvent_t& e : ev) cudaEventDestroy(e);   // the stream sync below covers them
    if (win.num_bytes) set_stream_window(st, cudaAccessPolicyWindow{});
    if ((e = cudaGetLastError())) return e;
    LzCtl hr;
    if ((e = cudaMemcpyAsync(&hr, w.ctl, sizeof(hr), cudaMemcpyDeviceToHost, st))) return e;
    if ((e = cudaStreamSynchronize(st))) return e;
    const int m = hr.m;
    *itercg = m;
    if (hr.done == 4) return cudaErrorLaunchTimeout;   // a staged copy never arrived
    *status = hr.done == 1 ? 0 : (hr.done == 2 ? 1 : 2);
    if (stats) { stats->iters = m; stats->pass1_launches = 2 * launched; }
    if (m < 1) return cudaErrorUnknown;

    // coefficients, then pass 2 over the regenerated vectors
    k_lz_coeffs<<<1, kThreads, 0, st>>>(w.ctl, w.hist, iflag);
    k_lz_source<T><<<nbr, kThreads, 0, st>>>(r1, phi, g.kferm, w.part, a.pl);
    count_launches(2);
    if (iflag == 2) {
        // every x_k from the stored basis, poles in chunks of 8 (one pass over
        // the basis per chunk); needs the whole basis in HBM
        if (!(m < a.hcap) || !w.pole_out) return cudaErrorInvalidValue;
        const unsigned nbx = (unsigned)((g.kferm + kThreads - 1) / kThreads);
        for (int k0 = 0; k0 < ndiag; k0 += 8) {
            k_lz_accum_poles<T><<<nbx, kThreads, 0, st>>>(a, m, k0, w.pole_out);
            count_launches(1);
        }
        return cudaGetLastError();
    }
    launch_scale(x, phi, anum[0], g.kferm, st);                       // x = a0 Phi (:628)
    if (iflag == 1) cudaMemsetAsync(w.xw, 0, sizeof(double2) * (size_t)ndiag * 16 * g.kvol, st);
    if (a.wcap > 0 ? m < a.wcap : m < a.hcap) {
        // every q_j (or, for the force, its wall slices) is still in HBM:
        // one streaming pass over the store reads the m stored vectors and
        // the solution once
        const double vb = (double)sizeof(T);
        const double nbytes = iflag == 0
            ? (double)m * g.kferm * vb + 2.0 * g.kferm * sizeof(double2)
            : (double)m * 16.0 * g.kvol * vb + (double)ndiag * 16.0 * g.kvol * sizeof(double2);
        w.timer.begin(timer_class<T>(2), st, nbytes);
        if (iflag == 0) {
            // a chunk of stored vectors per launch: x (FP64) is carried in
            // memory between chunks, so each element still sums j = 1..m in
            // order, and the pages a launch touches stay few
            const unsigned nbx = (unsigned)((g.kferm + kThreads - 1) / kThreads);
            for (int j0 = 1; j0 <= m; j0 += kAccumChunk) {
                const int j1 = j0 + kAccumChunk - 1 < m ? j0 + kAccumChunk - 1 : m;
                k_lz_accum_x<T><<<nbx, kThreads, 0, st>>>(a, j0, j1);
                count_launches(1);
            }
        } else if (a.wcap > 0) {
            launch_accum_walls<T, true>(a, m, ndiag, g.kvol, st);
        } else {
            launch_accum_walls<T, false>(a, m, ndiag, g.kvol, st);
        }
        w.timer.end(st);
    } else {
        for (int j = 1; j <= m; j++) {
            launch_pass2_any<T>(a, j, m, iflag, st, w.timer, imass);
            if (w.timer.enabled && w.timer.used >= KernelTimer::kPool - 2) {
                cudaStreamSynchronize(st);
                w.timer.collect();
            }
        }
    }
    if (w.timer.enabled) {
        cudaStreamSynchronize(st);
        w.timer.collect();
    }
    if (iflag == 1) {
        // X2 = M x_k on the walls, then derivs pole by pole (:733-740)
        launch_wall_dslash64(ndiag, w.x2w, w.xw, chif, g, am3, hpin, ibound, imass, st);
        const double* anum_dev = reinterpret_cast<const double*>(
            reinterpret_cast<const char*>(w.ctl) + offsetof(LzCtl, anum));
        launch_derivs_walls(ndiag, w.xw, w.x2w, anum_dev, imass, dSdchi, g, st);
    }
    return cudaGetLastError();
}

// Multi-shift solve.  anum[0..n], aden[0..n-1] as in the reference.
// iflag 0: x = a0 Phi + sum_k a_k x_k.  iflag 1: x = a0 Phi and the force
// contribution of every pole is accumulated into dSdchi (device, REAL*4).
cudaError_t lz_solve(LzWork& w, const Geom& g, const double2* phi, float res, int ndiag,
                     const double* anum, const double* aden, int iflag, const float* chif,
                     float am3, float hpin, int imass, int ibound, double2* x, float* dSdchi,
                     int* itercg, int* status, LzStats* stats, cudaStream_t st, int prec) {
    if (ndiag < 1 || ndiag > kMaxPoles) return cudaErrorInvalidValue;
    cudaError_t e = w.ensure(g, iflag == 1 ? ndiag : 1, prec, iflag == 1);
    if (e) return e;
    if (prec == kPrecF32)
        return lz_solve_t<float2>(w, g, phi, res, ndiag, anum, aden, iflag, chif, am3, hpin,
                                  imass, ibound, x, dSdchi, itercg, status, stats, st);
    return lz_solve_t<double2>(w, g, phi, res, ndiag, anum, aden, iflag, chif, am3, hpin, imass,
                               ibound, x, dSdchi, itercg, status, stats, st);
}

}  // namespace chdwf
