// row_stage.cuh -- shared-memory row staging for the stencil kernels.
//
// A "row" is the set of points with fixed (y, t): L*Ls consecutive points of
// every component plane (the layout has s innermost, then x), i.e. one
// contiguous run of L*Ls elements per plane.  A block walks a contiguous
// range of output rows rho = (f*Lt + t)*L + y of one flavour f.  For output
// row (f, t, y) the four Dirac planes of flavour f on rows y-1, y, y+1 (same
// t) and on rows t-1, t+1 (same y) are held in shared memory: they serve the
// diagonal term and the x, y, t and s hops.  Only the wall terms read
// global memory (the other flavour at the other wall, 2 of every Ls points,
// and chi), issued one output row ahead, as are the vectors a kernel streams
// besides its stencil input.
//
// The block is warp-specialised.  Lane 0 of its last warp is the producer:
// it moves rows into shared memory with 1-D bulk copies (cp.async.bulk, the
// TMA engine's untiled form, this GPU's own memory only, no multicast).  The
// other warps are consumers: each thread evaluates PPT adjacent points of
// the row (PPT = 2 for FP32/FP16 storage with Ls even, so every shared load
// is 16 or 8 bytes holding both points; else 1).  Two rings hold the rows:
//   * the window ring of kRowSlots rows along y.  The window rows of a block
//     are loaded in order: for each maximal run of output rows with the same
//     (f, t), rows y_a-1, y_a, ..., y_b (mod L), i.e. run length + 2 loads.
//     Output row k of a run needs loads u, u+1, u+2 (u = run base + k).
//     Load w is the (w / kRowSlots)-th use of slot w % kRowSlots;
//   * the t ring of kRowTEnt entries, entry k holding rows (t+1, y) and
//     (t-1, y) of the block's k-th output row; entry k is the
//     (k / kRowTEnt)-th use of its slot.
// Every slot has a "full" mbarrier (the producer's expect-tx arrival plus
// the copies' bytes) and an "empty" one (one arrival per consumer warp when
// the warp no longer needs the slot's rows).  The producer refills a slot
// only after its empty barrier has completed the previous use, so each slot
// has at most one copy in flight and both barriers' wait parities follow
// from the use count.  No block-wide barrier is taken inside the loop: a
// consumer warp goes on to the next row as soon as that row's copies have
// landed.
//
// Every wait is bounded (kRowWaitNs).  A thread whose wait runs out sets the
// block's error flag; the others see it at their next row and leave, the
// producer stops issuing, waits (bounded again) for the copies it has in
// flight, and the block reports the failure after its final barrier.
#pragma once
#include <cuda_fp16.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "dwf_stencil.cuh"

namespace chdwf {

constexpr int kRowSlots = 5;                      // window ring (rows along y)
constexpr int kRowTEnt = 3;                       // t ring entries (two rows each)
// mbarriers: full window, full t, empty window, empty t
constexpr int kRowFullT = kRowSlots;
constexpr int kRowEmptyY = kRowSlots + kRowTEnt;
constexpr int kRowEmptyT = 2 * kRowSlots + kRowTEnt;
constexpr int kRowBars = 2 * (kRowSlots + kRowTEnt);
constexpr uint64_t kRowWaitNs = 1000000000ull;   // 1 s per wait
constexpr unsigned kRowBarBytes = 128;            // mbarriers at the front of shared memory
static_assert(kRowBars * 8 <= (int)kRowBarBytes, "mbarriers exceed their area");
constexpr unsigned kRowSmemMax = 227 * 1024;

// Register budget of the row kernels and the block size it allows: a
// block's warps are spread over the SM's four sub-partitions, each with a
// quarter of the register file (16384), so ceil(warps / 4) * 32 * registers
// must not exceed 16384.
constexpr int kRowRegs = 128;
constexpr int kRowMaxThreads = 512;               // consumer warps + the producer warp
static_assert((kRowMaxThreads / 32 + 3) / 4 * 32 * kRowRegs <= 16384,
              "a row block does not fit a sub-partition's registers");

// Which stencil kernels run, from the environment variable CHDWF_STENCIL:
// 0 (unset): the autotuner's choice per lattice and precision (tune.cu);
// 1 ("legacy"): the point-gather kernels at 3 blocks a SM; 2 ("rows"): row
// kernels wherever they fit (tests use it to run them on small lattices);
// 3 ("gather4"): the point-gather kernels at 4 blocks a SM.
inline int stencil_mode() {
    const char* v = getenv("CHDWF_STENCIL");
    if (!v) return 0;
    if (strcmp(v, "legacy") == 0) return 1;
    if (strcmp(v, "rows") == 0) return 2;
    if (strcmp(v, "gather4") == 0) return 3;
    return 0;
}

// Launch plan of a row-staged kernel (host-computed, passed by value).
struct RowPlan {
    int Lrow;        // L*Ls points (elements per plane row)
    int nrows;       // 2*Lt*L output rows (flavour, t, y)
    unsigned smem;   // dynamic shared memory bytes
    int nthreads;    // block size: the consumer warps and the producer warp
    int ncw;         // consumer warps
    int ppt;         // points per consumer thread (1 or 2)
};

// Points per consumer thread for storage elements of elem bytes.
inline int row_ppt(const Geom& g, size_t elem) { return (elem <= 8 && g.Ls % 2 == 0) ? 2 : 1; }

// A row-staged launch needs: every bulk copy 16-byte aligned and a multiple
// of 16 bytes (Lrow*elem), the block within kRowMaxThreads, and both rings
// within the shared memory of one block.
inline bool row_plan(const Geom& g, size_t elem, RowPlan* p) {
    const int64_t Lrow = (int64_t)g.L * g.Ls;
    if ((Lrow * (int64_t)elem) % 16 != 0) return false;
    const int ppt = row_ppt(g, elem);
    const int64_t ncw = ((Lrow + ppt - 1) / ppt + 31) / 32;
    const int64_t nthreads = (ncw + 1) * 32;
    if (nthreads > kRowMaxThreads) return false;
    const int64_t smem =
        kRowBarBytes + (int64_t)(kRowSlots + 2 * kRowTEnt) * 4 * Lrow * (int64_t)elem;
    if (smem > kRowSmemMax) return false;
    p->Lrow = (int)Lrow;
    p->nrows = 2 * g.Lt * g.L;
    p->smem = (unsigned)smem;
    p->nthreads = (int)nthreads;
    p->ncw = (int)ncw;
    p->ppt = ppt;
    return true;
}

// ---- PTX helpers --------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// global -> shared bulk copy completing on bar (16-byte aligned, bytes % 16 == 0)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Wait for phase `parity` of bar to complete, for at most kRowWaitNs.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > kRowWaitNs) return false;
    }
}

// ---- block-wide deterministic sum for any block size (multiple of 32) -------
// Valid in thread 0; warps are added in order.
__device__ __forceinline__ double block_sum_any(double v, double* sh /* >= 32 */) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0) {
        const int nw = (int)(blockDim.x >> 5);
        for (int i = 0; i < nw; i++) r += sh[i];
    }
    __syncthreads();
    return r;
}

// Sum of n partials in a fixed order, the same value in every block and
// every thread (the row kernels' counterpart of sum_partials).
__device__ __forceinline__ double sum_partials_any(const double* part, int n) {
    __shared__ double sh[32];
    __shared__ double total;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += __ldcg(part + i);
    s = block_sum_any(s, sh);
    if (threadIdx.x == 0) total = s;
    __syncthreads();
    return total;
}

// The block's contiguous range of output rows.
__device__ __forceinline__ void row_range(int nrows, int* rho0, int* rho1) {
    const int64_t nb = gridDim.x, b = blockIdx.x;
    *rho0 = (int)(b * nrows / nb);
    *rho1 = (int)((b + 1) * nrows / nb);
}

// Storage -> arithmetic type of a staged element (FP16 storage computes in FP32).
template <class T, class S> struct RowCvt {
    __device__ __forceinline__ static T get(S v) { return v; }
};
template <> struct RowCvt<float2, __half2> {
    __device__ __forceinline__ static float2 get(__half2 v) { return __half22float2(v); }
};

// PPT adjacent staged elements from shared memory, converted to T.  For
// PPT = 2 the index is even, so the pair is one aligned 16-byte (FP32) or
// 8-byte (FP16) load.
template <class T, class S, int PPT> struct RowLd;
template <class T, class S> struct RowLd<T, S, 1> {
    __device__ __forceinline__ static void get(const S* p, int j, T* v) {
        v[0] = RowCvt<T, S>::get(p[j]);
    }
};
template <> struct RowLd<float2, float2, 2> {
    __device__ __forceinline__ static void get(const float2* p, int j, float2* v) {
        const float4 q = *reinterpret_cast<const float4*>(p + j);
        v[0] = make_float2(q.x, q.y);
        v[1] = make_float2(q.z, q.w);
    }
};
template <> struct RowLd<float2, __half2, 2> {
    __device__ __forceinline__ static void get(const __half2* p, int j, float2* v) {
        const uint2 q = *reinterpret_cast<const uint2*>(p + j);
        v[0] = __half22float2(*reinterpret_cast<const __half2*>(&q.x));
        v[1] = __half22float2(*reinterpret_cast<const __half2*>(&q.y));
    }
};

// Operands of the wall terms that are not in the staged rows: the other
// flavour's components on the other wall (same site, Dirac pair of the
// wall) for each of the thread's points that lies on a wall, and chi at the
// site.  Loaded one output row ahead (Body::pre).
template <class T, int PPT>
struct RowWall {
    T w[PPT][2];
    float c1, c2, c3;
};

template <bool DAG, int PPT, class T, class S>
__device__ __forceinline__ void row_wall_prefetch(RowWall<T, PPT>& rw, const S* __restrict__ gin,
                                                  const Geom& g, int f, int t, int y, int x,
                                                  int s, const float* __restrict__ chif) {
    const int Ls = g.Ls;
    const int site = x + g.L * (y + g.L * t);
    constexpr int WA = DAG ? 0 : 2;   // pair at s=Ls
    constexpr int WB = DAG ? 2 : 0;   // pair at s=1
    const int fo = 1 - f;
    bool any = false;
#pragma unroll
    for (int p = 0; p < PPT; p++) {
        const int sp = s + p;
        const bool atL = (sp == Ls - 1), at0 = (sp == 0);
        if (!(atL || at0)) continue;
        any = true;
        const int64_t other = (int64_t)Ls * site + (atL ? 0 : Ls - 1);
        const int d0 = atL ? WA : WB;
#pragma unroll
        for (int k = 0; k < 2; k++)
            rw.w[p][k] = RowCvt<T, S>::get(__ldg(gin + other + g.cs * (d0 + k + 4 * fo)));
    }
    if (any) {
        rw.c1 = __ldg(chif + site);
        rw.c2 = __ldg(chif + g.kvol + site);
        rw.c3 = __ldg(chif + 2 * g.kvol + site);
    }
}

// The four Dirac components of flavour f at PPT adjacent output points
// (s, s+1, ...) of a staged row, each point with the same operation sequence
// as dwf_apply_flavour (so the FP64 result is bit-identical to it and the
// FP32 result to the point-gather kernels').  c, yp, ym: shared rows y, y+1,
// y-1; tps, tms: shared rows t+1, t-1 (plane stride Lrow, storage type S);
// i = x*Ls + s; ixp, ixm: the x+-1 points of the row; site, it: the site
// and t of the row's points; rw: the wall operands (registers).
template <bool DAG, int IMASS, int PPT, class T, class S>
__device__ __forceinline__ void dwf_apply_rows(T acc[PPT][4], const S* c, const S* yp,
                                               const S* ym, const S* tps, const S* tms, int Lrow,
                                               int i, int ixp, int ixm, int s, int site, int it,
                                               const RowWall<T, PPT>& rw, const Geom& g, int f,
                                               typename real_of<T>::type diag,
                                               typename real_of<T>::type hpin, bool apbc) {
    typedef typename real_of<T>::type R;
    typedef RowCvt<T, S> C;
    constexpr int SF = DAG ? -1 : 1;
    const int Ls = g.Ls;
    T r[PPT][4];
    auto load = [&](const S* base, int j) {
#pragma unroll
        for (int d = 0; d < 4; d++) {
            T v[PPT];
            RowLd<T, S, PPT>::get(base, d * Lrow + j, v);
#pragma unroll
            for (int p = 0; p < PPT; p++) r[p][d] = v[p];
        }
    };
    // diagonal term (cheisdwf.f:2651-2667)
    load(c, i);
#pragma unroll
    for (int p = 0; p < PPT; p++)
#pragma unroll
        for (int d = 0; d < 4; d++) acc[p][d] = zscal(diag, r[p][d]);
    load(c, ixp);
#pragma unroll
    for (int p = 0; p < PPT; p++) hop<0, SF, false>(acc[p], r[p]);
    load(c, ixm);
#pragma unroll
    for (int p = 0; p < PPT; p++) hop<0, -SF, false>(acc[p], r[p]);
    load(yp, i);
#pragma unroll
    for (int p = 0; p < PPT; p++) hop<1, SF, false>(acc[p], r[p]);
    load(ym, i);
#pragma unroll
    for (int p = 0; p < PPT; p++) hop<1, -SF, false>(acc[p], r[p]);
    load(tps, i);
#pragma unroll
    for (int p = 0; p < PPT; p++) hop<2, SF, false>(acc[p], r[p]);
    load(tms, i);
#pragma unroll
    for (int p = 0; p < PPT; p++) hop<2, -SF, false>(acc[p], r[p]);
    // kappa = 1/2 (:2815-2829)
#pragma unroll
    for (int p = 0; p < PPT; p++)
#pragma unroll
        for (int d = 0; d < 4; d++) acc[p][d] = zscal((R)0.5, acc[p][d]);
    // antiperiodic boundary in t (:2831-2876): reverse the wrapped hop
    if (apbc && it == g.Lt - 1) {
        load(tps, i);
#pragma unroll
        for (int p = 0; p < PPT; p++) hop<2, SF, true>(acc[p], r[p]);
    }
    if (apbc && it == 0) {
        load(tms, i);
#pragma unroll
        for (int p = 0; p < PPT; p++) hop<2, -SF, true>(acc[p], r[p]);
    }
    // s hops with chiral projection (:2879-2908; M^dagger :3313-3342)
    constexpr int UP = DAG ? 0 : 2;
    constexpr int DN = DAG ? 2 : 0;
#pragma unroll
    for (int p = 0; p < PPT; p++) {
        const int sp = s + p, ip = i + p;
        if (sp < Ls - 1) {
#pragma unroll
            for (int d = UP; d < UP + 2; d++)
                acc[p][d] = zsub(acc[p][d], C::get(c[d * Lrow + ip + 1]));
        }
        if (sp > 0) {
#pragma unroll
            for (int d = DN; d < DN + 2; d++)
                acc[p][d] = zsub(acc[p][d], C::get(c[d * Lrow + ip - 1]));
        }
    }
    // wall coupling: this flavour's components on the other wall come from
    // the staged row (same site), the other flavour's and chi from rw
    constexpr int WA = DAG ? 0 : 2;
    constexpr int WB = DAG ? 2 : 0;
    const bool pin = (site == 0);
#pragma unroll
    for (int p = 0; p < PPT; p++) {
        const int sp = s + p, ip = i + p;
        const bool atL = (sp == Ls - 1), at0 = (sp == 0);
        if (!(atL || at0)) continue;
        const int io = ip - sp + (atL ? 0 : Ls - 1);   // the other wall's point in the row
        if (atL) {
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const T own = C::get(c[(WA + k) * Lrow + io]);
                wall_elem<DAG, IMASS, 0>(acc[p][WA + k], f == 0 ? own : rw.w[p][k],
                                         f == 0 ? rw.w[p][k] : own, f, rw.c1, rw.c2, rw.c3, pin,
                                         hpin);
            }
        } else {
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const T own = C::get(c[(WB + k) * Lrow + io]);
                wall_elem<DAG, IMASS, 1>(acc[p][WB + k], f == 0 ? own : rw.w[p][k],
                                         f == 0 ? rw.w[p][k] : own, f, rw.c1, rw.c2, rw.c3, pin,
                                         hpin);
            }
        }
    }
}

// ---- the producer: lane 0 of the block's last warp -----------------------------
// Issues the window loads and t entries in the order the consumers need
// them, each after its slot's previous use has been released, then waits
// (bounded) for the copies it has in flight.  The consumers' reads of a slot
// are ordered before its refill by the empty barrier alone (their arrive
// releases, the producer's wait acquires); no proxy fence is taken between
// copies, since one waits for the copies already in flight and would leave
// a single copy in flight at a time.
template <class T>
__device__ __forceinline__ void row_produce(const Geom& g, const RowPlan& rp, uint64_t* bar,
                                            T* slots, const T* src, int rho0, int rho1,
                                            volatile int* err) {
    const int L = g.L, Lt = g.Lt, Lrow = rp.Lrow;
    const int64_t cs = g.cs;
    const uint32_t bytes = (uint32_t)(Lrow * sizeof(T));
    T* tslots = slots + (int64_t)kRowSlots * 4 * Lrow;
    const int nk = rho1 - rho0;
    // window-load cursor: start of the current run, its length, offset in it
    int ra = rho0, o = 0;
    int len = min((ra / L + 1) * L, rho1) - ra;
    int issued = 0, t_issued = 0;
    // the output row of step k and the base u of its window loads
    const int run0 = rho0 / L;
    int f = run0 / Lt, t = run0 - f * Lt, y = rho0 - run0 * L;
    int u = 0;
    bool ok = true;
    for (int k = 0; k < nk && ok; k++) {
        if (k > 0) {
            u += 1;
            if (++y == L) {
                y = 0;
                u += 2;
                if (++t == Lt) {
                    t = 0;
                    ++f;
                }
            }
        }
        while (issued <= u + 2) {
            const int e = issued % kRowSlots;
            if (*err || (issued >= kRowSlots &&
                         !mbar_wait_bounded(bar + kRowEmptyY + e,
                                            (uint32_t)((issued / kRowSlots - 1) & 1)))) {
                ok = false;
                break;
            }
            const int wr = ra / L, wf = wr / Lt, wt = wr - wf * Lt;
            int wy = ra - wr * L - 1 + o;
            wy = wy < 0 ? wy + L : (wy >= L ? wy - L : wy);
            mbar_arrive_expect_tx(bar + e, 4 * bytes);
            T* dst = slots + (int64_t)e * 4 * Lrow;
            const int64_t off = (int64_t)Lrow * (wy + (int64_t)L * wt);
#pragma unroll
            for (int d = 0; d < 4; d++)
                bulk_g2s(dst + (int64_t)d * Lrow, src + cs * (4 * wf + d) + off, bytes, bar + e);
            issued++;
            if (++o == len + 2) {
                ra += len;
                o = 0;
                if (ra < rho1) len = min((ra / L + 1) * L, rho1) - ra;
            }
        }
        if (!ok) break;
        const int e = k % kRowTEnt;
        if (*err || (k >= kRowTEnt &&
                     !mbar_wait_bounded(bar + kRowEmptyT + e, (uint32_t)((k / kRowTEnt - 1) & 1)))) {
            ok = false;
            break;
        }
        const int tp = t + 1 == Lt ? 0 : t + 1, tm = t == 0 ? Lt - 1 : t - 1;
        mbar_arrive_expect_tx(bar + kRowFullT + e, 8 * bytes);
        T* dst = tslots + (int64_t)e * 8 * Lrow;
        const int64_t op = (int64_t)Lrow * (y + (int64_t)L * tp);
        const int64_t om = (int64_t)Lrow * (y + (int64_t)L * tm);
#pragma unroll
        for (int d = 0; d < 4; d++) {
            bulk_g2s(dst + (int64_t)d * Lrow, src + cs * (4 * f + d) + op, bytes, bar + kRowFullT + e);
            bulk_g2s(dst + (int64_t)(4 + d) * Lrow, src + cs * (4 * f + d) + om, bytes,
                     bar + kRowFullT + e);
        }
        t_issued++;
    }
    if (!ok) *err = 1;
    // the last use of every slot: its copies must land before the block ends
    for (int w = issued > kRowSlots ? issued - kRowSlots : 0; w < issued; w++)
        mbar_wait_bounded(bar + w % kRowSlots, (uint32_t)((w / kRowSlots) & 1));
    for (int e = t_issued > kRowTEnt ? t_issued - kRowTEnt : 0; e < t_issued; e++)
        mbar_wait_bounded(bar + kRowFullT + e % kRowTEnt, (uint32_t)((e / kRowTEnt) & 1));
}

// The loop over a block's rows.  Body::pre(f, t, y, x, s) issues the global
// loads a thread's points need besides the staged rows (wall operands,
// streamed vectors); it runs for the first row before the first wait and
// for row k+1 right after row k is computed, so those loads are in flight
// while the warp waits.  Body::compute(c, yp, ym, tp, tm, f, t, y, x, s, i,
// ixp, ixm) evaluates the thread's PPT points from the staged rows y, y+1,
// y-1 and t+1, t-1.  T is the storage type of the staged field src.  Called
// by every thread of the block; returns false if a copy timed out.
template <class T, int PPT, class Body>
__device__ __forceinline__ bool row_sweep(const Geom& g, const RowPlan& rp, unsigned char* sm,
                                          const T* src, Body& body) {
    __shared__ int s_err;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm);
    T* slots = reinterpret_cast<T*>(sm + kRowBarBytes);
    int rho0, rho1;
    row_range(rp.nrows, &rho0, &rho1);
    const int warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);
    if (threadIdx.x == 0) {
        s_err = 0;
        for (int k = 0; k < kRowSlots + kRowTEnt; k++) {
            mbar_init(bar + k, 1);
            mbar_init(bar + kRowEmptyY + k, (uint32_t)rp.ncw);
        }
        fence_mbar_init();
    }
    __syncthreads();
    volatile int* err = &s_err;
    const int nk = rho1 - rho0;
    if (nk > 0 && warp == rp.ncw) {
        if (lane == 0) row_produce<T>(g, rp, bar, slots, src, rho0, rho1, err);
    } else if (nk > 0) {
        const int Lrow = rp.Lrow, Ls = g.Ls, L = g.L, Lt = g.Lt;
        const T* tslots = slots + (int64_t)kRowSlots * 4 * Lrow;
        const int i = (int)threadIdx.x * PPT;
        const bool active = i < Lrow;
        const int x = active ? i / Ls : 0;
        const int s = active ? i - x * Ls : 0;
        const int ixp = (x + 1 == L ? 0 : x + 1) * Ls + s;
        const int ixm = (x == 0 ? L - 1 : x - 1) * Ls + s;
        const int run0 = rho0 / L;
        int f = run0 / Lt, t = run0 - f * Lt, y = rho0 - run0 * L;
        int u = 0;
        if (active) body.pre(f, t, y, x, s);
        for (int k = 0; k < nk; k++) {
            if (k > 0) {
                u += 1;
                if (++y == L) {
                    y = 0;
                    u += 2;
                    if (++t == Lt) {
                        t = 0;
                        ++f;
                    }
                }
            }
            if (__any_sync(0xffffffffu, *err != 0)) break;
            bool got = true;
#pragma unroll
            for (int w = 0; w < 3; w++)
                got &= mbar_wait_bounded(bar + (u + w) % kRowSlots,
                                         (uint32_t)(((u + w) / kRowSlots) & 1));
            got &= mbar_wait_bounded(bar + kRowFullT + k % kRowTEnt,
                                     (uint32_t)((k / kRowTEnt) & 1));
            if (!__all_sync(0xffffffffu, got)) {
                *err = 1;
                break;
            }
            // the next output row
            int fn = f, tn = t, yn = y + 1;
            const bool newrun = yn == L;
            if (newrun) {
                yn = 0;
                if (++tn == Lt) {
                    tn = 0;
                    ++fn;
                }
            }
            const bool more = k + 1 < nk;
            if (active) {
                const T* tr = tslots + (int64_t)(k % kRowTEnt) * 8 * Lrow;
                body.compute(slots + (int64_t)((u + 1) % kRowSlots) * 4 * Lrow,
                             slots + (int64_t)((u + 2) % kRowSlots) * 4 * Lrow,
                             slots + (int64_t)(u % kRowSlots) * 4 * Lrow, tr, tr + 4 * Lrow, f, t,
                             y, x, s, i, ixp, ixm);
                if (more) body.pre(fn, tn, yn, x, s);
            }
            __syncwarp();
            if (lane == 0) {
                // window loads the next row does not read, and this row's t entry
                if (more) {
                    const int nrel = newrun ? 3 : 1;
                    for (int w = u; w < u + nrel; w++) mbar_arrive(bar + kRowEmptyY + w % kRowSlots);
                }
                mbar_arrive(bar + kRowEmptyT + k % kRowTEnt);
            }
        }
    }
    __syncthreads();
    return s_err == 0;
}

}  // namespace chdwf
