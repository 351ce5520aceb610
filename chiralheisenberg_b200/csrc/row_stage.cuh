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
// and chi), issued one output row ahead.
//
// Rows reach shared memory by 1-D bulk copies (cp.async.bulk, the TMA
// engine's untiled form, this GPU's own memory only, no multicast) into two
// rings with one mbarrier per entry:
//   * the window ring of kRowSlots rows along y.  The window rows of a block
//     are loaded in order: for each maximal run of output rows with the same
//     (f, t), rows y_a-1, y_a, ..., y_b (mod L), i.e. run length + 2 loads.
//     Output row k of a run needs loads u, u+1, u+2 (u = run base + k);
//     after it the slot of load u is free and load u + kRowSlots is issued
//     into it, so up to kRowSlots - 3 rows are in flight ahead of the
//     computation.  Load w is the (w / kRowSlots)-th use of slot
//     w % kRowSlots, so its wait parity is (w / kRowSlots) & 1;
//   * the t ring of kRowTEnt entries, entry k holding rows (t+1, y) and
//     (t-1, y) of the block's k-th output row; after output row k, entry
//     k + kRowTEnt is issued into its slot (parity (k / kRowTEnt) & 1).
//
// Every wait is bounded (kRowWaitNs); a block whose copy does not arrive in
// time records an error and leaves the loop with the others at the next
// block barrier, after waiting (bounded again) for its copies in flight.
#pragma once
#include <cuda_fp16.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "dwf_stencil.cuh"

namespace chdwf {

constexpr int kRowSlots = 5;                      // window ring (rows along y)
constexpr int kRowTEnt = 3;                       // t ring entries (two rows each)
constexpr uint64_t kRowWaitNs = 1000000000ull;   // 1 s per wait
constexpr unsigned kRowBarBytes = 128;            // mbarriers at the front of shared memory
constexpr unsigned kRowSmemMax = 227 * 1024;

// Block size limit (one thread per point of a row) and the register budget
// that lets one such block of the largest size run on an SM: a block's warps
// are spread over the SM's four sub-partitions, each with a quarter of the
// register file (16384), so ceil(warps / 4) * 32 * registers <= 16384.
template <class T> struct RowMaxThreads;
template <> struct RowMaxThreads<double2> { static constexpr int value = 512; };
template <> struct RowMaxThreads<float2> { static constexpr int value = 768; };
template <class T> struct RowRegs;
template <> struct RowRegs<double2> { static constexpr int value = 112; };
template <> struct RowRegs<float2> { static constexpr int value = 80; };
static_assert((RowMaxThreads<double2>::value / 32 + 3) / 4 * 32 * RowRegs<double2>::value <= 16384,
              "FP64 row block does not fit a sub-partition's registers");
static_assert((RowMaxThreads<float2>::value / 32 + 3) / 4 * 32 * RowRegs<float2>::value <= 16384,
              "FP32 row block does not fit a sub-partition's registers");

// Which stencil kernels run, from the environment variable CHDWF_STENCIL:
// 0 (unset): the autotuner's choice per lattice and precision (tune.cu);
// 1 ("legacy"): the point-gather kernels only; 2 ("rows"): row kernels
// wherever they fit (tests use it to run them on small lattices).
inline int stencil_mode() {
    const char* v = getenv("CHDWF_STENCIL");
    if (!v) return 0;
    if (strcmp(v, "legacy") == 0) return 1;
    if (strcmp(v, "rows") == 0) return 2;
    return 0;
}

// Launch plan of a row-staged kernel (host-computed, passed by value).
struct RowPlan {
    int Lrow;        // L*Ls points (elements per plane row)
    int nrows;       // 2*Lt*L output rows (flavour, t, y)
    unsigned smem;   // dynamic shared memory bytes
    int nthreads;    // block size: Lrow rounded up to a warp
};

// A row-staged launch needs: every bulk copy 16-byte aligned and a multiple
// of 16 bytes (Lrow*elem), one thread per point of a row, and the ring of
// slots within the shared memory of one block.
inline bool row_plan(const Geom& g, size_t elem, int max_threads, RowPlan* p) {
    const int64_t Lrow = (int64_t)g.L * g.Ls;
    if ((Lrow * (int64_t)elem) % 16 != 0) return false;
    const int64_t nthreads = (Lrow + 31) / 32 * 32;
    if (nthreads > max_threads) return false;
    const int64_t smem =
        kRowBarBytes + (int64_t)(kRowSlots + 2 * kRowTEnt) * 4 * Lrow * (int64_t)elem;
    if (smem > kRowSmemMax) return false;
    p->Lrow = (int)Lrow;
    p->nrows = 2 * g.Lt * g.L;
    p->smem = (unsigned)smem;
    p->nthreads = (int)nthreads;
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
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
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

// ---- the rings of staged rows -------------------------------------------------
template <class T>
struct RowRing {
    uint64_t* bar;      // kRowSlots window mbarriers, then kRowTEnt t-ring mbarriers
    T* slots;           // kRowSlots x 4 planes x Lrow
    T* tslots;          // kRowTEnt x 8 planes x Lrow (t+1 rows, then t-1 rows)
    int Lrow, L, Lt;
    int64_t cs;         // plane stride (elements)
    // producer cursor (thread 0): run start, run length, offset in the run
    int p_rho_a, p_len, p_o;
    int rho0, rho1;
    int issued;         // window loads issued so far
    int t_issued;       // t-ring entries issued so far

    __device__ __forceinline__ T* slot(int w) const {
        return slots + (int64_t)(w % kRowSlots) * 4 * Lrow;
    }
    __device__ __forceinline__ T* tslot(int k) const {
        return tslots + (int64_t)(k % kRowTEnt) * 8 * Lrow;
    }
    __device__ __forceinline__ int run_len_from(int rho_a) const {
        const int end = (rho_a / L + 1) * L;
        return (end < rho1 ? end : rho1) - rho_a;
    }
    // thread 0: issue the next window-row load of the block's sequence
    __device__ __forceinline__ void issue_next(const T* src) {
        const int run = p_rho_a / L;
        const int f = run / Lt, t = run - f * Lt;
        const int ya = p_rho_a - run * L;
        int y = ya - 1 + p_o;
        y = y < 0 ? y + L : (y >= L ? y - L : y);
        const int w = issued;
        uint64_t* b = bar + (w % kRowSlots);
        const uint32_t bytes = (uint32_t)(Lrow * sizeof(T));
        mbar_arrive_expect_tx(b, 4 * bytes);
        T* dst = slot(w);
        const int64_t row_off = (int64_t)Lrow * (y + (int64_t)L * t);
#pragma unroll
        for (int d = 0; d < 4; d++)
            bulk_g2s(dst + (int64_t)d * Lrow, src + cs * (4 * f + d) + row_off, bytes, b);
        issued++;
        if (++p_o == p_len + 2) {
            p_rho_a += p_len;
            p_o = 0;
            if (p_rho_a < rho1) p_len = run_len_from(p_rho_a);
        }
    }
    __device__ __forceinline__ bool more() const { return p_rho_a < rho1; }
    // thread 0: issue t-ring entry t_issued, rows (t+1, y), (t-1, y) of the
    // block's output row rho0 + t_issued
    __device__ __forceinline__ void issue_t(const T* src) {
        const int k = t_issued;
        const int rho = rho0 + k;
        const int run = rho / L;
        const int f = run / Lt, t = run - f * Lt, y = rho - run * L;
        const int tp = t + 1 == Lt ? 0 : t + 1, tm = t == 0 ? Lt - 1 : t - 1;
        uint64_t* b = bar + kRowSlots + (k % kRowTEnt);
        const uint32_t bytes = (uint32_t)(Lrow * sizeof(T));
        mbar_arrive_expect_tx(b, 8 * bytes);
        T* dst = tslot(k);
        const int64_t op = (int64_t)Lrow * (y + (int64_t)L * tp);
        const int64_t om = (int64_t)Lrow * (y + (int64_t)L * tm);
#pragma unroll
        for (int d = 0; d < 4; d++) {
            bulk_g2s(dst + (int64_t)d * Lrow, src + cs * (4 * f + d) + op, bytes, b);
            bulk_g2s(dst + (int64_t)(4 + d) * Lrow, src + cs * (4 * f + d) + om, bytes, b);
        }
        t_issued++;
    }
};

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

// Operands of the wall terms that are not in the staged rows: the other
// flavour's components on the other wall (same site, Dirac pair of the
// wall) and chi at the site.  Loaded in Body::pre with the t neighbours, so
// their latency overlaps the wait for the staged rows.
template <class T>
struct RowWall {
    T w[2];
    float c1, c2, c3;
};

template <bool DAG, class T, class S>
__device__ __forceinline__ void row_wall_prefetch(RowWall<T>& rw, const S* __restrict__ gin,
                                                  const Geom& g, int f, int t, int y, int x,
                                                  int s, const float* __restrict__ chif) {
    const int Ls = g.Ls;
    const bool atL = (s == Ls - 1), at0 = (s == 0);
    if (!(atL || at0)) return;
    const int site = x + g.L * (y + g.L * t);
    const int64_t other = (int64_t)Ls * site + (atL ? 0 : Ls - 1);
    constexpr int WA = DAG ? 0 : 2;   // pair at s=Ls
    constexpr int WB = DAG ? 2 : 0;   // pair at s=1
    const int d0 = atL ? WA : WB;
    const int fo = 1 - f;
#pragma unroll
    for (int k = 0; k < 2; k++) rw.w[k] = RowCvt<T, S>::get(__ldg(gin + other + g.cs * (d0 + k + 4 * fo)));
    rw.c1 = __ldg(chif + site);
    rw.c2 = __ldg(chif + g.kvol + site);
    rw.c3 = __ldg(chif + 2 * g.kvol + site);
}

// The four Dirac components of flavour f at one output point of a staged
// row, with the same operation sequence as dwf_apply_flavour (so the FP64
// result is bit-identical to it).  c, yp, ym: shared rows y, y+1, y-1; tps,
// tms: shared rows t+1, t-1 (plane stride Lrow, storage type S); i = x*Ls + s;
// ixp, ixm: the x+-1 points of the row; rw: the wall operands (registers).
template <bool DAG, int IMASS, class T, class S>
__device__ __forceinline__ void dwf_apply_rows(T acc[4], const S* c, const S* yp, const S* ym,
                                               const S* tps, const S* tms, int Lrow, int i,
                                               int ixp, int ixm, const RowWall<T>& rw,
                                               const Geom& g, const PointIdx& q, int f,
                                               typename real_of<T>::type diag,
                                               typename real_of<T>::type hpin, bool apbc) {
    typedef typename real_of<T>::type R;
    typedef RowCvt<T, S> C;
    constexpr int SF = DAG ? -1 : 1;
    const int Ls = g.Ls;
    // diagonal term (cheisdwf.f:2651-2667)
#pragma unroll
    for (int d = 0; d < 4; d++) acc[d] = zscal(diag, C::get(c[d * Lrow + i]));
    T r[4];
#pragma unroll
    for (int d = 0; d < 4; d++) r[d] = C::get(c[d * Lrow + ixp]);
    hop<0, SF, false>(acc, r);
#pragma unroll
    for (int d = 0; d < 4; d++) r[d] = C::get(c[d * Lrow + ixm]);
    hop<0, -SF, false>(acc, r);
#pragma unroll
    for (int d = 0; d < 4; d++) r[d] = C::get(yp[d * Lrow + i]);
    hop<1, SF, false>(acc, r);
#pragma unroll
    for (int d = 0; d < 4; d++) r[d] = C::get(ym[d * Lrow + i]);
    hop<1, -SF, false>(acc, r);
#pragma unroll
    for (int d = 0; d < 4; d++) r[d] = C::get(tps[d * Lrow + i]);
    hop<2, SF, false>(acc, r);
#pragma unroll
    for (int d = 0; d < 4; d++) r[d] = C::get(tms[d * Lrow + i]);
    hop<2, -SF, false>(acc, r);
    // kappa = 1/2 (:2815-2829)
#pragma unroll
    for (int d = 0; d < 4; d++) acc[d] = zscal((R)0.5, acc[d]);
    // antiperiodic boundary in t (:2831-2876): reverse the wrapped hop
    if (apbc && q.it == g.Lt - 1) {
#pragma unroll
        for (int d = 0; d < 4; d++) r[d] = C::get(tps[d * Lrow + i]);
        hop<2, SF, true>(acc, r);
    }
    if (apbc && q.it == 0) {
#pragma unroll
        for (int d = 0; d < 4; d++) r[d] = C::get(tms[d * Lrow + i]);
        hop<2, -SF, true>(acc, r);
    }
    // s hops with chiral projection (:2879-2908; M^dagger :3313-3342)
    constexpr int UP = DAG ? 0 : 2;
    constexpr int DN = DAG ? 2 : 0;
    if (q.s < Ls - 1) {
#pragma unroll
        for (int d = UP; d < UP + 2; d++) acc[d] = zsub(acc[d], C::get(c[d * Lrow + i + 1]));
    }
    if (q.s > 0) {
#pragma unroll
        for (int d = DN; d < DN + 2; d++) acc[d] = zsub(acc[d], C::get(c[d * Lrow + i - 1]));
    }
    // wall coupling: this flavour's components on the other wall come from
    // the staged row (same site), the other flavour's and chi from rw
    constexpr int WA = DAG ? 0 : 2;
    constexpr int WB = DAG ? 2 : 0;
    const bool atL = (q.s == Ls - 1), at0 = (q.s == 0);
    if (!(atL || at0)) return;
    const bool pin = (q.site == 0);
    const int io = i - q.s + (atL ? 0 : Ls - 1);      // the other wall's point in the row
    if (atL) {
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const T own = C::get(c[(WA + k) * Lrow + io]);
            wall_elem<DAG, IMASS, 0>(acc[WA + k], f == 0 ? own : rw.w[k], f == 0 ? rw.w[k] : own,
                                     f, rw.c1, rw.c2, rw.c3, pin, hpin);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const T own = C::get(c[(WB + k) * Lrow + io]);
            wall_elem<DAG, IMASS, 1>(acc[WB + k], f == 0 ? own : rw.w[k], f == 0 ? rw.w[k] : own,
                                     f, rw.c1, rw.c2, rw.c3, pin, hpin);
        }
    }
}

__device__ __forceinline__ PointIdx row_point(const Geom& g, int t, int y, int x, int s) {
    PointIdx q;
    q.s = s;
    q.ix = x;
    q.iy = y;
    q.it = t;
    q.site = x + g.L * (y + g.L * t);
    q.p = s + (int64_t)g.Ls * q.site;
    return q;
}

// The loop over a block's rows.  Body::pre(f, t, y, x, s) issues the global
// loads a point needs besides the staged rows (wall operands, streamed
// vectors); it runs for the first row before the first wait and for row k+1
// right after row k is computed, so those loads are in flight while the
// block synchronises and waits.  Body::compute(c, yp, ym, tp, tm, f, t, y,
// x, s, i, ixp, ixm) evaluates the point from the staged rows y, y+1, y-1
// and t+1, t-1.  T is the storage type of the staged field src.  Returns
// false if a copy timed out.
template <class T, class Body>
__device__ __forceinline__ bool row_sweep(const Geom& g, const RowPlan& rp, unsigned char* sm,
                                          const T* src, Body& body) {
    __shared__ int s_err;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm);
    T* slots = reinterpret_cast<T*>(sm + kRowBarBytes);
    int rho0, rho1;
    row_range(rp.nrows, &rho0, &rho1);
    RowRing<T> rr;
    rr.bar = bar;
    rr.slots = slots;
    rr.tslots = slots + (int64_t)kRowSlots * 4 * rp.Lrow;
    rr.Lrow = rp.Lrow;
    rr.L = g.L;
    rr.Lt = g.Lt;
    rr.cs = g.cs;
    rr.rho0 = rho0;
    rr.rho1 = rho1;
    rr.issued = 0;
    rr.t_issued = 0;
    rr.p_rho_a = rho0;
    rr.p_o = 0;
    rr.p_len = rho0 < rho1 ? rr.run_len_from(rho0) : 0;
    if (threadIdx.x == 0) {
        s_err = 0;
        for (int k = 0; k < kRowSlots + kRowTEnt; k++) mbar_init(bar + k, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (rho0 >= rho1) return true;
    const int nk = rho1 - rho0;
    if (threadIdx.x == 0) {
        // the first output row's copies first, then the ones ahead
        while (rr.issued < 3 && rr.more()) rr.issue_next(src);
        rr.issue_t(src);
        while (rr.issued < kRowSlots && rr.more()) rr.issue_next(src);
        while (rr.t_issued < kRowTEnt && rr.t_issued < nk) rr.issue_t(src);
    }
    const int i = threadIdx.x;
    const bool active = i < rp.Lrow;
    const int Ls = g.Ls, L = g.L;
    const int x = active ? i / Ls : 0;
    const int s = active ? i - x * Ls : 0;
    const int ixp = (x + 1 == L ? 0 : x + 1) * Ls + s;
    const int ixm = (x == 0 ? L - 1 : x - 1) * Ls + s;
    int u = 0;
    int run_prev = rho0 / L;
    bool ok = true;
    int k = 0;
    if (active) {
        const int run = rho0 / L, f = run / g.Lt;
        body.pre(f, run - f * g.Lt, rho0 - run * L, x, s);
    }
    for (int rho = rho0; rho < rho1; rho++, k++) {
        const int run = rho / L;
        if (run != run_prev) {
            u += 2;
            run_prev = run;
        }
        const int f = run / g.Lt, t = run - f * g.Lt, y = rho - run * L;
        bool got = true;
#pragma unroll
        for (int w = 0; w < 3; w++)
            got &= mbar_wait_bounded(bar + (u + w) % kRowSlots, (uint32_t)(((u + w) / kRowSlots) & 1));
        got &= mbar_wait_bounded(bar + kRowSlots + k % kRowTEnt, (uint32_t)((k / kRowTEnt) & 1));
        if (!got) s_err = 1;
        __syncthreads();
        if (s_err) {
            ok = false;
            break;
        }
        if (active) {
            const T* tr = rr.tslot(k);
            body.compute(rr.slot(u + 1), rr.slot(u + 2), rr.slot(u), tr, tr + 4 * rp.Lrow, f, t,
                         y, x, s, i, ixp, ixm);
            if (rho + 1 < rho1) {
                const int rn = (rho + 1) / L, fn = rn / g.Lt;
                body.pre(fn, rn - fn * g.Lt, rho + 1 - rn * L, x, s);
            }
        }
        __syncthreads();   // every thread is done with window load u and t entry k
        u += 1;
        const int next_u = (rho + 1 < rho1 && (rho + 1) / L != run) ? u + 2 : u;
        if (threadIdx.x == 0) {
            fence_proxy_async_smem();
            while (rr.more() && rr.issued < next_u + kRowSlots) rr.issue_next(src);
            while (rr.t_issued < nk && rr.t_issued < k + 1 + kRowTEnt) rr.issue_t(src);
        }
    }
    if (!ok && threadIdx.x == 0) {
        // wait (bounded) for the copies still in flight before the block's
        // shared memory goes away
        for (int w = u; w < rr.issued; w++)
            mbar_wait_bounded(bar + w % kRowSlots, (uint32_t)((w / kRowSlots) & 1));
        for (int e = k; e < rr.t_issued; e++)
            mbar_wait_bounded(bar + kRowSlots + e % kRowTEnt, (uint32_t)((e / kRowTEnt) & 1));
    }
    __syncthreads();
    return ok;
}

}  // namespace chdwf
