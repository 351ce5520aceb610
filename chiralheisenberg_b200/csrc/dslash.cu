// dslash.cu -- FP64 domain-wall operator kernels (rhmc/cheisdwf.f:2634-3501)
// and the chi-force contraction derivs (rhmc/cheisdwf.f:747-849).
#include <cuda_fp16.h>

#include <cstdlib>
#include <cstring>

#include "dwf_stencil.cuh"
#include "internal.h"
#include "row_stage.cuh"

namespace chdwf {

struct LdF64 {
    const double2* __restrict__ p;
    __device__ __forceinline__ double2 operator()(int64_t j) const { return __ldg(p + j); }
};

// Flavour-split: two threads per point (split_point / split_flavour); OCC
// blocks a SM (the register budget).
template <bool DAG, int IMASS, int OCC>
__global__ void __launch_bounds__(kSplitThreads, OCC)
    k_dslash64(double2* __restrict__ out, const double2* __restrict__ in,
               const float* __restrict__ chif, Geom g, double diag, double hpin, int apbc) {
    const int64_t p = split_point();
    const int f = split_flavour();
    if (p >= g.npts) return;
    const PointIdx q = point_of(g, p);
    double2 acc[4];
    dwf_apply_flavour<DAG, IMASS>(acc, LdF64{in}, g, q, f, chif, diag, hpin, apbc != 0);
#pragma unroll
    for (int d = 0; d < 4; d++) out[p + g.cs * (d + 4 * f)] = acc[d];
}

static inline float diag_of(float am3) { return 2.0f * ((3.0f - am3) + 1.0f); }  // :2652

// ---- the operator on staged rows (row_stage.cuh) ------------------------------
// S: storage type (double2, float2 or __half2), T: arithmetic type.  Per
// element the operation sequence of k_dslash64 / k_dslash_lp.  A block
// whose staged copy does not arrive within the bounded wait writes NaN over
// its rows, so the failure reaches the caller's data.
template <class T> __device__ __forceinline__ T row_store(T v, T*) { return v; }
__device__ __forceinline__ __half2 row_store(float2 v, __half2*) { return __float22half2_rn(v); }

// Stores PPT adjacent output elements (one 16-byte or 8-byte store for a pair).
template <class S, class T, int PPT> struct RowSt;
template <class S, class T> struct RowSt<S, T, 1> {
    __device__ __forceinline__ static void put(S* o, const T* v) { *o = row_store(v[0], o); }
};
template <> struct RowSt<float2, float2, 2> {
    __device__ __forceinline__ static void put(float2* o, const float2* v) {
        *reinterpret_cast<float4*>(o) = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
    }
};
template <> struct RowSt<__half2, float2, 2> {
    __device__ __forceinline__ static void put(__half2* o, const float2* v) {
        const __half2 a = __float22half2_rn(v[0]), b = __float22half2_rn(v[1]);
        uint2 q;
        q.x = *reinterpret_cast<const uint32_t*>(&a);
        q.y = *reinterpret_cast<const uint32_t*>(&b);
        *reinterpret_cast<uint2*>(o) = q;
    }
};

template <class S, class T, bool DAG, int IMASS, int PPT>
struct OpRows {
    typedef typename real_of<T>::type Real;
    const S* __restrict__ in;
    S* __restrict__ out;
    const float* __restrict__ chif;
    const Geom& g;
    int Lrow;
    Real diag, hpin;
    int apbc;
    RowWall<T, PPT> rw;
    __device__ __forceinline__ void pre(int f, int t, int y, int x, int s) {
        row_wall_prefetch<DAG, PPT>(rw, in, g, f, t, y, x, s, chif);
    }
    __device__ __forceinline__ void compute(const S* c, const S* yp, const S* ym, const S* tps,
                                            const S* tms, int f, int t, int y, int x, int s,
                                            int i, int ixp, int ixm) {
        const int site = x + g.L * (y + g.L * t);
        T acc[PPT][4];
        dwf_apply_rows<DAG, IMASS, PPT>(acc, c, yp, ym, tps, tms, Lrow, i, ixp, ixm, s, site, t,
                                        rw, g, f, diag, hpin, apbc != 0);
        const int64_t p0 = s + (int64_t)g.Ls * site;
#pragma unroll
        for (int d = 0; d < 4; d++) {
            T v[PPT];
#pragma unroll
            for (int p = 0; p < PPT; p++) v[p] = acc[p][d];
            RowSt<S, T, PPT>::put(out + p0 + g.cs * (d + 4 * f), v);
        }
    }
};

template <class S, class T, bool DAG, int IMASS, int PPT>
__global__ void __maxnreg__(kRowRegs)
    k_dslash_rows(S* __restrict__ out, const S* __restrict__ in, const float* __restrict__ chif,
                  Geom g, RowPlan rp, typename real_of<T>::type diag,
                  typename real_of<T>::type hpin, int apbc) {
    extern __shared__ __align__(128) unsigned char row_smem[];
    OpRows<S, T, DAG, IMASS, PPT> body{in, out, chif, g, rp.Lrow, diag, hpin, apbc};
    if (row_sweep<S, PPT>(g, rp, row_smem, in, body)) return;
    int rho0, rho1;
    row_range(rp.nrows, &rho0, &rho1);
    const T nan = zmake<T>((typename real_of<T>::type)NAN, (typename real_of<T>::type)NAN);
    for (int rho = rho0; rho < rho1; rho++) {
        const int run = rho / g.L, f = run / g.Lt, t = run - f * g.Lt, y = rho - run * g.L;
        for (int i = threadIdx.x; i < rp.Lrow; i += blockDim.x)
            for (int d = 0; d < 4; d++)
                out[i + (int64_t)rp.Lrow * (y + (int64_t)g.L * t) + g.cs * (d + 4 * f)] =
                    row_store(nan, out);
    }
}

// Plan and grid of the row-staged operator, set up once per kernel and row
// shape: the blocks that fit on all SMs at once, at most one per row.
template <class S, class T, bool DAG, int IMASS, int PPT>
static bool op_rows_setup(const Geom& g, const RowPlan& rp, unsigned* nb) {
    static int cached_lrow = -1, cached_nrows = -1;
    static unsigned cached_nb = 0;
    if (cached_lrow == rp.Lrow && cached_nrows == rp.nrows) {
        *nb = cached_nb;
        return cached_nb > 0;
    }
    const void* k = (const void*)k_dslash_rows<S, T, DAG, IMASS, PPT>;
    int dev = 0, nsm = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    unsigned n = 0;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rp.smem) ==
            cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, rp.nthreads, rp.smem) ==
            cudaSuccess &&
        per_sm >= 1) {
        int64_t m = (int64_t)nsm * per_sm;
        if (m > rp.nrows) m = rp.nrows;
        if (m >= 1) n = (unsigned)m;
    }
    cudaGetLastError();
    cached_lrow = rp.Lrow;
    cached_nrows = rp.nrows;
    cached_nb = n;
    *nb = n;
    return n > 0;
}

template <class S, class T, bool DAG, int IMASS, int PPT>
static bool launch_op_rows(S* out, const S* in, const float* chif, const Geom& g,
                           const RowPlan& rp, typename real_of<T>::type diag,
                           typename real_of<T>::type hpin, int apbc, cudaStream_t st) {
    unsigned nb = 0;
    if (!op_rows_setup<S, T, DAG, IMASS, PPT>(g, rp, &nb)) return false;
    k_dslash_rows<S, T, DAG, IMASS, PPT><<<nb, rp.nthreads, rp.smem, st>>>(out, in, chif, g, rp,
                                                                           diag, hpin, apbc);
    count_launches(1);
    return true;
}

template <class S, class T, int PPT>
static bool launch_op_rows_ppt(bool dag, int imass, S* out, const S* in, const float* chif,
                               const Geom& g, const RowPlan& rp, typename real_of<T>::type diag,
                               typename real_of<T>::type hpin, int apbc, cudaStream_t st) {
#define OPR(D, I) launch_op_rows<S, T, D, I, PPT>(out, in, chif, g, rp, diag, hpin, apbc, st)
    if (!dag) return imass == 1 ? OPR(false, 1) : OPR(false, 3);
    return imass == 1 ? OPR(true, 1) : OPR(true, 3);
#undef OPR
}

template <class S, class T>
static bool launch_op_rows_any(bool dag, int imass, S* out, const S* in, const float* chif,
                               const Geom& g, typename real_of<T>::type diag,
                               typename real_of<T>::type hpin, int apbc, cudaStream_t st) {
    if (imass != 1 && imass != 3) return false;
    RowPlan rp;
    if (!row_plan(g, sizeof(S), &rp)) return false;
    if constexpr (sizeof(S) <= 8) {
        if (rp.ppt == 2)
            return launch_op_rows_ppt<S, T, 2>(dag, imass, out, in, chif, g, rp, diag, hpin, apbc,
                                               st);
    }
    return launch_op_rows_ppt<S, T, 1>(dag, imass, out, in, chif, g, rp, diag, hpin, apbc, st);
}

bool op_rows_launchable(const Geom& g, int elem) {
    RowPlan rp;
    unsigned nb = 0;
    if (!row_plan(g, (size_t)elem, &rp)) return false;
    if (elem == 16) return op_rows_setup<double2, double2, false, 1, 1>(g, rp, &nb);
    if (elem == 8)
        return rp.ppt == 2 ? op_rows_setup<float2, float2, false, 1, 2>(g, rp, &nb)
                           : op_rows_setup<float2, float2, false, 1, 1>(g, rp, &nb);
    return rp.ppt == 2 ? op_rows_setup<__half2, float2, false, 1, 2>(g, rp, &nb)
                       : op_rows_setup<__half2, float2, false, 1, 1>(g, rp, &nb);
}

void launch_dslash64(bool dag, int imass, double2* out, const double2* in, const float* chif,
                     const Geom& g, float am3, float hpin, int ibound, cudaStream_t st,
                     int variant) {
    const unsigned nb = split_blocks(g.npts);
    const double diag = (double)diag_of(am3), hp = (double)hpin;
    const int apbc = ibound == -1;
    const int shape = variant < 0 ? stencil_choice(g, 16, st) : variant;
    if (shape == kStencilRows &&
        launch_op_rows_any<double2, double2>(dag, imass, out, in, chif, g, diag, hp, apbc, st)) {
        note_stencil(kStencilRows, 1);
        return;
    }
    note_stencil(shape == kStencilGather4 ? kStencilGather4 : kStencilGather3, 1);
#define LAUNCH(D, I)                                                                          \
    do {                                                                                      \
        if (shape == kStencilGather4)                                                         \
            k_dslash64<D, I, 4><<<nb, kSplitThreads, 0, st>>>(out, in, chif, g, diag, hp, apbc); \
        else                                                                                  \
            k_dslash64<D, I, 3><<<nb, kSplitThreads, 0, st>>>(out, in, chif, g, diag, hp, apbc); \
    } while (0)
    if (!dag) {
        if (imass == 1) LAUNCH(false, 1); else if (imass == 3) LAUNCH(false, 3); else LAUNCH(false, 0);
    } else {
        if (imass == 1) LAUNCH(true, 1); else if (imass == 3) LAUNCH(true, 3); else LAUNCH(true, 0);
    }
    count_launches(1);
#undef LAUNCH
}

// ---- reduced-precision storage: FP32 spinors (complex64) and FP16 spinors
// (two halves per complex), FP32 arithmetic ----------------------------------
struct LdF32 {
    const float2* __restrict__ p;
    __device__ __forceinline__ float2 operator()(int64_t j) const { return __ldg(p + j); }
};
struct LdF16 {
    const __half2* __restrict__ p;
    __device__ __forceinline__ float2 operator()(int64_t j) const { return __half22float2(__ldg(p + j)); }
};

// One thread per point and both flavours: with FP32 arithmetic the registers
// already allow full occupancy, and this shape is the faster one there.
template <bool DAG, int IMASS, int HALF>
__global__ void __launch_bounds__(kThreads) k_dslash_lp(void* __restrict__ out,
                                                       const void* __restrict__ in,
                                                       const float* __restrict__ chif, Geom g,
                                                       float diag, float hpin, int apbc) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= g.npts) return;
    const PointIdx q = point_of(g, p);
    float2 acc[2][4];
    if (HALF) dwf_apply_point<DAG, IMASS>(acc, LdF16{(const __half2*)in}, g, q, chif, diag, hpin, apbc != 0);
    else dwf_apply_point<DAG, IMASS>(acc, LdF32{(const float2*)in}, g, q, chif, diag, hpin, apbc != 0);
#pragma unroll
    for (int f = 0; f < 2; f++)
#pragma unroll
        for (int d = 0; d < 4; d++) {
            const int64_t e = p + g.cs * (d + 4 * f);
            if (HALF) ((__half2*)out)[e] = __float22half2_rn(acc[f][d]);
            else ((float2*)out)[e] = acc[f][d];
        }
}

// FP32 storage with Ls even: a thread takes two adjacent points of one
// flavour with 16-byte loads (dwf_apply_flavour_pair); a block covers 128
// point pairs of both flavours.
template <bool DAG, int IMASS, int OCC>
__global__ void __launch_bounds__(kSplitThreads, OCC)
    k_dslash_f32_pair(float2* __restrict__ out, const float2* __restrict__ in,
                      const float* __restrict__ chif, Geom g, float diag, float hpin, int apbc) {
    const int64_t p = (int64_t)blockIdx.x * (2 * kSplitPoints) +
                      2 * (threadIdx.x & (kSplitPoints - 1));
    const int f = split_flavour();
    if (p >= g.npts) return;
    const PointIdx q = point_of(g, p);
    float2 acc[2][4];
    dwf_apply_flavour_pair<DAG, IMASS>(acc, in, g, q, f, chif, diag, hpin, apbc != 0);
#pragma unroll
    for (int d = 0; d < 4; d++) {
        const int64_t e = p + g.cs * (d + 4 * f);
        *reinterpret_cast<float4*>(out + e) =
            make_float4(acc[0][d].x, acc[0][d].y, acc[1][d].x, acc[1][d].y);
    }
}

// The same thread shape on a split-layout vector (the FP32 solver's Krylov
// vectors, see cpair): M only, for the autotuner, which times the shapes the
// solver's pass 1 will run.
template <int OCC>
__global__ void __launch_bounds__(kSplitThreads, OCC)
    k_dslash_f32_sp(float2* __restrict__ out, const float2* __restrict__ in,
                    const float* __restrict__ chif, Geom g, float diag) {
    const int64_t p = (int64_t)blockIdx.x * (2 * kSplitPoints) +
                      2 * (threadIdx.x & (kSplitPoints - 1));
    const int f = split_flavour();
    if (p >= g.npts) return;
    const PointIdx q = point_of(g, p);
    cpair acc[4];
    dwf_apply_flavour_pair_sp<false, 1>(acc, in, g, q, f, chif, diag, 0.0f, true);
#pragma unroll
    for (int d = 0; d < 4; d++) st_cpair(out, (uint32_t)(p + g.cs * (d + 4 * f)), acc[d]);
}

void launch_dslash_sp_m(float2* out, const float2* in, const float* chif, const Geom& g,
                        cudaStream_t st, int shape) {
    const unsigned nb2 = (unsigned)((g.npts + 2 * kSplitPoints - 1) / (2 * kSplitPoints));
    const float diag = diag_of(1.0f);
    if (shape == kStencilGather4)
        k_dslash_f32_sp<4><<<nb2, kSplitThreads, 0, st>>>(out, in, chif, g, diag);
    else
        k_dslash_f32_sp<3><<<nb2, kSplitThreads, 0, st>>>(out, in, chif, g, diag);
    count_launches(1);
}

// ---- FP16 storage, four points a thread ----------------------------------------
// Point q (s a multiple of 4) and its three successors s+1..s+3 of flavour f:
// each neighbour is one 16-byte load of four FP16 complex numbers (the layout
// has s innermost), as many bytes per load as the FP32 two-point kernel, and
// the index arithmetic and the wall path are shared by four points.  Each
// element goes through dwf_apply_flavour's operation sequence in FP32.
// Needs Ls a multiple of 4.  (Four FP32 points a thread, at the 128
// registers they need, ran 45% slower than the two-point kernel: two blocks
// an SM hide too little latency.)
__device__ __forceinline__ float2 h2_get(uint32_t w) {
    return __half22float2(*reinterpret_cast<const __half2*>(&w));
}
__device__ __forceinline__ uint32_t h2_bits(float2 v) {
    const __half2 h = __float22half2_rn(v);
    return *reinterpret_cast<const uint32_t*>(&h);
}
template <class S> struct Quad;
template <> struct Quad<__half2> {
    uint4 v;
    __device__ __forceinline__ void load(const __half2* p, int64_t n) {
        v = __ldg(reinterpret_cast<const uint4*>(p + n));
    }
    __device__ __forceinline__ float2 get(int k) const {
        return h2_get(k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w)));
    }
    __device__ __forceinline__ static void store(__half2* p, int64_t n, const float2* a) {
        uint4 o;
        o.x = h2_bits(a[0]);
        o.y = h2_bits(a[1]);
        o.z = h2_bits(a[2]);
        o.w = h2_bits(a[3]);
        *reinterpret_cast<uint4*>(p + n) = o;
    }
    typedef LdF16 Elem;
};
template <bool DAG, int IMASS, class S>
__device__ __forceinline__ void dwf_apply_flavour_quad(float2 acc[4][4], const S* __restrict__ in,
                                                       const Geom& g, const PointIdx& q, int f,
                                                       const float* __restrict__ chif,
                                                       float diag, float hpin, bool apbc) {
    constexpr int SF = DAG ? -1 : 1;
    const int L = g.L, Lt = g.Lt, Ls = g.Ls;
    const int64_t LsI = Ls, cs = g.cs, fo = g.cs * (4 * f);
    // diagonal term (:2651-2667)
#pragma unroll
    for (int d = 0; d < 4; d++) {
        Quad<S> v;
        v.load(in, q.p + fo + cs * d);
#pragma unroll
        for (int p = 0; p < 4; p++) acc[p][d] = zscal(diag, v.get(p));
    }
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
#define CHDWF_QUAD_HOP(N, MU, SIG, NEG)                                                   \
    {                                                                                    \
        Quad<S> v[4];                                                                    \
        _Pragma("unroll") for (int d = 0; d < 4; d++) v[d].load(in, (N) + cs * d);       \
        _Pragma("unroll") for (int p = 0; p < 4; p++) {                                  \
            float2 r[4];                                                                 \
            _Pragma("unroll") for (int d = 0; d < 4; d++) r[d] = v[d].get(p);            \
            hop<MU, SIG, NEG>(acc[p], r);                                                \
        }                                                                                \
    }
    CHDWF_QUAD_HOP(n_xp, 0, SF, false)
    CHDWF_QUAD_HOP(n_xm, 0, -SF, false)
    CHDWF_QUAD_HOP(n_yp, 1, SF, false)
    CHDWF_QUAD_HOP(n_ym, 1, -SF, false)
    CHDWF_QUAD_HOP(n_tp, 2, SF, false)
    CHDWF_QUAD_HOP(n_tm, 2, -SF, false)
    // kappa = 1/2 (:2815-2829)
#pragma unroll
    for (int p = 0; p < 4; p++)
#pragma unroll
        for (int d = 0; d < 4; d++) acc[p][d] = zscal(0.5f, acc[p][d]);
    // antiperiodic boundary in t (:2831-2876)
    if (apbc) {
        if (q.it == Lt - 1) CHDWF_QUAD_HOP(n_tp, 2, SF, true)
        if (q.it == 0) CHDWF_QUAD_HOP(n_tm, 2, -SF, true)
    }
#undef CHDWF_QUAD_HOP
    // s hops (:2879-2908; M^dagger :3313-3342): point p takes s+p+1 (the
    // next point of the group, or the next group's first) and s+p-1 (the
    // previous point, or the previous group's last)
    constexpr int UP = DAG ? 0 : 2;
    constexpr int DN = DAG ? 2 : 0;
    typedef typename Quad<S>::Elem Ld1;
    const Ld1 ld1{in};
#pragma unroll
    for (int d = UP; d < UP + 2; d++) {
        Quad<S> c;
        c.load(in, q.p + fo + cs * d);
#pragma unroll
        for (int p = 0; p < 3; p++) acc[p][d] = zsub(acc[p][d], c.get(p + 1));
        if (q.s + 4 < Ls) acc[3][d] = zsub(acc[3][d], ld1(q.p + 4 + fo + cs * d));
    }
#pragma unroll
    for (int d = DN; d < DN + 2; d++) {
        Quad<S> c;
        c.load(in, q.p + fo + cs * d);
        if (q.s > 0) acc[0][d] = zsub(acc[0][d], ld1(q.p - 1 + fo + cs * d));
#pragma unroll
        for (int p = 1; p < 4; p++) acc[p][d] = zsub(acc[p][d], c.get(p - 1));
    }
    // wall coupling: point 3 at s=Ls or point 0 at s=1 (one of them, Ls >= 8;
    // both for Ls = 4)
    const bool atL = (q.s + 4 == Ls), at0 = (q.s == 0);
    if (!(atL || at0)) return;
    const float c1f = __ldg(chif + q.site), c2f = __ldg(chif + g.kvol + q.site),
                c3f = __ldg(chif + 2 * g.kvol + q.site);
    const bool pin = (q.site == 0);
    if (atL && at0) {
        constexpr int WA = DAG ? 0 : 2;
        constexpr int WB = DAG ? 2 : 0;
        wall_terms<DAG, IMASS, WA, 0>(acc[3], ld1, cs, LsI * q.site, f, c1f, c2f, c3f, pin, hpin);
        wall_terms<DAG, IMASS, WB, 1>(acc[0], ld1, cs, LsI * q.site + Ls - 1, f, c1f, c2f, c3f,
                                      pin, hpin);
        return;
    }
    float2 w[4];
#pragma unroll
    for (int d = 0; d < 4; d++) w[d] = atL ? acc[3][d] : acc[0][d];
    wall_terms_rt<DAG, IMASS>(w, ld1, cs, atL ? LsI * q.site : LsI * q.site + Ls - 1, atL, f, c1f,
                              c2f, c3f, pin, hpin);
#pragma unroll
    for (int d = 0; d < 4; d++) {
        if (atL) acc[3][d] = w[d];
        else acc[0][d] = w[d];
    }
}

template <bool DAG, int IMASS, class S>
__global__ void __launch_bounds__(kSplitThreads, 2)
    k_dslash_quad(S* __restrict__ out, const S* __restrict__ in, const float* __restrict__ chif,
                  Geom g, float diag, float hpin, int apbc) {
    const int64_t p = (int64_t)blockIdx.x * (4 * kSplitPoints) +
                      4 * (threadIdx.x & (kSplitPoints - 1));
    const int f = split_flavour();
    if (p >= g.npts) return;
    const PointIdx q = point_of(g, p);
    float2 acc[4][4];
    dwf_apply_flavour_quad<DAG, IMASS, S>(acc, in, g, q, f, chif, diag, hpin, apbc != 0);
#pragma unroll
    for (int d = 0; d < 4; d++) {
        const float2 v[4] = {acc[0][d], acc[1][d], acc[2][d], acc[3][d]};
        Quad<S>::store(out, p + g.cs * (d + 4 * f), v);
    }
}

void launch_dslash_lp(bool dag, int imass, int half, void* out, const void* in, const float* chif,
                      const Geom& g, float am3, float hpin, int ibound, cudaStream_t st,
                      int variant) {
    const int shape = variant < 0 ? stencil_choice(g, half ? 4 : 8, st) : variant;
    if (shape == kStencilRows) {
        const float diag = diag_of(am3);
        const int apbc = ibound == -1;
        if (half ? launch_op_rows_any<__half2, float2>(dag, imass, (__half2*)out,
                                                       (const __half2*)in, chif, g, diag, hpin,
                                                       apbc, st)
                 : launch_op_rows_any<float2, float2>(dag, imass, (float2*)out,
                                                      (const float2*)in, chif, g, diag, hpin,
                                                      apbc, st)) {
            note_stencil(kStencilRows, 1);
            return;
        }
    }
    note_stencil(shape == kStencilGather4 && !half ? kStencilGather4 : kStencilGather3, 1);
    if (half && g.Ls % 4 == 0) {
        const unsigned nb4 = (unsigned)((g.npts + 4 * kSplitPoints - 1) / (4 * kSplitPoints));
        const float diag = diag_of(am3);
        const int apbc = ibound == -1;
        __half2* o = (__half2*)out;
        const __half2* i = (const __half2*)in;
#define PQ(D, I) k_dslash_quad<D, I, __half2><<<nb4, kSplitThreads, 0, st>>>(o, i, chif, g, diag, hpin, apbc)
        if (!dag) { if (imass == 3) PQ(false, 3); else PQ(false, 1); }
        else { if (imass == 3) PQ(true, 3); else PQ(true, 1); }
#undef PQ
        count_launches(1);
        return;
    }
    if (!half && pair_ok(g)) {
        const unsigned nb2 = (unsigned)((g.npts + 2 * kSplitPoints - 1) / (2 * kSplitPoints));
        const float diag = diag_of(am3);
        const int apbc = ibound == -1;
        float2* o = (float2*)out;
        const float2* i = (const float2*)in;
#define PR(D, I)                                                                             \
    do {                                                                                     \
        if (shape == kStencilGather4)                                                        \
            k_dslash_f32_pair<D, I, 4><<<nb2, kSplitThreads, 0, st>>>(o, i, chif, g, diag, hpin, \
                                                                     apbc);                  \
        else                                                                                 \
            k_dslash_f32_pair<D, I, 3><<<nb2, kSplitThreads, 0, st>>>(o, i, chif, g, diag, hpin, \
                                                                     apbc);                  \
    } while (0)
        if (!dag) { if (imass == 3) PR(false, 3); else PR(false, 1); }
        else { if (imass == 3) PR(true, 3); else PR(true, 1); }
#undef PR
        count_launches(1);
        return;
    }
    const unsigned nb = (unsigned)((g.npts + kThreads - 1) / kThreads);
    const float diag = diag_of(am3);
    const int apbc = ibound == -1;
#define LP(D, I, H) k_dslash_lp<D, I, H><<<nb, kThreads, 0, st>>>(out, in, chif, g, diag, hpin, apbc)
    if (half) {
        if (!dag) { if (imass == 3) LP(false, 3, 1); else LP(false, 1, 1); }
        else { if (imass == 3) LP(true, 3, 1); else LP(true, 1, 1); }
    } else {
        if (!dag) { if (imass == 3) LP(false, 3, 0); else LP(false, 1, 0); }
        else { if (imass == 3) LP(true, 3, 0); else LP(true, 1, 0); }
    }
#undef LP
    count_launches(1);
}

// M on npole stacked two-slice lattices: blockIdx.y = pole.
template <int IMASS>
__global__ void __launch_bounds__(kThreads) k_wall_dslash64(double2* __restrict__ out,
                                                           const double2* __restrict__ in,
                                                           const float* __restrict__ chif,
                                                           Geom g2, double diag, double hpin,
                                                           int apbc) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= g2.npts) return;
    const int64_t off = (int64_t)blockIdx.y * g2.kferm;
    const PointIdx q = point_of(g2, p);
    double2 acc[2][4];
    dwf_apply_point<false, IMASS>(acc, LdF64{in + off}, g2, q, chif, diag, hpin, apbc != 0);
#pragma unroll
    for (int f = 0; f < 2; f++)
#pragma unroll
        for (int d = 0; d < 4; d++) out[off + p + g2.cs * (d + 4 * f)] = acc[f][d];
}

void launch_wall_dslash64(int npole, double2* out, const double2* in, const float* chif,
                          const Geom& g, float am3, float hpin, int ibound, int imass,
                          cudaStream_t st) {
    const Geom g2 = make_geom(g.L, g.Lt, 2);
    const unsigned nb = (unsigned)((g2.npts + kThreads - 1) / kThreads);
    const dim3 grid(nb, npole);
    const double diag = (double)diag_of(am3), hp = (double)hpin;
    const int apbc = ibound == -1;
    if (imass == 1) k_wall_dslash64<1><<<grid, kThreads, 0, st>>>(out, in, chif, g2, diag, hp, apbc);
    else if (imass == 3) k_wall_dslash64<3><<<grid, kThreads, 0, st>>>(out, in, chif, g2, diag, hp, apbc);
    else k_wall_dslash64<0><<<grid, kThreads, 0, st>>>(out, in, chif, g2, diag, hp, apbc);
    count_launches(1);
}

// ---- derivs ---------------------------------------------------------------
// One term of derivs for one site and one Dirac index: R and X2 of both
// flavours; REAL*8 products, REAL*4 accumulation (cheisdwf.f:762-845).
template <int IMASS>
__device__ __forceinline__ void derivs_term(float* f, double2 r1, double2 r2, double2 y1,
                                            double2 y2, double tzi, bool lower) {
    r1 = zconj(r1);
    r2 = zconj(r2);
    const double2 c1 = zscal(tzi, zadd(zmul(r1, y2), zmul(r2, y1)));
    const double2 c2 = zscal(tzi, zsub(zmul(r1, y2), zmul(r2, y1)));
    const double2 c3 = zscal(tzi, zsub(zmul(r1, y1), zmul(r2, y2)));
    if (IMASS == 1) {
        f[0] = (float)__dsub_rn((double)f[0], c1.x);
        f[1] = (float)__dsub_rn((double)f[1], c2.y);
        f[2] = (float)__dsub_rn((double)f[2], c3.x);
    } else if (IMASS == 3) {
        if (lower) {   // Dirac 1,2 (:806-823)
            f[0] = (float)__dsub_rn((double)f[0], c1.y);
            f[1] = (float)__dadd_rn((double)f[1], c2.x);
            f[2] = (float)__dsub_rn((double)f[2], c3.y);
        } else {       // Dirac 3,4 (:825-843)
            f[0] = (float)__dadd_rn((double)f[0], c1.y);
            f[1] = (float)__dsub_rn((double)f[1], c2.x);
            f[2] = (float)__dadd_rn((double)f[2], c3.y);
        }
    }
}

// Per site, poles in order k=1..npole, Dirac 1,2 (R at s=Ls, X2 at s=1)
// then Dirac 3,4 (R at s=1, X2 at s=Ls) -- the accumulation order of
// qmrherm's force branch (cheisdwf.f:733-740) calling derivs.
template <int IMASS>
__global__ void __launch_bounds__(kThreads) k_derivs_walls(int npole,
                                                          const double2* __restrict__ xw,
                                                          const double2* __restrict__ x2w,
                                                          const double* __restrict__ anum1,
                                                          float* __restrict__ dS, Geom g2) {
    const int site = blockIdx.x * blockDim.x + threadIdx.x;
    if (site >= g2.kvol) return;
    float f[3] = {dS[site], dS[site + g2.kvol], dS[site + 2 * g2.kvol]};
    for (int k = 0; k < npole; k++) {
        const double tzi = -2 * anum1[k];
        const int64_t off = (int64_t)k * g2.kferm;
        const int64_t pL = 1 + 2 * (int64_t)site, p0 = 2 * (int64_t)site;
#pragma unroll
        for (int d = 0; d < 2; d++)
            derivs_term<IMASS>(f, xw[off + pL + g2.cs * d], xw[off + pL + g2.cs * (d + 4)],
                               x2w[off + p0 + g2.cs * d], x2w[off + p0 + g2.cs * (d + 4)], tzi, true);
#pragma unroll
        for (int d = 2; d < 4; d++)
            derivs_term<IMASS>(f, xw[off + p0 + g2.cs * d], xw[off + p0 + g2.cs * (d + 4)],
                               x2w[off + pL + g2.cs * d], x2w[off + pL + g2.cs * (d + 4)], tzi, false);
    }
    dS[site] = f[0];
    dS[site + g2.kvol] = f[1];
    dS[site + 2 * g2.kvol] = f[2];
}

void launch_derivs_walls(int npole, const double2* xw, const double2* x2w, const double* anum1,
                         int imass, float* dSdchi, const Geom& g, cudaStream_t st) {
    const Geom g2 = make_geom(g.L, g.Lt, 2);
    const unsigned nb = (unsigned)((g.kvol + kThreads - 1) / kThreads);
    if (imass == 1) k_derivs_walls<1><<<nb, kThreads, 0, st>>>(npole, xw, x2w, anum1, dSdchi, g2);
    else if (imass == 3) k_derivs_walls<3><<<nb, kThreads, 0, st>>>(npole, xw, x2w, anum1, dSdchi, g2);
    count_launches(1);
}

template <int IMASS>
__global__ void __launch_bounds__(kThreads) k_derivs_full(const double2* __restrict__ R,
                                                         const double2* __restrict__ X2,
                                                         double tzi, float* __restrict__ dS,
                                                         Geom g) {
    const int site = blockIdx.x * blockDim.x + threadIdx.x;
    if (site >= g.kvol) return;
    float f[3] = {dS[site], dS[site + g.kvol], dS[site + 2 * g.kvol]};
    const int64_t pL = (int64_t)g.Ls * site + g.Ls - 1, p0 = (int64_t)g.Ls * site;
#pragma unroll
    for (int d = 0; d < 2; d++)
        derivs_term<IMASS>(f, R[pL + g.cs * d], R[pL + g.cs * (d + 4)], X2[p0 + g.cs * d],
                           X2[p0 + g.cs * (d + 4)], tzi, true);
#pragma unroll
    for (int d = 2; d < 4; d++)
        derivs_term<IMASS>(f, R[p0 + g.cs * d], R[p0 + g.cs * (d + 4)], X2[pL + g.cs * d],
                           X2[pL + g.cs * (d + 4)], tzi, false);
    dS[site] = f[0];
    dS[site + g.kvol] = f[1];
    dS[site + 2 * g.kvol] = f[2];
}

void launch_derivs_full(const double2* R, const double2* X2, double anum, int imass,
                        float* dSdchi, const Geom& g, cudaStream_t st) {
    const unsigned nb = (unsigned)((g.kvol + kThreads - 1) / kThreads);
    const double tzi = -2 * anum;
    if (imass == 1) k_derivs_full<1><<<nb, kThreads, 0, st>>>(R, X2, tzi, dSdchi, g);
    else if (imass == 3) k_derivs_full<3><<<nb, kThreads, 0, st>>>(R, X2, tzi, dSdchi, g);
    count_launches(1);
}

}  // namespace chdwf
