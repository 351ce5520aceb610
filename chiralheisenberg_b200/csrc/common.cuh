// common.cuh -- shared device helpers for the chiral-Heisenberg domain-wall
// fermion kernels (sm_100a).
//
// Field layout in HBM is the reference's own Fortran layout
// (rhmc/cheisdwf.f:50-54, :2644-2645), 0-based:
//   spinor element (s, x, y, t, dirac d, flavour f) at
//     s + Ls*(x + L*(y + L*t)) + cs*(d + 4*f),   cs = Ls*kvol,
// i.e. eight component planes ("SoA over the 8 complex components"), each
// point-fastest with the fifth dimension s innermost.  One thread owns one
// lattice point (s, site) and all eight components, so every plane access of
// a warp is a contiguous, coalesced run of 16-byte (FP64) elements and the
// host<->device copies at the drop-in boundary are plain memcpys.  The
// solver's FP32 Krylov vectors (Ls even, never copied across the boundary)
// keep the same planes with each pair of adjacent s split by part: see
// cpair below.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace chdwf {

// Unsigned division by a divisor fixed at set-up, for numerators below 2^31:
// q = (umulhi(n, m) + n) >> l with l = ceil(log2 d) and
// m = floor(2^32 (2^l - d) / d) + 1 (Granlund and Montgomery, "Division by
// invariant integers using multiplication", PLDI 1994, the round-up method
// with an added numerator).  Three integer instructions instead of the
// reciprocal sequence a division by a run-time value compiles to.
struct FastDiv {
    uint32_t d, m, l;
};
inline FastDiv make_fastdiv(uint32_t d) {
    FastDiv f;
    f.d = d;
    f.l = 0;
    while ((1ull << f.l) < d) f.l++;
    f.m = (uint32_t)((((1ull << 32) * ((1ull << f.l) - d)) / d) + 1);
    return f;
}
__host__ __device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f) {
#ifdef __CUDA_ARCH__
    const uint32_t t = __umulhi(n, f.m);
#else
    const uint32_t t = (uint32_t)(((uint64_t)n * f.m) >> 32);
#endif
    return (t + n) >> f.l;
}

struct Geom {
    int L, Lt, Ls;
    int kvol;         // L*L*Lt
    int64_t npts;     // kvol*Ls
    int64_t cs;       // component-plane stride = npts
    int64_t kferm;    // 8*npts complex numbers
    FastDiv dLs, dL, dLL;   // division by Ls, L, L*L (point decoding)
};

// Lattices are limited to 2^31 - 1 points (kthird*ksize^2*ksizet), far
// beyond one GPU's memory; point indices then fit 32-bit arithmetic.
constexpr int64_t kMaxPoints = 2147483647LL;

inline bool geom_ok(int L, int Lt, int Ls) {
    return L >= 2 && Lt >= 2 && Ls >= 2 && (int64_t)L * L * Lt * Ls <= kMaxPoints;
}

inline Geom make_geom(int L, int Lt, int Ls) {
    Geom g;
    g.L = L; g.Lt = Lt; g.Ls = Ls;
    g.kvol = L * L * Lt;
    g.npts = (int64_t)g.kvol * Ls;
    g.cs = g.npts;
    g.kferm = 8 * g.npts;
    g.dLs = make_fastdiv((uint32_t)Ls);
    g.dL = make_fastdiv((uint32_t)L);
    g.dLL = make_fastdiv((uint32_t)L * (uint32_t)L);
    return g;
}

// ---- exact (non-contracted) double-complex arithmetic ---------------------
// The FP64 operator reproduces the reference's per-element operation order
// without fused multiply-add, so it agrees bit for bit with the CPU oracle.
__device__ __forceinline__ double2 zadd(double2 a, double2 b) {
    return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
__device__ __forceinline__ double2 zsub(double2 a, double2 b) {
    return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
}
__device__ __forceinline__ double2 zmuli(double2 a) { return make_double2(-a.y, a.x); }
__device__ __forceinline__ double2 zscal(double s, double2 a) {
    return make_double2(__dmul_rn(s, a.x), __dmul_rn(s, a.y));
}
__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                        __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 zconj(double2 a) { return make_double2(a.x, -a.y); }
// x + (i? i*y : y) or x - (...)
__device__ __forceinline__ double2 zcomb(double2 x, double2 y, bool use_i, int sgn) {
    double2 t = use_i ? zmuli(y) : y;
    return sgn > 0 ? zadd(x, t) : zsub(x, t);
}

// ---- single-precision complex (mixed-precision path) ----------------------
// Also without contraction: every kernel that evaluates the same per-element
// sequence (the pass-1 kernels and the regenerating pass 2, whatever their
// thread shape) then produces the same bits, so regenerated Lanczos vectors
// equal the first pass's.
//
// On sm_100 an addition or subtraction of FP32 complex numbers is one packed
// FP32x2 instruction (add/sub.rn.f32x2, written as PTX) instead of two scalar
// ones; per lane it rounds exactly as __fadd_rn / __fsub_rn.  Products stay
// scalar (__fmul_rn): measured on B200, the code generator fuses a packed
// multiply whose only use is a packed add or subtract into a packed fused
// multiply-add (one rounding instead of two), even with .rn, while scalar
// products feeding packed sums are left alone.  x +- i*y mixes the lanes and
// stays scalar.  Host builds of these helpers (the CPU tests of the element
// functions) use the scalar forms, which give the same bits.
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000)
#define CHDWF_F32X2 1
#endif
#ifdef CHDWF_F32X2
#define CHDWF_F2OP(NAME, OP)                                                               \
    __device__ __forceinline__ float2 NAME(float2 a, float2 b) {                           \
        float2 d;                                                                          \
        asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t" \
            OP " rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"                                 \
            : "=f"(d.x), "=f"(d.y)                                                         \
            : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));                                     \
        return d;                                                                          \
    }
CHDWF_F2OP(f2_add, "add.rn.f32x2")
CHDWF_F2OP(f2_sub, "sub.rn.f32x2")
#undef CHDWF_F2OP
#else
__device__ __forceinline__ float2 f2_add(float2 a, float2 b) {
    return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}
__device__ __forceinline__ float2 f2_sub(float2 a, float2 b) {
    return make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y));
}
#endif
__device__ __forceinline__ float2 f2_mul(float2 a, float2 b) {
    return make_float2(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
}
__device__ __forceinline__ float2 zadd(float2 a, float2 b) { return f2_add(a, b); }
__device__ __forceinline__ float2 zsub(float2 a, float2 b) { return f2_sub(a, b); }
__device__ __forceinline__ float2 zmuli(float2 a) { return make_float2(-a.y, a.x); }
__device__ __forceinline__ float2 zscal(float s, float2 a) { return f2_mul(make_float2(s, s), a); }
__device__ __forceinline__ float2 zmul(float2 a, float2 b) {
    return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                       __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float2 zconj(float2 a) { return make_float2(a.x, -a.y); }
// x +- y packed; x +- i*y = (x.x -+ y.y, x.y +- y.x) as two scalar operations
__device__ __forceinline__ float2 zcomb(float2 x, float2 y, bool use_i, int sgn) {
    if (!use_i) return sgn > 0 ? zadd(x, y) : zsub(x, y);
    return sgn > 0 ? make_float2(__fsub_rn(x.x, y.y), __fadd_rn(x.y, y.x))
                   : make_float2(__fadd_rn(x.x, y.y), __fsub_rn(x.y, y.x));
}

// ---- FP32 complex numbers of two adjacent points, split by part ------------
// The solver's FP32 Krylov vectors (Ls even) keep every aligned element pair
// (e, e+1), e even -- two adjacent s of one component -- as the 16 bytes
// (re_e, re_e+1, im_e, im_e+1): the "split" layout.  One 16-byte load then
// puts both real parts in one register pair and both imaginary parts in the
// other, so each complex operation on the two points, i*y included, is two
// packed instructions with no lane exchange; per element the IEEE operations
// are those of the float2 forms above.
struct cpair {
    float2 re, im;   // (point s, point s+1)
};
__device__ __forceinline__ cpair zadd(cpair a, cpair b) {
    return cpair{f2_add(a.re, b.re), f2_add(a.im, b.im)};
}
__device__ __forceinline__ cpair zsub(cpair a, cpair b) {
    return cpair{f2_sub(a.re, b.re), f2_sub(a.im, b.im)};
}
__device__ __forceinline__ cpair zscal(float s, cpair a) {
    const float2 ss = make_float2(s, s);
    return cpair{f2_mul(ss, a.re), f2_mul(ss, a.im)};
}
// x +- y, or x +- i*y: re = x.re -+ y.im, im = x.im +- y.re
__device__ __forceinline__ cpair zcomb(cpair x, cpair y, bool use_i, int sgn) {
    if (!use_i) return sgn > 0 ? zadd(x, y) : zsub(x, y);
    return sgn > 0 ? cpair{f2_sub(x.re, y.im), f2_add(x.im, y.re)}
                   : cpair{f2_add(x.re, y.im), f2_sub(x.im, y.re)};
}
__device__ __forceinline__ float2 cpair_pt(const cpair& c, int k) {   // point k as a complex
    return k ? make_float2(c.re.y, c.im.y) : make_float2(c.re.x, c.im.x);
}
// Element pair at even element e of a split-layout vector
__device__ __forceinline__ cpair ld_cpair(const float2* v, uint32_t e) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(v + e));
    return cpair{make_float2(q.x, q.y), make_float2(q.z, q.w)};
}
__device__ __forceinline__ void st_cpair(float2* v, uint32_t e, const cpair& c) {
    *reinterpret_cast<float4*>(v + e) = make_float4(c.re.x, c.re.y, c.im.x, c.im.y);
}
// Any element e of a split-layout vector
__device__ __forceinline__ float2 sp_get(const float2* v, int64_t e) {
    const float* f = reinterpret_cast<const float*>(v + (e & ~(int64_t)1));
    const int o = (int)(e & 1);
    return make_float2(__ldg(f + o), __ldg(f + 2 + o));
}
__device__ __forceinline__ void sp_put(float2* v, int64_t e, float2 x) {
    float* f = reinterpret_cast<float*>(v + (e & ~(int64_t)1));
    const int o = (int)(e & 1);
    f[o] = x.x;
    f[2 + o] = x.y;
}


template <class T> struct real_of;
template <> struct real_of<double2> { typedef double type; };
template <> struct real_of<float2> { typedef float type; };
template <class T> __device__ __forceinline__ T zmake(typename real_of<T>::type re,
                                                      typename real_of<T>::type im);
template <> __device__ __forceinline__ double2 zmake<double2>(double re, double im) {
    return make_double2(re, im);
}
template <> __device__ __forceinline__ float2 zmake<float2>(float re, float im) {
    return make_float2(re, im);
}

// ---- block reductions (deterministic order) -------------------------------
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NT / 32; i++) r += sh[i];
    }
    __syncthreads();
    return r;  // valid in thread 0
}

// Grid-wide sum of one double per thread: each block writes its block sum to
// part[blockIdx.x]; the block that arrives last (counted in *count) adds the
// partials in block order, stores the total in *total (thread 0), resets the
// counter for the next launch and returns true.  Every other block returns
// false.  The result does not depend on the order in which blocks finish.
template <int NT>
__device__ __forceinline__ bool last_block_total(double v, double* part, unsigned* count,
                                                 double* total) {
    __shared__ double sh[NT / 32];
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
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) s += ((volatile double*)part)[i];
    s = block_sum<NT>(s, sh);
    if (threadIdx.x == 0) {
        *total = s;
        *count = 0;
    }
    return true;
}

}  // namespace chdwf
