// multishift.cu -- per-shift solutions of (M^dag M + sigma_k) x_k = Phi with
// their true residuals (no reference routine returns them: qmrherm keeps
// x1(ndiag,kferm) internally, rhmc/cheisdwf.f:614,:689-695, and testinv,
// :854-890, checks each pole's true residual), in FP64 or with FP32 Krylov
// vectors and FP64 defect correction.
//
// FP64: the two-pass Lanczos solve (lanczos.cu) with every x_k formed from
// the stored basis, stopping by the reference's rule at res.
// FP32: the same solve with FP32 vectors stopped at max(res, 1e-6), x_k
// accumulated in FP64; then, per shift, while the FP64 true residual
// |Phi - (M^dag M + sigma_k) x_k| / |Phi| exceeds res: an FP32 CG on the
// shifted system with the FP64 residual as right-hand side, run until its
// own residual falls by 1e-4 (or stagnates), and its solution added to x_k
// in FP64 -- defect correction, each outer step recomputing the true
// residual in FP64.  The result meets the same true-residual target as FP64.
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/chdwf.h"
#include "ctx.h"
#include "lanczos.h"

using namespace chdwf;

namespace chdwf {
namespace {

unsigned nb_of(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// r = Phi - t - sigma x (FP64); partial sums of |r|^2 per block
__global__ void k_ms_resid(double2* __restrict__ r, const double2* __restrict__ phi,
                           const double2* __restrict__ t, const double2* __restrict__ x,
                           double sigma, int64_t n, double* __restrict__ part) {
    __shared__ double sh[kThreads / 32];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double2 v = make_double2(phi[i].x - t[i].x - sigma * x[i].x,
                                       phi[i].y - t[i].y - sigma * x[i].y);
        r[i] = v;
        s += v.x * v.x + v.y * v.y;
    }
    s = block_sum<kThreads>(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// FP32 vector kernels of the inner CG; reductions in FP64
__global__ void k_ms_to32(float2* __restrict__ o, const double2* __restrict__ i, double scale,
                          int64_t n) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < n) o[k] = make_float2((float)(i[k].x * scale), (float)(i[k].y * scale));
}
__global__ void k_ms_dot32(const float2* __restrict__ a, const float2* __restrict__ b, int64_t n,
                           double* __restrict__ part) {
    __shared__ double sh[kThreads / 32];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        s += (double)a[i].x * b[i].x + (double)a[i].y * b[i].y;
    s = block_sum<kThreads>(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}
// ap = t + sigma p
__global__ void k_ms_shift32(float2* __restrict__ ap, const float2* __restrict__ t,
                             const float2* __restrict__ p, float sigma, int64_t n) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < n) ap[k] = make_float2(t[k].x + sigma * p[k].x, t[k].y + sigma * p[k].y);
}
// e += alpha p ; r -= alpha ap
__global__ void k_ms_update32(float2* __restrict__ e, float2* __restrict__ r,
                              const float2* __restrict__ p, const float2* __restrict__ ap,
                              float alpha, int64_t n) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < n) {
        e[k] = make_float2(e[k].x + alpha * p[k].x, e[k].y + alpha * p[k].y);
        r[k] = make_float2(r[k].x - alpha * ap[k].x, r[k].y - alpha * ap[k].y);
    }
}
// p = r + beta p
__global__ void k_ms_dir32(float2* __restrict__ p, const float2* __restrict__ r, float beta,
                           int64_t n) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < n) p[k] = make_float2(r[k].x + beta * p[k].x, r[k].y + beta * p[k].y);
}
// x += scale * e (FP64)
__global__ void k_ms_add(double2* __restrict__ x, const float2* __restrict__ e, double scale,
                         int64_t n) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < n) x[k] = make_double2(x[k].x + scale * e[k].x, x[k].y + scale * e[k].y);
}

double host_sum(const double* part_dev, int nb, cudaStream_t st) {
    std::vector<double> h(nb);
    cudaMemcpyAsync(h.data(), part_dev, sizeof(double) * nb, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    double s = 0.0;
    for (double v : h) s += v;
    return s;
}

struct MsWork {
    double2 *t = nullptr, *r = nullptr;
    float2 *e = nullptr, *rr = nullptr, *p = nullptr, *ap = nullptr, *t32 = nullptr;
    double* part = nullptr;
    double2** xk_dev = nullptr;
    ~MsWork() {
        cudaFree(t); cudaFree(r); cudaFree(e); cudaFree(rr); cudaFree(p); cudaFree(ap);
        cudaFree(t32); cudaFree(part); cudaFree(xk_dev);
    }
};

// |Phi - (M^dag M + sigma) x|^2 into *r2 (FP64), residual vector in w.r
cudaError_t true_residual(Ctx* c, MsWork& w, const double2* phi, const double2* x, double sigma,
                          float hpin, int imass, double* r2) {
    const Geom& g = c->g;
    launch_dslash64(false, imass, w.t, x, c->chif, g, c->am3, hpin, c->ibound, c->stream);
    launch_dslash64(true, imass, c->spin[3], w.t, c->chif, g, c->am3, hpin, c->ibound, c->stream);
    const int nb = reduce_blocks(g.kferm);
    k_ms_resid<<<nb, kThreads, 0, c->stream>>>(w.r, phi, c->spin[3], x, sigma, g.kferm, w.part);
    count_launches(1);
    *r2 = host_sum(w.part, nb, c->stream);
    return cudaGetLastError();
}

// FP32 CG on (M^dag M + sigma) e = r/|r|, to a relative residual of tol or
// maxit iterations; e (FP32) holds the solution of the normalised system.
cudaError_t inner_cg32(Ctx* c, MsWork& w, float sigma, float hpin, int imass, double tol,
                       int maxit, int* iters) {
    const Geom& g = c->g;
    const int64_t n = g.kferm;
    const int nb = reduce_blocks(n), nbe = (int)nb_of(n);
    cudaStream_t st = c->stream;
    cudaMemsetAsync(w.e, 0, sizeof(float2) * n, st);
    cudaMemcpyAsync(w.p, w.rr, sizeof(float2) * n, cudaMemcpyDeviceToDevice, st);
    k_ms_dot32<<<nb, kThreads, 0, st>>>(w.rr, w.rr, n, w.part);
    double rr = host_sum(w.part, nb, st);
    const double rr0 = rr;
    int it = 0;
    for (; it < maxit && rr > tol * tol * rr0; it++) {
        launch_dslash_lp(false, imass, 0, w.t32, w.p, c->chif, g, c->am3, hpin, c->ibound, st);
        launch_dslash_lp(true, imass, 0, w.ap, w.t32, c->chif, g, c->am3, hpin, c->ibound, st);
        k_ms_shift32<<<nbe, kThreads, 0, st>>>(w.ap, w.ap, w.p, sigma, n);
        k_ms_dot32<<<nb, kThreads, 0, st>>>(w.p, w.ap, n, w.part);
        const double pap = host_sum(w.part, nb, st);
        if (!(pap > 0.0)) break;
        const double alpha = rr / pap;
        k_ms_update32<<<nbe, kThreads, 0, st>>>(w.e, w.rr, w.p, w.ap, (float)alpha, n);
        k_ms_dot32<<<nb, kThreads, 0, st>>>(w.rr, w.rr, n, w.part);
        const double rn = host_sum(w.part, nb, st);
        k_ms_dir32<<<nbe, kThreads, 0, st>>>(w.p, w.rr, (float)(rn / rr), n);
        count_launches(6);
        rr = rn;
    }
    *iters = it;
    return cudaGetLastError();
}

}  // namespace
}  // namespace chdwf

extern "C" int chdwf_multishift_dev(chdwf_ctx* ctx, const void* Phi, float res, const void* chi,
                                    float hpin, int imass, int n, const double* sigma,
                                    void* const* x, double* true_res, int prec, int* iters,
                                    int* refine_iters) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !Phi || !chi || !sigma || !x || !true_res || !iters || !refine_iters) return CHDWF_BAD_ARG;
    if (n < 1 || n > kMaxPoles || (prec != CHDWF_PREC_F64 && prec != CHDWF_PREC_F32)) return CHDWF_BAD_ARG;
    cudaSetDevice(c->device);
    const Geom& g = c->g;
    cudaStream_t st = c->stream;
    launch_round_chi((const double*)chi, c->chif, g.kvol, st);
    MsWork w;
    cudaError_t e;
    if ((e = cudaMalloc(&w.t, sizeof(double2) * g.kferm)) ||
        (e = cudaMalloc(&w.r, sizeof(double2) * g.kferm)) ||
        (e = cudaMalloc(&w.part, sizeof(double) * 8192)) ||
        (e = cudaMalloc(&w.xk_dev, sizeof(double2*) * n)))
        return c->status_of(e, "multishift");
    if (prec == CHDWF_PREC_F32 &&
        ((e = cudaMalloc(&w.e, sizeof(float2) * g.kferm)) ||
         (e = cudaMalloc(&w.rr, sizeof(float2) * g.kferm)) ||
         (e = cudaMalloc(&w.p, sizeof(float2) * g.kferm)) ||
         (e = cudaMalloc(&w.ap, sizeof(float2) * g.kferm)) ||
         (e = cudaMalloc(&w.t32, sizeof(float2) * g.kferm))))
        return c->status_of(e, "multishift");
    cudaMemcpyAsync(w.xk_dev, x, sizeof(double2*) * n, cudaMemcpyHostToDevice, st);
    std::vector<double> anum(n + 1, 1.0);
    anum[0] = 0.0;
    const float res1 = prec == CHDWF_PREC_F32 ? std::fmax(res, 1e-6f) : res;
    int st_code = 0;
    c->lz.pole_out = w.xk_dev;
    e = lz_solve(c->lz, g, (const double2*)Phi, res1, n, anum.data(), sigma, 2, c->chif, c->am3,
                 hpin, imass, c->ibound, nullptr, c->dS, iters, &st_code, &c->last_lz, st,
                 prec == CHDWF_PREC_F32 ? kPrecF32 : kPrecF64);
    c->lz.pole_out = nullptr;
    if (e) return c->status_of(e, "multishift (basis store too small for per-shift output?)");
    if (st_code == 1) { c->err = "multishift: iteration cap reached"; return CHDWF_ITER_CAP; }
    if (st_code == 2) { c->err = "multishift: non-finite value"; return CHDWF_NONFINITE; }
    double phi2 = 0.0;
    launch_norm2((const double2*)Phi, g.kferm, w.part, c->red, st);
    cudaMemcpyAsync(&phi2, c->red, sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    const double phin = std::sqrt(phi2);
    *refine_iters = 0;
    for (int k = 0; k < n; k++) {
        double2* xk = (double2*)x[k];
        double r2 = 0.0;
        if ((e = true_residual(c, w, (const double2*)Phi, xk, sigma[k], hpin, imass, &r2)))
            return c->status_of(e, "multishift residual");
        double rel = std::sqrt(r2) / phin;
        if (prec == CHDWF_PREC_F32) {
            // defect correction: FP32 CG on the FP64 residual, added in FP64
            for (int outer = 0; outer < 20 && rel > (double)res; outer++) {
                const double rn = std::sqrt(r2);
                k_ms_to32<<<nb_of(g.kferm), kThreads, 0, st>>>(w.rr, w.r, 1.0 / rn, g.kferm);
                count_launches(1);
                int it = 0;
                if ((e = inner_cg32(c, w, (float)sigma[k], hpin, imass, 1e-4, 4 * kMaxIter, &it)))
                    return c->status_of(e, "multishift refinement");
                *refine_iters += it;
                k_ms_add<<<nb_of(g.kferm), kThreads, 0, st>>>(xk, w.e, rn, g.kferm);
                count_launches(1);
                if ((e = true_residual(c, w, (const double2*)Phi, xk, sigma[k], hpin, imass, &r2)))
                    return c->status_of(e, "multishift residual");
                const double nrel = std::sqrt(r2) / phin;
                if (!(nrel < rel)) { rel = nrel; break; }   // stagnation
                rel = nrel;
            }
        }
        true_res[k] = rel;
    }
    return c->status_of(cudaStreamSynchronize(st), "multishift");
}
