// traj.cu -- resident trajectory blocks of program dwf3d (rhmc/cheisdwf.f:
// 207-399) for the C ABI: pseudofermion heatbath, hamilton, force, leapfrog
// updates, acceptance and the propagator solve of fermion(), with chi, chit,
// pp, dSdchi and Phi kept in HBM.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/chdwf.h"
#include "cg.h"
#include "ctx.h"
#include "lanczos.h"

using namespace chdwf;

namespace chdwf {

// R(s,i,d,f) = cmplx(ps(i,1), ps(i,2)) of gauss0 call c = s + Ls*(d + 4 f)
// (loop order of :221-230).
__global__ void k_build_source(double2* __restrict__ R, const float* __restrict__ ps, Geom g) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t ncall = 8 * (int64_t)g.Ls;
    if (t >= ncall * g.kvol) return;
    const int64_t c = t / g.kvol, i = t - c * g.kvol;
    const int s = (int)(c % g.Ls), df = (int)(c / g.Ls);
    const float* p = ps + c * 2 * (int64_t)g.kvol;
    R[s + (int64_t)g.Ls * i + g.cs * df] = make_double2((double)p[i], (double)p[g.kvol + i]);
}

// pp = pp - dSdchi*d in REAL*4 (:273-277, :300-311)
__global__ void k_update_p(float* __restrict__ pp, const float* __restrict__ dS, float d, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pp[i] = pp[i] - dS[i] * d;
}

// chit = chit + d*pp, the increment a REAL*4 product (:285-289)
__global__ void k_update_chi(double* __restrict__ chit, const float* __restrict__ pp, float d, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) chit[i] = __dadd_rn(chit[i], (double)(d * pp[i]));
}

// hp = 0.5 sum (pp*pp)_REAL*4, hg = sum chi^2 (:546-559); deterministic
__global__ void k_hamilton_bos(const float* __restrict__ pp, const double* __restrict__ chi, int n,
                               double* __restrict__ out) {
    __shared__ double sh[kThreads / 32];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float q = pp[i] * pp[i];
        a += (double)q;
        b += chi[i] * chi[i];
    }
    a = block_sum<kThreads>(a, sh);
    b = block_sum<kThreads>(b, sh);
    if (threadIdx.x == 0) { out[0] = a; out[1] = b; }
}

// wall source of fermion(): xi = 0 except xi(1, i+ioff, idsource, 1) = 1/ksize2
// for the ksize^2 sites of timeslice ittt (:944-976)
__global__ void k_wall_source(double2* __restrict__ xi, Geom g, int64_t ioff, int idsource,
                              double val) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t ksize2 = (int64_t)g.L * g.L;
    if (i < ksize2) xi[(int64_t)g.Ls * (i + ioff) + g.cs * (idsource - 1)] = make_double2(val, 0.0);
}

// copy of the two walls needed by the correlators: s=1 Dirac 1,2 and s=Ls
// Dirac 3,4, both flavours -> out[(w*2 + dd)*2 + f][kvol] complex, w=0: s=1
__global__ void k_extract_walls(const double2* __restrict__ xi, Geom g, double2* __restrict__ out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= 8 * (int64_t)g.kvol) return;
    const int64_t i = t % g.kvol;
    const int c = (int)(t / g.kvol);           // (w*2 + dd)*2 + f
    const int f = c & 1, dd = (c >> 1) & 1, w = c >> 2;
    const int d = w == 0 ? dd : dd + 2;
    const int s = w == 0 ? 0 : g.Ls - 1;
    out[t] = xi[s + (int64_t)g.Ls * i + g.cs * (d + 4 * f)];
}

// noise source of measure(): xi(s, i, d, f) = cmplx(eta(i,1), eta(i,2)) for
// both flavours (rhmc/cheisdwf.f:1196-1208, :1226-1242); xi is zero elsewhere
__global__ void k_noise_source(double2* __restrict__ xi, Geom g, const float* __restrict__ eta,
                               int s, int d) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= 2 * (int64_t)g.kvol) return;
    const int64_t i = t % g.kvol;
    const int f = (int)(t / g.kvol);
    xi[s + (int64_t)g.Ls * i + g.cs * (d + 4 * f)] =
        make_double2((double)eta[i], (double)eta[g.kvol + i]);
}

// one wall slice of one Dirac component, both flavours -> out[f][kvol]
__global__ void k_extract_slice(const double2* __restrict__ xi, Geom g, int s, int d,
                                double2* __restrict__ out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= 2 * (int64_t)g.kvol) return;
    const int64_t i = t % g.kvol;
    const int f = (int)(t / g.kvol);
    out[t] = xi[s + (int64_t)g.Ls * i + g.cs * (d + 4 * f)];
}

static unsigned nblk(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// launchers shared with the multi-pseudofermion blocks (ext.cu)
void launch_build_source(double2* R, const float* ps, const Geom& g, cudaStream_t st) {
    k_build_source<<<nblk(8 * (int64_t)g.Ls * g.kvol), kThreads, 0, st>>>(R, ps, g);
    count_launches(1);
}
void launch_hamilton_bos(const float* pp, const double* chi, int n, double* out, cudaStream_t st) {
    k_hamilton_bos<<<1, kThreads, 0, st>>>(pp, chi, n, out);
    count_launches(1);
}

cudaError_t Ctx::ensure_traj() {
    if (chit) return cudaSuccess;
    cudaError_t e;
    if ((e = cudaMalloc(&chit, sizeof(double) * 3 * g.kvol))) return e;
    if ((e = cudaMalloc(&pp, sizeof(float) * 3 * g.kvol))) return e;
    if ((e = cudaMalloc(&phi, sizeof(double2) * g.kferm))) return e;
    if ((e = cudaMalloc(&gauss, sizeof(float) * 16 * (size_t)g.kvol * g.Ls))) return e;
    if ((e = cudaMalloc(&walls, sizeof(double2) * 8 * (size_t)g.kvol))) return e;
    return cudaSuccess;
}

}  // namespace chdwf

#define CTX_OR_BAD(ctx)                          \
    Ctx* c = reinterpret_cast<Ctx*>(ctx);        \
    if (!c) return CHDWF_BAD_ARG;                \
    cudaSetDevice(c->device);                    \
    {                                            \
        cudaError_t e0 = c->ensure_traj();       \
        if (e0) return c->status_of(e0, "traj"); \
    }

static int traj_solver_status(Ctx* c, cudaError_t e, int st, const char* where) {
    if (e) return c->status_of(e, where);
    if (st == 1) { c->err = std::string(where) + ": iteration cap reached"; return CHDWF_ITER_CAP; }
    if (st == 2) { c->err = std::string(where) + ": non-finite value"; return CHDWF_NONFINITE; }
    return CHDWF_OK;
}

extern "C" {

int chdwf_traj_set_remez(chdwf_ctx* ctx, int which, const double* anum, const double* aden,
                         const double* bnum, const double* bden, int ndiag) {
    CTX_OR_BAD(ctx);
    if (!anum || !aden || !bnum || !bden || ndiag < 1 || ndiag > kMaxPoles) return CHDWF_BAD_ARG;
    RemezSet* r = which == 2 ? &c->rz2 : which == 4 ? &c->rz4 : which == 22 ? &c->rz2g : nullptr;
    if (!r) return CHDWF_BAD_ARG;
    r->n = ndiag;
    r->anum.assign(anum, anum + ndiag + 1);
    r->aden.assign(aden, aden + ndiag);
    r->bnum.assign(bnum, bnum + ndiag + 1);
    r->bden.assign(bden, bden + ndiag);
    return CHDWF_OK;
}

int chdwf_traj_set_chi(chdwf_ctx* ctx, const double* chi) {
    CTX_OR_BAD(ctx);
    if (!chi) return CHDWF_BAD_ARG;
    cudaMemcpyAsync(c->chid, chi, sizeof(double) * 3 * c->g.kvol, cudaMemcpyHostToDevice, c->stream);
    return c->status_of(cudaStreamSynchronize(c->stream), "traj_set_chi");
}

int chdwf_traj_get_chi(chdwf_ctx* ctx, double* chi, int trial) {
    CTX_OR_BAD(ctx);
    if (!chi) return CHDWF_BAD_ARG;
    cudaMemcpyAsync(chi, trial ? c->chit : c->chid, sizeof(double) * 3 * c->g.kvol,
                    cudaMemcpyDeviceToHost, c->stream);
    return c->status_of(cudaStreamSynchronize(c->stream), "traj_get_chi");
}

int chdwf_traj_begin(chdwf_ctx* ctx) {            // chit = chi (:213-216)
    CTX_OR_BAD(ctx);
    cudaMemcpyAsync(c->chit, c->chid, sizeof(double) * 3 * c->g.kvol, cudaMemcpyDeviceToDevice,
                    c->stream);
    return c->status_of(cudaGetLastError(), "traj_begin");
}

int chdwf_traj_heatbath(chdwf_ctx* ctx, const float* ps, float res, float am, float hpin, int imass,
                        int* itercg) {
    (void)am;
    CTX_OR_BAD(ctx);
    if (!ps || !itercg || c->rz4.n < 1) return CHDWF_BAD_ARG;
    const size_t n = 16 * (size_t)c->g.kvol * c->g.Ls;
    cudaMemcpyAsync(c->gauss, ps, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream);
    return chdwf_traj_heatbath_dev(ctx, c->gauss, res, am, hpin, imass, itercg);
}

int chdwf_traj_heatbath_dev(chdwf_ctx* ctx, const void* ps_dev, float res, float am, float hpin,
                            int imass, int* itercg) {
    (void)am;
    CTX_OR_BAD(ctx);
    if (!ps_dev || !itercg || c->rz4.n < 1) return CHDWF_BAD_ARG;
    k_build_source<<<nblk(8 * (int64_t)c->g.Ls * c->g.kvol), kThreads, 0, c->stream>>>(
        c->spin[0], (const float*)ps_dev, c->g); count_launches(1);
    launch_round_chi(c->chit, c->chif, c->g.kvol, c->stream);
    int st = 0;
    // Phi = (M^dagger M)^(1/4) R with the remez4 a-coefficients (:233), Phi <- X1 (:237-245)
    cudaError_t e = lz_solve(c->lz, c->g, c->spin[0], res, c->rz4.n, c->rz4.anum.data(),
                             c->rz4.aden.data(), 0, c->chif, c->am3, hpin, imass, c->ibound,
                             c->phi, c->dS, itercg, &st, &c->last_lz, c->stream, c->prec_accept);
    return traj_solver_status(c, e, st, "heatbath");
}

int chdwf_traj_set_momenta(chdwf_ctx* ctx, const float* pp) {
    CTX_OR_BAD(ctx);
    if (!pp) return CHDWF_BAD_ARG;
    cudaMemcpyAsync(c->pp, pp, sizeof(float) * 3 * c->g.kvol, cudaMemcpyHostToDevice, c->stream);
    return c->status_of(cudaGetLastError(), "traj_set_momenta");
}

int chdwf_traj_set_momenta_dev(chdwf_ctx* ctx, const void* pp_dev) {
    CTX_OR_BAD(ctx);
    if (!pp_dev) return CHDWF_BAD_ARG;
    cudaMemcpyAsync(c->pp, pp_dev, sizeof(float) * 3 * c->g.kvol, cudaMemcpyDeviceToDevice,
                    c->stream);
    return c->status_of(cudaGetLastError(), "traj_set_momenta_dev");
}

int chdwf_traj_get_momenta(chdwf_ctx* ctx, float* pp) {
    CTX_OR_BAD(ctx);
    if (!pp) return CHDWF_BAD_ARG;
    cudaMemcpyAsync(pp, c->pp, sizeof(float) * 3 * c->g.kvol, cudaMemcpyDeviceToHost, c->stream);
    return c->status_of(cudaStreamSynchronize(c->stream), "traj_get_momenta");
}

int chdwf_traj_get_force(chdwf_ctx* ctx, float* dSdchi) {
    CTX_OR_BAD(ctx);
    if (!dSdchi) return CHDWF_BAD_ARG;
    cudaMemcpyAsync(dSdchi, c->dS, sizeof(float) * 3 * c->g.kvol, cudaMemcpyDeviceToHost, c->stream);
    return c->status_of(cudaStreamSynchronize(c->stream), "traj_get_force");
}

int chdwf_traj_get_phi(chdwf_ctx* ctx, double* Phi) {
    CTX_OR_BAD(ctx);
    if (!Phi) return CHDWF_BAD_ARG;
    cudaMemcpyAsync(Phi, c->phi, sizeof(double2) * c->g.kferm, cudaMemcpyDeviceToHost, c->stream);
    return c->status_of(cudaStreamSynchronize(c->stream), "traj_get_phi");
}

int chdwf_traj_hamilton(chdwf_ctx* ctx, float res2, float am, float hpin, int imass, double* out,
                        int* itercg) {
    (void)am;
    CTX_OR_BAD(ctx);
    if (!out || !itercg || c->rz2.n < 1) return CHDWF_BAD_ARG;
    launch_round_chi(c->chit, c->chif, c->g.kvol, c->stream);
    k_hamilton_bos<<<1, kThreads, 0, c->stream>>>(c->pp, c->chit, 3 * c->g.kvol, c->red + 16); count_launches(1);
    int st = 0;
    cudaError_t e = lz_solve(c->lz, c->g, c->phi, res2, c->rz2.n, c->rz2.bnum.data(),
                             c->rz2.bden.data(), 0, c->chif, c->am3, hpin, imass, c->ibound,
                             c->spin[1], c->dS, itercg, &st, &c->last_lz, c->stream, c->prec_accept);   // :572
    if (e) return traj_solver_status(c, e, st, "hamilton");
    launch_redot(c->phi, c->spin[1], c->g.kferm, c->red + 32, c->red, c->stream);          // :578-580
    double h[3];
    cudaMemcpyAsync(h, c->red + 16, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(h + 2, c->red, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    e = cudaStreamSynchronize(c->stream);
    const double hp = h[0] * 0.5, hg = (double)c->beta * h[1], hf = h[2];
    out[0] = hg + hp + hf;
    out[1] = hg;
    out[2] = hp;
    out[3] = hg + hf;
    out[4] = hf;
    return traj_solver_status(c, e, st, "hamilton");
}

int chdwf_traj_force(chdwf_ctx* ctx, float res1, float am, float hpin, int imass, int* itg,
                     int* itf) {
    (void)am;
    CTX_OR_BAD(ctx);
    if (!itg || !itf || c->rz2g.n < 1) return CHDWF_BAD_ARG;
    launch_round_chi(c->chit, c->chif, c->g.kvol, c->stream);
    launch_dsdchi_init(c->chit, 2 * c->beta, c->dS, c->g.kvol, c->stream);       // :494-498
    int st1 = 0, st2 = 0;
    cudaError_t e = lz_solve(c->lz, c->g, c->phi, res1, c->rz2g.n, c->rz2g.bnum.data(),
                             c->rz2g.bden.data(), 0, c->chif, c->am3, hpin, imass, c->ibound,
                             c->spin[1], c->dS, itg, &st1, &c->last_lz, c->stream, c->prec_md);   // :505
    if (e || st1) return traj_solver_status(c, e, st1, "force (guidance solve)");
    e = lz_solve(c->lz, c->g, c->spin[1], res1, c->rz2g.n, c->rz2g.anum.data(),
                 c->rz2g.aden.data(), 1, c->chif, c->am3, hpin, imass, c->ibound, c->spin[2],
                 c->dS, itf, &st2, &c->last_lz, c->stream, c->prec_md);                           // :513
    return traj_solver_status(c, e, st2, "force (force solve)");
}

int chdwf_traj_update_momenta(chdwf_ctx* ctx, float d) {
    CTX_OR_BAD(ctx);
    const int n = 3 * c->g.kvol;
    k_update_p<<<nblk(n), kThreads, 0, c->stream>>>(c->pp, c->dS, d, n); count_launches(1);
    return c->status_of(cudaGetLastError(), "traj_update_momenta");
}

int chdwf_traj_update_chi(chdwf_ctx* ctx, float d) {
    CTX_OR_BAD(ctx);
    const int n = 3 * c->g.kvol;
    k_update_chi<<<nblk(n), kThreads, 0, c->stream>>>(c->chit, c->pp, d, n); count_launches(1);
    return c->status_of(cudaGetLastError(), "traj_update_chi");
}

int chdwf_traj_accept(chdwf_ctx* ctx) {           // chi = chit (:337-341)
    CTX_OR_BAD(ctx);
    cudaMemcpyAsync(c->chid, c->chit, sizeof(double) * 3 * c->g.kvol, cudaMemcpyDeviceToDevice,
                    c->stream);
    return c->status_of(cudaGetLastError(), "traj_accept");
}

int chdwf_traj_sync(chdwf_ctx* ctx) {
    CTX_OR_BAD(ctx);
    return c->status_of(cudaStreamSynchronize(c->stream), "traj_sync");
}

int chdwf_traj_propagator(chdwf_ctx* ctx, int ittt, int idsource, float res, float am, float hpin,
                          int imass, double* walls, int* itercg) {
    (void)am;
    CTX_OR_BAD(ctx);
    if (!walls || !itercg || ittt < 1 || ittt > c->g.Lt || idsource < 1 || idsource > 4)
        return CHDWF_BAD_ARG;
    const Geom& g = c->g;
    const int64_t ksize2 = (int64_t)g.L * g.L;
    double2* xi = c->spin[0];
    double2* Phi = c->spin[1];
    cudaMemsetAsync(xi, 0, sizeof(double2) * g.kferm, c->stream);                 // :945-953
    const double val = (double)(1.0f / (float)ksize2);                             // :961
    k_wall_source<<<nblk(ksize2), kThreads, 0, c->stream>>>(xi, g, (int64_t)(ittt - 1) * ksize2,
                                                             idsource, val); count_launches(1);
    launch_round_chi(c->chit, c->chif, g.kvol, c->stream);
    launch_dslash64(true, imass, Phi, xi, c->chif, g, c->am3, hpin, c->ibound, c->stream);  // :979
    cudaMemcpyAsync(xi, Phi, sizeof(double2) * g.kferm, cudaMemcpyDeviceToDevice, c->stream);  // :983-991
    int st = 0;
    cudaError_t e = cg_solve(c->cg, g, Phi, res, c->chif, c->am3, hpin, imass, c->ibound, xi,
                             itercg, &st, c->stream);                              // :996
    if (e) return traj_solver_status(c, e, st, "propagator");
    if (st == 1) fprintf(stdout, " # iterations of congrad exceeds niterc\n");
    k_extract_walls<<<nblk(8 * (int64_t)g.kvol), kThreads, 0, c->stream>>>(xi, g, c->walls); count_launches(1);
    cudaMemcpyAsync(walls, c->walls, sizeof(double2) * 8 * g.kvol, cudaMemcpyDeviceToHost, c->stream);
    e = cudaStreamSynchronize(c->stream);
    return traj_solver_status(c, e, st, "propagator");
}

int chdwf_traj_propagators(chdwf_ctx* ctx, int nsrc, const int* ittt, const int* idsource,
                           float res, float am, float hpin, int imass, double* walls,
                           int* itercg) {
    (void)am;
    CTX_OR_BAD(ctx);
    const Geom& g = c->g;
    if (nsrc < 1 || !ittt || !idsource || !walls || !itercg) return CHDWF_BAD_ARG;
    for (int i = 0; i < nsrc; i++)
        if (ittt[i] < 1 || ittt[i] > g.Lt || idsource[i] < 1 || idsource[i] > 4)
            return CHDWF_BAD_ARG;
    if (nsrc > c->prop_cap) {
        cudaFree(c->prop_x);
        cudaFree(c->prop_phi);
        c->prop_x = c->prop_phi = nullptr;
        c->prop_cap = 0;
        cudaError_t e;
        if ((e = cudaMalloc(&c->prop_x, sizeof(double2) * g.kferm * nsrc)) ||
            (e = cudaMalloc(&c->prop_phi, sizeof(double2) * g.kferm * nsrc)))
            return c->status_of(e, "propagators");
        c->prop_cap = nsrc;
    }
    const int64_t ksize2 = (int64_t)g.L * g.L;
    const double val = (double)(1.0f / (float)ksize2);                             // :961
    launch_round_chi(c->chit, c->chif, g.kvol, c->stream);
    std::vector<chdwf_cg_system> sys(nsrc);
    for (int i = 0; i < nsrc; i++) {
        double2* xi = c->prop_x + g.kferm * i;
        double2* Phi = c->prop_phi + g.kferm * i;
        cudaMemsetAsync(xi, 0, sizeof(double2) * g.kferm, c->stream);             // :945-953
        k_wall_source<<<nblk(ksize2), kThreads, 0, c->stream>>>(
            xi, g, (int64_t)(ittt[i] - 1) * ksize2, idsource[i], val);
        count_launches(1);
        launch_dslash64(true, imass, Phi, xi, c->chif, g, c->am3, hpin, c->ibound,
                        c->stream);                                                // :979
        cudaMemcpyAsync(xi, Phi, sizeof(double2) * g.kferm, cudaMemcpyDeviceToDevice,
                        c->stream);                                                // :983-991
        sys[i] = chdwf_cg_system{g.L, g.Lt, g.Ls, imass, hpin, c->am3, c->ibound, Phi, xi,
                                 c->chit};
    }
    std::vector<int> status(nsrc);
    int rc = chdwf_congrad_batch(ctx, sys.data(), nsrc, res, itercg, status.data());   // :996
    if (rc != CHDWF_OK && rc != CHDWF_ITER_CAP) return rc;
    for (int i = 0; i < nsrc; i++) {
        if (status[i] == CHDWF_ITER_CAP) fprintf(stdout, " # iterations of congrad exceeds niterc\n");
        k_extract_walls<<<nblk(8 * (int64_t)g.kvol), kThreads, 0, c->stream>>>(
            c->prop_x + g.kferm * i, g, c->walls);
        count_launches(1);
        cudaMemcpyAsync(walls + (size_t)16 * g.kvol * i, c->walls, sizeof(double2) * 8 * g.kvol,
                        cudaMemcpyDeviceToHost, c->stream);
    }
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e) return c->status_of(e, "propagators");
    return rc;
}

int chdwf_traj_noise_solve(chdwf_ctx* ctx, const float* eta, int swall, int idirac, float res,
                           float am, float hpin, int imass, double* slice, int* itercg) {
    (void)am;
    CTX_OR_BAD(ctx);
    const Geom& g = c->g;
    if (!eta || !slice || !itercg || (swall != 1 && swall != g.Ls) || idirac < 1 || idirac > 4 ||
        (imass != 1 && imass != 3))
        return CHDWF_BAD_ARG;
    double2* xi = c->spin[0];
    double2* Phi = c->spin[1];
    float* eta_d = c->gauss;                       // heatbath scratch, free between sweeps
    cudaMemcpyAsync(eta_d, eta, sizeof(float) * 2 * g.kvol, cudaMemcpyHostToDevice, c->stream);
    cudaMemsetAsync(xi, 0, sizeof(double2) * g.kferm, c->stream);
    k_noise_source<<<nblk(2 * (int64_t)g.kvol), kThreads, 0, c->stream>>>(
        xi, g, eta_d, swall - 1, idirac - 1); count_launches(1);
    launch_round_chi(c->chit, c->chif, g.kvol, c->stream);
    launch_dslash64(true, imass, Phi, xi, c->chif, g, c->am3, hpin, c->ibound, c->stream);  // :1273
    cudaMemcpyAsync(xi, Phi, sizeof(double2) * g.kferm, cudaMemcpyDeviceToDevice, c->stream);  // :1277-1282
    int st = 0;
    cudaError_t e = cg_solve(c->cg, g, Phi, res, c->chif, c->am3, hpin, imass, c->ibound, xi,
                             itercg, &st, c->stream);                              // :1284
    if (e) return traj_solver_status(c, e, st, "noise solve");
    if (st == 1) fprintf(stdout, " # iterations of congrad exceeds niterc\n");
    const int sread = swall == 1 ? g.Ls - 1 : 0;
    k_extract_slice<<<nblk(2 * (int64_t)g.kvol), kThreads, 0, c->stream>>>(
        xi, g, sread, idirac - 1, c->walls); count_launches(1);
    cudaMemcpyAsync(slice, c->walls, sizeof(double2) * 2 * g.kvol, cudaMemcpyDeviceToHost,
                    c->stream);
    e = cudaStreamSynchronize(c->stream);
    return traj_solver_status(c, e, st, "noise solve");
}

}  // extern "C"
