// api.cu -- the C ABI (include/chdwf.h): device context and the routine-level
// replacements of dslash, dslashd, qmrherm, derivs, congrad, force, hamilton.
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/chdwf.h"
#include "cg.h"
#include "ctx.h"
#include "lanczos.h"

using namespace chdwf;

namespace chdwf {

bool Ctx::fail(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return false;
    err = std::string(where) + ": " + cudaGetErrorString(e);
    return true;
}

int Ctx::status_of(cudaError_t e, const char* where) {
    if (e == cudaSuccess) e = cudaGetLastError();
    if (fail(e, where)) return CHDWF_CUDA_ERROR;
    return CHDWF_OK;
}

cudaError_t Ctx::ensure_fields() {
    if (spin[0]) return cudaSuccess;
    cudaError_t e;
    for (int i = 0; i < kSpin; i++)
        if ((e = cudaMalloc(&spin[i], sizeof(double2) * g.kferm))) return e;
    if ((e = cudaMalloc(&chid, sizeof(double) * 3 * g.kvol))) return e;
    if ((e = cudaMalloc(&chif, sizeof(float) * 3 * g.kvol))) return e;
    if ((e = cudaMalloc(&dS, sizeof(float) * 3 * g.kvol))) return e;
    if ((e = cudaMalloc(&red, sizeof(double) * 4096))) return e;
    return cudaSuccess;
}

Ctx::~Ctx() {
    cudaSetDevice(device);
    lz.release();
    cg.release();
    free_batch(batch);
    for (int i = 0; i < kSpin; i++)
        if (spin[i]) cudaFree(spin[i]);
    if (chid) cudaFree(chid);
    if (chif) cudaFree(chif);
    if (dS) cudaFree(dS);
    if (red) cudaFree(red);
    if (chit) cudaFree(chit);
    if (pp) cudaFree(pp);
    if (phi_slot[0] == nullptr && phi) phi_slot[0] = phi;   // field 0 is phi
    for (int i = 0; i < kMaxPf; i++)
        if (phi_slot[i]) cudaFree(phi_slot[i]);
    if (gauss) cudaFree(gauss);
    if (prop_x) cudaFree(prop_x);
    if (prop_phi) cudaFree(prop_phi);
    if (walls) cudaFree(walls);
    if (stream) cudaStreamDestroy(stream);
}

// Upload a host chi (kvol,3) real*8 and its REAL*4-rounded copy.
cudaError_t Ctx::upload_chi(const double* chi_host) {
    cudaError_t e = cudaMemcpyAsync(chid, chi_host, sizeof(double) * 3 * g.kvol,
                                    cudaMemcpyHostToDevice, stream);
    if (e) return e;
    launch_round_chi(chid, chif, g.kvol, stream);
    return cudaGetLastError();
}

}  // namespace chdwf

static thread_local std::string g_create_err;

extern "C" {

const char* chdwf_version(void) { return "chdwf-b200 0.1 (sm_100a)"; }

int chdwf_timing(chdwf_ctx* ctx, int enable) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c) return CHDWF_BAD_ARG;
    cudaSetDevice(c->device);
    if (enable < 0 || enable > 2) return CHDWF_BAD_ARG;
    if (enable) {
        c->lz.timer.enable();
        c->lz.timer.reset();
        c->lz.timer.chunks = enable == 2;
    } else {
        c->lz.timer.release();
    }
    return c->status_of(cudaGetLastError(), "timing");
}

int chdwf_timing_read_chunks(chdwf_ctx* ctx, double* us_per_iter, long long* iters) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !us_per_iter || !iters) return CHDWF_BAD_ARG;
    for (int k = 0; k < 2; k++) {
        iters[k] = c->lz.timer.chunk_iters[k];
        us_per_iter[k] = iters[k] > 0 ? 1e3 * c->lz.timer.chunk_ms[k] / (double)iters[k] : 0.0;
    }
    return CHDWF_OK;
}

long long chdwf_kernel_launches(void) { return launches_total(); }

int chdwf_stencil_launches(long long* counts) {
    if (!counts) return CHDWF_BAD_ARG;
    for (int k = 0; k < 3; k++) counts[k] = stencil_launches(k);
    return CHDWF_OK;
}

int chdwf_set_precision(chdwf_ctx* ctx, int md, int accept) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || md < 0 || md > 1 || accept < 0 || accept > 1) return CHDWF_BAD_ARG;
    c->prec_md = md;
    c->prec_accept = accept;
    return CHDWF_OK;
}

int chdwf_set_basis_store(chdwf_ctx* ctx, double max_bytes) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c) return CHDWF_BAD_ARG;
    cudaSetDevice(c->device);
    c->lz.basis_enabled = max_bytes != 0.0;
    c->lz.basis_max_bytes = max_bytes;
    // drop the current store; the next solve allocates within the new limit
    if (c->lz.basis) cudaFree(c->lz.basis);
    if (c->lz.basis32) cudaFree(c->lz.basis32);
    if (c->lz.wall) cudaFree(c->lz.wall);
    if (c->lz.wall32) cudaFree(c->lz.wall32);
    c->lz.basis = nullptr;
    c->lz.basis32 = nullptr;
    c->lz.wall = nullptr;
    c->lz.wall32 = nullptr;
    c->lz.hcap = c->lz.hcap32 = 0;
    c->lz.wcap = c->lz.wcap32 = 0;
    return c->status_of(cudaGetLastError(), "set_basis_store");
}

void* chdwf_get_stream(chdwf_ctx* ctx) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    return c ? (void*)c->stream : nullptr;
}

int chdwf_timing_read(chdwf_ctx* ctx, double* ms, long long* timed, long long* launched,
                      double* bytes) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !ms || !timed || !launched || !bytes) return CHDWF_BAD_ARG;
    for (int k = 0; k < KernelTimer::kClasses; k++) {
        ms[k] = c->lz.timer.total_ms[k];
        bytes[k] = c->lz.timer.total_bytes[k];
        timed[k] = c->lz.timer.count[k];
        launched[k] = c->lz.timer.launches[k];
    }
    return CHDWF_OK;
}

int chdwf_create(chdwf_ctx** out, int ksize, int ksizet, int kthird, int device) {
    if (!out) return CHDWF_BAD_ARG;
    *out = nullptr;
    if (!geom_ok(ksize, ksizet, kthird)) return CHDWF_BAD_ARG;
    cudaError_t e = cudaSetDevice(device);
    if (e) { g_create_err = cudaGetErrorString(e); return CHDWF_CUDA_ERROR; }
    Ctx* c = new Ctx();
    c->device = device;
    c->g = make_geom(ksize, ksizet, kthird);
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) ||
        (e = c->ensure_fields())) {
        g_create_err = cudaGetErrorString(e);
        delete c;
        return CHDWF_CUDA_ERROR;
    }
    *out = reinterpret_cast<chdwf_ctx*>(c);
    return CHDWF_OK;
}

void chdwf_destroy(chdwf_ctx* ctx) { delete reinterpret_cast<Ctx*>(ctx); }

int chdwf_set_para(chdwf_ctx* ctx, float beta, float am3, int ibound) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c) return CHDWF_BAD_ARG;
    c->beta = beta;
    c->am3 = am3;
    c->ibound = ibound;
    return CHDWF_OK;
}

const char* chdwf_last_error(const chdwf_ctx* ctx) {
    const Ctx* c = reinterpret_cast<const Ctx*>(ctx);
    if (!c) return g_create_err.c_str();
    return c->err.c_str();
}

static int dslash_host(Ctx* c, double* Phi, const double* R, const double* chi, float hpin,
                       int imass, bool dag) {
    if (!Phi || !R || !chi) return CHDWF_BAD_ARG;
    cudaSetDevice(c->device);
    const size_t bytes = sizeof(double2) * c->g.kferm;
    cudaError_t e;
    if ((e = c->upload_chi(chi))) return c->status_of(e, "dslash: chi upload");
    if ((e = cudaMemcpyAsync(c->spin[0], R, bytes, cudaMemcpyHostToDevice, c->stream)))
        return c->status_of(e, "dslash: R upload");
    launch_dslash64(dag, imass, c->spin[1], c->spin[0], c->chif, c->g, c->am3, hpin, c->ibound,
                    c->stream);
    if ((e = cudaMemcpyAsync(Phi, c->spin[1], bytes, cudaMemcpyDeviceToHost, c->stream)))
        return c->status_of(e, "dslash: Phi download");
    return c->status_of(cudaStreamSynchronize(c->stream), "dslash");
}

int chdwf_dslash(chdwf_ctx* ctx, double* Phi, const double* R, const double* chi, float am,
                 float hpin, int imass) {
    (void)am;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c) return CHDWF_BAD_ARG;
    return dslash_host(c, Phi, R, chi, hpin, imass, false);
}

int chdwf_dslashd(chdwf_ctx* ctx, double* Phi, const double* R, const double* chi, float am,
                  float hpin, int imass) {
    (void)am;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c) return CHDWF_BAD_ARG;
    return dslash_host(c, Phi, R, chi, hpin, imass, true);
}

int chdwf_dslash_dev(chdwf_ctx* ctx, void* Phi, const void* R, const void* chi, float hpin,
                     int imass, int dagger, void* stream) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !Phi || !R || !chi) return CHDWF_BAD_ARG;
    cudaSetDevice(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    launch_round_chi((const double*)chi, c->chif, c->g.kvol, st);
    launch_dslash64(dagger != 0, imass, (double2*)Phi, (const double2*)R, c->chif, c->g, c->am3,
                    hpin, c->ibound, st);
    return c->status_of(cudaGetLastError(), "dslash_dev");
}

int chdwf_dslash_dev_lp(chdwf_ctx* ctx, void* Phi, const void* R, const void* chi, float hpin,
                        int imass, int dagger, int prec, void* stream) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !Phi || !R || !chi || (prec != 1 && prec != 2)) return CHDWF_BAD_ARG;
    cudaSetDevice(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    launch_round_chi((const double*)chi, c->chif, c->g.kvol, st);
    launch_dslash_lp(dagger != 0, imass, prec == 2, Phi, R, c->chif, c->g, c->am3, hpin, c->ibound,
                     st);
    return c->status_of(cudaGetLastError(), "dslash_dev_lp");
}

static int solver_status(Ctx* c, cudaError_t e, int st, const char* where) {
    if (e) return c->status_of(e, where);
    if (st == 1) { c->err = std::string(where) + ": iteration cap reached"; return CHDWF_ITER_CAP; }
    if (st == 2) { c->err = std::string(where) + ": non-finite value"; return CHDWF_NONFINITE; }
    return CHDWF_OK;
}

int chdwf_qmrherm_dev(chdwf_ctx* ctx, const void* Phi, float res, int* itercg, float hpin,
                      int imass, const double* anum, const double* aden, int ndiag, int iflag,
                      const void* chi, void* x, void* dSdchi) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !Phi || !itercg || !anum || !aden || !chi || !x) return CHDWF_BAD_ARG;
    if (ndiag < 1 || ndiag > kMaxPoles || (iflag == 1 && !dSdchi)) return CHDWF_BAD_ARG;
    cudaSetDevice(c->device);
    launch_round_chi((const double*)chi, c->chif, c->g.kvol, c->stream);
    int st = 0;
    cudaError_t e = lz_solve(c->lz, c->g, (const double2*)Phi, res, ndiag, anum, aden, iflag,
                             c->chif, c->am3, hpin, imass, c->ibound, (double2*)x,
                             (float*)dSdchi, itercg, &st, &c->last_lz, c->stream);
    if (!e) e = cudaStreamSynchronize(c->stream);
    return solver_status(c, e, st, "qmrherm");
}

int chdwf_qmrherm(chdwf_ctx* ctx, const double* Phi, float res, int* itercg, float am,
                  float hpin, int imass, const double* anum, const double* aden, int ndiag,
                  int iflag, const double* chi, double* x, float* dSdchi) {
    (void)am;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !Phi || !x || !chi) return CHDWF_BAD_ARG;
    if (iflag == 1 && !dSdchi) return CHDWF_BAD_ARG;
    cudaSetDevice(c->device);
    const size_t bytes = sizeof(double2) * c->g.kferm;
    cudaError_t e;
    if ((e = c->upload_chi(chi))) return c->status_of(e, "qmrherm: chi upload");
    if ((e = cudaMemcpyAsync(c->spin[0], Phi, bytes, cudaMemcpyHostToDevice, c->stream)))
        return c->status_of(e, "qmrherm: Phi upload");
    if (iflag == 1 &&
        (e = cudaMemcpyAsync(c->dS, dSdchi, sizeof(float) * 3 * c->g.kvol, cudaMemcpyHostToDevice,
                             c->stream)))
        return c->status_of(e, "qmrherm: dSdchi upload");
    int st = 0;
    e = lz_solve(c->lz, c->g, c->spin[0], res, ndiag, anum, aden, iflag, c->chif, c->am3, hpin,
                 imass, c->ibound, c->spin[1], c->dS, itercg, &st, &c->last_lz, c->stream);
    if (e) return solver_status(c, e, st, "qmrherm");
    cudaMemcpyAsync(x, c->spin[1], bytes, cudaMemcpyDeviceToHost, c->stream);
    if (iflag == 1)
        cudaMemcpyAsync(dSdchi, c->dS, sizeof(float) * 3 * c->g.kvol, cudaMemcpyDeviceToHost,
                        c->stream);
    e = cudaStreamSynchronize(c->stream);
    return solver_status(c, e, st, "qmrherm");
}

int chdwf_derivs(chdwf_ctx* ctx, const double* R, const double* X2, double anum, int imass,
                 float* dSdchi) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !R || !X2 || !dSdchi) return CHDWF_BAD_ARG;
    cudaSetDevice(c->device);
    const size_t bytes = sizeof(double2) * c->g.kferm;
    cudaMemcpyAsync(c->spin[0], R, bytes, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(c->spin[1], X2, bytes, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(c->dS, dSdchi, sizeof(float) * 3 * c->g.kvol, cudaMemcpyHostToDevice, c->stream);
    launch_derivs_full(c->spin[0], c->spin[1], anum, imass, c->dS, c->g, c->stream);
    cudaMemcpyAsync(dSdchi, c->dS, sizeof(float) * 3 * c->g.kvol, cudaMemcpyDeviceToHost, c->stream);
    return c->status_of(cudaStreamSynchronize(c->stream), "derivs");
}

int chdwf_congrad_dev(chdwf_ctx* ctx, const void* Phi, float res, int* itercg, float hpin,
                      int imass, const void* chi, void* x) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !Phi || !itercg || !chi || !x) return CHDWF_BAD_ARG;
    cudaSetDevice(c->device);
    launch_round_chi((const double*)chi, c->chif, c->g.kvol, c->stream);
    int st = 0;
    cudaError_t e = cg_solve(c->cg, c->g, (const double2*)Phi, res, c->chif, c->am3, hpin, imass,
                             c->ibound, (double2*)x, itercg, &st, c->stream);
    if (st == 1) {
        // the reference prints this line to units 6 and 7 (rhmc/cheisdwf.f:1151-1153)
        fprintf(stdout, " # iterations of congrad exceeds niterc\n");
    }
    return solver_status(c, e, st, "congrad");
}

int chdwf_congrad(chdwf_ctx* ctx, const double* Phi, float res, int* itercg, float am,
                  float hpin, int imass, const double* chi, double* x) {
    (void)am;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !Phi || !x || !chi || !itercg) return CHDWF_BAD_ARG;
    cudaSetDevice(c->device);
    const size_t bytes = sizeof(double2) * c->g.kferm;
    cudaError_t e;
    if ((e = c->upload_chi(chi))) return c->status_of(e, "congrad: chi upload");
    cudaMemcpyAsync(c->spin[0], Phi, bytes, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(c->spin[1], x, bytes, cudaMemcpyHostToDevice, c->stream);
    int st = 0;
    e = cg_solve(c->cg, c->g, c->spin[0], res, c->chif, c->am3, hpin, imass, c->ibound,
                 c->spin[1], itercg, &st, c->stream);
    if (e) return solver_status(c, e, st, "congrad");
    if (st == 1) fprintf(stdout, " # iterations of congrad exceeds niterc\n");
    cudaMemcpyAsync(x, c->spin[1], bytes, cudaMemcpyDeviceToHost, c->stream);
    e = cudaStreamSynchronize(c->stream);
    return solver_status(c, e, st, "congrad");
}

int chdwf_force(chdwf_ctx* ctx, const double* Phi, float res1, float am, float hpin, int imass,
                const double* chi, const double* anum, const double* aden, const double* bnum,
                const double* bden, int ndiag, float* dSdchi, double* x, int* itg, int* itf) {
    (void)am;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !Phi || !chi || !anum || !aden || !bnum || !bden || !dSdchi || !x || !itg || !itf)
        return CHDWF_BAD_ARG;
    cudaSetDevice(c->device);
    const size_t bytes = sizeof(double2) * c->g.kferm;
    cudaError_t e;
    if ((e = c->upload_chi(chi))) return c->status_of(e, "force: chi upload");
    cudaMemcpyAsync(c->spin[0], Phi, bytes, cudaMemcpyHostToDevice, c->stream);
    launch_dsdchi_init(c->chid, 2 * c->beta, c->dS, c->g.kvol, c->stream);      // :494-498
    int st1 = 0, st2 = 0;
    e = lz_solve(c->lz, c->g, c->spin[0], res1, ndiag, bnum, bden, 0, c->chif, c->am3, hpin, imass,
                 c->ibound, c->spin[1], c->dS, itg, &st1, nullptr, c->stream);  // :505
    if (e) return solver_status(c, e, st1, "force (guidance solve)");
    e = lz_solve(c->lz, c->g, c->spin[1], res1, ndiag, anum, aden, 1, c->chif, c->am3, hpin, imass,
                 c->ibound, c->spin[2], c->dS, itf, &st2, nullptr, c->stream);  // :513
    if (e) return solver_status(c, e, st2, "force (force solve)");
    cudaMemcpyAsync(x, c->spin[2], bytes, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(dSdchi, c->dS, sizeof(float) * 3 * c->g.kvol, cudaMemcpyDeviceToHost, c->stream);
    e = cudaStreamSynchronize(c->stream);
    int s = solver_status(c, e, st1, "force (guidance solve)");
    if (s) return s;
    return solver_status(c, e, st2, "force (force solve)");
}

int chdwf_hamilton(chdwf_ctx* ctx, const double* Phi, float res2, float am, float hpin, int imass,
                   const double* chi, const float* pp, const double* bnum, const double* bden,
                   int ndiag, double* out, double* x, int* itercg) {
    (void)am;
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !Phi || !chi || !pp || !bnum || !bden || !out || !x || !itercg) return CHDWF_BAD_ARG;
    cudaSetDevice(c->device);
    const int kvol = c->g.kvol;
    // hp and hg are O(kvol) host sums in the reference's order and types
    // (rhmc/cheisdwf.f:546-559): REAL*4 products summed in REAL*8.
    double hp = 0.0, hg = 0.0;
    for (int a = 0; a < 3; a++)
        for (int i = 0; i < kvol; i++) hp = hp + (double)(pp[i + kvol * a] * pp[i + kvol * a]);
    hp = hp * 0.5;
    for (int a = 0; a < 3; a++)
        for (int i = 0; i < kvol; i++) hg = hg + chi[i + kvol * a] * chi[i + kvol * a];
    hg = (double)c->beta * hg;
    const size_t bytes = sizeof(double2) * c->g.kferm;
    cudaError_t e;
    if ((e = c->upload_chi(chi))) return c->status_of(e, "hamilton: chi upload");
    cudaMemcpyAsync(c->spin[0], Phi, bytes, cudaMemcpyHostToDevice, c->stream);
    int st = 0;
    e = lz_solve(c->lz, c->g, c->spin[0], res2, ndiag, bnum, bden, 0, c->chif, c->am3, hpin, imass,
                 c->ibound, c->spin[1], c->dS, itercg, &st, nullptr, c->stream);   // :572
    if (e) return solver_status(c, e, st, "hamilton");
    launch_redot(c->spin[0], c->spin[1], c->g.kferm, c->red + 8, c->red, c->stream);  // :578-580
    double hf = 0.0;
    cudaMemcpyAsync(&hf, c->red, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(x, c->spin[1], bytes, cudaMemcpyDeviceToHost, c->stream);
    e = cudaStreamSynchronize(c->stream);
    out[0] = hg + hp + hf;
    out[1] = hg;
    out[2] = hp;
    out[3] = hg + hf;
    out[4] = hf;
    return solver_status(c, e, st, "hamilton");
}

}  // extern "C"
