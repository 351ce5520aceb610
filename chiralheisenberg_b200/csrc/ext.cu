// ext.cu -- resident blocks of the multi-pseudofermion RHMC variant (no
// counterpart in the reference, which has one pseudofermion; rhmc/cheisdwf.f
// :218-345).
//
// With npf pseudofermion fields the fermion determinant det(M^dag M)^(1/2)
// is split into npf factors det(M^dag M)^(1/(2 npf)), each sampled by its own
// field:
//   heatbath  Phi_i = r_hb(M^dag M) R_i,   r_hb ~ x^(1/(4 npf)),
//             R_i from the same Gaussians as the reference's (gauss0, variance
//             1/2 per component), so S_i = R_i^dag R_i at the start;
//   action    S_i = Re Phi_i^dag r_act(M^dag M) Phi_i,   r_act ~ x^(-1/(2 npf));
//   force     dS_i/dchi from one multi-shift solve with r_act's poles and
//             the per-pole derivs term of the reference's qmrherm(iflag=1)
//             (rhmc/cheisdwf.f:729-742): for r(x) = a0 + sum a_k/(x + sigma_k)
//             the derivative of Phi^dag r(M^dag M) Phi is
//             -sum_k a_k x_k^dag d(M^dag M) x_k, x_k = (M^dag M + sigma_k)^-1 Phi.
// For npf = 1 these are the reference's remez4 (heatbath) and remez2
// (action) functions; its force instead splits (M^dag M)^(-1/2) into a
// guidance solve and a second set (rhmc/cheisdwf.f:470-518), equal in exact
// arithmetic.  The rational sets are made by chiralheisenberg_b200/remez.py.
#include <cstring>
#include <vector>

#include "../../include/chdwf.h"
#include "ctx.h"
#include "lanczos.h"

using namespace chdwf;

namespace chdwf {
// traj.cu: R = cmplx(ps(:,1), ps(:,2)) per gauss0 call, and the bosonic sums
// (hp: pp^2 in REAL*4 products, hg: chi^2) of hamilton
void launch_build_source(double2* R, const float* ps, const Geom& g, cudaStream_t st);
void launch_hamilton_bos(const float* pp, const double* chi, int n, double* out, cudaStream_t st);
}  // namespace chdwf

#define EXT_CTX(ctx)                             \
    Ctx* c = reinterpret_cast<Ctx*>(ctx);        \
    if (!c) return CHDWF_BAD_ARG;                \
    cudaSetDevice(c->device);                    \
    {                                            \
        cudaError_t e0 = c->ensure_traj();       \
        if (e0) return c->status_of(e0, "ext"); \
    }

static int ext_status(Ctx* c, cudaError_t e, int st, const char* where) {
    if (e) return c->status_of(e, where);
    if (st == 1) { c->err = std::string(where) + ": iteration cap reached"; return CHDWF_ITER_CAP; }
    if (st == 2) { c->err = std::string(where) + ": non-finite value"; return CHDWF_NONFINITE; }
    return CHDWF_OK;
}

extern "C" {

int chdwf_ext_set_remez(chdwf_ctx* ctx, int which, const double* num, const double* den, int n) {
    EXT_CTX(ctx);
    if (!num || !den || n < 1 || n > kMaxPoles || (which != 0 && which != 1)) return CHDWF_BAD_ARG;
    RemezSet& r = which == 0 ? c->rz_hb : c->rz_act;
    r.n = n;
    r.anum.assign(num, num + n + 1);
    r.aden.assign(den, den + n);
    return CHDWF_OK;
}

int chdwf_ext_select_pf(chdwf_ctx* ctx, int k) {
    EXT_CTX(ctx);
    if (k < 0 || k >= Ctx::kMaxPf) return CHDWF_BAD_ARG;
    if (!c->phi_slot[0]) c->phi_slot[0] = c->phi;
    if (!c->phi_slot[k]) {
        cudaError_t e = cudaMalloc(&c->phi_slot[k], sizeof(double2) * c->g.kferm);
        if (e) return c->status_of(e, "ext_select_pf");
    }
    c->phi = c->phi_slot[k];
    c->pf = k;
    return CHDWF_OK;
}

int chdwf_ext_heatbath_dev(chdwf_ctx* ctx, const void* ps_dev, float res, float hpin, int imass,
                           int* itercg) {
    EXT_CTX(ctx);
    if (!ps_dev || !itercg || c->rz_hb.n < 1) return CHDWF_BAD_ARG;
    launch_build_source(c->spin[0], (const float*)ps_dev, c->g, c->stream);
    launch_round_chi(c->chit, c->chif, c->g.kvol, c->stream);
    int st = 0;
    cudaError_t e = lz_solve(c->lz, c->g, c->spin[0], res, c->rz_hb.n, c->rz_hb.anum.data(),
                             c->rz_hb.aden.data(), 0, c->chif, c->am3, hpin, imass, c->ibound,
                             c->phi, c->dS, itercg, &st, &c->last_lz, c->stream, c->prec_accept);
    return ext_status(c, e, st, "ext heatbath");
}

int chdwf_ext_action(chdwf_ctx* ctx, float res, float hpin, int imass, double* hf, int* itercg) {
    EXT_CTX(ctx);
    if (!hf || !itercg || c->rz_act.n < 1) return CHDWF_BAD_ARG;
    launch_round_chi(c->chit, c->chif, c->g.kvol, c->stream);
    int st = 0;
    cudaError_t e = lz_solve(c->lz, c->g, c->phi, res, c->rz_act.n, c->rz_act.anum.data(),
                             c->rz_act.aden.data(), 0, c->chif, c->am3, hpin, imass, c->ibound,
                             c->spin[1], c->dS, itercg, &st, &c->last_lz, c->stream,
                             c->prec_accept);
    if (e) return ext_status(c, e, st, "ext action");
    launch_redot(c->phi, c->spin[1], c->g.kferm, c->red + 32, c->red, c->stream);
    cudaMemcpyAsync(hf, c->red, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    e = cudaStreamSynchronize(c->stream);
    return ext_status(c, e, st, "ext action");
}

int chdwf_ext_force(chdwf_ctx* ctx, float res, float hpin, int imass, int init, int* itercg) {
    EXT_CTX(ctx);
    if (!itercg || c->rz_act.n < 1) return CHDWF_BAD_ARG;
    launch_round_chi(c->chit, c->chif, c->g.kvol, c->stream);
    if (init) launch_dsdchi_init(c->chit, 2 * c->beta, c->dS, c->g.kvol, c->stream);
    // qmrherm(iflag=1) with weights a_k adds -X^dag d r(M^dag M) X to dSdchi:
    // in the reference's force, X = r_b(M^dag M) Phi ~ (M^dag M)^(-1/2) Phi and
    // r ~ x^(1/2), and -X^dag d(M^dag M)^(1/2) X is the derivative of
    // Phi^dag (M^dag M)^(-1/2) Phi (rhmc/cheisdwf.f:470-518).  The derivative
    // of Phi^dag r_act(M^dag M) Phi is +Phi^dag d r_act Phi: the same solve
    // with the weights negated.
    std::vector<double> w(c->rz_act.anum);
    for (size_t k = 1; k < w.size(); k++) w[k] = -w[k];
    int st = 0;
    cudaError_t e = lz_solve(c->lz, c->g, c->phi, res, c->rz_act.n, w.data(),
                             c->rz_act.aden.data(), 1, c->chif, c->am3, hpin, imass, c->ibound,
                             c->spin[2], c->dS, itercg, &st, &c->last_lz, c->stream, c->prec_md);
    return ext_status(c, e, st, "ext force");
}

int chdwf_ext_bosonic(chdwf_ctx* ctx, double* hp_hg) {
    EXT_CTX(ctx);
    if (!hp_hg) return CHDWF_BAD_ARG;
    launch_hamilton_bos(c->pp, c->chit, 3 * c->g.kvol, c->red + 16, c->stream);
    double h[2];
    cudaMemcpyAsync(h, c->red + 16, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    hp_hg[0] = 0.5 * h[0];
    hp_hg[1] = (double)c->beta * h[1];
    return c->status_of(e, "ext bosonic");
}

}  // extern "C"
