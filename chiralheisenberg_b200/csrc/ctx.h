// ctx.h -- the device context behind the opaque chdwf_ctx handle.
#pragma once
#include <string>

#include "cg.h"
#include "internal.h"
#include "lanczos.h"

namespace chdwf {

struct BatchWork;                       // batch.cu
void free_batch(BatchWork* w);

// One rational approximation as the reference reads it (rhmc/cheisdwf.f:
// 140-159): anum[0] = a0, anum[1..n], aden = sigma_1..n; same for b.
struct RemezSet {
    int n = 0;
    std::vector<double> anum, aden, bnum, bden;
};

struct Ctx {
    static constexpr int kSpin = 4;
    int device = 0;
    Geom g{};
    cudaStream_t stream = nullptr;
    float beta = 0.0f, am3 = 1.0f;      // /para/
    int ibound = -1;
    double2* spin[kSpin] = {nullptr, nullptr, nullptr, nullptr};   // general spinor slots
    double* chid = nullptr;             // chi (kvol,3) real*8
    float* chif = nullptr;              // chi rounded to REAL*4 for the wall coupling
    float* dS = nullptr;                // dSdchi (kvol,3) REAL*4
    double* red = nullptr;              // reduction scratch
    LzWork lz;
    CgWork cg;
    LzStats last_lz{};
    std::string err;
    // resident trajectory state (traj.cu)
    double* chit = nullptr;             // /trial/ chit
    float* pp = nullptr;                // /trial/ pp (REAL*4)
    double2* phi = nullptr;             // pseudofermion field
    float* gauss = nullptr;             // staging of the heatbath Gaussians
    double2* walls = nullptr;           // propagator wall slices
    RemezSet rz2, rz4, rz2g;
    // multi-pseudofermion variant (ext.cu): fields 1.. beyond phi, and its
    // two rational functions (heatbath: x^(1/(4 npf)); action and force:
    // x^(-1/(2 npf)))
    static constexpr int kMaxPf = 4;
    double2* phi_slot[kMaxPf] = {nullptr, nullptr, nullptr, nullptr};
    int pf = 0;                         // the field phi points to
    RemezSet rz_hb, rz_act;
    int prec_md = 0, prec_accept = 0;   // vector precision of the resident solves
    BatchWork* batch = nullptr;         // workspace of chdwf_congrad_batch
    double2* prop_x = nullptr;          // chdwf_traj_propagators: solutions and
    double2* prop_phi = nullptr;        // right-hand sides of nsrc sources
    int prop_cap = 0;

    ~Ctx();
    bool fail(cudaError_t e, const char* where);
    int status_of(cudaError_t e, const char* where);
    cudaError_t ensure_fields();
    cudaError_t ensure_traj();
    cudaError_t upload_chi(const double* chi_host);
};

}  // namespace chdwf
