// ctx.h -- the device context behind the opaque chdwf_ctx handle.
#pragma once
#include <string>

#include "cg.h"
#include "internal.h"
#include "lanczos.h"

namespace chdwf {

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

    ~Ctx();
    bool fail(cudaError_t e, const char* where);
    int status_of(cudaError_t e, const char* where);
    cudaError_t ensure_fields();
    cudaError_t upload_chi(const double* chi_host);
};

}  // namespace chdwf
