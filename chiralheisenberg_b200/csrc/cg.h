// cg.h -- CGNE propagator solver (congrad replacement).
#pragma once
#include "internal.h"

namespace chdwf {

struct CgCtl {
    int nx, done, iters, niterc;
    float alpha, beta, alphan, betad, resid, pad2_;
    unsigned count1, count2;
};

struct CgArgs {
    Geom g;
    double2 *x, *p, *r, *x1;
    const float* chif;
    double diag, hpin;
    int apbc;
    CgCtl* ctl;
    double* part;
    int* hflag;
};

struct CgWork {
    Geom geom{};
    CgCtl* ctl = nullptr;
    double* part = nullptr;
    double2 *x1 = nullptr, *p = nullptr, *r = nullptr;
    int* hflag_host = nullptr;
    int* hflag_dev = nullptr;
    ~CgWork();
    void release();
    cudaError_t ensure(const Geom& g);
};

// Solves M^dagger M x = Phi starting from x (in/out).  status 0 converged,
// 1 iteration cap (kthird*kvol), 2 non-finite.
cudaError_t cg_solve(CgWork& w, const Geom& g, const double2* phi, float res, const float* chif,
                     float am3, float hpin, int imass, int ibound, double2* x, int* itercg,
                     int* status, cudaStream_t st);

}  // namespace chdwf
