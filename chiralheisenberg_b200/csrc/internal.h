// internal.h -- host-side declarations shared by the CUDA translation units of
// libchdwf (not part of the public C ABI, which is include/chdwf.h).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "common.cuh"

namespace chdwf {

// Number of kernels this library has launched (all contexts); read through
// chdwf_kernel_launches().
void count_launches(long long n);
long long launches_total();
// Operator and pass-1 stencil launches by kernel shape (kStencil*), read
// through chdwf_stencil_launches().
void note_stencil(int shape, long long n);
long long stencil_launches(int shape);

constexpr int kMaxPoles = 32;
constexpr int kMaxIter = 5000;     // niterc of qmrherm (rhmc/cheisdwf.f:603)
constexpr int kThreads = 256;

// Device-resident control block of one multi-shift solve.  Written by the
// last block of each reduction kernel; the iteration index and the buffer
// rotation are read from here so every launch of the loop is identical
// (and therefore capturable in a CUDA graph).
struct LzCtl {
    int it_m;          // iteration j of the next pass-1 M launch (written by M^dagger)
    int it_md;         // iteration j of the next pass-1 M^dagger launch (written by M)
    int done;          // 0 running, 1 converged, 2 iteration cap, 3 non-finite,
                       // 4 a staged copy did not arrive (row kernels)
    int m;             // iteration at which the loop ended
    int npole;
    int niter_cap;
    int pad_;
    double phimod;     // |Phi|
    double thresh;     // arelax*resid, REAL*4 product promoted (cheisdwf.f:711-712)
    double sigma[kMaxPoles];
    double d[kMaxPoles];
    double rho[kMaxPoles];
    double anum[kMaxPoles];    // a_1..a_n (force weights / solution weights)
};

// Per-iteration scalar history (device), sized for kMaxIter iterations.
struct LzHist {
    double* alphat;    // [kMaxIter+2]  alpha~_j
    double* beta;      // [kMaxIter+2]  beta_j (beta_1 = |Phi|)
    double* invbeta;   // [kMaxIter+2]
    double* rho;       // [kMaxPoles][kMaxIter+2]
    double* mu;        // [kMaxPoles][kMaxIter+2]
    double* y;         // [kMaxPoles][kMaxIter+2]  coefficients of q_j in x_k
    double* c;         // [kMaxIter+2]             sum_k a_k y_kj
};

// Operator launchers (FP64, exact evaluation order).
// variant: -1 the tuned choice (stencil_choice), or one of the kStencil*
// shapes below (the row-staged one wherever its shared memory fits).
void launch_dslash64(bool dag, int imass, double2* out, const double2* in, const float* chif,
                     const Geom& g, float am3, float hpin, int ibound, cudaStream_t st,
                     int variant = -1);

// Operator on FP32 (half=0, complex64) or FP16 (half=1, two halves per
// complex) storage with FP32 arithmetic.
void launch_dslash_lp(bool dag, int imass, int half, void* out, const void* in, const float* chif,
                      const Geom& g, float am3, float hpin, int ibound, cudaStream_t st,
                      int variant = -1);

// Stencil kernel shapes: the point-gather kernels with 3 blocks of 256 a SM
// (80 registers a thread) or 4 (64 registers), or the row-staged kernels.
constexpr int kStencilGather3 = 0, kStencilRows = 1, kStencilGather4 = 2;

// Autotuner (tune.cu): the stencil shape for this lattice and element size
// (16: FP64, 8: FP32, 4: FP16 storage).  With CHDWF_STENCIL unset the first
// call for a (L, Lt, Ls, elem) times the operator in every shape on scratch
// vectors on stream st and keeps the fastest; "legacy" forces the
// point-gather kernels at 3 blocks a SM, "rows" the row-staged ones.
int stencil_choice(const Geom& g, int elem, cudaStream_t st);
// The same for the FP32 solver's split-layout vectors (Ls even): the
// point-gather shapes only, timed on the split-layout operator; "rows" and
// "legacy" give the 3-block shape, "gather4" the 4-block one.
int stencil_choice_split(const Geom& g, cudaStream_t st);
// M on split-layout FP32 vectors in a point-gather shape (the tuner's probe).
void launch_dslash_sp_m(float2* out, const float2* in, const float* chif, const Geom& g,
                        cudaStream_t st, int shape);
// Whether the row-staged operator of this element size (16 FP64, 8 FP32,
// 4 FP16 storage) can launch on this lattice and device: its rows fit the
// shared memory and a block fits an SM.
bool op_rows_launchable(const Geom& g, int elem);

// Wall-slice operator for npole stacked two-slice fields (s'=0 <-> s=1,
// s'=1 <-> s=Ls): computes M on the Ls=2 lattice of each pole.
void launch_wall_dslash64(int npole, double2* out, const double2* in, const float* chif,
                          const Geom& g, float am3, float hpin, int ibound, int imass,
                          cudaStream_t st);

// derivs over npole wall fields in pole order into REAL*4 dSdchi.
void launch_derivs_walls(int npole, const double2* xw, const double2* x2w, const double* anum1,
                         int imass, float* dSdchi, const Geom& g, cudaStream_t st);
// derivs of one pole on full fields (the reference routine itself).
void launch_derivs_full(const double2* R, const double2* X2, double anum, int imass,
                        float* dSdchi, const Geom& g, cudaStream_t st);

// small utilities (blas.cu)
void launch_round_chi(const double* chi, float* chif, int kvol, cudaStream_t st);
void launch_dsdchi_init(const double* chi, float twobeta, float* dS, int kvol, cudaStream_t st);
void launch_scale(double2* out, const double2* in, double a, int64_t n, cudaStream_t st);
// sum |v|^2 into *out (device), deterministic
void launch_norm2(const double2* v, int64_t n, double* partials, double* out, cudaStream_t st);
// Re <a, b> into *out
void launch_redot(const double2* a, const double2* b, int64_t n, double* partials, double* out,
                  cudaStream_t st);
int reduce_blocks(int64_t n);

}  // namespace chdwf
