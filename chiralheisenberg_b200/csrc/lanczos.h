// lanczos.h -- two-pass multi-shift Lanczos solver (qmrherm replacement).
#pragma once
#include <vector>

#include "internal.h"
#include "row_stage.cuh"

namespace chdwf {

// Kernel arguments; T is the complex type of the Krylov vectors: double2
// (the FP64 drop-in path) or float2 (mixed precision: FP32 vectors and
// stencil arithmetic, FP64 reductions, scalars and solution accumulation).
template <class T>
struct LzArgsT {
    typedef typename real_of<T>::type Real;
    Geom g;
    T *rb0, *rb1, *rb2;         // Lanczos residual ring: r_j lives in rb[j % 3] ...
    T* basis;                   // ... unless j < hcap: then in basis + j*kferm
    int hcap;
    T* vt;                      // M q_j
    const float* chif;          // chi rounded to REAL*4 (wall coupling)
    Real diag, hpin;
    int apbc;
    LzCtl* ctl;
    LzHist h;
    double* part;               // per-block partial sums
    int* hflag;                 // device view of the mapped host stop flag
    double2* x;                 // solution (iflag 0), FP64
    double2* xw;                // two-slice x_k per pole (iflag 1), FP64
    int npole;
    T* wbasis;                  // force solves: the two wall slices of each r_j,
    int wcap;                   // j < wcap, at wbasis + j*16*kvol (0: no wall store)
    int pl;                     // FP32 vectors in the split layout (cpair; Ls even)
    int rows;                   // pass 1 on the row-staged kernels (plan rp)
    int occ;                    // else the point-gather kernels at 3 or 4 blocks a SM
    RowPlan rp;
};

struct LzStats {
    int iters;
    int pass1_launches;
};

// Optional CUDA-event timing of the solver kernels by class (0: pass-1 M,
// 1: pass-1 M^dagger + update, 2: pass-2 accumulation from the stored basis,
// 3: pass-2 regeneration, M and M^dagger launches), with the algorithmic
// bytes of every timed launch.  Events bracket each launch on the solver's
// stream; durations are summed when the solve synchronises.
struct KernelTimer {
    // classes 0-3 as above for FP64 Krylov vectors, 4-7 the same for FP32
    static constexpr int kClasses = 8;
    static constexpr int kPool = 2 * kMaxIter + 256;
    bool enabled = false;
    cudaEvent_t ev[2 * kPool] = {};
    int cls[kPool] = {};
    double bytes[kPool] = {};
    int used = 0;
    double total_ms[kClasses] = {};
    double total_bytes[kClasses] = {};   // algorithmic bytes moved
    long long count[kClasses] = {};
    long long launches[kClasses] = {};
    void enable();
    void release();
    void begin(int c, cudaStream_t st, double nbytes);   // start event of one launch
    void end(cudaStream_t st);
    void collect();                       // after a synchronisation
    void reset();
    // Chunk mode: pass 1 stays on its graph replays, and events bracket each
    // replayed chunk instead of each launch, so the time per iteration
    // carries no per-launch dispatch.  Only chunks that end at or before the
    // solve's last iteration count.  Per vector precision (0 FP64, 1 FP32).
    static constexpr int kChunkPool = kMaxIter / 16 + 8;
    bool chunks = false;
    cudaEvent_t cev[2 * kChunkPool] = {};
    int cfirst[kChunkPool] = {};
    int cused = 0;
    double chunk_ms[2] = {};
    long long chunk_iters[2] = {};
    void chunk_begin(cudaStream_t st, int first);   // first iteration of the chunk
    void chunk_end(cudaStream_t st);
    void collect_chunks(int m, int chunk, int prec);   // after a synchronisation
};

struct LzGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned char> key;   // the kernel arguments it was captured with
    unsigned nb = 0;
    int imass = 0, chunk = 0;
};

// Side stream of the pass-1 loop: the scalar step of each iteration runs
// there, beside the M^dagger kernel, forked and joined with events.
struct LzSide {
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};

struct LzWork {
    Geom geom{};
    LzSide side;
    LzGraph graph[2][2];              // pass-1 chunk graph per vector precision and
                                      // per basis mode (full vectors / wall slices)
    LzCtl* ctl = nullptr;
    double* hist_mem = nullptr;
    LzHist hist{};
    double* part = nullptr;
    double2* rb[3] = {nullptr, nullptr, nullptr};
    double2* vt = nullptr;
    float2* rb32[3] = {nullptr, nullptr, nullptr};
    float2* vt32 = nullptr;
    // Lanczos basis kept in HBM: pass 2 then reads the stored vectors once
    // instead of regenerating them (2 operator applies per vector)
    double2* basis = nullptr;
    float2* basis32 = nullptr;
    int hcap = 0, hcap32 = 0;
    // Wall store of the force solves: the two wall slices of every Lanczos
    // vector (2/Ls of a vector), all that their pass 2 reads; their pass 1
    // then keeps only the three-vector ring, which stays in L2 for FP32.
    double2* wall = nullptr;
    float2* wall32 = nullptr;
    int wcap = 0, wcap32 = 0;
    int basis_enabled = 1;
    double basis_max_bytes = -1.0;   // per precision; < 0: 40% of the free HBM
    double2* xw = nullptr;
    double2* x2w = nullptr;
    int xw_poles = 0;
    int* hflag_host = nullptr;
    int* hflag_dev = nullptr;
    double2* const* pole_out = nullptr;   // iflag 2: device array of the x_k pointers
    KernelTimer timer;
    ~LzWork();
    void release();
    cudaError_t ensure(const Geom& g, int npole_max, int prec, bool walls);
};

// Precision of the Krylov vectors.
enum { kPrecF64 = 0, kPrecF32 = 1 };

// iflag 0: x = a0 Phi + sum_k a_k x_k; 1: force (see lanczos.cu); 2: every
// x_k into w.pole_out[k] (needs the stored basis; anum unused).
cudaError_t lz_solve(LzWork& w, const Geom& g, const double2* phi, float res, int ndiag,
                     const double* anum, const double* aden, int iflag, const float* chif,
                     float am3, float hpin, int imass, int ibound, double2* x, float* dSdchi,
                     int* itercg, int* status, LzStats* stats, cudaStream_t st,
                     int prec = kPrecF64);

}  // namespace chdwf
