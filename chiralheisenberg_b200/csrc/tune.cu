// tune.cu -- the autotuner of the stencil kernels.
//
// The domain-wall operator has three kernel shapes: the point-gather kernels
// (dwf_stencil.cuh: one thread per point and flavour, every neighbour read
// through L1/L2) at a register budget of 80 a thread (3 blocks of 256 a
// SM) or 64 (4 blocks, more warps in flight, some spills), and the
// row-staged kernels (row_stage.cuh: rows y-1..y+1 and t-1, t+1 staged in
// shared memory by bulk copies), where they can launch.  Which is fastest
// depends on the lattice and the precision.  On the first use of a (L, Lt,
// Ls, element size) the tuner applies M in every shape to scratch vectors on
// the caller's stream -- 2 warm-up and 5 timed applications each, CUDA
// events, L2 not flushed (all see the same cache state) -- and keeps the
// fastest, the 3-block point-gather kernel unless another shape is faster
// by more than kTuneMargin (10%).  The choice holds for
// the operator and for the multi-shift solver's pass 1, which use the same
// stencil at the same budgets.  The FP32 solver's Krylov vectors (Ls even)
// are in the split layout, which has point-gather kernels of its own: its
// choice is a separate entry, timed on the split-layout operator
// (stencil_choice_split).  The table is per process; chdwf_autotune_report
// prints it.
#include <cuda_fp16.h>

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/chdwf.h"
#include "internal.h"
#include "row_stage.cuh"

namespace chdwf {
namespace {

struct TuneEntry {
    int L, Lt, Ls, elem, device;
    int choice;
    float us[3];   // per shape (kStencil*), 0 when not timed
    int split;     // the FP32 solver's split-layout kernels
};
const char* shape_name(int k) {
    return k == kStencilRows ? "rows" : (k == kStencilGather4 ? "gather4" : "gather3");
}

// Another shape replaces the 3-block point-gather kernels only when the
// probe (M alone) finds it faster by more than 10%.  The solver's M^dagger
// kernel, the larger of the two, moves the other way: at 24^3x24 the probe
// put 4 blocks a SM within +-5% of 3 (either side, box to box), while the
// solver's M^dagger at 4 blocks took 23% (FP64) and 7% (FP32) longer.
constexpr float kTuneMargin = 0.10f;

std::mutex g_tune_mu;
std::vector<TuneEntry> g_tune;

// median microseconds of 5 applications (after 2) of variant v
float time_variant(const Geom& g, int elem, int v, void* out, const void* in, const float* chif,
                   cudaStream_t st, bool split = false) {
    auto apply = [&] {
        if (split)
            launch_dslash_sp_m((float2*)out, (const float2*)in, chif, g, st, v);
        else if (elem == 16)
            launch_dslash64(false, 1, (double2*)out, (const double2*)in, chif, g, 1.0f, 0.0f, -1,
                            st, v);
        else
            launch_dslash_lp(false, 1, elem == 4 ? 1 : 0, out, in, chif, g, 1.0f, 0.0f, -1, st,
                             v);
    };
    for (int k = 0; k < 2; k++) apply();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<float> ts;
    for (int k = 0; k < 5; k++) {
        cudaEventRecord(e0, st);
        apply();
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        ts.push_back(ms * 1e3f);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::sort(ts.begin(), ts.end());
    return ts[ts.size() / 2];
}

}  // namespace

int stencil_choice(const Geom& g, int elem, cudaStream_t st) {
    const int mode = stencil_mode();
    RowPlan rp;
    const bool rows_fit = row_plan(g, (size_t)elem, &rp);
    if (mode == 1) return kStencilGather3;
    if (mode == 3) return elem == 4 ? kStencilGather3 : kStencilGather4;
    if (mode == 2) return rows_fit && op_rows_launchable(g, elem) ? kStencilRows : kStencilGather3;
    int dev = 0;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        for (const TuneEntry& t : g_tune)
            if (t.L == g.L && t.Lt == g.Lt && t.Ls == g.Ls && t.elem == elem && t.device == dev &&
                !t.split)
                return t.choice;
    }
    // measure on scratch vectors (zeros: the same memory traffic)
    void *in = nullptr, *out = nullptr;
    float* chif = nullptr;
    const size_t bytes = (size_t)elem * g.kferm;
    TuneEntry t{g.L, g.Lt, g.Ls, elem, dev, kStencilGather3, {0.0f, 0.0f, 0.0f}, 0};
    if (cudaMalloc(&in, bytes) == cudaSuccess && cudaMalloc(&out, bytes) == cudaSuccess &&
        cudaMalloc(&chif, sizeof(float) * 3 * (size_t)g.kvol) == cudaSuccess) {
        cudaMemsetAsync(in, 0, bytes, st);
        cudaMemsetAsync(chif, 0, sizeof(float) * 3 * (size_t)g.kvol, st);
        // another shape replaces the point-gather kernel at 3 blocks a SM
        // only if it is faster by more than kTuneMargin
        float best = 0.0f;
        for (int k : {kStencilGather3, kStencilGather4, kStencilRows}) {
            if (k == kStencilRows && !(rows_fit && op_rows_launchable(g, elem))) continue;
            if (k == kStencilGather4 && elem == 4) continue;   // one FP16 gather kernel
            t.us[k] = time_variant(g, elem, k, out, in, chif, st);
            if (best == 0.0f || t.us[k] < best * (1.0f - kTuneMargin)) {
                best = t.us[k];
                t.choice = k;
            }
        }
    }
    cudaGetLastError();
    cudaFree(in);
    cudaFree(out);
    cudaFree(chif);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.push_back(t);
    return t.choice;
}

int stencil_choice_split(const Geom& g, cudaStream_t st) {
    const int mode = stencil_mode();
    if (mode == 1 || mode == 2) return kStencilGather3;
    if (mode == 3) return kStencilGather4;
    int dev = 0;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        for (const TuneEntry& t : g_tune)
            if (t.L == g.L && t.Lt == g.Lt && t.Ls == g.Ls && t.split && t.device == dev)
                return t.choice;
    }
    void *in = nullptr, *out = nullptr;
    float* chif = nullptr;
    const size_t bytes = sizeof(float2) * (size_t)g.kferm;
    TuneEntry t{g.L, g.Lt, g.Ls, 8, dev, kStencilGather3, {0.0f, 0.0f, 0.0f}, 1};
    if (cudaMalloc(&in, bytes) == cudaSuccess && cudaMalloc(&out, bytes) == cudaSuccess &&
        cudaMalloc(&chif, sizeof(float) * 3 * (size_t)g.kvol) == cudaSuccess) {
        cudaMemsetAsync(in, 0, bytes, st);
        cudaMemsetAsync(chif, 0, sizeof(float) * 3 * (size_t)g.kvol, st);
        float best = 0.0f;
        for (int k : {kStencilGather3, kStencilGather4}) {
            t.us[k] = time_variant(g, 8, k, out, in, chif, st, true);
            if (best == 0.0f || t.us[k] < best * (1.0f - kTuneMargin)) {
                best = t.us[k];
                t.choice = k;
            }
        }
    }
    cudaGetLastError();
    cudaFree(in);
    cudaFree(out);
    cudaFree(chif);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.push_back(t);
    return t.choice;
}

}  // namespace chdwf

extern "C" int chdwf_autotune_report(char* buf, int cap) {
    using namespace chdwf;
    std::string s = "[";
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        for (size_t i = 0; i < g_tune.size(); i++) {
            const TuneEntry& t = g_tune[i];
            char line[256];
            snprintf(line, sizeof(line),
                     "%s{\"L\": %d, \"Lt\": %d, \"Ls\": %d, \"elem_bytes\": %d, \"device\": %d, "
                     "\"layout\": \"%s\", \"gather3_us\": %.2f, \"gather4_us\": %.2f, "
                     "\"rows_us\": %.2f, \"choice\": \"%s\"}",
                     i ? ", " : "", t.L, t.Lt, t.Ls, t.elem, t.device, t.split ? "split" : "plain",
                     t.us[kStencilGather3], t.us[kStencilGather4], t.us[kStencilRows],
                     shape_name(t.choice));
            s += line;
        }
    }
    s += "]";
    if (!buf || cap <= 0) return (int)s.size() + 1;
    const int n = (int)s.size() < cap - 1 ? (int)s.size() : cap - 1;
    memcpy(buf, s.data(), n);
    buf[n] = 0;
    return (int)s.size() + 1;
}
