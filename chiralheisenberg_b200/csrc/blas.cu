// blas.cu -- small field utilities: chi rounding, force initialisation,
// scaling and deterministic reductions.
#include <atomic>

#include "internal.h"

namespace chdwf {

static std::atomic<long long> g_launches{0};
void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launches_total() { return g_launches.load(std::memory_order_relaxed); }

static std::atomic<long long> g_stencil[3];
void note_stencil(int shape, long long n) {
    if (shape >= 0 && shape < 3) g_stencil[shape].fetch_add(n, std::memory_order_relaxed);
}
long long stencil_launches(int shape) {
    return shape >= 0 && shape < 3 ? g_stencil[shape].load(std::memory_order_relaxed) : 0;
}

__global__ void k_round_chi(const double* __restrict__ chi, float* __restrict__ chif, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) chif[i] = (float)chi[i];
}

void launch_round_chi(const double* chi, float* chif, int kvol, cudaStream_t st) {
    const int n = 3 * kvol;
    k_round_chi<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(chi, chif, n); count_launches(1);
}

// dSdchi = 2*beta*chi with 2*beta a REAL*4 product (cheisdwf.f:494-498)
__global__ void k_dsdchi_init(const double* __restrict__ chi, float twob, float* __restrict__ dS,
                              int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dS[i] = (float)__dmul_rn((double)twob, chi[i]);
}

void launch_dsdchi_init(const double* chi, float twobeta, float* dS, int kvol, cudaStream_t st) {
    const int n = 3 * kvol;
    k_dsdchi_init<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(chi, twobeta, dS, n); count_launches(1);
}

__global__ void k_scale(double2* __restrict__ out, const double2* __restrict__ in, double a,
                        int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = zscal(a, in[i]);
}

void launch_scale(double2* out, const double2* in, double a, int64_t n, cudaStream_t st) {
    k_scale<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, st>>>(out, in, a, n); count_launches(1);
}

int reduce_blocks(int64_t n) {
    int64_t nb = (n + kThreads * 4 - 1) / (kThreads * 4);
    if (nb > 1184) nb = 1184;   // 8 blocks per SM on 148 SMs
    if (nb < 1) nb = 1;
    return (int)nb;
}

// Two-stage deterministic reductions: fixed per-thread stride, fixed tree.
__global__ void k_norm2_part(const double2* __restrict__ v, int64_t n, double* __restrict__ part) {
    __shared__ double sh[kThreads / 32];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double2 a = v[i];
        s += a.x * a.x + a.y * a.y;
    }
    s = block_sum<kThreads>(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_redot_part(const double2* __restrict__ a, const double2* __restrict__ b,
                             int64_t n, double* __restrict__ part) {
    __shared__ double sh[kThreads / 32];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double2 x = a[i], y = b[i];
        s += x.x * y.x + x.y * y.y;
    }
    s = block_sum<kThreads>(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_final_sum(const double* __restrict__ part, int nb, double* __restrict__ out) {
    __shared__ double sh[kThreads / 32];
    double s = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) s += part[i];
    s = block_sum<kThreads>(s, sh);
    if (threadIdx.x == 0) *out = s;
}

void launch_norm2(const double2* v, int64_t n, double* partials, double* out, cudaStream_t st) {
    const int nb = reduce_blocks(n);
    k_norm2_part<<<nb, kThreads, 0, st>>>(v, n, partials); count_launches(1);
    k_final_sum<<<1, kThreads, 0, st>>>(partials, nb, out); count_launches(1);
}

void launch_redot(const double2* a, const double2* b, int64_t n, double* partials, double* out,
                  cudaStream_t st) {
    const int nb = reduce_blocks(n);
    k_redot_part<<<nb, kThreads, 0, st>>>(a, b, n, partials); count_launches(1);
    k_final_sum<<<1, kThreads, 0, st>>>(partials, nb, out); count_launches(1);
}

}  // namespace chdwf
