// cg.cu -- congrad: CGNE on M^dagger M (rhmc/cheisdwf.f:1064-1157).
//
// Vectors are FP64 as in the reference; the scalars alpha, beta, alphad,
// alphan, betad, betan and resid are REAL*4 there (implicit typing), so they
// are REAL*4 here too.  The reference accumulates alphad and betan
// element by element in REAL*4 (:1105-1108, :1133-1136), an order no parallel
// reduction can follow; here each sum is formed in FP64 with a fixed tree and
// rounded to REAL*4 once.
#include <cstdio>
#include <cstring>

#include "cg.h"
#include "dwf_stencil.cuh"

namespace chdwf {

struct LdCg {
    const double2* __restrict__ p;
    __device__ __forceinline__ double2 operator()(int64_t j) const { return __ldg(p + j); }
};

__device__ __forceinline__ bool cg_last_block(double v, double* part, unsigned* count,
                                              double* total) {
    return last_block_total<kThreads>(v, part, count, total);
}

// The stencil kernels are flavour-split: two threads per point (one per
// flavour), grid split_blocks(npts).
// x1 = M p ; alphad = |x1|^2 ; alpha = alphan/alphad   (:1093-1117)
template <int IMASS>
__global__ void __launch_bounds__(kSplitThreads, 3) k_cg1(CgArgs a) {
    CgCtl* c = a.ctl;
    if (c->done) return;
    const int64_t p = split_point();
    const int f = split_flavour();
    double loc = 0.0;
    if (p < a.g.npts) {
        const PointIdx q = point_of(a.g, p);
        double2 acc[4];
        dwf_apply_flavour<false, IMASS>(acc, LdCg{a.p}, a.g, q, f, a.chif, a.diag, a.hpin,
                                        a.apbc != 0);
#pragma unroll
        for (int d = 0; d < 4; d++) {
            a.x1[p + a.g.cs * (d + 4 * f)] = acc[d];
            loc += acc[d].x * acc[d].x + acc[d].y * acc[d].y;
        }
    }
    double tot;
    if (!cg_last_block(loc, a.part, &c->count1, &tot)) return;
    if (threadIdx.x == 0 && c->nx > 1) {
        const float alphad = (float)tot;
        c->alpha = c->alphan / alphad;
    }
}

// x2 = M^dagger x1 ; x += alpha p (nx>1) ; r -= alpha x2 ; betan = |r|^2 (:1119-1141)
template <int IMASS>
__global__ void __launch_bounds__(kSplitThreads, 3) k_cg2(CgArgs a) {
    CgCtl* c = a.ctl;
    if (c->done) return;
    const int nx = c->nx;
    const double alpha = (double)c->alpha;
    const int64_t p = split_point();
    const int f = split_flavour();
    double loc = 0.0;
    if (p < a.g.npts) {
        const PointIdx q = point_of(a.g, p);
        double2 acc[4];
        dwf_apply_flavour<true, IMASS>(acc, LdCg{a.x1}, a.g, q, f, a.chif, a.diag, a.hpin,
                                       a.apbc != 0);
#pragma unroll
        for (int d = 0; d < 4; d++) {
            const int64_t e = p + a.g.cs * (d + 4 * f);
            if (nx > 1) a.x[e] = zadd(a.x[e], zscal(alpha, a.p[e]));
            const double2 r = zsub(a.r[e], zscal(alpha, acc[d]));
            a.r[e] = r;
            loc += r.x * r.x + r.y * r.y;
        }
    }
    double tot;
    if (!cg_last_block(loc, a.part, &c->count2, &tot)) return;
    if (threadIdx.x == 0) {
        const float betan = (float)tot;
        float beta = betan / c->betad;
        c->betad = betan;
        c->alphan = betan;
        if (nx == 1) beta = 0.0f;
        c->beta = beta;
        if (betan < c->resid) {
            c->done = 1;
            c->iters = nx;
        } else if (nx >= c->niterc) {
            c->done = 2;
            c->iters = nx;
        }
        if (!(betan == betan)) { c->done = 3; c->iters = nx; }
        if (c->done && a.hflag) {
            *(volatile int*)a.hflag = c->done;
            __threadfence_system();
        }
        // all other blocks finished (they were counted), so the iteration
        // index can advance for the next launches
        if (!c->done) c->nx = nx + 1;
    }
}

// p = r + beta p ; next iteration  (:1147-1150)
__global__ void __launch_bounds__(kThreads) k_cg3(CgArgs a) {
    CgCtl* c = a.ctl;
    if (c->done) return;
    const double beta = (double)c->beta;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < a.g.kferm) a.p[i] = zadd(a.r[i], zscal(beta, a.p[i]));
}

CgWork::~CgWork() { release(); }

void CgWork::release() {
    if (ctl) cudaFree(ctl);
    if (part) cudaFree(part);
    if (hflag_host) cudaFreeHost(hflag_host);
    if (x1) cudaFree(x1);
    if (p) cudaFree(p);
    if (r) cudaFree(r);
    ctl = nullptr; part = nullptr; hflag_host = nullptr; x1 = p = r = nullptr;
}

cudaError_t CgWork::ensure(const Geom& g) {
    if (ctl && g.kferm == geom.kferm && g.L == geom.L && g.Lt == geom.Lt) return cudaSuccess;
    release();
    geom = g;
    cudaError_t e;
    if ((e = cudaMalloc(&ctl, sizeof(CgCtl)))) return e;
    const int64_t nb = split_blocks(g.npts);
    if ((e = cudaMalloc(&part, sizeof(double) * (nb + 64)))) return e;
    if ((e = cudaMalloc(&x1, sizeof(double2) * g.kferm))) return e;
    if ((e = cudaMalloc(&p, sizeof(double2) * g.kferm))) return e;
    if ((e = cudaMalloc(&r, sizeof(double2) * g.kferm))) return e;
    if ((e = cudaHostAlloc(&hflag_host, sizeof(int), cudaHostAllocMapped))) return e;
    if ((e = cudaHostGetDevicePointer((void**)&hflag_dev, hflag_host, 0))) return e;
    return cudaSuccess;
}

cudaError_t cg_solve(CgWork& w, const Geom& g, const double2* phi, float res, const float* chif,
                     float am3, float hpin, int imass, int ibound, double2* x, int* itercg,
                     int* status, cudaStream_t st) {
    cudaError_t e = w.ensure(g);
    if (e) return e;
    CgCtl hc;
    memset(&hc, 0, sizeof(hc));
    hc.nx = 1;
    hc.alpha = 1.0f;                                  // :1090-1091
    hc.betad = 1.0f;
    hc.resid = (float)g.kferm * res * res;            // :1076
    hc.niterc = (int)(g.Ls * (int64_t)g.kvol);        // niterc = kthird*kvol
    if ((e = cudaMemcpyAsync(w.ctl, &hc, sizeof(hc), cudaMemcpyHostToDevice, st))) return e;
    *w.hflag_host = 0;
    // p = x ; r = Phi (:1086-1089)
    cudaMemcpyAsync(w.p, x, sizeof(double2) * g.kferm, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(w.r, phi, sizeof(double2) * g.kferm, cudaMemcpyDeviceToDevice, st);
    CgArgs a;
    memset(&a, 0, sizeof(a));
    a.g = g;
    a.x = x; a.p = w.p; a.r = w.r; a.x1 = w.x1;
    a.chif = chif;
    a.diag = (double)(2.0f * ((3.0f - am3) + 1.0f));
    a.hpin = (double)hpin;
    a.apbc = ibound == -1;
    a.ctl = w.ctl;
    a.part = w.part;
    a.hflag = w.hflag_dev;
    const unsigned nb = split_blocks(g.npts);
    const unsigned nbf = (unsigned)((g.kferm + kThreads - 1) / kThreads);
    const int chunk = 16;
    cudaEvent_t ev[2];
    cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
    int64_t launched = 0;
    int nchunk = 0;
    const int64_t cap = hc.niterc;
    while (launched < cap) {
        for (int c = 0; c < chunk && launched < cap; c++, launched++) {
            if (imass == 3) { k_cg1<3><<<nb, kThreads, 0, st>>>(a); count_launches(1); k_cg2<3><<<nb, kThreads, 0, st>>>(a); count_launches(1); }
            else { k_cg1<1><<<nb, kThreads, 0, st>>>(a); count_launches(1); k_cg2<1><<<nb, kThreads, 0, st>>>(a); count_launches(1); }
            k_cg3<<<nbf, kThreads, 0, st>>>(a); count_launches(1);
        }
        cudaEventRecord(ev[nchunk & 1], st);
        if (nchunk >= 1) {
            cudaEventSynchronize(ev[(nchunk - 1) & 1]);
            if (*(volatile int*)w.hflag_host) break;
        }
        nchunk++;
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if ((e = cudaGetLastError())) return e;
    CgCtl hr;
    if ((e = cudaMemcpyAsync(&hr, w.ctl, sizeof(hr), cudaMemcpyDeviceToHost, st))) return e;
    if ((e = cudaStreamSynchronize(st))) return e;
    *itercg = hr.iters;
    *status = hr.done == 1 ? 0 : (hr.done == 2 ? 1 : 2);
    return cudaSuccess;
}

// ---- congrad without any allocation ---------------------------------------
// For callers that cannot allocate device memory: a host program whose device
// memory is owned by another runtime's pool or reserved in full up front, or
// code that must not allocate (a real-time or otherwise allocation-free
// section).  The solver's scratch -- the REAL*4 copy of chi, the CG vectors
// x1, p, r, the per-block partial sums and the control block -- lives in one
// file-scope device array sized for kferm <= kStaticMaxFerm.  The array is
// shared by every call: calls whose GPU work overlaps (other streams, other
// host threads) race on it.  Each call clears the part that must start at
// zero (the control block) before its first kernel.
constexpr int64_t kStaticMaxFerm = 262144;            // 8*kvol*kthird, e.g. 16^3 x 8
constexpr int64_t kStaticMaxKvol = kStaticMaxFerm / 16;   // kthird >= 2
constexpr size_t kStaticBytes = 256 + 64 * 1024 +          // control block, partials
                                3 * kStaticMaxKvol * sizeof(float) +
                                3 * kStaticMaxFerm * sizeof(double2);
static __device__ __align__(256) unsigned char g_cg_scratch[kStaticBytes];

namespace {
constexpr int kMaxDevices = 64;
// Device address of the array per device ordinal.  Two host threads making
// their first call on a device at the same time both look it up and store
// the same value: a benign race, since cudaGetSymbolAddress returns one
// address per device.
unsigned char* g_scratch_addr[kMaxDevices] = {};
}  // namespace

}  // namespace chdwf

extern "C" int chdwf_congrad_static(const void* Phi, void* x, const void* chi, int ksize,
                                    int ksizet, int kthird, float am3, int ibound, float res,
                                    float hpin, int imass, int* itercg, void* stream) {
    using namespace chdwf;
    if (!Phi || !x || !chi || !itercg) return 4;
    if (imass != 1 && imass != 3) return 4;
    // sizes in 64-bit arithmetic first: kvol = ksize^2*ksizet is a 32-bit
    // int in the geometry and must not wrap before the size check
    if (!geom_ok(ksize, ksizet, kthird)) return 4;
    if (8 * (int64_t)ksize * ksize * ksizet * kthird > kStaticMaxFerm) return 4;
    const Geom g = make_geom(ksize, ksizet, kthird);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 3;
    // once per device: the device address of the array (its host-side name
    // is only a stand-in and must never be passed to a kernel)
    if (!g_scratch_addr[dev]) {
        void* ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_cg_scratch) != cudaSuccess || !ptr) return 3;
        g_scratch_addr[dev] = (unsigned char*)ptr;
    }
    // a sticky error from earlier work on this device fails here; a stale
    // non-sticky one is cleared so that it is not reported as this call's
    if (cudaGetLastError() != cudaSuccess && cudaPeekAtLastError() != cudaSuccess) return 3;
    unsigned char* base = g_scratch_addr[dev];
    CgCtl* ctl = reinterpret_cast<CgCtl*>(base);
    double* part = reinterpret_cast<double*>(base + 256);
    float* chif = reinterpret_cast<float*>(base + 256 + 64 * 1024);
    double2* x1 = reinterpret_cast<double2*>(base + 256 + 64 * 1024 +
                                             3 * kStaticMaxKvol * sizeof(float));
    double2* p = x1 + kStaticMaxFerm;
    double2* r = p + kStaticMaxFerm;
    cudaStream_t st = (cudaStream_t)stream;
    CgCtl hc;
    memset(&hc, 0, sizeof(hc));
    hc.nx = 1;
    hc.alpha = 1.0f;                                  // rhmc/cheisdwf.f:1090-1091
    hc.betad = 1.0f;
    hc.resid = (float)g.kferm * res * res;            // :1076
    hc.niterc = (int)(g.Ls * (int64_t)g.kvol);
    if (cudaMemcpyAsync(ctl, &hc, sizeof(hc), cudaMemcpyHostToDevice, st) != cudaSuccess) return 3;
    launch_round_chi((const double*)chi, chif, g.kvol, st);
    cudaMemcpyAsync(p, x, sizeof(double2) * g.kferm, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(r, Phi, sizeof(double2) * g.kferm, cudaMemcpyDeviceToDevice, st);
    CgArgs a;
    memset(&a, 0, sizeof(a));
    a.g = g;
    a.x = (double2*)x; a.p = p; a.r = r; a.x1 = x1;
    a.chif = chif;
    a.diag = (double)(2.0f * ((3.0f - am3) + 1.0f));
    a.hpin = (double)hpin;
    a.apbc = ibound == -1;
    a.ctl = ctl;
    a.part = part;
    a.hflag = nullptr;
    const unsigned nb = split_blocks(g.npts);
    const unsigned nbf = (unsigned)((g.kferm + kThreads - 1) / kThreads);
    // chunks of 16 iterations; the done flag is copied into a host stack
    // variable after each chunk (launches after convergence return at once)
    const int64_t cap = hc.niterc;
    int64_t launched = 0;
    CgCtl hr;
    memset(&hr, 0, sizeof(hr));
    while (launched < cap) {
        for (int c = 0; c < 16 && launched < cap; c++, launched++) {
            if (imass == 3) { k_cg1<3><<<nb, kThreads, 0, st>>>(a); k_cg2<3><<<nb, kThreads, 0, st>>>(a); }
            else { k_cg1<1><<<nb, kThreads, 0, st>>>(a); k_cg2<1><<<nb, kThreads, 0, st>>>(a); }
            k_cg3<<<nbf, kThreads, 0, st>>>(a);
            count_launches(3);
        }
        // a failed launch or copy ends the solve at once instead of launching
        // on until the iteration cap
        if (cudaGetLastError() != cudaSuccess) return 3;
        if (cudaMemcpyAsync(&hr, ctl, sizeof(hr), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return 3;
        if (hr.done) break;
    }
    *itercg = hr.iters;
    if (hr.done == 2) {
        fprintf(stdout, " # iterations of congrad exceeds niterc\n");   // :1151-1153
        return 1;
    }
    if (hr.done == 3) return 2;
    return 0;
}
