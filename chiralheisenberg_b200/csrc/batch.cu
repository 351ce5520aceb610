// batch.cu -- many independent propagator solves in one set of launches.
//
// fermion() (rhmc/cheisdwf.f:897-1058) solves M^dagger M x = Phi with congrad
// (:1064-1157) once per source, one after the other.  On small lattices each
// iteration of one solve is a few microseconds of GPU work, so a sequence of
// solves is bound by kernel launches and host round trips.  Here nsys solves
// -- on lattices of different sizes, with their own chi, imass and hpin --
// advance together: one launch per CG stage covers the blocks of every
// still-running system, each system keeps its own REAL*4 scalars (the types of
// congrad) and stops on its own criterion.
#include <cstring>
#include <vector>

#include "../../include/chdwf.h"
#include "cg.h"
#include "ctx.h"
#include "dwf_stencil.cuh"

namespace chdwf {

struct BSys {
    Geom g;
    int64_t off;        // element offset of the system's vectors in the batch buffers
    int64_t chioff;     // offset of its REAL*4 chi planes
    double diag, hpin;
    int apbc, imass;
    int blk0, nblk;     // its blocks in the point grid
    int eblk0, neblk;   // its blocks in the element grid (p = r + beta p)
    double2* x;
    const double2* phi;
};

struct BArgs {
    const BSys* sys;
    const int* blk2sys;
    const int* eblk2sys;
    double2 *p, *r, *x1;
    const float* chif;
    CgCtl* ctl;         // one per system
    double* part;       // one per block
    int* active;        // number of running systems (device)
    int* hflag;         // mapped host copy: 1 when none is running
};

struct LdB {
    const double2* __restrict__ p;
    __device__ __forceinline__ double2 operator()(int64_t j) const { return __ldg(p + j); }
};

__device__ __forceinline__ bool sys_last_block(double v, double* part, unsigned* count, int blk0,
                                               int nblk, double* total) {
    __shared__ double sh[kThreads / 32];
    __shared__ bool is_last;
    v = block_sum<kThreads>(v, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = v;
        __threadfence();
        is_last = (atomicAdd(count, 1u) == (unsigned)nblk - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    double s = 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) s += ((volatile double*)part)[blk0 + i];
    s = block_sum<kThreads>(s, sh);
    if (threadIdx.x == 0) {
        *total = s;
        *count = 0;
    }
    return true;
}

template <bool DAG>
__device__ __forceinline__ void apply_sys(double2 acc[4], const double2* in, const BSys& S,
                                          const PointIdx& q, int f, const float* chif) {
    if (S.imass == 3)
        dwf_apply_flavour<DAG, 3>(acc, LdB{in}, S.g, q, f, chif, S.diag, S.hpin, S.apbc != 0);
    else
        dwf_apply_flavour<DAG, 1>(acc, LdB{in}, S.g, q, f, chif, S.diag, S.hpin, S.apbc != 0);
}

// x1 = M p ; alphad = |x1|^2 ; alpha = alphan/alphad (rhmc/cheisdwf.f:1093-1117)
// Flavour-split stencil kernels: a system's point blocks cover
// kSplitPoints points each, two threads per point.
__global__ void __launch_bounds__(kSplitThreads, 2) k_bcg1(BArgs a) {
    const int s = a.blk2sys[blockIdx.x];
    const BSys S = a.sys[s];
    CgCtl* c = a.ctl + s;
    if (c->done) return;
    const int64_t p = (int64_t)(blockIdx.x - S.blk0) * kSplitPoints +
                      (threadIdx.x & (kSplitPoints - 1));
    const int f = split_flavour();
    double loc = 0.0;
    if (p < S.g.npts) {
        const PointIdx q = point_of(S.g, p);
        double2 acc[4];
        apply_sys<false>(acc, a.p + S.off, S, q, f, a.chif + S.chioff);
#pragma unroll
        for (int d = 0; d < 4; d++) {
            a.x1[S.off + p + S.g.cs * (d + 4 * f)] = acc[d];
            loc += acc[d].x * acc[d].x + acc[d].y * acc[d].y;
        }
    }
    double tot;
    if (!sys_last_block(loc, a.part, &c->count1, S.blk0, S.nblk, &tot)) return;
    if (threadIdx.x == 0 && c->nx > 1) c->alpha = c->alphan / (float)tot;
}

// x2 = M^dagger x1 ; x += alpha p ; r -= alpha x2 ; betan = |r|^2 (:1119-1141)
__global__ void __launch_bounds__(kSplitThreads, 2) k_bcg2(BArgs a) {
    const int s = a.blk2sys[blockIdx.x];
    const BSys S = a.sys[s];
    CgCtl* c = a.ctl + s;
    if (c->done) return;
    const int nx = c->nx;
    const double alpha = (double)c->alpha;
    const int64_t p = (int64_t)(blockIdx.x - S.blk0) * kSplitPoints +
                      (threadIdx.x & (kSplitPoints - 1));
    const int f = split_flavour();
    double loc = 0.0;
    if (p < S.g.npts) {
        const PointIdx q = point_of(S.g, p);
        double2 acc[4];
        apply_sys<true>(acc, a.x1 + S.off, S, q, f, a.chif + S.chioff);
#pragma unroll
        for (int d = 0; d < 4; d++) {
            const int64_t e = p + S.g.cs * (d + 4 * f);
            if (nx > 1) S.x[e] = zadd(S.x[e], zscal(alpha, a.p[S.off + e]));
            const double2 r = zsub(a.r[S.off + e], zscal(alpha, acc[d]));
            a.r[S.off + e] = r;
            loc += r.x * r.x + r.y * r.y;
        }
    }
    double tot;
    if (!sys_last_block(loc, a.part, &c->count2, S.blk0, S.nblk, &tot)) return;
    if (threadIdx.x == 0) {
        const float betan = (float)tot;
        float beta = betan / c->betad;
        c->betad = betan;
        c->alphan = betan;
        if (nx == 1) beta = 0.0f;
        c->beta = beta;
        if (betan < c->resid) { c->done = 1; c->iters = nx; }
        else if (nx >= c->niterc) { c->done = 2; c->iters = nx; }
        if (!(betan == betan)) { c->done = 3; c->iters = nx; }
        if (c->done) {
            if (atomicSub(a.active, 1) == 1 && a.hflag) {
                *(volatile int*)a.hflag = 1;
                __threadfence_system();
            }
        } else {
            c->nx = nx + 1;
        }
    }
}

// p = r + beta p (:1147-1150)
__global__ void __launch_bounds__(kThreads) k_bcg3(BArgs a) {
    const int s = a.eblk2sys[blockIdx.x];
    const BSys S = a.sys[s];
    const CgCtl* c = a.ctl + s;
    if (c->done) return;
    const double beta = (double)c->beta;
    const int64_t i = (int64_t)(blockIdx.x - S.eblk0) * blockDim.x + threadIdx.x;
    if (i < S.g.kferm) a.p[S.off + i] = zadd(a.r[S.off + i], zscal(beta, a.p[S.off + i]));
}

__global__ void k_bround_chi(const double* __restrict__ chi, float* __restrict__ chif, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) chif[i] = (float)chi[i];
}

// Batch workspace, kept in the context and reallocated when a larger batch
// arrives.
struct BatchWork {
    int64_t cap_elems = 0, cap_chi = 0;
    int cap_sys = 0, cap_blk = 0, cap_eblk = 0;
    double2 *p = nullptr, *r = nullptr, *x1 = nullptr;
    float* chif = nullptr;
    BSys* sys = nullptr;
    int *blk2sys = nullptr, *eblk2sys = nullptr, *active = nullptr;
    CgCtl* ctl = nullptr;
    double* part = nullptr;
    int* hflag_host = nullptr;
    int* hflag_dev = nullptr;
    // a chunk of CG iterations captured as a CUDA graph, reused while the
    // batch layout (kernel arguments and grids) stays the same
    cudaGraphExec_t chunk = nullptr;
    std::vector<unsigned char> chunk_key;
    void drop_graph() {
        if (chunk) cudaGraphExecDestroy(chunk);
        chunk = nullptr;
        chunk_key.clear();
    }
    void release() {
        drop_graph();
        cudaFree(p); cudaFree(r); cudaFree(x1); cudaFree(chif); cudaFree(sys);
        cudaFree(blk2sys); cudaFree(eblk2sys); cudaFree(active); cudaFree(ctl); cudaFree(part);
        if (hflag_host) cudaFreeHost(hflag_host);
        hflag_host = nullptr;
        cap_elems = cap_chi = 0;
        cap_sys = cap_blk = cap_eblk = 0;
        p = r = x1 = nullptr;
        chif = nullptr;
        sys = nullptr;
        blk2sys = eblk2sys = active = nullptr;
        ctl = nullptr;
        part = nullptr;
        hflag_dev = nullptr;
    }
    cudaError_t reserve(int64_t elems, int64_t chis, int nsys, int nblk, int neblk) {
        if (p && elems <= cap_elems && chis <= cap_chi && nsys <= cap_sys && nblk <= cap_blk &&
            neblk <= cap_eblk)
            return cudaSuccess;
        release();
        cudaError_t e;
        if ((e = cudaMalloc(&p, sizeof(double2) * elems)) ||
            (e = cudaMalloc(&r, sizeof(double2) * elems)) ||
            (e = cudaMalloc(&x1, sizeof(double2) * elems)) ||
            (e = cudaMalloc(&chif, sizeof(float) * chis)) ||
            (e = cudaMalloc(&sys, sizeof(BSys) * nsys)) ||
            (e = cudaMalloc(&ctl, sizeof(CgCtl) * nsys)) ||
            (e = cudaMalloc(&blk2sys, sizeof(int) * nblk)) ||
            (e = cudaMalloc(&eblk2sys, sizeof(int) * neblk)) ||
            (e = cudaMalloc(&part, sizeof(double) * nblk)) ||
            (e = cudaMalloc(&active, sizeof(int))) ||
            (e = cudaHostAlloc(&hflag_host, sizeof(int), cudaHostAllocMapped)) ||
            (e = cudaHostGetDevicePointer((void**)&hflag_dev, hflag_host, 0)))
            return e;
        cap_elems = elems; cap_chi = chis; cap_sys = nsys; cap_blk = nblk; cap_eblk = neblk;
        return cudaSuccess;
    }
};

void free_batch(BatchWork* w) {
    if (w) {
        w->release();
        delete w;
    }
}

}  // namespace chdwf

using namespace chdwf;

extern "C" int chdwf_congrad_batch(chdwf_ctx* ctx, const chdwf_cg_system* in, int nsys, float res,
                                   int* itercg, int* status) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !in || nsys < 1 || !itercg || !status) return CHDWF_BAD_ARG;
    cudaSetDevice(c->device);
    if (!c->batch) c->batch = new BatchWork();
    BatchWork& w = *c->batch;
    cudaStream_t st = c->stream;
    std::vector<BSys> sys(nsys);
    std::vector<int> b2s, e2s;
    int64_t elems = 0, chis = 0;
    for (int i = 0; i < nsys; i++) {
        const chdwf_cg_system& s = in[i];
        if (!geom_ok(s.ksize, s.ksizet, s.kthird) || !s.Phi || !s.x || !s.chi ||
            (s.imass != 1 && s.imass != 3))
            return CHDWF_BAD_ARG;
        BSys& b = sys[i];
        b.g = make_geom(s.ksize, s.ksizet, s.kthird);
        b.off = elems;
        b.chioff = chis;
        b.diag = (double)(2.0f * ((3.0f - s.am3) + 1.0f));
        b.hpin = (double)s.hpin;
        b.apbc = s.ibound == -1;
        b.imass = s.imass;
        b.blk0 = (int)b2s.size();
        b.nblk = (int)split_blocks(b.g.npts);
        for (int k = 0; k < b.nblk; k++) b2s.push_back(i);
        b.eblk0 = (int)e2s.size();
        b.neblk = (int)((b.g.kferm + kThreads - 1) / kThreads);
        for (int k = 0; k < b.neblk; k++) e2s.push_back(i);
        b.x = (double2*)s.x;
        b.phi = (const double2*)s.Phi;
        elems += b.g.kferm;
        chis += 3 * (int64_t)b.g.kvol;
    }
    cudaError_t e = w.reserve(elems, chis, nsys, (int)b2s.size(), (int)e2s.size());
    if (e) return c->status_of(e, "congrad_batch: workspace");
    std::vector<CgCtl> ctl(nsys);
    int64_t maxcap = 0;
    for (int i = 0; i < nsys; i++) {
        CgCtl& h = ctl[i];
        memset(&h, 0, sizeof(h));
        h.nx = 1;
        h.alpha = 1.0f;                                   // :1090-1091
        h.betad = 1.0f;
        h.resid = (float)sys[i].g.kferm * res * res;      // :1076
        h.niterc = (int)(sys[i].g.Ls * (int64_t)sys[i].g.kvol);
        if (h.niterc > maxcap) maxcap = h.niterc;
    }
    cudaMemcpyAsync(w.sys, sys.data(), sizeof(BSys) * nsys, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(w.ctl, ctl.data(), sizeof(CgCtl) * nsys, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(w.blk2sys, b2s.data(), sizeof(int) * b2s.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(w.eblk2sys, e2s.data(), sizeof(int) * e2s.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(w.active, &nsys, sizeof(int), cudaMemcpyHostToDevice, st);
    *w.hflag_host = 0;
    for (int i = 0; i < nsys; i++) {           // p = x, r = Phi, chi rounded (:1086-1089)
        const int64_t kf = sys[i].g.kferm;
        cudaMemcpyAsync(w.p + sys[i].off, in[i].x, sizeof(double2) * kf, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(w.r + sys[i].off, in[i].Phi, sizeof(double2) * kf, cudaMemcpyDeviceToDevice, st);
        const int n = 3 * sys[i].g.kvol;
        k_bround_chi<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(
            (const double*)in[i].chi, w.chif + sys[i].chioff, n);
        count_launches(1);
    }
    BArgs a;
    memset(&a, 0, sizeof(a));    // padding too: the struct is the graph's key
    a.sys = w.sys;
    a.blk2sys = w.blk2sys;
    a.eblk2sys = w.eblk2sys;
    a.p = w.p; a.r = w.r; a.x1 = w.x1;
    a.chif = w.chif;
    a.ctl = w.ctl;
    a.part = w.part;
    a.active = w.active;
    a.hflag = w.hflag_dev;
    const unsigned nb = (unsigned)b2s.size(), nbe = (unsigned)e2s.size();
    // the chunk of kChunk iterations as a graph: every launch of the loop is
    // identical (the iteration state lives in the per-system control blocks),
    // so one capture serves every chunk of this and later batches of the
    // same layout
    constexpr int kChunk = 16;
    {
        std::vector<unsigned char> key(sizeof(a) + 2 * sizeof(unsigned));
        memcpy(key.data(), &a, sizeof(a));
        memcpy(key.data() + sizeof(a), &nb, sizeof(unsigned));
        memcpy(key.data() + sizeof(a) + sizeof(unsigned), &nbe, sizeof(unsigned));
        if (!w.chunk || w.chunk_key != key) {
            w.drop_graph();
            cudaGraph_t g = nullptr;
            if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                for (int k = 0; k < kChunk; k++) {
                    k_bcg1<<<nb, kThreads, 0, st>>>(a);
                    k_bcg2<<<nb, kThreads, 0, st>>>(a);
                    k_bcg3<<<nbe, kThreads, 0, st>>>(a);
                }
                if (cudaStreamEndCapture(st, &g) == cudaSuccess && g) {
                    if (cudaGraphInstantiate(&w.chunk, g, 0) != cudaSuccess) w.chunk = nullptr;
                    cudaGraphDestroy(g);
                }
            }
            cudaGetLastError();
            if (w.chunk) w.chunk_key = key;
        }
    }
    cudaEvent_t ev[2];
    cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
    int64_t launched = 0;
    int nchunk = 0;
    while (launched < maxcap) {
        if (w.chunk) {
            cudaGraphLaunch(w.chunk, st);
            launched += kChunk;
            count_launches(3 * kChunk);
        } else {
            for (int k = 0; k < kChunk && launched < maxcap; k++, launched++) {
                k_bcg1<<<nb, kThreads, 0, st>>>(a);
                k_bcg2<<<nb, kThreads, 0, st>>>(a);
                k_bcg3<<<nbe, kThreads, 0, st>>>(a);
                count_launches(3);
            }
        }
        cudaEventRecord(ev[nchunk & 1], st);
        if (nchunk >= 1) {
            cudaEventSynchronize(ev[(nchunk - 1) & 1]);
            if (*(volatile int*)w.hflag_host) break;
        }
        nchunk++;
    }
    cudaEventSynchronize(ev[nchunk & 1]);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    cudaMemcpyAsync(ctl.data(), w.ctl, sizeof(CgCtl) * nsys, cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st))) return c->status_of(e, "congrad_batch");
    int worst = CHDWF_OK;
    for (int i = 0; i < nsys; i++) {
        itercg[i] = ctl[i].iters;
        status[i] = ctl[i].done == 1 ? CHDWF_OK
                    : ctl[i].done == 2 ? CHDWF_ITER_CAP
                                       : CHDWF_NONFINITE;
        if (status[i] > worst) worst = status[i];
    }
    return worst;
}
