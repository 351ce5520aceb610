// batch.cu -- many independent propagator solves in one set of launches.
//
// fermion() (rhmc/cheisdwf.f:897-1058) solves M^dagger M x = Phi with congrad
// (:1064-1157) once per source, one after the other.  On small lattices each
// iteration of one solve is a few microseconds of GPU work, so a sequence of
// solves is bound by kernel launches and host round trips.  Here nsys solves
// -- on lattices of different sizes, with their own chi, imass and hpin --
// advance together: one launch per CG stage covers the blocks of every
// still-running system, each system keeps its own REAL*4 scalars (the types of
// congrad) and stops on its own criterion.  Systems that share a lattice, chi
// and parameters (the sources of one ensemble) are grouped, up to kRhs to a
// group: the operator kernels apply M to all members at a point in one
// thread (multiple right-hand sides), and the iteration loop is replayed as
// a CUDA graph.  Each member's arithmetic, block partition and reduction
// order are those of congrad on its own, so the results equal
// chdwf_congrad_dev's.
#include <cstring>
#include <vector>

#include "../../include/chdwf.h"
#include "cg.h"
#include "ctx.h"
#include "dwf_stencil.cuh"

namespace chdwf {

// Systems on the same lattice with the same chi, imass, hpin, am3 and ibound
// (the sources of one ensemble) form a group of up to kRhs members: one
// thread applies the operator to every member's vector at its point, sharing
// the point's index arithmetic and chi, and the launch covers all of them.
constexpr int kRhs = 4;

struct BGrp {
    Geom g;
    int64_t off;        // element offset of member 0's vectors (member r: off + r*kferm)
    int64_t chioff;     // offset of the group's REAL*4 chi planes
    double diag, hpin;
    int apbc, imass;
    int blk0, nblk;     // the group's blocks in the point grid
    int eblk0, neblk;   // its blocks in the element grid (p = r + beta p)
    int nrhs, sys0;     // members: systems sys0 .. sys0 + nrhs - 1
    double2* x[kRhs];   // members' solutions (the callers' buffers)
};

struct BArgs {
    const BGrp* grp;
    const int* blk2grp;
    const int* eblk2grp;
    double2 *p, *r, *x1;
    const float* chif;
    CgCtl* ctl;         // one per system
    double* part;       // kRhs per block
    unsigned* gcount;   // two block counters per group
    int* active;        // number of running systems (device)
    int* hflag;         // mapped host copy: 1 when none is running
};

struct LdB {
    const double2* __restrict__ p;
    __device__ __forceinline__ double2 operator()(int64_t j) const { return __ldg(p + j); }
};

// Block sums of the kRhs members' partials into part[block*kRhs + r]; the
// group's last block (counted in *count) adds the partials of its blocks in
// block order into tot[r], resets the counter and returns true.
__device__ __forceinline__ bool grp_last_block(const double* loc, double* part, unsigned* count,
                                               int blk0, int nblk, double* tot) {
    __shared__ double sh[kThreads / 32];
    __shared__ bool is_last;
#pragma unroll
    for (int r = 0; r < kRhs; r++) {
        const double v = block_sum<kThreads>(loc[r], sh);
        if (threadIdx.x == 0) part[(int64_t)blockIdx.x * kRhs + r] = v;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        is_last = (atomicAdd(count, 1u) == (unsigned)nblk - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
#pragma unroll
    for (int r = 0; r < kRhs; r++) {
        double s = 0.0;
        for (int i = threadIdx.x; i < nblk; i += blockDim.x)
            s += ((volatile double*)part)[(int64_t)(blk0 + i) * kRhs + r];
        s = block_sum<kThreads>(s, sh);
        tot[r] = s;     // valid in thread 0
    }
    if (threadIdx.x == 0) *count = 0;
    return true;
}

template <bool DAG>
__device__ __forceinline__ void apply_grp(double2 acc[4], const double2* in, const BGrp& S,
                                          const PointIdx& q, int f, const float* chif) {
    if (S.imass == 3)
        dwf_apply_flavour<DAG, 3>(acc, LdB{in}, S.g, q, f, chif, S.diag, S.hpin, S.apbc != 0);
    else
        dwf_apply_flavour<DAG, 1>(acc, LdB{in}, S.g, q, f, chif, S.diag, S.hpin, S.apbc != 0);
}

// Which members still run (the flags were set by the previous launch's last
// blocks, so they are the same in every block of this launch).
__device__ __forceinline__ int running_mask(const BArgs& a, const BGrp& S) {
    int m = 0;
    for (int r = 0; r < S.nrhs; r++)
        if (!a.ctl[S.sys0 + r].done) m |= 1 << r;
    return m;
}

// x1 = M p ; alphad = |x1|^2 ; alpha = alphan/alphad (rhmc/cheisdwf.f:1093-1117)
// for every running member.  Flavour-split: kSplitPoints points per block,
// two threads per point.
__global__ void __launch_bounds__(kSplitThreads, 2) k_bcg1(BArgs a) {
    const int G = a.blk2grp[blockIdx.x];
    const BGrp& S = a.grp[G];
    const int run = running_mask(a, S);
    if (!run) return;
    const int64_t p = (int64_t)(blockIdx.x - S.blk0) * kSplitPoints +
                      (threadIdx.x & (kSplitPoints - 1));
    const int f = split_flavour();
    const int64_t kf = S.g.kferm;
    double loc[kRhs] = {0.0, 0.0, 0.0, 0.0};
    if (p < S.g.npts) {
        const PointIdx q = point_of(S.g, p);
#pragma unroll
        for (int r = 0; r < kRhs; r++) {
            if (!(run >> r & 1)) continue;
            double2 acc[4];
            apply_grp<false>(acc, a.p + S.off + r * kf, S, q, f, a.chif + S.chioff);
#pragma unroll
            for (int d = 0; d < 4; d++) {
                a.x1[S.off + r * kf + p + S.g.cs * (d + 4 * f)] = acc[d];
                loc[r] += acc[d].x * acc[d].x + acc[d].y * acc[d].y;
            }
        }
    }
    double tot[kRhs];
    if (!grp_last_block(loc, a.part, a.gcount + 2 * G, S.blk0, S.nblk, tot)) return;
    if (threadIdx.x == 0)
        for (int r = 0; r < S.nrhs; r++) {
            CgCtl* c = a.ctl + S.sys0 + r;
            if ((run >> r & 1) && c->nx > 1) c->alpha = c->alphan / (float)tot[r];
        }
}

// x2 = M^dagger x1 ; x += alpha p ; r -= alpha x2 ; betan = |r|^2 (:1119-1141)
__global__ void __launch_bounds__(kSplitThreads, 2) k_bcg2(BArgs a) {
    const int G = a.blk2grp[blockIdx.x];
    const BGrp& S = a.grp[G];
    const int run = running_mask(a, S);
    if (!run) return;
    const int64_t p = (int64_t)(blockIdx.x - S.blk0) * kSplitPoints +
                      (threadIdx.x & (kSplitPoints - 1));
    const int f = split_flavour();
    const int64_t kf = S.g.kferm;
    double loc[kRhs] = {0.0, 0.0, 0.0, 0.0};
    if (p < S.g.npts) {
        const PointIdx q = point_of(S.g, p);
#pragma unroll
        for (int r = 0; r < kRhs; r++) {
            if (!(run >> r & 1)) continue;
            const CgCtl* c = a.ctl + S.sys0 + r;
            const int nx = c->nx;
            const double alpha = (double)c->alpha;
            double2 acc[4];
            apply_grp<true>(acc, a.x1 + S.off + r * kf, S, q, f, a.chif + S.chioff);
#pragma unroll
            for (int d = 0; d < 4; d++) {
                const int64_t e = p + S.g.cs * (d + 4 * f);
                const int64_t eb = S.off + r * kf + e;
                if (nx > 1) S.x[r][e] = zadd(S.x[r][e], zscal(alpha, a.p[eb]));
                const double2 rv = zsub(a.r[eb], zscal(alpha, acc[d]));
                a.r[eb] = rv;
                loc[r] += rv.x * rv.x + rv.y * rv.y;
            }
        }
    }
    double tot[kRhs];
    if (!grp_last_block(loc, a.part, a.gcount + 2 * G + 1, S.blk0, S.nblk, tot)) return;
    if (threadIdx.x != 0) return;
    for (int r = 0; r < S.nrhs; r++) {
        if (!(run >> r & 1)) continue;
        CgCtl* c = a.ctl + S.sys0 + r;
        const int nx = c->nx;
        const float betan = (float)tot[r];
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
    const int G = a.eblk2grp[blockIdx.x];
    const BGrp& S = a.grp[G];
    const int64_t i = (int64_t)(blockIdx.x - S.eblk0) * blockDim.x + threadIdx.x;
    if (i >= S.g.kferm) return;
    for (int r = 0; r < S.nrhs; r++) {
        const CgCtl* c = a.ctl + S.sys0 + r;
        if (c->done) continue;
        const double beta = (double)c->beta;
        const int64_t e = S.off + r * S.g.kferm + i;
        a.p[e] = zadd(a.r[e], zscal(beta, a.p[e]));
    }
}

__global__ void k_bround_chi(const double* __restrict__ chi, float* __restrict__ chif, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) chif[i] = (float)chi[i];
}

// Batch workspace, kept in the context and reallocated when a larger batch
// arrives.
struct BatchWork {
    int64_t cap_elems = 0, cap_chi = 0;
    int cap_sys = 0, cap_grp = 0, cap_blk = 0, cap_eblk = 0;
    double2 *p = nullptr, *r = nullptr, *x1 = nullptr;
    float* chif = nullptr;
    BGrp* grp = nullptr;
    int *blk2grp = nullptr, *eblk2grp = nullptr, *active = nullptr;
    CgCtl* ctl = nullptr;
    double* part = nullptr;
    unsigned* gcount = nullptr;
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
        cudaFree(p); cudaFree(r); cudaFree(x1); cudaFree(chif); cudaFree(grp);
        cudaFree(blk2grp); cudaFree(eblk2grp); cudaFree(active); cudaFree(ctl); cudaFree(part);
        cudaFree(gcount);
        if (hflag_host) cudaFreeHost(hflag_host);
        hflag_host = nullptr;
        cap_elems = cap_chi = 0;
        cap_sys = cap_grp = cap_blk = cap_eblk = 0;
        p = r = x1 = nullptr;
        chif = nullptr;
        grp = nullptr;
        blk2grp = eblk2grp = active = nullptr;
        ctl = nullptr;
        part = nullptr;
        gcount = nullptr;
        hflag_dev = nullptr;
    }
    cudaError_t reserve(int64_t elems, int64_t chis, int nsys, int ngrp, int nblk, int neblk) {
        if (p && elems <= cap_elems && chis <= cap_chi && nsys <= cap_sys && ngrp <= cap_grp &&
            nblk <= cap_blk && neblk <= cap_eblk)
            return cudaSuccess;
        release();
        cudaError_t e;
        if ((e = cudaMalloc(&p, sizeof(double2) * elems)) ||
            (e = cudaMalloc(&r, sizeof(double2) * elems)) ||
            (e = cudaMalloc(&x1, sizeof(double2) * elems)) ||
            (e = cudaMalloc(&chif, sizeof(float) * chis)) ||
            (e = cudaMalloc(&grp, sizeof(BGrp) * ngrp)) ||
            (e = cudaMalloc(&ctl, sizeof(CgCtl) * nsys)) ||
            (e = cudaMalloc(&blk2grp, sizeof(int) * nblk)) ||
            (e = cudaMalloc(&eblk2grp, sizeof(int) * neblk)) ||
            (e = cudaMalloc(&part, sizeof(double) * kRhs * nblk)) ||
            (e = cudaMalloc(&gcount, sizeof(unsigned) * 2 * ngrp)) ||
            (e = cudaMalloc(&active, sizeof(int))) ||
            (e = cudaHostAlloc(&hflag_host, sizeof(int), cudaHostAllocMapped)) ||
            (e = cudaHostGetDevicePointer((void**)&hflag_dev, hflag_host, 0)))
            return e;
        cap_elems = elems; cap_chi = chis; cap_sys = nsys; cap_grp = ngrp;
        cap_blk = nblk; cap_eblk = neblk;
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
    for (int i = 0; i < nsys; i++) {
        const chdwf_cg_system& s = in[i];
        if (!geom_ok(s.ksize, s.ksizet, s.kthird) || !s.Phi || !s.x || !s.chi ||
            (s.imass != 1 && s.imass != 3))
            return CHDWF_BAD_ARG;
    }
    // consecutive systems with the same lattice, chi and parameters form a
    // group of up to kRhs members (systems keep their order: member r of a
    // group starting at system i is system i + r)
    auto same = [&](const chdwf_cg_system& u, const chdwf_cg_system& v) {
        return u.ksize == v.ksize && u.ksizet == v.ksizet && u.kthird == v.kthird &&
               u.imass == v.imass && u.hpin == v.hpin && u.am3 == v.am3 && u.ibound == v.ibound &&
               u.chi == v.chi;
    };
    std::vector<BGrp> grp;
    std::vector<int> b2g, e2g;
    int64_t elems = 0, chis = 0;
    for (int i = 0; i < nsys;) {
        int n = 1;
        while (n < kRhs && i + n < nsys && same(in[i], in[i + n])) n++;
        const chdwf_cg_system& s = in[i];
        BGrp b;
        memset(&b, 0, sizeof(b));
        b.g = make_geom(s.ksize, s.ksizet, s.kthird);
        b.off = elems;
        b.chioff = chis;
        b.diag = (double)(2.0f * ((3.0f - s.am3) + 1.0f));
        b.hpin = (double)s.hpin;
        b.apbc = s.ibound == -1;
        b.imass = s.imass;
        b.nrhs = n;
        b.sys0 = i;
        for (int r = 0; r < n; r++) b.x[r] = (double2*)in[i + r].x;
        const int G = (int)grp.size();
        b.blk0 = (int)b2g.size();
        b.nblk = (int)split_blocks(b.g.npts);
        for (int k = 0; k < b.nblk; k++) b2g.push_back(G);
        b.eblk0 = (int)e2g.size();
        b.neblk = (int)((b.g.kferm + kThreads - 1) / kThreads);
        for (int k = 0; k < b.neblk; k++) e2g.push_back(G);
        elems += n * b.g.kferm;
        chis += 3 * (int64_t)b.g.kvol;
        grp.push_back(b);
        i += n;
    }
    const int ngrp = (int)grp.size();
    cudaError_t e = w.reserve(elems, chis, nsys, ngrp, (int)b2g.size(), (int)e2g.size());
    if (e) return c->status_of(e, "congrad_batch: workspace");
    std::vector<CgCtl> ctl(nsys);
    int64_t maxcap = 0;
    for (const BGrp& b : grp)
        for (int r = 0; r < b.nrhs; r++) {
            CgCtl& h = ctl[b.sys0 + r];
            memset(&h, 0, sizeof(h));
            h.nx = 1;
            h.alpha = 1.0f;                                   // :1090-1091
            h.betad = 1.0f;
            h.resid = (float)b.g.kferm * res * res;           // :1076
            h.niterc = (int)(b.g.Ls * (int64_t)b.g.kvol);
            if (h.niterc > maxcap) maxcap = h.niterc;
        }
    cudaMemcpyAsync(w.grp, grp.data(), sizeof(BGrp) * ngrp, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(w.ctl, ctl.data(), sizeof(CgCtl) * nsys, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(w.blk2grp, b2g.data(), sizeof(int) * b2g.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(w.eblk2grp, e2g.data(), sizeof(int) * e2g.size(), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(w.gcount, 0, sizeof(unsigned) * 2 * ngrp, st);
    cudaMemcpyAsync(w.active, &nsys, sizeof(int), cudaMemcpyHostToDevice, st);
    *w.hflag_host = 0;
    for (const BGrp& b : grp) {                // p = x, r = Phi, chi rounded (:1086-1089)
        const int64_t kf = b.g.kferm;
        for (int r = 0; r < b.nrhs; r++) {
            cudaMemcpyAsync(w.p + b.off + r * kf, in[b.sys0 + r].x, sizeof(double2) * kf,
                            cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(w.r + b.off + r * kf, in[b.sys0 + r].Phi, sizeof(double2) * kf,
                            cudaMemcpyDeviceToDevice, st);
        }
        const int n = 3 * b.g.kvol;
        k_bround_chi<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(
            (const double*)in[b.sys0].chi, w.chif + b.chioff, n);
        count_launches(1);
    }
    BArgs a;
    memset(&a, 0, sizeof(a));    // padding too: the struct is the graph's key
    a.grp = w.grp;
    a.blk2grp = w.blk2grp;
    a.eblk2grp = w.eblk2grp;
    a.p = w.p; a.r = w.r; a.x1 = w.x1;
    a.chif = w.chif;
    a.ctl = w.ctl;
    a.part = w.part;
    a.gcount = w.gcount;
    a.active = w.active;
    a.hflag = w.hflag_dev;
    const unsigned nb = (unsigned)b2g.size(), nbe = (unsigned)e2g.size();
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
