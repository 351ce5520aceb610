// program.cpp -- host driver mirroring program dwf3d (rhmc/cheisdwf.f:1-466)
// over the resident C ABI: random numbers and control flow on the host, every
// field operation on the GPU.
//
// The random stream of a trajectory does not depend on the fields: the
// heatbath Gaussians, the momenta, the trajectory-end draws and the
// Metropolis draw are fixed by the generator state alone.  The driver
// therefore generates trajectory n+1's heatbath Gaussians on a host thread
// while trajectory n runs on the GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <future>
#include <string>
#include <vector>

#include "../../include/chdwf.h"
#include "../../include/chdwf_program.h"
#include "fortio.h"
#include "rng.h"

namespace {

struct Draws {                       // the random numbers of one trajectory
    std::vector<float> gauss;        // 2*4*kthird gauss0 calls, (kvol,2) each
    std::vector<float> pp;           // pp(kvol,3) from two gaussp calls
    std::vector<float> ytest;        // trajectory-end draws, one per MD step
    float x = 0.0f;                  // Metropolis draw
    float yferm = 0.0f;              // fermion()'s draw (measurement sweeps)
    bool measured = false;
    chdwf::Rng::State state_after{};  // generator state after these draws
};

}  // namespace

struct Staged {                      // a trajectory's random inputs already in HBM
    Draws d;
    int slot = -1;                   // its device buffers in the driver's pool
};

struct StageSlot {                   // device buffers for one staged trajectory
    float* gauss_dev = nullptr;
    float* pp_dev = nullptr;
};

struct chdwf_prog {
    chdwf_ctx* ctx = nullptr;
    std::deque<Staged> staged;
    int L = 0, Lt = 0, Ls = 0, kvol = 0;
    float dt = 0.1f, beta = 0.5f, am3 = 1.0f, am = 0.0f, hpin = 0.0f;
    int imass = 1, iterl = 1, iprint = 5, measure = 1, isweep = 0;
    float rescga = 0.000000001f, rescgg = 0.000001f, rescgm = 0.000000001f;   // :32-33
    // multi-pseudofermion variant (chdwf_prog_set_ext): npf > 0 selects it
    int ext_npf = 0, ext_nsteps = 10, ext_integrator = 1;
    float ext_lambda = 0.1931833275037836f;
    chdwf::Rng rng;
    bool have_next = false;
    std::future<Draws> next;
    std::vector<float> cferm;        // cferm1(0:Lt-1,2), cferm2 as complex64 pairs
    chdwf_run_sums sums{};           // running sums of the main program
    int cg_caps = 0;                 // congrad iteration caps not yet reported
    std::string err;
    chdwf::Rng::State last_state{};  // generator after the last completed sweep
    // Device buffers of staged trajectories, allocated on first use and
    // reused: a sweep never allocates or frees device memory.
    std::vector<StageSlot> pool;
    std::vector<int> free_slots;

    // heatbath Gaussians of one trajectory: 2*4*kthird gauss0 calls of
    // (kvol,2) per pseudofermion field
    size_t gauss_floats() const {
        return 16 * (size_t)kvol * Ls * (size_t)(ext_npf > 0 ? ext_npf : 1);
    }
    int take_slot() {
        if (!free_slots.empty()) {
            const int k = free_slots.back();
            free_slots.pop_back();
            return k;
        }
        StageSlot sl;
        if (cudaMalloc(&sl.gauss_dev, sizeof(float) * gauss_floats()) ||
            cudaMalloc(&sl.pp_dev, sizeof(float) * 3 * (size_t)kvol)) {
            cudaFree(sl.gauss_dev);
            cudaGetLastError();
            return -1;
        }
        pool.push_back(sl);
        return (int)pool.size() - 1;
    }
    void release_pool() {
        for (StageSlot& sl : pool) {
            cudaFree(sl.gauss_dev);
            cudaFree(sl.pp_dev);
        }
        pool.clear();
        free_slots.clear();
    }

    // Drop prefetched or staged draws and rewind the generator to the end
    // of the last completed sweep, so the stream continues exactly there.
    void discard_pending() {
        if (have_next) {
            next.wait();
            have_next = false;
        }
        for (Staged& s : staged)
            if (s.slot >= 0) free_slots.push_back(s.slot);
        staged.clear();
        rng.set_state(last_state);
    }

    // All random numbers of the next trajectory, in the reference's order.
    Draws draw(int sweep_index) {
        if (ext_npf > 0) return draw_ext();
        Draws d;
        const int64_t kv = kvol;
        d.gauss.resize(16 * (size_t)kv * Ls);
        for (int c = 0; c < 8 * Ls; c++) rng.gauss0(kv, d.gauss.data() + (size_t)c * 2 * kv);  // :221-230
        std::vector<float> ps(2 * kv);
        d.pp.resize(3 * kv);
        rng.gaussp(kv, ps.data());                                                          // :249-253
        std::memcpy(d.pp.data(), ps.data(), sizeof(float) * 2 * kv);
        rng.gaussp(kv, ps.data());                                                          // :254-257
        std::memcpy(d.pp.data() + 2 * kv, ps.data(), sizeof(float) * kv);
        const float proby = 1.0f / (float)iterl;                                            // :164
        for (int iter = 1; iter <= 1000; iter++) {                                          // :281
            const float y = rng.rano_yrun();                                                // :298
            d.ytest.push_back(y);
            if (y < proby) break;
        }
        d.x = rng.rano_yrun();                                                              // :329
        d.measured = measure && (sweep_index / iprint) * iprint == sweep_index;
        if (d.measured) d.yferm = rng.rano_yran();                                          // :929
        d.state_after = rng.state();
        return d;
    }

    // The multi-pseudofermion variant's random numbers: the heatbath
    // Gaussians of each field in turn (the reference's gauss0 order within a
    // field), the momenta as the reference draws them, and the Metropolis
    // draw; the trajectory has a fixed number of steps, so there are no
    // trajectory-end draws.  No measurement.
    Draws draw_ext() {
        Draws d;
        const int64_t kv = kvol;
        d.gauss.resize(gauss_floats());
        for (int c = 0; c < 8 * Ls * ext_npf; c++)
            rng.gauss0(kv, d.gauss.data() + (size_t)c * 2 * kv);
        std::vector<float> ps(2 * kv);
        d.pp.resize(3 * kv);
        rng.gaussp(kv, ps.data());
        std::memcpy(d.pp.data(), ps.data(), sizeof(float) * 2 * kv);
        rng.gaussp(kv, ps.data());
        std::memcpy(d.pp.data() + 2 * kv, ps.data(), sizeof(float) * kv);
        d.x = rng.rano_yrun();
        d.measured = false;
        d.state_after = rng.state();
        return d;
    }

    void prefetch(int sweep_index) {
        next = std::async(std::launch::async, [this, sweep_index] { return draw(sweep_index); });
        have_next = true;
    }
};

namespace {

int fermion(chdwf_prog* p, float yferm, float* aviter) {
    // fermion(res, aviter, am, hpin, imass), rhmc/cheisdwf.f:897-1058
    const int L = p->L, Lt = p->Lt, kvol = p->kvol;
    const int ksize2 = L * L, nsource = 5;
    const float akappa = 0.5f;
    std::vector<float> cf1(4 * Lt, 0.0f), cf2(4 * Lt, 0.0f);
    std::vector<double> walls(2 * 8 * (size_t)kvol);
    // prop00(kvol,3:4,1:2,2), prop0L(kvol,3:4,3:4,2) complex64
    std::vector<float> prop00(2 * 8 * (size_t)kvol), prop0L(2 * 8 * (size_t)kvol);
    auto PI = [kvol](int64_t i, int a, int b, int f) { return 2 * (i + kvol * (a + 2 * (b + 2 * (int64_t)f))); };
    int iter = 0;
    const int ittt0 = (int)((float)Lt * yferm) + 1;                              // :929
    int ittt = 0;
    // the 2*nsource congrad solves of the loops below (:937-996) are
    // independent and share chi: they run as one batched solve, each with
    // the arithmetic of its own congrad call
    std::vector<int> src_t, src_d, its(2 * nsource);
    for (int ksource = 1; ksource <= nsource; ksource++)
        for (int idsource = 3; idsource <= 4; idsource++) {
            src_t.push_back((ittt0 + ksource * (Lt / nsource)) % Lt + 1);
            src_d.push_back(idsource);
        }
    std::vector<double> all_walls(2 * 8 * (size_t)kvol * 2 * nsource);
    {
        const int rc = chdwf_traj_propagators(p->ctx, 2 * nsource, src_t.data(), src_d.data(),
                                              p->rescgm, p->am, p->hpin, p->imass,
                                              all_walls.data(), its.data());
        if (rc != CHDWF_OK && rc != CHDWF_ITER_CAP) return rc;
        for (int i = 0; i < 2 * nsource; i++)
            if (its[i] >= p->Ls * kvol) p->cg_caps++;    // congrad's message (:1151-1153)
    }
    for (int ksource = 1; ksource <= nsource; ksource++) {
        ittt = (ittt0 + ksource * (Lt / nsource)) % Lt + 1;                        // :937
        for (int idsource = 3; idsource <= 4; idsource++) {
            const int isrc = 2 * (ksource - 1) + (idsource - 3);
            std::memcpy(walls.data(), all_walls.data() + 2 * 8 * (size_t)kvol * isrc,
                        sizeof(double) * 2 * 8 * (size_t)kvol);
            iter += its[isrc];
            // walls[(w*2 + dd)*2 + f][kvol]: w=0 s=1 Dirac 1,2; w=1 s=Ls Dirac 3,4
            for (int f = 0; f < 2; f++)
                for (int dd = 0; dd < 2; dd++)
                    for (int64_t i = 0; i < kvol; i++) {
                        const double* a = &walls[2 * (((0 * 2 + dd) * 2 + f) * (int64_t)kvol + i)];
                        const double* b = &walls[2 * (((1 * 2 + dd) * 2 + f) * (int64_t)kvol + i)];
                        const int64_t pa = PI(i, idsource - 3, dd, f), pb = PI(i, idsource - 3, dd, f);
                        prop00[pa] = (float)a[0];
                        prop00[pa + 1] = (float)a[1];
                        prop0L[pb] = (float)b[0];
                        prop0L[pb + 1] = (float)b[1];
                    }
        }
        // correlators (:1014-1034); gamval(3,3..4)*akappa = (0,+-0.5), gamin = 1,2
        for (int idd = 3; idd <= 4; idd++)
            for (int it = 0; it < Lt; it++) {
                const int itt = (ittt + it - 1) % Lt + 1;
                const int isign = itt >= ittt ? 1 : -1;   // ibound = -1 (:85)
                const int64_t ioff = (int64_t)(itt - 1) * ksize2;
                const double gim = idd == 3 ? 0.5 : -0.5;
                for (int f = 0; f < 2; f++)
                    for (int64_t i = 0; i < ksize2; i++) {
                        const float sk = (float)isign * akappa;
                        const int64_t pl = PI(i + ioff, idd - 3, idd - 3, f);
                        float* c1 = &cf1[2 * (it + Lt * f)];
                        c1[0] = c1[0] + sk * prop0L[pl];
                        c1[1] = c1[1] + sk * prop0L[pl + 1];
                        // (isign*gamval) * prop00, gamval = (0, gim)
                        const double gre = (double)isign * 0.0, gimv = (double)isign * gim;
                        const int64_t p0 = PI(i + ioff, idd - 3, idd - 3, f);
                        const double pr = prop00[p0], pim = prop00[p0 + 1];
                        const double tre = gre * pr - gimv * pim, tim = gre * pim + gimv * pr;
                        float* c2 = &cf2[2 * (it + Lt * f)];
                        c2[0] = (float)((double)c2[0] + tre);
                        c2[1] = (float)((double)c2[1] + tim);
                    }
            }
    }
    for (int i = 0; i < 4 * Lt; i++) {
        cf1[i] = cf1[i] / (float)nsource;
        cf2[i] = cf2[i] / (float)nsource;
    }
    p->cferm.assign(cf1.begin(), cf1.end());
    p->cferm.insert(p->cferm.end(), cf2.begin(), cf2.end());
    *aviter = (float)iter / (float)(2 * nsource);
    return CHDWF_OK;
}

}  // namespace

extern "C" {

int chdwf_prog_create(chdwf_prog** out, int ksize, int ksizet, int kthird, float dt, float beta,
                      float am3, float am, float hpin, int imass, int iterl, int device) {
    if (!out || iterl < 1 || (imass != 1 && imass != 3)) return CHDWF_BAD_ARG;
    chdwf_prog* p = new chdwf_prog();
    int rc = chdwf_create(&p->ctx, ksize, ksizet, kthird, device);
    if (rc != CHDWF_OK) { delete p; return rc; }
    chdwf_set_para(p->ctx, beta, am3, -1);
    p->L = ksize; p->Lt = ksizet; p->Ls = kthird; p->kvol = ksize * ksize * ksizet;
    p->dt = dt; p->beta = beta; p->am3 = am3; p->am = am; p->hpin = hpin;
    p->imass = imass; p->iterl = iterl;
    // sread without a 'con' file (:1467-1468): chi = 0.1/beta, default seed
    std::vector<double> chi(3 * (size_t)p->kvol, (double)(0.1f / beta));
    chdwf_traj_set_chi(p->ctx, chi.data());
    p->rng.startup((double)693764523745.0f);
    p->last_state = p->rng.state();
    *out = p;
    return CHDWF_OK;
}

void chdwf_prog_destroy(chdwf_prog* p) {
    if (!p) return;
    if (p->have_next) p->next.wait();
    p->release_pool();
    chdwf_destroy(p->ctx);
    delete p;
}

// Draw the random inputs of the next ntraj sweeps now and copy them to HBM,
// so those sweeps start with every input resident.
int chdwf_prog_stage(chdwf_prog* p, int ntraj) {
    if (!p || ntraj < 0) return CHDWF_BAD_ARG;
    if (p->have_next) {                  // a prefetched trajectory comes first
        Staged s;
        s.d = p->next.get();
        p->have_next = false;
        p->staged.push_back(std::move(s));
        ntraj--;
    }
    const int base = p->isweep + (int)p->staged.size();
    for (int k = 0; k < ntraj; k++) {
        Staged s;
        s.d = p->draw(base + 1 + k);
        p->staged.push_back(std::move(s));
    }
    for (Staged& s : p->staged) {
        if (s.slot >= 0) continue;
        s.slot = p->take_slot();
        if (s.slot < 0) return CHDWF_CUDA_ERROR;
        const StageSlot& sl = p->pool[s.slot];
        cudaMemcpy(sl.gauss_dev, s.d.gauss.data(), sizeof(float) * s.d.gauss.size(),
                   cudaMemcpyHostToDevice);
        cudaMemcpy(sl.pp_dev, s.d.pp.data(), sizeof(float) * s.d.pp.size(), cudaMemcpyHostToDevice);
    }
    return cudaDeviceSynchronize() == cudaSuccess ? CHDWF_OK : CHDWF_CUDA_ERROR;
}

chdwf_ctx* chdwf_prog_context(chdwf_prog* p) { return p ? p->ctx : nullptr; }

int chdwf_prog_set_remez(chdwf_prog* p, int which, const double* anum, const double* aden,
                         const double* bnum, const double* bden, int ndiag) {
    if (!p) return CHDWF_BAD_ARG;
    return chdwf_traj_set_remez(p->ctx, which, anum, aden, bnum, bden, ndiag);
}

int chdwf_prog_set_chi(chdwf_prog* p, const double* chi) {
    if (!p) return CHDWF_BAD_ARG;
    return chdwf_traj_set_chi(p->ctx, chi);
}

int chdwf_prog_get_chi(chdwf_prog* p, double* chi) {
    if (!p) return CHDWF_BAD_ARG;
    return chdwf_traj_get_chi(p->ctx, chi, 0);
}

int chdwf_prog_startup(chdwf_prog* p, double seed) {
    if (!p) return CHDWF_BAD_ARG;
    p->discard_pending();
    p->rng.startup(seed);
    p->last_state = p->rng.state();
    return CHDWF_OK;
}

// rranget after the last completed sweep (the value the reference would
// checkpoint there)
double chdwf_prog_seed(chdwf_prog* p) {
    if (!p) return 0.0;
    return p->last_state.ds[1] * 16777216.0 + p->last_state.ds[0];
}

struct ProgState {
    chdwf::Rng::State rng;
    int isweep;
    chdwf_run_sums sums;
};

int chdwf_prog_state_size(void) { return (int)sizeof(ProgState); }

int chdwf_prog_get_state(chdwf_prog* p, void* buf, int nbytes) {
    if (!p || !buf || nbytes < (int)sizeof(ProgState)) return CHDWF_BAD_ARG;
    ProgState s;
    s.rng = p->last_state;
    s.isweep = p->isweep;
    s.sums = p->sums;
    std::memcpy(buf, &s, sizeof(s));
    return CHDWF_OK;
}

int chdwf_prog_set_state(chdwf_prog* p, const void* buf, int nbytes) {
    if (!p || !buf || nbytes < (int)sizeof(ProgState)) return CHDWF_BAD_ARG;
    ProgState s;
    std::memcpy(&s, buf, sizeof(s));
    p->discard_pending();
    p->rng.set_state(s.rng);
    p->last_state = s.rng;
    p->isweep = s.isweep;
    p->sums = s.sums;
    return CHDWF_OK;
}

int chdwf_prog_set_measure(chdwf_prog* p, int iprint, int measure) {
    if (!p || iprint < 1) return CHDWF_BAD_ARG;
    p->discard_pending();
    p->iprint = iprint;
    p->measure = measure;
    return CHDWF_OK;
}

int chdwf_prog_set_residuals(chdwf_prog* p, float rescga, float rescgg, float rescgm) {
    if (!p) return CHDWF_BAD_ARG;
    p->rescga = rescga; p->rescgg = rescgg; p->rescgm = rescgm;
    return CHDWF_OK;
}

int chdwf_prog_correlators(chdwf_prog* p, float* cferm) {
    if (!p || !cferm) return CHDWF_BAD_ARG;
    if (p->cferm.empty()) return CHDWF_BAD_ARG;
    std::memcpy(cferm, p->cferm.data(), sizeof(float) * p->cferm.size());
    return CHDWF_OK;
}

int chdwf_prog_set_ext(chdwf_prog* p, int npf, int nsteps, int integrator, float lambda) {
    if (!p || npf < 0 || npf > 4 || nsteps < 1 || (integrator != 0 && integrator != 1))
        return CHDWF_BAD_ARG;
    p->discard_pending();
    p->release_pool();                   // staged buffers are sized by npf
    p->ext_npf = npf;
    p->ext_nsteps = nsteps;
    p->ext_integrator = integrator;
    p->ext_lambda = lambda;
    if (npf == 0) return chdwf_ext_select_pf(p->ctx, 0);
    return CHDWF_OK;
}

namespace {

// One trajectory of the multi-pseudofermion variant: heatbath of every
// field, H0, a fixed number of integrator steps, H1 and the Metropolis test
// (the reference's sequence, rhmc/cheisdwf.f:213-345, with npf fields and
// the chosen integrator).  Omelyan's second-order minimum-norm integrator
// (I.P. Omelyan, I.M. Mryglod, R. Folk, Comput. Phys. Commun. 151 (2003)
// 272) per step: p -= l dt F; chi += dt/2 p; p -= (1-2l) dt F;
// chi += dt/2 p; p -= l dt F, with the last force of a step shared with
// the first of the next (2 nsteps + 1 force evaluations).  Leapfrog: the
// reference's scheme with a fixed step count.
int ext_sweep(chdwf_prog* p, chdwf_sweep_record* rec) {
    chdwf_ctx* c = p->ctx;
    const int kvol = p->kvol, npf = p->ext_npf;
    Staged stg;
    if (!p->staged.empty()) {
        stg = std::move(p->staged.front());
        p->staged.pop_front();
    } else {
        stg.d = p->have_next ? p->next.get() : p->draw_ext();
        p->have_next = false;
    }
    Draws& d = stg.d;
    p->last_state = d.state_after;
    if (stg.slot < 0) {                  // draws not yet in HBM: copy them now
        stg.slot = p->take_slot();
        if (stg.slot < 0) return CHDWF_CUDA_ERROR;
        const StageSlot& s0 = p->pool[stg.slot];
        cudaMemcpy(s0.gauss_dev, d.gauss.data(), sizeof(float) * d.gauss.size(),
                   cudaMemcpyHostToDevice);
        cudaMemcpy(s0.pp_dev, d.pp.data(), sizeof(float) * d.pp.size(), cudaMemcpyHostToDevice);
    }
    struct Back {
        chdwf_prog* p;
        int slot;
        ~Back() { if (slot >= 0) p->free_slots.push_back(slot); }
    } back{p, stg.slot};
    const StageSlot& sl = p->pool[stg.slot];
    int rc;
#define CK(x) do { rc = (x); if (rc != CHDWF_OK) { p->err = chdwf_last_error(c); return rc; } } while (0)
    chdwf_run_sums& A = p->sums;
    CK(chdwf_traj_begin(c));
    const size_t per_pf = 16 * (size_t)kvol * p->Ls;
    for (int i = 0; i < npf; i++) {
        int it = 0;
        CK(chdwf_ext_select_pf(c, i));
        CK(chdwf_ext_heatbath_dev(c, sl.gauss_dev + per_pf * i, p->rescga, p->hpin, p->imass, &it));
        rec->it_pf += it;
    }
    A.ancgpf = A.ancgpf + (float)rec->it_pf;
    if (p->staged.empty()) p->prefetch(p->isweep + 1);
    CK(chdwf_traj_set_momenta_dev(c, sl.pp_dev));
    auto hamiltonian = [&](double* H, double* S, double* hg, double* hp, int* its) -> int {
        double b[2];
        int r2 = chdwf_ext_bosonic(c, b);
        if (r2 != CHDWF_OK) return r2;
        double hf = 0.0;
        for (int i = 0; i < npf; i++) {
            double h = 0.0;
            int it = 0;
            if ((r2 = chdwf_ext_select_pf(c, i)) != CHDWF_OK) return r2;
            if ((r2 = chdwf_ext_action(c, p->rescga, p->hpin, p->imass, &h, &it)) != CHDWF_OK)
                return r2;
            hf += h;
            *its += it;
        }
        *hp = b[0];
        *hg = b[1];
        *H = b[1] + b[0] + hf;
        *S = b[1] + hf;
        return CHDWF_OK;
    };
    double hg = 0.0, hp = 0.0;
    CK(hamiltonian(&rec->H0, &rec->S0, &hg, &hp, &rec->it_h0));
    A.ancgh = A.ancgh + (float)rec->it_h0;
    if (p->isweep == 1) A.gaction = (float)(hg / (double)kvol);
    rec->action = (float)(rec->S0 / (double)kvol);
    rec->paction = (float)(hp / (double)kvol);
    auto force = [&]() -> int {
        for (int i = 0; i < npf; i++) {
            int it = 0, r2;
            if ((r2 = chdwf_ext_select_pf(c, i)) != CHDWF_OK) return r2;
            if ((r2 = chdwf_ext_force(c, p->rescgg, p->hpin, p->imass, i == 0, &it)) != CHDWF_OK)
                return r2;
            rec->it_force += it;
        }
        rec->nforce++;
        return CHDWF_OK;
    };
    const float dt = p->dt;
    const int ns = p->ext_nsteps;
    if (p->ext_integrator == 1) {
        const float l = p->ext_lambda;
        const float d_l = l * dt, d_m = (1.0f - 2.0f * l) * dt, d_2l = 2.0f * l * dt;
        const float half = 0.5f * dt;
        CK(force());
        CK(chdwf_traj_update_momenta(c, d_l));
        for (int k = 1; k <= ns; k++) {
            CK(chdwf_traj_update_chi(c, half));
            CK(force());
            CK(chdwf_traj_update_momenta(c, d_m));
            CK(chdwf_traj_update_chi(c, half));
            CK(force());
            CK(chdwf_traj_update_momenta(c, k < ns ? d_2l : d_l));
        }
    } else {
        CK(force());
        CK(chdwf_traj_update_momenta(c, 0.5f * dt));
        for (int k = 1; k <= ns; k++) {
            CK(chdwf_traj_update_chi(c, dt));
            CK(force());
            CK(chdwf_traj_update_momenta(c, k < ns ? dt : 0.5f * dt));
        }
    }
    rec->nsteps = ns;
    rec->ended = 1;
    A.itot = A.itot + ns;
    A.ancgf = A.ancgf + (float)rec->it_force;
    CK(hamiltonian(&rec->H1, &rec->S1, &rec->hg, &rec->hp, &rec->it_h1));
    A.ancgh = A.ancgh + (float)rec->it_h1;
    rec->dH = rec->H0 - rec->H1;
    rec->dS = rec->S0 - rec->S1;
    rec->y = (float)std::exp(rec->dH);
    A.yav = A.yav + rec->y;
    A.yyav = A.yyav + rec->y * rec->y;
    rec->x = d.x;
    if (rec->x < rec->y) {
        rec->accepted = 1;
        CK(chdwf_traj_accept(c));
        A.naccp = A.naccp + 1;
        rec->action = (float)(rec->S1 / (double)kvol);
        A.gaction = (float)(rec->hg / (double)kvol);
        rec->paction = (float)(rec->hp / (double)kvol);
    }
    rec->gaction = A.gaction;
    A.actiona = A.actiona + rec->action;
    std::vector<float> pp(3 * (size_t)kvol);
    CK(chdwf_traj_get_momenta(c, pp.data()));
    float vel2 = 0.0f;
    for (size_t i = 0; i < pp.size(); i++) vel2 = vel2 + pp[i] * pp[i];
    rec->vel2 = vel2 / (float)kvol;
    A.vel2a = A.vel2a + rec->vel2;
    A.nsweep = A.nsweep + 1;
#undef CK
    return CHDWF_OK;
}

}  // namespace

// One sweep of the main loop (rhmc/cheisdwf.f:207-399).
int chdwf_prog_sweep(chdwf_prog* p, chdwf_sweep_record* rec) {
    if (!p || !rec) return CHDWF_BAD_ARG;
    std::memset(rec, 0, sizeof(*rec));
    if (p->ext_npf > 0) {
        p->isweep++;
        return ext_sweep(p, rec);
    }
    chdwf_ctx* c = p->ctx;
    const int kvol = p->kvol;
    p->isweep++;
    Staged stg;
    const bool from_stage = !p->staged.empty();
    if (from_stage) {
        stg = std::move(p->staged.front());
        p->staged.pop_front();
    } else {
        stg.d = p->have_next ? p->next.get() : p->draw(p->isweep);
        p->have_next = false;
    }
    Draws& d = stg.d;
    p->last_state = d.state_after;
    struct Back {                    // the slot returns to the pool, whatever the outcome
        chdwf_prog* p;
        int slot;
        ~Back() { if (slot >= 0) p->free_slots.push_back(slot); }
    } back{p, stg.slot};
    const StageSlot* sl = stg.slot >= 0 ? &p->pool[stg.slot] : nullptr;
    int rc;
#define CK(x) do { rc = (x); if (rc != CHDWF_OK) { p->err = chdwf_last_error(c); return rc; } } while (0)
    CK(chdwf_traj_begin(c));                                                        // :213-216
    if (from_stage)
        CK(chdwf_traj_heatbath_dev(c, sl->gauss_dev, p->rescga, p->am, p->hpin, p->imass,
                                   &rec->it_pf));                                   // :218-245
    else
        CK(chdwf_traj_heatbath(c, d.gauss.data(), p->rescga, p->am, p->hpin, p->imass,
                               &rec->it_pf));
    chdwf_run_sums& A = p->sums;
    A.ancgpf = A.ancgpf + (float)rec->it_pf;                                       // :235
    if (p->staged.empty()) p->prefetch(p->isweep + 1);   // next trajectory's draws, overlapped
    if (from_stage) CK(chdwf_traj_set_momenta_dev(c, sl->pp_dev));                 // :249-257
    else CK(chdwf_traj_set_momenta(c, d.pp.data()));
    double h[5];
    CK(chdwf_traj_hamilton(c, p->rescga, p->am, p->hpin, p->imass, h, &rec->it_h0));  // :261
    A.ancgh = A.ancgh + (float)rec->it_h0;                                          // :575
    rec->H0 = h[0];
    rec->S0 = h[3];
    if (p->isweep == 1) A.gaction = (float)(h[1] / (double)kvol);
    rec->action = (float)(h[3] / (double)kvol);
    rec->paction = (float)(h[2] / (double)kvol);
    int itg = 0, itf = 0;
    auto force_sums = [&] {                                                         // :507, :515
        A.ancg = A.ancg + (float)itg;
        A.ancgf = A.ancgf + (float)itf;
        rec->it_guid += itg; rec->it_force += itf; rec->nforce++;
    };
    CK(chdwf_traj_force(c, p->rescgg, p->am, p->hpin, p->imass, &itg, &itf));       // :272
    force_sums();
    CK(chdwf_traj_update_momenta(c, p->dt * 0.5f));                                 // :273-277
    const int nsteps = (int)d.ytest.size();
    const float proby = 1.0f / (float)p->iterl;
    for (int iter = 1; iter <= nsteps; iter++) {                                    // :281-315
        CK(chdwf_traj_update_chi(c, p->dt));
        CK(chdwf_traj_force(c, p->rescgg, p->am, p->hpin, p->imass, &itg, &itf));
        force_sums();
        rec->nsteps = iter;
        if (d.ytest[iter - 1] < proby) {
            CK(chdwf_traj_update_momenta(c, p->dt * 0.5f));
            rec->ended = 1;
            A.itot = A.itot + iter;                                                 // :305
            break;
        }
        CK(chdwf_traj_update_momenta(c, p->dt));
    }
    CK(chdwf_traj_hamilton(c, p->rescga, p->am, p->hpin, p->imass, h, &rec->it_h1));  // :321
    A.ancgh = A.ancgh + (float)rec->it_h1;
    rec->H1 = h[0]; rec->S1 = h[3]; rec->hg = h[1]; rec->hp = h[2];
    rec->dH = rec->H0 - rec->H1;
    rec->dS = rec->S0 - rec->S1;
    rec->y = (float)std::exp(rec->dH);
    A.yav = A.yav + rec->y;                                                         // :326-327
    A.yyav = A.yyav + rec->y * rec->y;
    rec->x = d.x;
    rec->accepted = 0;
    if (rec->x < rec->y) {                                                          // :331-344
        rec->accepted = 1;
        CK(chdwf_traj_accept(c));
        A.naccp = A.naccp + 1;
        rec->action = (float)(h[3] / (double)kvol);
        A.gaction = (float)(h[1] / (double)kvol);
        rec->paction = (float)(h[2] / (double)kvol);
    }
    rec->gaction = A.gaction;           // kept from the last sweep that set it (:264, :342)
    A.actiona = A.actiona + rec->action;                                            // :348
    std::vector<float> pp(3 * (size_t)kvol);
    CK(chdwf_traj_get_momenta(c, pp.data()));
    float vel2 = 0.0f;                                                              // :349-355
    for (size_t i = 0; i < pp.size(); i++) vel2 = vel2 + pp[i] * pp[i];
    rec->vel2 = vel2 / (float)kvol;
    A.vel2a = A.vel2a + rec->vel2;                                                  // :356
    if (d.measured) {                                                               // :359-399
        rec->measured = 1;
        CK(chdwf_traj_begin(c));                                                    // chit = chi
        std::vector<double> chi(3 * (size_t)kvol);
        CK(chdwf_traj_get_chi(c, chi.data(), 0));
        float susctot = 0.0f, condmod = 0.0f;
        for (int a = 0; a < 3; a++) {
            float cnd = 0.0f;
            for (int i = 0; i < kvol; i++) cnd = (float)((double)cnd + chi[i + (size_t)kvol * a]);
            float su = cnd * cnd;
            cnd = cnd / (float)kvol;
            condmod = condmod + cnd * cnd;
            su = su / (float)kvol;
            susctot = susctot + su;
            rec->cond[a] = cnd;
            rec->susc[a] = su;
        }
        rec->condmod = std::sqrt(condmod);
        rec->susctot = susctot;
        A.condmoda = A.condmoda + rec->condmod;                                     // :382-386
        A.susca = A.susca + susctot;
        for (int a = 0; a < 3; a++) A.conda[a] = A.conda[a] + rec->cond[a];
        CK(fermion(p, d.yferm, &rec->ancgm));
        A.pbpa = A.pbpa + 0.0f;             // pbp: 'measure' is not called (:392-394)
        A.ancgma = A.ancgma + rec->ancgm;                                           // :395-396
        A.ipbp = A.ipbp + 1;
    }
    A.nsweep = A.nsweep + 1;
#undef CK
    return CHDWF_OK;
}

int chdwf_prog_measure(chdwf_prog* p, float res, float* psibarpsi, float* susclsing,
                       float* aviter, double* parts) {
    // measure(psibarpsi, res, aviter, am, hpin, imass), rhmc/cheisdwf.f:1164-1453,
    // on chi with the program's am, hpin, imass (1 or 3)
    if (!p || !psibarpsi || !susclsing || !aviter) return CHDWF_BAD_ARG;
    if (p->imass != 1 && p->imass != 3) return CHDWF_BAD_ARG;
    chdwf_ctx* c = p->ctx;
    const int64_t kvol = p->kvol;
    constexpr int knoise = 10;
    p->discard_pending();                 // the draws continue the generator's stream
    int rc = chdwf_traj_begin(c);         // the solves run on chit = chi
    if (rc != CHDWF_OK) { p->err = chdwf_last_error(c); return rc; }
    std::vector<float> ps(2 * kvol), pt(2 * kvol);
    std::vector<double> slice(4 * kvol);
    float pbp[knoise];
    int iter = 0;
    for (int inoise = 0; inoise < knoise; inoise++) {
        p->rng.gauss0(kvol, ps.data());                                            // :1187
        p->rng.gauss0(kvol, pt.data());                                            // :1189
        double p1r = 0.0, p1i = 0.0, p2r = 0.0, p2i = 0.0;
        for (int idsource = 1; idsource <= 2; idsource++) {
            for (int w = 0; w < 2; w++) {
                // w=0: ps on s=1, Dirac idsource, read s=kthird (:1194-1294);
                // w=1: pt on s=kthird, Dirac idsource+2, read s=1 (:1303-1393)
                const float* eta = w == 0 ? ps.data() : pt.data();
                const int d = w == 0 ? idsource : idsource + 2;
                int it = 0;
                rc = chdwf_traj_noise_solve(c, eta, w == 0 ? 1 : p->Ls, d, res, p->am, p->hpin,
                                            p->imass, slice.data(), &it);
                if (rc != CHDWF_OK && rc != CHDWF_ITER_CAP) {
                    p->err = chdwf_last_error(c);
                    p->last_state = p->rng.state();
                    return rc;
                }
                if (rc == CHDWF_ITER_CAP) p->cg_caps++;
                iter += it;
                double ar = w == 0 ? p1r : p2r, ai = w == 0 ? p1i : p2i;
                for (int64_t t = 0; t < 2 * kvol; t++) {       // f outer, i inner
                    const int64_t i = t % kvol;
                    const double xr = (double)eta[i], xi = (double)eta[kvol + i];
                    const double yr = slice[2 * t], yi = slice[2 * t + 1];
                    // conjg(x)*y, then the running sum
                    const double mr = xr * yr - (-xi) * yi, mi = xr * yi + (-xi) * yr;
                    ar = ar + mr;
                    ai = ai + mi;
                }
                if (w == 0) { p1r = ar; p1i = ai; } else { p2r = ar; p2i = ai; }
            }
        }
        const double kv = (double)kvol;
        if (p->imass == 1) {                                                      // :1418-1421
            p1r = p1r / kv; p1i = p1i / kv;
            p2r = p2r / kv; p2i = p2i / kv;
        } else {                                                                  // :1422-1425
            // (0,-1)*p1 and (0,+1)*p2 as complex products
            const double a1 = 0.0 * p1r - (-1.0) * p1i, b1 = 0.0 * p1i + (-1.0) * p1r;
            const double a2 = 0.0 * p2r - 1.0 * p2i, b2 = 0.0 * p2i + 1.0 * p2r;
            p1r = a1 / kv; p1i = b1 / kv;
            p2r = a2 / kv; p2i = b2 / kv;
        }
        pbp[inoise] = (float)(p1r + p2r);
        if (parts) {                                                              // write(100)
            parts[4 * inoise] = p1r; parts[4 * inoise + 1] = p1i;
            parts[4 * inoise + 2] = p2r; parts[4 * inoise + 3] = p2i;
        }
    }
    p->last_state = p->rng.state();
    float pb = 0.0f, sus = 0.0f;                                                  // :1440-1449
    for (int i = 0; i < knoise; i++) {
        pb = pb + pbp[i];
        for (int j = knoise - 1; j >= i + 1; j--) sus = sus + pbp[i] * pbp[j];
    }
    *psibarpsi = pb / (float)knoise;
    *susclsing = (float)(2 * kvol) * sus / (float)(knoise * (knoise - 1));
    *aviter = (float)iter / (float)(4 * knoise);                                  // :1451
    return CHDWF_OK;
}

const char* chdwf_prog_last_error(chdwf_prog* p) { return p ? p->err.c_str() : ""; }

int chdwf_prog_sums(chdwf_prog* p, chdwf_run_sums* out) {
    if (!p || !out) return CHDWF_BAD_ARG;
    *out = p->sums;
    return CHDWF_OK;
}

int chdwf_prog_reset_sums(chdwf_prog* p) {
    if (!p) return CHDWF_BAD_ARG;
    const float g = p->sums.gaction;
    p->sums = chdwf_run_sums{};
    p->sums.gaction = g;
    return CHDWF_OK;
}

// Averages printed at the end of a run (rhmc/cheisdwf.f:413-431), in the
// reference's REAL*4 arithmetic and evaluation order.
int chdwf_prog_averages(chdwf_prog* p, chdwf_run_averages* out) {
    if (!p || !out) return CHDWF_BAD_ARG;
    const chdwf_run_sums& A = p->sums;
    const int iter2 = A.nsweep;
    if (iter2 < 1) return CHDWF_BAD_ARG;
    chdwf_run_averages v{};
    v.iter2 = iter2;
    v.naccp = A.naccp;
    const float n = (float)iter2, np = (float)A.ipbp, nt = (float)A.itot;
    v.actiona = A.actiona / n;
    v.vel2a = A.vel2a / n;
    v.condmoda = A.condmoda / np;
    v.susca = A.susca / np;
    for (int a = 0; a < 3; a++) v.conda[a] = A.conda[a] / np;
    v.pbpa = A.pbpa / np;
    v.ancg = A.ancg / nt;
    v.ancgf = A.ancgf / nt;
    v.ancgh = A.ancgh / (float)(2 * iter2);
    v.ancgpf = A.ancgpf / n;
    v.ancgma = A.ancgma / np;
    v.yav = A.yav / n;
    const float yy = A.yyav / n - v.yav * v.yav;
    v.yyav = std::sqrt(yy / (float)(iter2 - 1));
    v.atraj = p->dt * (float)A.itot / n;
    *out = v;
    return CHDWF_OK;
}

// sread (rhmc/cheisdwf.f:1455-1478)
int chdwf_prog_read_con(chdwf_prog* p, const char* path, double* seed) {
    if (!p || !path || !seed) return CHDWF_BAD_ARG;
    std::vector<double> chi(3 * (size_t)p->kvol);
    const int rc = chdwf::fio::con_read(path, p->kvol, chi.data(), seed, nullptr);
    if (rc == 2) {
        p->err = std::string("not a configuration of this lattice: ") + path;
        return CHDWF_BAD_ARG;
    }
    if (rc == 1) {                       // no 'con': chi = 0.1/beta, default seed (:1468-1469)
        std::fill(chi.begin(), chi.end(), (double)(0.1f / p->beta));
        *seed = (double)693764523745.0f;
    }
    p->discard_pending();
    return chdwf_traj_set_chi(p->ctx, chi.data());
}

// rranget + swrite (rhmc/cheisdwf.f:402-404, :1480-1489)
int chdwf_prog_write_con(chdwf_prog* p, const char* path) {
    if (!p || !path) return CHDWF_BAD_ARG;
    std::vector<double> chi(3 * (size_t)p->kvol);
    const int rc = chdwf_traj_get_chi(p->ctx, chi.data(), 0);
    if (rc != CHDWF_OK) return rc;
    if (chdwf::fio::con_write(path, p->kvol, chi.data(), chdwf_prog_seed(p)) != 0) {
        p->err = std::string("cannot write ") + path;
        return CHDWF_BAD_ARG;
    }
    return CHDWF_OK;
}

int chdwf_prog_take_cg_caps(chdwf_prog* p) {
    if (!p) return 0;
    const int n = p->cg_caps;
    p->cg_caps = 0;
    return n;
}

}  // extern "C"
