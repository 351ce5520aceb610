"""CPU check of the element arithmetic of three CUDA kernel families against
the oracle, bit for bit, without a GPU.

The FP64 RHMC operator (dwf_apply_flavour of chiralheisenberg_b200/csrc/
dwf_stencil.cuh, the body of every FP64 M and M^dagger kernel), the
single-precision HMC operator and force (csrc/hmc.cu) and the Thirring link
operator, coef and derivs (csrc/thirring.cu) compute each output element in
registers with round-to-nearest intrinsics (__dadd_rn, __fmul_rn, ...) and
no fused multiply-add.  Host IEEE arithmetic
compiled with -ffp-contract=off rounds the same way, so the same element
functions, compiled for the host with those intrinsics mapped to plain
operators, must reproduce the oracle's sequential sweeps exactly.  This test
includes dwf_stencil.cuh as it is (with host stand-ins for the warp and
atomic intrinsics of common.cuh, which the element function does not
call), extracts the element functions and per-element kernels of the two
.cu files (between the section comments named below), compiles each with
g++ into a small program, runs every element over random inputs, and
compares.

A fourth program compares the FP32 two-point operator on the solver's
split vector layout (dwf_apply_flavour_pair_sp, whose additions are packed
FP32x2 instructions on the GPU) with the plain-layout one, element by
element, and a fifth checks that layout's element accessors.

It checks the arithmetic of the kernel bodies only; the device build, the
launch shapes and the solvers are checked by the -m gpu tests.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "chiralheisenberg_b200", "csrc")
CUDA_INC = "/usr/local/cuda/include"

PRELUDE = r'''
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>
#define __forceinline__
#define __constant__
static int64_t g_tid;
static const int kThreads = 256;
static inline float __fadd_rn(float a, float b) { return a + b; }
static inline float __fsub_rn(float a, float b) { return a - b; }
static inline float __fmul_rn(float a, float b) { return a * b; }
static inline double __dadd_rn(double a, double b) { return a + b; }
static inline double __dsub_rn(double a, double b) { return a - b; }
static inline double __dmul_rn(double a, double b) { return a * b; }
static inline float __double2float_rn(double a) { return (float)a; }
template <class T> static inline T __ldg(const T* p) { return *p; }
'''

ZOPS = r'''
static inline double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
static inline double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
static inline double2 zscal(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
static inline double2 zmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
static inline double2 zconj(double2 a) { return make_double2(a.x, -a.y); }
'''

HMC_MAIN = r'''
struct Geom { int L, Lt, Ls; int kvol; int64_t npts, cs, kferm; };
int main(int argc, char** argv) {
    int L = atoi(argv[1]), Lt = atoi(argv[2]), Ls = atoi(argv[3]), imass = atoi(argv[4]);
    float beta = atof(argv[5]);
    Geom g; g.L = L; g.Lt = Lt; g.Ls = Ls; g.kvol = L * L * Lt; g.npts = (int64_t)g.kvol * Ls;
    g.cs = g.npts; g.kferm = 8 * g.npts;
    std::vector<float2> R(g.kferm), out(g.kferm), outd(g.kferm);
    std::vector<float> chi(3 * g.kvol), dS(3 * g.kvol);
    FILE* f = fopen(argv[6], "rb");
    if (fread(R.data(), sizeof(float2), g.kferm, f) != (size_t)g.kferm) return 1;
    if (fread(chi.data(), 4, 3 * g.kvol, f) != (size_t)(3 * g.kvol)) return 1;
    fclose(f);
    const float diag = (3.0f - 1.0f) + 1.0f;
    for (g_tid = 0; g_tid < g.kferm; g_tid++) {
        if (imass == 1) { k_hmc_dslash<false,1>(out.data(), R.data(), chi.data(), g, diag, 1);
                          k_hmc_dslash<true,1>(outd.data(), R.data(), chi.data(), g, diag, 1); }
        else { k_hmc_dslash<false,3>(out.data(), R.data(), chi.data(), g, diag, 1);
               k_hmc_dslash<true,3>(outd.data(), R.data(), chi.data(), g, diag, 1); }
    }
    for (g_tid = 0; g_tid < g.kvol; g_tid++) {
        if (imass == 1) k_hmc_derivs<1>(R.data(), chi.data(), g, 2.0f * beta, diag, 1, dS.data());
        else k_hmc_derivs<3>(R.data(), chi.data(), g, 2.0f * beta, diag, 1, dS.data());
    }
    f = fopen(argv[7], "wb");
    fwrite(out.data(), sizeof(float2), g.kferm, f); fwrite(outd.data(), sizeof(float2), g.kferm, f);
    fwrite(dS.data(), 4, 3 * g.kvol, f); fclose(f);
    return 0;
}
'''

THR_MAIN = r'''
int main(int argc, char** argv) {
    int L = atoi(argv[1]), Lt = atoi(argv[2]), Ls = atoi(argv[3]), imass = atoi(argv[4]);
    float am = atof(argv[5]); double anum = atof(argv[6]);
    TGeom g; g.L = L; g.Lt = Lt; g.Ls = Ls; g.kvol = L * L * Lt; g.kferm = 4 * (int64_t)g.kvol * Ls;
    const int64_t n3 = 3 * (int64_t)g.kvol;
    std::vector<double2> R(g.kferm), X2(g.kferm), u(n3), out(g.kferm), outd(g.kferm);
    std::vector<float> theta(n3), dS0(n3, 0.f), dS1(n3, 0.f);
    FILE* f = fopen(argv[7], "rb");
    if (fread(R.data(), 16, g.kferm, f) != (size_t)g.kferm) return 1;
    if (fread(X2.data(), 16, g.kferm, f) != (size_t)g.kferm) return 1;
    if (fread(theta.data(), 4, n3, f) != (size_t)n3) return 1;
    fclose(f);
    for (g_tid = 0; g_tid < n3; g_tid++) k_thr_coef(theta.data(), u.data(), g);
    const double diag = (double)((3.0f - 1.0f) + 1.0f);
    for (int dag = 0; dag < 2; dag++) {
        double2 zk = imass == 1 ? make_double2((double)am, 0.0)
                                : make_double2(0.0, dag ? (double)am : (double)(-am));
        double2* o = dag ? outd.data() : out.data();
        for (g_tid = 0; g_tid < g.kferm; g_tid++) {
            if (!dag) { if (imass == 1) k_thr_dslash<false,1>(o, R.data(), u.data(), g, diag, zk, nullptr, 0);
                        else if (imass == 3) k_thr_dslash<false,3>(o, R.data(), u.data(), g, diag, zk, nullptr, 0);
                        else k_thr_dslash<false,5>(o, R.data(), u.data(), g, diag, zk, nullptr, 0); }
            else { if (imass == 1) k_thr_dslash<true,1>(o, R.data(), u.data(), g, diag, zk, nullptr, 0);
                   else if (imass == 3) k_thr_dslash<true,3>(o, R.data(), u.data(), g, diag, zk, nullptr, 0);
                   else k_thr_dslash<true,5>(o, R.data(), u.data(), g, diag, zk, nullptr, 0); }
        }
    }
    const double tz = (double)(float)(2.0 * anum);
    for (g_tid = 0; g_tid < n3; g_tid++) {
        k_thr_derivs(R.data(), X2.data(), g, tz, 0, dS0.data());
        k_thr_derivs(R.data(), X2.data(), g, tz, 1, dS1.data());
    }
    f = fopen(argv[8], "wb");
    fwrite(u.data(), 16, n3, f); fwrite(out.data(), 16, g.kferm, f); fwrite(outd.data(), 16, g.kferm, f);
    fwrite(dS0.data(), 4, n3, f); fwrite(dS1.data(), 4, n3, f); fclose(f);
    return 0;
}
'''


RHMC_PROGRAM = r'''
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cstring>
#define __forceinline__ inline
#define __shared__
static inline double __dadd_rn(double a, double b) { return a + b; }
static inline double __dsub_rn(double a, double b) { return a - b; }
static inline double __dmul_rn(double a, double b) { return a * b; }
static inline float __fadd_rn(float a, float b) { return a + b; }
static inline float __fsub_rn(float a, float b) { return a - b; }
static inline float __fmul_rn(float a, float b) { return a * b; }
template <class T> static inline T __ldg(const T* p) { return *p; }
static uint3 threadIdx, blockIdx;
static dim3 blockDim, gridDim;
static inline double __shfl_down_sync(unsigned, double v, int) { return v; }
static inline void __syncthreads() {}
static inline void __threadfence() {}
static inline unsigned atomicAdd(unsigned* p, unsigned v) { unsigned o = *p; *p += v; return o; }
#include "dwf_stencil.cuh"
using namespace chdwf;
struct Ld { const double2* p; double2 operator()(int64_t j) const { return p[j]; } };
int main(int argc, char** argv) {
    int L = atoi(argv[1]), Lt = atoi(argv[2]), Ls = atoi(argv[3]), imass = atoi(argv[4]);
    int dag = atoi(argv[5]);
    double hpin = atof(argv[6]);
    Geom g = make_geom(L, Lt, Ls);
    std::vector<double2> R(g.kferm), out(g.kferm);
    std::vector<float> chif(3 * g.kvol);
    FILE* f = fopen(argv[7], "rb");
    if (fread(R.data(), 16, g.kferm, f) != (size_t)g.kferm) return 1;
    if (fread(chif.data(), 4, 3 * g.kvol, f) != (size_t)(3 * g.kvol)) return 1;
    fclose(f);
    const double diag = (double)(2.0f * ((3.0f - 1.0f) + 1.0f));
    const Ld ld{R.data()};
    for (int64_t p = 0; p < g.npts; p++) {
        const PointIdx q = point_of(g, p);
        for (int fl = 0; fl < 2; fl++) {
            double2 acc[4];
            if (dag) {
                if (imass == 1) dwf_apply_flavour<true, 1>(acc, ld, g, q, fl, chif.data(), diag, hpin, true);
                else dwf_apply_flavour<true, 3>(acc, ld, g, q, fl, chif.data(), diag, hpin, true);
            } else {
                if (imass == 1) dwf_apply_flavour<false, 1>(acc, ld, g, q, fl, chif.data(), diag, hpin, true);
                else dwf_apply_flavour<false, 3>(acc, ld, g, q, fl, chif.data(), diag, hpin, true);
            }
            for (int d = 0; d < 4; d++) out[p + g.cs * (d + 4 * fl)] = acc[d];
        }
    }
    f = fopen(argv[8], "wb");
    fwrite(out.data(), 16, g.kferm, f);
    fclose(f);
    return 0;
}
'''


# The FP32 two-point operator in both vector layouts: the plain one
# (dwf_apply_flavour_pair, the standalone FP32 operator) and the split layout
# of the solver's Krylov vectors (dwf_apply_flavour_pair_sp).  Every element
# must come out with the same bits.  Prints the number of differing elements.
SPLIT_PROGRAM = RHMC_PROGRAM.split("using namespace chdwf;")[0] + r"""
using namespace chdwf;
int main(int argc, char** argv) {
    int L = atoi(argv[1]), Lt = atoi(argv[2]), Ls = atoi(argv[3]);
    Geom g = make_geom(L, Lt, Ls);
    std::vector<float2> in(g.kferm), insp(g.kferm);
    std::vector<float> chif(3 * g.kvol);
    FILE* f = fopen(argv[4], "rb");
    if (fread(in.data(), 8, g.kferm, f) != (size_t)g.kferm) return 1;
    if (fread(chif.data(), 4, 3 * g.kvol, f) != (size_t)(3 * g.kvol)) return 1;
    fclose(f);
    float* sp = reinterpret_cast<float*>(insp.data());
    for (int64_t e = 0; e < g.kferm; e += 2) {
        sp[2 * e] = in[e].x; sp[2 * e + 1] = in[e + 1].x;
        sp[2 * e + 2] = in[e].y; sp[2 * e + 3] = in[e + 1].y;
    }
    const float diag = 2.0f * ((3.0f - 1.0f) + 1.0f), hpin = 0.3f;
    long long bad = 0, n = 0;
    for (int dag = 0; dag < 2; dag++)
    for (int imass = 1; imass <= 3; imass += 2)
    for (int apbc = 0; apbc < 2; apbc++)
    for (int64_t p = 0; p < g.npts; p += 2) {
        const PointIdx q = point_of(g, p);
        for (int fl = 0; fl < 2; fl++) {
            float2 a[2][4];
            cpair c[4];
#define RUN(D, I) { dwf_apply_flavour_pair<D, I>(a, in.data(), g, q, fl, chif.data(), diag, hpin, apbc); \
                    dwf_apply_flavour_pair_sp<D, I>(c, insp.data(), g, q, fl, chif.data(), diag, hpin, apbc); }
            if (dag) { if (imass == 1) RUN(true, 1) else RUN(true, 3) }
            else { if (imass == 1) RUN(false, 1) else RUN(false, 3) }
#undef RUN
            for (int d = 0; d < 4; d++)
                for (int k = 0; k < 2; k++) {
                    const float2 v = cpair_pt(c[d], k);
                    n++;
                    if (memcmp(&v, &a[k][d], sizeof(float2)) != 0) bad++;
                }
        }
    }
    printf("%lld %lld\n", bad, n);
    return 0;
}
"""


# Element accessors of the split layout (common.cuh): sp_put of a plain
# vector, read back with sp_get and as element pairs with ld_cpair /
# cpair_pt, then a st_cpair round trip.  Prints the number of mismatches.
ACCESS_PROGRAM = RHMC_PROGRAM.split("using namespace chdwf;")[0] + r"""
using namespace chdwf;
int main(int argc, char** argv) {
    const int64_t n = atoll(argv[1]);
    std::vector<float2> plain(n), sp(n), back(n);
    for (int64_t e = 0; e < n; e++) plain[e] = make_float2(0.5f * e + 0.25f, -1.0f * e - 0.75f);
    for (int64_t e = n - 1; e >= 0; e--) sp_put(sp.data(), e, plain[e]);   // any order
    long long bad = 0;
    for (int64_t e = 0; e < n; e++) {
        const float2 v = sp_get(sp.data(), e);
        if (v.x != plain[e].x || v.y != plain[e].y) bad++;
    }
    const float* f = reinterpret_cast<const float*>(sp.data());
    for (int64_t e = 0; e < n; e += 2) {
        if (f[2 * e] != plain[e].x || f[2 * e + 1] != plain[e + 1].x ||
            f[2 * e + 2] != plain[e].y || f[2 * e + 3] != plain[e + 1].y) bad++;
        const cpair c = ld_cpair(sp.data(), (uint32_t)e);
        for (int k = 0; k < 2; k++) {
            const float2 v = cpair_pt(c, k);
            if (v.x != plain[e + k].x || v.y != plain[e + k].y) bad++;
        }
        st_cpair(back.data(), (uint32_t)e, c);
    }
    if (memcmp(back.data(), sp.data(), sizeof(float2) * n) != 0) bad++;
    printf("%lld\n", bad);
    return 0;
}
"""


def _section(src, start, end):
    a, b = src.find(start), src.find(end)
    assert a >= 0 and b > a, f"section markers moved: {start!r} .. {end!r}"
    return src[a:b]


def _hostify(body):
    body = body.replace("__global__ void __launch_bounds__(kThreads)", "void")
    body = body.replace("__global__ void", "void")
    return body.replace("blockIdx.x * (int64_t)blockDim.x + threadIdx.x", "g_tid")


def _build(tmp, name, code, extra=()):
    cxx = shutil.which("g++")
    if cxx is None or not os.path.isdir(CUDA_INC):
        pytest.skip("needs g++ and the CUDA headers")
    src = os.path.join(tmp, name + ".cpp")
    exe = os.path.join(tmp, name)
    with open(src, "w") as f:
        f.write(code)
    subprocess.run([cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-w", "-I", CUDA_INC,
                    *extra, "-o", exe, src], check=True)
    return exe


@pytest.fixture(scope="module")
def rhmc_exe(tmp_path_factory):
    return _build(str(tmp_path_factory.mktemp("rhmc")), "rhmc", RHMC_PROGRAM,
                  extra=["-I", CSRC])


@pytest.fixture(scope="module")
def split_exe(tmp_path_factory):
    return _build(str(tmp_path_factory.mktemp("split")), "split", SPLIT_PROGRAM,
                  extra=["-I", CSRC])


@pytest.fixture(scope="module")
def access_exe(tmp_path_factory):
    return _build(str(tmp_path_factory.mktemp("access")), "access", ACCESS_PROGRAM,
                  extra=["-I", CSRC])


@pytest.fixture(scope="module")
def hmc_exe(tmp_path_factory):
    src = open(os.path.join(CSRC, "hmc.cu")).read()
    body = _section(src, "// ---- REAL*4 complex arithmetic", "// ---- congrad (mh/cheisdwf_hmc.f:625-716)")
    body += _section(src, "template <int IMASS>\n__global__ void __launch_bounds__(kThreads) k_hmc_derivs",
                     "// R(s, i, d, f) = cmplx")
    code = PRELUDE + HMC_MAIN.split("int main")[0] + "namespace X {\n" + _hostify(body) + \
        "}\nusing namespace X;\nint main" + HMC_MAIN.split("int main")[1]
    return _build(str(tmp_path_factory.mktemp("hmc")), "hmc", code)


@pytest.fixture(scope="module")
def thr_exe(tmp_path_factory):
    src = open(os.path.join(CSRC, "thirring.cu")).read()
    body = _section(src, "struct TGeom {", "// ---- multi-shift solver kernels")
    code = PRELUDE + ZOPS + "namespace X {\n" + _hostify(body) + "}\nusing namespace X;\n" + THR_MAIN
    return _build(str(tmp_path_factory.mktemp("thr")), "thr", code)


@pytest.mark.parametrize("shape", [(4, 4, 4), (3, 2, 5), (6, 4, 8)])
@pytest.mark.parametrize("imass", [1, 3])
@pytest.mark.parametrize("dag", [0, 1])
def test_rhmc_fp64_operator_element_matches_oracle(rhmc_exe, tmp_path, shape, imass, dag):
    """The FP64 M and M^dagger element function, with the pinning term."""
    L, Lt, Ls = shape
    rng = np.random.default_rng(L * 100 + Lt * 10 + Ls + imass)
    lat = po.make_lat(L, Lt, Ls, beta=0.475)
    sh = po.spinor_shape(lat)
    R = rng.standard_normal(sh) + 1j * rng.standard_normal(sh)
    chi = rng.standard_normal((3, L * L * Lt))
    hpin = np.float32(0.3)
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(fin, "wb") as f:
        f.write(R.tobytes())
        f.write(chi.astype(np.float32).tobytes())
    subprocess.run([rhmc_exe, str(L), str(Lt), str(Ls), str(imass), str(dag), repr(float(hpin)),
                    fin, fout], check=True)
    out = np.fromfile(fout, dtype=np.complex128).reshape(sh)
    assert np.array_equal(out, po.dslash(lat, R, chi, hpin=hpin, imass=imass, dag=bool(dag)))


@pytest.mark.parametrize("shape", [(4, 4, 4), (3, 2, 6), (6, 4, 8), (4, 3, 2)])
def test_fp32_split_layout_matches_plain_pair(split_exe, tmp_path, shape):
    """The FP32 solver's split-layout two-point operator (packed on the GPU)
    against the plain-layout one: same bits for M and M^dagger, both mass
    terms, both time boundaries, the pinning term, Ls = 2 included."""
    L, Lt, Ls = shape
    rng = np.random.default_rng(L * 100 + Lt * 10 + Ls)
    n = 8 * L * L * Lt * Ls
    R = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    chi = rng.standard_normal(3 * L * L * Lt).astype(np.float32)
    fin = str(tmp_path / "in.bin")
    with open(fin, "wb") as f:
        f.write(R.tobytes())
        f.write(chi.tobytes())
    out = subprocess.run([split_exe, str(L), str(Lt), str(Ls), fin], check=True,
                         capture_output=True, text=True).stdout.split()
    bad, total = int(out[0]), int(out[1])
    assert total == 2 * 2 * 2 * n and bad == 0, (bad, total)


def test_split_layout_accessors(access_exe):
    """sp_put / sp_get / ld_cpair / st_cpair agree with the split layout's
    definition: element pair (e, e+1), e even, stored as (re_e, re_e+1,
    im_e, im_e+1)."""
    out = subprocess.run([access_exe, "4096"], check=True, capture_output=True,
                         text=True).stdout.split()
    assert int(out[0]) == 0


@pytest.mark.parametrize("shape", [(4, 4, 4), (3, 2, 5), (6, 4, 8)])
@pytest.mark.parametrize("imass", [1, 3])
def test_hmc_element_kernels_match_oracle(hmc_exe, tmp_path, shape, imass):
    L, Lt, Ls = shape
    rng = np.random.default_rng(L * 100 + Lt * 10 + Ls + imass)
    sh = (2, 4, Lt, L, L, Ls)
    R = (rng.standard_normal(sh) + 1j * rng.standard_normal(sh)).astype(np.complex64)
    chi = (0.7 * rng.standard_normal((3, L * L * Lt))).astype(np.float32)
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(fin, "wb") as f:
        f.write(R.tobytes())
        f.write(chi.tobytes())
    subprocess.run([hmc_exe, str(L), str(Lt), str(Ls), str(imass), "0.475", fin, fout], check=True)
    raw = np.fromfile(fout, dtype=np.uint8)
    n = R.size * 8
    out = np.frombuffer(raw[:n].tobytes(), dtype=np.complex64).reshape(sh)
    outd = np.frombuffer(raw[n:2 * n].tobytes(), dtype=np.complex64).reshape(sh)
    dS = np.frombuffer(raw[2 * n:].tobytes(), dtype=np.float32).reshape(3, -1)
    lat = po.make_lat(L, Lt, Ls, beta=0.475)
    assert np.array_equal(out, po.hmc_dslash(lat, R, chi, imass))
    assert np.array_equal(outd, po.hmc_dslash(lat, R, chi, imass, dag=True))
    assert np.array_equal(dS, po.hmc_derivs(lat, R, chi, imass))


@pytest.mark.parametrize("shape", [(4, 4, 4), (3, 2, 5), (2, 6, 3)])
@pytest.mark.parametrize("imass", [1, 3, 5])
def test_thirring_element_kernels_match_oracle(thr_exe, tmp_path, shape, imass):
    L, Lt, Ls = shape
    lat = po.make_lat(L, Lt, Ls)
    sh, kv = po.thr_shape(lat), po.kvol(lat)
    rng = np.random.default_rng(L * 100 + Lt * 10 + Ls + imass)
    R = rng.standard_normal(sh) + 1j * rng.standard_normal(sh)
    X2 = rng.standard_normal(sh) + 1j * rng.standard_normal(sh)
    theta = (0.3 * rng.standard_normal((3, kv))).astype(np.float32)
    am, anum = np.float32(0.2), 0.3141592653589793
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(fin, "wb") as f:
        f.write(R.tobytes())
        f.write(X2.tobytes())
        f.write(theta.tobytes())
    subprocess.run([thr_exe, str(L), str(Lt), str(Ls), str(imass), repr(float(am)), repr(anum),
                    fin, fout], check=True)
    raw = np.fromfile(fout, dtype=np.uint8)
    off = [0]

    def take(count, dt):
        size = count * np.dtype(dt).itemsize
        v = np.frombuffer(raw[off[0]:off[0] + size].tobytes(), dtype=dt)
        off[0] += size
        return v

    u = take(3 * kv, np.complex128).reshape(3, kv)
    out = take(R.size, np.complex128).reshape(sh)
    outd = take(R.size, np.complex128).reshape(sh)
    d0 = take(3 * kv, np.float32).reshape(3, kv)
    d1 = take(3 * kv, np.float32).reshape(3, kv)
    uo = po.thr_coef(lat, theta)
    assert np.array_equal(u, uo)
    assert np.array_equal(out, po.thr_dslash(lat, R, uo, am, imass))
    assert np.array_equal(outd, po.thr_dslash(lat, R, uo, am, imass, dag=True))
    assert np.array_equal(d0, po.thr_derivs(lat, R, X2, anum, 0))
    assert np.array_equal(d1, po.thr_derivs(lat, R, X2, anum, 1))
