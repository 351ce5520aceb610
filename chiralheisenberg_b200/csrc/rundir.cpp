// rundir.cpp -- program dwf3d (rhmc/cheisdwf.f:1-466) run in a directory,
// with the reference's input files and output streams, over the host driver
// of chdwf_program.h; and the C entry points of the on-disk formats.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/chdwf.h"
#include "../../include/chdwf_program.h"
#include "fortio.h"

using chdwf::fio::ListRecord;
using chdwf::fio::edit_e;
using chdwf::fio::edit_f;
using chdwf::fio::edit_i;

namespace {

// remez2/remez4/remez2g as the reads at rhmc/cheisdwf.f:138-158 take them:
// anum(0); n records 'anum(i) aden(i)'; bnum(0); n records 'bnum(i) bden(i)'.
bool read_remez(const std::string& path, int n, std::vector<double>* an, std::vector<double>* ad,
                std::vector<double>* bn, std::vector<double>* bd) {
    chdwf::fio::ListReader r(path.c_str());
    if (!r.ok()) return false;
    an->assign(n + 1, 0.0); ad->assign(n, 0.0);
    bn->assign(n + 1, 0.0); bd->assign(n, 0.0);
    std::vector<std::string> t;
    auto block = [&](std::vector<double>* num, std::vector<double>* den) {
        if (!r.read(1, &t) || !chdwf::fio::to_real8(t[0], &(*num)[0])) return false;
        for (int i = 1; i <= n; i++)
            if (!r.read(2, &t) || !chdwf::fio::to_real8(t[0], &(*num)[i]) ||
                !chdwf::fio::to_real8(t[1], &(*den)[i - 1]))
                return false;
        return true;
    };
    return block(an, ad) && block(bn, bd);
}

struct Files {                       // the units the main program writes
    FILE* out7 = nullptr;            // 'output'
    FILE* f98 = nullptr;             // 'control'
    FILE* f11 = nullptr; FILE* f12 = nullptr; FILE* f13 = nullptr; FILE* f14 = nullptr;
    FILE* f5001 = nullptr; FILE* f5011 = nullptr; FILE* f5002 = nullptr; FILE* f5012 = nullptr;
    ~Files() {
        for (FILE* f : {out7, f98, f11, f12, f13, f14, f5001, f5011, f5002, f5012})
            if (f) fclose(f);
    }
};

void put(FILE* f, const std::string& s) { fputs(s.c_str(), f); }

}  // namespace

extern "C" {

int chdwf_con_read(const char* path, int kvol, double* chi, double* seed, int* single) {
    if (!path || !chi || !seed || kvol < 1) return CHDWF_BAD_ARG;
    const int rc = chdwf::fio::con_read(path, kvol, chi, seed, single);
    return rc == 0 ? CHDWF_OK : (rc == 1 ? CHDWF_NOT_FOUND : CHDWF_BAD_ARG);
}

int chdwf_con_write(const char* path, int kvol, const double* chi, double seed) {
    if (!path || !chi || kvol < 1) return CHDWF_BAD_ARG;
    return chdwf::fio::con_write(path, kvol, chi, seed) == 0 ? CHDWF_OK : CHDWF_BAD_ARG;
}

int chdwf_format_list(char* out, int cap, const char* kinds, const double* values) {
    if (!out || !kinds || !values) return -1;
    ListRecord r;
    for (int i = 0; kinds[i]; i++) {
        if (kinds[i] == 'i') r.i((long long)values[i]);
        else if (kinds[i] == 'f') r.r4((float)values[i]);
        else if (kinds[i] == 'd') r.r8(values[i]);
        else return -1;
    }
    const std::string s = r.line();
    if ((int)s.size() + 1 > cap) return -1;
    std::memcpy(out, s.c_str(), s.size() + 1);
    return (int)s.size();
}

int chdwf_format_edit(char* out, int cap, char kind, int w, int d, double value) {
    if (!out || w < 1 || d < 0) return -1;
    std::string s;
    if (kind == 'I') s = edit_i((long long)value, w);
    else if (kind == 'F') s = edit_f(value, w, d);
    else if (kind == 'E') s = edit_e(value, w, d);
    else return -1;
    if ((int)s.size() + 1 > cap) return -1;
    std::memcpy(out, s.c_str(), s.size() + 1);
    return (int)s.size();
}

int chdwf_run_dir(const char* dir, int ksize, int ksizet, int kthird, int device) {
    if (!dir) return CHDWF_BAD_ARG;
    const std::string D = dir;
    auto path = [&D](const char* f) { return D + "/" + f; };
    // parameter(ndiag=25, ndiagg=12), the residuals and iprint (:31-35, :91)
    const int ndiag = 25, ndiagg = 12, icheck = 5;
    const float respbp = 0.000001f, rescgg = 0.000001f, rescga = 0.000000001f;

    // read(25,*) dt,beta,am3,am,hpin,imass,iterl,iter2 (:117)
    chdwf::fio::ListReader mid(path("midout").c_str());
    if (!mid.ok()) return CHDWF_NOT_FOUND;
    std::vector<std::string> t;
    float dt, beta, am3, am, hpin;
    int imass, iterl, iter2;
    using namespace chdwf::fio;
    if (!mid.read(8, &t) || !to_real4(t[0], &dt) || !to_real4(t[1], &beta) ||
        !to_real4(t[2], &am3) || !to_real4(t[3], &am) || !to_real4(t[4], &hpin) ||
        !to_int(t[5], &imass) || !to_int(t[6], &iterl) || !to_int(t[7], &iter2) || iter2 < 1)
        return CHDWF_BAD_ARG;

    std::vector<double> r[3][4];
    const char* rnames[3] = {"remez2", "remez4", "remez2g"};
    const int rpoles[3] = {ndiag, ndiag, ndiagg};
    for (int k = 0; k < 3; k++)
        if (!read_remez(path(rnames[k]), rpoles[k], &r[k][0], &r[k][1], &r[k][2], &r[k][3]))
            return CHDWF_NOT_FOUND;

    chdwf_prog* p = nullptr;
    int rc = chdwf_prog_create(&p, ksize, ksizet, kthird, dt, beta, am3, am, hpin, imass, iterl,
                               device);
    if (rc != CHDWF_OK) return rc;
    struct Guard {
        chdwf_prog* p;
        ~Guard() { chdwf_prog_destroy(p); }
    } guard{p};
    const int which[3] = {2, 4, 22};
    for (int k = 0; k < 3; k++) {
        rc = chdwf_prog_set_remez(p, which[k], r[k][0].data(), r[k][1].data(), r[k][2].data(),
                                  r[k][3].data(), rpoles[k]);
        if (rc != CHDWF_OK) return rc;
    }

    Files F;
    F.out7 = fopen(path("output").c_str(), "w");
    F.f98 = fopen(path("control").c_str(), "a");
    F.f11 = fopen(path("fort.11").c_str(), "a");
    F.f12 = fopen(path("fort.12").c_str(), "a");
    F.f13 = fopen(path("fort.13").c_str(), "a");
    F.f14 = fopen(path("fort.14").c_str(), "a");
    F.f5001 = fopen(path("fort.5001").c_str(), "a");
    F.f5011 = fopen(path("fort.5011").c_str(), "a");
    F.f5002 = fopen(path("fort.5002").c_str(), "a");
    F.f5012 = fopen(path("fort.5012").c_str(), "a");
    for (FILE* f : {F.out7, F.f98, F.f11, F.f12, F.f13, F.f14, F.f5001, F.f5011, F.f5002, F.f5012})
        if (!f) return CHDWF_BAD_ARG;

    double seed = 0.0;                                                   // sread (:118-120)
    rc = chdwf_prog_read_con(p, path("con").c_str(), &seed);
    if (rc != CHDWF_OK) return rc;
    put(F.out7, ListRecord().a("seed: ").r8(seed).line());              // :126
    rc = chdwf_prog_startup(p, seed);                                    // :128-130
    if (rc != CHDWF_OK) return rc;

    // heading (:161-176)
    const float traj = (float)iterl * dt;
    put(F.out7, " ksize=" + edit_i(ksize, 3) + " ksizet=" + edit_i(ksizet, 3) + "\n");
    put(F.out7, " kthird=" + edit_i(kthird, 3) + "\n");
    put(F.out7, " time step: dt=" + edit_f(dt, 6, 4) + " trajectory length=" +
                    edit_f(traj, 9, 6) + "\n");
    put(F.out7, " # trajectories=" + edit_i(iter2, 6) + " beta=" + edit_f(beta, 9, 6) + "\n");
    put(F.out7, " am3=" + edit_f(am3, 6, 4) + " am=" + edit_f(am, 6, 4) + " hpin=" +
                    edit_f(hpin, 7, 4) + "\n");
    put(F.out7, " imass=" + edit_i(imass, 2) + "\n");
    put(F.out7, " Stopping residuals: guidance: " + edit_e(rescgg, 9, 4) + " acceptance: " +
                    edit_e(rescga, 9, 4) + " estimator: " + edit_e(respbp, 9, 4) + "\n");
    put(F.out7, ListRecord().a("seed: ").r8(chdwf_prog_seed(p)).line());   // :180-182

    const int Lt = ksizet;
    std::vector<float> cf(8 * (size_t)Lt);
    for (int isweep = 1; isweep <= iter2; isweep++) {                   // :207-411
        chdwf_sweep_record rec;
        rc = chdwf_prog_sweep(p, &rec);
        if (rc != CHDWF_OK) return rc;
        put(F.f98, ListRecord().r8(rec.dH).r8(rec.dS).i(rec.accepted).line());           // :345
        put(F.f11, ListRecord().i(isweep).r4(rec.gaction).r4(rec.paction).line());       // :347
        if (rec.measured) {                                                              // :387-389
            put(F.f12, ListRecord().r4(rec.cond[0]).r4(rec.cond[1]).r4(rec.cond[2]).line());
            put(F.f13, ListRecord().r4(rec.susc[0]).r4(rec.susc[1]).r4(rec.susc[2]).line());
            put(F.f14, ListRecord().r4(rec.condmod).r4(rec.susctot).line());
            for (int n = chdwf_prog_take_cg_caps(p); n > 0; n--)                     // :1151-1153
                put(F.out7, " # iterations of congrad exceeds niterc\n");
            rc = chdwf_prog_correlators(p, cf.data());
            if (rc != CHDWF_OK) return rc;
            // cferm1(it,f) at cf[2(it + Lt f)], cferm2 after it (:1036-1047)
            const float* c1 = cf.data();
            const float* c2 = cf.data() + 4 * Lt;
            for (int it = 0; it < Lt; it++) {
                put(F.f5001, ListRecord().i(it).r4(c1[2 * it]).r4(c1[2 * it + 1]).line());
                put(F.f5011, ListRecord().i(it).r4(c2[2 * it]).r4(c2[2 * it + 1]).line());
                put(F.f5002, ListRecord().i(it).r4(c1[2 * (it + Lt)]).r4(c1[2 * (it + Lt) + 1]).line());
                put(F.f5012, ListRecord().i(it).r4(c2[2 * (it + Lt)]).r4(c2[2 * (it + Lt) + 1]).line());
            }
            for (FILE* f : {F.f5001, F.f5011, F.f5002, F.f5012}) fflush(f);
        }
        if ((isweep / icheck) * icheck == isweep) {                                     // :400-411
            rc = chdwf_prog_write_con(p, path("con").c_str());
            if (rc != CHDWF_OK) return rc;
            for (FILE* f : {F.f12, F.f13, F.f14}) fflush(f);
        }
        fflush(F.f98);
    }

    chdwf_run_averages a;                                               // :413-431
    rc = chdwf_prog_averages(p, &a);
    if (rc != CHDWF_OK) return rc;
    put(F.out7, " averages for last " + edit_i(a.iter2, 6) + " trajectories\n");         // 9022
    put(F.out7, "  # of acceptances: " + edit_i(a.naccp, 6) + " average trajectory length= " +
                    edit_f(a.atraj, 8, 3) + "\n");
    put(F.out7, "  <exp-dH>=" + edit_e(a.yav, 11, 4) + " +/-" + edit_e(a.yyav, 10, 3) + "\n");
    put(F.out7, "  av. # QMR itr. guidance: " + edit_f(a.ancg, 9, 3) + "; acceptance: " +
                    edit_f(a.ancgh, 9, 3) + "\n");
    put(F.out7, "  force: " + edit_f(a.ancgf, 9, 3) + "; pseudofermion: " +
                    edit_f(a.ancgpf, 9, 3) + "\n\n");
    put(F.out7, "  measurement: " + edit_f(a.ancgma, 9, 3) + "\n\n");
    put(F.out7, "  condmod=" + edit_e(a.condmoda, 11, 3) + " susc=" + edit_e(a.susca, 11, 3) + "\n");
    put(F.out7, " cond components=" + edit_e(a.conda[0], 11, 3) + edit_e(a.conda[1], 11, 3) +
                    edit_e(a.conda[2], 11, 3) + "\n");
    put(F.out7, "  psibarpsi=" + edit_e(a.pbpa, 11, 3) + "\n");
    put(F.out7, "  mean square velocity=" + edit_e(a.vel2a, 10, 3) + "; action per site=" +
                    edit_e(a.actiona, 10, 3) + "\n\n\n");
    put(F.out7, "\n\n");                                                 // 9024 twice: 1x alone
    rc = chdwf_prog_write_con(p, path("con").c_str());                   // :456-463
    if (rc != CHDWF_OK) return rc;
    put(F.out7, ListRecord().a("seed: ").r8(chdwf_prog_seed(p)).line());
    return CHDWF_OK;
}

}  // extern "C"
