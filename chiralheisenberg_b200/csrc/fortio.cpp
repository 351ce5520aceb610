// fortio.cpp -- the reference program's on-disk formats (see fortio.h).
#include "fortio.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>

namespace chdwf {
namespace fio {

namespace {

std::string rjust(const std::string& s, int w) {
    if ((int)s.size() >= w) return s;
    return std::string((size_t)(w - (int)s.size()), ' ') + s;
}

// Decimal digits of |v| rounded to nd significant digits: the digit string
// and the decimal exponent X with |v| ~ 0.d1d2...dnd x 10^X.
void sig_digits(double a, int nd, std::string* digits, int* X) {
    char buf[512];
    snprintf(buf, sizeof buf, "%.*e", nd - 1, a);
    const char* e = strchr(buf, 'e');
    digits->clear();
    for (const char* c = buf; c < e; c++)
        if (*c >= '0' && *c <= '9') digits->push_back(*c);
    *X = atoi(e + 1) + 1;
}

// Exponent field: E+ee (or E+eee for e = 3).  An Ew.d exponent beyond two
// digits drops the letter (+eee), as the standard's E editing does.
std::string exp_part(int X, int e) {
    const int ax = X < 0 ? -X : X;
    char buf[32];
    if (e == 2 && ax > 99) snprintf(buf, sizeof buf, "%c%03d", X < 0 ? '-' : '+', ax);
    else snprintf(buf, sizeof buf, "E%c%0*d", X < 0 ? '-' : '+', e, ax);
    return buf;
}

std::string nonfinite(double v, int w) {
    if (std::isnan(v)) return rjust("NaN", w);
    return rjust(v < 0 ? "-Infinity" : "Infinity", w);
}

}  // namespace

std::string edit_i(long long v, int w) {
    char buf[32];
    snprintf(buf, sizeof buf, "%lld", v);
    if ((int)strlen(buf) > w) return std::string((size_t)w, '*');
    return rjust(buf, w);
}

std::string edit_f(double v, int w, int d) {
    if (!std::isfinite(v)) return nonfinite(v, w);
    char buf[512];
    snprintf(buf, sizeof buf, "%.*f", d, std::fabs(v));
    std::string s = buf;
    const std::string sign = std::signbit(v) ? "-" : "";
    if ((int)(sign.size() + s.size()) > w && s.size() > 1 && s[0] == '0' && s[1] == '.')
        s.erase(0, 1);                               // the optional leading zero
    s = sign + s;
    if ((int)s.size() > w) return std::string((size_t)w, '*');
    return rjust(s, w);
}

std::string edit_e(double v, int w, int d) {
    if (!std::isfinite(v)) return nonfinite(v, w);
    const double a = std::fabs(v);
    std::string digits;
    int X = 0;
    if (a == 0.0) digits.assign((size_t)d, '0');
    else sig_digits(a, d, &digits, &X);
    const std::string sign = std::signbit(v) ? "-" : "";
    const std::string body = "." + digits + exp_part(X, 2);
    std::string s = sign + "0" + body;
    if ((int)s.size() > w) s = sign + body;
    if ((int)s.size() > w) return std::string((size_t)w, '*');
    return rjust(s, w);
}

// List-directed REAL output: G editing with d significant digits and an
// e-digit exponent.  Values that round to [0.1, 10^d) are written in F form
// (d-k decimals for k integer digits) followed by e+2 blanks; the others in
// E form with one digit before the point.
std::string edit_g_list(double v, int w, int d, int e) {
    if (!std::isfinite(v)) return nonfinite(v, w);
    d = std::min(std::max(d, 1), 40);            // gfortran uses 9 (REAL*4) and 17 (REAL*8)
    const double a = std::fabs(v);
    const std::string sign = std::signbit(v) ? "-" : "";
    const int tail = e + 2;
    char buf[512];
    if (a == 0.0) {
        snprintf(buf, sizeof buf, "%.*f", d - 1, 0.0);
        return rjust(sign + buf, w - tail) + std::string((size_t)tail, ' ');
    }
    snprintf(buf, sizeof buf, "%.*e", d - 1, a);
    const char* ep = strchr(buf, 'e');
    const int E = atoi(ep + 1);
    const int k = E + 1;                         // integer digits of the F form
    if (k >= 0 && k <= d) {
        char fb[512];
        snprintf(fb, sizeof fb, "%.*f", d - k, a);
        return rjust(sign + fb, w - tail) + std::string((size_t)tail, ' ');
    }
    return rjust(sign + std::string(buf, (size_t)(ep - buf)) + exp_part(E, e), w);
}

// ---- list-directed records -------------------------------------------------
void ListRecord::sep() {
    s_ += ' ';          // the record's leading blank, then one separator per item
    first_ = false;
}

ListRecord& ListRecord::i(long long v) {
    sep();
    s_ += edit_i(v, 11);
    return *this;
}

ListRecord& ListRecord::r4(float v) {
    sep();
    s_ += edit_g_list((double)v, 16, 9, 2);
    return *this;
}

ListRecord& ListRecord::r8(double v) {
    sep();
    s_ += edit_g_list(v, 25, 17, 3);
    return *this;
}

ListRecord& ListRecord::a(const char* str) {
    if (first_) sep();
    s_ += str;
    return *this;
}

// ---- con --------------------------------------------------------------------
int con_read(const char* path, int kvol, double* chi, double* seed, int* single) {
    FILE* f = fopen(path, "rb");
    if (!f) return 1;
    int32_t n1 = 0, n2 = -1;
    int rc = 2;
    const int64_t ndp = 24LL * kvol + 8, nsp = 12LL * kvol + 8;
    if (fread(&n1, 4, 1, f) == 1 && (n1 == ndp || n1 == nsp)) {
        std::vector<unsigned char> rec((size_t)n1);
        if (fread(rec.data(), 1, rec.size(), f) == rec.size() && fread(&n2, 4, 1, f) == 1 &&
            n2 == n1) {
            const bool sp = n1 == nsp;
            const size_t nchi = 3 * (size_t)kvol;
            if (sp) {
                std::vector<float> c(nchi);
                std::memcpy(c.data(), rec.data(), 4 * nchi);
                for (size_t i = 0; i < nchi; i++) chi[i] = (double)c[i];
                std::memcpy(seed, rec.data() + 4 * nchi, 8);
            } else {
                std::memcpy(chi, rec.data(), 8 * nchi);
                std::memcpy(seed, rec.data() + 8 * nchi, 8);
            }
            if (single) *single = sp ? 1 : 0;
            rc = 0;
        }
    }
    fclose(f);
    return rc;
}

int con_write(const char* path, int kvol, const double* chi, double seed) {
    FILE* f = fopen(path, "wb");
    if (!f) return 1;
    const int32_t n = (int32_t)(24LL * kvol + 8);
    bool ok = fwrite(&n, 4, 1, f) == 1;
    ok = ok && fwrite(chi, 8, 3 * (size_t)kvol, f) == 3 * (size_t)kvol;
    ok = ok && fwrite(&seed, 8, 1, f) == 1;
    ok = ok && fwrite(&n, 4, 1, f) == 1;
    ok = (fclose(f) == 0) && ok;
    return ok ? 0 : 1;
}

// ---- list-directed input ----------------------------------------------------
ListReader::ListReader(const char* path) { f_ = fopen(path, "r"); }

ListReader::~ListReader() {
    if (f_) fclose(f_);
}

bool ListReader::read(int n, std::vector<std::string>* out) {
    out->clear();
    if (!f_) return false;
    int got = 0;
    std::string line;
    auto is_sep = [](char c) { return c == ' ' || c == '\t' || c == ',' || c == '\r'; };
    while (got < n) {
        line.clear();
        int ch;
        bool any = false;
        while ((ch = fgetc(f_)) != EOF) {
            any = true;
            if (ch == '\n') break;
            line.push_back((char)ch);
        }
        if (!any) return false;
        size_t i = 0;
        while (got < n && i < line.size()) {
            while (i < line.size() && is_sep(line[i])) i++;
            if (i >= line.size()) break;
            if (line[i] == '/') return false;        // slash: values left undefined
            size_t j = i;
            while (j < line.size() && !is_sep(line[j])) j++;
            std::string tok = line.substr(i, j - i);
            for (char& c : tok)
                if (c == 'D' || c == 'd') c = 'E';
            out->push_back(tok);
            got++;
            i = j;
        }
    }
    return true;
}

bool to_real4(const std::string& t, float* v) {
    char* end = nullptr;
    *v = strtof(t.c_str(), &end);     // decimal -> REAL*4 in one rounding
    return end != t.c_str() && *end == '\0';
}

bool to_real8(const std::string& t, double* v) {
    char* end = nullptr;
    *v = strtod(t.c_str(), &end);
    return end != t.c_str() && *end == '\0';
}

bool to_int(const std::string& t, int* v) {
    char* end = nullptr;
    const long x = strtol(t.c_str(), &end, 10);
    *v = (int)x;
    return end != t.c_str() && *end == '\0';
}

}  // namespace fio
}  // namespace chdwf
