// fortio.h -- the reference program's on-disk formats: the 'con' checkpoint
// (Fortran unformatted sequential, rhmc/cheisdwf.f:1455-1489 and the
// single-precision variant read by rhmc/sp_to_dp.f), list-directed output
// in the layout gfortran's runtime produces (fort.11-14, 'control',
// fort.5001-5012), the explicit edit descriptors of 'output' (formats 9001,
// 9004, 9022, 9024), and the list-directed reads of 'midout' and the Remez
// files.
#pragma once
#include <cstdio>
#include <string>
#include <vector>

namespace chdwf {
namespace fio {

// ---- list-directed output -------------------------------------------------
// One record of a list-directed WRITE: a leading blank, then every item in
// its default field.  INTEGER(4) takes 11 columns, REAL(4) G16.9E2 and
// REAL(8) G25.17E3 with the 1P scale of the exponent form; every item after
// the first is preceded by one separator blank.
class ListRecord {
public:
    ListRecord& i(long long v);
    ListRecord& r4(float v);
    ListRecord& r8(double v);
    ListRecord& a(const char* s);      // character item, as is
    std::string line() const { return s_ + "\n"; }
private:
    void sep();
    std::string s_;
    bool first_ = true;
};

// ---- explicit edit descriptors -------------------------------------------
std::string edit_i(long long v, int w);          // Iw
std::string edit_f(double v, int w, int d);      // Fw.d
std::string edit_e(double v, int w, int d);      // Ew.d (0.ddddE+ee)
std::string edit_g_list(double v, int w, int d, int e);   // list-directed G

// ---- 'con' ----------------------------------------------------------------
// Reads one unformatted record holding chi(kvol,3) and seed.  A REAL*8 chi
// (the record cheisdwf.f's swrite writes) and a REAL*4 chi (the older
// configurations, converted by sp_to_dp.f) are told apart by the record
// length; *single reports which.  Returns 0, 1 if the file is missing, 2 if
// its record does not hold a kvol-site configuration.
int con_read(const char* path, int kvol, double* chi, double* seed, int* single);
// Writes chi (REAL*8) and seed as one record, as swrite does.  Returns 0 or 1.
int con_write(const char* path, int kvol, const double* chi, double seed);

// ---- list-directed input ----------------------------------------------------
// Reads records from a text file as successive list-directed READs do: each
// read starts at a new record and takes values (blank- or comma-separated,
// 'D' exponents accepted) across as many records as it needs.
class ListReader {
public:
    explicit ListReader(const char* path);
    ~ListReader();
    ListReader(const ListReader&) = delete;
    ListReader& operator=(const ListReader&) = delete;
    bool ok() const { return f_ != nullptr; }
    bool read(int n, std::vector<std::string>* out);   // one READ of n values
private:
    FILE* f_ = nullptr;
};

// Conversions of one list-directed value to the variable's type.
bool to_real4(const std::string& t, float* v);
bool to_real8(const std::string& t, double* v);
bool to_int(const std::string& t, int* v);

}  // namespace fio
}  // namespace chdwf
