// rng.cpp -- host random numbers of program dwf3d (see rng.h).
#include "rng.h"

#include <cmath>

namespace chdwf {

namespace {
constexpr double kM1 = 15184245.0, kM2 = 2651554.0;      // DM(1), DM(2)
constexpr double k24 = 16777216.0, k48 = 281474976710656.0;
// tpi = 2.0*acos(-1.0) evaluated in REAL*4 (rhmc/cheisdwf.f:93)
const float kTwoPi = 2.0f * static_cast<float>(3.14159265358979323846);
}  // namespace

void Rng::set_seed(double seed) {
    ds_[1] = std::trunc(seed / k24);
    ds_[0] = seed - ds_[1] * k24;
}

double Rng::seed() const { return ds_[1] * k24 + ds_[0]; }

float Rng::rranf() {
    // low half times low multiplier, carry into the high half; all products
    // stay below 2^53 so the double arithmetic is exact
    double lo = ds_[0] * kM1;
    const double carry = std::trunc(lo / k24);
    lo = lo - carry * k24;
    const double hi = ds_[0] * kM2 + ds_[1] * kM1 + carry;
    ds_[1] = hi - std::trunc(hi / k24) * k24;
    ds_[0] = lo;
    return static_cast<float>((ds_[1] * k24 + ds_[0]) / k48);
}

float Rng::rano(float& y) {
    if (idum_ < 0) {
        idum_ = 1;
        for (int j = 0; j < 97; j++) (void)rranf();
        for (int j = 0; j < 97; j++) v_[j] = rranf();
        y = rranf();
    }
    int j = 1 + static_cast<int>(97.0f * y);
    if (j > 97) j = 97;
    if (j < 1) j = 1;
    y = v_[j - 1];
    const float out = y;
    v_[j - 1] = rranf();
    return out;
}

Rng::State Rng::state() const {
    State s;
    s.ds[0] = ds_[0];
    s.ds[1] = ds_[1];
    for (int j = 0; j < 97; j++) s.v[j] = v_[j];
    s.yran = yran_;
    s.yrun = yrun_;
    s.idum = idum_;
    return s;
}

void Rng::set_state(const State& s) {
    ds_[0] = s.ds[0];
    ds_[1] = s.ds[1];
    for (int j = 0; j < 97; j++) v_[j] = s.v[j];
    yran_ = s.yran;
    yrun_ = s.yrun;
    idum_ = s.idum;
}

void Rng::startup(double seed) {
    set_seed(seed);
    idum_ = -1;
    yran_ = 0.0f;
    yrun_ = 0.0f;
    (void)rano(yran_);
}

void Rng::gauss0(int64_t kvol, float* ps) {
    for (int64_t i = 0; i < kvol; i++) ps[kvol + i] = std::sqrt(-std::log(rano(yran_)));
    for (int64_t i = 0; i < kvol; i++) {
        const float theta = kTwoPi * rano(yran_);
        ps[i] = ps[kvol + i] * std::sin(theta);
        ps[kvol + i] = ps[kvol + i] * std::cos(theta);
    }
}

void Rng::gaussp(int64_t kvol, float* ps) {
    for (int64_t i = 0; i < kvol; i++) ps[kvol + i] = std::sqrt(-2.0f * std::log(rano(yran_)));
    for (int64_t i = 0; i < kvol; i++) {
        const float theta = kTwoPi * rano(yran_);
        ps[i] = ps[kvol + i] * std::sin(theta);
        ps[kvol + i] = ps[kvol + i] * std::cos(theta);
    }
}

}  // namespace chdwf
