// rng.h -- the reference's random-number generator, host side.
//
// RRANF is a 48-bit multiplicative congruential generator carried as two
// 24-bit halves in double precision (rhmc/cheisdwf.f:1765-1801); rano is the
// Numerical-Recipes shuffle over a 97-entry table (:1722-1751), called with
// one of two "last output" variables: yran (/ranseed/, used by the Gaussian
// generators and fermion) and yrun (a main-program local, used for the
// trajectory-end test and the Metropolis draw, :298, :329).  Every draw of a
// trajectory is independent of the fields, so a whole trajectory's stream can
// be generated ahead of the GPU work.
#pragma once
#include <stdint.h>

namespace chdwf {

class Rng {
public:
    // rranset(seed); idum=-1; one rano(yran) call (rhmc/cheisdwf.f:125-130)
    void startup(double seed);
    void set_seed(double seed);                 // RRANSET / G900ST
    double seed() const;                        // RRANGET / G900GT
    float rranf();                              // one LCG step, SNGL of the result
    float rano_yran() { return rano(yran_); }
    float rano_yrun() { return rano(yrun_); }
    // gauss0 (variance 1/2, :1701-1718) and gaussp (variance 1, :1678-1695):
    // ps(kvol,2): ps[0..kvol) and ps[kvol..2kvol)
    void gauss0(int64_t kvol, float* ps);
    void gaussp(int64_t kvol, float* ps);

    // Complete generator state: the LCG halves, the shuffle table and both
    // "last output" variables.  The reference checkpoints only the LCG seed
    // (rhmc/cheisdwf.f:401-411), so its resumed runs differ from
    // uninterrupted ones; restoring this state resumes exactly.
    struct State {
        double ds[2];
        float v[97];
        float yran, yrun;
        int idum;
    };
    State state() const;
    void set_state(const State& s);

private:
    float rano(float& y);
    double ds_[2] = {0.0, 0.0};
    float v_[97] = {};
    float yran_ = 0.0f, yrun_ = 0.0f;
    int idum_ = -1;
};

}  // namespace chdwf
