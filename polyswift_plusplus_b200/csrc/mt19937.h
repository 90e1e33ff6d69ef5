// MT19937 with the conversions of psstd/PsRandom (host side of the engine).
//
// init_genrand(seed) (psstd/PsRandom.cpp:86-98), tempering as PsRandom::int32
// (psstd/PsRandom.h:305-318), real() = u32 * 2^-32 on LP64
// (psstd/PsRandom.h:165-170), Marsaglia polar Gaussian with one cached value
// (psstd/PsRandom.h:327-364).  Used for the reference's "random" field
// initialisation and for the updater noise, which must consume the stream in
// the reference's order.
#pragma once

#include <math.h>
#include <stdint.h>

namespace psb {

class Mt19937 {
 public:
  explicit Mt19937(uint32_t seed = 5489u) { seed_(seed); }

  void seed_(uint32_t s) {
    mt_[0] = s;
    for (int j = 1; j < 624; ++j)
      mt_[j] = (uint32_t)(1812433253u * (mt_[j - 1] ^ (mt_[j - 1] >> 30)) + (uint32_t)j);
    idx_ = 624;
    have_gauss_ = false;
    gauss_ = 0.0;
  }

  uint32_t u32() {
    if (idx_ >= 624) refill_();
    uint32_t y = mt_[idx_++];
    y ^= (y >> 11);
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= (y >> 18);
    return y;
  }

  double real() { return (double)u32() * (1.0 / 4294967296.0); }

  double gauss() {
    if (!have_gauss_) {
      double v1, v2, r;
      do {
        v1 = (2.0 * real()) - 1.0;
        v2 = (2.0 * real()) - 1.0;
        r = (v1 * v1) + (v2 * v2);
      } while ((r >= 1.0) || (r == 0.0));
      const double fac = sqrt(-2.0 * log(r) / r);
      gauss_ = v1 * fac;
      have_gauss_ = true;
      return v2 * fac;
    }
    have_gauss_ = false;
    return gauss_;
  }

  // The whole generator state, e.g. to continue the stream on the device.
  void get_state(uint32_t* mt, int* idx, bool* have_gauss, double* gauss) const {
    for (int k = 0; k < 624; ++k) mt[k] = mt_[k];
    *idx = idx_;
    *have_gauss = have_gauss_;
    *gauss = gauss_;
  }
  void set_state(const uint32_t* mt, int idx, bool have_gauss, double gauss) {
    for (int k = 0; k < 624; ++k) mt_[k] = mt[k];
    idx_ = idx;
    have_gauss_ = have_gauss;
    gauss_ = gauss;
  }

 private:
  void refill_() {
    for (int k = 0; k < 624; ++k) {
      uint32_t y = (mt_[k] & 0x80000000u) | (mt_[(k + 1) % 624] & 0x7fffffffu);
      uint32_t v = mt_[(k + 397) % 624] ^ (y >> 1);
      if (y & 1u) v ^= 0x9908b0dfu;
      mt_[k] = v;
    }
    idx_ = 0;
  }
  uint32_t mt_[624];
  int idx_;
  bool have_gauss_;
  double gauss_;
};

}  // namespace psb
