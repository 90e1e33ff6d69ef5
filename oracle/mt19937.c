/*
 * MT19937 restatement of psstd/PsRandom (TEST INFRASTRUCTURE -- oracle only).
 *
 * Follows the published Matsumoto-Nishimura MT19937 (init_genrand, the
 * tempering of PsRandom::int32 psstd/PsRandom.h:305-318) and the reference's
 * conversions:
 *   real()             u32 * 2^-32 on LP64 (psstd/PsRandom.h:165-170)
 *   psRandomGaussian   Marsaglia polar method with a cached second value
 *                      (psstd/PsRandom.h:327-364)
 *   seeding            psSrandom(randomSeed + rank) (pstrol/PsDomain.cpp:213)
 * Pinned in tests against numpy's independent MT19937 (legacy seeding).
 */
#include <math.h>
#include <stdint.h>

#include "mt19937.h"

#define MT_N 624
#define MT_M 397
#define MATRIX_A 0x9908b0dfUL
#define UPPER 0x80000000UL
#define LOWER 0x7fffffffUL

void mt_seed(mt_state* s, uint32_t seed) {
  /* init_genrand: psstd/PsRandom.cpp:86-98 */
  s->mt[0] = seed;
  for (int j = 1; j < MT_N; ++j) {
    s->mt[j] = (uint32_t)(1812433253UL * (s->mt[j - 1] ^ (s->mt[j - 1] >> 30)) + (uint32_t)j);
  }
  s->idx = MT_N;
  s->have_gauss = 0;
  s->gauss = 0.0;
}

static void mt_refill(mt_state* s) {
  for (int k = 0; k < MT_N; ++k) {
    uint32_t y = (s->mt[k] & UPPER) | (s->mt[(k + 1) % MT_N] & LOWER);
    uint32_t v = s->mt[(k + MT_M) % MT_N] ^ (y >> 1);
    if (y & 1u) v ^= (uint32_t)MATRIX_A;
    s->mt[k] = v;
  }
  s->idx = 0;
}

uint32_t mt_u32(mt_state* s) {
  if (s->idx >= MT_N) mt_refill(s);
  uint32_t y = s->mt[s->idx++];
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9d2c5680UL;
  y ^= (y << 15) & 0xefc60000UL;
  y ^= (y >> 18);
  return y;
}

double mt_real(mt_state* s) {
  /* LP64 branch of PsRandom::real(): (long)int32() * (1/4294967296.0) */
  return (double)mt_u32(s) * (1.0 / 4294967296.0);
}

double mt_gauss(mt_state* s) {
  /* psRandomGaussian<double> (psstd/PsRandom.h:327-364) */
  if (!s->have_gauss) {
    double v1, v2, r;
    do {
      double u = mt_real(s);
      v1 = (2.0 * u) - 1.0;
      u = mt_real(s);
      v2 = (2.0 * u) - 1.0;
      r = (v1 * v1) + (v2 * v2);
    } while ((r >= 1.0) || (r == 0.0));
    double fac = sqrt(-2.0 * log(r) / r);
    s->gauss = v1 * fac;
    s->have_gauss = 1;
    return v2 * fac;
  }
  s->have_gauss = 0;
  return s->gauss;
}
