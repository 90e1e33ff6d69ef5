/* MT19937 state for the oracle (TEST INFRASTRUCTURE). */
#ifndef PSWIFT_ORACLE_MT_H
#define PSWIFT_ORACLE_MT_H
#include <stdint.h>

typedef struct mt_state {
  uint32_t mt[624];
  int idx;
  int have_gauss;
  double gauss;
} mt_state;

void mt_seed(mt_state* s, uint32_t seed);
uint32_t mt_u32(mt_state* s);
double mt_real(mt_state* s);
double mt_gauss(mt_state* s);

#endif
