/*
 * Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3", SC'11), restated from the
 * paper for the oracle.  It stands in for gfortran's random_number in the
 * reference (src/work/util.f90:33-110, src/ionization/ionize.f90:429), whose
 * stream is seeded from /dev/urandom and is not reproducible; the device
 * library implements the same generator so that both sides draw the same
 * numbers for the same (key, counter).
 *
 * Test infrastructure: only tests/, bench.py's CPU baseline and the smoke
 * check use the oracle.
 */
#ifndef ORACLE_PHILOX_H
#define ORACLE_PHILOX_H
#include <stdint.h>

static inline void ora_philox4x32_10(const uint32_t ctr_in[4], uint32_t k0, uint32_t k1,
                                     uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n1 = lo1;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    uint32_t n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* 53-bit uniform in [0,1) from two 32-bit words. */
static inline double ora_u53(uint32_t a, uint32_t b) {
  uint64_t m = ((uint64_t)a << 21) | (uint64_t)(b >> 11);
  return (double)m * (1.0 / 9007199254740992.0);
}
/* 32-bit uniform in [0,1). */
static inline double ora_u32(uint32_t a) { return (double)a * (1.0 / 4294967296.0); }

#endif
