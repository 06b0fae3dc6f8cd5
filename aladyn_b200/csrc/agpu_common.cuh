// agpu_common.cuh — device-side helpers shared by the FP64 and FP32-split
// kernels of the B200 PIC step: the Philox4x32-10 generator, the packed
// charge/part_ind/wgh slot, grid geometry and the handle's device state.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/aladyn_gpu.h"

#define AGPU_HD __host__ __device__ __forceinline__

// Geometry of the single-domain box (the reference's ix1..ix2 etc., Fortran
// 1-based indices; arrays are column-major (n1p, n2p, n3p, comp)).
struct Geo {
  int ndim, n1p, n2p, n3p, ix1, ix2, jy1, jy2, kz1, kz2, nf, nc;
  long long ncell;  // n1p*n2p*n3p
  uint32_t dm1, dm2;  // div31 multipliers of n1p and n2p (geo_divisors)
  int ds1, ds2;       // and their shifts
};

// floor(n / d) for 0 <= n < 2^31 and d >= 2 with one multiply-high
// (Granlund and Montgomery, PLDI 1994, Theorem 4.2, N = 31): with
// l = ceil(log2 d) and m = ceil(2^(31+l) / d), m d - 2^(31+l) < d <= 2^l, so
// floor(n / d) = floor(n m / 2^(31+l)); m < 2^32 for every d >= 2.
AGPU_HD uint32_t div31(uint32_t n, uint32_t m, int sh) {
#ifdef __CUDA_ARCH__
  return __umulhi(n, m) >> sh;
#else
  return (uint32_t)(((uint64_t)n * m) >> 32) >> sh;
#endif
}

inline void div31_constants(uint32_t d, uint32_t& m, int& sh) {
  int l = 0;
  while ((1ull << l) < d) ++l;
  m = (uint32_t)(((1ull << (31 + l)) + d - 1) / d);
  sh = l - 1;  // the shift after the high word: 31 + l - 32
}

// Fills the divisor constants of a Geo whose n1p, n2p are set (both >= 2).
inline void geo_divisors(Geo& g) {
  div31_constants((uint32_t)g.n1p, g.dm1, g.ds1);
  div31_constants((uint32_t)g.n2p, g.dm2, g.ds2);
}

// Fortran node (i, j, k) of a linear cell index 0 <= c < 2^31 (goff's inverse).
AGPU_HD void cell_split(const Geo& g, int c, int& i, int& j, int& k) {
  const uint32_t r = div31((uint32_t)c, g.dm1, g.ds1);
  const uint32_t q = div31(r, g.dm2, g.ds2);
  i = c - (int)r * g.n1p + 1;
  j = (int)r - (int)q * g.n2p + 1;
  k = (int)q + 1;
}

// Linear offset of Fortran node (i, j, k) (1-based) in one component.
AGPU_HD long long goff(const Geo& g, int i, int j, int k) {
  return (long long)(i - 1) + (long long)g.n1p * ((long long)(j - 1) + (long long)g.n2p * (long long)(k - 1));
}

// ---- Philox4x32-10 (Salmon et al., SC'11), written from the paper ----------
AGPU_HD void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                           uint32_t out[4]) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}
AGPU_HD double u53(uint32_t a, uint32_t b) {
  uint64_t m = ((uint64_t)a << 21) | (uint64_t)(b >> 11);
  return (double)m * (1.0 / 9007199254740992.0);
}
AGPU_HD double u32d(uint32_t a) { return (double)a * (1.0 / 4294967296.0); }

// Ionization draw of ion n (0-based, in species order) of species ic at step
// iter: the same counter layout the oracle uses.
AGPU_HD double ionz_draw(uint64_t seed, long long n, int iter, int ic) {
  uint32_t r[4];
  philox4x32_10((uint32_t)n, (uint32_t)((unsigned long long)n >> 32), (uint32_t)iter, 0x494f0000u | (uint32_t)ic,
                (uint32_t)seed, (uint32_t)(seed >> 32), r);
  return u53(r[0], r[1]);
}

// ---- packed slot: int16 charge | int16 part_ind | float wgh -------------
AGPU_HD int slot_charge(uint64_t b) { return (int)(int16_t)(uint16_t)(b & 0xffffu); }
AGPU_HD int slot_part_ind(uint64_t b) { return (int)(int16_t)(uint16_t)((b >> 16) & 0xffffu); }
__device__ __forceinline__ float slot_wgh(uint64_t b) { return __uint_as_float((uint32_t)(b >> 32)); }
__device__ __forceinline__ uint64_t make_slot(int charge, int part_ind, float wgh) {
  return (uint64_t)(uint16_t)(int16_t)charge | ((uint64_t)(uint16_t)(int16_t)part_ind << 16) |
         ((uint64_t)__float_as_uint(wgh) << 32);
}
__device__ __forceinline__ uint64_t dbits(double d) { return (uint64_t)__double_as_longlong(d); }
__device__ __forceinline__ double bitsd(uint64_t b) { return __longlong_as_double((long long)b); }

// ---- error word -----------------------------------------------------------
__device__ __forceinline__ void raise_err(unsigned int* err, unsigned int bit) { atomicOr(err, bit); }

// Grid-size helper: a multiple of the SM count (148 on B200) times resident
// blocks, capped by the work.
static inline int grid_for(long long n, int block, int sms, int per_sm = 8) {
  long long need = (n + block - 1) / block;
  long long cap = (long long)sms * per_sm;
  if (need < 1) need = 1;
  return (int)(need < cap ? need : cap);
}
