// Host-side checks of the binning and index helpers shared with the device
// kernels (compiled by nvcc, run on the CPU; no CUDA call is made):
//   * div31: floor(n / d) by multiply-high for every d in 2..5000 and random
//     large d, on edge and random n < 2^31;
//   * cell_split inverts goff on random nodes of several grids;
//   * tile_key / tile_key_c: the key packs (tile, row, octant) as
//     tile * nsub + row * nq + octant, nodes outside the tiles map to nkeys,
//     and the compile-time variant agrees with the run-time one.
// Prints "host logic ok <checks>" and exits 0, or the first failure and 1.
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "agpu_bin.cuh"

using namespace agpu;

static uint64_t rng_state = 0x9E3779B97F4A7C15ull;
static uint64_t rnd() {  // splitmix64
  uint64_t z = (rng_state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

#define FAIL(...)                  \
  do {                             \
    std::printf("FAIL: ");         \
    std::printf(__VA_ARGS__);      \
    std::printf("\n");             \
    return 1;                      \
  } while (0)

int main() {
  long long checks = 0;
  // div31
  for (int rep = 0; rep < 5000 + 2000; ++rep) {
    const uint32_t d = rep < 4999 ? (uint32_t)(rep + 2) : (uint32_t)(2 + rnd() % 0x7FFFFFFEull);
    uint32_t m;
    int sh;
    div31_constants(d, m, sh);
    const uint32_t edge[] = {0u, 1u, d - 1u, d, d + 1u, 0x7FFFFFFFu, 0x7FFFFFFEu, (0x7FFFFFFFu / d) * d,
                             (0x7FFFFFFFu / d) * d - 1u};
    for (uint32_t n : edge) {
      if (n > 0x7FFFFFFFu) continue;
      if (div31(n, m, sh) != n / d) FAIL("div31 n=%u d=%u", n, d);
      ++checks;
    }
    for (int k = 0; k < 64; ++k) {
      const uint32_t n = (uint32_t)(rnd() & 0x7FFFFFFFu);
      if (div31(n, m, sh) != n / d) FAIL("div31 n=%u d=%u", n, d);
      ++checks;
    }
  }
  // cell_split o goff, tile keys
  const int grids[][4] = {{3, 64, 32, 16}, {3, 96, 40, 24}, {3, 1024, 256, 256}, {2, 1024, 256, 1}, {2, 70, 37, 1}};
  for (const auto& gr : grids) {
    Geo g{};
    g.ndim = gr[0];
    g.n1p = gr[1] + 5;
    g.n2p = gr[2] + 5;
    g.n3p = gr[0] == 3 ? gr[3] + 5 : 1;
    g.ncell = (long long)g.n1p * g.n2p * g.n3p;
    geo_divisors(g);
    TileGeo t{};
    t.tx = 16;
    t.ty = g.ndim == 3 ? 8 : 16;
    t.tz = g.ndim == 3 ? 4 : 1;
    t.ntx = (gr[1] + 1 + t.tx - 1) / t.tx;
    t.nty = (gr[2] + 1 + t.ty - 1) / t.ty;
    t.ntz = g.ndim == 3 ? (gr[3] + 1 + t.tz - 1) / t.tz : 1;
    t.ntiles = t.ntx * t.nty * t.ntz;
    t.nq = g.ndim == 3 ? 8 : 4;
    t.nsub = t.ty * t.tz * t.nq;
    t.nkeys = t.ntiles * t.nsub;
    for (int k = 0; k < 20000; ++k) {
      const int i = 1 + (int)(rnd() % g.n1p), j = 1 + (int)(rnd() % g.n2p), kk = 1 + (int)(rnd() % g.n3p);
      const long long c = goff(g, i, j, kk);
      int a, b, e;
      cell_split(g, (int)c, a, b, e);
      if (a != i || b != j || e != kk) FAIL("cell_split (%d,%d,%d) -> (%d,%d,%d)", i, j, kk, a, b, e);
      const int kz = g.ndim == 3 ? kk : 3;
      const int oct = (int)(rnd() % t.nq);
      const int key = tile_key(t, i, j, kz, oct);
      const bool in = i >= 3 && j >= 3 && kz >= 3 && (i - 3) / t.tx < t.ntx && (j - 3) / t.ty < t.nty &&
                      (kz - 3) / t.tz < t.ntz;
      if (!in) {
        if (key != t.nkeys) FAIL("outside node (%d,%d,%d) key %d", i, j, kz, key);
      } else {
        const int tile = key / t.nsub, sub = key % t.nsub;
        const int ta = (i - 3) / t.tx, tb = (j - 3) / t.ty, tc = (kz - 3) / t.tz;
        if (tile != ta + t.ntx * (tb + t.nty * tc)) FAIL("tile of (%d,%d,%d)", i, j, kz);
        if (sub % t.nq != oct) FAIL("octant of (%d,%d,%d)", i, j, kz);
        const int row = sub / t.nq;
        if (row != ((j - 3) - tb * t.ty) + t.ty * ((kz - 3) - tc * t.tz)) FAIL("row of (%d,%d,%d)", i, j, kz);
        const int kc = g.ndim == 3 ? tile_key_c<16, 8, 4, 8>(t, i, j, kz, oct) : tile_key_c<16, 16, 1, 4>(t, i, j, kz, oct);
        if (kc != key) FAIL("tile_key_c %d != tile_key %d", kc, key);
      }
      checks += 2;
    }
  }
  // octants
  const float v[2] = {-0.25f, 0.25f};
  for (int q = 0; q < 8; ++q) {
    const int o = offset_octant(v[q & 1], v[(q >> 1) & 1], v[(q >> 2) & 1], 3);
    if (o != q) FAIL("octant %d -> %d", q, o);
    if (offset_octant(v[q & 1], v[(q >> 1) & 1], v[(q >> 2) & 1], 2) != (q & 3)) FAIL("quadrant %d", q);
    ++checks;
  }
  std::printf("host logic ok %lld\n", checks);
  return 0;
}
