// agpu_tile.h — arguments of the tiled gather/push/deposit kernels.
#pragma once
#include <cuda_runtime.h>

#include "agpu_bin.cuh"
#include "agpu_kernels.h"

namespace agpu {

// Tile extents in nodes (3D and 2D).  32 nodes along x: the FP32 split
// kernel gives each warp one x-row of a tile, one node per lane, so that its
// shared-memory stencil reads are 32 consecutive words.
constexpr int TILE3_X = 32, TILE3_Y = 4, TILE3_Z = 4;
constexpr int TILE2_X = 32, TILE2_Y = 8;

struct TileArgs32 {
  Geo g;
  TileGeo t;
  const float* ebf;
  float* jhi;
  float* jlo;
  Part32 p;
  const int* perm;
  const int* tstart;
  int* key;   // new key per particle (tile and row; nkeys = removed)
  int* hist;  // next histogram, nkeys + 1 bins
  float dth, lfact, dtx, dty, dtz;
  int initial;
  unsigned int* err;
  // further chunks of dense tiles: (tile, chunk) pairs and the counters
  // (count, next); null: every tile's CTA runs all its chunks
  int* work;
  unsigned int* work_n;
  int work_cap;
};

struct TileArgs64 {
  Geo g;
  TileGeo t;
  const double* ebf;
  double* jc;
  double *x, *y, *z, *px, *py, *pz;
  const double* slot;
  const int* perm;
  const int* tstart;
  int* key;
  int* hist;
  double xmn, ymn, zmn, dx_inv, dy_inv, dz_inv;
  double dt, dth, lfact;
  double gxmin, gxmax, gymin, gymax, gzmin, gzmax;
  double vdt;  // comoving frame: dt * vbeam subtracted from x after the push (0: off)
  int initial;
  unsigned int* err;
};

TileGeo make_tiles(const Geo& g, int nx, int ny, int nz);
int tile_push32(const TileArgs32& a, cudaStream_t st, int sms);
int tile32_list_cap(int ndim);
// the cubic shape extension (agpu_tile32c.cu)
void tile_push32_cubic(const TileArgs32& a, cudaStream_t st);
void tile_push64(const TileArgs64& a, cudaStream_t st);
void hist_reset(int* hist, const int* tstart, const TileGeo& t, long long np, bool first, unsigned long long* pushed,
                cudaStream_t st);

}  // namespace agpu
