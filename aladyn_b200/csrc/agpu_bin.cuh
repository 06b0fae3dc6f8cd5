// agpu_bin.cuh — spatial tiles of the particle binning (tile geometry and
// node -> tile key), shared by the tiled push kernels and the binning pass.
#pragma once
#include "agpu_common.cuh"

namespace agpu {

// A tile is TX x TY x TZ integer nodes; node i (Fortran) of an alive particle
// lies in [3, nx+3], so tiles cover nodes 3.. in steps of TX.
struct TileGeo {
  int tx, ty, tz;     // tile extent in nodes
  int ntx, nty, ntz;  // tiles per axis
  int ntiles;         // ntx*nty*ntz; key ntiles = removed particle
};

AGPU_HD int tile_key(const TileGeo& t, int i, int j, int k) {
  int a = (i - 3), b = (j - 3), c = (k - 3);
  if (a < 0 || b < 0 || c < 0) return t.ntiles;
  a /= t.tx;
  b /= t.ty;
  c /= t.tz;
  if (a >= t.ntx || b >= t.nty || c >= t.ntz) return t.ntiles;
  return a + t.ntx * (b + t.nty * c);
}

// tile_key for a kernel compiled for the tile extent (TX, TY, TZ) == (t.tx, t.ty, t.tz).
template <int TX, int TY, int TZ>
AGPU_HD int tile_key_c(const TileGeo& t, int i, int j, int k) {
  unsigned a = (unsigned)(i - 3), b = (unsigned)(j - 3), c = (unsigned)(k - 3);
  a /= TX;
  b /= TY;
  c /= TZ;
  if (a >= (unsigned)t.ntx || b >= (unsigned)t.nty || c >= (unsigned)t.ntz) return t.ntiles;
  return (int)a + t.ntx * ((int)b + t.nty * (int)c);
}

// Warp-aggregated histogram increment of key (all active lanes call it).
__device__ __forceinline__ void hist_add(int* hist, int key) {
  unsigned int act = __activemask();
  unsigned int peers = __match_any_sync(act, key);
  int leader = __ffs(peers) - 1;
  if ((threadIdx.x & 31) == leader) atomicAdd(&hist[key], __popc(peers));
}

struct Scratch;
struct Part32View;
void bin_keys_split(const int* cell, long long np, const Geo& g, const TileGeo& t, int* key, int* hist, unsigned int* err,
                    cudaStream_t st, int sms);
void bin_keys_abs(const double* x, const double* y, const double* z, long long np, const Geo& g, const TileGeo& t,
                  double xmn, double ymn, double zmn, double dxi, double dyi, double dzi, int* key, int* hist,
                  unsigned int* err, cudaStream_t st, int sms);
void bin_finish(const int* key, long long np, const TileGeo& t, const int* hist, int* start, int* cursor, int* perm,
                cudaStream_t st, int sms);
long long perm_compact64(const int* perm, long long nalive, double* part, double* tmp, long long cap, int ndv, bool xbox,
                         double x0, double x1, Scratch& s, cudaStream_t st);
long long perm_compact32(const int* perm, long long nalive, const Part32View& src, const Part32View& dst, bool xbox, int n1p,
                         int nx, Scratch& s, cudaStream_t st);

}  // namespace agpu
