// agpu_bin.cuh — spatial tiles of the particle binning (tile geometry and
// node -> tile key), shared by the tiled push kernels and the binning pass.
#pragma once
#include "agpu_common.cuh"

namespace agpu {

// A tile is TX x TY x TZ integer nodes; node i (Fortran) of an alive particle
// lies in [3, nx+3], so tiles cover nodes 3.. in steps of TX.  The binning
// key of a particle is its tile, its row (y, z) inside the tile and the
// octant of its offset from its node (quadrant in 2D):
//   key = tile * nsub + (ly + ty * lz) * nq + octant,  nsub = ty * tz * nq,
// so tile t's particles are perm[tstart[t * nsub] .. tstart[(t + 1) * nsub]),
// row by row and, inside a row, octant by octant.  A row's octant bucket
// holds about one particle per cell of the row (the lattice points of a cell
// start in different octants and a cell's particles spread over them), so
// a warp of the tile kernel covers one or two buckets: consecutive cells of
// one row, about two lanes per cell, whatever order the window compactions
// and tile changes left the records in.  Its shared-memory reads then hit
// distinct banks and its atomics few lanes per address.  Key nkeys =
// ntiles * nsub marks a removed particle.
struct TileGeo {
  int tx, ty, tz;     // tile extent in nodes
  int ntx, nty, ntz;  // tiles per axis
  int ntiles;         // ntx*nty*ntz
  int nq;             // offset octants (3D: 8) or quadrants (2D: 4)
  int nsub;           // keys per tile, ty*tz*nq
  int nkeys;          // ntiles*nsub; key nkeys = removed particle
};

// octant (quadrant) of a particle's offsets from its node
AGPU_HD int offset_octant(float ox, float oy, float oz, int ndim) {
  return (ox >= 0.f ? 1 : 0) + (oy >= 0.f ? 2 : 0) + ((ndim == 3 && oz >= 0.f) ? 4 : 0);
}

AGPU_HD int tile_key(const TileGeo& t, int i, int j, int k, int oct) {
  const int a = (i - 3), b = (j - 3), c = (k - 3);
  if (a < 0 || b < 0 || c < 0) return t.nkeys;
  const int ta = a / t.tx, tb = b / t.ty, tc = c / t.tz;
  if (ta >= t.ntx || tb >= t.nty || tc >= t.ntz) return t.nkeys;
  const int tile = ta + t.ntx * (tb + t.nty * tc);
  return tile * t.nsub + ((b - tb * t.ty) + t.ty * (c - tc * t.tz)) * t.nq + oct;
}

// tile_key for a kernel compiled for the tile extent (TX, TY, TZ) == (t.tx,
// t.ty, t.tz) and NQ == t.nq.
template <int TX, int TY, int TZ, int NQ>
AGPU_HD int tile_key_c(const TileGeo& t, int i, int j, int k, int oct) {
  const unsigned a = (unsigned)(i - 3), b = (unsigned)(j - 3), c = (unsigned)(k - 3);
  const unsigned ta = a / TX, tb = b / TY, tc = c / TZ;
  if (ta >= (unsigned)t.ntx || tb >= (unsigned)t.nty || tc >= (unsigned)t.ntz) return t.nkeys;
  const int tile = (int)ta + t.ntx * ((int)tb + t.nty * (int)tc);
  return tile * (TY * TZ * NQ) + ((int)(b - tb * TY) + TY * (int)(c - tc * TZ)) * NQ + oct;
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
void bin_keys_split(const int* cell, const float* ox, const float* oy, const float* oz, long long np, const Geo& g,
                    const TileGeo& t, int* key, int* hist, unsigned int* err, cudaStream_t st, int sms);
void bin_keys_abs(const double* x, const double* y, const double* z, long long np, const Geo& g, const TileGeo& t,
                  double xmn, double ymn, double zmn, double dxi, double dyi, double dzi, int* key, int* hist,
                  unsigned int* err, cudaStream_t st, int sms);
// Returns the number of kernels it launched.
int bin_finish(const int* key, long long np, const TileGeo& t, const int* hist, int* start, int* cursor, int* perm,
               int* scan_tmp, cudaStream_t st, int sms);
// ints of bin_finish's scan_tmp
int bin_scan_tmp_ints(const TileGeo& t);
long long perm_compact64(const int* perm, long long nalive, double* part, double* tmp, long long cap, int ndv, bool xbox,
                         double x0, double x1, Scratch& s, cudaStream_t st);
long long perm_compact32(const int* perm, long long nalive, const Part32View& src, const Part32View& dst, bool xbox, int n1p,
                         int nx, Scratch& s, cudaStream_t st);

}  // namespace agpu
