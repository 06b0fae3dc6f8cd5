// agpu_bin.cu — per-step binning of particles by spatial tile: a key per
// particle (its tile and row inside the tile, or the removed bin), a
// histogram, an exclusive scan and a scatter of particle indices into the
// permutation perm, so that tile t's particles are
// perm[tstart[t * nsub] .. tstart[(t + 1) * nsub]), row by row.  The particle records stay
// where they are; the permutation is rebuilt every step from the keys that
// the push kernel writes, and the records are physically reordered along it
// whenever the window compaction copies them.
#include "agpu_bin.cuh"
#include "agpu_multi.h"
#include "agpu_util.h"
#include "agpu_select.cuh"

namespace agpu {

// keys from the split form's node index and offsets
__global__ void k_keys_split(const int* cell, const float* ox, const float* oy, const float* oz, long long np, Geo g,
                             TileGeo t, int* key, int* hist, unsigned int* err) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < np; n += (long long)gridDim.x * blockDim.x) {
    int c = cell[n];
    int i, j, k;
    cell_split(g, c, i, j, k);
    if (g.ndim != 3) k = 3;
    int kk = tile_key(t, i, j, k, offset_octant(ox[n], oy[n], (g.ndim == 3) ? oz[n] : 0.f, g.ndim));
    key[n] = kk;
    if (kk == t.nkeys) raise_err(err, AGPU_EBIT_INDEX);  // a record outside the node range
    hist_add(hist, kk);
  }
}

// keys from FP64 absolute positions: node = int(3 + x_loc + 0.5) (qden)
__global__ void k_keys_abs(const double* x, const double* y, const double* z, long long np, Geo g, TileGeo t,
                           double xmn, double ymn, double zmn, double dxi, double dyi, double dzi, int* key, int* hist,
                           unsigned int* err) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < np; n += (long long)gridDim.x * blockDim.x) {
    double xx = 3.0 + dxi * (x[n] - xmn);
    double yy = 3.0 + dyi * (y[n] - ymn);
    int i = (xx > -1e9 && xx < 2e9) ? (int)(xx + 0.5) : -1;
    int j = (yy > -1e9 && yy < 2e9) ? (int)(yy + 0.5) : -1;
    int k = 3;
    float sz = 0.f;
    if (g.ndim == 3) {
      double zz = 3.0 + dzi * (z[n] - zmn);
      k = (zz > -1e9 && zz < 2e9) ? (int)(zz + 0.5) : -1;
      sz = (float)(zz - (double)k);
    }
    int kk = tile_key(t, i, j, k, offset_octant((float)(xx - (double)i), (float)(yy - (double)j), sz, g.ndim));
    key[n] = kk;
    if (kk == t.nkeys) raise_err(err, AGPU_EBIT_INDEX);  // a record outside the node range
    hist_add(hist, kk);
  }
}

// Exclusive scan of hist[0..nb) into start[0..nb], one block.
__device__ void d_scan_int(const int* hist, int nb, int* start) {
  __shared__ long long part[1024];
  int per = (nb + blockDim.x - 1) / blockDim.x;
  int lo = threadIdx.x * per, hi = min(lo + per, nb);
  long long s = 0;
  for (int b = lo; b < hi; ++b) s += hist[b];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long run = 0;
    for (int q = 0; q < (int)blockDim.x; ++q) {
      long long v = part[q];
      part[q] = run;
      run += v;
    }
    start[nb] = (int)run;
  }
  __syncthreads();
  long long run = part[threadIdx.x];
  for (int b = lo; b < hi; ++b) {
    start[b] = (int)run;
    run += hist[b];
  }
}
__global__ void k_scan_int(const int* hist, int nb, int* start) { d_scan_int(hist, nb, start); }

// perm[start[key] + rank] = n, ranks from warp-aggregated cursors.  Each warp
// takes SC_U consecutive runs of 32 records per pass, so that SC_U cursor
// atomics (one round trip to L2 each) are in flight together; the lanes of
// a run with one key get consecutive slots in lane order.  Warp-uniform loop
// (blockDim a multiple of 32).
constexpr int SC_U = 4;
__device__ void d_perm_scatter(const int* key, long long np, const int* start, int* cursor, int* perm, long long bid_,
                               long long nb_) {
  const int lane = threadIdx.x & 31;
  const long long warp = (bid_ * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = (nb_ * (long long)blockDim.x) >> 5;
  for (long long base = warp * 32 * SC_U; base < np; base += nwarps * 32 * SC_U) {
    int kk[SC_U], b[SC_U], rank[SC_U], lead[SC_U];
#pragma unroll
    for (int u = 0; u < SC_U; ++u) {
      const long long n = base + u * 32 + lane;
      kk[u] = (n < np) ? key[n] : -1;
    }
#pragma unroll
    for (int u = 0; u < SC_U; ++u) {
      const unsigned peers = __match_any_sync(0xffffffffu, kk[u]);
      lead[u] = __ffs(peers) - 1;
      rank[u] = __popc(peers & ((1u << lane) - 1u));
      b[u] = 0;
      if (lane == lead[u] && kk[u] >= 0) b[u] = atomicAdd(&cursor[kk[u]], __popc(peers));
    }
#pragma unroll
    for (int u = 0; u < SC_U; ++u) {
      const int bb = __shfl_sync(0xffffffffu, b[u], lead[u]);
      if (kk[u] >= 0) perm[start[kk[u]] + bb + rank[u]] = (int)(base + u * 32 + lane);
    }
  }
}
__global__ void k_perm_scatter(const int* key, long long np, const int* start, int* cursor, int* perm) {
  d_perm_scatter(key, np, start, cursor, perm, blockIdx.x, gridDim.x);
}

void bin_keys_split(const int* cell, const float* ox, const float* oy, const float* oz, long long np, const Geo& g,
                    const TileGeo& t, int* key, int* hist, unsigned int* err, cudaStream_t st, int sms) {
  if (np <= 0) return;
  k_keys_split<<<grid_for(np, 256, sms, 16), 256, 0, st>>>(cell, ox, oy, oz, np, g, t, key, hist, err);
}
void bin_keys_abs(const double* x, const double* y, const double* z, long long np, const Geo& g, const TileGeo& t,
                  double xmn, double ymn, double zmn, double dxi, double dyi, double dzi, int* key, int* hist,
                  unsigned int* err, cudaStream_t st, int sms) {
  if (np <= 0) return;
  k_keys_abs<<<grid_for(np, 256, sms, 16), 256, 0, st>>>(x, y, z, np, g, t, xmn, ymn, zmn, dxi, dyi, dzi, key, hist, err);
}
// ---- exclusive scan of many bins: block sums, a scan of the block sums,
// then each block's scan offset by its block's start -------------------------
constexpr int SCAN_ITEMS = 16, SCAN_THREADS = 256, SCAN_BLOCK = SCAN_ITEMS * SCAN_THREADS;

__device__ __forceinline__ int block_exclusive_sum(int v, int* s_warp, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += u;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      const int x = s_warp[w];
      s_warp[w] = run;
      run += x;
    }
    *total = run;
  }
  __syncthreads();
  return s_warp[warp] + inc - v;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_sums(const int* hist, int n, int* bsum) {
  __shared__ int s_warp[SCAN_THREADS / 32];
  __shared__ int s_total;
  const int base = blockIdx.x * SCAN_BLOCK;
  int v = 0;
  for (int e = threadIdx.x; e < SCAN_BLOCK; e += blockDim.x)
    if (base + e < n) v += hist[base + e];
  block_exclusive_sum(v, s_warp, &s_total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = s_total;
}

// start[i] = boff[block] + exclusive sum inside the block; start[n] = total
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_apply(const int* hist, int n, const int* boff, int* start) {
  __shared__ int s_warp[SCAN_THREADS / 32];
  __shared__ int s_total;
  const int base = blockIdx.x * SCAN_BLOCK + threadIdx.x * SCAN_ITEMS;
  int v[SCAN_ITEMS];
  int sum = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    v[k] = (base + k < n) ? hist[base + k] : 0;
    sum += v[k];
  }
  int run = boff[blockIdx.x] + block_exclusive_sum(sum, s_warp, &s_total);
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    if (base + k < n) start[base + k] = run;
    run += v[k];
    if (base + k == n - 1) start[n] = run;
  }
}

// hist has nkeys+1 bins (the last one: removed particles).  scan_tmp holds
// bin_scan_tmp_ints(t) ints.  Returns the kernels launched.
int bin_finish(const int* key, long long np, const TileGeo& t, const int* hist, int* start, int* cursor, int* perm,
               int* scan_tmp, cudaStream_t st, int sms) {
  const int n = t.nkeys + 1;
  const int nb = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
  if (nb <= 1) {
    k_scan_int<<<1, 1024, 0, st>>>(hist, n, start);
  } else {
    int* bsum = scan_tmp;
    int* boff = scan_tmp + nb + 1;
    k_scan_sums<<<nb, SCAN_THREADS, 0, st>>>(hist, n, bsum);
    k_scan_int<<<1, 1024, 0, st>>>(bsum, nb, boff);
    k_scan_apply<<<nb, SCAN_THREADS, 0, st>>>(hist, n, boff, start);
  }
  cudaMemsetAsync(cursor, 0, sizeof(int) * n, st);
  if (np > 0) k_perm_scatter<<<grid_for(np, 256, sms, 16), 256, 0, st>>>(key, np, start, cursor, perm);
  return (nb <= 1 ? 1 : 3) + (np > 0 ? 1 : 0);
}
int bin_scan_tmp_ints(const TileGeo& t) { return 2 * ((t.nkeys + 1) / SCAN_BLOCK + 3); }

// ---- compaction along the permutation (physical reorder by tile) --------
struct PermAlive {
  const int* perm;
  long long nalive;
  __device__ bool operator()(long long q) const { return q < nalive; }
};
struct PermAliveInBox64 {
  const int* perm;
  long long nalive;
  const double* x;
  double x0, x1;
  __device__ bool operator()(long long q) const {
    if (q >= nalive) return false;
    double a = x[perm[q]];
    return a > x0 && a <= x1;
  }
};
struct PermMove64 {
  const int* perm;
  const double* src;
  double* dst;
  long long ld;
  int ndv;
  __device__ void operator()(long long q, long long o) const {
    long long p = perm[q];
    for (int c = 0; c < ndv; ++c) dst[(long long)c * ld + o] = src[(long long)c * ld + p];
  }
};
long long perm_compact64(const int* perm, long long nalive, double* part, double* tmp, long long cap, int ndv, bool xbox,
                         double x0, double x1, Scratch& s, cudaStream_t st) {
  PermMove64 mv{perm, part, tmp, cap, ndv};
  if (xbox) {
    PermAliveInBox64 pr{perm, nalive, part, x0, x1};
    return select_run(pr, mv, nalive, s, st);
  }
  PermAlive pr{perm, nalive};
  return select_run(pr, mv, nalive, s, st);
}

struct PermAliveInBox32 {
  const int* perm;
  long long nalive;
  const int* cell;
  const float* ox;
  int n1p, nx;
  __device__ bool operator()(long long q) const {
    if (q >= nalive) return false;
    int p = perm[q];
    int i = cell[p] % n1p + 1;
    int m = i - 3;
    float o = ox[p];
    return ((m > 0) || (m == 0 && o > 0.f)) && ((m < nx) || (m == nx && o <= 0.f));
  }
};
struct PermMove32 {
  const int* perm;
  Part32View src, dst;
  __device__ void operator()(long long q, long long o) const {
    int p = perm[q];
    dst.cell[o] = src.cell[p];
    dst.ox[o] = src.ox[p];
    dst.oy[o] = src.oy[p];
    dst.px[o] = src.px[p];
    dst.py[o] = src.py[p];
    dst.slot[o] = src.slot[p];
    if (src.oz) {
      dst.oz[o] = src.oz[p];
      dst.pz[o] = src.pz[p];
    }
  }
};
long long perm_compact32(const int* perm, long long nalive, const Part32View& src, const Part32View& dst, bool xbox, int n1p,
                         int nx, Scratch& s, cudaStream_t st) {
  PermMove32 mv{perm, src, dst};
  if (xbox) {
    PermAliveInBox32 pr{perm, nalive, src.cell, src.ox, n1p, nx};
    return select_run(pr, mv, nalive, s, st);
  }
  PermAlive pr{perm, nalive};
  return select_run(pr, mv, nalive, s, st);
}


// ---- multi-instance binning: scan (one block per instance), scatter ------
namespace {
__global__ void km_scan(const MultiInst* __restrict__ d) {
  const MultiInst& m = d[blockIdx.x];
  d_scan_int(m.ta.hist, m.ta.t.nkeys + 1, const_cast<int*>(m.ta.tstart));
}
__global__ void km_scatter(const MultiInst* __restrict__ d) {
  const MultiInst& m = d[blockIdx.y];
  d_perm_scatter(m.ta.key, m.np, m.ta.tstart, m.cursor, const_cast<int*>(m.ta.perm), blockIdx.x, gridDim.x);
}
}  // namespace

void multi_bin32(const MultiInst* d, const MultiPlan& pl, cudaStream_t st, int* launches) {
  km_scan<<<pl.n, 1024, 0, st>>>(d);
  km_scatter<<<dim3(pl.gx_parts, pl.n), 256, 0, st>>>(d);
  *launches += 2;
}

}  // namespace agpu
