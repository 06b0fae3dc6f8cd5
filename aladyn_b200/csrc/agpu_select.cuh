// agpu_select.cuh — stable selection (order-preserving compaction and
// append) templated on a predicate and a mover; shared by agpu_util.cu and
// agpu_bin.cu.
#pragma once
#include "agpu_common.cuh"
#include "agpu_util.h"

namespace agpu {

// ============================================================================
// Stable selection.  Each block owns SEL_CHUNK consecutive elements; warp w
// of the block owns the w-th run of 32*SEL_ITEMS of them and walks it in
// 32-element groups with a ballot, so reads and writes stay coalesced and
// the kept elements leave in their original order (the reference compacts
// in order: mpi_part_interface.f90:496-519).
// ============================================================================
template <class Pred>
__global__ void __launch_bounds__(SEL_BLOCK) k_sel_count(Pred pr, long long n, long long* blockcnt) {
  __shared__ int wsum[SEL_BLOCK / 32];
  long long base = (long long)blockIdx.x * SEL_CHUNK;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  long long wbase = base + (long long)warp * 32 * SEL_ITEMS;
  int cnt = 0;
  for (int it = 0; it < SEL_ITEMS; ++it) {
    long long i = wbase + it * 32 + lane;
    bool keep = (i < n) && pr(i);
    cnt += __popc(__ballot_sync(0xffffffffu, keep));
  }
  if (lane == 0) wsum[warp] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long s = 0;
    for (int w = 0; w < SEL_BLOCK / 32; ++w) s += wsum[w];
    blockcnt[blockIdx.x] = s;
  }
}

// Exclusive scan of the block counts in one block; total into *total.
static __global__ void k_scan_blocks(long long* cnt, long long nb, long long* total) {
  __shared__ long long part[1024];
  long long per = (nb + blockDim.x - 1) / blockDim.x;
  long long lo = threadIdx.x * per, hi = min(lo + per, nb);
  long long s = 0;
  for (long long b = lo; b < hi; ++b) s += cnt[b];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long run = 0;
    for (int t = 0; t < (int)blockDim.x; ++t) {
      long long v = part[t];
      part[t] = run;
      run += v;
    }
    *total = run;
  }
  __syncthreads();
  long long run = part[threadIdx.x];
  for (long long b = lo; b < hi; ++b) {
    long long v = cnt[b];
    cnt[b] = run;
    run += v;
  }
}

template <class Pred, class Move>
__global__ void __launch_bounds__(SEL_BLOCK) k_sel_scatter(Pred pr, Move mv, long long n, const long long* blockoff) {
  __shared__ int wsum[SEL_BLOCK / 32];
  __shared__ long long woff[SEL_BLOCK / 32];
  long long base = (long long)blockIdx.x * SEL_CHUNK;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  long long wbase = base + (long long)warp * 32 * SEL_ITEMS;
  int cnt = 0;
  for (int it = 0; it < SEL_ITEMS; ++it) {
    long long i = wbase + it * 32 + lane;
    bool keep = (i < n) && pr(i);
    cnt += __popc(__ballot_sync(0xffffffffu, keep));
  }
  if (lane == 0) wsum[warp] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long s = blockoff[blockIdx.x];
    for (int w = 0; w < SEL_BLOCK / 32; ++w) {
      woff[w] = s;
      s += wsum[w];
    }
  }
  __syncthreads();
  long long o = woff[warp];
  for (int it = 0; it < SEL_ITEMS; ++it) {
    long long i = wbase + it * 32 + lane;
    bool keep = (i < n) && pr(i);
    unsigned int m = __ballot_sync(0xffffffffu, keep);
    if (keep) mv(i, o + __popc(m & ((1u << lane) - 1u)));
    o += __popc(m);
  }
}

template <class Pred, class Move>
long long select_run(Pred pr, Move mv, long long n, Scratch& s, cudaStream_t st) {
  if (n <= 0) return 0;
  long long nb = (n + SEL_CHUNK - 1) / SEL_CHUNK;
  k_sel_count<Pred><<<(unsigned)nb, SEL_BLOCK, 0, st>>>(pr, n, s.blockcnt);
  k_scan_blocks<<<1, 1024, 0, st>>>(s.blockcnt, nb, s.total);
  k_sel_scatter<Pred, Move><<<(unsigned)nb, SEL_BLOCK, 0, st>>>(pr, mv, n, s.blockcnt);
  long long tot = 0;
  cudaMemcpyAsync(s.h_total, s.total, sizeof(long long), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  tot = *s.h_total;
  return tot;
}

}  // namespace agpu
