// agpu_tile32.cu — tiled gather + push + deposit of the FP32 split form.
//
// One CTA of 256 threads per spatial tile of TX x TY x TZ nodes (3D 32x4x4,
// 2D 32x8).  The tile's particles are the permutation range
// perm[tstart[t] .. tstart[t+1]) of the binning pass (every particle's
// nearest node lies inside the tile).  The CTA
//   1. stages the tile's field components plus a one-node guard (the qlh
//      gather stencil) into shared memory and zeroes a shared FP32 current
//      tile with a two-node guard (the Esirkepov window of a particle that
//      moves at most one node);
//   2. sorts the tile's particles by node in shared memory (counting sort:
//      per-node counts, a block scan, a scatter of the record indices);
//   3. gives every thread one node at a time, the threads of a warp the 32
//      consecutive nodes of one x-row: the thread gathers, pushes
//      (exact-gamma Boris) and deposits each particle of its node in turn.
//      A particle that keeps its nearest node (most of them) deposits on
//      the fixed 3x3[x3] slots around that node, so its Esirkepov terms are
//      summed in FP32 registers over all particles of the node and reach
//      shared memory once per node (54 shared atomics per node in 3D
//      instead of per particle).  A particle that changes node is queued
//      per warp and deposited on its full window by 32 lanes at a time;
//   4. flushes the shared currents once to the global (hi, lo) pair with
//      the TwoSum error of each global add accumulated into lo (compensated
//      accumulation), and writes each particle's new tile key and the next
//      histogram.
// Every current contribution is an FP32 product summed in FP32: no fixed
// point, so the discrete continuity of the Esirkepov currents holds to FP32
// round-off.  A tile with more particles than the shared node list holds
// (a dense tile, more than 1.5 times the mean at 8 particles per cell) runs
// the same gather, push and full-window deposit one particle per thread.
#include "agpu_bin.cuh"
#include "agpu_common.cuh"
#include "agpu_multi.h"
#include "agpu_tile.h"

namespace agpu {

namespace {

constexpr int NT = 256;  // threads per CTA
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ void wq(float s, float a[3]) {
  float s2 = s * s;
  a[1] = 0.75f - s2;
  a[2] = 0.5f * (0.25f + s2 + s);
  a[0] = 1.f - a[1] - a[2];
}

// New shape on the 5-slot window (slot 0 = old node - 2; the new node is
// old node + ih - 1) and the running sum cur(q) = sum_{m <= q} (S0 - S1).
__device__ __forceinline__ void esirk1(const float a0[3], const float a1[3], int ih, float axh[5], float cur[5]) {
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    int m = q - ih;
    axh[q] = (m == 0) ? a1[0] : (m == 1) ? a1[1] : (m == 2) ? a1[2] : 0.f;
  }
  cur[0] = -axh[0];
  cur[1] = cur[0] + a0[0] - axh[1];
  cur[2] = cur[1] + a0[1] - axh[2];
  cur[3] = cur[2] + a0[2] - axh[3];
  cur[4] = cur[3] - axh[4];
}

__device__ __forceinline__ int renorm(float& s) {
  int m = (s >= 0.5f) ? 1 : ((s < -0.5f) ? -1 : 0);
  s = s - (float)m;
  return m;
}
__device__ __forceinline__ bool inside(int node, float o, int n) {
  int m = node - 3;
  return ((m > 0) || (m == 0 && o > 0.f)) && ((m < n) || (m == n && o <= 0.f));
}

// Tile constants of the split-form kernel.
template <int NDIM>
struct CT {
  static constexpr int TX = (NDIM == 3) ? TILE3_X : TILE2_X;
  static constexpr int TY = (NDIM == 3) ? TILE3_Y : TILE2_Y;
  static constexpr int TZ = (NDIM == 3) ? TILE3_Z : 1;
  static constexpr int NCELL = TX * TY * TZ;
  static constexpr int NPASS = NCELL / NT;  // nodes per thread
  static constexpr int FX = TX + 2, FY = TY + 2, FZ = (NDIM == 3) ? TZ + 2 : 1;
  static constexpr int JX = TX + 4, JY = TY + 4, JZ = (NDIM == 3) ? TZ + 4 : 1;
  static constexpr int FV = FX * FY * FZ, JV = JX * JY * JZ;
  static constexpr int NF = (NDIM == 3) ? 6 : 3, NC = (NDIM == 3) ? 3 : 2;
  static constexpr int NSUB = TY * TZ * ((NDIM == 3) ? 8 : 4);  // binning keys per tile
  static constexpr int LIST_CAP = (NDIM == 3) ? 6144 : 4096;  // node-sorted record indices
  static constexpr int QCAP = 48;                               // mover queue entries per warp
  static constexpr int QDRAIN = 16;                             // drain the queue from this fill on
  static constexpr int QW = 8;                                  // words per queue entry
  static constexpr int NACC = (NDIM == 3) ? 54 : 12;            // register sums of a node
  // dynamic shared memory, in 4-byte words (the 8-byte slot staging first);
  // two staging buffers: the copy of record k+1 never lands on the words
  // that record k is read from
  static constexpr int W_SLOT = 0;                  // 2 x NT packed slots of the next records
  static constexpr int W_REC = W_SLOT + 4 * NT;     // 2 x 6 x NT offsets and momenta of the next records
  static constexpr int W_F = W_REC + 12 * NT;
  static constexpr int W_J = W_F + NF * FV;
  static constexpr int W_START = W_J + NC * JV;
  static constexpr int W_CUR = W_START + NCELL + 1;
  static constexpr int W_LIST = W_CUR + NCELL;
  static constexpr int W_Q = W_LIST + LIST_CAP;
  static constexpr int WORDS = W_Q + (NT / 32) * QW * QCAP;
  static_assert(QCAP >= QDRAIN - 1 + 32, "a warp adds at most 32 entries per iteration");
  static_assert(NCELL % NT == 0 && TX == 32, "one x-row of 32 nodes per warp");
};

// One particle record as the push reads it.
struct Rec {
  float ox, oy, oz, px, py, pz;
  uint64_t slot;
};

// Asynchronous 4- and 8-byte copies global -> shared (cp.async, sm_80+):
// the next record of a thread's node is fetched while it pushes the
// current one, without holding registers for the loads.
__device__ __forceinline__ void cpa4(void* sdst, const void* gsrc) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cpa8(void* sdst, const void* gsrc) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gsrc) : "memory");
}
// 4-byte copy, or a zero fill (no read) when !valid
__device__ __forceinline__ void cpa4z(void* sdst, const void* gsrc, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
  const int n = valid ? 4 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(gsrc), "r"(n) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// What a push leaves for the deposit.
struct Moved {
  float sx, sy, sz;     // offsets before the push
  float nsx, nsy, nsz;  // offsets after it, from the new nearest node
  int mi, mj, mk;       // node change (-1, 0, 1)
  float wght;           // charge * weight (real(charge * wgh, sp))
  bool keep;            // still inside the box
};

template <int NDIM>
__device__ __forceinline__ Rec load_rec(const TileArgs32& a, int p) {
  Rec r;
  r.ox = a.p.ox[p];
  r.oy = a.p.oy[p];
  r.oz = (NDIM == 3) ? a.p.oz[p] : 0.f;
  r.px = a.p.px[p];
  r.py = a.p.py[p];
  r.pz = (NDIM == 3) ? a.p.pz[p] : 0.f;
  r.slot = a.p.slot[p];
  return r;
}

// Gather (qlh shapes from the staged fields; fx, fy, fz = local field
// coordinates of node i0-1, j0-1, k0-1), init_lpf_momenta on the first step,
// the exact-gamma Boris push, the new position and record of particle p, and
// its new binning key.
template <int NDIM>
__device__ __forceinline__ Moved push_one(const TileArgs32& a, const float* __restrict__ sF, int* sHist, int kbase,
                                          int p, const Rec& rec, int i0, int j0, int k0, int fx, int fy, int fz, int nx,
                                          int ny, int nz, bool interior, int nodekey) {
  using C = CT<NDIM>;
  constexpr int FX = C::FX, FY = C::FY, FV = C::FV;
  const Geo& g = a.g;
  Moved o;
  float sx = rec.ox, sy = rec.oy, sz = rec.oz;
  float pp[3] = {rec.px, rec.py, rec.pz};
  const uint64_t sl = rec.slot;
  float ax1[3], ay1[3], az1[3] = {0.f, 1.f, 0.f};
  wq(sx, ax1);
  wq(sy, ay1);
  if (NDIM == 3) wq(sz, az1);
  const float axh[2] = {0.5f - sx, sx + 0.5f};
  const float ayh[2] = {0.5f - sy, sy + 0.5f};
  const float azh[2] = {0.5f - sz, sz + 0.5f};
  float ap[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (NDIM == 3) {
    const float* e1 = sF;
    const float* e2 = sF + FV;
    const float* e3 = sF + 2 * FV;
    const float* b1 = sF + 3 * FV;
    const float* b2 = sF + 4 * FV;
    const float* b3 = sF + 5 * FV;
#pragma unroll
    for (int k1 = 0; k1 < 3; ++k1) {
#pragma unroll
      for (int j1 = 0; j1 < 3; ++j1) {
        int q = fx + FX * (fy + j1 + FY * (fz + k1));
        ap[0] += ay1[j1] * az1[k1] * (axh[0] * e1[q] + axh[1] * e1[q + 1]);
      }
#pragma unroll
      for (int j1 = 0; j1 < 2; ++j1) {
        int q = fx + FX * (fy + j1 + FY * (fz + k1));
        float dv = ayh[j1] * az1[k1];
        ap[1] += dv * (ax1[0] * e2[q] + ax1[1] * e2[q + 1] + ax1[2] * e2[q + 2]);
        ap[5] += dv * (axh[0] * b3[q] + axh[1] * b3[q + 1]);
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < 2; ++k1) {
#pragma unroll
      for (int j1 = 0; j1 < 2; ++j1) {
        int q = fx + FX * (fy + j1 + FY * (fz + k1));
        ap[3] += ayh[j1] * azh[k1] * (ax1[0] * b1[q] + ax1[1] * b1[q + 1] + ax1[2] * b1[q + 2]);
      }
#pragma unroll
      for (int j1 = 0; j1 < 3; ++j1) {
        int q = fx + FX * (fy + j1 + FY * (fz + k1));
        float dv = ay1[j1] * azh[k1];
        ap[4] += dv * (axh[0] * b2[q] + axh[1] * b2[q + 1]);
        ap[2] += dv * (ax1[0] * e3[q] + ax1[1] * e3[q + 1] + ax1[2] * e3[q + 2]);
      }
    }
  } else {
    const float* e1 = sF;
    const float* e2 = sF + FV;
    const float* b3 = sF + 2 * FV;
#pragma unroll
    for (int j1 = 0; j1 < 3; ++j1) {
      int q = fx + FX * (fy + j1);
      ap[0] += ay1[j1] * (axh[0] * e1[q] + axh[1] * e1[q + 1]);
    }
#pragma unroll
    for (int j1 = 0; j1 < 2; ++j1) {
      int q = fx + FX * (fy + j1);
      ap[1] += ayh[j1] * (ax1[0] * e2[q] + ax1[1] * e2[q + 1] + ax1[2] * e2[q + 2]);
      ap[5] += ayh[j1] * (axh[0] * b3[q] + axh[1] * b3[q + 1]);
    }
  }
  const float qc = (float)slot_charge(sl);
  if (a.initial) {
    // init_lpf_momenta (boris_push.f90:34-73): p^0 -> p^{-1/2}
    float alp0 = a.dth * a.lfact * qc;
    float gi = rsqrtf(1.f + pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2]);
    float v0 = gi * pp[0], v1 = gi * pp[1], v2 = gi * pp[2];
    float e[6];
#pragma unroll
    for (int cc = 0; cc < 6; ++cc) e[cc] = -alp0 * ap[cc];
    pp[0] = pp[0] + e[0] + v1 * e[5] - v2 * e[4];
    pp[1] = pp[1] + e[1] + v2 * e[3] - v0 * e[5];
    pp[2] = pp[2] + e[2] + v0 * e[4] - v1 * e[3];
  }
  // exact-gamma Boris (boris_push.f90:75-168)
  const float alp = a.dth * a.lfact * qc;
  const float vp[3] = {pp[0] + alp * ap[0], pp[1] + alp * ap[1], pp[2] + alp * ap[2]};
  const float bb[3] = {alp * ap[3], alp * ap[4], alp * ap[5]};
  const float b2v = bb[0] * bb[0] + bb[1] * bb[1] + bb[2] * bb[2];
  const float bv = bb[0] * vp[0] + bb[1] * vp[1] + bb[2] * vp[2];
  const float gam02 = 1.f + vp[0] * vp[0] + vp[1] * vp[1] + vp[2] * vp[2] - b2v;
  const float gam2 = 0.5f * (gam02 + sqrtf(gam02 * gam02 + 4.f * (b2v + bv * bv)));
  const float gam = sqrtf(gam2);
  const float inv = 1.f / (b2v + gam2);
  float pn[3];
  pn[0] = 2.f * (gam2 * vp[0] + bb[0] * bv + gam * (vp[1] * bb[2] - vp[2] * bb[1])) * inv - pp[0];
  pn[1] = 2.f * (gam2 * vp[1] + bb[1] * bv + gam * (vp[2] * bb[0] - vp[0] * bb[2])) * inv - pp[1];
  pn[2] = (NDIM == 3) ? 2.f * (gam2 * vp[2] + bb[2] * bv + gam * (vp[0] * bb[1] - vp[1] * bb[0])) * inv - pp[2] : 0.f;
  const float dtg = rsqrtf(1.f + pn[0] * pn[0] + pn[1] * pn[1] + pn[2] * pn[2]);
  float nsx = sx + a.dtx * dtg * pn[0];
  float nsy = sy + a.dty * dtg * pn[1];
  float nsz = (NDIM == 3) ? sz + a.dtz * dtg * pn[2] : 0.f;
  const int mi = renorm(nsx), mj = renorm(nsy), mk = (NDIM == 3) ? renorm(nsz) : 0;
  const int i1n = i0 + mi, j1n = j0 + mj, k1n = k0 + mk;
  a.p.ox[p] = nsx;
  a.p.oy[p] = nsy;
  a.p.px[p] = pn[0];
  a.p.py[p] = pn[1];
  if (NDIM == 3) {
    a.p.oz[p] = nsz;
    a.p.pz[p] = pn[2];
  }
  if (!(pn[0] == pn[0] && pn[1] == pn[1] && pn[2] == pn[2])) raise_err(a.err, AGPU_EBIT_NONFINITE);
  bool keep = true;
  if ((mi | mj | mk) == 0 && interior) {
    // kept its node, away from the box edges: same cell, same tile row,
    // new octant; the next histogram counted in shared memory
    const int nkey = nodekey + offset_octant(nsx, nsy, nsz, NDIM);
    a.key[p] = nkey;
    atomicAdd(&sHist[nkey - kbase], 1);
  } else {
    a.p.cell[p] = (int)goff(g, i1n, j1n, k1n);
    keep = inside(i1n, nsx, nx) && inside(j1n, nsy, ny);
    if (NDIM == 3) keep = keep && inside(k1n, nsz, nz);
    const int nkey = keep ? tile_key_c<C::TX, C::TY, C::TZ, (NDIM == 3) ? 8 : 4>(
                                a.t, i1n, j1n, (NDIM == 3) ? k1n : 3, offset_octant(nsx, nsy, nsz, NDIM))
                          : a.t.nkeys;
    a.key[p] = nkey;
    // keys of this tile counted in shared memory, added to the global
    // histogram once per tile
    if ((unsigned)(nkey - kbase) < (unsigned)C::NSUB)
      atomicAdd(&sHist[nkey - kbase], 1);
    else
      hist_add(a.hist, nkey);
  }
  o.sx = sx;
  o.sy = sy;
  o.sz = sz;
  o.nsx = nsx;
  o.nsy = nsy;
  o.nsz = nsz;
  o.mi = mi;
  o.mj = mj;
  o.mk = mk;
  o.wght = qc * slot_wgh(sl);
  o.keep = keep;
  return o;
}

// Esirkepov deposit of one particle on its full window (grid_part_connect.f90:
// 956-1334) into the shared FP32 current tile; (lx, ly, lz) = local current
// coordinates of window slot 0 (old node - 2).  The old-plane and new-plane
// terms are regrouped onto the window slots: each component is one dense
// product over (x0..x1) x (y0..y1) [x (z0..z1)], its last slot along its own
// axis skipped (the running sum ends there at sum(S0) - sum(S1) = 0).  Each
// window is compacted to the four slots x0 .. x0+3 that can be non-zero.
template <int NDIM>
__device__ __forceinline__ void deposit_window(float* sJ, int lx, int ly, int lz, const Moved& m) {
  using C = CT<NDIM>;
  constexpr int JX = C::JX, JY = C::JY, JV = C::JV;
  const float wsc = m.wght;
  float ax0[3], ay0[3], axn[3], ayn[3];
  wq(m.sx, ax0);
  wq(m.sy, ay0);
  wq(m.nsx, axn);
  wq(m.nsy, ayn);
  float* sJx = sJ;
  float* sJy = sJ + JV;
  if (NDIM == 2) {
    float sxh[5], cx[5], syh[5], cy[5];
    const int ih = m.mi + 1, jh = m.mj + 1;
    esirk1(ax0, axn, ih, sxh, cx);
    esirk1(ay0, ayn, jh, syh, cy);
    const int x0 = ih < 1 ? ih : 1, x1 = (ih + 2) > 3 ? ih + 2 : 3;
    const int y0 = jh < 1 ? jh : 1, y1 = (jh + 2) > 3 ? jh + 2 : 3;
    float wxs[5], wys[5];
#pragma unroll
    for (int u = 0; u < 5; ++u) {
      cx[u] *= wsc;
      cy[u] *= wsc;
      wxs[u] = sxh[u] + ((u >= 1 && u <= 3) ? ax0[u - 1] : 0.f);
      wys[u] = syh[u] + ((u >= 1 && u <= 3) ? ay0[u - 1] : 0.f);
    }
    float cxc[4], cyc[4], wxc[4], wyc[4];  // index s = window slot x0+s (y0+s)
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      cxc[s] = x0 ? cx[s + 1] : cx[s];
      wxc[s] = x0 ? wxs[s + 1] : wxs[s];
      cyc[s] = y0 ? cy[s + 1] : cy[s];
      wyc[s] = y0 ? wys[s + 1] : wys[s];
    }
    const int nxw = x1 - x0, nyw = y1 - y0;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      if (t > nyw) continue;
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        if (s > nxw) continue;
        const int o = lx + x0 + s + JX * (ly + y0 + t);
        if (s < nxw) atomicAdd(&sJx[o], wyc[t] * cxc[s]);
        if (t < nyw) atomicAdd(&sJy[o], wxc[s] * cyc[t]);
      }
    }
  } else {
    float az0[3], azn[3];
    wq(m.sz, az0);
    wq(m.nsz, azn);
    float* sJz = sJ + 2 * JV;
    float sxh[5], cx[5], syh[5], cy[5], szh[5], cz[5];
    const int ih = m.mi + 1, jh = m.mj + 1, kh = m.mk + 1;
    esirk1(ax0, axn, ih, sxh, cx);
    esirk1(ay0, ayn, jh, syh, cy);
    esirk1(az0, azn, kh, szh, cz);
    const int x0 = ih < 1 ? ih : 1, x1 = (ih + 2) > 3 ? ih + 2 : 3;
    const int y0 = jh < 1 ? jh : 1, y1 = (jh + 2) > 3 ? jh + 2 : 3;
    const int z0 = kh < 1 ? kh : 1, z1 = (kh + 2) > 3 ? kh + 2 : 3;
    float wx0[5], wx1[5], wy0[5], wy1[5], b0[5], b1[5];
#pragma unroll
    for (int u = 0; u < 5; ++u) {
      cx[u] *= wsc;
      cy[u] *= wsc;
      const float a0x = (u >= 1 && u <= 3) ? ax0[u - 1] : 0.f;
      const float a0y = (u >= 1 && u <= 3) ? ay0[u - 1] : 0.f;
      wx0[u] = 0.5f * sxh[u] + a0x;  // axh0
      wx1[u] = sxh[u] + 0.5f * a0x;  // axh1
      wy0[u] = 0.5f * syh[u] + a0y;  // ayh0
      wy1[u] = syh[u] + 0.5f * a0y;  // ayh1
      b0[u] = a0y;                   // old y shape on slots 1..3
      b1[u] = syh[u];                // new y shape
    }
    float cxc[4], wx0c[4], wx1c[4], cyc[4], wy0c[4], wy1c[4], b0c[4], b1c[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      cxc[s] = x0 ? cx[s + 1] : cx[s];
      wx0c[s] = x0 ? wx0[s + 1] : wx0[s];
      wx1c[s] = x0 ? wx1[s + 1] : wx1[s];
      cyc[s] = y0 ? cy[s + 1] : cy[s];
      wy0c[s] = y0 ? wy0[s + 1] : wy0[s];
      wy1c[s] = y0 ? wy1[s + 1] : wy1[s];
      b0c[s] = y0 ? b0[s + 1] : b0[s];
      b1c[s] = y0 ? b1[s + 1] : b1[s];
    }
    const int nxw = x1 - x0, nyw = y1 - y0;
    for (int w = z0; w <= z1; ++w) {
      const int m0 = w - 1;
      const float A0 = (m0 == 0) ? az0[0] : (m0 == 1) ? az0[1] : (m0 == 2) ? az0[2] : 0.f;
      const float A1 = (w == 0) ? szh[0] : (w == 1) ? szh[1] : (w == 2) ? szh[2] : (w == 3) ? szh[3] : szh[4];
      const float czw = wsc * ((w == 0) ? cz[0] : (w == 1) ? cz[1] : (w == 2) ? cz[2] : (w == 3) ? cz[3] : cz[4]);
      const int ow = lx + x0 + JX * (ly + y0 + JY * (lz + w));
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        if (t > nyw) continue;
        const float wyv = wy0c[t] * A0 + wy1c[t] * A1;
        const float cyv = cyc[t];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          if (s > nxw) continue;
          const int o = ow + s + JX * t;
          if (s < nxw) atomicAdd(&sJx[o], cxc[s] * wyv);
          if (t < nyw) atomicAdd(&sJy[o], cyv * (wx0c[s] * A0 + wx1c[s] * A1));
          if (w < z1) atomicAdd(&sJz[o], czw * (wx0c[s] * b0c[t] + wx1c[s] * b1c[t]));
        }
      }
    }
  }
}

// Esirkepov terms of a particle that keeps its nearest node, added to the
// node's register sums.  The window is slots 1..3 around the node; the
// component along each axis skips slot 3 (identically zero).  Layout:
// 3D acc[0..17] = Jx(s<2, t<3, r<3), acc[18..35] = Jy(s<3, t<2, r<3),
// acc[36..53] = Jz(s<3, t<3, r<2); 2D acc[0..5] = Jx(s<2, t<3),
// acc[6..11] = Jy(s<3, t<2); index s = x slot - 1 etc.
template <int NDIM>
__device__ __forceinline__ void accumulate_stay(float* acc, const Moved& m) {
  const float wsc = m.wght;
  float ax0[3], ay0[3], axn[3], ayn[3];
  wq(m.sx, ax0);
  wq(m.sy, ay0);
  wq(m.nsx, axn);
  wq(m.nsy, ayn);
  float cx[2], cy[2];
  cx[0] = (-0.f + ax0[0]) - axn[0];
  cy[0] = (-0.f + ay0[0]) - ayn[0];
  cx[1] = (cx[0] + ax0[1]) - axn[1];
  cy[1] = (cy[0] + ay0[1]) - ayn[1];
  cx[0] *= wsc;
  cx[1] *= wsc;
  cy[0] *= wsc;
  cy[1] *= wsc;
  if (NDIM == 2) {
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      const float wy = ayn[t] + ay0[t];
#pragma unroll
      for (int s = 0; s < 2; ++s) acc[s * 3 + t] += wy * cx[s];
    }
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const float wx = axn[s] + ax0[s];
#pragma unroll
      for (int t = 0; t < 2; ++t) acc[6 + s * 2 + t] += wx * cy[t];
    }
  } else {
    float az0[3], azn[3];
    wq(m.sz, az0);
    wq(m.nsz, azn);
    float cz[2];
    cz[0] = (-0.f + az0[0]) - azn[0];
    cz[1] = (cz[0] + az0[1]) - azn[1];
    cz[0] *= wsc;
    cz[1] *= wsc;
    float wx0[3], wx1[3], wy0[3], wy1[3];
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      wx0[s] = 0.5f * axn[s] + ax0[s];
      wx1[s] = axn[s] + 0.5f * ax0[s];
      wy0[s] = 0.5f * ayn[s] + ay0[s];
      wy1[s] = ayn[s] + 0.5f * ay0[s];
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const float A0 = az0[r], A1 = azn[r];
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        const float wyv = wy0[t] * A0 + wy1[t] * A1;
#pragma unroll
        for (int s = 0; s < 2; ++s) acc[(s * 3 + t) * 3 + r] += cx[s] * wyv;
      }
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const float wxv = wx0[s] * A0 + wx1[s] * A1;
#pragma unroll
        for (int t = 0; t < 2; ++t) acc[18 + (s * 2 + t) * 3 + r] += cy[t] * wxv;
      }
    }
#pragma unroll
    for (int s = 0; s < 3; ++s) {
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        const float wxy = wx0[s] * ay0[t] + wx1[s] * ayn[t];
#pragma unroll
        for (int r = 0; r < 2; ++r) acc[36 + (s * 3 + t) * 2 + r] += cz[r] * wxy;
      }
    }
  }
}

// The node's register sums into the shared current tile ((lx, ly, lz) =
// local current coordinates of slot 0, node - 2).
template <int NDIM>
__device__ __forceinline__ void flush_stay(float* sJ, int lx, int ly, int lz, const float* acc) {
  using C = CT<NDIM>;
  constexpr int JX = C::JX, JY = C::JY, JV = C::JV;
  if (NDIM == 2) {
#pragma unroll
    for (int s = 0; s < 2; ++s)
#pragma unroll
      for (int t = 0; t < 3; ++t) atomicAdd(&sJ[lx + 1 + s + JX * (ly + 1 + t)], acc[s * 3 + t]);
#pragma unroll
    for (int s = 0; s < 3; ++s)
#pragma unroll
      for (int t = 0; t < 2; ++t) atomicAdd(&sJ[JV + lx + 1 + s + JX * (ly + 1 + t)], acc[6 + s * 2 + t]);
  } else {
    const int b = lx + 1 + JX * (ly + 1 + JY * (lz + 1));
#pragma unroll
    for (int s = 0; s < 2; ++s)
#pragma unroll
      for (int t = 0; t < 3; ++t)
#pragma unroll
        for (int r = 0; r < 3; ++r) atomicAdd(&sJ[b + s + JX * (t + JY * r)], acc[(s * 3 + t) * 3 + r]);
#pragma unroll
    for (int s = 0; s < 3; ++s)
#pragma unroll
      for (int t = 0; t < 2; ++t)
#pragma unroll
        for (int r = 0; r < 3; ++r) atomicAdd(&sJ[JV + b + s + JX * (t + JY * r)], acc[18 + (s * 2 + t) * 3 + r]);
#pragma unroll
    for (int s = 0; s < 3; ++s)
#pragma unroll
      for (int t = 0; t < 3; ++t)
#pragma unroll
        for (int r = 0; r < 2; ++r)
          atomicAdd(&sJ[2 * JV + b + s + JX * (t + JY * r)], acc[36 + (s * 3 + t) * 2 + r]);
  }
}

// Mover queue of a warp: entry e, word j at q[j * QCAP + e].  Word 0 packs
// the tile-local node (bits 0-9) and the node changes + 1 (bits 10-15).
template <int NDIM>
__device__ __forceinline__ void queue_put(float* q, int e, int lc, const Moved& m) {
  constexpr int QC = CT<NDIM>::QCAP;
  q[0 * QC + e] = __int_as_float(lc | ((m.mi + 1) << 10) | ((m.mj + 1) << 12) | ((m.mk + 1) << 14));
  q[1 * QC + e] = m.sx;
  q[2 * QC + e] = m.sy;
  q[3 * QC + e] = m.sz;
  q[4 * QC + e] = m.nsx;
  q[5 * QC + e] = m.nsy;
  q[6 * QC + e] = m.nsz;
  q[7 * QC + e] = m.wght;
}
template <int NDIM>
__device__ __forceinline__ void queue_deposit(float* sJ, const float* q, int e) {
  using C = CT<NDIM>;
  constexpr int QC = C::QCAP;
  const int w0 = __float_as_int(q[e]);
  const int lc = w0 & 1023;
  Moved m;
  m.mi = ((w0 >> 10) & 3) - 1;
  m.mj = ((w0 >> 12) & 3) - 1;
  m.mk = ((w0 >> 14) & 3) - 1;
  m.sx = q[1 * QC + e];
  m.sy = q[2 * QC + e];
  m.sz = q[3 * QC + e];
  m.nsx = q[4 * QC + e];
  m.nsy = q[5 * QC + e];
  m.nsz = q[6 * QC + e];
  m.wght = q[7 * QC + e];
  m.keep = true;
  deposit_window<NDIM>(sJ, lc % C::TX, (lc / C::TX) % C::TY, lc / (C::TX * C::TY), m);
}

}  // namespace

// Particles [beg, end) of tile t (at most LIST_CAP of them).
template <int NDIM>
__device__ __forceinline__ void d32_chunk(const TileArgs32& a, const int t, const int beg, const int end) {
  using C = CT<NDIM>;
  constexpr int TX = C::TX, TY = C::TY, TZ = C::TZ, NCELL = C::NCELL;
  constexpr int FX = C::FX, FY = C::FY, JX = C::JX, JY = C::JY, JV = C::JV;
  constexpr int NF = C::NF, NC = C::NC;
  extern __shared__ __align__(16) float smem[];
  float* sF = smem + C::W_F;
  float* sJ = smem + C::W_J;
  int* sStart = reinterpret_cast<int*>(smem + C::W_START);
  int* sCur = reinterpret_cast<int*>(smem + C::W_CUR);
  int* sList = reinterpret_cast<int*>(smem + C::W_LIST);
  __shared__ int sWarp[NT / 32];
  __shared__ int sHist[C::NSUB];

  const Geo g = a.g;
  const int tx = t % a.t.ntx, ty = (t / a.t.ntx) % a.t.nty, tz = t / (a.t.ntx * a.t.nty);
  const int i0t = 3 + tx * TX, j0t = 3 + ty * TY, k0t = (NDIM == 3) ? 3 + tz * TZ : 1;
  const int nx = g.ix2 - g.ix1 + 1, ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  // 1: stage fields (nodes i0t-1 .. i0t+TX), one x-row of FX nodes per
  // warp and pass (lane = node, the first FX - 32 lanes take the rest), as
  // asynchronous copies that complete while the CTA zeroes its currents and
  // sorts its particles (nodes outside the array are zero-filled)
  __syncthreads();  // a previous chunk of this CTA has finished with shared memory
  {
    constexpr int NROW = NF * FY * C::FZ;
    const int gi0 = i0t - 1 + lane, gi1 = gi0 + 32;
    const bool in0 = gi0 >= 1 && gi0 <= g.n1p, in1 = (lane < FX - 32) && gi1 <= g.n1p;
    for (int row = warp; row < NROW; row += NT / 32) {
      const int c = row / (FY * C::FZ), r = row - c * (FY * C::FZ);
      const int gj = j0t - 1 + r % FY, gk = (NDIM == 3) ? k0t - 1 + r / FY : 1;
      const bool rin = gj >= 1 && gj <= g.n2p && gk >= 1 && gk <= g.n3p;
      const float* src = a.ebf + g.ncell * c + goff(g, gi0, gj, gk);
      cpa4z(&sF[row * FX + lane], (rin && in0) ? src : a.ebf, rin && in0);
      if (lane < FX - 32) cpa4z(&sF[row * FX + 32 + lane], (rin && in1) ? src + 32 : a.ebf, rin && in1);
    }
    cpa_commit();
  }
  for (int e = threadIdx.x; e < NC * JV; e += NT) sJ[e] = 0.f;
  for (int e = threadIdx.x; e < NCELL; e += NT) sCur[e] = 0;
  for (int e = threadIdx.x; e < C::NSUB; e += NT) sHist[e] = 0;
  const int kbase = t * C::NSUB;
  __syncthreads();

  {
    // 2: counting sort of the tile's particles by node; each thread holds
    // its (at most LIST_CAP / NT) record indices and nodes in registers, all
    // loads of a thread in flight together
    // (the slots past the chunk's particles are skipped: nu is the same
    // for the whole CTA)
    constexpr int U = (C::LIST_CAP + NT - 1) / NT;
    const int nu = (end - beg + NT - 1) / NT;
    int pv[U], lv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      pv[u] = -1;
      lv[u] = 0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (u >= nu) break;
      const int q = beg + threadIdx.x + u * NT;
      pv[u] = (q < end) ? __ldg(&a.perm[q]) : -1;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (u >= nu) break;
      lv[u] = (pv[u] >= 0) ? a.p.cell[pv[u]] : 0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (u >= nu) break;
      if (pv[u] < 0) continue;
      int i0, j0, k0;
      cell_split(g, lv[u], i0, j0, k0);
      const unsigned lx = (unsigned)(i0 - i0t), ly = (unsigned)(j0 - j0t), lz = (unsigned)(k0 - k0t);
      if (lx < (unsigned)TX && ly < (unsigned)TY && (NDIM == 2 || lz < (unsigned)TZ)) {
        lv[u] = lx + TX * (ly + TY * lz);
        atomicAdd(&sCur[lv[u]], 1);
      } else {
        raise_err(a.err, AGPU_EBIT_INDEX);  // not binned in this tile: drop it
        a.key[pv[u]] = a.t.nkeys;
        hist_add(a.hist, a.t.nkeys);
        pv[u] = -1;
      }
    }
    __syncthreads();
    {
      // exclusive scan of the NCELL counts, C::NPASS consecutive per thread
      int c[C::NPASS], s = 0;
#pragma unroll
      for (int u = 0; u < C::NPASS; ++u) {
        c[u] = sCur[threadIdx.x * C::NPASS + u];
        s += c[u];
      }
      int incl = s;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += v;
      }
      if (lane == 31) sWarp[warp] = incl;
      __syncthreads();
      int wbase = 0;
#pragma unroll
      for (int w = 0; w < NT / 32; ++w) wbase += (w < warp) ? sWarp[w] : 0;
      int st = wbase + incl - s;
#pragma unroll
      for (int u = 0; u < C::NPASS; ++u) {
        sStart[threadIdx.x * C::NPASS + u] = st;
        sCur[threadIdx.x * C::NPASS + u] = st;
        st += c[u];
      }
      if (threadIdx.x == NT - 1) sStart[NCELL] = st;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (u >= nu) break;
      if (pv[u] >= 0) sList[atomicAdd(&sCur[lv[u]], 1)] = pv[u];
    }
    cpa_wait_all();  // this thread's field copies; the barrier makes all of them visible
    __syncthreads();

    // 3: one node per thread, pass by pass (a warp = one x-row of 32 nodes);
    // the next record of the node is copied into the thread's staging slot
    // while the current one is pushed
    float* qw = smem + C::W_Q + warp * (C::QW * C::QCAP);
    float* stg0 = smem + C::W_REC + threadIdx.x;
    uint64_t* stg_slot0 = reinterpret_cast<uint64_t*>(smem + C::W_SLOT) + threadIdx.x;
    auto fetch = [&](int p, int b) {
      float* stg = stg0 + b * (6 * NT);
      cpa4(stg + 0 * NT, a.p.ox + p);
      cpa4(stg + 1 * NT, a.p.oy + p);
      if (NDIM == 3) cpa4(stg + 2 * NT, a.p.oz + p);
      cpa4(stg + 3 * NT, a.p.px + p);
      cpa4(stg + 4 * NT, a.p.py + p);
      if (NDIM == 3) cpa4(stg + 5 * NT, a.p.pz + p);
      cpa8(stg_slot0 + b * NT, a.p.slot + p);
    };
    int qn = 0;  // entries in this warp's mover queue (warp-uniform)
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll 1
    for (int pass = 0; pass < C::NPASS; ++pass) {
      const int lc = pass * NT + threadIdx.x;
      const int lx = lc % TX, ly = (lc / TX) % TY, lz = lc / (TX * TY);
      const int i0 = i0t + lx, j0 = j0t + ly, k0 = (NDIM == 3) ? k0t + lz : 1;
      const int cs = sStart[lc], nk = sStart[lc + 1] - cs;
      const int nmax = __reduce_max_sync(FULL, nk);
      // a node strictly inside the box keeps every particle that stays on it
      const bool interior = (unsigned)(i0 - 4) < (unsigned)(nx - 1) && (unsigned)(j0 - 4) < (unsigned)(ny - 1) &&
                            (NDIM == 2 || (unsigned)(k0 - 4) < (unsigned)(nz - 1));
      const int nodekey = kbase + (ly + TY * lz) * ((NDIM == 3) ? 8 : 4);
      float acc[C::NACC];
#pragma unroll
      for (int u = 0; u < C::NACC; ++u) acc[u] = 0.f;
      int pnext = (nk > 0) ? sList[cs] : 0;
      if (nk > 0) fetch(pnext, 0);
      cpa_commit();
#pragma unroll 1
      for (int k = 0; k < nmax; ++k) {
        bool mover = false;
        Moved m;
        cpa_wait_all();
        const int p = pnext;
        const float* stg = stg0 + (k & 1) * (6 * NT);
        Rec rec;
        rec.ox = stg[0];
        rec.oy = stg[NT];
        rec.oz = (NDIM == 3) ? stg[2 * NT] : 0.f;
        rec.px = stg[3 * NT];
        rec.py = stg[4 * NT];
        rec.pz = (NDIM == 3) ? stg[5 * NT] : 0.f;
        rec.slot = stg_slot0[(k & 1) * NT];
        if (k + 1 < nk) {
          pnext = sList[cs + k + 1];
          fetch(pnext, (k + 1) & 1);
        }
        cpa_commit();
        if (k < nk) {
          m = push_one<NDIM>(a, sF, sHist, kbase, p, rec, i0, j0, k0, lx, ly, lz, nx, ny, nz, interior, nodekey);
          if (m.keep) {
            if (m.mi == 0 && m.mj == 0 && m.mk == 0)
              accumulate_stay<NDIM>(acc, m);
            else
              mover = true;
          }
        }
        const unsigned mm = __ballot_sync(FULL, mover);
        if (mover) queue_put<NDIM>(qw, qn + __popc(mm & lt), lc, m);
        qn += __popc(mm);
        if (qn >= C::QDRAIN) {
          // rare: hand the node sums over first so that no register sum is
          // live across the full-window deposits
          if (nk > 0) flush_stay<NDIM>(sJ, lx, ly, lz, acc);
#pragma unroll
          for (int u = 0; u < C::NACC; ++u) acc[u] = 0.f;
          const int d = qn < 32 ? qn : 32;
          __syncwarp();
          if (lane < d) queue_deposit<NDIM>(sJ, qw, qn - d + lane);
          qn -= d;
          __syncwarp();
        }
      }
      if (nk > 0) flush_stay<NDIM>(sJ, lx, ly, lz, acc);
    }
    __syncwarp();
    if (lane < qn) queue_deposit<NDIM>(sJ, qw, lane);
  }
  __syncthreads();
  // 4: the tile's histogram counts, then one compensated flush of its
  // currents (nodes i0t-2 ..)
  for (int e = threadIdx.x; e < C::NSUB; e += NT)
    if (sHist[e]) atomicAdd(&a.hist[kbase + e], sHist[e]);
  // x-rows of JX nodes, R per warp and pass (lane = node, the first
  // JX - 32 lanes take the rest): the rows' global adds in flight together,
  // then their TwoSum errors into lo
  {
    constexpr int NROW = NC * JY * C::JZ;
    const int gi0 = i0t - 2 + lane;
    const bool xin0 = gi0 >= 1 && gi0 <= g.n1p, xin1 = (lane < JX - 32) && gi0 + 32 <= g.n1p;
    constexpr int R = 8;  // rows of a warp in flight
    for (int row0 = warp; row0 < NROW; row0 += R * (NT / 32)) {
      float v[2 * R], old[2 * R];
      long long o[R];
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int row = row0 + u * (NT / 32);
        v[2 * u] = v[2 * u + 1] = 0.f;
        o[u] = 0;
        if (row < NROW) {
          const int c = row / (JY * C::JZ), r = row - c * (JY * C::JZ);
          const int gj = j0t - 2 + r % JY, gk = (NDIM == 3) ? k0t - 2 + r / JY : 1;
          const bool rin = gj >= 1 && gj <= g.n2p && gk >= 1 && gk <= g.n3p;
          v[2 * u] = sJ[row * JX + lane];
          v[2 * u + 1] = (lane < JX - 32) ? sJ[row * JX + 32 + lane] : 0.f;
          const bool in0 = rin && xin0, in1 = rin && xin1;
          if ((v[2 * u] != 0.f && !in0) || (v[2 * u + 1] != 0.f && !in1)) {
            raise_err(a.err, AGPU_EBIT_INDEX);
            if (!in0) v[2 * u] = 0.f;
            if (!in1) v[2 * u + 1] = 0.f;
          }
          o[u] = g.ncell * c + goff(g, gi0, gj, gk);
        }
      }
#pragma unroll
      for (int e = 0; e < 2 * R; ++e)
        old[e] = (v[e] != 0.f) ? atomicAdd(&a.jhi[o[e >> 1] + 32 * (e & 1)], v[e]) : 0.f;
#pragma unroll
      for (int e = 0; e < 2 * R; ++e) {
        if (v[e] == 0.f) continue;
        const float sm = __fadd_rn(old[e], v[e]);
        const float bp = __fsub_rn(sm, old[e]);
        const float err = __fadd_rn(__fsub_rn(old[e], __fsub_rn(sm, bp)), __fsub_rn(v[e], bp));
        if (err != 0.f) atomicAdd(&a.jlo[o[e >> 1] + 32 * (e & 1)], err);
      }
    }
  }
}

// Tile t, first chunk of at most LIST_CAP particles; the CTA lists the
// tile's further chunks (a dense tile) as (tile, chunk) pairs for
// k32_tile_more.
template <int NDIM>
__device__ __forceinline__ void d32_tile_first(const TileArgs32& a, const int t) {
  constexpr int CAP = CT<NDIM>::LIST_CAP;
  const int beg = a.tstart[t * a.t.nsub], end = a.tstart[(t + 1) * a.t.nsub];
  if (beg >= end) return;
  const int nch = (end - beg + CAP - 1) / CAP;
  if (nch > 1 && threadIdx.x == 0) {
    const unsigned base = atomicAdd(&a.work_n[0], (unsigned)(nch - 1));
    for (int c = 1; c < nch; ++c) {
      const unsigned e = base + (unsigned)(c - 1);
      if (e < (unsigned)a.work_cap) {
        a.work[2 * e] = t;
        a.work[2 * e + 1] = c;
      } else {
        raise_err(a.err, AGPU_EBIT_CAPACITY);  // cannot happen: the list holds capacity / LIST_CAP chunks
      }
    }
  }
  d32_chunk<NDIM>(a, t, beg, min(end, beg + CAP));
}

// Tile t, all its chunks in turn (the multi-instance kernel, no work list).
template <int NDIM>
__device__ __forceinline__ void d32_tile_all(const TileArgs32& a, const int t) {
  constexpr int CAP = CT<NDIM>::LIST_CAP;
  const int beg = a.tstart[t * a.t.nsub], end = a.tstart[(t + 1) * a.t.nsub];
  for (int c = beg; c < end; c += CAP) d32_chunk<NDIM>(a, t, c, min(end, c + CAP));
}

template <int NDIM>
__global__ void __launch_bounds__(NT, (NDIM == 3) ? 2 : 3) k32_tile(TileArgs32 a) {
  d32_tile_first<NDIM>(a, blockIdx.x);
}

// The listed further chunks of dense tiles, pulled by a fixed grid of CTAs
// from a shared counter (the list is complete: k32_tile has finished).
template <int NDIM>
__global__ void __launch_bounds__(NT, (NDIM == 3) ? 2 : 3) k32_tile_more(TileArgs32 a) {
  constexpr int CAP = CT<NDIM>::LIST_CAP;
  __shared__ unsigned s_item;
  const unsigned total = min(a.work_n[0], (unsigned)a.work_cap);
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(&a.work_n[1], 1u);
    __syncthreads();
    const unsigned item = s_item;
    if (item >= total) return;
    const int t = a.work[2 * item], c = a.work[2 * item + 1];
    const int beg = a.tstart[t * a.t.nsub], end = a.tstart[(t + 1) * a.t.nsub];
    d32_chunk<NDIM>(a, t, beg + c * CAP, min(end, beg + (c + 1) * CAP));
  }
}

// One block per tile of any instance: instance i owns the global tiles
// [tile_off[i], tile_off[i+1]).
template <int NDIM>
__global__ void __launch_bounds__(NT, (NDIM == 3) ? 2 : 3) km32_tile(const MultiInst* __restrict__ d,
                                                                      const int* __restrict__ tile_off, int n) {
  const int b = blockIdx.x;
  int lo = 0, hi = n;  // tile_off[lo] <= b < tile_off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&tile_off[mid]) <= b) lo = mid; else hi = mid;
  }
  // the instance's arguments in shared memory: read from the global
  // descriptor they would be reloaded after every global store (which the
  // compiler cannot prove does not alias them)
  __shared__ TileArgs32 sa;
  if (threadIdx.x == 0) sa = d[lo].ta;
  __syncthreads();
  d32_tile_all<NDIM>(sa, b - __ldg(&tile_off[lo]));
}

size_t tile32_smem(int ndim) { return sizeof(float) * (size_t)((ndim == 3) ? CT<3>::WORDS : CT<2>::WORDS); }

int tile32_list_cap(int ndim) { return (ndim == 3) ? CT<3>::LIST_CAP : CT<2>::LIST_CAP; }

// Returns the kernels launched (the work-list counters are reset here).
int tile_push32(const TileArgs32& a, cudaStream_t st, int sms) {
  if (a.t.ntiles <= 0) return 0;
  const size_t sm = tile32_smem(a.g.ndim);
  if (a.work) cudaMemsetAsync(a.work_n, 0, 2 * sizeof(unsigned int), st);
  if (a.g.ndim == 3) {
    auto k = k32_tile<3>;
    auto k2 = k32_tile_more<3>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<a.t.ntiles, NT, sm, st>>>(a);
    if (a.work) k2<<<2 * sms, NT, sm, st>>>(a);
  } else {
    auto k = k32_tile<2>;
    auto k2 = k32_tile_more<2>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<a.t.ntiles, NT, sm, st>>>(a);
    if (a.work) k2<<<3 * sms, NT, sm, st>>>(a);
  }
  return a.work ? 2 : 1;
}

void multi_tile32(const MultiInst* d, const int* tile_off, const MultiPlan& pl, cudaStream_t st, int* launches) {
  if (pl.total_tiles <= 0) return;
  const size_t sm = tile32_smem(pl.ndim);
  if (pl.ndim == 3) {
    auto k = km32_tile<3>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<pl.total_tiles, NT, sm, st>>>(d, tile_off, pl.n);
  } else {
    auto k = km32_tile<2>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<pl.total_tiles, NT, sm, st>>>(d, tile_off, pl.n);
  }
  *launches += 1;
}

}  // namespace agpu
