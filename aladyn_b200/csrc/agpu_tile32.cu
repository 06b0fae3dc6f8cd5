// agpu_tile32.cu — tiled gather + push + deposit of the FP32 split form.
//
// One CTA per spatial tile of TX x TY x TZ nodes.  The tile's particles are
// the permutation range perm[tstart[t] .. tstart[t+1]) built by the binning
// pass, so every particle's node lies inside the tile.  The CTA
//   1. stages the six field components of the tile plus a one-node guard
//      (the qlh gather stencil) into shared memory,
//   2. zeroes a shared current tile with a two-node guard (the Esirkepov
//      window of a particle that moves at most one node) and finds the
//      tile's largest |charge * weight|,
//   3. gathers, pushes (exact-gamma Boris) and deposits every particle, the
//      deposit going into shared memory as int32 fixed point with integer
//      shared atomics (on sm_100a several times the throughput of FP32
//      shared atomics, and unaffected by lanes that hit the same node); the
//      tile's scale 2^30 / (max|q w| * max(particles, 512)) bounds every
//      node's sum below 2^31 and every single contribution below 2^22 (one
//      particle adds at most 1.69 |q w| to a node), so each contribution is
//      rounded to an integer by one FMA with 1.5 * 2^23 (no conversion
//      instruction), and integer sums make the tile's currents independent
//      of the order,
//   4. flushes the shared currents to the global (hi, lo) pair once, each
//      fixed-point sum converted exactly to FP64 and split into hi + lo,
//      with the TwoSum error of each global add accumulated into lo,
//   5. writes each particle's new tile key and the next histogram.
#include "agpu_bin.cuh"
#include "agpu_common.cuh"
#include "agpu_multi.h"
#include "agpu_tile.h"

namespace agpu {

namespace {

__device__ __forceinline__ void kadd_g(float* hi, float* lo, float v) {
  float old = atomicAdd(hi, v);
  float s = __fadd_rn(old, v);
  float bp = __fsub_rn(s, old);
  float err = __fadd_rn(__fsub_rn(old, __fsub_rn(s, bp)), __fsub_rn(v, bp));
  if (err != 0.f) atomicAdd(lo, err);
}

// Fixed-point contribution x * y, already in units of the tile's scale and
// below 2^22 in magnitude by construction: x * y + 1.5 * 2^23, rounded once,
// lies in [2^23, 2^24) where the float spacing is 1, so its bit pattern minus
// that of 1.5 * 2^23 is x * y rounded to the nearest integer (ties to even).
__device__ __forceinline__ void fx_add(int* a, float x, float y) {
  atomicAdd(a, __float_as_int(__fmaf_rn(x, y, 12582912.f)) - 0x4B400000);
}

__device__ __forceinline__ void wq(float s, float a[3]) {
  float s2 = s * s;
  a[1] = 0.75f - s2;
  a[2] = 0.5f * (0.25f + s2 + s);
  a[0] = 1.f - a[1] - a[2];
}

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

}  // namespace

template <int NDIM, int TX, int TY, int TZ>
__device__ __forceinline__ void d32_tile(const TileArgs32& a, const int t) {
  constexpr int FX = TX + 2, FY = TY + 2, FZ = (NDIM == 3) ? TZ + 2 : 1;
  constexpr int JX = TX + 4, JY = TY + 4, JZ = (NDIM == 3) ? TZ + 4 : 1;
  constexpr int FV = FX * FY * FZ, JV = JX * JY * JZ;
  constexpr int NF = (NDIM == 3) ? 6 : 3, NC = (NDIM == 3) ? 3 : 2;
  extern __shared__ float smem[];
  float* sF = smem;                                  // NF * FV
  int* sJ = reinterpret_cast<int*>(smem + NF * FV);  // NC * JV, fixed point
  __shared__ unsigned int s_wmax;

  const Geo g = a.g;
  const int beg = a.tstart[t * a.t.nsub], end = a.tstart[(t + 1) * a.t.nsub];
  if (beg >= end) return;
  const int tx = t % a.t.ntx, ty = (t / a.t.ntx) % a.t.nty, tz = t / (a.t.ntx * a.t.nty);
  const int i0t = 3 + tx * TX, j0t = 3 + ty * TY, k0t = (NDIM == 3) ? 3 + tz * TZ : 1;

  // 1-2: stage fields (nodes i0t-1 .. i0t+TX), zero currents
  for (int e = threadIdx.x; e < NF * FV; e += blockDim.x) {
    int c = e / FV, r = e - c * FV;
    int lx = r % FX, ly = (r / FX) % FY, lz = r / (FX * FY);
    int gi = i0t - 1 + lx, gj = j0t - 1 + ly, gk = (NDIM == 3) ? k0t - 1 + lz : 1;
    float v = 0.f;
    if (gi >= 1 && gi <= g.n1p && gj >= 1 && gj <= g.n2p && gk >= 1 && gk <= g.n3p)
      v = __ldg(&a.ebf[g.ncell * c + goff(g, gi, gj, gk)]);
    sF[e] = v;
  }
  for (int e = threadIdx.x; e < NC * JV; e += blockDim.x) sJ[e] = 0;
  if (threadIdx.x == 0) s_wmax = 0u;
  __syncthreads();
  {
    // largest |charge * weight| of the tile (non-negative floats order as
    // their bit patterns)
    float wl = 0.f;
    for (int q = beg + threadIdx.x; q < end; q += blockDim.x) {
      const uint64_t sl = a.p.slot[a.perm[q]];
      wl = fmaxf(wl, fabsf((float)slot_charge(sl) * slot_wgh(sl)));
    }
    if (!(wl <= 3.0e38f)) wl = 3.0e38f;  // NaN / inf weights: keep the scale finite
    for (int o = 16; o > 0; o >>= 1) wl = fmaxf(wl, __shfl_xor_sync(0xffffffffu, wl, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&s_wmax, __float_as_uint(wl));
  }
  __syncthreads();
  const float wtile = __uint_as_float(s_wmax) * (float)max(end - beg, 512);
  float fsc = 1073741824.f / wtile;  // 2^30 / (max|q w| * max(particles, 512))
  if (!(fsc < 1.0e30f)) fsc = 1.0e30f;

  const int nx = g.ix2 - g.ix1 + 1, ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  for (int q = beg + threadIdx.x; q < end; q += blockDim.x) {
    const int p = a.perm[q];
    const int c = a.p.cell[p];
    int i0, j0, k0;
    cell_split(g, c, i0, j0, k0);
    float sx = a.p.ox[p], sy = a.p.oy[p], sz = (NDIM == 3) ? a.p.oz[p] : 0.f;
    float pp[3] = {a.p.px[p], a.p.py[p], (NDIM == 3) ? a.p.pz[p] : 0.f};
    const uint64_t sl = a.p.slot[p];
    // local field coordinates of node i0-1 (the first stencil node)
    const int fx = i0 - i0t, fy = j0 - j0t, fz = (NDIM == 3) ? k0 - k0t : 0;
    if ((unsigned)fx >= (unsigned)TX || (unsigned)fy >= (unsigned)TY || (NDIM == 3 && (unsigned)fz >= (unsigned)TZ)) {
      raise_err(a.err, AGPU_EBIT_INDEX);  // not binned in this tile: drop it
      a.key[p] = a.t.nkeys;
      hist_add(a.hist, a.t.nkeys);
      continue;
    }
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
          int o = fx + FX * (fy + j1 + FY * (fz + k1));
          ap[0] += ay1[j1] * az1[k1] * (axh[0] * e1[o] + axh[1] * e1[o + 1]);
        }
#pragma unroll
        for (int j1 = 0; j1 < 2; ++j1) {
          int o = fx + FX * (fy + j1 + FY * (fz + k1));
          float dv = ayh[j1] * az1[k1];
          ap[1] += dv * (ax1[0] * e2[o] + ax1[1] * e2[o + 1] + ax1[2] * e2[o + 2]);
          ap[5] += dv * (axh[0] * b3[o] + axh[1] * b3[o + 1]);
        }
      }
#pragma unroll
      for (int k1 = 0; k1 < 2; ++k1) {
#pragma unroll
        for (int j1 = 0; j1 < 2; ++j1) {
          int o = fx + FX * (fy + j1 + FY * (fz + k1));
          ap[3] += ayh[j1] * azh[k1] * (ax1[0] * b1[o] + ax1[1] * b1[o + 1] + ax1[2] * b1[o + 2]);
        }
#pragma unroll
        for (int j1 = 0; j1 < 3; ++j1) {
          int o = fx + FX * (fy + j1 + FY * (fz + k1));
          float dv = ay1[j1] * azh[k1];
          ap[4] += dv * (axh[0] * b2[o] + axh[1] * b2[o + 1]);
          ap[2] += dv * (ax1[0] * e3[o] + ax1[1] * e3[o + 1] + ax1[2] * e3[o + 2]);
        }
      }
    } else {
      const float* e1 = sF;
      const float* e2 = sF + FV;
      const float* b3 = sF + 2 * FV;
#pragma unroll
      for (int j1 = 0; j1 < 3; ++j1) {
        int o = fx + FX * (fy + j1);
        ap[0] += ay1[j1] * (axh[0] * e1[o] + axh[1] * e1[o + 1]);
      }
#pragma unroll
      for (int j1 = 0; j1 < 2; ++j1) {
        int o = fx + FX * (fy + j1);
        ap[1] += ayh[j1] * (ax1[0] * e2[o] + ax1[1] * e2[o + 1] + ax1[2] * e2[o + 2]);
        ap[5] += ayh[j1] * (axh[0] * b3[o] + axh[1] * b3[o + 1]);
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
    a.p.cell[p] = (int)goff(g, i1n, j1n, k1n);
    a.p.ox[p] = nsx;
    a.p.oy[p] = nsy;
    a.p.px[p] = pn[0];
    a.p.py[p] = pn[1];
    if (NDIM == 3) {
      a.p.oz[p] = nsz;
      a.p.pz[p] = pn[2];
    }
    if (!(pn[0] == pn[0] && pn[1] == pn[1] && pn[2] == pn[2])) raise_err(a.err, AGPU_EBIT_NONFINITE);
    bool keep = inside(i1n, nsx, nx) && inside(j1n, nsy, ny);
    if (NDIM == 3) keep = keep && inside(k1n, nsz, nz);
    int nkey = keep ? tile_key_c<TX, TY, TZ, (NDIM == 3) ? 8 : 4>(a.t, i1n, j1n, (NDIM == 3) ? k1n : 3,
                                                                   offset_octant(nsx, nsy, nsz, NDIM))
                    : a.t.nkeys;
    a.key[p] = nkey;
    hist_add(a.hist, nkey);
    if (!keep) continue;
    // Esirkepov deposit into the shared tile (grid_part_connect.f90:956-1334).
    // Old-plane and new-plane terms are regrouped onto the particle's 5-slot
    // windows (slot 0 = old node - 2): each current component is one dense
    // product over (x0..x1) x (y0..y1) [x (z0..z1)].  Along its own axis a
    // component's running sum ends at sum(S0) - sum(S1) = 0 in the last slot
    // (x1 for Jx, y1 for Jy, z1 for Jz), so that slot is not deposited: 54
    // instead of 81 shared atomics (3D) for a particle that stays in its cell.
    const float wght = qc * slot_wgh(sl);
    const float wsc = wght * fsc;  // charge x weight in fixed-point units
    float ax0[3], ay0[3], axn[3], ayn[3];
    wq(sx, ax0);
    wq(sy, ay0);
    wq(nsx, axn);
    wq(nsy, ayn);
    // local J coordinates of window slot 0 (node i0-2)
    const int lx = i0 - i0t, ly = j0 - j0t;
    int* sJx = sJ;
    int* sJy = sJ + JV;
    // When no lane of the warp changes cell, every window is slots 1..3 and
    // the deposit is a fixed 3 x 3 [x 3] loop without predicates; otherwise
    // each window is compacted to the four slots x0 .. x0+3 that can be
    // non-zero.  Both forms evaluate the same expressions per node.
    const bool stay = (mi == 0) && (mj == 0) && (NDIM == 2 || mk == 0);
    const bool warp_stays = __all_sync(__activemask(), stay);
    if (NDIM == 2) {
      if (warp_stays) {
        float cx[3], cy[3], wxs[3], wys[3];  // index s = window slot s+1
        cx[0] = (-0.f + ax0[0]) - axn[0];
        cy[0] = (-0.f + ay0[0]) - ayn[0];
        cx[1] = (cx[0] + ax0[1]) - axn[1];
        cy[1] = (cy[0] + ay0[1]) - ayn[1];
#pragma unroll
        for (int s = 0; s < 3; ++s) {
          cx[s] *= wsc;
          cy[s] *= wsc;
          wxs[s] = axn[s] + ax0[s];
          wys[s] = ayn[s] + ay0[s];
        }
#pragma unroll
        for (int t = 0; t < 3; ++t) {
#pragma unroll
          for (int s = 0; s < 3; ++s) {
            const int o = lx + 1 + s + JX * (ly + 1 + t);
            if (s < 2) fx_add(&sJx[o], wys[t], cx[s]);
            if (t < 2) fx_add(&sJy[o], wxs[s], cy[t]);
          }
        }
      } else {
        float sxh[5], cx[5], syh[5], cy[5];
        const int ih = mi + 1, jh = mj + 1;
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
            if (s < nxw) fx_add(&sJx[o], wyc[t], cxc[s]);
            if (t < nyw) fx_add(&sJy[o], wxc[s], cyc[t]);
          }
        }
      }
    } else {
      float az0[3], azn[3];
      wq(sz, az0);
      wq(nsz, azn);
      int* sJz = sJ + 2 * JV;
      if (warp_stays) {
        float cx[3], cy[3], cz[3], wx0[3], wx1[3], wy0[3], wy1[3];  // index s = window slot s+1
        cx[0] = (-0.f + ax0[0]) - axn[0];
        cy[0] = (-0.f + ay0[0]) - ayn[0];
        cz[0] = (-0.f + az0[0]) - azn[0];
        cx[1] = (cx[0] + ax0[1]) - axn[1];
        cy[1] = (cy[0] + ay0[1]) - ayn[1];
        cz[1] = (cz[0] + az0[1]) - azn[1];
#pragma unroll
        for (int s = 0; s < 3; ++s) {
          cx[s] *= wsc;
          cy[s] *= wsc;
          wx0[s] = 0.5f * axn[s] + ax0[s];
          wx1[s] = axn[s] + 0.5f * ax0[s];
          wy0[s] = 0.5f * ayn[s] + ay0[s];
          wy1[s] = ayn[s] + 0.5f * ay0[s];
        }
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          const float A0 = az0[r], A1 = azn[r];
          const float czw = wsc * cz[r];
          const int ow = lx + 1 + JX * (ly + 1 + JY * (k0 - k0t + 1 + r));
#pragma unroll
          for (int t = 0; t < 3; ++t) {
            const float wyv = wy0[t] * A0 + wy1[t] * A1;
#pragma unroll
            for (int s = 0; s < 3; ++s) {
              const int o = ow + s + JX * t;
              if (s < 2) fx_add(&sJx[o], cx[s], wyv);
              if (t < 2) fx_add(&sJy[o], cy[t], wx0[s] * A0 + wx1[s] * A1);
              if (r < 2) fx_add(&sJz[o], czw, wx0[s] * ay0[t] + wx1[s] * ayn[t]);
            }
          }
        }
      } else {
        float sxh[5], cx[5], syh[5], cy[5], szh[5], cz[5];
        const int ih = mi + 1, jh = mj + 1, kh = mk + 1;
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
        // index s = window slot x0+s (y0+s)
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
          const int ow = lx + x0 + JX * (ly + y0 + JY * (k0 - k0t + w));
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            if (t > nyw) continue;
            const float wyv = wy0c[t] * A0 + wy1c[t] * A1;
            const float cyv = cyc[t];
#pragma unroll
            for (int s = 0; s < 4; ++s) {
              if (s > nxw) continue;
              const int o = ow + s + JX * t;
              if (s < nxw) fx_add(&sJx[o], cxc[s], wyv);
              if (t < nyw) fx_add(&sJy[o], cyv, wx0c[s] * A0 + wx1c[s] * A1);
              if (w < z1) fx_add(&sJz[o], czw, wx0c[s] * b0c[t] + wx1c[s] * b1c[t]);
            }
          }
        }
      }
    }
  }
  __syncthreads();
  // 4: one compensated flush of the tile's currents (nodes i0t-2 ..)
  const double inv_sc = 1.0 / (double)fsc;
  for (int e = threadIdx.x; e < NC * JV; e += blockDim.x) {
    const int iv = sJ[e];
    if (iv == 0) continue;
    int c = e / JV, rr = e - c * JV;
    int lx = rr % JX, ly = (rr / JX) % JY, lz = rr / (JX * JY);
    int gi = i0t - 2 + lx, gj = j0t - 2 + ly, gk = (NDIM == 3) ? k0t - 2 + lz : 1;
    if (gi < 1 || gi > g.n1p || gj < 1 || gj > g.n2p || gk < 1 || gk > g.n3p) {
      raise_err(a.err, AGPU_EBIT_INDEX);
      continue;
    }
    long long o = g.ncell * c + goff(g, gi, gj, gk);
    const double dv = (double)iv * inv_sc;
    const float vh = (float)dv;
    const float vl = (float)(dv - (double)vh);
    kadd_g(&a.jhi[o], &a.jlo[o], vh);
    if (vl != 0.f) atomicAdd(&a.jlo[o], vl);
  }
}

template <int NDIM, int TX, int TY, int TZ>
__global__ void __launch_bounds__(256, 4) k32_tile(TileArgs32 a) {
  d32_tile<NDIM, TX, TY, TZ>(a, blockIdx.x);
}

// One block per tile of any instance: instance i owns the global tiles
// [tile_off[i], tile_off[i+1]).
template <int NDIM, int TX, int TY, int TZ>
__global__ void __launch_bounds__(256, 4) km32_tile(const MultiInst* __restrict__ d, const int* __restrict__ tile_off,
                                                    int n) {
  const int b = blockIdx.x;
  int lo = 0, hi = n;  // tile_off[lo] <= b < tile_off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&tile_off[mid]) <= b) lo = mid; else hi = mid;
  }
  d32_tile<NDIM, TX, TY, TZ>(d[lo].ta, b - __ldg(&tile_off[lo]));
}

size_t tile32_smem(int ndim, int tx, int ty, int tz) {
  if (ndim == 3) return sizeof(float) * (6 * (tx + 2) * (ty + 2) * (tz + 2) + 3 * (tx + 4) * (ty + 4) * (tz + 4));
  return sizeof(float) * (3 * (tx + 2) * (ty + 2) + 2 * (tx + 4) * (ty + 4));
}

void tile_push32(const TileArgs32& a, cudaStream_t st) {
  if (a.t.ntiles <= 0) return;
  if (a.g.ndim == 3) {
    size_t sm = tile32_smem(3, TILE3_X, TILE3_Y, TILE3_Z);
    auto k = k32_tile<3, TILE3_X, TILE3_Y, TILE3_Z>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<a.t.ntiles, 256, sm, st>>>(a);
  } else {
    size_t sm = tile32_smem(2, TILE2_X, TILE2_Y, 1);
    auto k = k32_tile<2, TILE2_X, TILE2_Y, 1>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<a.t.ntiles, 256, sm, st>>>(a);
  }
}

void multi_tile32(const MultiInst* d, const int* tile_off, const MultiPlan& pl, cudaStream_t st, int* launches) {
  if (pl.total_tiles <= 0) return;
  if (pl.ndim == 3) {
    size_t sm = tile32_smem(3, TILE3_X, TILE3_Y, TILE3_Z);
    auto k = km32_tile<3, TILE3_X, TILE3_Y, TILE3_Z>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<pl.total_tiles, 256, sm, st>>>(d, tile_off, pl.n);
  } else {
    size_t sm = tile32_smem(2, TILE2_X, TILE2_Y, 1);
    auto k = km32_tile<2, TILE2_X, TILE2_Y, 1>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<pl.total_tiles, 256, sm, st>>>(d, tile_off, pl.n);
  }
  *launches += 1;
}

}  // namespace agpu
