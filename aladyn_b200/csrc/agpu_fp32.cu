// agpu_fp32.cu — the FP32 "split" form of the PIC step on sm_100a.
//
// Positions are an int32 node index (the reference's nearest-node index
// int(3 + x_loc + 0.5)) plus an FP32 offset in [-0.5, 0.5), so the window
// shift is an exact integer decrement and long runs lose no resolution;
// fields, momenta, spline weights and currents are FP32.  Currents are
// accumulated as a compensated pair (hi, lo): every atomic add returns the
// old value, the TwoSum rounding error of that add is accumulated into lo.
#include "agpu_common.cuh"
#include "agpu_kernels.h"
#include "agpu_multi.h"
#include "agpu_yee.cuh"
#include "agpu_yee_fused.cuh"

namespace agpu {

void field_bd32(const Dev32& d, cudaStream_t st, int sms) { field_bd_t<float>(d.ebf, d.g, st, sms); }
void jfold32(const Dev32& d, cudaStream_t st, int sms) {
  jfold_t<float>(d.jhi, d.g, st, sms);
  jfold_t<float>(d.jlo, d.g, st, sms);
}
void yee32(const Dev32& d, const YeeC& c, cudaStream_t st, int sms) { yee_t<float>(d.ebf, d.jhi, d.jlo, d.g, c, st, sms); }
void yee32_fused(const float* fin, float* fout, const float* jhi, const float* jlo, const Geo& g, const YeeC& c,
                 cudaStream_t st) {
  yee_fused_t<float>(fin, fout, jhi, jlo, g, c, st);
}

// Compensated accumulation: hi += v with the rounding error of that add
// (Knuth TwoSum on the value the atomic saw) added into lo.
__device__ __forceinline__ void kadd(float* hi, float* lo, float v) {
  float old = atomicAdd(hi, v);
  float s = __fadd_rn(old, v);
  float bp = __fsub_rn(s, old);
  float err = __fadd_rn(__fsub_rn(old, __fsub_rn(s, bp)), __fsub_rn(v, bp));
  if (err != 0.f) atomicAdd(lo, err);
}

// Quadratic (integer node) and linear (half node) weights from the offset.
__device__ __forceinline__ void wq(float s, float a[3]) {
  float s2 = s * s;
  a[1] = 0.75f - s2;
  a[2] = 0.5f * (0.25f + s2 + s);
  a[0] = 1.f - a[1] - a[2];
}

// 1-D Esirkepov DS shape with the new shape shifted by ih in {0,1,2}.
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

// Renormalise an offset that moved by less than one cell.
__device__ __forceinline__ int renorm(float& s) {
  int m = (s >= 0.5f) ? 1 : ((s < -0.5f) ? -1 : 0);
  s = s - (float)m;
  return m;
}
__device__ __forceinline__ bool inside(int node, float o, int n) {
  int m = node - 3;
  return ((m > 0) || (m == 0 && o > 0.f)) && ((m < n) || (m == n && o <= 0.f));
}

template <int NDIM>
__global__ void __launch_bounds__(256) k32_push_dep(PushArgs32 a) {
  const Geo g = a.g;
  const float* __restrict__ ef = a.ebf;
  const int nx = g.ix2 - g.ix1 + 1, ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < a.np; n += (long long)gridDim.x * blockDim.x) {
    int c = a.p.cell[n];
    int i0, j0, k0;
    cell_split(g, c, i0, j0, k0);
    float sx = a.p.ox[n], sy = a.p.oy[n], sz = (NDIM == 3) ? a.p.oz[n] : 0.f;
    float pp[3] = {a.p.px[n], a.p.py[n], (NDIM == 3) ? a.p.pz[n] : 0.f};
    uint64_t sl = a.p.slot[n];
    // bounds: gather touches i0-1..i0+1, deposit ii0-2..ii0+2 (and new node)
    bool bad = (i0 < 3 || i0 > g.n1p - 2 || j0 < 3 || j0 > g.n2p - 2);
    if (NDIM == 3) bad = bad || (k0 < 3 || k0 > g.n3p - 2);
    if (bad) {
      raise_err(a.err, AGPU_EBIT_INDEX);
      atomicAdd(a.removed, 1ull);  // outside the box: the compaction drops it
      continue;
    }
    float ax1[3], ay1[3], az1[3] = {0.f, 1.f, 0.f};
    wq(sx, ax1);
    wq(sy, ay1);
    float axh[2] = {1.f - (sx + 0.5f), sx + 0.5f};
    float ayh[2] = {1.f - (sy + 0.5f), sy + 0.5f};
    float azh[2] = {1.f - (sz + 0.5f), sz + 0.5f};
    if (NDIM == 3) wq(sz, az1);
    const int i = i0 - 1, j = j0 - 1, k = (NDIM == 3) ? k0 - 1 : 1;
    float ap[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (NDIM == 3) {
      const float* e1 = ef;
      const float* e2 = ef + g.ncell;
      const float* e3 = ef + 2 * g.ncell;
      const float* b1 = ef + 3 * g.ncell;
      const float* b2 = ef + 4 * g.ncell;
      const float* b3 = ef + 5 * g.ncell;
#pragma unroll
      for (int k1 = 0; k1 <= 2; ++k1) {
#pragma unroll
        for (int j1 = 0; j1 <= 2; ++j1) {
          long long o = goff(g, i, j + j1, k + k1);
          float dv = ay1[j1] * az1[k1];
          ap[0] += dv * (axh[0] * __ldg(&e1[o]) + axh[1] * __ldg(&e1[o + 1]));
        }
#pragma unroll
        for (int j1 = 0; j1 <= 1; ++j1) {
          long long o = goff(g, i, j + j1, k + k1);
          float dv = ayh[j1] * az1[k1];
          ap[1] += dv * (ax1[0] * __ldg(&e2[o]) + ax1[1] * __ldg(&e2[o + 1]) + ax1[2] * __ldg(&e2[o + 2]));
          ap[5] += dv * (axh[0] * __ldg(&b3[o]) + axh[1] * __ldg(&b3[o + 1]));
        }
      }
#pragma unroll
      for (int k1 = 0; k1 <= 1; ++k1) {
#pragma unroll
        for (int j1 = 0; j1 <= 1; ++j1) {
          long long o = goff(g, i, j + j1, k + k1);
          float dv = ayh[j1] * azh[k1];
          ap[3] += dv * (ax1[0] * __ldg(&b1[o]) + ax1[1] * __ldg(&b1[o + 1]) + ax1[2] * __ldg(&b1[o + 2]));
        }
#pragma unroll
        for (int j1 = 0; j1 <= 2; ++j1) {
          long long o = goff(g, i, j + j1, k + k1);
          float dv = ay1[j1] * azh[k1];
          ap[4] += dv * (axh[0] * __ldg(&b2[o]) + axh[1] * __ldg(&b2[o + 1]));
          ap[2] += dv * (ax1[0] * __ldg(&e3[o]) + ax1[1] * __ldg(&e3[o + 1]) + ax1[2] * __ldg(&e3[o + 2]));
        }
      }
    } else {
      const float* e1 = ef;
      const float* e2 = ef + g.ncell;
      const float* b3 = ef + 2 * g.ncell;
#pragma unroll
      for (int j1 = 0; j1 <= 2; ++j1) {
        long long o = goff(g, i, j + j1, 1);
        ap[0] += ay1[j1] * (axh[0] * __ldg(&e1[o]) + axh[1] * __ldg(&e1[o + 1]));
      }
#pragma unroll
      for (int j1 = 0; j1 <= 1; ++j1) {
        long long o = goff(g, i, j + j1, 1);
        ap[1] += ayh[j1] * (ax1[0] * __ldg(&e2[o]) + ax1[1] * __ldg(&e2[o + 1]) + ax1[2] * __ldg(&e2[o + 2]));
        ap[2] += ayh[j1] * (axh[0] * __ldg(&b3[o]) + axh[1] * __ldg(&b3[o + 1]));
      }
      // 2D TE layout (Ex, Ey, Bz) -> (E, B) vectors with Bz in slot 5
      ap[5] = ap[2];
      ap[2] = 0.f;
    }
    const float q = (float)slot_charge(sl);
    if (a.initial) {
      float alp0 = a.dth * a.lfact * q;
      float gam_inv = rsqrtf(1.f + pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2]);
      float vp[3] = {gam_inv * pp[0], gam_inv * pp[1], gam_inv * pp[2]};
      float e[6];
#pragma unroll
      for (int cc = 0; cc < 6; ++cc) e[cc] = -alp0 * ap[cc];
      pp[0] = pp[0] + e[0] + vp[1] * e[5] - vp[2] * e[4];
      pp[1] = pp[1] + e[1] + vp[2] * e[3] - vp[0] * e[5];
      pp[2] = pp[2] + e[2] + vp[0] * e[4] - vp[1] * e[3];
    }
    // exact-gamma Boris push (boris_push.f90:75-168) in FP32
    float alp = a.dth * a.lfact * q;
    float vp[3] = {pp[0] + alp * ap[0], pp[1] + alp * ap[1], pp[2] + alp * ap[2]};
    float bb[3] = {alp * ap[3], alp * ap[4], alp * ap[5]};
    float b2v = bb[0] * bb[0] + bb[1] * bb[1] + bb[2] * bb[2];
    float bv = bb[0] * vp[0] + bb[1] * vp[1] + bb[2] * vp[2];
    float gam02 = 1.f + vp[0] * vp[0] + vp[1] * vp[1] + vp[2] * vp[2] - b2v;
    float gam2 = 0.5f * (gam02 + sqrtf(gam02 * gam02 + 4.f * (b2v + bv * bv)));
    float gam = sqrtf(gam2);
    float inv = 1.f / (b2v + gam2);
    float pn[3];
    pn[0] = 2.f * (gam2 * vp[0] + bb[0] * bv + gam * (vp[1] * bb[2] - vp[2] * bb[1])) * inv - pp[0];
    pn[1] = 2.f * (gam2 * vp[1] + bb[1] * bv + gam * (vp[2] * bb[0] - vp[0] * bb[2])) * inv - pp[1];
    pn[2] = 2.f * (gam2 * vp[2] + bb[2] * bv + gam * (vp[0] * bb[1] - vp[1] * bb[0])) * inv - pp[2];
    if (NDIM == 2) pn[2] = 0.f;
    float dtg = rsqrtf(1.f + pn[0] * pn[0] + pn[1] * pn[1] + pn[2] * pn[2]);
    float nsx = sx + a.dtx * dtg * pn[0];
    float nsy = sy + a.dty * dtg * pn[1];
    float nsz = sz + ((NDIM == 3) ? a.dtz * dtg * pn[2] : 0.f);
    int i1n = i0 + renorm(nsx);
    int j1n = j0 + renorm(nsy);
    int k1n = k0 + ((NDIM == 3) ? renorm(nsz) : 0);
    a.p.cell[n] = (int)goff(g, i1n, j1n, k1n);
    a.p.ox[n] = nsx;
    a.p.oy[n] = nsy;
    a.p.px[n] = pn[0];
    a.p.py[n] = pn[1];
    if (NDIM == 3) {
      a.p.oz[n] = nsz;
      a.p.pz[n] = pn[2];
    }
    if (!(pn[0] == pn[0] && pn[1] == pn[1] && pn[2] == pn[2])) raise_err(a.err, AGPU_EBIT_NONFINITE);
    bool keep = inside(i1n, nsx, nx) && inside(j1n, nsy, ny);
    if (NDIM == 3) keep = keep && inside(k1n, nsz, nz);
    unsigned int leave = __ballot_sync(__activemask(), !keep);
    if (!keep) {
      if ((threadIdx.x & 31) == (__ffs(leave) - 1)) atomicAdd(a.removed, (unsigned long long)__popc(leave));
      continue;
    }
    // Esirkepov deposit (grid_part_connect.f90:956-1334) from the split
    // positions: old node i0 offset sx, new node i1n offset nsx.
    const float wght = q * slot_wgh(sl);
    float ax0[3], ay0[3], axn[3], ayn[3];
    wq(sx, ax0);
    wq(sy, ay0);
    wq(nsx, axn);
    wq(nsy, ayn);
    float sxh[5], cx[5], syh[5], cy[5];
    int ih = i1n - i0 + 1, jh = j1n - j0 + 1;  // in {0,1,2}: renorm moves at most one node
    esirk1(ax0, axn, ih, sxh, cx);
    esirk1(ay0, ayn, jh, syh, cy);
    // the reference loops only over x0..x1 = min(ih,1)..max(ih+2,3)
    const int x0 = ih < 1 ? ih : 1, x1 = (ih + 2) > 3 ? ih + 2 : 3;
    const int y0 = jh < 1 ? jh : 1, y1 = (jh + 2) > 3 ? jh + 2 : 3;
#pragma unroll
    for (int qq = 0; qq < 5; ++qq) {
      cx[qq] = (qq < x0 || qq > x1) ? 0.f : cx[qq] * wght;
      cy[qq] = (qq < y0 || qq > y1) ? 0.f : cy[qq] * wght;
    }
    const int ib = i0 - 2, jb = j0 - 2;  // J index of window slot 0
    float* jxh = a.jhi;
    float* jxl = a.jlo;
    float* jyh = a.jhi + g.ncell;
    float* jyl = a.jlo + g.ncell;
    if (NDIM == 2) {
      float wxs[5], wys[5];
#pragma unroll
      for (int qq = 0; qq < 5; ++qq) {
        wxs[qq] = sxh[qq] + ((qq >= 1 && qq <= 3) ? ax0[qq - 1] : 0.f);
        wys[qq] = syh[qq] + ((qq >= 1 && qq <= 3) ? ay0[qq - 1] : 0.f);
      }
#pragma unroll
      for (int j1 = 0; j1 < 5; ++j1) {
#pragma unroll
        for (int i1 = 0; i1 < 5; ++i1) {
          long long o = goff(g, ib + i1, jb + j1, 1);
          float vx = wys[j1] * cx[i1];
          float vy = wxs[i1] * cy[j1];
          if (vx != 0.f) kadd(&jxh[o], &jxl[o], vx);
          if (vy != 0.f) kadd(&jyh[o], &jyl[o], vy);
        }
      }
    } else {
      float az0[3], azn[3], szh[5], cz[5];
      wq(sz, az0);
      wq(nsz, azn);
      int kh = k1n - k0 + 1;
      esirk1(az0, azn, kh, szh, cz);
      const int z0 = kh < 1 ? kh : 1, z1 = (kh + 2) > 3 ? kh + 2 : 3;
#pragma unroll
      for (int qq = 0; qq < 5; ++qq) cz[qq] = (qq < z0 || qq > z1) ? 0.f : cz[qq] * wght;
      // 3-point shapes on the old / new planes, 5-wide shifted sums
      float wx0[5], wx1[5], wy0[5], wy1[5];
#pragma unroll
      for (int qq = 0; qq < 5; ++qq) {
        float a0x = (qq >= 1 && qq <= 3) ? ax0[qq - 1] : 0.f;
        float a0y = (qq >= 1 && qq <= 3) ? ay0[qq - 1] : 0.f;
        wx0[qq] = 0.5f * sxh[qq] + a0x;  // axh0
        wx1[qq] = sxh[qq] + 0.5f * a0x;  // axh1
        wy0[qq] = 0.5f * syh[qq] + a0y;  // ayh0
        wy1[qq] = syh[qq] + 0.5f * a0y;  // ayh1
      }
      const int kb0 = k0 - 1, kb1 = k1n - 1, jb0 = j0 - 1, jb1 = j1n - 1;
      float* jzh = a.jhi + 2 * g.ncell;
      float* jzl = a.jlo + 2 * g.ncell;
#pragma unroll
      for (int k1 = 0; k1 < 3; ++k1) {
#pragma unroll
        for (int j1 = 0; j1 < 5; ++j1) {
          float d0 = wy0[j1] * az0[k1], d1 = wy1[j1] * azn[k1];
          float e0 = cy[j1] * az0[k1], e1 = cy[j1] * azn[k1];
#pragma unroll
          for (int i1 = 0; i1 < 5; ++i1) {
            long long o0 = goff(g, ib + i1, jb + j1, kb0 + k1);
            long long o1 = goff(g, ib + i1, jb + j1, kb1 + k1);
            float v;
            v = d0 * cx[i1];
            if (v != 0.f) kadd(&jxh[o0], &jxl[o0], v);
            v = d1 * cx[i1];
            if (v != 0.f) kadd(&jxh[o1], &jxl[o1], v);
            v = wx0[i1] * e0;
            if (v != 0.f) kadd(&jyh[o0], &jyl[o0], v);
            v = wx1[i1] * e1;
            if (v != 0.f) kadd(&jyh[o1], &jyl[o1], v);
          }
        }
      }
      const int kb = k0 - 2;
#pragma unroll
      for (int k1 = 0; k1 < 5; ++k1) {
#pragma unroll
        for (int j1 = 0; j1 < 3; ++j1) {
          float d0 = ay0[j1] * cz[k1], d1 = ayn[j1] * cz[k1];
#pragma unroll
          for (int i1 = 0; i1 < 5; ++i1) {
            long long o0 = goff(g, ib + i1, jb0 + j1, kb + k1);
            long long o1 = goff(g, ib + i1, jb1 + j1, kb + k1);
            float v;
            v = wx0[i1] * d0;
            if (v != 0.f) kadd(&jzh[o0], &jzl[o0], v);
            v = wx1[i1] * d1;
            if (v != 0.f) kadd(&jzh[o1], &jzl[o1], v);
          }
        }
      }
    }
  }
}

void push_deposit32(const PushArgs32& a, cudaStream_t st, int sms) {
  if (a.np <= 0) return;
  int grid = grid_for(a.np, 256, sms, 8);
  if (a.g.ndim == 3)
    k32_push_dep<3><<<grid, 256, 0, st>>>(a);
  else
    k32_push_dep<2><<<grid, 256, 0, st>>>(a);
}

}  // namespace agpu

namespace agpu {

// ============================================================================
// A15/A16 in the split form: |E|^2 on each ion with the qqh shapes
// (set_ion_efield, grid_part_connect.f90:288-410) from the node + offset,
// then the one-level draw of part_ionize (ionize.f90:390-450) against the
// FP64 table.  Node index of the integer-node shape: i0 (offset s); of the
// half-node shape: int(i0 + s) = i0 (s >= 0) or i0 - 1, offset s -/+ 0.5.
// ============================================================================
__global__ void k32_ion_efield(IonArgs32 a) {
  const Geo g = a.g;
  const float* E1 = a.ebf;
  const float* E2 = a.ebf + g.ncell;
  const float* E3 = a.ebf + 2 * g.ncell;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < a.np; n += (long long)gridDim.x * blockDim.x) {
    int c = a.cell[n];
    int i0, j0, k0;
    cell_split(g, c, i0, j0, k0);
    float sv[3] = {a.ox[n], a.oy[n], (g.ndim == 3) ? a.oz[n] : 0.f};
    int nd[3] = {i0, j0, k0};
    float w1[3][3], wh[3][3];
    int ib[3], ih[3];
    for (int d = 0; d < 3; ++d) {
      float s = sv[d], s2 = s * s;
      w1[d][1] = 0.75f - s2;
      w1[d][2] = 0.5f * (0.25f + s2 + s);
      w1[d][0] = 1.f - w1[d][1] - w1[d][2];
      ib[d] = nd[d] - 1;
      int hn = (s >= 0.f) ? nd[d] : nd[d] - 1;
      float sh = (s >= 0.f) ? s - 0.5f : s + 0.5f;
      float h2 = sh * sh;
      wh[d][1] = 0.75f - h2;
      wh[d][2] = 0.5f * (0.25f + h2 + sh);
      wh[d][0] = 1.f - wh[d][1] - wh[d][2];
      ih[d] = hn - 1;
    }
    bool bad = ib[0] < 1 || ib[0] > g.n1p - 2 || ih[0] < 1 || ih[0] > g.n1p - 2 || ib[1] < 1 || ib[1] > g.n2p - 2 ||
               ih[1] < 1 || ih[1] > g.n2p - 2;
    if (g.ndim == 3) bad = bad || ib[2] < 1 || ib[2] > g.n3p - 2 || ih[2] < 1 || ih[2] > g.n3p - 2;
    if (bad) {
      raise_err(a.err, AGPU_EBIT_INDEX);
      a.ef2[n] = 0.0;
      continue;
    }
    float ef = 0.f;
    if (g.ndim == 2) {
      for (int jp = 0; jp < 3; ++jp)
        for (int ip = 0; ip < 3; ++ip) {
          float e = E1[goff(g, ih[0] + ip, ib[1] + jp, 1)];
          ef += wh[0][ip] * w1[1][jp] * e * e;
          float f = E2[goff(g, ib[0] + ip, ih[1] + jp, 1)];
          ef += w1[0][ip] * wh[1][jp] * f * f;
        }
    } else {
      for (int kp = 0; kp < 3; ++kp)
        for (int jp = 0; jp < 3; ++jp)
          for (int ip = 0; ip < 3; ++ip) {
            float e = E1[goff(g, ih[0] + ip, ib[1] + jp, ib[2] + kp)];
            ef += wh[0][ip] * w1[1][jp] * w1[2][kp] * e * e;
            float f = E2[goff(g, ib[0] + ip, ih[1] + jp, ib[2] + kp)];
            ef += w1[0][ip] * wh[1][jp] * w1[2][kp] * f * f;
            float h = E3[goff(g, ib[0] + ip, ib[1] + jp, ih[2] + kp)];
            ef += w1[0][ip] * w1[1][jp] * wh[2][kp] * h * h;
          }
    }
    a.ef2[n] = (double)ef;
  }
}

__global__ void k32_ionize(IonArgs32 a) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < a.np; n += (long long)gridDim.x * blockDim.x) {
    double ef2 = a.ef2[n];
    int nk = 0;
    if (ef2 > 0.) nk = (int)llround(a.de_inv * sqrt(ef2));
    if (nk > a.n_ge + 1) {
      raise_err(a.err, AGPU_EBIT_IONZ_INDEX);
      nk = a.n_ge + 1;
    }
    uint64_t sl = a.slot[n];
    int z0 = slot_charge(sl);
    double pr = ionz_draw(a.seed, n, a.iter, a.ic);
    double thr = (z0 >= 0 && z0 <= a.zmax) ? a.wtab[(long long)nk + (long long)(a.n_ge + 2) * z0] : 0.0;
    int fl = 0;
    if (pr < thr) {
      a.slot[n] = make_slot(z0 + 1, slot_part_ind(sl), slot_wgh(sl));
      fl = 1;
    }
    a.flag[n] = fl;
  }
}


// ---- multi-instance field phases (one row of blocks per instance) ---------
namespace {

__global__ void km_pre(const MultiInst* __restrict__ d) {
  const MultiInst& m = d[blockIdx.y];
  const Geo g = m.ta.g;
  const long long bid_ = blockIdx.x, nb_ = gridDim.x;
  const long long nj = g.ncell * g.nc;
  GRID_STRIDE(q, nj) {
    m.ta.jhi[q] = 0.f;
    m.ta.jlo[q] = 0.f;
  }
  const int nt = m.ta.t.nkeys;
  GRID_STRIDE(b, (long long)nt + 1) {
    m.cursor[b] = 0;
    if (b == nt) {
      const int alive = m.ta.tstart[nt];
      m.ta.hist[b] = (int)(m.np - alive);  // the records already dead
      *m.pushed += (unsigned long long)alive;
      *m.removed = 0ull;
      *m.fmax = 0.0;
    } else {
      m.ta.hist[b] = 0;
    }
  }
  d_field_bd_x<float>(m.ebf, g, g.nf, bid_, nb_);
}
__global__ void km_bd_y(const MultiInst* __restrict__ d) {
  const MultiInst& m = d[blockIdx.y];
  d_field_bd_y<float>(m.ebf, m.ta.g, m.ta.g.nf, blockIdx.x, gridDim.x);
}
__global__ void km_bd_z(const MultiInst* __restrict__ d) {
  const MultiInst& m = d[blockIdx.y];
  d_field_bd_z<float>(m.ebf, m.ta.g, m.ta.g.nf, blockIdx.x, gridDim.x);
}
__global__ void km_fold_x(const MultiInst* __restrict__ d) {
  const MultiInst& m = d[blockIdx.y];
  d_jfold_x<float>(m.ta.jhi, m.ta.g, blockIdx.x, gridDim.x);
  d_jfold_x<float>(m.ta.jlo, m.ta.g, blockIdx.x, gridDim.x);
}
__global__ void km_fold_y(const MultiInst* __restrict__ d) {
  const MultiInst& m = d[blockIdx.y];
  d_jfold_y<float>(m.ta.jhi, m.ta.g, blockIdx.x, gridDim.x);
  d_jfold_y<float>(m.ta.jlo, m.ta.g, blockIdx.x, gridDim.x);
}
__global__ void km_fold_z(const MultiInst* __restrict__ d) {
  const MultiInst& m = d[blockIdx.y];
  d_jfold_z<float>(m.ta.jhi, m.ta.g, blockIdx.x, gridDim.x);
  d_jfold_z<float>(m.ta.jlo, m.ta.g, blockIdx.x, gridDim.x);
}
__global__ void km_ef_bds(const MultiInst* __restrict__ d, int full_dt) {
  const MultiInst& m = d[blockIdx.y];
  d_ef_bds<float>(m.ebf, m.ta.g, m.yc, full_dt ? m.yc.dt : 0.0, blockIdx.x, gridDim.x);
}
__global__ void km_bf_bds(const MultiInst* __restrict__ d) {
  const MultiInst& m = d[blockIdx.y];
  d_bf_bds<float>(m.ebf, m.ta.g, m.yc, m.yc.dt, blockIdx.x, gridDim.x);
}
template <int NDIM>
__global__ void __launch_bounds__(256) km_rote(const MultiInst* __restrict__ d) {
  const MultiInst& m = d[blockIdx.y];
  d_rote<float, NDIM>(m.ebf, m.ta.g, m.yc, 0.5 * m.yc.dt, blockIdx.x, gridDim.x);
}
template <int NDIM>
__global__ void __launch_bounds__(256) km_rotb_j(const MultiInst* __restrict__ d) {
  const MultiInst& m = d[blockIdx.y];
  d_rotb_j<float, NDIM>(m.ebf, m.ta.jhi, m.ta.jlo, m.ta.g, m.yc, m.yc.dt, blockIdx.x, gridDim.x);
}

}  // namespace

void multi_pre32(const MultiInst* d, const MultiPlan& pl, cudaStream_t st, int* launches) {
  km_pre<<<dim3(pl.gx_cells, pl.n), 256, 0, st>>>(d);
  *launches += 1;
}
void multi_field_bd32(const MultiInst* d, const MultiPlan& pl, cudaStream_t st, int* launches) {
  km_bd_y<<<dim3(pl.gx_faces, pl.n), 256, 0, st>>>(d);
  *launches += 1;
  if (pl.ndim == 3) {
    km_bd_z<<<dim3(pl.gx_faces, pl.n), 256, 0, st>>>(d);
    *launches += 1;
  }
}
// the order of yee_t (curr_and_fields_util.f90:176-260): ef_bds(0), rote(dt/2),
// bf_bds(dt), rotb + current(dt), ef_bds(dt), rote(dt/2)
void multi_fields32(const MultiInst* d, const MultiPlan& pl, cudaStream_t st, int* launches) {
  km_fold_x<<<dim3(pl.gx_faces, pl.n), 256, 0, st>>>(d);
  km_fold_y<<<dim3(pl.gx_faces, pl.n), 256, 0, st>>>(d);
  *launches += 2;
  if (pl.ndim == 3) {
    km_fold_z<<<dim3(pl.gx_faces, pl.n), 256, 0, st>>>(d);
    *launches += 1;
  }
  const dim3 gf(pl.gx_faces, pl.n), gc(pl.gx_cells, pl.n);
  km_ef_bds<<<gf, 256, 0, st>>>(d, 0);
  if (pl.ndim == 3) km_rote<3><<<gc, 256, 0, st>>>(d); else km_rote<2><<<gc, 256, 0, st>>>(d);
  km_bf_bds<<<gf, 256, 0, st>>>(d);
  if (pl.ndim == 3) km_rotb_j<3><<<gc, 256, 0, st>>>(d); else km_rotb_j<2><<<gc, 256, 0, st>>>(d);
  km_ef_bds<<<gf, 256, 0, st>>>(d, 1);
  if (pl.ndim == 3) km_rote<3><<<gc, 256, 0, st>>>(d); else km_rote<2><<<gc, 256, 0, st>>>(d);
  *launches += 6;
}

}  // namespace agpu
