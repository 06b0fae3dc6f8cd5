// agpu_fp64_dep.cuh — FP64 shape functions and the Esirkepov deposit of one
// particle move, shared by the standard FP64 step (agpu_fp64.cu) and the
// envelope step (agpu_env.cu).  Include only from units compiled with
// -fmad=false: the arithmetic keeps the reference's statement order.
#pragma once
#include "agpu_common.cuh"

namespace agpu {

// ============================================================================
// Shapes (src/particles/grid_part_lib.f90)
// ============================================================================
// qlh per dimension (110-143, 212-259): quadratic on integer nodes, linear on
// half nodes, index shifted by -1.
__device__ __forceinline__ int qlh64(double xp, double ax[3], double axh[2]) {
  double xx = 3.0 + xp;
  int i = (int)(xx + 0.5);
  double sx = xx - (double)i;
  double sx2 = sx * sx;
  ax[1] = 0.75 - sx2;
  ax[2] = 0.5 * (0.25 + sx2 + sx);
  ax[0] = 1. - ax[1] - ax[2];
  axh[1] = sx + 0.5;
  axh[0] = 1. - axh[1];
  return i - 1;
}
// qden per dimension (337-358, 388-417): no shift.
__device__ __forceinline__ int qden64(double xp, double ax[3]) {
  double xx = 3.0 + xp;
  int i = (int)(xx + 0.5);
  double sx = xx - (double)i;
  double sx2 = sx * sx;
  ax[1] = 0.75 - sx2;
  ax[2] = 0.5 * (0.25 + sx2 + sx);
  ax[0] = 1. - ax[1] - ax[2];
  return i;
}
// qqh per dimension (170-210, 261-320).
__device__ __forceinline__ void qqh64(double xp, double ax[3], double axh[3], int* ix, int* ihx) {
  double xx = 3.0 + xp;
  int i = (int)(xx + 0.5);
  double sx = xx - (double)i;
  double sx2 = sx * sx;
  ax[1] = 0.75 - sx2;
  ax[2] = 0.5 * (0.25 + sx2 + sx);
  ax[0] = 1. - ax[1] - ax[2];
  int ih = (int)(xx);
  sx = xx - (double)ih - 0.5;
  sx2 = sx * sx;
  axh[1] = 0.75 - sx2;
  axh[2] = 0.5 * (0.25 + sx2 + sx);
  axh[0] = 1. - axh[1] - axh[2];
  *ix = i - 1;
  *ihx = ih - 1;
}

// ============================================================================
// Esirkepov deposit of one move (grid_part_connect.f90:956-1334) with FP64
// atomics (or plain adds when the caller serialises the particles).
// ============================================================================
template <bool SERIAL>
__device__ __forceinline__ void jadd(double* p, double v) {
  if (SERIAL)
    *p = *p + v;
  else
    atomicAdd(p, v);
}

// 1-D Esirkepov "DS" shape: axh[0..4] holds the new shape shifted by ih,
// curr[0..4] the cumulative differences (grid_part_connect.f90:1020-1030).
__device__ __forceinline__ void esirk_1d(const double a0[3], const double a1[3], int ih, double axh[5], double curr[5]) {
#pragma unroll
  for (int q = 0; q < 5; ++q) axh[q] = 0.;
  // ih in {0,1,2}: branch-free placement into registers
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    int m = q - ih;
    axh[q] = (m == 0) ? a1[0] : (m == 1) ? a1[1] : (m == 2) ? a1[2] : 0.;
  }
  curr[0] = -axh[0];
  curr[1] = curr[0] + a0[0] - axh[1];
  curr[2] = curr[1] + a0[1] - axh[2];
  curr[3] = curr[2] + a0[2] - axh[3];
  curr[4] = curr[3] - axh[4];
}

template <bool SERIAL>
__device__ __forceinline__ bool esirkepov2d(const Geo& g, double* jc, double xn, double yn, double xo, double yo,
                                            float wght) {
  double ax0[3], ay0[3], ax1[3], ay1[3], axh[5], ayh[5], currx[5], curry[5];
  int ii0 = qden64(xo, ax0);
  int jj0 = qden64(yo, ay0);
  int i = qden64(xn, ax1);
  int j = qden64(yn, ay1);
  int ih = i - ii0 + 1;
  // a move of more than one cell (dt beyond the CFL limit) has no slot
  if ((unsigned)ih > 2u || (unsigned)(j - jj0 + 1) > 2u) return false;
  esirk_1d(ax0, ax1, ih, axh, currx);
  axh[1] = axh[1] + ax0[0];
  axh[2] = axh[2] + ax0[1];
  axh[3] = axh[3] + ax0[2];
  double w = (double)wght;
#pragma unroll
  for (int q = 0; q < 5; ++q) currx[q] = w * currx[q];
  int x0 = ih < 1 ? ih : 1;
  int x1 = (ih + 2) > 3 ? ih + 2 : 3;
  int jh = j - jj0 + 1;
  esirk_1d(ay0, ay1, jh, ayh, curry);
#pragma unroll
  for (int q = 0; q < 5; ++q) curry[q] = w * curry[q];
  ayh[1] = ayh[1] + ay0[0];
  ayh[2] = ayh[2] + ay0[1];
  ayh[3] = ayh[3] + ay0[2];
  int y0 = jh < 1 ? jh : 1;
  int y1 = (jh + 2) > 3 ? jh + 2 : 3;
  jj0 = jj0 - 1;
  jh = jj0 - 1;
  ii0 = ii0 - 1;
  ih = ii0 - 1;
  double* jx = jc;
  double* jy = jc + g.ncell;
  for (int j1 = y0; j1 <= y1; ++j1) {
    int j2 = jh + j1;
    for (int i1 = x0; i1 <= x1; ++i1) jadd<SERIAL>(&jx[goff(g, ih + i1, j2, 1)], ayh[j1] * currx[i1]);
  }
  for (int j1 = y0; j1 <= y1; ++j1) {
    int j2 = jh + j1;
    for (int i1 = x0; i1 <= x1; ++i1) jadd<SERIAL>(&jy[goff(g, ih + i1, j2, 1)], axh[i1] * curry[j1]);
  }
  return true;
}

template <bool SERIAL>
__device__ __forceinline__ bool esirkepov3d(const Geo& g, double* jc, const double xn[3], const double xo[3],
                                            float wght) {
  double ax0[3], ay0[3], az0[3], ax1[3], ay1[3], az1[3];
  double axh[5], ayh[5], azh[5], axh0[5], axh1[5], ayh0[5], ayh1[5];
  double currx[5], curry[5], currz[5];
  int ii0 = qden64(xo[0], ax0), jj0 = qden64(xo[1], ay0), kk0 = qden64(xo[2], az0);
  int i = qden64(xn[0], ax1), j = qden64(xn[1], ay1), k = qden64(xn[2], az1);
  if ((unsigned)(i - ii0 + 1) > 2u || (unsigned)(j - jj0 + 1) > 2u || (unsigned)(k - kk0 + 1) > 2u) return false;
  double w = (double)wght;

  int ih = i - ii0 + 1;
  esirk_1d(ax0, ax1, ih, axh, currx);
#pragma unroll
  for (int q = 0; q < 5; ++q) currx[q] = w * currx[q];
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    axh0[q] = 0.5 * axh[q];
    axh1[q] = axh[q];
  }
#pragma unroll
  for (int i1 = 1; i1 <= 3; ++i1) {
    axh0[i1] = axh0[i1] + ax0[i1 - 1];
    axh1[i1] = axh1[i1] + 0.5 * ax0[i1 - 1];
  }
  int x0 = ih < 1 ? ih : 1;
  int x1 = (ih + 2) > 3 ? ih + 2 : 3;
  i = i - 1;
  ii0 = ii0 - 1;

  int jh = j - jj0 + 1;
  esirk_1d(ay0, ay1, jh, ayh, curry);
#pragma unroll
  for (int q = 0; q < 5; ++q) curry[q] = w * curry[q];
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    ayh0[q] = 0.5 * ayh[q];
    ayh1[q] = ayh[q];
  }
#pragma unroll
  for (int i1 = 1; i1 <= 3; ++i1) {
    ayh0[i1] = ayh0[i1] + ay0[i1 - 1];
    ayh1[i1] = ayh1[i1] + 0.5 * ay0[i1 - 1];
  }
  int y0 = jh < 1 ? jh : 1;
  int y1 = (jh + 2) > 3 ? jh + 2 : 3;
  jj0 = jj0 - 1;
  j = j - 1;

  int kh = k - kk0 + 1;
  esirk_1d(az0, az1, kh, azh, currz);
#pragma unroll
  for (int q = 0; q < 5; ++q) currz[q] = w * currz[q];
  kk0 = kk0 - 1;
  k = k - 1;
  int z0 = kh < 1 ? kh : 1;
  int z1 = (kh + 2) > 3 ? kh + 2 : 3;

  double* jx = jc;
  double* jy = jc + g.ncell;
  double* jz = jc + 2 * g.ncell;
  jh = jj0 - 1;
  ih = ii0 - 1;
  for (int k1 = 0; k1 <= 2; ++k1)
    for (int j1 = y0; j1 <= y1; ++j1) {
      int j2 = jh + j1;
      double dvol = ayh0[j1] * az0[k1];
      double dvolh = ayh1[j1] * az1[k1];
      for (int i1 = x0; i1 <= x1; ++i1) {
        int i2 = ih + i1;
        jadd<SERIAL>(&jx[goff(g, i2, j2, kk0 + k1)], dvol * currx[i1]);
        jadd<SERIAL>(&jx[goff(g, i2, j2, k + k1)], dvolh * currx[i1]);
      }
    }
  for (int k1 = 0; k1 <= 2; ++k1)
    for (int j1 = y0; j1 <= y1; ++j1) {
      int j2 = jh + j1;
      double dvol = curry[j1] * az0[k1];
      double dvolh = curry[j1] * az1[k1];
      for (int i1 = x0; i1 <= x1; ++i1) {
        int i2 = ih + i1;
        jadd<SERIAL>(&jy[goff(g, i2, j2, kk0 + k1)], axh0[i1] * dvol);
        jadd<SERIAL>(&jy[goff(g, i2, j2, k + k1)], axh1[i1] * dvolh);
      }
    }
  kh = kk0 - 1;
  for (int k1 = z0; k1 <= z1; ++k1) {
    int k2 = kh + k1;
    for (int j1 = 0; j1 <= 2; ++j1) {
      double dvol = ay0[j1] * currz[k1];
      double dvolh = ay1[j1] * currz[k1];
      for (int i1 = x0; i1 <= x1; ++i1) {
        int i2 = ih + i1;
        jadd<SERIAL>(&jz[goff(g, i2, jj0 + j1, k2)], axh0[i1] * dvol);
        jadd<SERIAL>(&jz[goff(g, i2, j + j1, k2)], axh1[i1] * dvolh);
      }
    }
  }
  return true;
}

// ============================================================================
// iform = 2: the non-conserving deposit ncdef_2d_curr / ncdef_3d_curr
// (grid_part_connect.f90:1338-1512): half the particle's q w dt v on the qlh
// shapes at the old and at the new position (xn, xo local).  q w dt / gamma
// as the reference forms it from the push's dt / gamma (ebfp(ch), kept when
// iform = 2); p the momenta at t^{n+1/2}.
// ============================================================================
template <bool SERIAL>
__device__ __forceinline__ void ncdef3d(const Geo& g, double* jc, const double xn[3], const double xo[3],
                                        const double p[3], float wght, double dtg) {
  double ax0[3], ay0[3], az0[3], axh0[2], ayh0[2], azh0[2];
  double ax1[3], ay1[3], az1[3], axh1[2], ayh1[2], azh1[2];
  const double gam_inv = (double)wght * dtg;
  double vp[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) vp[c] = 0.5 * gam_inv * p[c];
  const int ii0 = qlh64(xo[0], ax0, axh0), jj0 = qlh64(xo[1], ay0, ayh0), kk0 = qlh64(xo[2], az0, azh0);
  const int i = qlh64(xn[0], ax1, axh1), j = qlh64(xn[1], ay1, ayh1), k = qlh64(xn[2], az1, azh1);
  const int ih0 = ii0, jh0 = jj0, kh0 = kk0, ih = i, jh = j, kh = k;
  double* jx = jc;
  double* jy = jc + g.ncell;
  double* jz = jc + 2 * g.ncell;
  for (int k1 = 0; k1 <= 2; ++k1) {
    for (int j1 = 0; j1 <= 2; ++j1) {
      const double dvol = vp[0] * ay1[j1] * az1[k1];
      for (int i1 = 0; i1 <= 1; ++i1) jadd<SERIAL>(&jx[goff(g, ih + i1, j + j1, k + k1)], dvol * axh1[i1]);
    }
    for (int j1 = 0; j1 <= 2; ++j1) {
      const double dvol = vp[0] * ay0[j1] * az0[k1];
      for (int i1 = 0; i1 <= 1; ++i1) jadd<SERIAL>(&jx[goff(g, ih0 + i1, jj0 + j1, kk0 + k1)], dvol * axh0[i1]);
    }
  }
  for (int k1 = 0; k1 <= 2; ++k1) {
    for (int j1 = 0; j1 <= 1; ++j1) {
      const double dvol = vp[1] * ayh0[j1] * az0[k1];
      for (int i1 = 0; i1 <= 2; ++i1) jadd<SERIAL>(&jy[goff(g, ii0 + i1, jh0 + j1, kk0 + k1)], dvol * ax0[i1]);
    }
    for (int j1 = 0; j1 <= 1; ++j1) {
      const double dvol = vp[1] * ayh1[j1] * az1[k1];
      for (int i1 = 0; i1 <= 2; ++i1) jadd<SERIAL>(&jy[goff(g, i + i1, jh + j1, k + k1)], dvol * ax1[i1]);
    }
  }
  for (int k1 = 0; k1 <= 1; ++k1) {
    for (int j1 = 0; j1 <= 2; ++j1) {
      const double dvol = vp[2] * ay0[j1] * azh0[k1];
      for (int i1 = 0; i1 <= 2; ++i1) jadd<SERIAL>(&jz[goff(g, ii0 + i1, jj0 + j1, kh0 + k1)], dvol * ax0[i1]);
    }
    for (int j1 = 0; j1 <= 2; ++j1) {
      const double dvol = vp[2] * ay1[j1] * azh1[k1];
      for (int i1 = 0; i1 <= 2; ++i1) jadd<SERIAL>(&jz[goff(g, i + i1, j + j1, kh + k1)], dvol * ax1[i1]);
    }
  }
}

template <bool SERIAL>
__device__ __forceinline__ void ncdef2d(const Geo& g, double* jc, double xn, double yn, double xo, double yo, double p1,
                                        double p2, float wght, double dtg) {
  double ax0[3], ay0[3], axh0[2], ayh0[2], ax1[3], ay1[3], axh1[2], ayh1[2];
  double vp1 = (double)wght * dtg * p1, vp2 = (double)wght * dtg * p2;
  vp1 = 0.5 * vp1;
  vp2 = 0.5 * vp2;
  const int ii0 = qlh64(xo, ax0, axh0), jj0 = qlh64(yo, ay0, ayh0);
  const int i = qlh64(xn, ax1, axh1), j = qlh64(yn, ay1, ayh1);
  const int ih0 = ii0, jh0 = jj0, ih = i, jh = j;
  double* jx = jc;
  double* jy = jc + g.ncell;
  for (int j1 = 0; j1 <= 2; ++j1) {
    double dvol = vp1 * ay1[j1];
    for (int i1 = 0; i1 <= 1; ++i1) jadd<SERIAL>(&jx[goff(g, ih + i1, j + j1, 1)], dvol * axh1[i1]);
    dvol = vp1 * ay0[j1];
    for (int i1 = 0; i1 <= 1; ++i1) jadd<SERIAL>(&jx[goff(g, ih0 + i1, jj0 + j1, 1)], dvol * axh0[i1]);
  }
  for (int j1 = 0; j1 <= 1; ++j1) {
    double dvol = vp2 * ayh0[j1];
    for (int i1 = 0; i1 <= 2; ++i1) jadd<SERIAL>(&jy[goff(g, ii0 + i1, jh0 + j1, 1)], dvol * ax0[i1]);
    dvol = vp2 * ayh1[j1];
    for (int i1 = 0; i1 <= 2; ++i1) jadd<SERIAL>(&jy[goff(g, i + i1, jh + j1, 1)], dvol * ax1[i1]);
  }
}

}  // namespace agpu
