// agpu_yee.cuh — field kernels templated on the storage type: boundary
// extrapolation (A1), current fold (A13) and the leapfrog Yee update with
// Mur-type open boundaries (A14).  Included by agpu_fp64.cu (T = double,
// compiled without FMA contraction so the statement order of the reference
// is kept bit for bit) and agpu_fp32.cu (T = float).
#pragma once
#include "agpu_common.cuh"
#include "agpu_kernels.h"

namespace agpu {

// Every kernel body is a device function over "its" blocks bid_ of nb_, so
// that the same body runs as a single-instance kernel (bid_ = blockIdx.x) or
// inside a kernel that serves many instances at once (one row of blocks per
// instance).
#define GRID_STRIDE(t, total) \
  for (long long t = bid_ * (long long)blockDim.x + threadIdx.x; t < (total); t += nb_ * (long long)blockDim.x)

// ---- A1: field_xyzbd (src/parallel/mpi_field_interface.f90:53-198) --------
template <typename T>
__device__ __forceinline__ void d_field_bd_x(T* ebf, Geo g, int nc, long long bid_, long long nb_) {
  int ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  long long total = (long long)ny * nz * nc;
  GRID_STRIDE(t, total) {
    int iy = g.jy1 + (int)(t % ny);
    int iz = g.kz1 + (int)((t / ny) % nz);
    int ik = (int)(t / ((long long)ny * nz));
    T* f = ebf + g.ncell * ik;
    f[goff(g, g.ix1 - 1, iy, iz)] = (T)2. * f[goff(g, g.ix1, iy, iz)] - f[goff(g, g.ix1 + 1, iy, iz)];
    f[goff(g, g.ix2 + 1, iy, iz)] = (T)2. * f[goff(g, g.ix2, iy, iz)] - f[goff(g, g.ix2 - 1, iy, iz)];
  }
}
template <typename T>
__global__ void k_field_bd_x(T* ebf, Geo g, int nc) {
  d_field_bd_x<T>(ebf, g, nc, blockIdx.x, gridDim.x);
}
template <typename T>
__device__ __forceinline__ void d_field_bd_y(T* ebf, Geo g, int nc, long long bid_, long long nb_) {
  int nxe = g.ix2 - g.ix1 + 3, nz = g.kz2 - g.kz1 + 1;
  long long total = (long long)nxe * nz * nc;
  GRID_STRIDE(t, total) {
    int ix = g.ix1 - 1 + (int)(t % nxe);
    int iz = g.kz1 + (int)((t / nxe) % nz);
    int ik = (int)(t / ((long long)nxe * nz));
    T* f = ebf + g.ncell * ik;
    f[goff(g, ix, g.jy1 - 1, iz)] = (T)2. * f[goff(g, ix, g.jy1, iz)] - f[goff(g, ix, g.jy1 + 1, iz)];
    f[goff(g, ix, g.jy2 + 1, iz)] = (T)2. * f[goff(g, ix, g.jy2, iz)] - f[goff(g, ix, g.jy2 - 1, iz)];
  }
}
template <typename T>
__global__ void k_field_bd_y(T* ebf, Geo g, int nc) {
  d_field_bd_y<T>(ebf, g, nc, blockIdx.x, gridDim.x);
}
template <typename T>
__device__ __forceinline__ void d_field_bd_z(T* ebf, Geo g, int nc, long long bid_, long long nb_) {
  int nxe = g.ix2 - g.ix1 + 3, nye = g.jy2 - g.jy1 + 3;
  long long total = (long long)nxe * nye * nc;
  GRID_STRIDE(t, total) {
    int ix = g.ix1 - 1 + (int)(t % nxe);
    int iy = g.jy1 - 1 + (int)((t / nxe) % nye);
    int ik = (int)(t / ((long long)nxe * nye));
    T* f = ebf + g.ncell * ik;
    f[goff(g, ix, iy, g.kz1 - 1)] = (T)2 * f[goff(g, ix, iy, g.kz1)] - f[goff(g, ix, iy, g.kz1 + 1)];
    f[goff(g, ix, iy, g.kz2 + 1)] = (T)2 * f[goff(g, ix, iy, g.kz2)] - f[goff(g, ix, iy, g.kz2 - 1)];
  }
}
template <typename T>
__global__ void k_field_bd_z(T* ebf, Geo g, int nc) {
  d_field_bd_z<T>(ebf, g, nc, blockIdx.x, gridDim.x);
}
template <typename T>
void field_bd_t(T* ebf, const Geo& g, cudaStream_t st, int sms) {
  int nc = g.nf;
  k_field_bd_x<T><<<grid_for((long long)(g.jy2 - g.jy1 + 1) * (g.kz2 - g.kz1 + 1) * nc, 256, sms), 256, 0, st>>>(ebf, g, nc);
  k_field_bd_y<T><<<grid_for((long long)(g.ix2 - g.ix1 + 3) * (g.kz2 - g.kz1 + 1) * nc, 256, sms), 256, 0, st>>>(ebf, g, nc);
  if (g.ndim == 3)
    k_field_bd_z<T><<<grid_for((long long)(g.ix2 - g.ix1 + 3) * (g.jy2 - g.jy1 + 3) * nc, 256, sms), 256, 0, st>>>(ebf, g, nc);
}

// ---- A13: jc_xyzbd (src/parallel/mpi_curr_interface.f90:551-643) ----------
template <typename T>
__device__ __forceinline__ void d_jfold_x(T* jc, Geo g, long long bid_, long long nb_) {
  int ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  long long total = (long long)ny * nz * g.nc;
  GRID_STRIDE(t, total) {
    int j = g.jy1 + (int)(t % ny);
    int k = g.kz1 + (int)((t / ny) % nz);
    int ik = (int)(t / ((long long)ny * nz));
    T* c = jc + g.ncell * ik;
    long long a = goff(g, g.ix1, j, k);
    c[a] = c[a] + c[a - 1];
    c[a - 1] = (T)0;
    long long b = goff(g, g.ix2, j, k);
    c[b] = c[b] + c[b + 1] + c[b + 2];
    c[b + 1] = (T)0;
    c[b + 2] = (T)0;
  }
}
template <typename T>
__global__ void k_jfold_x(T* jc, Geo g) {
  d_jfold_x<T>(jc, g, blockIdx.x, gridDim.x);
}
template <typename T>
__device__ __forceinline__ void d_jfold_y(T* jc, Geo g, long long bid_, long long nb_) {
  int nx = g.ix2 - g.ix1 + 1, nz = g.kz2 - g.kz1 + 1;
  long long total = (long long)nx * nz * g.nc;
  long long sy = g.n1p;
  GRID_STRIDE(t, total) {
    int ix = g.ix1 + (int)(t % nx);
    int iz = g.kz1 + (int)((t / nx) % nz);
    int ik = (int)(t / ((long long)nx * nz));
    T* c = jc + g.ncell * ik;
    long long a = goff(g, ix, g.jy1, iz);
    c[a] = c[a] + c[a - sy] + c[a - 2 * sy];
    c[a - 2 * sy] = (T)0;
    c[a - sy] = (T)0;
    long long b = goff(g, ix, g.jy2, iz);
    c[b] = c[b] + c[b + sy] + c[b + 2 * sy];
    c[b + sy] = (T)0;
    c[b + 2 * sy] = (T)0;
  }
}
template <typename T>
__global__ void k_jfold_y(T* jc, Geo g) {
  d_jfold_y<T>(jc, g, blockIdx.x, gridDim.x);
}
template <typename T>
__device__ __forceinline__ void d_jfold_z(T* jc, Geo g, long long bid_, long long nb_) {
  int nx = g.ix2 - g.ix1 + 1, ny = g.jy2 - g.jy1 + 1;
  long long total = (long long)nx * ny * g.nc;
  long long sz = (long long)g.n1p * g.n2p;
  GRID_STRIDE(t, total) {
    int ix = g.ix1 + (int)(t % nx);
    int iy = g.jy1 + (int)((t / nx) % ny);
    int ik = (int)(t / ((long long)nx * ny));
    T* c = jc + g.ncell * ik;
    long long a = goff(g, ix, iy, g.kz1);
    c[a] = c[a] + c[a - sz];
    c[a - sz] = (T)0;
    long long b = goff(g, ix, iy, g.kz2);
    c[b] = c[b] + c[b + sz] + c[b + 2 * sz];
    c[b + sz] = (T)0;
    c[b + 2 * sz] = (T)0;
  }
}
template <typename T>
__global__ void k_jfold_z(T* jc, Geo g) {
  d_jfold_z<T>(jc, g, blockIdx.x, gridDim.x);
}
template <typename T>
void jfold_t(T* jc, const Geo& g, cudaStream_t st, int sms) {
  k_jfold_x<T><<<grid_for((long long)(g.jy2 - g.jy1 + 1) * (g.kz2 - g.kz1 + 1) * g.nc, 256, sms), 256, 0, st>>>(jc, g);
  k_jfold_y<T><<<grid_for((long long)(g.ix2 - g.ix1 + 1) * (g.kz2 - g.kz1 + 1) * g.nc, 256, sms), 256, 0, st>>>(jc, g);
  if (g.ndim == 3)
    k_jfold_z<T><<<grid_for((long long)(g.ix2 - g.ix1 + 1) * (g.jy2 - g.jy1 + 1) * g.nc, 256, sms), 256, 0, st>>>(jc, g);
}

// ---- A14: Yee (advance_lpf_fields, curr_and_fields_util.f90:176-260) ------

// ef_bds (src/fields/grid_fields.f90:1204-1354): right-face Mur boundary of E.
template <typename T>
__device__ __forceinline__ void d_ef_bds(T* ebf, Geo g, YeeC c, double dtl, long long bid_, long long nb_) {
  int ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1, nx = g.ix2 - g.ix1 + 1;
  long long nfx = (long long)ny * nz, nfy = (long long)nx * nz, nfz = (g.ndim == 3) ? (long long)nx * ny : 0;
  int nf = g.nf;
  T* E1 = ebf;
  T* E2 = ebf + g.ncell;
  T* E3 = ebf + 2 * g.ncell;
  T* B1 = ebf + 3 * g.ncell;
  T* B2 = ebf + 4 * g.ncell;
  T* Bn = ebf + (nf - 1) * g.ncell;
  const T one = (T)1., two = (T)2.;
  GRID_STRIDE(t, nfx + nfy + nfz) {
    if (t < nfx) {
      int j = g.jy1 + (int)(t % ny), k = g.kz1 + (int)(t / ny);
      T aphx = (T)(1.0 * c.dx_inv * dtl);
      long long o = goff(g, g.ix2, j, k);
      E2[o + 1] = (two * Bn[o] - (one - aphx) * E2[o]) / (one + aphx);
      if (nf > 3) E3[o + 1] = -(two * B2[o] + (one - aphx) * E3[o]) / (one + aphx);
    } else if (t < nfx + nfy) {
      long long u = t - nfx;
      int i = g.ix1 + (int)(u % nx), k = g.kz1 + (int)(u / nx);
      T aphy = (T)(c.ty4 * c.dy_inv * dtl);  // loc_yg(ny, 4) dy_inv dt
      long long o = goff(g, i, g.jy2, k), o1 = o + g.n1p;
      E1[o1] = -(two * Bn[o] + (one - aphy) * E1[o]) / (one + aphy);
      if (nf > 3) E3[o1] = (two * B1[o] - (one - aphy) * E3[o]) / (one + aphy);
    } else {
      long long u = t - nfx - nfy;
      int i = g.ix1 + (int)(u % nx), j = g.jy1 + (int)(u / nx);
      T aphz = (T)(c.tz4 * c.dz_inv * dtl);  // loc_zg(nz, 4) dz_inv dt
      long long o = goff(g, i, j, g.kz2), o1 = o + (long long)g.n1p * g.n2p;
      E1[o1] = (two * B2[o] - (one - aphz) * E1[o]) / (one + aphz);
      E2[o1] = -(two * B1[o] + (one - aphz) * E2[o]) / (one + aphz);
    }
  }
}
template <typename T>
__global__ void k_ef_bds(T* ebf, Geo g, YeeC c, double dtl) {
  d_ef_bds<T>(ebf, g, c, dtl, blockIdx.x, gridDim.x);
}
// bf_bds (src/fields/grid_fields.f90:1069-1202): left-face Mur boundary of B.
template <typename T>
__device__ __forceinline__ void d_bf_bds(T* ebf, Geo g, YeeC c, double dtl, long long bid_, long long nb_) {
  int ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1, nx = g.ix2 - g.ix1 + 1;
  long long nfx = (long long)ny * nz, nfy = (long long)nx * nz, nfz = (g.ndim == 3) ? (long long)nx * ny : 0;
  int nf = g.nf;
  T* E1 = ebf;
  T* E2 = ebf + g.ncell;
  T* E3 = ebf + 2 * g.ncell;
  T* B1 = ebf + 3 * g.ncell;
  T* B2 = ebf + 4 * g.ncell;
  T* Bn = ebf + (nf - 1) * g.ncell;
  const T one = (T)1., two = (T)2.;
  GRID_STRIDE(t, nfx + nfy + nfz) {
    if (t < nfx) {
      int j = g.jy1 + (int)(t % ny), k = g.kz1 + (int)(t / ny);
      T aphx = (T)(1.0 * c.dx_inv * dtl);
      long long o = goff(g, g.ix1, j, k);
      Bn[o - 1] = -(two * E2[o] + (one - aphx) * Bn[o]) / (one + aphx);
      if (nf > 3) B2[o - 1] = (two * E3[o] - (one - aphx) * B2[o]) / (one + aphx);
    } else if (t < nfx + nfy) {
      long long u = t - nfx;
      int i = g.ix1 + (int)(u % nx), k = g.kz1 + (int)(u / nx);
      T aphy = (T)(c.by3 * c.dy_inv * dtl);  // loc_yg(1, 3) dy_inv dt
      long long o = goff(g, i, g.jy1, k), o1 = o - g.n1p;
      T v = two * E1[o] - (one - aphy) * Bn[o];
      Bn[o1] = v / (one + aphy);
      if (nf > 3) {
        T w = -two * E3[o] - (one - aphy) * B1[o];
        B1[o1] = w / (one + aphy);
      }
    } else {
      long long u = t - nfx - nfy;
      int i = g.ix1 + (int)(u % nx), j = g.jy1 + (int)(u / nx);
      T aphz = (T)(c.bz3 * c.dz_inv * dtl);  // loc_zg(1, 3) dz_inv dt
      long long o = goff(g, i, j, g.kz1), o1 = o - (long long)g.n1p * g.n2p;
      T v = two * E2[o] - (one - aphz) * B1[o];
      B1[o1] = v / (one + aphz);
      T w = -two * E1[o] - (one - aphz) * B2[o];
      B2[o1] = w / (one + aphz);
    }
  }
}
template <typename T>
__global__ void k_bf_bds(T* ebf, Geo g, YeeC c, double dtl) {
  d_bf_bds<T>(ebf, g, c, dtl, blockIdx.x, gridDim.x);
}

// rote (grid_fields.f90:1405-1478): B -= dtf curl E, interior.
template <typename T, int NDIM>
__device__ __forceinline__ void d_rote(T* ebf, Geo g, YeeC c, double dtf, long long bid_, long long nb_) {
  int nx = g.ix2 - g.ix1 + 1, ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  long long total = (long long)nx * ny * nz;
  double aphxd = dtf * c.dx_inv, aphyd = dtf * c.dy_inv, aphzd = dtf * c.dz_inv;
  T aph1 = (T)(aphxd * c.se1), aph2 = (T)(aphxd * c.se2);
  T sdhy = (T)(1.0 * aphyd), sdhz = (T)(1.0 * aphzd);
  const T* E1 = ebf;
  const T* E2 = ebf + g.ncell;
  const T* E3 = ebf + 2 * g.ncell;
  long long sy = g.n1p, sz = (long long)g.n1p * g.n2p;
  GRID_STRIDE(t, total) {
    int i = g.ix1 + (int)(t % nx);
    int j = g.jy1 + (int)((t / nx) % ny);
    int k = g.kz1 + (int)(t / ((long long)nx * ny));
    long long o = goff(g, i, j, k);
    if (NDIM == 2) {
      T* Bz = ebf + 2 * g.ncell;
      Bz[o] = Bz[o] - aph1 * (E2[o + 1] - E2[o]) + sdhy * (E1[o + sy] - E1[o]) - aph2 * (E2[o + 2] - E2[o - 1]);
    } else {
      T* Bx = ebf + 3 * g.ncell;
      T* By = ebf + 4 * g.ncell;
      T* Bz = ebf + 5 * g.ncell;
      Bz[o] = Bz[o] - aph1 * (E2[o + 1] - E2[o]) + sdhy * (E1[o + sy] - E1[o]) - aph2 * (E2[o + 2] - E2[o - 1]);
      Bx[o] = Bx[o] - sdhy * (E3[o + sy] - E3[o]) + sdhz * (E2[o + sz] - E2[o]);
      By[o] = By[o] + aph1 * (E3[o + 1] - E3[o]) - sdhz * (E1[o + sz] - E1[o]) + aph2 * (E3[o + 2] - E3[o - 1]);
    }
  }
}
template <typename T, int NDIM>
__global__ void __launch_bounds__(256) k_rote(T* ebf, Geo g, YeeC c, double dtf) {
  d_rote<T, NDIM>(ebf, g, c, dtf, blockIdx.x, gridDim.x);
}

// rotb (grid_fields.f90:1480-1552) + E -= ompe * (djc * J)
// (curr_and_fields_util.f90:111-115, 227-231).  jlo (optional) holds the
// compensation term of a two-float current.
template <typename T, int NDIM>
__device__ __forceinline__ void d_rotb_j(T* ebf, const T* jc, const T* jlo, Geo g, YeeC c, double dtf, long long bid_, long long nb_) {
  int nx = g.ix2 - g.ix1 + 1, ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  long long total = (long long)nx * ny * nz;
  double aphxd = dtf * c.dx_inv, aphyd = dtf * c.dy_inv, aphzd = dtf * c.dz_inv;
  T aph1 = (T)(aphxd * c.se1), aph2 = (T)(aphxd * c.se2);
  T sdy = (T)(1.0 * aphyd), sdz = (T)(aphzd * 1.0);
  T ompe = (T)c.ompe, djc1 = (T)c.djc1, djc2 = (T)c.djc2, djc3 = (T)c.djc3;
  T* E1 = ebf;
  T* E2 = ebf + g.ncell;
  long long sy = g.n1p, sz = (long long)g.n1p * g.n2p;
  GRID_STRIDE(t, total) {
    int i = g.ix1 + (int)(t % nx);
    int j = g.jy1 + (int)((t / nx) % ny);
    int k = g.kz1 + (int)(t / ((long long)nx * ny));
    long long o = goff(g, i, j, k);
    T j1 = jc[o], j2 = jc[o + g.ncell];
    if (jlo) {
      j1 = j1 + jlo[o];
      j2 = j2 + jlo[o + g.ncell];
    }
    if (NDIM == 2) {
      const T* Bz = ebf + 2 * g.ncell;
      T ex = E1[o] + sdy * (Bz[o] - Bz[o - sy]);
      T ey = E2[o] - aph1 * (Bz[o] - Bz[o - 1]) - aph2 * (Bz[o + 1] - Bz[o - 2]);
      E1[o] = ex - ompe * (djc1 * j1);
      E2[o] = ey - ompe * (djc2 * j2);
    } else {
      T* E3 = ebf + 2 * g.ncell;
      const T* Bx = ebf + 3 * g.ncell;
      const T* By = ebf + 4 * g.ncell;
      const T* Bz = ebf + 5 * g.ncell;
      T j3 = jc[o + 2 * g.ncell];
      if (jlo) j3 = j3 + jlo[o + 2 * g.ncell];
      T ex = E1[o] + sdy * (Bz[o] - Bz[o - sy]);
      T ey = E2[o] - aph1 * (Bz[o] - Bz[o - 1]) - aph2 * (Bz[o + 1] - Bz[o - 2]);
      ex = ex - sdz * (By[o] - By[o - sz]);
      ey = ey + sdz * (Bx[o] - Bx[o - sz]);
      T ez = E3[o] + aph1 * (By[o] - By[o - 1]) - sdy * (Bx[o] - Bx[o - sy]) + aph2 * (By[o + 1] - By[o - 2]);
      E1[o] = ex - ompe * (djc1 * j1);
      E2[o] = ey - ompe * (djc2 * j2);
      E3[o] = ez - ompe * (djc3 * j3);
    }
  }
}
template <typename T, int NDIM>
__global__ void __launch_bounds__(256) k_rotb_j(T* ebf, const T* jc, const T* jlo, Geo g, YeeC c, double dtf) {
  d_rotb_j<T, NDIM>(ebf, jc, jlo, g, c, dtf, blockIdx.x, gridDim.x);
}

// Single-instance forms of the two sweeps: one thread per node, blocks of
// 128 x 2 nodes over (i, j) and one z plane per grid layer, so the node
// indices come without the 64-bit divisions of the grid-stride bodies (which
// serve the multi-instance kernels).  Every node's arithmetic is that of
// d_rote / d_rotb_j, in the same order.  Measured on the 1024x256x256 grid:
// the FP32 phase 2.42 -> 2.06 ms; marching each thread over several z planes
// (carrying the z-neighbour loads) was slower.
constexpr int YEE_BX = 128, YEE_BY = 2;

template <typename T, int NDIM>
__global__ void __launch_bounds__(YEE_BX* YEE_BY) k_rote_n(T* ebf, Geo g, YeeC c, double dtf) {
  const int i = g.ix1 + blockIdx.x * YEE_BX + threadIdx.x;
  const int j = g.jy1 + blockIdx.y * YEE_BY + threadIdx.y;
  if (i > g.ix2 || j > g.jy2) return;
  const double aphxd = dtf * c.dx_inv, aphyd = dtf * c.dy_inv, aphzd = dtf * c.dz_inv;
  const T aph1 = (T)(aphxd * c.se1), aph2 = (T)(aphxd * c.se2);
  // loc_yg(jj, 4) * aphy, loc_zg(kk, 4) * aphz (1 on a uniform axis)
  const int kn = (NDIM == 3) ? g.kz1 + (int)blockIdx.z : 1;
  const T sdhy = (T)((c.my4 ? c.my4[j - 2] : 1.0) * aphyd);
  const T sdhz = (T)((c.mz4 && NDIM == 3 ? c.mz4[kn - 2] : 1.0) * aphzd);
  const T* __restrict__ E1 = ebf;
  const T* __restrict__ E2 = ebf + g.ncell;
  const T* __restrict__ E3 = ebf + 2 * g.ncell;
  const long long sy = g.n1p, sz = (long long)g.n1p * g.n2p;
  if (NDIM == 2) {
    const long long o = goff(g, i, j, 1);
    T* Bz = ebf + 2 * g.ncell;
    Bz[o] = Bz[o] - aph1 * (E2[o + 1] - E2[o]) + sdhy * (E1[o + sy] - E1[o]) - aph2 * (E2[o + 2] - E2[o - 1]);
    return;
  }
  T* __restrict__ Bx = ebf + 3 * g.ncell;
  T* __restrict__ By = ebf + 4 * g.ncell;
  T* __restrict__ Bz = ebf + 5 * g.ncell;
  const long long o = goff(g, i, j, kn);
  Bz[o] = Bz[o] - aph1 * (E2[o + 1] - E2[o]) + sdhy * (E1[o + sy] - E1[o]) - aph2 * (E2[o + 2] - E2[o - 1]);
  Bx[o] = Bx[o] - sdhy * (E3[o + sy] - E3[o]) + sdhz * (E2[o + sz] - E2[o]);
  By[o] = By[o] + aph1 * (E3[o + 1] - E3[o]) - sdhz * (E1[o + sz] - E1[o]) + aph2 * (E3[o + 2] - E3[o - 1]);
}

template <typename T, int NDIM>
__global__ void __launch_bounds__(YEE_BX* YEE_BY) k_rotb_j_n(T* ebf, const T* jc, const T* jlo, Geo g, YeeC c, double dtf) {
  const int i = g.ix1 + blockIdx.x * YEE_BX + threadIdx.x;
  const int j = g.jy1 + blockIdx.y * YEE_BY + threadIdx.y;
  if (i > g.ix2 || j > g.jy2) return;
  const double aphxd = dtf * c.dx_inv, aphyd = dtf * c.dy_inv, aphzd = dtf * c.dz_inv;
  const T aph1 = (T)(aphxd * c.se1), aph2 = (T)(aphxd * c.se2);
  // loc_yg(jj, 3) * aphy, aphz * loc_zg(kk, 3) (1 on a uniform axis)
  const int kn = (NDIM == 3) ? g.kz1 + (int)blockIdx.z : 1;
  const T sdy = (T)((c.my3 ? c.my3[j - 2] : 1.0) * aphyd);
  const T sdz = (T)(aphzd * (c.mz3 && NDIM == 3 ? c.mz3[kn - 2] : 1.0));
  const T ompe = (T)c.ompe, djc1 = (T)c.djc1, djc2 = (T)c.djc2, djc3 = (T)c.djc3;
  T* __restrict__ E1 = ebf;
  T* __restrict__ E2 = ebf + g.ncell;
  const long long sy = g.n1p, sz = (long long)g.n1p * g.n2p;
  const long long o = goff(g, i, j, kn);
  T j1 = jc[o], j2 = jc[o + g.ncell];
  if (jlo) {
    j1 = j1 + jlo[o];
    j2 = j2 + jlo[o + g.ncell];
  }
  if (NDIM == 2) {
    const T* Bz = ebf + 2 * g.ncell;
    T ex = E1[o] + sdy * (Bz[o] - Bz[o - sy]);
    T ey = E2[o] - aph1 * (Bz[o] - Bz[o - 1]) - aph2 * (Bz[o + 1] - Bz[o - 2]);
    if (c.my3) {
      // curr_mpi_collect on a stretched y: dery (djc jx), derhy (djc jy)
      E1[o] = ex - ompe * ((T)c.my3[j - 2] * (djc1 * j1));
      E2[o] = ey - ompe * ((T)c.my4[j - 2] * (djc2 * j2));
      return;
    }
    E1[o] = ex - ompe * (djc1 * j1);
    E2[o] = ey - ompe * (djc2 * j2);
    return;
  }
  T* __restrict__ E3 = ebf + 2 * g.ncell;
  const T* __restrict__ Bx = ebf + 3 * g.ncell;
  const T* __restrict__ By = ebf + 4 * g.ncell;
  const T* __restrict__ Bz = ebf + 5 * g.ncell;
  T j3 = jc[o + 2 * g.ncell];
  if (jlo) j3 = j3 + jlo[o + 2 * g.ncell];
  T ex = E1[o] + sdy * (Bz[o] - Bz[o - sy]);
  T ey = E2[o] - aph1 * (Bz[o] - Bz[o - 1]) - aph2 * (Bz[o + 1] - Bz[o - 2]);
  ex = ex - sdz * (By[o] - By[o - sz]);
  ey = ey + sdz * (Bx[o] - Bx[o - sz]);
  T ez = E3[o] + aph1 * (By[o] - By[o - 1]) - sdy * (Bx[o] - Bx[o - sy]) + aph2 * (By[o + 1] - By[o - 2]);
  if (c.my3) {
    // curr_mpi_collect on stretched y and z: dery derz, derhy derz, dery derhz
    const T dery = (T)c.my3[j - 2], derhy = (T)c.my4[j - 2];
    const T derz = (T)c.mz3[kn - 2], derhz = (T)c.mz4[kn - 2];
    E1[o] = ex - ompe * ((dery * derz) * (djc1 * j1));
    E2[o] = ey - ompe * ((derhy * derz) * (djc2 * j2));
    E3[o] = ez - ompe * ((dery * derhz) * (djc3 * j3));
    return;
  }
  E1[o] = ex - ompe * (djc1 * j1);
  E2[o] = ey - ompe * (djc2 * j2);
  E3[o] = ez - ompe * (djc3 * j3);
}

// ---- comoving frame: field_xadvect (src/fields/grid_fields.f90:210-324) ----

// x ghosts: f(ix1-1) = f(ix1+1), f(ix2+1) = f(ix2), components ic1..ic2
template <typename T>
__global__ void k_xadv_ghost(T* ebf, Geo g, int ic1, int ic2) {
  const int ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  const long long rows = (long long)ny * nz;
  const long long total = rows * (ic2 - ic1 + 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int ic = ic1 + (int)(t / rows);
    const long long r = t - (long long)(ic - ic1) * rows;
    const int j = g.jy1 + (int)(r % ny), k = g.kz1 + (int)(r / ny);
    T* row = ebf + g.ncell * (ic - 1) + goff(g, 1, j, k) - 1;  // row[i] = f(i)
    row[g.ix1 - 1] = row[g.ix1 + 1];
    row[g.ix2 + 1] = row[g.ix2];
  }
}
// explicit step of one component into the row buffer, then back
template <typename T>
__global__ void k_xadv_explicit(const T* f, double* tmp, Geo g, double aphx_exp) {
  const int i = g.ix1 + blockIdx.x * YEE_BX + threadIdx.x;
  const int j = g.jy1 + blockIdx.y * YEE_BY + threadIdx.y;
  if (i > g.ix2 || j > g.jy2) return;
  const long long o = goff(g, i, j, g.ndim == 3 ? g.kz1 + (int)blockIdx.z : 1);
  tmp[o] = f[o] - aphx_exp * (f[o + 1] - f[o - 1]);
}
template <typename T>
__global__ void k_xadv_copy(T* f, const double* tmp, Geo g) {
  const int i = g.ix1 + blockIdx.x * YEE_BX + threadIdx.x;
  const int j = g.jy1 + blockIdx.y * YEE_BY + threadIdx.y;
  if (i > g.ix2 || j > g.jy2) return;
  const long long o = goff(g, i, j, g.ndim == 3 ? g.kz1 + (int)blockIdx.z : 1);
  f[o] = tmp[o];
}
// implicit step: one thread per row (component ic1..ic2), the Thomas sweeps
// in place in trid_der1's order
template <typename T>
__global__ void k_xadv_implicit(T* ebf, Geo g, int ic1, int ic2, XAdv x) {
  const int ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  const long long rows = (long long)ny * nz;
  const long long total = rows * (ic2 - ic1 + 1);
  const int n = g.ix2 - g.ix1 + 1;
  const double a = x.a, an = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int ic = ic1 + (int)(t / rows);
    const long long r = t - (long long)(ic - ic1) * rows;
    const int j = g.jy1 + (int)(r % ny), k = g.kz1 + (int)(r / ny);
    T* u = ebf + g.ncell * (ic - 1) + goff(g, g.ix1, j, k) - 1;  // u[kk] = f(ix1 + kk - 1), kk = 1..n
    u[1] = u[1] / x.bet[1];
    for (int kk = 2; kk <= n - 1; ++kk) u[kk] = (u[kk] - a * u[kk - 1]) / x.bet[kk];
    u[n] = (u[n] - an * u[n - 1]) / x.bet[n];
    for (int kk = n - 1; kk >= 1; --kk) u[kk] = u[kk] - x.w1[kk + 1] * u[kk + 1];
  }
}
template <typename T>
void xadvect_t(T* ebf, const Geo& g, int ic1, int ic2, int isch, const XAdv& x, cudaStream_t st, int sms) {
  const long long rows = (long long)(g.jy2 - g.jy1 + 1) * (g.kz2 - g.kz1 + 1) * (ic2 - ic1 + 1);
  k_xadv_ghost<T><<<grid_for(rows, 256, sms), 256, 0, st>>>(ebf, g, ic1, ic2);
  if (isch == 0) {
    const dim3 blk(YEE_BX, YEE_BY, 1);
    const dim3 grd((g.ix2 - g.ix1 + YEE_BX) / YEE_BX, (g.jy2 - g.jy1 + YEE_BY) / YEE_BY, g.ndim == 3 ? g.kz2 - g.kz1 + 1 : 1);
    for (int ic = ic1; ic <= ic2; ++ic) {
      k_xadv_explicit<T><<<grd, blk, 0, st>>>(ebf + g.ncell * (ic - 1), x.tmp, g, x.aphx_exp);
      k_xadv_copy<T><<<grd, blk, 0, st>>>(ebf + g.ncell * (ic - 1), x.tmp, g);
    }
  } else {
    k_xadv_implicit<T><<<(int)((rows + 127) / 128), 128, 0, st>>>(ebf, g, ic1, ic2, x);
  }
}

// xa: the comoving frame's advection scratch (c.vbeam > 0), else null;
// hk: a y slab's halo exchange after each boundary sweep, else null
template <typename T>
void yee_t(T* ebf, const T* jc, const T* jlo, const Geo& g, const YeeC& c, cudaStream_t st, int sms,
           const XAdv* xa = nullptr, YeeHook* hk = nullptr) {
  long long faces = (long long)(g.jy2 - g.jy1 + 1) * (g.kz2 - g.kz1 + 1) + (long long)(g.ix2 - g.ix1 + 1) * (g.kz2 - g.kz1 + 1) +
                    (g.ndim == 3 ? (long long)(g.ix2 - g.ix1 + 1) * (g.jy2 - g.jy1 + 1) : 0);
  int gf = grid_for(faces, 256, sms);
  const dim3 blk(YEE_BX, YEE_BY, 1);
  const dim3 grd((g.ix2 - g.ix1 + YEE_BX) / YEE_BX, (g.jy2 - g.jy1 + YEE_BY) / YEE_BY,
                 g.ndim == 3 ? g.kz2 - g.kz1 + 1 : 1);
  double dt = c.dt, dth = 0.5 * dt;
  // the comoving frame's advection substeps (curr_and_fields_util.f90:200-258)
  const bool adv = xa && c.vbeam > 0.0;
  const int nb1 = g.nc + 1, nb2 = g.nf, ne1 = 1, ne2 = g.nc;
  auto halo = [&](int point) {
    if (hk && !hk->rc) hk->rc = hk->fn(hk->ctx, point);
    return hk && hk->rc;
  };
  k_ef_bds<T><<<gf, 256, 0, st>>>(ebf, g, c, 0.0);
  if (halo(AGPU_HALO_E)) return;
  if (adv) xadvect_t<T>(ebf, g, nb1, nb2, 0, *xa, st, sms);
  if (g.ndim == 3) k_rote_n<T, 3><<<grd, blk, 0, st>>>(ebf, g, c, dth); else k_rote_n<T, 2><<<grd, blk, 0, st>>>(ebf, g, c, dth);
  k_bf_bds<T><<<gf, 256, 0, st>>>(ebf, g, c, dt);
  if (halo(AGPU_HALO_B)) return;
  if (adv) xadvect_t<T>(ebf, g, ne1, ne2, 0, *xa, st, sms);
  if (g.ndim == 3) k_rotb_j_n<T, 3><<<grd, blk, 0, st>>>(ebf, jc, jlo, g, c, dt); else k_rotb_j_n<T, 2><<<grd, blk, 0, st>>>(ebf, jc, jlo, g, c, dt);
  if (adv) xadvect_t<T>(ebf, g, ne1, ne2, 2, *xa, st, sms);
  k_ef_bds<T><<<gf, 256, 0, st>>>(ebf, g, c, dt);
  if (halo(AGPU_HALO_E)) return;
  if (g.ndim == 3) k_rote_n<T, 3><<<grd, blk, 0, st>>>(ebf, g, c, dth); else k_rote_n<T, 2><<<grd, blk, 0, st>>>(ebf, g, c, dth);
  if (adv) xadvect_t<T>(ebf, g, nb1, nb2, 2, *xa, st, sms);
}

}  // namespace agpu
