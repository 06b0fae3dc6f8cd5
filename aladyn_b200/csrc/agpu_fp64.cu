// agpu_fp64.cu — the plain FP64 form of the PIC step on sm_100a.
//
// Compiled with -fmad=false: every expression keeps the reference's
// statement order and rounding (no fused multiply-add), so cell indices,
// momenta and positions reproduce the Fortran arithmetic bit for bit given
// the same fields; the currents differ only by the order of the atomic sums
// unless the deterministic (serial) deposit is selected.
#include "agpu_common.cuh"
#include "agpu_fp64_dep.cuh"
#include "agpu_kernels.h"
#include "agpu_yee.cuh"
#include "agpu_yee_fused.cuh"

namespace agpu {

void field_bd64(const Dev64& d, cudaStream_t st, int sms) { field_bd_t<double>(d.ebf, d.g, st, sms); }

// ============================================================================
// Cubic shape extension (AGPU_SHAPE_CUBIC; no counterpart in the reference):
// cubic B-spline weights on integer nodes (the weights of cden_3d_wgh,
// grid_part_lib.f90:419-454), quadratic on half nodes (qqh), and Esirkepov's
// deposit with 4-point shapes on 6-slot windows.  Same arithmetic, in the
// same order, as the oracle's restatement.
// ============================================================================
__device__ __forceinline__ int cden64(double xp, double a[4]) {
  const double one_sixth = 1.0 / 6.0, two_third = 2.0 / 3.0;
  double xx = 3.0 + xp;
  int i = (int)xx;
  double sx = xx - (double)i;
  double sx2 = sx * sx;
  double sx3 = sx2 * sx;
  a[1] = two_third - sx2 + 0.5 * sx3;
  a[2] = one_sixth + 0.5 * (sx + sx2 - sx3);
  a[3] = one_sixth * sx3;
  a[0] = 1. - a[1] - a[2] - a[3];
  return i;
}
__device__ __forceinline__ int qhalf64(double xp, double a[3]) {
  double xx = 3.0 + xp;
  int h = (int)xx;
  double sx = xx - (double)h - 0.5;
  double sx2 = sx * sx;
  a[1] = 0.75 - sx2;
  a[2] = 0.5 * (0.25 + sx2 + sx);
  a[0] = 1. - a[1] - a[2];
  return h;
}

// Gather of the 2 (2D: Ex, Ey, Bz) or 6 field components; false when the
// stencil leaves the array.  Per point (w_x * (w_y * w_z)) * F.
__device__ __forceinline__ bool gather_cubic64(const Geo& g, const double* __restrict__ ebf, const double* xl, int ndim,
                                               double ap[6]) {
  double ax[4], ay[4], az[4] = {0., 1., 0., 0.}, axh[3], ayh[3], azh[3] = {0., 1., 0.};
  const int fx = cden64(xl[0], ax), hx = qhalf64(xl[0], axh);
  const int fy = cden64(xl[1], ay), hy = qhalf64(xl[1], ayh);
  int kz0 = 1, kh0 = 1, nzi = 1;
  if (ndim == 3) {
    const int fz = cden64(xl[2], az), hz = qhalf64(xl[2], azh);
    kz0 = fz - 1;
    kh0 = hz - 1;
    nzi = 4;
    if (kz0 < 1 || fz + 2 > g.n3p) return false;
  }
  if (fx - 1 < 1 || fx + 2 > g.n1p || fy - 1 < 1 || fy + 2 > g.n2p) return false;
  const int ix0 = fx - 1, iy0 = fy - 1, hx0 = hx - 1, hy0 = hy - 1;
  const double* wzi = (ndim == 3) ? az : az + 1;
  const double* E1 = ebf;
  const double* E2 = ebf + g.ncell;
  for (int c = 0; c < 6; ++c) ap[c] = 0.;
  for (int k1 = 0; k1 < nzi; ++k1)
    for (int j1 = 0; j1 < 4; ++j1) {
      double dvol = ay[j1] * wzi[k1];
      for (int i1 = 0; i1 < 3; ++i1) ap[0] += (axh[i1] * dvol) * __ldg(&E1[goff(g, hx0 + i1, iy0 + j1, kz0 + k1)]);
    }
  for (int k1 = 0; k1 < nzi; ++k1)
    for (int j1 = 0; j1 < 3; ++j1) {
      double dvol = ayh[j1] * wzi[k1];
      for (int i1 = 0; i1 < 4; ++i1) ap[1] += (ax[i1] * dvol) * __ldg(&E2[goff(g, ix0 + i1, hy0 + j1, kz0 + k1)]);
    }
  if (ndim == 2) {
    const double* B3 = ebf + 2 * g.ncell;
    for (int j1 = 0; j1 < 3; ++j1) {
      double dvol = ayh[j1];
      for (int i1 = 0; i1 < 3; ++i1) ap[2] += (axh[i1] * dvol) * __ldg(&B3[goff(g, hx0 + i1, hy0 + j1, 1)]);
    }
    return true;
  }
  const double* E3 = ebf + 2 * g.ncell;
  const double* B1 = ebf + 3 * g.ncell;
  const double* B2 = ebf + 4 * g.ncell;
  const double* B3 = ebf + 5 * g.ncell;
  for (int k1 = 0; k1 < 3; ++k1)
    for (int j1 = 0; j1 < 4; ++j1) {
      double dvol = ay[j1] * azh[k1];
      for (int i1 = 0; i1 < 4; ++i1) ap[2] += (ax[i1] * dvol) * __ldg(&E3[goff(g, ix0 + i1, iy0 + j1, kh0 + k1)]);
    }
  for (int k1 = 0; k1 < 3; ++k1)
    for (int j1 = 0; j1 < 3; ++j1) {
      double dvol = ayh[j1] * azh[k1];
      for (int i1 = 0; i1 < 4; ++i1) ap[3] += (ax[i1] * dvol) * __ldg(&B1[goff(g, ix0 + i1, hy0 + j1, kh0 + k1)]);
    }
  for (int k1 = 0; k1 < 3; ++k1)
    for (int j1 = 0; j1 < 4; ++j1) {
      double dvol = ay[j1] * azh[k1];
      for (int i1 = 0; i1 < 3; ++i1) ap[4] += (axh[i1] * dvol) * __ldg(&B2[goff(g, hx0 + i1, iy0 + j1, kh0 + k1)]);
    }
  for (int k1 = 0; k1 < 4; ++k1)
    for (int j1 = 0; j1 < 3; ++j1) {
      double dvol = ayh[j1] * az[k1];
      for (int i1 = 0; i1 < 3; ++i1) ap[5] += (axh[i1] * dvol) * __ldg(&B3[goff(g, hx0 + i1, hy0 + j1, kz0 + k1)]);
    }
  return true;
}

// 1-D window: old shape on slots 1..4 (slot 0 = old floor node - 2), new on
// sh..sh+3, running current; returns the node of slot 0.
__device__ __forceinline__ int cubic_window64(double x0l, double x1l, double s0[6], double s1[6], double cur[6], int* lo,
                                              int* hi) {
  double a0[4], a1[4];
  const int f0 = cden64(x0l, a0);
  const int f1 = cden64(x1l, a1);
  const int sh = f1 - f0 + 1;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    s0[q] = (q >= 1 && q <= 4) ? a0[q - 1] : 0.;
    const int m = q - sh;
    s1[q] = (sh >= 0 && sh <= 2 && m >= 0 && m <= 3) ? a1[m] : 0.;
  }
  cur[0] = s0[0] - s1[0];
#pragma unroll
  for (int q = 1; q < 6; ++q) cur[q] = cur[q - 1] + s0[q] - s1[q];
  *lo = sh < 1 ? sh : 1;
  *hi = (sh + 3) > 4 ? sh + 3 : 4;
  return f0 - 2;
}

template <bool SERIAL>
__device__ bool esirkepov_cubic64(const Geo& g, double* jc, const double* xn, const double* xo, float wght, int ndim) {
  double sx0[6], sx1[6], cx[6], sy0[6], sy1[6], cy[6], sz0[6], sz1[6], cz[6];
  int x0, x1, y0, y1, z0 = 0, z1 = 0;
  const int bx = cubic_window64(xo[0], xn[0], sx0, sx1, cx, &x0, &x1);
  const int by = cubic_window64(xo[1], xn[1], sy0, sy1, cy, &y0, &y1);
  int bz = 1;
  if (ndim == 3) bz = cubic_window64(xo[2], xn[2], sz0, sz1, cz, &z0, &z1);
  const double w = (double)wght;
  bool ok = true;
  double* jx = jc;
  double* jy = jc + g.ncell;
  if (ndim == 2) {
    for (int v = y0; v <= y1; ++v)
      for (int u = x0; u <= x1; ++u) {
        const int i = bx + u, j = by + v;
        if (i < 1 || i > g.n1p || j < 1 || j > g.n2p) {
          ok = false;
          continue;
        }
        const long long o = goff(g, i, j, 1);
        jadd<SERIAL>(&jx[o], (w * cx[u]) * (sy0[v] + sy1[v]));
        jadd<SERIAL>(&jy[o], (sx0[u] + sx1[u]) * (w * cy[v]));
      }
    return ok;
  }
  double wx0[6], wx1[6], wy0[6], wy1[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    wx0[q] = 0.5 * sx1[q] + sx0[q];
    wx1[q] = sx1[q] + 0.5 * sx0[q];
    wy0[q] = 0.5 * sy1[q] + sy0[q];
    wy1[q] = sy1[q] + 0.5 * sy0[q];
  }
  double* jz = jc + 2 * g.ncell;
  for (int ww = z0; ww <= z1; ++ww)
    for (int v = y0; v <= y1; ++v)
      for (int u = x0; u <= x1; ++u) {
        const int i = bx + u, j = by + v, k = bz + ww;
        if (i < 1 || i > g.n1p || j < 1 || j > g.n2p || k < 1 || k > g.n3p) {
          ok = false;
          continue;
        }
        const long long o = goff(g, i, j, k);
        jadd<SERIAL>(&jx[o], (w * cx[u]) * (wy0[v] * sz0[ww] + wy1[v] * sz1[ww]));
        jadd<SERIAL>(&jy[o], (w * cy[v]) * (wx0[u] * sz0[ww] + wx1[u] * sz1[ww]));
        jadd<SERIAL>(&jz[o], (w * cz[ww]) * (wx0[u] * sy0[v] + wx1[u] * sy1[v]));
      }
  return ok;
}

// ============================================================================
// A2-A12 fused: gather (set_part{2,3}d_hcell_acc, grid_part_connect.f90:
// 89-285) -> charge multiply (curr_and_fields_util.f90:58-72) ->
// [init_lpf_momenta (boris_push.f90:34-73)] -> exact-gamma Boris push
// (boris_push.f90:75-168) -> box-edge test of cell_part_dist(.false.)
// (mpi_part_interface.f90:467-523) -> Esirkepov deposit of the particles that
// stay.  The reference runs these as separate sweeps with ebfp as scratch;
// per particle the arithmetic is identical, and a particle that leaves the
// box is exactly one that the reference removes before its deposit.
// ============================================================================

// set_local_*_positions (grid_part_lib.f90:458-519): y and z in cells, by
// the stretched axes' map when the grid is stretched
__device__ __forceinline__ double ly(const PushArgs64& a, double y) {
  return a.str ? str_map(a.sy, y) : a.dy_inv * (y - a.ymn);
}
__device__ __forceinline__ double lz(const PushArgs64& a, double z) {
  return a.str ? str_map(a.sz, z) : a.dz_inv * (z - a.zmn);
}

// A slab of a y (and z) decomposition: a particle that left through sides
// shared with neighbours, and through no physical side, moves on to them
// (part_prl_exchange, y first, then z).  The reference deposits it there,
// from its old position in the neighbour's ghost rows; here the slab it
// leaves deposits it into its own ghost rows, which the current exchange
// then adds to the neighbour's rows: the same terms on the same nodes.
__device__ __forceinline__ bool emigrant(const PushArgs64& a, double x, double y, double z) {
  if (!(x > a.gxmin && x <= a.gxmax)) return false;
  const bool yin = y > a.gymin && y <= a.gymax;
  const bool yok = yin || (a.dd_ylo && y <= a.gymin) || (a.dd_yhi && y > a.gymax);
  if (a.g.ndim < 3) return yok && !yin;
  const bool zin = z > a.gzmin && z <= a.gzmax;
  const bool zok = zin || (a.dd_zlo && z <= a.gzmin) || (a.dd_zhi && z > a.gzmax);
  return yok && zok && !(yin && zin);
}

template <bool SERIAL, int SHAPE>
__global__ void __launch_bounds__(256) k64_push_dep_3d(PushArgs64 a) {
  const Geo g = a.g;
  const double* __restrict__ ex = a.ebf;
  long long stride = SERIAL ? 1 : (long long)gridDim.x * blockDim.x;
  long long first = SERIAL ? 0 : blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (SERIAL && (blockIdx.x != 0 || threadIdx.x != 0)) return;
  for (long long n = first; n < a.np; n += stride) {
    double x = a.x[n], y = a.y[n], z = a.z[n];
    double pp[3] = {a.px[n], a.py[n], a.pz[n]};
    uint64_t sl = dbits(a.slot[n]);
    // set_local_3d_positions
    double xo[3] = {a.dx_inv * (x - a.xmn), ly(a, y), lz(a, z)};
    double ap[6] = {0, 0, 0, 0, 0, 0};
    if (SHAPE == AGPU_SHAPE_CUBIC) {
      if (!gather_cubic64(g, ex, xo, 3, ap)) {
        raise_err(a.err, AGPU_EBIT_INDEX);
        atomicAdd(a.removed, 1ull);  // outside the box: the compaction drops it
        continue;
      }
    } else {
      double ax1[3], axh[2], ay1[3], ayh[2], az1[3], azh[2];
      int i = qlh64(xo[0], ax1, axh);
      int j = qlh64(xo[1], ay1, ayh);
      int k = qlh64(xo[2], az1, azh);
      // gather needs i..i+2, the deposit i-1..i+3 (old node i+1 +- 2)
      if (i < 2 || i > g.n1p - 3 || j < 2 || j > g.n2p - 3 || k < 2 || k > g.n3p - 3) {
        raise_err(a.err, AGPU_EBIT_INDEX);
        atomicAdd(a.removed, 1ull);  // outside the box: the compaction drops it
        continue;
      }
      int ih = i, jh = j, kh = k;
      const double* e1 = ex;
      const double* e2 = ex + g.ncell;
      const double* e3 = ex + 2 * g.ncell;
      const double* b1 = ex + 3 * g.ncell;
      const double* b2 = ex + 4 * g.ncell;
      const double* b3 = ex + 5 * g.ncell;
  #pragma unroll
      for (int k1 = 0; k1 <= 2; ++k1) {
        int k2 = k + k1;
  #pragma unroll
        for (int j1 = 0; j1 <= 2; ++j1) {
          int j2 = j + j1;
          double dvol = ay1[j1] * az1[k1];
  #pragma unroll
          for (int i1 = 0; i1 <= 1; ++i1) ap[0] = ap[0] + axh[i1] * dvol * __ldg(&e1[goff(g, i1 + ih, j2, k2)]);
        }
  #pragma unroll
        for (int j1 = 0; j1 <= 1; ++j1) {
          int j2 = jh + j1;
          double dvol = ayh[j1] * az1[k1];
  #pragma unroll
          for (int i1 = 0; i1 <= 2; ++i1) ap[1] = ap[1] + ax1[i1] * dvol * __ldg(&e2[goff(g, i + i1, j2, k2)]);
  #pragma unroll
          for (int i1 = 0; i1 <= 1; ++i1) ap[5] = ap[5] + axh[i1] * dvol * __ldg(&b3[goff(g, i1 + ih, j2, k2)]);
        }
      }
  #pragma unroll
      for (int k1 = 0; k1 <= 1; ++k1) {
        int k2 = kh + k1;
  #pragma unroll
        for (int j1 = 0; j1 <= 1; ++j1) {
          int j2 = jh + j1;
          double dvol = ayh[j1] * azh[k1];
  #pragma unroll
          for (int i1 = 0; i1 <= 2; ++i1) ap[3] = ap[3] + ax1[i1] * dvol * __ldg(&b1[goff(g, i1 + i, j2, k2)]);
        }
  #pragma unroll
        for (int j1 = 0; j1 <= 2; ++j1) {
          int j2 = j + j1;
          double dvol = ay1[j1] * azh[k1];
  #pragma unroll
          for (int i1 = 0; i1 <= 1; ++i1) ap[4] = ap[4] + axh[i1] * dvol * __ldg(&b2[goff(g, ih + i1, j2, k2)]);
  #pragma unroll
          for (int i1 = 0; i1 <= 2; ++i1) ap[2] = ap[2] + ax1[i1] * dvol * __ldg(&e3[goff(g, i1 + i, j2, k2)]);
        }
      }
    }
    // field_charge_multiply
    double q = (double)slot_charge(sl);
#pragma unroll
    for (int c = 0; c < 6; ++c) ap[c] = q * ap[c];
    if (a.initial) {
      double alp0 = a.dth * a.lfact;
      double efp[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) efp[c] = -alp0 * ap[c];
      double gam2 = 1. + (pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2]);
      double gam_inv = 1. / sqrt(gam2);
      double vp[3] = {gam_inv * pp[0], gam_inv * pp[1], gam_inv * pp[2]};
      pp[0] = pp[0] + efp[0] + vp[1] * efp[5] - vp[2] * efp[4];
      pp[1] = pp[1] + efp[1] + vp[2] * efp[3] - vp[0] * efp[5];
      pp[2] = pp[2] + efp[2] + vp[0] * efp[4] - vp[1] * efp[3];
    }
    // lpf_momenta_and_positions, 3D
    double alp = a.dth * a.lfact;
    double efp[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) efp[c] = alp * ap[c];
    double vp[3] = {pp[0] + efp[0], pp[1] + efp[1], pp[2] + efp[2]};
    double bb[3] = {efp[3], efp[4], efp[5]};
    double gam02 = 1. + (vp[0] * vp[0] + vp[1] * vp[1] + vp[2] * vp[2]);
    double b2v = bb[0] * bb[0] + bb[1] * bb[1] + bb[2] * bb[2];
    double bv = bb[0] * vp[0] + bb[1] * vp[1] + bb[2] * vp[2];
    gam02 = gam02 - b2v;
    double gam2 = 0.5 * (gam02 + sqrt(gam02 * gam02 + 4. * (b2v + bv * bv)));
    double gam = sqrt(gam2);
    double vph[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) vph[c] = gam2 * vp[c] + bb[c] * bv;
    vph[0] = vph[0] + gam * (vp[1] * bb[2] - vp[2] * bb[1]);
    vph[1] = vph[1] + gam * (vp[2] * bb[0] - vp[0] * bb[2]);
    vph[2] = vph[2] + gam * (vp[0] * bb[1] - vp[1] * bb[0]);
#pragma unroll
    for (int c = 0; c < 3; ++c) vph[c] = vph[c] / (b2v + gam2);
    double pn[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) pn[c] = 2. * vph[c] - pp[c];
    gam2 = 1. + (pn[0] * pn[0] + pn[1] * pn[1] + pn[2] * pn[2]);
    double dtg = a.dt / sqrt(gam2);
    double xnew = x + dtg * pn[0];
    double ynew = y + dtg * pn[1];
    double znew = z + dtg * pn[2];
    if (a.vdt > 0.) xnew = xnew - a.vdt;  // comoving frame (boris_push.f90:161-166)
    a.px[n] = pn[0];
    a.py[n] = pn[1];
    a.pz[n] = pn[2];
    a.x[n] = xnew;
    a.y[n] = ynew;
    a.z[n] = znew;
    if (!(pn[0] == pn[0] && pn[1] == pn[1] && pn[2] == pn[2])) raise_err(a.err, AGPU_EBIT_NONFINITE);
    // cell_part_dist(.false.): keep gmin < x <= gmax along x, y, z
    bool keep = (xnew > a.gxmin && xnew <= a.gxmax) && (ynew > a.gymin && ynew <= a.gymax) &&
                (znew > a.gzmin && znew <= a.gzmax);
    if (!keep) {
      a.flag[n] = 1;
      atomicAdd(a.removed, 1ull);
      if (!emigrant(a, xnew, ynew, znew)) continue;
    }
    double xn[3] = {a.dx_inv * (xnew - a.xmn), ly(a, ynew), lz(a, znew)};
    float wght = (float)slot_charge(sl) * slot_wgh(sl);
    if (SHAPE != AGPU_SHAPE_CUBIC && a.iform == 2) {
      ncdef3d<SERIAL>(g, a.jc, xn, xo, pn, wght, dtg);
      continue;
    }
    const bool dep_ok = (SHAPE == AGPU_SHAPE_CUBIC) ? esirkepov_cubic64<SERIAL>(g, a.jc, xn, xo, wght, 3)
                                                   : esirkepov3d<SERIAL>(g, a.jc, xn, xo, wght);
    if (!dep_ok) raise_err(a.err, AGPU_EBIT_INDEX);
  }
}

template <bool SERIAL, int SHAPE>
__global__ void __launch_bounds__(256) k64_push_dep_2d(PushArgs64 a) {
  const Geo g = a.g;
  const double* __restrict__ ex = a.ebf;
  long long stride = SERIAL ? 1 : (long long)gridDim.x * blockDim.x;
  long long first = SERIAL ? 0 : blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (SERIAL && (blockIdx.x != 0 || threadIdx.x != 0)) return;
  for (long long n = first; n < a.np; n += stride) {
    double x = a.x[n], y = a.y[n];
    double pp1 = a.px[n], pp2 = a.py[n];
    uint64_t sl = dbits(a.slot[n]);
    double xl = a.dx_inv * (x - a.xmn);
    double yl = ly(a, y);
    double ap1 = 0., ap2 = 0., ap3 = 0.;
    if (SHAPE == AGPU_SHAPE_CUBIC) {
      double apc[6];
      const double xl2[2] = {xl, yl};
      if (!gather_cubic64(g, ex, xl2, 2, apc)) {
        raise_err(a.err, AGPU_EBIT_INDEX);
        atomicAdd(a.removed, 1ull);  // outside the box: the compaction drops it
        continue;
      }
      ap1 = apc[0];
      ap2 = apc[1];
      ap3 = apc[2];
    } else {
      double ax1[3], axh[2], ay1[3], ayh[2];
      int i = qlh64(xl, ax1, axh);
      int j = qlh64(yl, ay1, ayh);
      if (i < 2 || i > g.n1p - 3 || j < 2 || j > g.n2p - 3) {
        raise_err(a.err, AGPU_EBIT_INDEX);
        atomicAdd(a.removed, 1ull);  // outside the box: the compaction drops it
        continue;
      }
      int ih = i, jh = j;
      const double* e1 = ex;
      const double* e2 = ex + g.ncell;
      const double* b3 = ex + 2 * g.ncell;
  #pragma unroll
      for (int j1 = 0; j1 <= 2; ++j1) {
        int j2 = j + j1;
        double dvol = ay1[j1];
  #pragma unroll
        for (int i1 = 0; i1 <= 1; ++i1) {
          double dvol1 = axh[i1] * dvol;
          ap1 = ap1 + dvol1 * __ldg(&e1[goff(g, i1 + ih, j2, 1)]);
        }
      }
  #pragma unroll
      for (int j1 = 0; j1 <= 1; ++j1) {
        int j2 = jh + j1;
        double dvol = ayh[j1];
  #pragma unroll
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol1 = ax1[i1] * dvol;
          ap2 = ap2 + dvol1 * __ldg(&e2[goff(g, i + i1, j2, 1)]);
        }
  #pragma unroll
        for (int i1 = 0; i1 <= 1; ++i1) {
          double dvol1 = axh[i1] * dvol;
          ap3 = ap3 + dvol1 * __ldg(&b3[goff(g, i1 + ih, j2, 1)]);
        }
      }
    }
    double q = (double)slot_charge(sl);
    ap1 = q * ap1;
    ap2 = q * ap2;
    ap3 = q * ap3;
    if (a.initial) {
      double alp0 = a.dth * a.lfact;
      double efp1 = -alp0 * ap1, efp2 = -alp0 * ap2, efp3 = -alp0 * ap3;
      double gam2 = 1. + (pp1 * pp1 + pp2 * pp2);
      double gam_inv = 1. / sqrt(gam2);
      double vp1 = pp1 * gam_inv, vp2 = pp2 * gam_inv;
      pp1 = pp1 + efp1 + vp2 * efp3;
      pp2 = pp2 + efp2 - vp1 * efp3;
    }
    double alp = a.dth * a.lfact;
    double efp1 = alp * ap1, efp2 = alp * ap2, efp3 = alp * ap3;
    double vp1 = pp1 + efp1, vp2 = pp2 + efp2, vp3 = efp3;
    double gam02 = 1. + (vp1 * vp1 + vp2 * vp2);
    double b2 = vp3 * vp3;
    gam02 = gam02 - b2;
    double gam2 = 0.5 * (gam02 + sqrt(gam02 * gam02 + 4. * b2));
    double gam = sqrt(gam2);
    double vph1 = gam2 * vp1 + gam * vp2 * vp3;
    double vph2 = gam2 * vp2 - gam * vp1 * vp3;
    vph1 = vph1 / (gam2 + b2);
    vph2 = vph2 / (gam2 + b2);
    double pn1 = 2. * vph1 - pp1;
    double pn2 = 2. * vph2 - pp2;
    gam2 = 1. + (pn1 * pn1 + pn2 * pn2);
    double dtg = a.dt / sqrt(gam2);
    double xnew = x + dtg * pn1;
    double ynew = y + dtg * pn2;
    if (a.vdt > 0.) xnew = xnew - a.vdt;  // comoving frame (boris_push.f90:161-166)
    a.px[n] = pn1;
    a.py[n] = pn2;
    a.x[n] = xnew;
    a.y[n] = ynew;
    if (!(pn1 == pn1 && pn2 == pn2)) raise_err(a.err, AGPU_EBIT_NONFINITE);
    bool keep = (xnew > a.gxmin && xnew <= a.gxmax) && (ynew > a.gymin && ynew <= a.gymax);
    if (!keep) {
      a.flag[n] = 1;
      atomicAdd(a.removed, 1ull);
      if (!emigrant(a, xnew, ynew, 0.)) continue;
    }
    float wght = (float)slot_charge(sl) * slot_wgh(sl);
    if (SHAPE != AGPU_SHAPE_CUBIC && a.iform == 2) {
      ncdef2d<SERIAL>(g, a.jc, a.dx_inv * (xnew - a.xmn), ly(a, ynew), xl, yl, pn1, pn2, wght, dtg);
      continue;
    }
    bool dep_ok;
    if (SHAPE == AGPU_SHAPE_CUBIC) {
      const double xn2[2] = {a.dx_inv * (xnew - a.xmn), ly(a, ynew)}, xo2[2] = {xl, yl};
      dep_ok = esirkepov_cubic64<SERIAL>(g, a.jc, xn2, xo2, wght, 2);
    } else {
      dep_ok = esirkepov2d<SERIAL>(g, a.jc, a.dx_inv * (xnew - a.xmn), ly(a, ynew), xl, yl, wght);
    }
    if (!dep_ok) raise_err(a.err, AGPU_EBIT_INDEX);
  }
}

void push_deposit64(const PushArgs64& a, cudaStream_t st, int sms, bool serial) {
  if (a.np <= 0) return;
  int block = 256;
  int grid = serial ? 1 : grid_for(a.np, block, sms, 8);
  const bool cubic = a.shape == AGPU_SHAPE_CUBIC;
  if (a.g.ndim == 3) {
    if (serial)
      cubic ? k64_push_dep_3d<true, 1><<<1, 32, 0, st>>>(a) : k64_push_dep_3d<true, 0><<<1, 32, 0, st>>>(a);
    else
      cubic ? k64_push_dep_3d<false, 1><<<grid, block, 0, st>>>(a) : k64_push_dep_3d<false, 0><<<grid, block, 0, st>>>(a);
  } else {
    if (serial)
      cubic ? k64_push_dep_2d<true, 1><<<1, 32, 0, st>>>(a) : k64_push_dep_2d<true, 0><<<1, 32, 0, st>>>(a);
    else
      cubic ? k64_push_dep_2d<false, 1><<<grid, block, 0, st>>>(a) : k64_push_dep_2d<false, 0><<<grid, block, 0, st>>>(a);
  }
}

void jfold64(const Dev64& d, cudaStream_t st, int sms) { jfold_t<double>(d.jc, d.g, st, sms); }

void yee64(const Dev64& d, const YeeC& c, cudaStream_t st, int sms, const XAdv* xa, YeeHook* hk) {
  yee_t<double>(d.ebf, d.jc, (const double*)nullptr, d.g, c, st, sms, xa, hk);
}
void yee64_fused(const double* fin, double* fout, const double* jc, const Geo& g, const YeeC& c, cudaStream_t st) {
  yee_fused_t<double>(fin, fout, jc, (const double*)nullptr, g, c, st);
}

// ============================================================================
// A15: set_ion_efield (grid_part_connect.f90:288-410): |E|^2 on each ion with
// the qqh shapes.
// ============================================================================
__global__ void k64_ion_efield(IonArgs64 a) {
  const Geo g = a.g;
  const double* E1 = a.ebf;
  const double* E2 = a.ebf + g.ncell;
  const double* E3 = a.ebf + 2 * g.ncell;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < a.np; n += (long long)gridDim.x * blockDim.x) {
    double ef_sqr = 0.;
    double xl = a.dx_inv * (a.x[n] - a.xmn);
    double yl = a.dy_inv * (a.y[n] - a.ymn);
    double ax1[3], axh[3], ay1[3], ayh[3], az1[3], azh[3];
    int i, ih, j, jh, k = 1, kh = 1;
    qqh64(xl, ax1, axh, &i, &ih);
    qqh64(yl, ay1, ayh, &j, &jh);
    int imin = min(i, ih), jmin = min(j, jh);
    if (imin < 1 || max(i, ih) > g.n1p - 2 || jmin < 1 || max(j, jh) > g.n2p - 2) {
      raise_err(a.err, AGPU_EBIT_INDEX);
      a.ef2[n] = 0.0;
      continue;
    }
    if (g.ndim == 2) {
      for (int jp1 = 0; jp1 <= 2; ++jp1) {
        double dvol = ay1[jp1];
        for (int ip1 = 0; ip1 <= 2; ++ip1) {
          double e = E1[goff(g, ih + ip1, j + jp1, 1)];
          ef_sqr = ef_sqr + axh[ip1] * dvol * e * e;
        }
      }
      for (int jp1 = 0; jp1 <= 2; ++jp1) {
        double dvol = ayh[jp1];
        for (int ip1 = 0; ip1 <= 2; ++ip1) {
          double e = E2[goff(g, i + ip1, jh + jp1, 1)];
          ef_sqr = ef_sqr + ax1[ip1] * dvol * e * e;
        }
      }
    } else {
      double zl = a.dz_inv * (a.z[n] - a.zmn);
      qqh64(zl, az1, azh, &k, &kh);
      if (min(k, kh) < 1 || max(k, kh) > g.n3p - 2) {
        raise_err(a.err, AGPU_EBIT_INDEX);
        a.ef2[n] = 0.0;
        continue;
      }
      for (int kp1 = 0; kp1 <= 2; ++kp1) {
        int kp2 = k + kp1;
        for (int jp1 = 0; jp1 <= 2; ++jp1) {
          double dvol = ay1[jp1] * az1[kp1];
          for (int ip1 = 0; ip1 <= 2; ++ip1) {
            double e = E1[goff(g, ip1 + ih, j + jp1, kp2)];
            ef_sqr = ef_sqr + axh[ip1] * dvol * e * e;
          }
        }
        for (int jp1 = 0; jp1 <= 2; ++jp1) {
          double dvol = ayh[jp1] * az1[kp1];
          for (int ip1 = 0; ip1 <= 2; ++ip1) {
            double e = E2[goff(g, i + ip1, jh + jp1, kp2)];
            ef_sqr = ef_sqr + ax1[ip1] * dvol * e * e;
          }
        }
      }
      for (int kp1 = 0; kp1 <= 2; ++kp1) {
        int kp2 = kh + kp1;
        for (int jp1 = 0; jp1 <= 2; ++jp1) {
          double dvol = ay1[jp1] * azh[kp1];
          for (int ip1 = 0; ip1 <= 2; ++ip1) {
            double e = E3[goff(g, ip1 + i, j + jp1, kp2)];
            ef_sqr = ef_sqr + ax1[ip1] * dvol * e * e;
          }
        }
      }
    }
    a.ef2[n] = ef_sqr;
  }
}

// A16: part_ionize, ionz_lev = 1 (ionize.f90:390-450) with the nk index of
// ionization_cycle (ionize.f90:496-506): flag[n] = 1 when ion n ionizes.
__global__ void k64_ionize(IonArgs64 a) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < a.np; n += (long long)gridDim.x * blockDim.x) {
    double ef2 = a.ef2[n];
    int nk = 0;
    if (ef2 > 0.) {
      double ef = sqrt(ef2);
      nk = (int)llround(a.de_inv * ef);
    }
    if (nk > a.n_ge + 1) {
      raise_err(a.err, AGPU_EBIT_IONZ_INDEX);
      nk = a.n_ge + 1;
    }
    uint64_t sl = dbits(a.slot[n]);
    int z0 = slot_charge(sl);
    double pr = ionz_draw(a.seed, n, a.iter, a.ic);
    double thr = (z0 >= 0 && z0 <= a.zmax) ? a.wtab[(long long)nk + (long long)(a.n_ge + 2) * z0] : 0.0;
    int fl = 0;
    if (pr < thr) {
      a.slot[n] = bitsd(make_slot(z0 + 1, slot_part_ind(sl), slot_wgh(sl)));
      fl = 1;
    }
    a.flag[n] = fl;
  }
}

}  // namespace agpu
