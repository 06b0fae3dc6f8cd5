// agpu_tile64.cu — tiled gather + push + deposit of the plain FP64 form.
//
// Same tiling as agpu_tile32.cu (one CTA per tile, fields staged in shared
// memory), with the reference's FP64 statement order: the gather reads the
// same field values from shared memory as the untiled kernel does from
// global memory, so positions and momenta stay bit-identical to the oracle;
// only the order of the current sums changes.  The FP64 currents go straight
// to global memory with FP64 atomics (resolved in L2), which on sm_100a is
// faster than FP64 atomics in shared memory; the shared accumulation variant
// (SHJ) is kept for comparison.  Compiled with -fmad=false.
#include "agpu_bin.cuh"
#include "agpu_common.cuh"
#include "agpu_tile.h"

namespace agpu {

namespace {

__device__ __forceinline__ int qlh_d(double xp, double ax[3], double axh[2]) {
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
__device__ __forceinline__ int qden_d(double xp, double ax[3]) {
  double xx = 3.0 + xp;
  int i = (int)(xx + 0.5);
  double sx = xx - (double)i;
  double sx2 = sx * sx;
  ax[1] = 0.75 - sx2;
  ax[2] = 0.5 * (0.25 + sx2 + sx);
  ax[0] = 1. - ax[1] - ax[2];
  return i;
}
__device__ __forceinline__ void esirk_d(const double a0[3], const double a1[3], int ih, double axh[5], double cur[5]) {
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    int m = q - ih;
    axh[q] = (m == 0) ? a1[0] : (m == 1) ? a1[1] : (m == 2) ? a1[2] : 0.;
  }
  cur[0] = -axh[0];
  cur[1] = cur[0] + a0[0] - axh[1];
  cur[2] = cur[1] + a0[1] - axh[2];
  cur[3] = cur[2] + a0[2] - axh[3];
  cur[4] = cur[3] - axh[4];
}

}  // namespace

template <int NDIM, int TX, int TY, int TZ, bool SHJ>
__global__ void __launch_bounds__(256, 2) k64_tile(TileArgs64 a) {
  constexpr int FX = TX + 2, FY = TY + 2, FZ = (NDIM == 3) ? TZ + 2 : 1;
  constexpr int JX = TX + 4, JY = TY + 4, JZ = (NDIM == 3) ? TZ + 4 : 1;
  constexpr int FV = FX * FY * FZ, JV = JX * JY * JZ;
  constexpr int NF = (NDIM == 3) ? 6 : 3, NC = (NDIM == 3) ? 3 : 2;
  extern __shared__ double smd[];
  double* sF = smd;
  double* sJ = smd + NF * FV;  // used when SHJ: currents summed in shared memory

  const Geo g = a.g;
  const int t = blockIdx.x;
  const int beg = a.tstart[t * a.t.nsub], end = a.tstart[(t + 1) * a.t.nsub];
  if (beg >= end) return;
  const int tx = t % a.t.ntx, ty = (t / a.t.ntx) % a.t.nty, tz = t / (a.t.ntx * a.t.nty);
  const int i0t = 3 + tx * TX, j0t = 3 + ty * TY, k0t = (NDIM == 3) ? 3 + tz * TZ : 1;
  // current accumulation at local tile coordinates (node i0t-2+lx, ...)
  auto addJ = [&](int c, int lx, int ly, int lz, double v) {
    if (SHJ)
      atomicAdd(&sJ[c * JV + lx + JX * (ly + JY * lz)], v);
    else
      atomicAdd(&a.jc[g.ncell * c + goff(g, i0t - 2 + lx, j0t - 2 + ly, (NDIM == 3) ? k0t - 2 + lz : 1)], v);
  };
  for (int e = threadIdx.x; e < NF * FV; e += blockDim.x) {
    int c = e / FV, r = e - c * FV;
    int lx = r % FX, ly = (r / FX) % FY, lz = r / (FX * FY);
    int gi = i0t - 1 + lx, gj = j0t - 1 + ly, gk = (NDIM == 3) ? k0t - 1 + lz : 1;
    double v = 0.;
    if (gi >= 1 && gi <= g.n1p && gj >= 1 && gj <= g.n2p && gk >= 1 && gk <= g.n3p)
      v = __ldg(&a.ebf[g.ncell * c + goff(g, gi, gj, gk)]);
    sF[e] = v;
  }
  if (SHJ)
    for (int e = threadIdx.x; e < NC * JV; e += blockDim.x) sJ[e] = 0.;
  __syncthreads();

  for (int q = beg + threadIdx.x; q < end; q += blockDim.x) {
    const int p = a.perm[q];
    const double x = a.x[p], y = a.y[p], z = (NDIM == 3) ? a.z[p] : 0.;
    double pp[3] = {a.px[p], a.py[p], (NDIM == 3) ? a.pz[p] : 0.};
    const uint64_t sl = dbits(a.slot[p]);
    const double xo[3] = {a.dx_inv * (x - a.xmn), a.dy_inv * (y - a.ymn), (NDIM == 3) ? a.dz_inv * (z - a.zmn) : 0.};
    double ax1[3], axh[2], ay1[3], ayh[2], az1[3], azh[2];
    const int i = qlh_d(xo[0], ax1, axh);
    const int j = qlh_d(xo[1], ay1, ayh);
    const int k = (NDIM == 3) ? qlh_d(xo[2], az1, azh) : 0;
    const int fx = i - (i0t - 1), fy = j - (j0t - 1), fz = (NDIM == 3) ? k - (k0t - 1) : 0;
    if ((unsigned)fx >= (unsigned)TX || (unsigned)fy >= (unsigned)TY || (NDIM == 3 && (unsigned)fz >= (unsigned)TZ)) {
      raise_err(a.err, AGPU_EBIT_INDEX);
      a.key[p] = a.t.nkeys;
      hist_add(a.hist, a.t.nkeys);
      continue;
    }
    double ap[6] = {0, 0, 0, 0, 0, 0};
    if (NDIM == 3) {
      const double* e1 = sF;
      const double* e2 = sF + FV;
      const double* e3 = sF + 2 * FV;
      const double* b1 = sF + 3 * FV;
      const double* b2 = sF + 4 * FV;
      const double* b3 = sF + 5 * FV;
      // set_part3d_hcell_acc loop order (grid_part_connect.f90:222-281)
#pragma unroll
      for (int k1 = 0; k1 <= 2; ++k1) {
#pragma unroll
        for (int j1 = 0; j1 <= 2; ++j1) {
          double dvol = ay1[j1] * az1[k1];
          int o = fx + FX * (fy + j1 + FY * (fz + k1));
#pragma unroll
          for (int i1 = 0; i1 <= 1; ++i1) ap[0] = ap[0] + axh[i1] * dvol * e1[o + i1];
        }
#pragma unroll
        for (int j1 = 0; j1 <= 1; ++j1) {
          double dvol = ayh[j1] * az1[k1];
          int o = fx + FX * (fy + j1 + FY * (fz + k1));
#pragma unroll
          for (int i1 = 0; i1 <= 2; ++i1) ap[1] = ap[1] + ax1[i1] * dvol * e2[o + i1];
#pragma unroll
          for (int i1 = 0; i1 <= 1; ++i1) ap[5] = ap[5] + axh[i1] * dvol * b3[o + i1];
        }
      }
#pragma unroll
      for (int k1 = 0; k1 <= 1; ++k1) {
#pragma unroll
        for (int j1 = 0; j1 <= 1; ++j1) {
          double dvol = ayh[j1] * azh[k1];
          int o = fx + FX * (fy + j1 + FY * (fz + k1));
#pragma unroll
          for (int i1 = 0; i1 <= 2; ++i1) ap[3] = ap[3] + ax1[i1] * dvol * b1[o + i1];
        }
#pragma unroll
        for (int j1 = 0; j1 <= 2; ++j1) {
          double dvol = ay1[j1] * azh[k1];
          int o = fx + FX * (fy + j1 + FY * (fz + k1));
#pragma unroll
          for (int i1 = 0; i1 <= 1; ++i1) ap[4] = ap[4] + axh[i1] * dvol * b2[o + i1];
#pragma unroll
          for (int i1 = 0; i1 <= 2; ++i1) ap[2] = ap[2] + ax1[i1] * dvol * e3[o + i1];
        }
      }
    } else {
      const double* e1 = sF;
      const double* e2 = sF + FV;
      const double* b3 = sF + 2 * FV;
      // set_part2d_hcell_acc (grid_part_connect.f90:110-138)
#pragma unroll
      for (int j1 = 0; j1 <= 2; ++j1) {
        double dvol = ay1[j1];
        int o = fx + FX * (fy + j1);
#pragma unroll
        for (int i1 = 0; i1 <= 1; ++i1) {
          double dvol1 = axh[i1] * dvol;
          ap[0] = ap[0] + dvol1 * e1[o + i1];
        }
      }
#pragma unroll
      for (int j1 = 0; j1 <= 1; ++j1) {
        double dvol = ayh[j1];
        int o = fx + FX * (fy + j1);
#pragma unroll
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol1 = ax1[i1] * dvol;
          ap[1] = ap[1] + dvol1 * e2[o + i1];
        }
#pragma unroll
        for (int i1 = 0; i1 <= 1; ++i1) {
          double dvol1 = axh[i1] * dvol;
          ap[2] = ap[2] + dvol1 * b3[o + i1];
        }
      }
    }
    const double qc = (double)slot_charge(sl);
    double xnew, ynew, znew = 0.;
    if (NDIM == 3) {
#pragma unroll
      for (int c = 0; c < 6; ++c) ap[c] = qc * ap[c];
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
#pragma unroll
      for (int c = 0; c < 3; ++c) pp[c] = 2. * vph[c] - pp[c];
      gam2 = 1. + (pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2]);
      double dtg = a.dt / sqrt(gam2);
      xnew = x + dtg * pp[0];
      ynew = y + dtg * pp[1];
      znew = z + dtg * pp[2];
      a.pz[p] = pp[2];
      a.z[p] = znew;
    } else {
      ap[0] = qc * ap[0];
      ap[1] = qc * ap[1];
      ap[2] = qc * ap[2];
      if (a.initial) {
        double alp0 = a.dth * a.lfact;
        double efp1 = -alp0 * ap[0], efp2 = -alp0 * ap[1], efp3 = -alp0 * ap[2];
        double gam2 = 1. + (pp[0] * pp[0] + pp[1] * pp[1]);
        double gam_inv = 1. / sqrt(gam2);
        double vp1 = pp[0] * gam_inv, vp2 = pp[1] * gam_inv;
        pp[0] = pp[0] + efp1 + vp2 * efp3;
        pp[1] = pp[1] + efp2 - vp1 * efp3;
      }
      double alp = a.dth * a.lfact;
      double efp1 = alp * ap[0], efp2 = alp * ap[1], efp3 = alp * ap[2];
      double vp1 = pp[0] + efp1, vp2 = pp[1] + efp2, vp3 = efp3;
      double gam02 = 1. + (vp1 * vp1 + vp2 * vp2);
      double b2 = vp3 * vp3;
      gam02 = gam02 - b2;
      double gam2 = 0.5 * (gam02 + sqrt(gam02 * gam02 + 4. * b2));
      double gam = sqrt(gam2);
      double vph1 = gam2 * vp1 + gam * vp2 * vp3;
      double vph2 = gam2 * vp2 - gam * vp1 * vp3;
      vph1 = vph1 / (gam2 + b2);
      vph2 = vph2 / (gam2 + b2);
      double pn1 = 2. * vph1 - pp[0];
      double pn2 = 2. * vph2 - pp[1];
      pp[0] = pn1;
      pp[1] = pn2;
      gam2 = 1. + (pn1 * pn1 + pn2 * pn2);
      double dtg = a.dt / sqrt(gam2);
      xnew = x + dtg * pn1;
      ynew = y + dtg * pn2;
    }
    // comoving frame (boris_push.f90:161-166)
    if (a.vdt > 0.) xnew = xnew - a.vdt;
    a.px[p] = pp[0];
    a.py[p] = pp[1];
    a.x[p] = xnew;
    a.y[p] = ynew;
    if (!(pp[0] == pp[0] && pp[1] == pp[1] && pp[2] == pp[2])) raise_err(a.err, AGPU_EBIT_NONFINITE);
    bool keep = (xnew > a.gxmin && xnew <= a.gxmax) && (ynew > a.gymin && ynew <= a.gymax);
    if (NDIM == 3) keep = keep && (znew > a.gzmin && znew <= a.gzmax);
    const double xn[3] = {a.dx_inv * (xnew - a.xmn), a.dy_inv * (ynew - a.ymn),
                          (NDIM == 3) ? a.dz_inv * (znew - a.zmn) : 0.};
    double ax0[3], ay0[3], az0[3], axn[3], ayn[3], azn[3];
    const int ii0 = qden_d(xo[0], ax0), jj0 = qden_d(xo[1], ay0);
    const int in = qden_d(xn[0], axn), jn = qden_d(xn[1], ayn);
    const int kk0 = (NDIM == 3) ? qden_d(xo[2], az0) : 0;
    const int kn = (NDIM == 3) ? qden_d(xn[2], azn) : 0;
    const int ih = in - ii0 + 1, jh = jn - jj0 + 1, kh = (NDIM == 3) ? kn - kk0 + 1 : 1;
    if (keep && ((unsigned)ih > 2u || (unsigned)jh > 2u || (unsigned)kh > 2u)) {
      raise_err(a.err, AGPU_EBIT_INDEX);  // moved more than one cell: no window slot
      keep = false;
    }
    const int oct = offset_octant((float)(3.0 + xn[0] - (double)in), (float)(3.0 + xn[1] - (double)jn),
                                  (NDIM == 3) ? (float)(3.0 + xn[2] - (double)kn) : 0.f, NDIM);
    int nkey = keep ? tile_key(a.t, in, jn, (NDIM == 3) ? kn : 3, oct) : a.t.nkeys;
    a.key[p] = nkey;
    hist_add(a.hist, nkey);
    if (!keep) continue;
    // Esirkepov (grid_part_connect.f90:979-1059, 1168-1334) into shared
    const double w = (double)((float)slot_charge(sl) * slot_wgh(sl));
    double sxh[5], cx[5], syh[5], cy[5];
    esirk_d(ax0, axn, ih, sxh, cx);
    esirk_d(ay0, ayn, jh, syh, cy);
    const int x0 = ih < 1 ? ih : 1, x1 = (ih + 2) > 3 ? ih + 2 : 3;
    const int y0 = jh < 1 ? jh : 1, y1 = (jh + 2) > 3 ? jh + 2 : 3;
    const int lx = ii0 - i0t, ly = jj0 - j0t;  // J slot 0 = node ii0-2
    if (NDIM == 2) {
      sxh[1] = sxh[1] + ax0[0];
      sxh[2] = sxh[2] + ax0[1];
      sxh[3] = sxh[3] + ax0[2];
#pragma unroll
      for (int u = 0; u < 5; ++u) cx[u] = w * cx[u];
#pragma unroll
      for (int u = 0; u < 5; ++u) cy[u] = w * cy[u];
      syh[1] = syh[1] + ay0[0];
      syh[2] = syh[2] + ay0[1];
      syh[3] = syh[3] + ay0[2];
      for (int j1 = y0; j1 <= y1; ++j1)
        for (int i1 = x0; i1 <= x1; ++i1) addJ(0, lx + i1, ly + j1, 0, syh[j1] * cx[i1]);
      for (int j1 = y0; j1 <= y1; ++j1)
        for (int i1 = x0; i1 <= x1; ++i1) addJ(1, lx + i1, ly + j1, 0, sxh[i1] * cy[j1]);
    } else {
      // regrouped onto the 5-slot windows (slot 0 = old node - 2): old-plane
      // and new-plane terms of the reference loops land on the same slots
      double axh0[5], axh1[5], ayh0[5], ayh1[5], szh[5], cz[5], b1[5];
#pragma unroll
      for (int u = 0; u < 5; ++u) cx[u] = w * cx[u];
#pragma unroll
      for (int u = 0; u < 5; ++u) {
        axh0[u] = 0.5 * sxh[u];
        axh1[u] = sxh[u];
      }
#pragma unroll
      for (int i1 = 1; i1 <= 3; ++i1) {
        axh0[i1] = axh0[i1] + ax0[i1 - 1];
        axh1[i1] = axh1[i1] + 0.5 * ax0[i1 - 1];
      }
#pragma unroll
      for (int u = 0; u < 5; ++u) cy[u] = w * cy[u];
#pragma unroll
      for (int u = 0; u < 5; ++u) {
        ayh0[u] = 0.5 * syh[u];
        ayh1[u] = syh[u];
        int m = u - jh;
        b1[u] = (m == 0) ? ayn[0] : (m == 1) ? ayn[1] : (m == 2) ? ayn[2] : 0.;
      }
#pragma unroll
      for (int i1 = 1; i1 <= 3; ++i1) {
        ayh0[i1] = ayh0[i1] + ay0[i1 - 1];
        ayh1[i1] = ayh1[i1] + 0.5 * ay0[i1 - 1];
      }
      esirk_d(az0, azn, kh, szh, cz);
      const int z0 = kh < 1 ? kh : 1, z1 = (kh + 2) > 3 ? kh + 2 : 3;
      const int lzb = kk0 - k0t;  // local z of slot 0 (node kk0-2)
      for (int ws = z0; ws <= z1; ++ws) {
        const int m0 = ws - 1, m1 = ws - kh;
        const double A0 = (m0 == 0) ? az0[0] : (m0 == 1) ? az0[1] : (m0 == 2) ? az0[2] : 0.;
        const double A1 = (m1 == 0) ? azn[0] : (m1 == 1) ? azn[1] : (m1 == 2) ? azn[2] : 0.;
        const double czw = w * ((ws == 0) ? cz[0] : (ws == 1) ? cz[1] : (ws == 2) ? cz[2] : (ws == 3) ? cz[3] : cz[4]);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          if (v < y0 || v > y1) continue;
          const double wyv = ayh0[v] * A0 + ayh1[v] * A1;
          const double b0v = (v >= 1 && v <= 3) ? ay0[v - 1] : 0.;
#pragma unroll
          for (int u = 0; u < 5; ++u) {
            if (u < x0 || u > x1) continue;
            addJ(0, lx + u, ly + v, lzb + ws, wyv * cx[u]);
            addJ(1, lx + u, ly + v, lzb + ws, cy[v] * (axh0[u] * A0 + axh1[u] * A1));
            addJ(2, lx + u, ly + v, lzb + ws, czw * (axh0[u] * b0v + axh1[u] * b1[v]));
          }
        }
      }
    }
  }
  if (!SHJ) return;
  __syncthreads();
  for (int e = threadIdx.x; e < NC * JV; e += blockDim.x) {
    double v = sJ[e];
    if (v == 0.) continue;
    int c = e / JV, rr = e - c * JV;
    int lx = rr % JX, ly = (rr / JX) % JY, lz = rr / (JX * JY);
    int gi = i0t - 2 + lx, gj = j0t - 2 + ly, gk = (NDIM == 3) ? k0t - 2 + lz : 1;
    if (gi < 1 || gi > g.n1p || gj < 1 || gj > g.n2p || gk < 1 || gk > g.n3p) {
      raise_err(a.err, AGPU_EBIT_INDEX);
      continue;
    }
    atomicAdd(&a.jc[g.ncell * c + goff(g, gi, gj, gk)], v);
  }
}

size_t tile64_smem(int ndim, int tx, int ty, int tz) {
  if (ndim == 3) return sizeof(double) * (6 * (tx + 2) * (ty + 2) * (tz + 2) + 3 * (tx + 4) * (ty + 4) * (tz + 4));
  return sizeof(double) * (3 * (tx + 2) * (ty + 2) + 2 * (tx + 4) * (ty + 4));
}

void tile_push64(const TileArgs64& a, cudaStream_t st) {
  if (a.t.ntiles <= 0) return;
  if (a.g.ndim == 3) {
    size_t sm = sizeof(double) * 6 * (TILE3_X + 2) * (TILE3_Y + 2) * (TILE3_Z + 2);
    auto k = k64_tile<3, TILE3_X, TILE3_Y, TILE3_Z, false>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<a.t.ntiles, 256, sm, st>>>(a);
  } else {
    size_t sm = sizeof(double) * 3 * (TILE2_X + 2) * (TILE2_Y + 2);
    auto k = k64_tile<2, TILE2_X, TILE2_Y, 1, false>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<a.t.ntiles, 256, sm, st>>>(a);
  }
}

// Histogram of the next binning: tile bins zero, the removed bin keeps the
// particles already removed (they are not revisited by any tile).
// Next histogram zeroed, the dead bin seeded with the records already dead;
// with `pushed` set, the alive count of this push (tstart[nkeys]) is added
// to it (the deferred-count mode keeps the push count on the device).
__global__ void k_hist_reset(int* hist, const int* tstart, int nkeys, int np, int first, unsigned long long* pushed) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= nkeys; b += gridDim.x * blockDim.x) {
    hist[b] = (b == nkeys && !first) ? (np - tstart[nkeys]) : 0;
    if (b == nkeys && pushed) *pushed += (unsigned long long)tstart[nkeys];
  }
}
void hist_reset(int* hist, const int* tstart, const TileGeo& t, long long np, bool first, unsigned long long* pushed,
                cudaStream_t st) {
  k_hist_reset<<<(t.nkeys + 256) / 256, 256, 0, st>>>(hist, tstart, t.nkeys, (int)np, first ? 1 : 0, pushed);
}

TileGeo make_tiles(const Geo& g, int nx, int ny, int nz) {
  TileGeo t;
  if (g.ndim == 3) {
    t.tx = TILE3_X;
    t.ty = TILE3_Y;
    t.tz = TILE3_Z;
  } else {
    t.tx = TILE2_X;
    t.ty = TILE2_Y;
    t.tz = 1;
  }
  // alive nodes 3 .. n+3 (n+1 nodes per axis)
  t.ntx = (nx + 1 + t.tx - 1) / t.tx;
  t.nty = (ny + 1 + t.ty - 1) / t.ty;
  t.ntz = (g.ndim == 3) ? (nz + 1 + t.tz - 1) / t.tz : 1;
  t.ntiles = t.ntx * t.nty * t.ntz;
  t.nq = (g.ndim == 3) ? 8 : 4;
  t.nsub = t.ty * t.tz * t.nq;
  t.nkeys = t.ntiles * t.nsub;
  return t;
}

}  // namespace agpu
