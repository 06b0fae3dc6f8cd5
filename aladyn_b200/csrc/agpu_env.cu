// agpu_env.cu — the envelope cycle (the reference's Env_cycle,
// src/ALaDyn.F90:111-130) on sm_100a, FP64 form.
//
// env_lpf2_evolve (src/dynamics/env_evolve_in_time.f90:196-361) for species
// 0 in a fixed frame: the laser is the complex envelope A of its vector
// potential, advanced by the explicit Maxwell envelope solver
// (env_maxw_solve), and the particles feel the wake fields plus the
// ponderomotive force of F = |A|^2/2.  Compiled with -fmad=false: every
// expression keeps the reference's statement order, so given the same
// inputs the grid arrays and particles equal the CPU restatement bit for bit
// (the density and current sums in the deterministic, serial mode).  Grid
// kernels run one thread per node; the particle kernels one thread per
// particle with global-memory stencils (the envelope route runs on the PWFA
// set-up, not on the tiled benchmark path).  The stretch factors
// loc_yg/loc_zg(:,3:4) of a uniform grid are 1 and are left out (x * 1 == x
// exactly).
#include "agpu_env.h"
#include "agpu_fp64_dep.cuh"

namespace agpu {
namespace {

// Interior node t of an nx*ny*nz box starting at (ix1, jy1, kz1).
__device__ __forceinline__ void interior_node(const Geo& g, long long t, int& i, int& j, int& k) {
  const int nx = g.ix2 - g.ix1 + 1, ny = g.jy2 - g.jy1 + 1;
  i = g.ix1 + (int)(t % nx);
  j = g.jy1 + (int)((t / nx) % ny);
  k = g.kz1 + (int)(t / ((long long)nx * ny));
}
__host__ __device__ __forceinline__ long long interior_count(const Geo& g) {
  return (long long)(g.ix2 - g.ix1 + 1) * (g.jy2 - g.jy1 + 1) * (g.kz2 - g.kz1 + 1);
}
#define GRID_LOOP(t, total) \
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (total); t += (long long)gridDim.x * blockDim.x)

// env_amp_prepare (env_evolve_in_time.f90:129-158): av(1) = |A^n|^2 / 2.
__global__ void k_env_amp(const double* __restrict__ env, double* __restrict__ av, Geo g) {
  const long long total = interior_count(g);
  GRID_LOOP(t, total) {
    int i, j, k;
    interior_node(g, t, i, j, k);
    const long long o = goff(g, i, j, k);
    const double e1 = env[o], e2 = env[g.ncell + o];
    av[o] = 0.5 * (e1 * e1 + e2 * e2);
  }
}

// env_grad (src/fields/grid_fields.f90:426-586), der_ord < 4, one rank:
// av(2) = D_x F at i+1/2, av(3) = D_y F at j+1/2, av(4) = D_z F at k+1/2,
// one-sided at ix2 and jy2; in 3D the edge planes kz1, kz2 first extrapolate
// F into the ghost planes kz1-1, kz2+1 (written to av(1)).
__global__ void k_env_grad(double* av, Geo g, double dxi, double dyi, double dzi) {
  const long long total = interior_count(g);
  double* gx = av + g.ncell;
  double* gy = av + 2 * g.ncell;
  double* gz = av + 3 * g.ncell;
  GRID_LOOP(t, total) {
    int i, j, k;
    interior_node(g, t, i, j, k);
    const long long o = goff(g, i, j, k);
    const double f0 = av[o];
    if (i == g.ix2)
      gx[o] = dxi * (2. * av[o - 1] - 3. * av[o - 2] + av[o - 3]);
    else
      gx[o] = dxi * (av[o + 1] - f0);
    const long long sy = g.n1p;
    if (j == g.jy2)
      gy[o] = dyi * (2. * f0 - 3. * av[o - sy] + av[o - 2 * sy]);
    else
      gy[o] = dyi * (av[o + sy] - f0);
    if (g.ndim == 3) {
      const long long sz = (long long)g.n1p * g.n2p;
      if (k == g.kz2) {
        const double gh = 2. * f0 - av[o - sz];
        av[o + sz] = gh;
        gz[o] = dzi * (gh - f0);
      } else if (k == g.kz1) {
        av[o - sz] = 2. * f0 - av[o + sz];
        gz[o] = dzi * (av[o + sz] - f0);
      } else {
        gz[o] = dzi * (av[o + sz] - f0);
      }
    }
  }
}

__device__ __forceinline__ bool in_stencil(int lo, int n) { return lo >= 1 && lo + 2 <= n; }

// The atomic-mode Esirkepov deposit of one 3D move: the terms of
// esirkepov3d (grid_part_connect.f90:1168-1334) with every window loop
// unrolled over its five slots, so the window arrays stay in registers, and
// where the old-plane and new-plane terms of a component land on the same
// node (the particle keeps its z node for Jx and Jy, its y node for Jz) the
// two terms are summed before one atomic add instead of two.  The sums then
// round differently from the reference's two adds (the serial mode keeps
// esirkepov3d); the atomic mode's sum order is not the reference's anyway.
__device__ __forceinline__ bool esirkepov3d_sum(const Geo& g, double* jc, const double xn[3], const double xo[3],
                                                float wght) {
  double ax0[3], ay0[3], az0[3], ax1[3], ay1[3], az1[3];
  double axh[5], ayh[5], azh[5], axh0[5], axh1[5], ayh0[5], ayh1[5];
  double currx[5], curry[5], currz[5];
  const int ii0 = qden64(xo[0], ax0), jj0 = qden64(xo[1], ay0), kk0 = qden64(xo[2], az0);
  const int i = qden64(xn[0], ax1), j = qden64(xn[1], ay1), k = qden64(xn[2], az1);
  if ((unsigned)(i - ii0 + 1) > 2u || (unsigned)(j - jj0 + 1) > 2u || (unsigned)(k - kk0 + 1) > 2u) return false;
  const double w = (double)wght;
  const int ih = i - ii0 + 1, jh = j - jj0 + 1, kh = k - kk0 + 1;
  esirk_1d(ax0, ax1, ih, axh, currx);
  esirk_1d(ay0, ay1, jh, ayh, curry);
  esirk_1d(az0, az1, kh, azh, currz);
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    currx[q] = w * currx[q];
    curry[q] = w * curry[q];
    currz[q] = w * currz[q];
    axh0[q] = 0.5 * axh[q];
    axh1[q] = axh[q];
    ayh0[q] = 0.5 * ayh[q];
    ayh1[q] = ayh[q];
  }
#pragma unroll
  for (int q = 1; q <= 3; ++q) {
    axh0[q] = axh0[q] + ax0[q - 1];
    axh1[q] = axh1[q] + 0.5 * ax0[q - 1];
    ayh0[q] = ayh0[q] + ay0[q - 1];
    ayh1[q] = ayh1[q] + 0.5 * ay0[q - 1];
  }
  const int x0 = ih < 1 ? ih : 1, x1 = (ih + 2) > 3 ? ih + 2 : 3;
  const int y0 = jh < 1 ? jh : 1, y1 = (jh + 2) > 3 ? jh + 2 : 3;
  const int z0 = kh < 1 ? kh : 1, z1 = (kh + 2) > 3 ? kh + 2 : 3;
  const long long sy = g.n1p, sz = (long long)g.n1p * g.n2p;
  // slot (i1, j1, k1) of the window of component c sits at base + i1 + sy j1 + sz k1
  const long long bx0 = goff(g, ii0 - 2, jj0 - 2, kk0 - 1), bx1 = goff(g, ii0 - 2, jj0 - 2, k - 1);
  const long long bz0 = goff(g, ii0 - 2, jj0 - 1, kk0 - 2), bz1 = goff(g, ii0 - 2, j - 1, kk0 - 2);
  const bool samek = (k == kk0), samej = (j == jj0);
  double* jx = jc;
  double* jy = jc + g.ncell;
  double* jz = jc + 2 * g.ncell;
#pragma unroll
  for (int k1 = 0; k1 <= 2; ++k1)
#pragma unroll
    for (int j1 = 0; j1 < 5; ++j1) {
      if (j1 < y0 || j1 > y1) continue;
      const double dvol = ayh0[j1] * az0[k1], dvolh = ayh1[j1] * az1[k1];
      const double cvol = curry[j1] * az0[k1], cvolh = curry[j1] * az1[k1];
#pragma unroll
      for (int i1 = 0; i1 < 5; ++i1) {
        if (i1 < x0 || i1 > x1) continue;
        const long long o0 = bx0 + i1 + sy * j1 + sz * k1, o1 = bx1 + i1 + sy * j1 + sz * k1;
        const double ax = dvol * currx[i1], bx = dvolh * currx[i1];
        const double ay = axh0[i1] * cvol, by = axh1[i1] * cvolh;
        if (samek) {
          atomicAdd(&jx[o0], ax + bx);
          atomicAdd(&jy[o0], ay + by);
        } else {
          atomicAdd(&jx[o0], ax);
          atomicAdd(&jx[o1], bx);
          atomicAdd(&jy[o0], ay);
          atomicAdd(&jy[o1], by);
        }
      }
    }
#pragma unroll
  for (int k1 = 0; k1 < 5; ++k1) {
    if (k1 < z0 || k1 > z1) continue;
#pragma unroll
    for (int j1 = 0; j1 <= 2; ++j1) {
      const double dvol = ay0[j1] * currz[k1], dvolh = ay1[j1] * currz[k1];
#pragma unroll
      for (int i1 = 0; i1 < 5; ++i1) {
        if (i1 < x0 || i1 > x1) continue;
        const long long o0 = bz0 + i1 + sy * j1 + sz * k1, o1 = bz1 + i1 + sy * j1 + sz * k1;
        const double az = axh0[i1] * dvol, bz = axh1[i1] * dvolh;
        if (samej) {
          atomicAdd(&jz[o0], az + bz);
        } else {
          atomicAdd(&jz[o0], az);
          atomicAdd(&jz[o1], bz);
        }
      }
    }
  }
  return true;
}

// set_env_acc (src/particles/grid_part_connect.f90:414-615) ->
// lpf_env_momenta (src/dynamics/boris_push.f90:170-223) ->
// set_env_density (grid_part_connect.f90:884-952), per particle: the qqh
// gather at x^n of (E, B), F and grad F, the approximate gamma, the Boris
// rotation p^{n-1/2} -> p^{n+1/2}, and the qden deposit of wgh/gam_new into
// den.  The reference runs the three as separate sweeps with ebfp as
// scratch; per particle the arithmetic is identical.
template <bool SERIAL, int NDIM>
__global__ void __launch_bounds__(256) k_env_acc(EnvArgs a) {
  const Geo g = a.g;
  const long long stride = SERIAL ? 1 : (long long)gridDim.x * blockDim.x;
  const long long first = SERIAL ? 0 : blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (SERIAL && (blockIdx.x != 0 || threadIdx.x != 0)) return;
  const double dth = 0.5 * a.dt;
  const double alp = 0.5 * a.dt * a.lfact;
  const double* __restrict__ ef = a.ebf;
  const double* __restrict__ av = a.av;
  const long long nc = g.ncell;
  for (long long n = first; n < a.np; n += stride) {
    const uint64_t sl = dbits(a.slot[n]);
    const double charge = (double)slot_charge(sl);
    const double wgh = (double)slot_wgh(sl);
    double ax1[3], axh1[3], ay1[3], ayh1[3], az1[3], azh1[3];
    int i, ih, j, jh, k = 1, kh = 1;
    const double xl = a.dx_inv * (a.x[n] - a.xmn);
    const double yl = a.dy_inv * (a.y[n] - a.ymn);
    qqh64(xl, ax1, axh1, &i, &ih);
    qqh64(yl, ay1, ayh1, &j, &jh);
    if (NDIM == 2) {
      if (!in_stencil(i, g.n1p) || !in_stencil(ih, g.n1p) || !in_stencil(j, g.n2p) || !in_stencil(jh, g.n2p)) {
        raise_err(a.err, AGPU_EBIT_INDEX);
        continue;
      }
      const double u1 = a.px[n], u2 = a.py[n];
      double ap[7] = {0, 0, 0, 0, 0, 0, 0};
      for (int j1 = 0; j1 <= 2; ++j1) {
        const int j2 = j + j1;
        const double dvol = ay1[j1];
        for (int i1 = 0; i1 <= 2; ++i1) ap[6] = ap[6] + ax1[i1] * dvol * av[goff(g, i + i1, j2, 1)];
        for (int i1 = 0; i1 <= 2; ++i1) {
          const double dvol1 = dvol * axh1[i1];
          const long long o = goff(g, ih + i1, j2, 1);
          ap[1] = ap[1] + dvol1 * ef[o];
          ap[4] = ap[4] + dvol1 * av[nc + o];
        }
      }
      for (int j1 = 0; j1 <= 2; ++j1) {
        const int j2 = jh + j1;
        const double dvol = ayh1[j1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          const double dvol1 = dvol * ax1[i1];
          const long long o = goff(g, i + i1, j2, 1);
          ap[2] = ap[2] + dvol1 * ef[nc + o];
          ap[5] = ap[5] + dvol1 * av[2 * nc + o];
        }
        for (int i1 = 0; i1 <= 2; ++i1) ap[3] = ap[3] + axh1[i1] * dvol * ef[2 * nc + goff(g, ih + i1, j2, 1)];
      }
      const double gam2 = 1. + u1 * u1 + u2 * u2 + ap[6];
      for (int c = 1; c <= 3; ++c) ap[c] = charge * ap[c];
      for (int c = 4; c <= 5; ++c) ap[c] = 0.5 * charge * charge * ap[c];
      const double aa1 = dth * (ap[1] * u1 + ap[2] * u2);
      const double b1 = dth * (ap[4] * u1 + ap[5] * u2);
      const double gam = sqrt(gam2);
      const double dgam = (aa1 * gam - b1) / gam2;
      const double gam_inv = (gam - dgam) / gam2;
      for (int c = 3; c <= 5; ++c) ap[c] = ap[c] * gam_inv;
      const double f1 = ap[1] - ap[4], f2 = ap[2] - ap[5], f3 = ap[3];
      const double wghp = wgh * gam_inv;
      // lpf_env_momenta, curr_ndim = 2
      const double efp1 = alp * f1, efp2 = alp * f2, efp3 = alp * f3;
      const double vp1 = u1 + efp1, vp2 = u2 + efp2;
      const double bb1 = efp3;
      const double b2 = 1. + bb1 * bb1;
      double vph1 = vp1 + vp2 * bb1;
      double vph2 = vp2 - vp1 * bb1;
      vph1 = vph1 / b2;
      vph2 = vph2 / b2;
      const double pn1 = 2. * vph1 - u1, pn2 = 2. * vph2 - u2;
      a.px[n] = pn1;
      a.py[n] = pn2;
      if (!(pn1 == pn1 && pn2 == pn2)) raise_err(a.err, AGPU_EBIT_NONFINITE);
      // set_env_density: qden at x^n, nodes i-1..i+1 of the qden index
      double dx1[3], dy1[3];
      const int iq = qden64(xl, dx1) - 1, jq = qden64(yl, dy1) - 1;
      for (int j1 = 0; j1 <= 2; ++j1) {
        const double dvol = dy1[j1] * wghp;
        for (int i1 = 0; i1 <= 2; ++i1) {
          const double dvol1 = dvol * dx1[i1];
          jadd<SERIAL>(&a.den[goff(g, i1 + iq, jq + j1, 1)], dvol1);
        }
      }
      continue;
    }
    const double zl = a.dz_inv * (a.z[n] - a.zmn);
    qqh64(zl, az1, azh1, &k, &kh);
    if (!in_stencil(i, g.n1p) || !in_stencil(ih, g.n1p) || !in_stencil(j, g.n2p) || !in_stencil(jh, g.n2p) ||
        !in_stencil(k, g.n3p) || !in_stencil(kh, g.n3p)) {
      raise_err(a.err, AGPU_EBIT_INDEX);
      continue;
    }
    const double u1 = a.px[n], u2 = a.py[n], u3 = a.pz[n];
    double ap[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int k1 = 0; k1 <= 2; ++k1) {
      const int k2 = k + k1;
      for (int j1 = 0; j1 <= 2; ++j1) {
        const int j2 = j + j1;
        const double dvol = ay1[j1] * az1[k1];
        for (int i1 = 0; i1 <= 2; ++i1) ap[10] = ap[10] + ax1[i1] * dvol * av[goff(g, i1 + i, j2, k2)];
        for (int i1 = 0; i1 <= 2; ++i1) {
          const double dvol1 = dvol * axh1[i1];
          const long long o = goff(g, i1 + ih, j2, k2);
          ap[1] = ap[1] + dvol1 * ef[o];
          ap[7] = ap[7] + dvol1 * av[nc + o];
        }
      }
      for (int j1 = 0; j1 <= 2; ++j1) {
        const int j2 = jh + j1;
        const double dvol = ayh1[j1] * az1[k1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          const double dvol1 = dvol * ax1[i1];
          const long long o = goff(g, i + i1, j2, k2);
          ap[2] = ap[2] + dvol1 * ef[nc + o];
          ap[8] = ap[8] + dvol1 * av[2 * nc + o];
        }
        for (int i1 = 0; i1 <= 2; ++i1) ap[6] = ap[6] + axh1[i1] * dvol * ef[5 * nc + goff(g, i1 + ih, j2, k2)];
      }
    }
    for (int k1 = 0; k1 <= 2; ++k1) {
      const int k2 = kh + k1;
      for (int j1 = 0; j1 <= 2; ++j1) {
        const int j2 = jh + j1;
        const double dvol = ayh1[j1] * azh1[k1];
        for (int i1 = 0; i1 <= 2; ++i1) ap[4] = ap[4] + ax1[i1] * dvol * ef[3 * nc + goff(g, i1 + i, j2, k2)];
      }
      for (int j1 = 0; j1 <= 2; ++j1) {
        const int j2 = j + j1;
        const double dvol = ay1[j1] * azh1[k1];
        for (int i1 = 0; i1 <= 2; ++i1) ap[5] = ap[5] + axh1[i1] * dvol * ef[4 * nc + goff(g, ih + i1, j2, k2)];
        for (int i1 = 0; i1 <= 2; ++i1) {
          const double dvol1 = dvol * ax1[i1];
          const long long o = goff(g, i1 + i, j2, k2);
          ap[3] = ap[3] + dvol1 * ef[2 * nc + o];
          ap[9] = ap[9] + dvol1 * av[3 * nc + o];
        }
      }
    }
    const double gam2 = 1. + u1 * u1 + u2 * u2 + u3 * u3 + ap[10];
    for (int c = 1; c <= 6; ++c) ap[c] = charge * ap[c];
    for (int c = 7; c <= 9; ++c) ap[c] = 0.5 * charge * charge * ap[c];
    const double aa1 = dth * (ap[1] * u1 + ap[2] * u2 + ap[3] * u3);
    const double b1 = dth * (ap[7] * u1 + ap[8] * u2 + ap[9] * u3);
    const double gam = sqrt(gam2);
    const double dgam = (aa1 * gam - b1) / gam2;
    const double gam_inv = (gam - dgam) / gam2;
    for (int c = 4; c <= 9; ++c) ap[c] = ap[c] * gam_inv;
    double fp[6];
    for (int c = 0; c < 3; ++c) fp[c] = ap[c + 1] - ap[c + 7];
    for (int c = 3; c < 6; ++c) fp[c] = ap[c + 1];
    const double wghp = wgh * gam_inv;
    // lpf_env_momenta, curr_ndim = 3
    const double pp[3] = {u1, u2, u3};
    double efp[6], vp[3], bb[3], vph[3];
    for (int c = 0; c < 6; ++c) efp[c] = alp * fp[c];
    for (int c = 0; c < 3; ++c) vp[c] = efp[c] + pp[c];
    for (int c = 0; c < 3; ++c) bb[c] = efp[3 + c];
    const double b2 = 1. + (bb[0] * bb[0] + bb[1] * bb[1] + bb[2] * bb[2]);
    const double bv = bb[0] * vp[0] + bb[1] * vp[1] + bb[2] * vp[2];
    vph[0] = vp[0] + vp[1] * bb[2] - vp[2] * bb[1] + bb[0] * bv;
    vph[1] = vp[1] + vp[2] * bb[0] - vp[0] * bb[2] + bb[1] * bv;
    vph[2] = vp[2] + vp[0] * bb[1] - vp[1] * bb[0] + bb[2] * bv;
    for (int c = 0; c < 3; ++c) vph[c] = vph[c] / b2;
    double pn[3];
    for (int c = 0; c < 3; ++c) pn[c] = 2. * vph[c] - pp[c];
    a.px[n] = pn[0];
    a.py[n] = pn[1];
    a.pz[n] = pn[2];
    if (!(pn[0] == pn[0] && pn[1] == pn[1] && pn[2] == pn[2])) raise_err(a.err, AGPU_EBIT_NONFINITE);
    // set_env_density
    double dx1[3], dy1[3], dz1[3];
    const int iq = qden64(xl, dx1) - 1, jq = qden64(yl, dy1) - 1, kq = qden64(zl, dz1) - 1;
    for (int k1 = 0; k1 <= 2; ++k1)
      for (int j1 = 0; j1 <= 2; ++j1) {
        const double dvol = dy1[j1] * dz1[k1] * wghp;
        for (int i1 = 0; i1 <= 2; ++i1) {
          const double dvol1 = dvol * dx1[i1];
          jadd<SERIAL>(&a.den[goff(g, i1 + iq, jq + j1, kq + k1)], dvol1);
        }
      }
  }
}

// den_zyxbd (src/parallel/mpi_curr_interface.f90, from env_den_collect,
// env_evolve_in_time.f90:37-78), one rank: the first ghost layer is added to
// the second interior layer, which is then copied onto the edge node; z,
// then y, then x; the ghosts keep their values.
__global__ void k_den_fold_z(double* d, Geo g) {
  const int nx = g.ix2 - g.ix1 + 1, ny = g.jy2 - g.jy1 + 1;
  const long long sz = (long long)g.n1p * g.n2p;
  GRID_LOOP(t, (long long)nx * ny) {
    const int ix = g.ix1 + (int)(t % nx), iy = g.jy1 + (int)(t / nx);
    const long long b = goff(g, ix, iy, 1);
    const int k1 = g.kz1, k2 = g.kz2;
    double* c = d + b;
    c[k1 * sz] = c[k1 * sz] + c[(k1 - 2) * sz];
    c[(k1 - 1) * sz] = c[k1 * sz];
    c[(k2 - 2) * sz] = c[(k2 - 2) * sz] + c[k2 * sz];
    c[(k2 - 1) * sz] = c[(k2 - 2) * sz];
  }
}
__global__ void k_den_fold_y(double* d, Geo g, int iby) {
  const int nx = g.ix2 - g.ix1 + 1, nz = g.kz2 - g.kz1 + 1;
  const long long sy = g.n1p;
  GRID_LOOP(t, (long long)nx * nz) {
    const int ix = g.ix1 + (int)(t % nx), k = g.kz1 + (int)(t / nx);
    double* c = d + goff(g, ix, 1, k);  // row j = 1
    const int j1 = g.jy1, j2 = g.jy2;
    if (iby == 0 || iby == 1) {
      c[j1 * sy] = c[j1 * sy] + c[(j1 - 2) * sy];
      if (iby == 0)
        c[(j1 - 1) * sy] = c[j1 * sy];
      else
        c[(j1 - 2) * sy] = 0.0;
    }
    if (iby < 2) {
      c[(j2 - 2) * sy] = c[(j2 - 2) * sy] + c[j2 * sy];
      c[(j2 - 1) * sy] = c[(j2 - 2) * sy];
    }
  }
}
__global__ void k_den_fold_x(double* d, Geo g) {
  const int ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  GRID_LOOP(t, (long long)ny * nz) {
    const int iy = g.jy1 + (int)(t % ny), k = g.kz1 + (int)(t / ny);
    double* c = d + goff(g, 1, iy, k);  // column i = 1
    const int i1 = g.ix1, i2 = g.ix2;
    c[i1] = c[i1] + c[i1 - 2];
    c[i1 - 1] = c[i1];
    c[i2 - 2] = c[i2 - 2] + c[i2];
    c[i2 - 1] = c[i2 - 2];
  }
}

// env_bds(env, 2, 2) (src/fields/grid_fields.f90:864-1067) on env(1:2), in
// the reference's three passes: the x ghosts copy the edge node (a one-term
// DOT_PRODUCT summed from zero), then the y ghosts over the widened x range
// and the z ghosts over the widened x and y ranges take the quadratic
// extrapolation (e2 - e1) - 2 e1 + 3 e0 of the first three interior planes
// (alpha = 1 on a uniform grid); ib = 1 is the parity copy.
__global__ void k_env_bds_x(double* env, Geo g, int ibx) {
  const int ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  GRID_LOOP(t, 2LL * ny * nz) {
    const int c = (int)(t % 2);
    const int j = g.jy1 + (int)((t / 2) % ny), k = g.kz1 + (int)(t / (2LL * ny));
    double* e = env + c * g.ncell + goff(g, 1, j, k) - 1;  // e[i] = env(i, j, k, c+1)
    const int i1 = g.ix1, i2 = g.ix2;
    const double par = (c == 0) ? -1.0 : 1.0;
    for (int point = 2; point >= 1; --point) {
      const int i = i1 - point;
      e[i] = (ibx == 1) ? par * e[2 * i1 - i] : 0.0 + 1.0 * e[i1];
    }
    for (int point = 1; point <= 2; ++point) {
      const int i = i2 + point;
      e[i] = (ibx == 1) ? par * e[2 * i2 - i] : 0.0 + 1.0 * e[i2];
    }
  }
}
__global__ void k_env_bds_y(double* env, Geo g, int iby) {
  const int nxw = g.ix2 - g.ix1 + 5, nz = g.kz2 - g.kz1 + 1;
  const long long sy = g.n1p;
  GRID_LOOP(t, 2LL * nxw * nz) {
    const int c = (int)(t % 2);
    const int i = g.ix1 - 2 + (int)((t / 2) % nxw), k = g.kz1 + (int)(t / (2LL * nxw));
    double* e = env + c * g.ncell + goff(g, i, 1, k) - sy;  // e[j * sy] = env(i, j, k, c+1)
    const int j1 = g.jy1, j2 = g.jy2;
    const double par = (c == 0) ? 1.0 : -1.0;
    const double lo = (e[(j1 + 2) * sy] - e[(j1 + 1) * sy]) - 2 * e[(j1 + 1) * sy] + 3 * e[j1 * sy];
    const double hi = (e[(j2 - 2) * sy] - e[(j2 - 1) * sy]) - 2 * e[(j2 - 1) * sy] + 3 * e[j2 * sy];
    for (int j = j1 - 2; j <= j1 - 1; ++j) e[j * sy] = (iby == 1) ? par * e[(2 * j1 - j) * sy] : lo;
    for (int j = j2 + 1; j <= j2 + 2; ++j) e[j * sy] = (iby == 1) ? par * e[(2 * j2 - j) * sy] : hi;
  }
}
__global__ void k_env_bds_z(double* env, Geo g, int ibz) {
  const int nxw = g.ix2 - g.ix1 + 5, nyw = g.jy2 - g.jy1 + 5;
  const long long sz = (long long)g.n1p * g.n2p;
  GRID_LOOP(t, 2LL * nxw * nyw) {
    const int c = (int)(t % 2);
    const int i = g.ix1 - 2 + (int)((t / 2) % nxw), j = g.jy1 - 2 + (int)(t / (2LL * nxw));
    double* e = env + c * g.ncell + goff(g, i, j, 1) - sz;  // e[k * sz] = env(i, j, k, c+1)
    const int k1 = g.kz1, k2 = g.kz2;
    const double lo = (e[(k1 + 2) * sz] - e[(k1 + 1) * sz]) - 2 * e[(k1 + 1) * sz] + 3 * e[k1 * sz];
    const double hi = (e[(k2 - 2) * sz] - e[(k2 - 1) * sz]) - 2 * e[(k2 - 1) * sz] + 3 * e[k2 * sz];
    for (int k = k1 - 2; k <= k1 - 1; ++k) e[k * sz] = (ibz == 1) ? e[(2 * k1 - k) * sz] : lo;
    for (int k = k2 + 1; k <= k2 + 2; ++k) e[k * sz] = (ibz == 1) ? e[(2 * k2 - k) * sz] : hi;
  }
}

struct SolveC {
  double ompe, dt2, kfact, dx1_inv, aph1, aph2, dx4_1, dx4_2, dy2, dz2;
  int der3;
};

// advance_lpf_envelope (src/dynamics/curr_and_fields_util.f90:262-299),
// ib = 2: the source -ompe chi A (chi = av(3)), potential_lapl
// (src/fields/grid_fields.f90:1356-1403) and pp_lapl (326-424) for
// S(A) = [D^2 - omp^2 chi] A, first_ader, and the second-order time
// combination of env_maxw_solve (588-694) into av(1:2).  The reference adds
// the terms in passes over the whole grid; each pass only reads env and the
// node's own sum, so one thread per node adds them in the same order.
__global__ void k_env_solve(const double* __restrict__ env, double* av, Geo g, SolveC s) {
  const long long total = interior_count(g);
  const long long nc = g.ncell, sy = g.n1p, sz = (long long)g.n1p * g.n2p;
  const double* E1 = env;
  const double* E2 = env + nc;
  const double* E3 = env + 2 * nc;
  const double* E4 = env + 3 * nc;
  GRID_LOOP(t, total) {
    int i, j, k;
    interior_node(g, t, i, j, k);
    const long long o = goff(g, i, j, k);
    const double a3 = av[2 * nc + o];
    double c[2];
    c[0] = -s.ompe * a3 * E1[o];
    c[1] = -s.ompe * a3 * E2[o];
    for (int q = 0; q < 2; ++q) {
      const double* e = env + q * nc;
      c[q] = c[q] + s.dx4_1 * (e[o + 1] + e[o - 1] - 2. * e[o]);
    }
    if (s.der3)
      for (int q = 0; q < 2; ++q) {
        const double* e = env + q * nc;
        c[q] = c[q] + s.dx4_2 * (e[o + 2] + e[o - 2] - 2. * e[o]);
      }
    for (int q = 0; q < 2; ++q) {
      const double* e = env + q * nc;
      c[q] = c[q] + s.dy2 * ((e[o + sy] - e[o]) - (e[o] - e[o - sy]));
    }
    if (g.ndim == 3)
      for (int q = 0; q < 2; ++q) {
        const double* e = env + q * nc;
        c[q] = c[q] + s.dz2 * ((e[o + sz] - e[o]) - (e[o] - e[o - sz]));
      }
    if (!s.der3) {
      c[0] = c[0] - s.dx1_inv * (E2[o + 1] - E2[o - 1]);
      c[1] = c[1] + s.dx1_inv * (E1[o + 1] - E1[o - 1]);
    } else {
      c[0] = c[0] - s.aph1 * (E2[o + 1] - E2[o - 1]) - s.aph2 * (E2[o + 2] - E2[o - 2]);
      c[1] = c[1] + s.aph1 * (E1[o + 1] - E1[o - 1]) + s.aph2 * (E1[o + 2] - E1[o - 2]);
    }
    av[o] = s.dt2 * c[0] + 2. * E1[o] - E3[o] + s.kfact * E4[o];
    av[nc + o] = s.dt2 * c[1] + 2. * E2[o] - E4[o] - s.kfact * E3[o];
  }
}

// The update of env_maxw_solve (A^{n-1} <- A^n, A^n <- A^{n+1}) and
// env_fields_average (env_evolve_in_time.f90:103-127):
// av(1) = ((A^{n+1} + A^n)/2)^2 / 2 = (1/8)((e1 + e3)^2 + (e2 + e4)^2).
__global__ void k_env_update(double* env, double* av, Geo g, double k2_fact, double kfact) {
  const long long total = interior_count(g);
  const long long nc = g.ncell;
  const double frac = 1.0 / 8.;
  GRID_LOOP(t, total) {
    int i, j, k;
    interior_node(g, t, i, j, k);
    const long long o = goff(g, i, j, k);
    const double e1 = env[o], e2 = env[nc + o];
    const double c1 = av[o], c2 = av[nc + o];
    env[2 * nc + o] = e1;
    env[3 * nc + o] = e2;
    const double n1 = k2_fact * (c1 - kfact * c2);
    const double n2 = k2_fact * (c2 + kfact * c1);
    env[o] = n1;
    env[nc + o] = n2;
    const double sa = n1 + e1, sb = n2 + e2;
    av[o] = frac * (sa * sa + sb * sb);
  }
}

// env_lpf_solve (src/fields/grid_fields.f90:696-858) with ib = 0, the
// comoving frame's reduced envelope solver, in three passes.  Pass 1, per
// node: the source -ompe chi A, the transverse Laplacian (pp_lapl) added,
// and on the row j = jy1 alone the factor -dt (the reference's
// `do j = jy1, jy1`).
__global__ void k_env_lpf_src(const double* __restrict__ env, double* av, Geo g, double ompe, double dy2, double dz2,
                              double dtl) {
  const long long total = interior_count(g);
  const long long nc = g.ncell, sy = g.n1p, sz = (long long)g.n1p * g.n2p;
  GRID_LOOP(t, total) {
    int i, j, k;
    interior_node(g, t, i, j, k);
    const long long o = goff(g, i, j, k);
    const double a3 = av[2 * nc + o];
    double c[2];
    c[0] = -ompe * a3 * env[o];
    c[1] = -ompe * a3 * env[nc + o];
    for (int q = 0; q < 2; ++q) {
      const double* e = env + q * nc;
      c[q] = c[q] + dy2 * ((e[o + sy] - e[o]) - (e[o] - e[o - sy]));
    }
    if (g.ndim == 3)
      for (int q = 0; q < 2; ++q) {
        const double* e = env + q * nc;
        c[q] = c[q] + dz2 * ((e[o + sz] - e[o]) - (e[o] - e[o - sz]));
      }
    if (j == g.jy1) {
      c[0] = -dtl * c[0];
      c[1] = -dtl * c[1];
    }
    av[o] = c[0];
    av[nc + o] = c[1];
  }
}
// Pass 2: first_der's centred x-derivative with the om0 rotation into
// (t1, t2); the row's x ghosts of av(1:2), which the reference leaves as
// they are, travel along so that pass 3 reads the same neighbours.
__global__ void k_env_lpf_der1(const double* __restrict__ av, double* t1, double* t2, Geo g, double om0, double dx1_inv) {
  const long long total = interior_count(g);
  const long long nc = g.ncell;
  GRID_LOOP(t, total) {
    int i, j, k;
    interior_node(g, t, i, j, k);
    const long long o = goff(g, i, j, k);
    const double* a1 = av;
    const double* a2 = av + nc;
    t1[o] = om0 * a2[o] + dx1_inv * (a1[o + 1] - a1[o - 1]);
    t2[o] = -om0 * a1[o] + dx1_inv * (a2[o + 1] - a2[o - 1]);
    if (i == g.ix1) {
      t1[o - 1] = a1[o - 1];
      t2[o - 1] = a2[o - 1];
    }
    if (i == g.ix2) {
      t1[o + 1] = a1[o + 1];
      t2[o + 1] = a2[o + 1];
    }
  }
}
// Pass 3: explicit_mat_inv's three-point inversion (u - dx2_norm D2 u) / om0^2,
// then A^{n+1} = A^{n-1} + u, the shift A^{n-1} <- A^n, A^n <- A^{n+1}, and
// env_fields_average's av(1) = (1/8)((A^{n+1} + A^n)^2) of the update.
__global__ void k_env_lpf_inv(double* env, double* av, const double* __restrict__ t1, const double* __restrict__ t2, Geo g,
                              double dx2_norm, double om2) {
  const long long total = interior_count(g);
  const long long nc = g.ncell;
  const double frac = 1.0 / 8.;
  GRID_LOOP(t, total) {
    int i, j, k;
    interior_node(g, t, i, j, k);
    const long long o = goff(g, i, j, k);
    double v[2];
    const double* tq[2] = {t1, t2};
    for (int q = 0; q < 2; ++q) {
      const double* u = tq[q];
      const double w = dx2_norm * (u[o + 1] - 2. * u[o] + u[o - 1]);
      v[q] = (u[o] - w) / om2;
    }
    const double e1 = env[o], e2 = env[nc + o];
    v[0] = v[0] + env[2 * nc + o];
    v[1] = v[1] + env[3 * nc + o];
    env[2 * nc + o] = e1;
    env[3 * nc + o] = e2;
    env[o] = v[0];
    env[nc + o] = v[1];
    av[nc + o] = v[1];
    const double sa = v[0] + e1, sb = v[1] + e2;
    av[o] = frac * (sa * sa + sb * sb);
  }
}

// set_env_grad_interp (grid_part_connect.f90:760-882) -> lpf_env_positions
// (src/dynamics/boris_push.f90:225-295, vbeam = 0) -> the box test of
// cell_part_dist(.false.) (mpi_part_interface.f90:467-523) -> Esirkepov
// deposit (grid_part_connect.f90:956-1334) of the particles that stay, from
// x^n to x^{n+1} with the packed weight (iform < 2).
template <bool SERIAL, int NDIM>
__global__ void __launch_bounds__(256) k_env_pos(EnvArgs a) {
  const Geo g = a.g;
  const long long stride = SERIAL ? 1 : (long long)gridDim.x * blockDim.x;
  const long long first = SERIAL ? 0 : blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (SERIAL && (blockIdx.x != 0 || threadIdx.x != 0)) return;
  const double dt_lp = a.dt;
  const double* __restrict__ av = a.av;
  const long long nc = g.ncell;
  for (long long n = first; n < a.np; n += stride) {
    double ax1[3], axh1[3], ay1[3], ayh1[3], az1[3], azh1[3];
    int i, ih, j, jh, k = 1, kh = 1;
    const double x = a.x[n], y = a.y[n];
    const double xl = a.dx_inv * (x - a.xmn);
    const double yl = a.dy_inv * (y - a.ymn);
    qqh64(xl, ax1, axh1, &i, &ih);
    qqh64(yl, ay1, ayh1, &j, &jh);
    const float wght = (float)slot_charge(dbits(a.slot[n])) * slot_wgh(dbits(a.slot[n]));
    if (NDIM == 2) {
      if (!in_stencil(i, g.n1p) || !in_stencil(ih, g.n1p) || !in_stencil(j, g.n2p) || !in_stencil(jh, g.n2p)) {
        raise_err(a.err, AGPU_EBIT_INDEX);
        a.flag[n] = 1;
        atomicAdd(a.removed, 1ull);
        continue;
      }
      double ap[4] = {0, 0, 0, 0};
      for (int j1 = 0; j1 <= 2; ++j1) {
        const int j2 = j + j1;
        const double dvol = ay1[j1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          const double dvol1 = dvol * axh1[i1];
          ap[1] = ap[1] + dvol1 * av[nc + goff(g, i1 + ih, j2, 1)];
          ap[3] = ap[3] + ax1[i1] * dvol * av[goff(g, i1 + i, j2, 1)];
        }
      }
      for (int j1 = 0; j1 <= 2; ++j1) {
        const int j2 = jh + j1;
        const double dvol = ayh1[j1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          const double dvol1 = dvol * ax1[i1];
          ap[2] = ap[2] + dvol1 * av[2 * nc + goff(g, i + i1, j2, 1)];
        }
      }
      const double pp1 = a.px[n], pp2 = a.py[n];
      const double gam2 = 1. + (pp1 * pp1 + pp2 * pp2) + ap[3];
      const double gam = sqrt(gam2);
      const double gam3 = gam2 * gam;
      const double b2 = 0.25 * (pp1 * ap[1] + pp2 * ap[2]);
      double gam_inv = 1. / gam;
      gam_inv = gam_inv * (1. - dt_lp * b2 / gam3);
      const double vp1 = dt_lp * gam_inv * pp1, vp2 = dt_lp * gam_inv * pp2;
      double xn = x + vp1;
      const double yn = y + vp2;
      if (a.vdt > 0.) xn = xn - a.vdt;  // comoving frame (boris_push.f90:288-294)
      a.x[n] = xn;
      a.y[n] = yn;
      const bool keep = (xn > a.gxmin && xn <= a.gxmax) && (yn > a.gymin && yn <= a.gymax);
      if (!keep) {
        a.flag[n] = 1;
        atomicAdd(a.removed, 1ull);
        continue;
      }
      if (a.iform == 2) {
        ncdef2d<SERIAL>(g, a.jc, a.dx_inv * (xn - a.xmn), a.dy_inv * (yn - a.ymn), xl, yl, pp1, pp2, wght,
                        dt_lp * gam_inv);
        continue;
      }
      if (!esirkepov2d<SERIAL>(g, a.jc, a.dx_inv * (xn - a.xmn), a.dy_inv * (yn - a.ymn), xl, yl, wght))
        raise_err(a.err, AGPU_EBIT_INDEX);
      continue;
    }
    const double z = a.z[n];
    const double zl = a.dz_inv * (z - a.zmn);
    qqh64(zl, az1, azh1, &k, &kh);
    if (!in_stencil(i, g.n1p) || !in_stencil(ih, g.n1p) || !in_stencil(j, g.n2p) || !in_stencil(jh, g.n2p) ||
        !in_stencil(k, g.n3p) || !in_stencil(kh, g.n3p)) {
      raise_err(a.err, AGPU_EBIT_INDEX);
      a.flag[n] = 1;
      atomicAdd(a.removed, 1ull);
      continue;
    }
    double ap[5] = {0, 0, 0, 0, 0};
    for (int k1 = 0; k1 <= 2; ++k1) {
      int k2 = k + k1;
      for (int j1 = 0; j1 <= 2; ++j1) {
        const int j2 = j + j1;
        const double dvol = ay1[j1] * az1[k1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          const double dvol1 = dvol * axh1[i1];
          ap[1] = ap[1] + dvol1 * av[nc + goff(g, i1 + ih, j2, k2)];
          ap[4] = ap[4] + ax1[i1] * dvol * av[goff(g, i1 + i, j2, k2)];
        }
      }
      for (int j1 = 0; j1 <= 2; ++j1) {
        const int j2 = jh + j1;
        const double dvol = ayh1[j1] * az1[k1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          const double dvol1 = dvol * ax1[i1];
          ap[2] = ap[2] + dvol1 * av[2 * nc + goff(g, i + i1, j2, k2)];
        }
      }
      k2 = kh + k1;
      for (int j1 = 0; j1 <= 2; ++j1) {
        const int j2 = j + j1;
        const double dvol = ay1[j1] * azh1[k1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          const double dvol1 = dvol * ax1[i1];
          ap[3] = ap[3] + dvol1 * av[3 * nc + goff(g, i + i1, j2, k2)];
        }
      }
    }
    const double pp[3] = {a.px[n], a.py[n], a.pz[n]};
    const double gam2 = 1. + (pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2]) + ap[4];
    const double gam = sqrt(gam2);
    const double gam3 = gam2 * gam;
    const double b2 = 0.25 * (pp[0] * ap[1] + pp[1] * ap[2] + pp[2] * ap[3]);
    double gam_inv = 1. / sqrt(gam2);
    gam_inv = gam_inv * (1. - dt_lp * b2 / gam3);
    double vp[3];
    for (int c = 0; c < 3; ++c) vp[c] = dt_lp * gam_inv * pp[c];
    double xn = x + vp[0];
    const double yn = y + vp[1], zn = z + vp[2];
    if (a.vdt > 0.) xn = xn - a.vdt;  // comoving frame (boris_push.f90:288-294)
    a.x[n] = xn;
    a.y[n] = yn;
    a.z[n] = zn;
    const bool keep =
        (xn > a.gxmin && xn <= a.gxmax) && (yn > a.gymin && yn <= a.gymax) && (zn > a.gzmin && zn <= a.gzmax);
    if (!keep) {
      a.flag[n] = 1;
      atomicAdd(a.removed, 1ull);
      continue;
    }
    const double xo[3] = {xl, yl, zl};
    const double xnl[3] = {a.dx_inv * (xn - a.xmn), a.dy_inv * (yn - a.ymn), a.dz_inv * (zn - a.zmn)};
    if (a.iform == 2) {
      ncdef3d<SERIAL>(g, a.jc, xnl, xo, pp, wght, dt_lp * gam_inv);
      continue;
    }
    const bool dep_ok = SERIAL ? esirkepov3d<true>(g, a.jc, xnl, xo, wght) : esirkepov3d_sum(g, a.jc, xnl, xo, wght);
    if (!dep_ok) raise_err(a.err, AGPU_EBIT_INDEX);
  }
}

// init_gprof_envelope_field / init_envelope_field
// (src/fields/init_grid_fields.f90:274-399 / 140-272): the pulse's A at
// t and t - dt added on the interior nodes.
__global__ void k_env_pulse(EnvPulseArgs a, double* env, Geo g) {
  const double pi = acos(-1.0);
  const double pih = 0.5 * acos(-1.0);
  const long long total = interior_count(g);
  const long long nc = g.ncell;
  GRID_LOOP(t, total) {
    int i, j, k;
    interior_node(g, t, i, j, k);
    const double zz = (a.ndim == 3) ? (a.zmn + a.dz * (double)(k - 3) - a.zcent) / a.wy : 0.0;
    const double yy = (a.ymn + a.dy * (double)(j - 3) - a.ycent) / a.wy;
    const double r2 = (a.ndim == 3) ? (yy * yy + zz * zz) : yy * yy;
    double xx = a.xmn + a.dx * (double)(i - 3);
    xx = xx - a.xf0;
    double phi0, phi1, phi, ar, ai, ampl1, ampl0;
    if (a.g_prof) {
      phi1 = (xx - a.t) / a.wx;
      phi0 = (xx - a.tm) / a.wx;
      if (a.plane_wave) {
        phi = atan(xx);
        ar = a.ee0 * cos(phi);
        ai = -a.ee0 * sin(phi);
      } else {
        xx = xx / a.zra;
        const double w2 = 1. / (1. + xx * xx);
        const double phx = atan(xx);
        phi = phx - xx * r2 * w2;
        const double ws = (a.ndim == 3) ? sqrt(w2) : sqrt(sqrt(w2));
        ar = a.ee0 * cos(phi) * ws * exp(-w2 * r2);
        ai = -a.ee0 * sin(phi) * ws * exp(-w2 * r2);
      }
      ampl1 = exp(-phi1 * phi1);
      ampl0 = exp(-phi0 * phi0);
    } else {
      if (a.plane_wave || a.ndim < 3) {
        phi1 = pi * (xx - a.t) / a.wx;
        phi0 = pi * (xx - a.tm) / a.wx;
      } else {
        phi1 = pi * (a.t - xx) / a.wx;
        phi0 = pi * (a.tm - xx) / a.wx;
      }
      if (fabs(phi1) > pih) phi1 = pih;
      if (fabs(phi0) > pih) phi0 = pih;
      if (a.plane_wave) {
        phi = 0.0;
        ar = a.ee0 * cos(phi);
        ai = -a.ee0 * sin(phi);
      } else {
        xx = xx / a.zra;
        const double w2 = 1. / (1. + xx * xx);
        const double phx = atan(xx);
        phi = phx - xx * r2 * w2;
        const double ws = (a.ndim == 3) ? sqrt(w2) : sqrt(sqrt(w2));
        ar = a.ee0 * cos(phi) * ws * exp(-w2 * r2);
        ai = -a.ee0 * sin(phi) * ws * exp(-w2 * r2);
      }
      ampl1 = cos(phi1) * cos(phi1);
      ampl0 = cos(phi0) * cos(phi0);
    }
    const long long o = goff(g, i, j, k);
    env[o] = env[o] + ampl1 * ar;
    env[nc + o] = env[nc + o] + ampl1 * ai;
    env[2 * nc + o] = env[2 * nc + o] + ampl0 * ar;
    env[3 * nc + o] = env[3 * nc + o] + ampl0 * ai;
  }
}

int grid_blocks(long long n, int sms) { return grid_for(n, 256, sms, 16); }

}  // namespace

void env_amp_grad(const EnvArgs& a, cudaStream_t st, int sms) {
  const long long n = interior_count(a.g);
  k_env_amp<<<grid_blocks(n, sms), 256, 0, st>>>(a.env, a.av, a.g);
  k_env_grad<<<grid_blocks(n, sms), 256, 0, st>>>(a.av, a.g, a.dx_inv, a.dy_inv, a.dz_inv);
}

void env_acc_momenta(const EnvArgs& a, cudaStream_t st, int sms, bool serial) {
  if (a.np <= 0) return;
  const int nb = grid_for(a.np, 256, sms, 8);
  if (a.g.ndim == 3) {
    if (serial) k_env_acc<true, 3><<<1, 1, 0, st>>>(a);
    else k_env_acc<false, 3><<<nb, 256, 0, st>>>(a);
  } else {
    if (serial) k_env_acc<true, 2><<<1, 1, 0, st>>>(a);
    else k_env_acc<false, 2><<<nb, 256, 0, st>>>(a);
  }
}

void env_den_collect(const EnvArgs& a, cudaStream_t st, int sms) {
  const Geo& g = a.g;
  const long long nx = g.ix2 - g.ix1 + 1, ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  if (g.ndim > 2 && a.ibz == 0) k_den_fold_z<<<grid_blocks(nx * ny, sms), 256, 0, st>>>(a.den, g);
  k_den_fold_y<<<grid_blocks(nx * nz, sms), 256, 0, st>>>(a.den, g, a.iby);
  if (a.ibx < 2) k_den_fold_x<<<grid_blocks(ny * nz, sms), 256, 0, st>>>(a.den, g);
  cudaMemcpyAsync(a.av, a.den, sizeof(double) * g.ncell, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(a.av + 2 * g.ncell, a.den, sizeof(double) * g.ncell, cudaMemcpyDeviceToDevice, st);
}

void env_advance(const EnvArgs& a, cudaStream_t st, int sms) {
  const Geo& g = a.g;
  const long long ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  const long long nxw = g.ix2 - g.ix1 + 5, nyw = g.jy2 - g.jy1 + 5;
  k_env_bds_x<<<grid_blocks(2 * ny * nz, sms), 256, 0, st>>>(a.env, g, a.ibx);
  k_env_bds_y<<<grid_blocks(2 * nxw * nz, sms), 256, 0, st>>>(a.env, g, a.iby);
  if (g.ndim == 3) k_env_bds_z<<<grid_blocks(2 * nxw * nyw, sms), 256, 0, st>>>(a.env, g, a.ibz);
  const long long n = interior_count(g);
  if (a.vdt > 0.) {
    // comoving frame: env_lpf_solve with ib = 0 (curr_and_fields_util.f90:276, 292-293)
    const double om0 = a.om0;
    const double dx_norm = a.dx_inv / om0;
    k_env_lpf_src<<<grid_blocks(n, sms), 256, 0, st>>>(a.env, a.av, g, a.ompe, a.dy_inv * a.dy_inv, a.dz_inv * a.dz_inv,
                                                      a.dt);
    k_env_lpf_der1<<<grid_blocks(n, sms), 256, 0, st>>>(a.av, a.den, a.xtmp, g, om0, 0.5 * a.dx_inv);
    k_env_lpf_inv<<<grid_blocks(n, sms), 256, 0, st>>>(a.env, a.av, a.den, a.xtmp, g, dx_norm * dx_norm, om0 * om0);
    k_env_grad<<<grid_blocks(n, sms), 256, 0, st>>>(a.av, g, a.dx_inv, a.dy_inv, a.dz_inv);
    return;
  }
  SolveC s;
  s.ompe = a.ompe;
  s.dt2 = a.dt * a.dt;
  s.kfact = a.om0 * a.dt;
  s.dx1_inv = a.om0 * a.dx_inv;
  s.der3 = (a.der_ord == 3) ? 1 : 0;
  s.aph1 = 1.;
  s.aph2 = 0.;
  if (s.der3) {
    s.aph1 = s.dx1_inv * a.opt_der1;
    s.aph2 = s.dx1_inv * 0.5 * (1. - a.opt_der1);
  }
  const double dx2 = a.dx_inv * a.dx_inv;
  double cf1 = 1., cf2 = 0.;
  if (a.der_ord > 2) {
    cf1 = 1. - 4. * a.hord_der2;
    cf2 = a.hord_der2;
  }
  s.dx4_1 = cf1 * dx2;
  s.dx4_2 = cf2 * dx2;
  s.dy2 = a.dy_inv * a.dy_inv;
  s.dz2 = a.dz_inv * a.dz_inv;
  k_env_solve<<<grid_blocks(n, sms), 256, 0, st>>>(a.env, a.av, g, s);
  const double k2_fact = 1. / (1. + s.kfact * s.kfact);
  k_env_update<<<grid_blocks(n, sms), 256, 0, st>>>(a.env, a.av, g, k2_fact, s.kfact);
  k_env_grad<<<grid_blocks(n, sms), 256, 0, st>>>(a.av, g, a.dx_inv, a.dy_inv, a.dz_inv);
}

void env_positions_deposit(const EnvArgs& a, cudaStream_t st, int sms, bool serial) {
  if (a.np <= 0) return;
  const int nb = grid_for(a.np, 256, sms, 8);
  if (a.g.ndim == 3) {
    if (serial) k_env_pos<true, 3><<<1, 1, 0, st>>>(a);
    else k_env_pos<false, 3><<<nb, 256, 0, st>>>(a);
  } else {
    if (serial) k_env_pos<true, 2><<<1, 1, 0, st>>>(a);
    else k_env_pos<false, 2><<<nb, 256, 0, st>>>(a);
  }
}

void env_init_pulse(const EnvPulseArgs& a, double* env, const Geo& g, cudaStream_t st, int sms) {
  k_env_pulse<<<grid_blocks(interior_count(g), sms), 256, 0, st>>>(a, env, g);
}

}  // namespace agpu
