// agpu_yee_fused.cuh — the whole leapfrog Yee step (A14: ef_bds(0), rote(dt/2),
// bf_bds(dt), rotb + current(dt), ef_bds(dt), rote(dt/2), the order of
// advance_lpf_fields, src/fields/curr_and_fields_util.f90:176-260) in one
// kernel that streams along z (in chunks of YF_KC planes per CTA).
//
// Each CTA owns a column tile (TX x TY nodes of the full (n1p, n2p) plane) and
// writes every node of its columns, k = 1..n3p, into a second field array:
// neighbouring tiles recompute the halo they need from the input array, so
// the update cannot be in place.  Per z-plane m the CTA keeps, in shared
// memory over its tile plus a halo of (-4..+5) x (-1..+2) nodes:
//   E0(m), E0(m+1)   E after the first ef_bds (the right-face Mur values),
//   B(m) -> B1/2(m)  B after the first rote, with bf_bds's left-face values,
//   E0(m) -> En(m)   E after rotb + current, with the second ef_bds,
// three E planes and three B planes in rings, and emits plane m-1:
//   B_new(m-1) = B1/2(m-1) - dt/2 curl En(m-1, m).
// Every face value is computed by the same formula, from the same operands,
// as the face kernels of agpu_yee.cuh, and every interior value by the same
// expression as k_rote / k_rotb_j, so the result equals the six-kernel path
// (bit for bit in FP64 without contraction).  Reads and writes each field
// word once (plus the halo, served from L2) instead of about 33 words per
// cell for the six sweeps.
#pragma once
#include "agpu_common.cuh"
#include "agpu_kernels.h"

namespace agpu {

constexpr int YF_TX = 32, YF_TY = 8;
constexpr int YF_RW = YF_TX + 9, YF_RH = YF_TY + 3;  // region x: X0-4 .. X0+TX+4, y: Y0-1 .. Y0+TY+1
constexpr int YF_RP = YF_RW * YF_RH;
constexpr int YF_KC = 4;  // output planes per CTA along z (blockIdx.z = chunk)

template <typename T, int NDIM>
__global__ void __launch_bounds__(256, 6) k_yee_fused(const T* __restrict__ fin, T* __restrict__ fout,
                                                   const T* __restrict__ jc, const T* __restrict__ jlo, Geo g,
                                                   YeeC c) {
  extern __shared__ unsigned char yf_smem[];
  T* sE = reinterpret_cast<T*>(yf_smem);  // 3 slots x 3 comps x RP
  T* sB = sE + 9 * YF_RP;                 // 3 slots x 3 comps x RP
  const int X0 = 1 + blockIdx.x * YF_TX, Y0 = 1 + blockIdx.y * YF_TY;
  const int xr0 = X0 - 4, yr0 = Y0 - 1;
  const int ix1 = g.ix1, ix2 = g.ix2, jy1 = g.jy1, jy2 = g.jy2, kz1 = g.kz1, kz2 = g.kz2;
  const long long nc3 = g.ncell;
  const int nf = g.nf;
  const T one = (T)1., two = (T)2.;
  // coefficients exactly as the face kernels and k_rote / k_rotb_j form them
  const double dt = c.dt, dth = 0.5 * dt;
  const T aphx0 = (T)(1.0 * c.dx_inv * 0.0), aphy0 = (T)(1.0 * c.dy_inv * 0.0), aphz0 = (T)(1.0 * c.dz_inv * 0.0);
  const T aphx1 = (T)(1.0 * c.dx_inv * dt), aphy1 = (T)(1.0 * c.dy_inv * dt), aphz1 = (T)(1.0 * c.dz_inv * dt);
  const double ahx = dth * c.dx_inv, ahy = dth * c.dy_inv, ahz = dth * c.dz_inv;
  const T r_aph1 = (T)(ahx * c.se1), r_aph2 = (T)(ahx * c.se2), r_sdhy = (T)(1.0 * ahy), r_sdhz = (T)(1.0 * ahz);
  const double afx = dt * c.dx_inv, afy = dt * c.dy_inv, afz = dt * c.dz_inv;
  const T b_aph1 = (T)(afx * c.se1), b_aph2 = (T)(afx * c.se2), b_sdy = (T)(1.0 * afy), b_sdz = (T)(afz * 1.0);
  const T ompe = (T)c.ompe, djc1 = (T)c.djc1, djc2 = (T)c.djc2, djc3 = (T)c.djc3;
  const int n1p = g.n1p, n2p = g.n2p;

  auto gidx = [&](int i, int j, int k) -> long long { return goff(g, i, j, k); };
  auto in_arr = [&](int i, int j) { return i >= 1 && i <= n1p && j >= 1 && j <= n2p; };
  auto interior_ij = [&](int i, int j) { return i >= ix1 && i <= ix2 && j >= jy1 && j <= jy2; };
  // component c of slot s at region point r
  auto E = [&](int s, int comp, int r) -> T& { return sE[(s * 3 + comp) * YF_RP + r]; };
  auto B = [&](int s, int comp, int r) -> T& { return sB[(s * 3 + comp) * YF_RP + r]; };
  const int BN = 2;  // B3 (Bz) component index in the slots; 2D keeps its Bz there too

  // ---- planes outside kz1-1 .. kz2+1: copied for the owned columns ---------
  auto copy_plane = [&](int k) {
    for (int q = threadIdx.x; q < YF_TX * YF_TY; q += blockDim.x) {
      const int i = X0 + q % YF_TX, j = Y0 + q / YF_TX;
      if (!in_arr(i, j)) continue;
      const long long o = gidx(i, j, k);
      for (int cc = 0; cc < nf; ++cc) fout[cc * nc3 + o] = fin[cc * nc3 + o];
    }
  };
  // this CTA's interior output planes c0..c1 (3D)
  const int c0 = kz1 + blockIdx.z * YF_KC;
  const int c1 = min(kz2, c0 + YF_KC - 1);
  if (NDIM == 3 || blockIdx.z == 0) {
    if (c0 == kz1)
      for (int k = 1; k < kz1 - 1; ++k) copy_plane(k);
    if (c1 == kz2)
      for (int k = kz2 + 2; k <= g.n3p; ++k) copy_plane(k);
  }

  // ---- load plane k into E slot se / B slot sb, then its first ef_bds faces --
  auto load_plane = [&](int k, int se, int sb) {
    for (int r = threadIdx.x; r < YF_RP; r += blockDim.x) {
      const int i = xr0 + r % YF_RW, j = yr0 + r / YF_RW;
      const bool ok = in_arr(i, j) && k >= 1 && k <= g.n3p;
      const long long o = ok ? gidx(i, j, k) : 0;
      if (NDIM == 3) {
        for (int cc = 0; cc < 3; ++cc) {
          E(se, cc, r) = ok ? fin[cc * nc3 + o] : (T)0;
          B(sb, cc, r) = ok ? fin[(3 + cc) * nc3 + o] : (T)0;
        }
      } else {
        E(se, 0, r) = ok ? fin[o] : (T)0;
        E(se, 1, r) = ok ? fin[nc3 + o] : (T)0;
        B(sb, BN, r) = ok ? fin[2 * nc3 + o] : (T)0;
      }
    }
  };
  // ef_bds(dtl) x- and y-faces of E slot se from E slot sef / B slot sbf (the
  // face-interior operands: E0 and B for the first call, En and B1/2 for the
  // second), on plane k
  auto ef_faces = [&](int k, int se, int sef, int sbf, T aphx, T aphy) {
    if (k < kz1 || k > kz2) return;
    for (int r = threadIdx.x; r < YF_RP; r += blockDim.x) {
      const int i = xr0 + r % YF_RW, j = yr0 + r / YF_RW;
      if (i == ix2 + 1 && j >= jy1 && j <= jy2 && r % YF_RW > 0) {
        const int ro = r - 1;  // (ix2, j)
        E(se, 1, r) = (two * B(sbf, BN, ro) - (one - aphx) * E(sef, 1, ro)) / (one + aphx);
        if (NDIM == 3) E(se, 2, r) = -(two * B(sbf, 1, ro) + (one - aphx) * E(sef, 2, ro)) / (one + aphx);
      } else if (j == jy2 + 1 && i >= ix1 && i <= ix2 && r >= YF_RW) {
        const int ro = r - YF_RW;  // (i, jy2)
        E(se, 0, r) = -(two * B(sbf, BN, ro) + (one - aphy) * E(sef, 0, ro)) / (one + aphy);
        if (NDIM == 3) E(se, 2, r) = (two * B(sbf, 0, ro) - (one - aphy) * E(sef, 2, ro)) / (one + aphy);
      }
    }
  };
  // first ef_bds z-face: E1, E2 on plane kz2+1 from E and B on plane kz2
  // (interior columns only); aphz is 0 for the first call, dt dz_inv for the
  // second
  auto ef_zface = [&](int se_top, int se_k2, int sb_k2, T aphz) {
    for (int r = threadIdx.x; r < YF_RP; r += blockDim.x) {
      const int i = xr0 + r % YF_RW, j = yr0 + r / YF_RW;
      if (!interior_ij(i, j)) continue;
      E(se_top, 0, r) = (two * B(sb_k2, 1, r) - (one - aphz) * E(se_k2, 0, r)) / (one + aphz);
      E(se_top, 1, r) = -(two * B(sb_k2, 0, r) + (one - aphz) * E(se_k2, 1, r)) / (one + aphz);
    }
  };
  // B1/2 = B - dt/2 curl E0 on plane m (rote), interior points whose stencil
  // lies in the region: x-1 .. x+2, y+1, z+1
  auto rote = [&](int m, int se, int se_up, int sb, T aph1, T aph2, T sdhy, T sdhz, int li0, int li1, int lj0,
                  int lj1) {
    for (int r = threadIdx.x; r < YF_RP; r += blockDim.x) {
      const int li = r % YF_RW, lj = r / YF_RW;
      if (li < li0 || li > li1 || lj < lj0 || lj > lj1) continue;
      const int i = xr0 + li, j = yr0 + lj;
      if (!interior_ij(i, j) || m < kz1 || m > kz2) continue;
      const int ry = r + YF_RW;
      B(sb, BN, r) = B(sb, BN, r) - aph1 * (E(se, 1, r + 1) - E(se, 1, r)) + sdhy * (E(se, 0, ry) - E(se, 0, r)) -
                     aph2 * (E(se, 1, r + 2) - E(se, 1, r - 1));
      if (NDIM == 3) {
        B(sb, 0, r) = B(sb, 0, r) - sdhy * (E(se, 2, ry) - E(se, 2, r)) + sdhz * (E(se_up, 1, r) - E(se, 1, r));
        B(sb, 1, r) = B(sb, 1, r) + aph1 * (E(se, 2, r + 1) - E(se, 2, r)) - sdhz * (E(se_up, 0, r) - E(se, 0, r)) +
                      aph2 * (E(se, 2, r + 2) - E(se, 2, r - 1));
      }
    }
  };
  // bf_bds(dt) x- and y-faces of B slot sb on plane m from E0 and B1/2
  auto bf_faces = [&](int m, int se, int sb) {
    if (m < kz1 || m > kz2) return;
    for (int r = threadIdx.x; r < YF_RP; r += blockDim.x) {
      const int i = xr0 + r % YF_RW, j = yr0 + r / YF_RW;
      if (i == ix1 - 1 && j >= jy1 && j <= jy2 && r % YF_RW < YF_RW - 1) {
        const int ro = r + 1;  // (ix1, j)
        B(sb, BN, r) = -(two * E(se, 1, ro) + (one - aphx1) * B(sb, BN, ro)) / (one + aphx1);
        if (NDIM == 3) B(sb, 1, r) = (two * E(se, 2, ro) - (one - aphx1) * B(sb, 1, ro)) / (one + aphx1);
      } else if (j == jy1 - 1 && i >= ix1 && i <= ix2 && r + YF_RW < YF_RP) {
        const int ro = r + YF_RW;  // (i, jy1)
        T v = two * E(se, 0, ro) - (one - aphy1) * B(sb, BN, ro);
        B(sb, BN, r) = v / (one + aphy1);
        if (NDIM == 3) {
          T w = -two * E(se, 2, ro) - (one - aphy1) * B(sb, 0, ro);
          B(sb, 0, r) = w / (one + aphy1);
        }
      }
    }
  };
  // bf_bds(dt) z-face: B1, B2 on plane kz1-1 from E0 and B1/2 on plane kz1
  auto bf_zface = [&](int sb_bot, int se_k1, int sb_k1) {
    for (int r = threadIdx.x; r < YF_RP; r += blockDim.x) {
      const int i = xr0 + r % YF_RW, j = yr0 + r / YF_RW;
      if (!interior_ij(i, j)) continue;
      T v = two * E(se_k1, 1, r) - (one - aphz1) * B(sb_k1, 0, r);
      B(sb_bot, 0, r) = v / (one + aphz1);
      T w = -two * E(se_k1, 0, r) - (one - aphz1) * B(sb_k1, 1, r);
      B(sb_bot, 1, r) = w / (one + aphz1);
    }
  };
  // En = E0 + dt curl B1/2 - ompe djc J on plane m (rotb + current), in place
  auto rotb = [&](int m, int se, int sb, int sb_dn) {
    for (int r = threadIdx.x; r < YF_RP; r += blockDim.x) {
      const int li = r % YF_RW, lj = r / YF_RW;
      if (li < 3 || li > YF_RW - 4 || lj < 1 || lj > YF_RH - 2) continue;
      const int i = xr0 + li, j = yr0 + lj;
      if (!interior_ij(i, j) || m < kz1 || m > kz2) continue;
      const long long o = gidx(i, j, m);
      T j1 = jc[o], j2 = jc[o + nc3];
      if (jlo) {
        j1 = j1 + jlo[o];
        j2 = j2 + jlo[o + nc3];
      }
      const int ry = r - YF_RW;
      T ex = E(se, 0, r) + b_sdy * (B(sb, BN, r) - B(sb, BN, ry));
      T ey = E(se, 1, r) - b_aph1 * (B(sb, BN, r) - B(sb, BN, r - 1)) - b_aph2 * (B(sb, BN, r + 1) - B(sb, BN, r - 2));
      if (NDIM == 2) {
        E(se, 0, r) = ex - ompe * (djc1 * j1);
        E(se, 1, r) = ey - ompe * (djc2 * j2);
      } else {
        T j3 = jc[o + 2 * nc3];
        if (jlo) j3 = j3 + jlo[o + 2 * nc3];
        ex = ex - b_sdz * (B(sb, 1, r) - B(sb_dn, 1, r));
        ey = ey + b_sdz * (B(sb, 0, r) - B(sb_dn, 0, r));
        T ez = E(se, 2, r) + b_aph1 * (B(sb, 1, r) - B(sb, 1, r - 1)) - b_sdy * (B(sb, 0, r) - B(sb, 0, ry)) +
               b_aph2 * (B(sb, 1, r + 1) - B(sb, 1, r - 2));
        E(se, 0, r) = ex - ompe * (djc1 * j1);
        E(se, 1, r) = ey - ompe * (djc2 * j2);
        E(se, 2, r) = ez - ompe * (djc3 * j3);
      }
    }
  };
  // the last rote of plane m and the outputs of plane m for the owned columns:
  // B = B1/2 - dt/2 curl En at interior points, else the B slot's value; E from
  // the E slot
  auto finish_plane = [&](int m, int se, int se_up, int sb) {
    for (int q = threadIdx.x; q < YF_TX * YF_TY; q += blockDim.x) {
      const int li = 4 + q % YF_TX, lj = 1 + q / YF_TX;
      const int i = xr0 + li, j = yr0 + lj;
      if (!in_arr(i, j)) continue;
      const int r = li + YF_RW * lj;
      const long long o = gidx(i, j, m);
      T bz = B(sb, BN, r), bx = (NDIM == 3) ? B(sb, 0, r) : (T)0, by = (NDIM == 3) ? B(sb, 1, r) : (T)0;
      if (interior_ij(i, j) && m >= kz1 && m <= kz2) {
        const int ry = r + YF_RW;
        bz = bz - r_aph1 * (E(se, 1, r + 1) - E(se, 1, r)) + r_sdhy * (E(se, 0, ry) - E(se, 0, r)) -
             r_aph2 * (E(se, 1, r + 2) - E(se, 1, r - 1));
        if (NDIM == 3) {
          bx = bx - r_sdhy * (E(se, 2, ry) - E(se, 2, r)) + r_sdhz * (E(se_up, 1, r) - E(se, 1, r));
          by = by + r_aph1 * (E(se, 2, r + 1) - E(se, 2, r)) - r_sdhz * (E(se_up, 0, r) - E(se, 0, r)) +
               r_aph2 * (E(se, 2, r + 2) - E(se, 2, r - 1));
        }
      }
      if (NDIM == 3) {
        fout[o] = E(se, 0, r);
        fout[nc3 + o] = E(se, 1, r);
        fout[2 * nc3 + o] = E(se, 2, r);
        fout[3 * nc3 + o] = bx;
        fout[4 * nc3 + o] = by;
        fout[5 * nc3 + o] = bz;
      } else {
        fout[o] = E(se, 0, r);
        fout[nc3 + o] = E(se, 1, r);
        fout[2 * nc3 + o] = bz;
      }
    }
  };

  // ---- the step ------------------------------------------------------------
  auto slot = [](int k) { return ((k % 3) + 3) % 3; };
  if (NDIM == 2) {
    load_plane(1, 0, 0);
    __syncthreads();
    ef_faces(1, 0, 0, 0, aphx0, aphy0);
    __syncthreads();
    rote(1, 0, 0, 0, r_aph1, r_aph2, r_sdhy, r_sdhz, 1, YF_RW - 3, 0, YF_RH - 2);
    __syncthreads();
    bf_faces(1, 0, 0);
    __syncthreads();
    rotb(1, 0, 0, 0);
    __syncthreads();
    ef_faces(1, 0, 0, 0, aphx1, aphy1);
    __syncthreads();
    finish_plane(1, 0, 0, 0);
    return;
  }
  // planes c0-1, c0, c0+1.  Plane kz1-1 is an output of the first chunk (B
  // gets bf_bds's z-face); for a later chunk, plane c0-1 belongs to the chunk
  // below and its B1/2 (with its faces) is recomputed here.
  load_plane(c0 - 1, slot(c0 - 1), slot(c0 - 1));
  load_plane(c0, slot(c0), slot(c0));
  load_plane(c0 + 1, slot(c0 + 1), slot(c0 + 1));
  __syncthreads();
  if (c0 - 1 >= kz1) ef_faces(c0 - 1, slot(c0 - 1), slot(c0 - 1), slot(c0 - 1), aphx0, aphy0);
  ef_faces(c0, slot(c0), slot(c0), slot(c0), aphx0, aphy0);
  if (c0 + 1 <= kz2)
    ef_faces(c0 + 1, slot(c0 + 1), slot(c0 + 1), slot(c0 + 1), aphx0, aphy0);
  else
    ef_zface(slot(c0 + 1), slot(c0), slot(c0), aphz0);
  __syncthreads();
  if (c0 - 1 >= kz1) {
    const int sp = slot(c0 - 1);
    rote(c0 - 1, sp, slot(c0), sp, r_aph1, r_aph2, r_sdhy, r_sdhz, 1, YF_RW - 3, 0, YF_RH - 2);
    __syncthreads();
    bf_faces(c0 - 1, sp, sp);
    __syncthreads();
  }
  // the last plane whose En this CTA needs: c1 + 1 (or the top face plane)
  const int mlast = (c1 == kz2) ? kz2 : c1 + 1;
  for (int m = c0; m <= mlast; ++m) {
    const int sm = slot(m), su = slot(m + 1), sd = slot(m - 1);
    rote(m, sm, su, sm, r_aph1, r_aph2, r_sdhy, r_sdhz, 1, YF_RW - 3, 0, YF_RH - 2);  // B1/2(m)
    __syncthreads();
    bf_faces(m, sm, sm);
    if (m == kz1) bf_zface(sd, sm, sm);
    __syncthreads();
    rotb(m, sm, sm, sd);  // En(m)
    __syncthreads();
    ef_faces(m, sm, sm, sm, aphx1, aphy1);
    __syncthreads();
    if ((m - 1 >= c0 || m - 1 == kz1 - 1) && m - 1 <= c1) {
      finish_plane(m - 1, sd, sm, sd);  // B_new(m-1) and the outputs of plane m-1
      __syncthreads();
    }
    if (m + 2 <= mlast + 1) {  // plane m+2 into the slot of m-1
      load_plane(m + 2, sd, sd);
      __syncthreads();
      if (m + 2 <= kz2)
        ef_faces(m + 2, sd, sd, sd, aphx0, aphy0);
      else
        ef_zface(sd, su, su, aphz0);
      __syncthreads();
    }
  }
  if (c1 == kz2) {
    const int s2 = slot(kz2), s3 = slot(kz2 + 1);
    ef_zface(s3, s2, s2, aphz1);  // the second ef_bds z-face, from En(kz2) and B1/2(kz2)
    __syncthreads();
    finish_plane(kz2, s2, s3, s2);
    finish_plane(kz2 + 1, s3, s3, s3);
  }
}

// fout = the fields after one leapfrog step of fin (fout != fin)
template <typename T>
void yee_fused_t(const T* fin, T* fout, const T* jc, const T* jlo, const Geo& g, const YeeC& c, cudaStream_t st) {
  const int nchunk = (g.ndim == 3) ? (g.kz2 - g.kz1 + 1 + YF_KC - 1) / YF_KC : 1;
  dim3 grid((g.n1p + YF_TX - 1) / YF_TX, (g.n2p + YF_TY - 1) / YF_TY, nchunk);
  const size_t sm = sizeof(T) * 18 * YF_RP;
  if (g.ndim == 3) {
    cudaFuncSetAttribute(k_yee_fused<T, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_yee_fused<T, 3><<<grid, 256, sm, st>>>(fin, fout, jc, jlo, g, c);
  } else {
    cudaFuncSetAttribute(k_yee_fused<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_yee_fused<T, 2><<<grid, 256, sm, st>>>(fin, fout, jc, jlo, g, c);
  }
}

}  // namespace agpu
