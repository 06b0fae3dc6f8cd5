// agpu_tile32c.cu — tiled gather + push + deposit of the FP32 split form
// with the cubic shape extension (AGPU_SHAPE_CUBIC; the reference has no
// cubic gather or deposit).  Same organisation as the quadratic tile kernel
// (agpu_tile32.cu): one CTA per tile, fields staged in shared memory, the
// deposit into an int32 fixed-point shared tile, one compensated flush.
// Differences: cubic B-spline weights on integer nodes (nodes f-1..f+2 of the
// floor node f) and quadratic weights on half nodes for the gather (a two-node
// field guard), and Esirkepov's scheme with 4-point shapes on 6-slot windows
// (a three-node current guard), in the regrouped form
//   Jx(u,v,w) = w cx(u) (wy0(v) Sz0(w) + wy1(v) Sz1(w))   (and cyclic),
// wy0 = Sy0 + Sy1/2, wy1 = Sy1 + Sy0/2; each component skips the last slot
// of its own axis, where the running sum is identically zero.
#include "agpu_bin.cuh"
#include "agpu_common.cuh"
#include "agpu_tile.h"

namespace agpu {

namespace {

__device__ __forceinline__ void kadd_gc(float* hi, float* lo, float v) {
  float old = atomicAdd(hi, v);
  float s = __fadd_rn(old, v);
  float bp = __fsub_rn(s, old);
  float err = __fadd_rn(__fsub_rn(old, __fsub_rn(s, bp)), __fsub_rn(v, bp));
  if (err != 0.f) atomicAdd(lo, err);
}
// Fixed-point contribution x * y in units of the tile's scale, below 2^22 in
// magnitude by construction: rounded to the nearest integer by one FMA with
// 1.5 * 2^23 (the sum lies in [2^23, 2^24), where the float spacing is 1).
__device__ __forceinline__ void fx_addc(int* a, float x, float y) {
  atomicAdd(a, __float_as_int(__fmaf_rn(x, y, 12582912.f)) - 0x4B400000);
}

// cubic B-spline weights at nodes f-1..f+2, s in [0, 1) from the floor node f
__device__ __forceinline__ void wcub(float s, float a[4]) {
  const float s2 = s * s, s3 = s2 * s;
  a[1] = 0.6666667f - s2 + 0.5f * s3;
  a[2] = 0.16666667f + 0.5f * (s + s2 - s3);
  a[3] = 0.16666667f * s3;
  a[0] = 1.f - a[1] - a[2] - a[3];
}
// quadratic weights at half nodes h-1..h+1 (h = f), offset s - 1/2
__device__ __forceinline__ void wqh(float s, float a[3]) {
  const float t = s - 0.5f, t2 = t * t;
  a[1] = 0.75f - t2;
  a[2] = 0.5f * (0.25f + t2 + t);
  a[0] = 1.f - a[1] - a[2];
}
// floor node of (nearest node i, offset o in [-0.5, 0.5)): f = i or i - 1
__device__ __forceinline__ int floor_of(int i, float o, float* s) {
  if (o >= 0.f) {
    *s = o;
    return i;
  }
  *s = o + 1.f;
  return i - 1;
}
__device__ __forceinline__ int renorm_c(float& s) {
  int m = (s >= 0.5f) ? 1 : ((s < -0.5f) ? -1 : 0);
  s = s - (float)m;
  return m;
}
__device__ __forceinline__ bool inside_c(int node, float o, int n) {
  int m = node - 3;
  return ((m > 0) || (m == 0 && o > 0.f)) && ((m < n) || (m == n && o <= 0.f));
}
// 1-D cubic window: old shape on slots 1..4, new on sh..sh+3 (sh = f1-f0+1)
__device__ __forceinline__ void cwin(float s0, float s1v, int sh, float a0s[6], float a1s[6], float cur[6]) {
  float a0[4], a1[4];
  wcub(s0, a0);
  wcub(s1v, a1);
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    a0s[q] = (q >= 1 && q <= 4) ? a0[q - 1] : 0.f;
    const int m = q - sh;
    a1s[q] = (m == 0) ? a1[0] : (m == 1) ? a1[1] : (m == 2) ? a1[2] : (m == 3) ? a1[3] : 0.f;
  }
  cur[0] = a0s[0] - a1s[0];
#pragma unroll
  for (int q = 1; q < 6; ++q) cur[q] = cur[q - 1] + a0s[q] - a1s[q];
}

}  // namespace

size_t tile32c_smem(int ndim, int tx, int ty, int tz) {
  if (ndim == 3) return sizeof(float) * (6 * (tx + 4) * (ty + 4) * (tz + 4) + 3 * (tx + 6) * (ty + 6) * (tz + 6));
  return sizeof(float) * (3 * (tx + 4) * (ty + 4) + 2 * (tx + 6) * (ty + 6));
}

template <int NDIM, int TX, int TY, int TZ>
__global__ void __launch_bounds__(256, 3) k32c_tile(TileArgs32 a) {
  constexpr int FX = TX + 4, FY = TY + 4, FZ = (NDIM == 3) ? TZ + 4 : 1;
  constexpr int JX = TX + 6, JY = TY + 6, JZ = (NDIM == 3) ? TZ + 6 : 1;
  constexpr int FV = FX * FY * FZ, JV = JX * JY * JZ;
  constexpr int NF = (NDIM == 3) ? 6 : 3, NC = (NDIM == 3) ? 3 : 2;
  extern __shared__ float smem[];
  float* sF = smem;                                  // NF * FV, origin node i0t - 2
  int* sJ = reinterpret_cast<int*>(smem + NF * FV);  // NC * JV, origin node i0t - 3
  __shared__ unsigned int s_wmax;

  const Geo g = a.g;
  const int t = blockIdx.x;
  const int beg = a.tstart[t * a.t.nsub], end = a.tstart[(t + 1) * a.t.nsub];
  if (beg >= end) return;
  const int tx = t % a.t.ntx, ty = (t / a.t.ntx) % a.t.nty, tz = t / (a.t.ntx * a.t.nty);
  const int i0t = 3 + tx * TX, j0t = 3 + ty * TY, k0t = (NDIM == 3) ? 3 + tz * TZ : 1;

  for (int e = threadIdx.x; e < NF * FV; e += blockDim.x) {
    int c = e / FV, r = e - c * FV;
    int lx = r % FX, ly = (r / FX) % FY, lz = r / (FX * FY);
    int gi = i0t - 2 + lx, gj = j0t - 2 + ly, gk = (NDIM == 3) ? k0t - 2 + lz : 1;
    float v = 0.f;
    if (gi >= 1 && gi <= g.n1p && gj >= 1 && gj <= g.n2p && gk >= 1 && gk <= g.n3p)
      v = __ldg(&a.ebf[g.ncell * c + goff(g, gi, gj, gk)]);
    sF[e] = v;
  }
  for (int e = threadIdx.x; e < NC * JV; e += blockDim.x) sJ[e] = 0;
  if (threadIdx.x == 0) s_wmax = 0u;
  __syncthreads();
  {
    float wl = 0.f;
    for (int q = beg + threadIdx.x; q < end; q += blockDim.x) {
      const uint64_t sl = a.p.slot[a.perm[q]];
      wl = fmaxf(wl, fabsf((float)slot_charge(sl) * slot_wgh(sl)));
    }
    if (!(wl <= 3.0e38f)) wl = 3.0e38f;
    for (int o = 16; o > 0; o >>= 1) wl = fmaxf(wl, __shfl_xor_sync(0xffffffffu, wl, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&s_wmax, __float_as_uint(wl));
  }
  __syncthreads();
  // one particle adds at most (4/3)|q w| to a node: the scale keeps every
  // node's sum below 2^31
  // 2^30 / (max|q w| * max(particles, 512)): node sums below 2^31 (one
  // particle adds at most 4/3 |q w| to a node), single contributions below 2^22
  float fsc = 1073741824.f / (__uint_as_float(s_wmax) * (float)max(end - beg, 512));
  if (!(fsc < 1.0e30f)) fsc = 1.0e30f;

  const int nx = g.ix2 - g.ix1 + 1, ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  for (int q = beg + threadIdx.x; q < end; q += blockDim.x) {
    const int p = a.perm[q];
    const int c = a.p.cell[p];
    int i0, j0, k0;
    cell_split(g, c, i0, j0, k0);
    float ox = a.p.ox[p], oy = a.p.oy[p], oz = (NDIM == 3) ? a.p.oz[p] : 0.f;
    float pp[3] = {a.p.px[p], a.p.py[p], (NDIM == 3) ? a.p.pz[p] : 0.f};
    const uint64_t sl = a.p.slot[p];
    if ((unsigned)(i0 - i0t) >= (unsigned)TX || (unsigned)(j0 - j0t) >= (unsigned)TY ||
        (NDIM == 3 && (unsigned)(k0 - k0t) >= (unsigned)TZ)) {
      raise_err(a.err, AGPU_EBIT_INDEX);
      a.key[p] = a.t.nkeys;
      hist_add(a.hist, a.t.nkeys);
      continue;
    }
    float sx, sy, sz = 0.f;
    const int fx = floor_of(i0, ox, &sx), fy = floor_of(j0, oy, &sy);
    const int fz = (NDIM == 3) ? floor_of(k0, oz, &sz) : 1;
    // local offsets of the first stencil node (floor - 1) in the staged fields
    const int lx = fx - i0t + 1, ly = fy - j0t + 1, lz = (NDIM == 3) ? fz - k0t + 1 : 0;
    float ax[4], ay[4], az[4] = {0.f, 1.f, 0.f, 0.f}, axh[3], ayh[3], azh[3] = {0.f, 1.f, 0.f};
    wcub(sx, ax);
    wcub(sy, ay);
    wqh(sx, axh);
    wqh(sy, ayh);
    if (NDIM == 3) {
      wcub(sz, az);
      wqh(sz, azh);
    }
    float ap[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (NDIM == 3) {
      const float* e1 = sF;
      const float* e2 = sF + FV;
      const float* e3 = sF + 2 * FV;
      const float* b1 = sF + 3 * FV;
      const float* b2 = sF + 4 * FV;
      const float* b3 = sF + 5 * FV;
#pragma unroll
      for (int k1 = 0; k1 < 4; ++k1) {
#pragma unroll
        for (int j1 = 0; j1 < 4; ++j1) {
          const int o = lx + FX * (ly + j1 + FY * (lz + k1));
          const float w = ay[j1] * az[k1];
          ap[0] += w * (axh[0] * e1[o] + axh[1] * e1[o + 1] + axh[2] * e1[o + 2]);
        }
#pragma unroll
        for (int j1 = 0; j1 < 3; ++j1) {
          const int o = lx + FX * (ly + j1 + FY * (lz + k1));
          const float w = ayh[j1] * az[k1];
          ap[1] += w * (ax[0] * e2[o] + ax[1] * e2[o + 1] + ax[2] * e2[o + 2] + ax[3] * e2[o + 3]);
          ap[5] += w * (axh[0] * b3[o] + axh[1] * b3[o + 1] + axh[2] * b3[o + 2]);
        }
      }
#pragma unroll
      for (int k1 = 0; k1 < 3; ++k1) {
#pragma unroll
        for (int j1 = 0; j1 < 4; ++j1) {
          const int o = lx + FX * (ly + j1 + FY * (lz + k1));
          const float w = ay[j1] * azh[k1];
          ap[2] += w * (ax[0] * e3[o] + ax[1] * e3[o + 1] + ax[2] * e3[o + 2] + ax[3] * e3[o + 3]);
          ap[4] += w * (axh[0] * b2[o] + axh[1] * b2[o + 1] + axh[2] * b2[o + 2]);
        }
#pragma unroll
        for (int j1 = 0; j1 < 3; ++j1) {
          const int o = lx + FX * (ly + j1 + FY * (lz + k1));
          const float w = ayh[j1] * azh[k1];
          ap[3] += w * (ax[0] * b1[o] + ax[1] * b1[o + 1] + ax[2] * b1[o + 2] + ax[3] * b1[o + 3]);
        }
      }
    } else {
      const float* e1 = sF;
      const float* e2 = sF + FV;
      const float* b3 = sF + 2 * FV;
#pragma unroll
      for (int j1 = 0; j1 < 4; ++j1) {
        const int o = lx + FX * (ly + j1);
        ap[0] += ay[j1] * (axh[0] * e1[o] + axh[1] * e1[o + 1] + axh[2] * e1[o + 2]);
      }
#pragma unroll
      for (int j1 = 0; j1 < 3; ++j1) {
        const int o = lx + FX * (ly + j1);
        ap[1] += ayh[j1] * (ax[0] * e2[o] + ax[1] * e2[o + 1] + ax[2] * e2[o + 2] + ax[3] * e2[o + 3]);
        ap[5] += ayh[j1] * (axh[0] * b3[o] + axh[1] * b3[o + 1] + axh[2] * b3[o + 2]);
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
    float nox = ox + a.dtx * dtg * pn[0];
    float noy = oy + a.dty * dtg * pn[1];
    float noz = (NDIM == 3) ? oz + a.dtz * dtg * pn[2] : 0.f;
    const int mi = renorm_c(nox), mj = renorm_c(noy), mk = (NDIM == 3) ? renorm_c(noz) : 0;
    const int i1n = i0 + mi, j1n = j0 + mj, k1n = k0 + mk;
    a.p.cell[p] = (int)goff(g, i1n, j1n, k1n);
    a.p.ox[p] = nox;
    a.p.oy[p] = noy;
    a.p.px[p] = pn[0];
    a.p.py[p] = pn[1];
    if (NDIM == 3) {
      a.p.oz[p] = noz;
      a.p.pz[p] = pn[2];
    }
    if (!(pn[0] == pn[0] && pn[1] == pn[1] && pn[2] == pn[2])) raise_err(a.err, AGPU_EBIT_NONFINITE);
    bool keep = inside_c(i1n, nox, nx) && inside_c(j1n, noy, ny);
    if (NDIM == 3) keep = keep && inside_c(k1n, noz, nz);
    int nkey = keep ? tile_key_c<TX, TY, TZ, (NDIM == 3) ? 8 : 4>(a.t, i1n, j1n, (NDIM == 3) ? k1n : 3,
                                                                   offset_octant(nox, noy, noz, NDIM))
                    : a.t.nkeys;
    a.key[p] = nkey;
    hist_add(a.hist, nkey);
    if (!keep) continue;
    // cubic Esirkepov deposit: slot 0 of each window is the old floor node - 2
    const float wsc = qc * slot_wgh(sl) * fsc;  // charge x weight in fixed-point units
    float s1x, s1y, s1z = 0.f;
    const int gx = floor_of(i1n, nox, &s1x), gy = floor_of(j1n, noy, &s1y);
    const int gz = (NDIM == 3) ? floor_of(k1n, noz, &s1z) : 1;
    const int shx = gx - fx + 1, shy = gy - fy + 1, shz = gz - fz + 1;
    if ((unsigned)shx > 2u || (unsigned)shy > 2u || (NDIM == 3 && (unsigned)shz > 2u)) {
      raise_err(a.err, AGPU_EBIT_INDEX);  // moved more than one node: not depositable
      continue;
    }
    float sx0[6], sx1[6], cx[6], sy0[6], sy1[6], cy[6];
    cwin(sx, s1x, shx, sx0, sx1, cx);
    cwin(sy, s1y, shy, sy0, sy1, cy);
    const int x0 = shx < 1 ? shx : 1, x1 = (shx + 3) > 4 ? shx + 3 : 4;
    const int y0 = shy < 1 ? shy : 1, y1 = (shy + 3) > 4 ? shy + 3 : 4;
    int* sJx = sJ;
    int* sJy = sJ + JV;
    // When no lane of the warp changes floor node, every window is slots
    // 1..4 and the deposit is a fixed 4 x 4 [x 4] loop without predicates
    // (the same expressions as the general loop).
    const bool stay = shx == 1 && shy == 1 && (NDIM == 2 || shz == 1);
    const bool warp_stays = __all_sync(__activemask(), stay);
    if (NDIM == 2 && warp_stays) {
#pragma unroll
      for (int v = 1; v <= 4; ++v) {
        const float wyv = sy0[v] + sy1[v];
        const float cyv = wsc * cy[v];
#pragma unroll
        for (int u = 1; u <= 4; ++u) {
          const int o = lx + u + JX * (ly + v);
          if (u < 4) fx_addc(&sJx[o], wsc * cx[u], wyv);
          if (v < 4) fx_addc(&sJy[o], sx0[u] + sx1[u], cyv);
        }
      }
    } else if (NDIM == 2) {
#pragma unroll
      for (int v = 0; v < 6; ++v) {
        if (v < y0 || v > y1) continue;
        const float wyv = sy0[v] + sy1[v];
        const float cyv = wsc * cy[v];
#pragma unroll
        for (int u = 0; u < 6; ++u) {
          if (u < x0 || u > x1) continue;
          const int o = lx + u + JX * (ly + v);
          if (u < x1) fx_addc(&sJx[o], wsc * cx[u], wyv);
          if (v < y1) fx_addc(&sJy[o], sx0[u] + sx1[u], cyv);
        }
      }
    } else {
      float sz0[6], sz1[6], cz[6];
      cwin(sz, s1z, shz, sz0, sz1, cz);
      const int z0 = shz < 1 ? shz : 1, z1 = (shz + 3) > 4 ? shz + 3 : 4;
      float wx0[6], wx1[6], wy0[6], wy1[6];
#pragma unroll
      for (int q2 = 0; q2 < 6; ++q2) {
        wx0[q2] = 0.5f * sx1[q2] + sx0[q2];
        wx1[q2] = sx1[q2] + 0.5f * sx0[q2];
        wy0[q2] = 0.5f * sy1[q2] + sy0[q2];
        wy1[q2] = sy1[q2] + 0.5f * sy0[q2];
        cx[q2] *= wsc;
        cy[q2] *= wsc;
        cz[q2] *= wsc;
      }
      int* sJz = sJ + 2 * JV;
      if (warp_stays) {
#pragma unroll
        for (int w = 1; w <= 4; ++w) {
          const float A0 = sz0[w], A1 = sz1[w], czw = cz[w];
          const int ow = lx + JX * (ly + JY * (lz + w));
#pragma unroll
          for (int v = 1; v <= 4; ++v) {
            const float wyv = wy0[v] * A0 + wy1[v] * A1;
            const float cyv = cy[v];
#pragma unroll
            for (int u = 1; u <= 4; ++u) {
              const int o = ow + u + JX * v;
              if (u < 4) fx_addc(&sJx[o], cx[u], wyv);
              if (v < 4) fx_addc(&sJy[o], cyv, wx0[u] * A0 + wx1[u] * A1);
              if (w < 4) fx_addc(&sJz[o], czw, wx0[u] * sy0[v] + wx1[u] * sy1[v]);
            }
          }
        }
      } else {
        for (int w = z0; w <= z1; ++w) {
          const float A0 = (w == 0) ? sz0[0] : (w == 1) ? sz0[1] : (w == 2) ? sz0[2] : (w == 3) ? sz0[3] : (w == 4) ? sz0[4] : sz0[5];
          const float A1 = (w == 0) ? sz1[0] : (w == 1) ? sz1[1] : (w == 2) ? sz1[2] : (w == 3) ? sz1[3] : (w == 4) ? sz1[4] : sz1[5];
          const float czw = (w == 0) ? cz[0] : (w == 1) ? cz[1] : (w == 2) ? cz[2] : (w == 3) ? cz[3] : (w == 4) ? cz[4] : cz[5];
          const int ow = lx + JX * (ly + JY * (lz + w));
#pragma unroll
          for (int v = 0; v < 6; ++v) {
            if (v < y0 || v > y1) continue;
            const float wyv = wy0[v] * A0 + wy1[v] * A1;
            const float cyv = cy[v];
#pragma unroll
            for (int u = 0; u < 6; ++u) {
              if (u < x0 || u > x1) continue;
              const int o = ow + u + JX * v;
              if (u < x1) fx_addc(&sJx[o], cx[u], wyv);
              if (v < y1) fx_addc(&sJy[o], cyv, wx0[u] * A0 + wx1[u] * A1);
              if (w < z1) fx_addc(&sJz[o], czw, wx0[u] * sy0[v] + wx1[u] * sy1[v]);
            }
          }
        }
      }
    }
  }
  __syncthreads();
  // compensated flush of the tile's currents (nodes i0t-3 ..)
  const double inv_sc = 1.0 / (double)fsc;
  for (int e = threadIdx.x; e < NC * JV; e += blockDim.x) {
    const int iv = sJ[e];
    if (iv == 0) continue;
    int c = e / JV, rr = e - c * JV;
    int lx = rr % JX, ly = (rr / JX) % JY, lz = rr / (JX * JY);
    int gi = i0t - 3 + lx, gj = j0t - 3 + ly, gk = (NDIM == 3) ? k0t - 3 + lz : 1;
    if (gi < 1 || gi > g.n1p || gj < 1 || gj > g.n2p || gk < 1 || gk > g.n3p) {
      raise_err(a.err, AGPU_EBIT_INDEX);
      continue;
    }
    long long o = g.ncell * c + goff(g, gi, gj, gk);
    const double dv = (double)iv * inv_sc;
    const float vh = (float)dv;
    const float vl = (float)(dv - (double)vh);
    kadd_gc(&a.jhi[o], &a.jlo[o], vh);
    if (vl != 0.f) atomicAdd(&a.jlo[o], vl);
  }
}

void tile_push32_cubic(const TileArgs32& a, cudaStream_t st) {
  if (a.t.ntiles <= 0) return;
  if (a.g.ndim == 3) {
    size_t sm = tile32c_smem(3, TILE3_X, TILE3_Y, TILE3_Z);
    auto k = k32c_tile<3, TILE3_X, TILE3_Y, TILE3_Z>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<a.t.ntiles, 256, sm, st>>>(a);
  } else {
    size_t sm = tile32c_smem(2, TILE2_X, TILE2_Y, 1);
    auto k = k32c_tile<2, TILE2_X, TILE2_Y, 1>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<a.t.ntiles, 256, sm, st>>>(a);
  }
}

}  // namespace agpu
