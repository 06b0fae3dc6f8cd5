// agpu_envar.cu — the reductions of the reference's Envar diagnostics
// (src/diagnostics/diag_part_and_fields.f90:485-719) with energy_momenta
// (172-220) and energy_spect (126-142), in FP64 on the device.
//
// Per species, over the alive records:
//   ek(1:curr_ndim)  3D: sum p_k (unweighted, as energy_momenta sums them);
//                    2D: sum wgh p_k
//   ek(4)            3D: sum wgh (y pz - z py)
//   ek(6)            sum real(charge * wgh, sp)
//   ek(7)            sum wgh (gamma - 1)
//   ekmax            max (gamma - 1)
//   psig(1:curr_ndim) sum (p_k - ek(k)/np)^2 (Envar 594-604, the mean being
//                    ek(k)/np also where ek(k) is weighted)
//   nde(1:ne)        energy_spect: bin min(nint(pmass (gamma - 1) / de) + 1, ne)
//                    with de = pmass ekmax / ne, weight wgh; empty when
//                    pmass ekmax < 1e-6
// and over the interior nodes: sum F_c^2 per component, max |F_c| and
// max sum_{c <= curr_ndim} E_c^2.  gamma = sqrt(1 + p1^2 + p2^2 [+ p3^2])
// in the reference's order; this file is built without FMA contraction.
// Sums use FP64 atomics (their order varies); maxima are exact.
#include "../../include/aladyn_gpu.h"
#include "agpu_common.cuh"
#include "agpu_util.h"

namespace agpu {

namespace {

constexpr int NE = AGPU_NE;

__device__ __forceinline__ double wsum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double wmax(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ void amax_nonneg(double* a, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(a), (unsigned long long)__double_as_longlong(v));
}

// One record: momenta, the y and z positions (3D) and the packed slot.
struct ERec {
  double p[3], y, z;
  uint64_t slot;
};

struct ESrc {
  // FP64 form: part(cap, ndv); split form: the SoA records
  const double* part;
  long long ld;
  Part32View sp;
  bool split;
  const int* perm;  // alive records along the tile permutation, or null
  long long n;
  int nd;
  Geo g;
  double ymn, zmn, dy, dz;
};

__device__ __forceinline__ ERec erec(const ESrc& s, long long qq) {
  const long long q = s.perm ? (long long)s.perm[qq] : qq;
  ERec r;
  r.p[2] = 0.0;
  r.y = r.z = 0.0;
  if (!s.split) {
    for (int c = 0; c < s.nd; ++c) r.p[c] = s.part[(long long)(s.nd + c) * s.ld + q];
    if (s.nd == 3) {
      r.y = s.part[s.ld + q];
      r.z = s.part[2 * s.ld + q];
    }
    r.slot = dbits(s.part[(long long)(2 * s.nd) * s.ld + q]);
  } else {
    r.p[0] = (double)s.sp.px[q];
    r.p[1] = (double)s.sp.py[q];
    if (s.nd == 3) {
      r.p[2] = (double)s.sp.pz[q];
      // the absolute position as agpu_get_species returns it
      const int c = s.sp.cell[q];
      const int rr = c / s.g.n1p;
      const int j = rr % s.g.n2p + 1, k = rr / s.g.n2p + 1;
      r.y = s.ymn + ((double)(j - 3) + (double)s.sp.oy[q]) * s.dy;
      r.z = s.zmn + ((double)(k - 3) + (double)s.sp.oz[q]) * s.dz;
    }
    r.slot = s.sp.slot[q];
  }
  return r;
}

__device__ __forceinline__ double gamma_of(const ERec& r, int nd) {
  return (nd == 3) ? sqrt(1. + r.p[0] * r.p[0] + r.p[1] * r.p[1] + r.p[2] * r.p[2])
                   : sqrt(1. + r.p[0] * r.p[0] + r.p[1] * r.p[1]);
}

// out[0..6] = ek(1:7), out[7] = ekmax
__global__ void k_envar_p1(ESrc s, double* out) {
  double ek[7] = {0, 0, 0, 0, 0, 0, 0}, emax = 0.0;
  for (long long qq = blockIdx.x * (long long)blockDim.x + threadIdx.x; qq < s.n; qq += (long long)gridDim.x * blockDim.x) {
    const ERec r = erec(s, qq);
    const double gam1 = gamma_of(r, s.nd) - 1.;
    const float wf = slot_wgh(r.slot);
    const double w = (double)wf;
    const int ch = slot_charge(r.slot);
    if (s.nd == 3) {
      for (int k = 0; k < 3; ++k) ek[k] += r.p[k];
      ek[3] += w * (r.y * r.p[2] - r.z * r.p[1]);
    } else {
      for (int k = 0; k < 2; ++k) ek[k] += w * r.p[k];
    }
    ek[5] += (double)((float)ch * wf);
    ek[6] += w * gam1;
    emax = fmax(emax, gam1);
  }
  for (int c = 0; c < 7; ++c) {
    const double v = wsum(ek[c]);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&out[c], v);
  }
  const double m = wmax(emax);
  if ((threadIdx.x & 31) == 0) amax_nonneg(&out[7], m);
}

// out[8..10] = psig, out[16..16+NE) = nde; in: out[0..7] of pass 1, np
__global__ void k_envar_p2(ESrc s, double* out, double pmass) {
  __shared__ double sh[NE];
  for (int b = threadIdx.x; b < NE; b += blockDim.x) sh[b] = 0.0;
  __syncthreads();
  const double np_norm = (s.n > 0) ? 1.0 / (double)s.n : 1.0;
  const double mean[3] = {out[0] * np_norm, out[1] * np_norm, out[2] * np_norm};
  const double ekem = pmass * out[7];
  const bool spect = !(ekem < 1.e-06);
  const double de = ekem / (double)NE;
  double ps[3] = {0, 0, 0};
  for (long long qq = blockIdx.x * (long long)blockDim.x + threadIdx.x; qq < s.n; qq += (long long)gridDim.x * blockDim.x) {
    const ERec r = erec(s, qq);
    for (int k = 0; k < s.nd; ++k) {
      const double sg = r.p[k] - mean[k];
      ps[k] += sg * sg;
    }
    if (spect) {
      const double xx = pmass * (gamma_of(r, s.nd) - 1.) / de;
      int ix = (int)round(xx);
      ix = min(ix + 1, NE);
      atomicAdd(&sh[ix - 1], (double)slot_wgh(r.slot));
    }
  }
  for (int k = 0; k < 3; ++k) {
    const double v = wsum(ps[k]);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&out[8 + k], v);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < NE; b += blockDim.x)
    if (sh[b] != 0.0) atomicAdd(&out[16 + b], sh[b]);
}

// one warp per interior x-row: out[0..5] sum F_c^2, out[6..11] max |F_c|,
// out[12] max sum_{c < nc} E_c^2
template <typename T>
__global__ void k_envar_fields(const T* ebf, Geo g, double* out) {
  const int nx = g.ix2 - g.ix1 + 1, ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  const long long nrows = (long long)ny * nz;
  double acc[6] = {0, 0, 0, 0, 0, 0}, mx[6] = {0, 0, 0, 0, 0, 0}, e2 = 0.0;
  const int lane = threadIdx.x & 31;
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = warp; r < nrows; r += nwarps) {
    const int j = g.jy1 + (int)(r % ny), k = g.kz1 + (int)(r / ny);
    const long long o0 = goff(g, g.ix1, j, k);
    for (int i = lane; i < nx; i += 32) {
      const long long o = o0 + i;
      double ef2 = 0.0;
      for (int c = 0; c < g.nf; ++c) {
        const double v = (double)ebf[g.ncell * c + o];
        acc[c] += v * v;
        mx[c] = fmax(mx[c], fabs(v));
        if (c < g.nc) ef2 += v * v;
      }
      e2 = fmax(e2, ef2);
    }
  }
  for (int c = 0; c < g.nf; ++c) {
    const double v = wsum(acc[c]);
    const double m = wmax(mx[c]);
    if (lane == 0) {
      if (v != 0.0) atomicAdd(&out[c], v);
      amax_nonneg(&out[6 + c], m);
    }
  }
  const double m = wmax(e2);
  if (lane == 0) amax_nonneg(&out[12], m);
}

}  // namespace

void envar_species(const double* part, long long ld, const Part32View* sp, const int* perm, long long n, const Geo& g,
                   double ymn, double zmn, double dy, double dz, double pmass, double* d_out, cudaStream_t st, int sms) {
  ESrc s;
  s.part = part;
  s.ld = ld;
  s.split = sp != nullptr;
  if (sp) s.sp = *sp;
  s.perm = perm;
  s.n = n;
  s.nd = g.ndim;
  s.g = g;
  s.ymn = ymn;
  s.zmn = zmn;
  s.dy = dy;
  s.dz = dz;
  if (n <= 0) return;
  const int grid = grid_for(n, 256, sms, 8);
  k_envar_p1<<<grid, 256, 0, st>>>(s, d_out);
  k_envar_p2<<<grid, 256, 0, st>>>(s, d_out, pmass);
}

void envar_fields64(const double* ebf, const Geo& g, double* d_out, cudaStream_t st, int sms) {
  const long long rows = (long long)(g.jy2 - g.jy1 + 1) * (g.kz2 - g.kz1 + 1);
  k_envar_fields<double><<<grid_for(rows * 32, 256, sms, 8), 256, 0, st>>>(ebf, g, d_out);
}
void envar_fields32(const float* ebf, const Geo& g, double* d_out, cudaStream_t st, int sms) {
  const long long rows = (long long)(g.jy2 - g.jy1 + 1) * (g.kz2 - g.kz1 + 1);
  k_envar_fields<float><<<grid_for(rows * 32, 256, sms, 8), 256, 0, st>>>(ebf, g, d_out);
}

}  // namespace agpu
