// agpu_beam.cu — PWFA bunch set-up on the device: the bunch charge density
// (set_grid_charge, src/particles/grid_part_util.f90:240-334), the FP64
// sine-transform Poisson solve (fft_3d_psolv / fft_2d_psolv with
// beam_potential / beam_2d_potential, src/IO/psolve.f90:39-238) and the
// bunch fields (initial_beam_fields, src/fields/init_grid_fields.f90:32-134).
//
// The reference runs FFTW's RODFT00 (DST-I) along each axis
// (src/fft/modern_fft_lib.F90:675-775).  Here each 1-D DST-I of length n is a
// batched cuFFT D2Z of the odd extension of length N = 2(n+1):
//   z = [0, x_0 .. x_{n-1}, 0, -x_{n-1} .. -x_0],  Z = DFT(z)  =>
//   RODFT00(x)_k = 2 sum_j x_j sin(pi (j+1)(k+1)/(n+1)) = -Im Z_{k+1}.
// A pack kernel writes the extensions of all lines of one axis, one batched
// transform runs, an unpack kernel writes -Im Z back (with the forward scale
// of the reference).  Compiled with -fmad=false: the deposit and the field
// stencils keep the reference's roundings.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "agpu_beam.h"

namespace agpu {

namespace {

__device__ __forceinline__ int qden_b(double xp, double ax[3]) {
  double xx = 3.0 + xp;
  int i = (int)(xx + 0.5);
  double sx = xx - (double)i;
  double sx2 = sx * sx;
  ax[1] = 0.75 - sx2;
  ax[2] = 0.5 * (0.25 + sx2 + sx);
  ax[0] = 1. - ax[1] - ax[2];
  return i;
}

// set_grid_charge: one thread per bunch record; wght = real(charge*wgh, sp),
// ax0 = wght*ax0, den(i2,j2,k2) += ax0(i1)*(az0(k1)*ay0(j1)).  Records whose
// 3-node stencil leaves the array are skipped and flagged.
__global__ void k_beam_charge(BeamArgs a, const double* __restrict__ rec, long long ld, long long nb,
                              double* __restrict__ den, unsigned int* err) {
  const Geo g = a.g;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nb; n += (long long)gridDim.x * blockDim.x) {
    const int ch = g.ndim == 3 ? 6 : 4;
    uint64_t b = (uint64_t)__double_as_longlong(rec[(long long)ch * ld + n]);
    float wgh = __uint_as_float((uint32_t)(b >> 32));
    float wght = (float)(int)(int16_t)(uint16_t)(b & 0xffffu) * wgh;
    double ax0[3], ay0[3], az0[3] = {1., 0., 0.};
    double xl = a.dx_inv * (rec[n] - a.xmn);
    double yl = a.dy_inv * (rec[ld + n] - a.ymn);
    if (!(fabs(xl) < 1e9) || !(fabs(yl) < 1e9)) {
      atomicOr(err, (unsigned int)AGPU_EBIT_INDEX);
      continue;
    }
    int i = qden_b(xl, ax0) - 1;
    int j = qden_b(yl, ay0) - 1;
    int k = 1;
    for (int q = 0; q < 3; ++q) ax0[q] = (double)wght * ax0[q];
    bool ok = i >= 1 && i <= g.n1p - 2 && j >= 1 && j <= g.n2p - 2;
    if (g.ndim == 3) {
      double zl = a.dz_inv * (rec[2 * ld + n] - a.zmn);
      if (!(fabs(zl) < 1e9)) {
        atomicOr(err, (unsigned int)AGPU_EBIT_INDEX);
        continue;
      }
      k = qden_b(zl, az0) - 1;
      ok = ok && k >= 1 && k <= g.n3p - 2;
    }
    if (!ok) {
      atomicOr(err, (unsigned int)AGPU_EBIT_INDEX);
      continue;
    }
    if (g.ndim == 2) {
      for (int j1 = 0; j1 <= 2; ++j1)
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol = ax0[i1] * ay0[j1];
          atomicAdd(den + goff(g, i + i1, j + j1, 1), dvol);
        }
    } else {
      for (int k1 = 0; k1 <= 2; ++k1)
        for (int j1 = 0; j1 <= 2; ++j1) {
          double dvol = az0[k1] * ay0[j1];
          for (int i1 = 0; i1 <= 2; ++i1) atomicAdd(den + goff(g, i + i1, j + j1, k + k1), ax0[i1] * dvol);
        }
    }
  }
}

// Interior of the field-layout array <-> compact w(n1, n2, n3).
__global__ void k_interior_copy(double* __restrict__ rho, double* __restrict__ w, Geo g, int n1, int n2, int n3,
                                int to_compact) {
  long long total = (long long)n1 * n2 * n3;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % n1);
    long long r = q / n1;
    int j = (int)(r % n2);
    int k = (int)(r / n2);
    long long o = goff(g, g.ix1 + i, g.jy1 + j, g.kz1 + k);
    if (to_compact)
      w[q] = rho[o];
    else
      rho[o] = w[q];
  }
}

// Line geometry of one axis of the compact array w(n1, n2, n3): line l has
// its first element at base(l) and elements at stride.
struct Lines {
  int n;             // transform length
  long long count;   // number of lines
  long long stride;  // element stride along the axis
  int na;            // extent of the faster of the two other axes
  long long sa, sb;  // strides of the two other axes
  AGPU_HD long long base(long long l) const { return (l % na) * sa + (l / na) * sb; }
};

Lines axis_lines(int dir, int n1, int n2, int n3) {
  Lines L;
  long long s2 = n1, s3 = (long long)n1 * n2;
  if (dir == 1) {
    L.n = n1; L.stride = 1; L.na = n2; L.sa = s2; L.sb = s3; L.count = (long long)n2 * n3;
  } else if (dir == 2) {
    L.n = n2; L.stride = s2; L.na = n1; L.sa = 1; L.sb = s3; L.count = (long long)n1 * n3;
  } else {
    L.n = n3; L.stride = s3; L.na = n1; L.sa = 1; L.sb = s2; L.count = (long long)n1 * n2;
  }
  return L;
}

// Odd extensions of all lines: ext[l*N + m], N = 2(n+1).
__global__ void k_pack_odd(const double* __restrict__ w, double* __restrict__ ext, Lines L) {
  const long long N = 2LL * (L.n + 1);
  const long long total = L.count * N;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    long long l = q / N;
    int m = (int)(q - l * N);
    const double* line = w + L.base(l);
    double v = 0.0;
    if (m >= 1 && m <= L.n)
      v = line[(long long)(m - 1) * L.stride];
    else if (m >= L.n + 2)
      v = -line[(long long)(2 * L.n + 1 - m) * L.stride];
    ext[q] = v;
  }
}

// w(line, k) = [sc *] (-Im Z_{k+1}); Z has N/2+1 = n+2 entries per line.
__global__ void k_unpack_sine(const cufftDoubleComplex* __restrict__ z, double* __restrict__ w, Lines L, double sc,
                              int scale) {
  const long long M = (long long)L.n + 2;
  const long long total = L.count * (long long)L.n;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    long long l = q / L.n;
    int k = (int)(q - l * L.n);
    double y = -z[l * M + k + 1].y;
    w[L.base(l) + (long long)k * L.stride] = scale ? sc * y : y;
  }
}

__global__ void k_scale(double* w, long long n, double s) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    w[q] = s * w[q];
}

// beam_potential (psolve.f90:66-115) for ndim = 3, beam_2d_potential
// (psolve.f90:39-64) for ndim = 2 (no kx term).
__global__ void k_divide(double* w, int n1, int n2, int n3, const double* __restrict__ skx,
                         const double* __restrict__ sky, const double* __restrict__ skz, double gam2, int three_d) {
  long long total = (long long)n1 * n2 * n3;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    int ix = (int)(q % n1);
    long long r = q / n1;
    int iy = (int)(r % n2);
    int iz = (int)(r / n2);
    double ak2p = skz[iz] * skz[iz] + sky[iy] * sky[iy];
    if (three_d) {
      if (ak2p > 0.0) {
        double ak2 = ak2p + skx[ix] * skx[ix] / gam2;
        w[q] = w[q] / ak2;
      } else if (ix >= 1) {
        double ak2 = skx[ix] * skx[ix] / gam2;
        w[q] = w[q] / ak2;
      }
    } else {
      w[q] = ak2p > 0.0 ? w[q] / ak2p : 0.0;
    }
  }
}

// Wavenumbers of the sine transform (set_grid_param.f90:967-987).
void sine_k(std::vector<double>& sk, int n, double d, double l_box) {
  double wk = std::acos(-1.0) / l_box;
  for (int i = 1; i <= n; ++i) {
    double ak = wk * (double)i;
    sk[i - 1] = 2. * std::sin(0.5 * d * ak) / d;
  }
}

// One DST-I pass along dir over the compact array w (forward scales by sc).
int dst_pass(double* w, int dir, int n1, int n2, int n3, bool forward, double sc, double* ext, cufftDoubleComplex* spec,
             cudaStream_t st, int sms, int* launches) {
  Lines L = axis_lines(dir, n1, n2, n3);
  long long N = 2LL * (L.n + 1);
  cufftHandle plan;
  if (cufftCreate(&plan) != CUFFT_SUCCESS) return AGPU_E_CUDA;
  long long n_arr[1] = {N};
  long long inembed[1] = {N}, onembed[1] = {N / 2 + 1};
  size_t ws = 0;
  int rc = 0;
  if (cufftMakePlanMany64(plan, 1, n_arr, inembed, 1, N, onembed, 1, N / 2 + 1, CUFFT_D2Z, L.count, &ws) !=
      CUFFT_SUCCESS)
    rc = AGPU_E_CUDA;
  if (!rc && cufftSetStream(plan, st) != CUFFT_SUCCESS) rc = AGPU_E_CUDA;
  if (!rc) {
    k_pack_odd<<<grid_for(L.count * N, 256, sms, 16), 256, 0, st>>>(w, ext, L);
    if (cufftExecD2Z(plan, ext, spec) != CUFFT_SUCCESS) rc = AGPU_E_CUDA;
    k_unpack_sine<<<grid_for(L.count * L.n, 256, sms, 16), 256, 0, st>>>(spec, w, L, sc, forward ? 1 : 0);
    *launches += 2;
  }
  cufftDestroy(plan);
  if (!rc && cudaGetLastError() != cudaSuccess) rc = AGPU_E_CUDA;
  return rc;
}

}  // namespace

void beam_charge(const BeamArgs& a, const double* rec, long long ld, long long nb, double* den, unsigned int* err,
                 cudaStream_t st, int sms) {
  if (nb <= 0) return;
  k_beam_charge<<<grid_for(nb, 256, sms, 8), 256, 0, st>>>(a, rec, ld, nb, den, err);
}

int beam_potential(const BeamArgs& a, double* rho, cudaStream_t st, int sms, int* launches) {
  const Geo& g = a.g;
  const int n1 = a.nx, n2 = a.ny, n3 = g.ndim == 3 ? a.nz : 1;
  const long long ncell = (long long)n1 * n2 * n3;
  std::vector<double> hkx(n1 + 2, 0.0), hky(n2 + 2, 0.0), hkz(n3 + 2, 0.0);
  sine_k(hkx, n1, a.dx, a.lx_box);
  if (n2 > 1) sine_k(hky, n2, a.dy, a.ly_box);
  if (n3 > 1) sine_k(hkz, n3, a.dz, a.lz_box);
  // scratch: compact w, the largest odd-extension set and its spectrum
  long long ext_n = 0, spec_n = 0;
  for (int dir = 1; dir <= 3; ++dir) {
    Lines L = axis_lines(dir, n1, n2, n3);
    long long N = 2LL * (L.n + 1);
    ext_n = std::max(ext_n, L.count * N);
    spec_n = std::max(spec_n, L.count * (N / 2 + 1));
  }
  double *w = nullptr, *ext = nullptr, *dk = nullptr;
  cufftDoubleComplex* spec = nullptr;
  int rc = 0;
  if (cudaMalloc(&w, sizeof(double) * ncell) != cudaSuccess || cudaMalloc(&ext, sizeof(double) * ext_n) != cudaSuccess ||
      cudaMalloc(&spec, sizeof(cufftDoubleComplex) * spec_n) != cudaSuccess ||
      cudaMalloc(&dk, sizeof(double) * (size_t)(n1 + n2 + n3 + 6)) != cudaSuccess) {
    cudaGetLastError();
    rc = AGPU_E_NOMEM;
  }
  if (!rc) {
    double *dkx = dk, *dky = dk + n1 + 2, *dkz = dk + n1 + n2 + 4;
    cudaMemcpyAsync(dkx, hkx.data(), sizeof(double) * (n1 + 2), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dky, hky.data(), sizeof(double) * (n2 + 2), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dkz, hkz.data(), sizeof(double) * (n3 + 2), cudaMemcpyHostToDevice, st);
    k_interior_copy<<<grid_for(ncell, 256, sms, 16), 256, 0, st>>>(rho, w, g, n1, n2, n3, 1);
    *launches += 1;
    // forward scales: 1/(2(n1+2)) along x (logical_dimension(kind, n1+1)),
    // 1/(2(n+1)) along y and z (modern_fft_lib.F90:686-748)
    const double scx = 1. / (double)(2 * (n1 + 1 + 1));
    const double scy = 1. / (double)(2 * (n2 + 1));
    const double scz = 1. / (double)(2 * (n3 + 1));
    if (g.ndim == 3) {
      rc = dst_pass(w, 1, n1, n2, n3, true, scx, ext, spec, st, sms, launches);
      if (!rc && n2 > 2) rc = dst_pass(w, 2, n1, n2, n3, true, scy, ext, spec, st, sms, launches);
      if (!rc && n2 > 2 && n3 > 2) rc = dst_pass(w, 3, n1, n2, n3, true, scz, ext, spec, st, sms, launches);
    } else if (n2 > 2) {
      rc = dst_pass(w, 2, n1, n2, n3, true, scy, ext, spec, st, sms, launches);
    }
    if (!rc) {
      k_scale<<<grid_for(ncell, 256, sms, 16), 256, 0, st>>>(w, ncell, a.ompe);
      k_divide<<<grid_for(ncell, 256, sms, 16), 256, 0, st>>>(w, n1, n2, n3, dkx, dky, dkz, a.gam2, g.ndim == 3);
      *launches += 2;
    }
    if (g.ndim == 3) {
      if (!rc && n3 > 1) rc = dst_pass(w, 3, n1, n2, n3, false, 1.0, ext, spec, st, sms, launches);
      if (!rc && n2 > 1) rc = dst_pass(w, 2, n1, n2, n3, false, 1.0, ext, spec, st, sms, launches);
      if (!rc) rc = dst_pass(w, 1, n1, n2, n3, false, 1.0, ext, spec, st, sms, launches);
    } else if (!rc && n2 > 1) {
      rc = dst_pass(w, 2, n1, n2, n3, false, 1.0, ext, spec, st, sms, launches);
    }
    if (!rc) {
      k_interior_copy<<<grid_for(ncell, 256, sms, 16), 256, 0, st>>>(rho, w, g, n1, n2, n3, 0);
      *launches += 1;
    }
  }
  if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = AGPU_E_CUDA;
  cudaFree(w);
  cudaFree(ext);
  cudaFree(spec);
  cudaFree(dk);
  return rc;
}

namespace {

// ---- initial_beam_fields (init_grid_fields.f90:32-134), single domain -----

// Ghost extrapolations of the potential: pe1y (jy2+1), pe1x (ix2+1, both
// components) and, in 3D, pe1z (kz2+1).  They write disjoint ghost cells and
// read interior ones.
__global__ void k_beam_extrap(double* __restrict__ p1, double* __restrict__ p2, Geo g) {
  const int ni = g.ix2 - g.ix1 + 1, nj = g.jy2 - g.jy1 + 1, nk = g.kz2 - g.kz1 + 1;
  const long long ny_side = (long long)ni * nk, nx_side = (long long)nj * nk;
  const long long nz_side = g.ndim == 3 ? (long long)ni * nj : 0;
  const long long total = ny_side + nx_side + nz_side;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    if (q < ny_side) {
      int i = g.ix1 + (int)(q % ni), k = g.kz1 + (int)(q / ni), j = g.jy2;
      p1[goff(g, i, j + 1, k)] = 3. * (p1[goff(g, i, j, k)] - p1[goff(g, i, j - 1, k)]) + p1[goff(g, i, j - 2, k)];
    } else if (q < ny_side + nx_side) {
      long long r = q - ny_side;
      int j = g.jy1 + (int)(r % nj), k = g.kz1 + (int)(r / nj), i = g.ix2;
      p1[goff(g, i + 1, j, k)] = p1[goff(g, i, j, k)];
      p2[goff(g, i + 1, j, k)] = 2. * p2[goff(g, i, j, k)] - p2[goff(g, i - 1, j, k)];
    } else {
      long long r = q - ny_side - nx_side;
      int i = g.ix1 + (int)(r % ni), j = g.jy1 + (int)(r / ni), k = g.kz2;
      p1[goff(g, i, j, k + 1)] = 2. * p1[goff(g, i, j, k)] - p1[goff(g, i, j, k - 1)];
    }
  }
}

struct BeamFieldArgs {
  Geo g;
  double dx_inv, dy_inv, dz_inv, g2, bet;
};

// Bunch fields of one cell and their sum into the field array: Ex, Ey, and
// Bz (2D) or Ez, By, Bz (3D); Bx and every cell outside the reference's loop
// ranges receive + 0.0, as ebf(:,:,:,1:nf) += ebf_bunch(:,:,:,1:nf) does.
// In 3D the second potential component becomes 0.5 (Ez(i) + Ez(i+1)) with
// Ez(ix2+1) = 0 (never written in the reference's ebf_bunch).
template <typename T>
__global__ void k_beam_fields(BeamFieldArgs a, const double* __restrict__ p1, double* __restrict__ p2, T* ebf) {
  const Geo g = a.g;
  const double sdhy = 1.0 * a.dy_inv, sdhz = 1.0 * a.dz_inv;  // loc_yg(:,3) = loc_zg(:,3) = 1 (uniform)
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.ncell; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % g.n1p) + 1;
    long long r = q / g.n1p;
    int j = (int)(r % g.n2p) + 1;
    int k = (int)(r / g.n2p) + 1;
    double e[6] = {0., 0., 0., 0., 0., 0.};
    const bool in_jk = j >= g.jy1 && j <= g.jy2 && k >= g.kz1 && k <= g.kz2;
    if (in_jk && i >= g.ix1 && i <= g.ix2 + 1) {
      e[1] = -sdhy * (p1[goff(g, i, j + 1, k)] - p1[goff(g, i, j, k)]);
      if (i <= g.ix2) {
        e[0] = -a.dx_inv * (p1[goff(g, i + 1, j, k)] - p1[goff(g, i, j, k)]) / a.g2;
        double ey1 = -sdhy * (p1[goff(g, i + 1, j + 1, k)] - p1[goff(g, i + 1, j, k)]);
        double bz = 0.5 * a.bet * (e[1] + ey1);
        if (g.ndim == 2) {
          e[2] = bz;
        } else {
          e[5] = bz;
          e[2] = -sdhz * (p1[goff(g, i, j, k + 1)] - p1[goff(g, i, j, k)]);
          double ez1 = (i + 1 <= g.ix2) ? -sdhz * (p1[goff(g, i + 1, j, k + 1)] - p1[goff(g, i + 1, j, k)]) : 0.0;
          double pz = 0.5 * (e[2] + ez1);
          p2[q] = pz;
          e[4] = -a.bet * pz;
        }
      }
    }
    for (int c = 0; c < g.nf; ++c) {
      T* f = ebf + (long long)c * g.ncell + q;
      *f = (T)((double)*f + e[c]);
    }
  }
}

__global__ void k_scaled_copy(const double* __restrict__ a, double* __restrict__ b, long long n, double s) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    b[q] = s * a[q];
}

}  // namespace

void beam_fields(const BeamArgs& a, double* p1, double* p2, double* ebf64, float* ebf32, cudaStream_t st, int sms,
                 int* launches) {
  const Geo& g = a.g;
  // jc(:,:,:,2) = bet0*jc(:,:,:,1) over the whole array (beam_inject)
  k_scaled_copy<<<grid_for(g.ncell, 256, sms, 16), 256, 0, st>>>(p1, p2, g.ncell, a.bet0);
  long long ne = (long long)(g.ix2 - g.ix1 + 1) * (g.kz2 - g.kz1 + 1) + (long long)(g.jy2 - g.jy1 + 1) * (g.kz2 - g.kz1 + 1) +
                 (g.ndim == 3 ? (long long)(g.ix2 - g.ix1 + 1) * (g.jy2 - g.jy1 + 1) : 0);
  k_beam_extrap<<<grid_for(ne, 256, sms, 8), 256, 0, st>>>(p1, p2, g);
  BeamFieldArgs f{g, a.dx_inv, a.dy_inv, a.dz_inv, a.gam2, a.bet0};
  if (ebf64)
    k_beam_fields<double><<<grid_for(g.ncell, 256, sms, 16), 256, 0, st>>>(f, p1, p2, ebf64);
  else
    k_beam_fields<float><<<grid_for(g.ncell, 256, sms, 16), 256, 0, st>>>(f, p1, p2, ebf32);
  *launches += 3;
}

}  // namespace agpu
