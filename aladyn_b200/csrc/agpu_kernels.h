// agpu_kernels.h — internal interface between the C-ABI host code
// (agpu_api.cu) and the kernel translation units (agpu_fp64.cu,
// agpu_fp32.cu, agpu_util.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "agpu_common.cuh"

namespace agpu {
struct YeeC {
  double dx_inv, dy_inv, dz_inv, dt, se1, se2, ompe, djc1, djc2, djc3;
  double vbeam;  // comoving frame: the x advection speed of the fields (0: off)
  // stretched y / z (null: uniform): loc_yg(jj, 3), loc_yg(jj, 4),
  // loc_zg(kk, 3), loc_zg(kk, 4), jj = j - 2, kk = k - 2 (device arrays)
  const double* my3 = nullptr;
  const double* my4 = nullptr;
  const double* mz3 = nullptr;
  const double* mz4 = nullptr;
  // the Mur faces' factors: loc_yg(1, 3) (bf_bds, y = ymin), loc_yg(ny, 4)
  // (ef_bds, y = ymax), loc_zg(1, 3), loc_zg(nz, 4)
  double by3 = 1.0, ty4 = 1.0, bz3 = 1.0, tz4 = 1.0;
};

// One stretched transverse axis (map2dy_part_sind / map2dz_part_sind,
// src/grid/stretched_grid.f90:45-143): a particle coordinate in cells of the
// uniform computational grid (node index - 1 of the integer nodes).
struct StrAxis {
  double cnst, smin, smax, xs, dl_inv, dli_inv, ratio, nl_stretch, init_cell, n;
};
AGPU_HD double str_inv(const StrAxis& s, double yp) {
  // invert_stretched_grid: dli_inv atan(ratio (y + const - xs)) + nl_stretch
  return s.dli_inv * atan(s.ratio * (yp + s.cnst - s.xs)) + s.nl_stretch;
}
AGPU_HD double str_map(const StrAxis& s, double yp) {
  if (yp <= s.smin) return str_inv(s, yp) - s.init_cell;
  if (yp >= s.smax) {
    const double ym = 2 * 0.0 - yp;  // mirrored about the symmetry centre 0
    return (s.n - str_inv(s, ym)) - s.init_cell;
  }
  return (yp + s.cnst) * s.dl_inv - s.init_cell;  // invert_uniform_grid
}
// Scratch of the comoving frame's field advection (field_xadvect,
// src/fields/grid_fields.f90:210-324): a one-component buffer for the
// explicit step and the coefficients of the implicit step's tridiagonal
// solve (trid_der1, grid_fields.f90:37-77, with b1 = bn = 1, c1 = an = 0),
// the same for every row: bet[k], w1[k], k = 1..nx, a = -aphx_exp.
struct XAdv {
  double* tmp;
  const double* bet;
  const double* w1;
  double a, aphx_exp;
};
// A slab of a y decomposition: the host's exchange, called between the
// Yee sweeps with the point (AGPU_HALO_E after each ef_bds, AGPU_HALO_B after
// bf_bds); a non-zero return is kept in rc and the sweeps stop.
struct YeeHook {
  int (*fn)(void* ctx, int point);
  void* ctx;
  int rc;
};
}  // namespace agpu

namespace agpu {

// Device state of the FP64 form.
struct Dev64 {
  Geo g;
  double* ebf;  // (n1p, n2p, n3p, nf)
  double* jc;   // (n1p, n2p, n3p, nc), raw sums before djc
};


struct PushArgs64 {
  Geo g;
  const double* ebf;
  double* jc;
  double *x, *y, *z, *px, *py, *pz;
  const double* slot;
  int* flag;  // set to 1 for particles that leave the box
  long long np;
  double xmn, ymn, zmn, dx_inv, dy_inv, dz_inv;
  double dt, dth, lfact;
  double gxmin, gxmax, gymin, gymax, gzmin, gzmax;
  double vdt;  // comoving frame: dt * vbeam subtracted from x after the push (0: off)
  int initial;
  int shape;  // AGPU_SHAPE_QUADRATIC or AGPU_SHAPE_CUBIC
  int iform;  // 0, 1: Esirkepov; 2: the non-conserving ncdef deposit
  // y and z sides shared with neighbouring slabs: a particle that leaves
  // through one (and no physical side) still deposits its current here
  int dd_ylo = 0, dd_yhi = 0, dd_zlo = 0, dd_zhi = 0;
  // stretched y and z (str != 0): particle coordinates through str_map
  int str = 0;
  StrAxis sy{}, sz{};
  unsigned long long* removed;
  unsigned int* err;
};

struct IonArgs64 {
  Geo g;
  const double* ebf;
  const double *x, *y, *z;
  double* slot;
  double* ef2;
  int* flag;
  long long np;
  double xmn, ymn, zmn, dx_inv, dy_inv, dz_inv;
  const double* wtab;
  int n_ge, zmax, iter, ic;
  double de_inv;
  uint64_t seed;
  unsigned int* err;
};

void field_bd64(const Dev64& d, cudaStream_t st, int sms);
void push_deposit64(const PushArgs64& a, cudaStream_t st, int sms, bool serial);
void jfold64(const Dev64& d, cudaStream_t st, int sms);
void yee64(const Dev64& d, const YeeC& c, cudaStream_t st, int sms, const XAdv* xa = nullptr, YeeHook* hk = nullptr);
// the whole leapfrog step in one z-streaming kernel, fin -> fout (fout != fin)
void yee64_fused(const double* fin, double* fout, const double* jc, const Geo& g, const YeeC& c, cudaStream_t st);
__global__ void k64_ion_efield(IonArgs64 a);
__global__ void k64_ionize(IonArgs64 a);

// ---------------------------------------------------------------------------
// FP32 split form
// ---------------------------------------------------------------------------
// Particle record: int32 linear node index of the nearest integer node
// (the reference's qden index int(3 + x_loc + 0.5), Fortran 1-based, linear
// over (n1p, n2p, n3p)), FP32 offsets (3 + x_loc) - ix in [-0.5, 0.5),
// FP32 momenta and the 8-byte packed charge/part_ind/wgh slot.
struct Dev32 {
  Geo g;
  float* ebf;   // (n1p, n2p, n3p, nf)
  float* jhi;   // (n1p, n2p, n3p, nc) compensated sum: value = jhi + jlo
  float* jlo;
};

struct Part32 {
  int* cell;
  float *ox, *oy, *oz;
  float *px, *py, *pz;
  uint64_t* slot;
};

struct PushArgs32 {
  Geo g;
  const float* ebf;
  float* jhi;
  float* jlo;
  Part32 p;
  int* flag;
  long long np;
  float dt, dth, lfact;
  float dtx, dty, dtz;  // dt * d{x,y,z}_inv
  int initial;
  unsigned long long* removed;
  unsigned int* err;
};


struct IonArgs32 {
  Geo g;
  const float* ebf;
  const int* cell;
  const float *ox, *oy, *oz;
  uint64_t* slot;
  double* ef2;
  int* flag;
  long long np;
  const double* wtab;
  int n_ge, zmax, iter, ic;
  double de_inv;
  uint64_t seed;
  unsigned int* err;
};
__global__ void k32_ion_efield(IonArgs32 a);
__global__ void k32_ionize(IonArgs32 a);

void field_bd32(const Dev32& d, cudaStream_t st, int sms);
void push_deposit32(const PushArgs32& a, cudaStream_t st, int sms);
void jfold32(const Dev32& d, cudaStream_t st, int sms);
void yee32(const Dev32& d, const YeeC& c, cudaStream_t st, int sms);
void yee32_fused(const float* fin, float* fout, const float* jhi, const float* jlo, const Geo& g, const YeeC& c,
                 cudaStream_t st);

}  // namespace agpu
