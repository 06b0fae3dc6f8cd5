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
};
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
  // y sides shared with a neighbouring slab: a particle that leaves through
  // one (and stays in the x and z box) still deposits its current here
  int dd_ylo = 0, dd_yhi = 0;
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
