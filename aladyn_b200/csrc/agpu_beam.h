// agpu_beam.h — interface of agpu_beam.cu (PWFA bunch set-up: charge
// density, sine-transform Poisson solve, bunch fields).
#pragma once
#include <cuda_runtime.h>

#include "agpu_common.cuh"

namespace agpu {

struct BeamArgs {
  Geo g;
  int nx, ny, nz;  // interior nodes per axis
  double dx, dy, dz, dx_inv, dy_inv, dz_inv;
  double xmn, ymn, zmn;
  double lx_box, ly_box, lz_box;  // x(n1)-x(1), y(n2+1)-y(1), z(n3+1)-z(1)
  double ompe, gam2, bet0;
};

// set_grid_charge of nb FP64 records (columns of leading dimension ld) added
// into den (one field-layout component).
void beam_charge(const BeamArgs& a, const double* rec, long long ld, long long nb, double* den, unsigned int* err,
                 cudaStream_t st, int sms);
// fft_3d_psolv / fft_2d_psolv (ft_mod = 2, sym = 1): the interior of rho is
// replaced by the potential.  Allocates its scratch and cuFFT plans, and
// synchronises the stream before returning.  Returns 0 or an AGPU_E_* code.
int beam_potential(const BeamArgs& a, double* rho, cudaStream_t st, int sms, int* launches);
// p2 = bet0 p1, the ghost extrapolations, and ebf += the bunch fields
// (exactly one of ebf64 / ebf32 non-null).
void beam_fields(const BeamArgs& a, double* p1, double* p2, double* ebf64, float* ebf32, cudaStream_t st, int sms,
                 int* launches);

}  // namespace agpu
