// agpu_env.h — interface of agpu_env.cu: the kernels of the envelope cycle
// (env_lpf2_evolve, src/dynamics/env_evolve_in_time.f90:196-361) in the
// FP64 form.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "agpu_common.cuh"

namespace agpu {

// Device state of one envelope step.  env(n1p,n2p,n3p,4): A^n (Re, Im),
// A^{n-1}; av(n1p,n2p,n3p,ndim+1): the reference's jc during the envelope
// part of the step; den(n1p,n2p,n3p): <q^2 n w / gam> before it is copied
// into av(1) and av(3).
struct EnvArgs {
  Geo g;
  const double* ebf;
  double* env;
  double* av;
  double* den;
  double* jc;  // raw Esirkepov sums (curr_ndim components)
  // species 0, SoA columns of capacity length (z, pz null in 2D)
  double *x, *y, *z, *px, *py, *pz;
  const double* slot;
  int* flag;
  long long np;
  double xmn, ymn, zmn, dx_inv, dy_inv, dz_inv;
  double dt, lfact, ompe;
  double gxmin, gxmax, gymin, gymax, gzmin, gzmax;
  double vdt;  // comoving frame: dt * vbeam subtracted from x after the push (0: off)
  // comoving frame: a second ncell scratch for the reduced envelope solver
  // (den is the first; both free once den has been copied into av)
  double* xtmp;
  double om0, opt_der1, hord_der2;
  int der_ord, ibx, iby, ibz, iform;
  unsigned long long* removed;
  unsigned int* err;
};

// init_gprof_envelope_field / init_envelope_field for one pulse
struct EnvPulseArgs {
  int ndim, g_prof, plane_wave;
  double ee0, t, tm, xf0, wx, wy, zra, ycent, zcent;
  double xmn, ymn, zmn, dx, dy, dz;
};

// av(1) = |A^n|^2 / 2 on the interior (av zeroed by the caller), then env_grad
void env_amp_grad(const EnvArgs& a, cudaStream_t st, int sms);
// set_env_acc + lpf_env_momenta + set_env_density (into den, zeroed by the
// caller); serial: one thread, particles in order
void env_acc_momenta(const EnvArgs& a, cudaStream_t st, int sms, bool serial);
// den_zyxbd on den, then av(1) = av(3) = den
void env_den_collect(const EnvArgs& a, cudaStream_t st, int sms);
// env_bds + the source term + env_maxw_solve (env_lpf_solve with ib = 0 in
// the comoving frame, a.vdt > 0), then env_fields_average and env_grad
void env_advance(const EnvArgs& a, cudaStream_t st, int sms);
// set_env_grad_interp + lpf_env_positions + the box test of
// cell_part_dist(.false.) + the Esirkepov deposit of the kept particles
void env_positions_deposit(const EnvArgs& a, cudaStream_t st, int sms, bool serial);
void env_init_pulse(const EnvPulseArgs& a, double* env, const Geo& g, cudaStream_t st, int sms);

}  // namespace agpu
