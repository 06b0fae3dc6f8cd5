/*
 * aladyn_oracle.c — CPU FP64 restatement of ALaDyn's per-timestep PIC cycle.
 *
 * TEST INFRASTRUCTURE ONLY.  The product (aladyn_b200/, the CUDA library)
 * never links, loads or calls this file; tests/, the smoke check and
 * bench.py's CPU baseline use it as the checker.
 *
 * parity unpinned: the reference is a Fortran 2003 + MPI + FFTW program that
 * cannot be compiled in this image (no Fortran compiler, no MPI, no FFTW) and
 * ships no tests, golden vectors or known-answer data.  This restatement is
 * pinned instead to the reference's source text, line by line (each function
 * cites the file:line it follows, paths relative to the ALaDyn project root),
 * and to the method's own invariants checked in tests/: partition of unity of
 * every shape set, discrete continuity of the Esirkepov current, vacuum Yee
 * dispersion, |p| conservation in a pure magnetic field, and the closed-form
 * one-level ionization probability.
 *
 * Arithmetic follows the Fortran statement order with no FMA contraction
 * (compile with -ffp-contract=off), matching gfortran -O2 on generic x86-64
 * with -fdefault-real-8; real(sp) roundings of the reference are kept.
 * Indices are the Fortran 1-based ones, arrays use the Fortran layouts.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/aladyn_gpu.h"
#include "philox.h"

#define ORA_NGE 10000 /* n_ge, src/ionization/ionz_data.f90:55 */

typedef struct ora_sim {
  agpu_params p;
  int n1p, n2p, n3p, ix1, ix2, jy1, jy2, kz1, kz2, ndv, nf, nc;
  double* ebf;
  double* jc;
  double* part[4];
  int64_t np[4], cap[4];
  double* ebfp;
  int64_t ebfp_cap;
  /* window state (lp_window_xshift saved variables, window.f90:279-280) */
  double xlapse;
  int wi1;
  /* plasma lattice sources (particles_inject, window.f90:106-184) */
  agpu_plasma src[4];
  int has_src[4];
  int64_t nptx[4], sptx_max[4];
  int npty[4], nptz[4];
  /* ionization tables w_one_lev(0:n_ge+1, 0:zmax) per ion species */
  double* wtab[4];
  int zmax[4];
  double de_inv[4];
  double lp_max[4];
  int at_num[4], ion_min[4], ionz_model[4];
  int nsp_ionz; /* species index bound: ions 1..nsp_ionz-1 ionize */
  uint32_t error_bits;
  int nthreads; /* >1: threaded CPU baseline (per-thread current copies) */
  /* envelope model: env(n1p,n2p,n3p,4) and the step's jc(:,:,:,1:ndim+1) */
  double* env;
  double* av;
  int nav;
  agpu_env_params ep;
  /* stretched y and z (set_grid, stretched_grid.f90): the particle maps and
     loc_yg(0:ny+1, 3:4), loc_zg(0:nz+1, 3:4) */
  int str;
  agpu_stretch_axis sy, sz;
  double *ym3, *ym4, *zm3, *zm4;
} ora_sim;

/* ---- layout helpers (Fortran 1-based) ---------------------------------- */
#define EBF(s, i, j, k, c)                                                            \
  (s)->ebf[((size_t)(i)-1) +                                                          \
           (size_t)(s)->n1p * (((size_t)(j)-1) +                                      \
                               (size_t)(s)->n2p * (((size_t)(k)-1) + (size_t)(s)->n3p * ((size_t)(c)-1)))]
#define JC(s, i, j, k, c)                                                             \
  (s)->jc[((size_t)(i)-1) +                                                           \
          (size_t)(s)->n1p * (((size_t)(j)-1) +                                       \
                              (size_t)(s)->n2p * (((size_t)(k)-1) + (size_t)(s)->n3p * ((size_t)(c)-1)))]
#define PART(s, ic, n, c) (s)->part[ic][(size_t)((c)-1) * (size_t)(s)->cap[ic] + (size_t)((n)-1)]
#define PT(s, n, c) (s)->ebfp[(size_t)((c)-1) * (size_t)(s)->ebfp_cap + (size_t)((n)-1)]

/* packed charge / part_ind / wgh slot (precision_def.F90:33-40) */
typedef struct {
  int16_t charge;
  int16_t part_ind;
  float wgh;
} ora_pack;
static inline ora_pack ora_unpack(double w) {
  ora_pack r;
  uint64_t b;
  memcpy(&b, &w, 8);
  r.charge = (int16_t)(uint16_t)(b & 0xffffu);
  r.part_ind = (int16_t)(uint16_t)((b >> 16) & 0xffffu);
  uint32_t fb = (uint32_t)(b >> 32);
  memcpy(&r.wgh, &fb, 4);
  return r;
}
static inline double ora_pack_slot(int16_t charge, int16_t part_ind, float wgh) {
  uint32_t fb;
  memcpy(&fb, &wgh, 4);
  uint64_t b = (uint64_t)(uint16_t)charge | ((uint64_t)(uint16_t)part_ind << 16) | ((uint64_t)fb << 32);
  double w;
  memcpy(&w, &b, 8);
  return w;
}

/* Fortran nint: round half away from zero. */
static inline int ora_nint(double x) { return (int)lround(x); }

static const double shx = 3.0; /* real(sp) shx = 3., grid_part_lib.f90:32 */

/* ======================================================================== */
/* lifecycle                                                                */
/* ======================================================================== */
ora_sim* ora_create(const agpu_params* p) {
  ora_sim* s = (ora_sim*)calloc(1, sizeof(ora_sim));
  if (!s) return NULL;
  s->p = *p;
  /* v_alloc: n1p = nxp + ihx with nxp = nx_loc + 2, ihx = 3
     (src/work/array_alloc.f90:63-71, src/work/pstruct_data.f90:40) */
  s->n1p = p->nx + 5;
  s->n2p = p->ny + 5;
  s->n3p = (p->ndim == 3) ? p->nz + 5 : 1;
  /* p_ind(1) = min(sh_ix=3, n_loc), p_ind(2) = n_loc + p_ind(1) - 1
     (set_grid_param.f90:604-609, 811-829) */
  s->ix1 = 3;
  s->ix2 = p->nx + 2;
  s->jy1 = 3;
  s->jy2 = p->ny + 2;
  s->kz1 = (p->ndim == 3) ? 3 : 1;
  s->kz2 = (p->ndim == 3) ? p->nz + 2 : 1;
  s->ndv = (p->ndim == 3) ? 7 : 5;
  s->nf = p->nfield;
  s->nc = p->curr_ndim;
  size_t ncell = (size_t)s->n1p * s->n2p * s->n3p;
  s->ebf = (double*)calloc(ncell * s->nf, sizeof(double));
  s->jc = (double*)calloc(ncell * s->nc, sizeof(double));
  int64_t maxcap = 1;
  for (int ic = 0; ic < 4; ++ic) {
    s->cap[ic] = p->capacity[ic] > 0 ? p->capacity[ic] : 1;
    if (ic < p->nsp) s->part[ic] = (double*)calloc((size_t)s->cap[ic] * s->ndv, sizeof(double));
    if (s->cap[ic] > maxcap) maxcap = s->cap[ic];
  }
  s->ebfp_cap = maxcap;
  s->ebfp = (double*)calloc((size_t)maxcap * s->ndv, sizeof(double));
  s->nsp_ionz = 1;
  s->nthreads = 1;
  return s;
}

void ora_destroy(ora_sim* s) {
  if (!s) return;
  free(s->ebf);
  free(s->jc);
  for (int ic = 0; ic < 4; ++ic) {
    free(s->part[ic]);
    free(s->wtab[ic]);
  }
  free(s->ebfp);
  free(s->env);
  free(s->av);
  free(s->ym3);
  free(s->ym4);
  free(s->zm3);
  free(s->zm4);
  free(s);
}

/* map2dy_part_sind / map2dz_part_sind (src/grid/stretched_grid.f90:45-143):
   a stretched coordinate in cells of the uniform computational grid. */
static double ora_str_inv(const agpu_stretch_axis* a, double yp) {
  return a->dli_inv * atan(a->ratio * (yp + a->cnst - a->xs)) + a->nl_stretch;
}
static double ora_str_map(const agpu_stretch_axis* a, double yp) {
  double yl;
  if (yp <= a->smin) {
    yl = ora_str_inv(a, yp) - a->init_cell;
  } else if (yp >= a->smax) {
    yp = 2 * 0.0 - yp;
    yl = ora_str_inv(a, yp);
    yl = (double)a->n - yl - a->init_cell;
  } else {
    yl = (yp + a->cnst) * a->dl_inv - a->init_cell;
  }
  return yl;
}
/* set_local_*_positions (grid_part_lib.f90:458-519) along y and z */
static inline double ora_ly(const ora_sim* s, double y) {
  return s->str ? ora_str_map(&s->sy, y) : s->p.dy_inv * (y - s->p.ymn);
}
static inline double ora_lz(const ora_sim* s, double z) {
  return s->str ? ora_str_map(&s->sz, z) : s->p.dz_inv * (z - s->p.zmn);
}
/* metric factors loc_yg(jj, 3|4), loc_zg(kk, 3|4) (1 on a uniform grid) */
static inline double ora_my(const ora_sim* s, int jj, int c) {
  return s->str ? (c == 3 ? s->ym3[jj] : s->ym4[jj]) : 1.0;
}
static inline double ora_mz(const ora_sim* s, int kk, int c) {
  return (s->str && s->p.ndim == 3) ? (c == 3 ? s->zm3[kk] : s->zm4[kk]) : 1.0;
}

int ora_set_stretch(ora_sim* s, const agpu_stretch* st) {
  if (!st->on) {
    s->str = 0;
    return 0;
  }
  if (st->y.n != s->p.ny || (s->p.ndim == 3 && st->z.n != s->p.nz)) return AGPU_E_ARG;
  const int ny = s->p.ny, nz = s->p.ndim == 3 ? s->p.nz : 0;
  free(s->ym3);
  free(s->ym4);
  free(s->zm3);
  free(s->zm4);
  s->ym3 = (double*)malloc(sizeof(double) * (size_t)(ny + 2));
  s->ym4 = (double*)malloc(sizeof(double) * (size_t)(ny + 2));
  memcpy(s->ym3, st->y.d1, sizeof(double) * (size_t)(ny + 2));
  memcpy(s->ym4, st->y.d1h, sizeof(double) * (size_t)(ny + 2));
  s->zm3 = s->zm4 = NULL;
  if (s->p.ndim == 3) {
    s->zm3 = (double*)malloc(sizeof(double) * (size_t)(nz + 2));
    s->zm4 = (double*)malloc(sizeof(double) * (size_t)(nz + 2));
    memcpy(s->zm3, st->z.d1, sizeof(double) * (size_t)(nz + 2));
    memcpy(s->zm4, st->z.d1h, sizeof(double) * (size_t)(nz + 2));
  }
  s->sy = st->y;
  s->sz = st->z;
  s->str = 1;
  return 0;
}

void ora_set_threads(ora_sim* s, int n) { s->nthreads = n > 0 ? n : 1; }

int ora_dims(const ora_sim* s, int* out) {
  out[0] = s->n1p; out[1] = s->n2p; out[2] = s->n3p;
  out[3] = s->ix1; out[4] = s->ix2; out[5] = s->jy1; out[6] = s->jy2;
  out[7] = s->kz1; out[8] = s->kz2; out[9] = s->ndv;
  return 0;
}

int ora_set_fields(ora_sim* s, const double* ebf) {
  memcpy(s->ebf, ebf, sizeof(double) * (size_t)s->n1p * s->n2p * s->n3p * s->nf);
  return 0;
}
int ora_get_fields(const ora_sim* s, double* ebf) {
  memcpy(ebf, s->ebf, sizeof(double) * (size_t)s->n1p * s->n2p * s->n3p * s->nf);
  return 0;
}
int ora_get_currents(const ora_sim* s, double* jc) {
  memcpy(jc, s->jc, sizeof(double) * (size_t)s->n1p * s->n2p * s->n3p * s->nc);
  return 0;
}
int ora_set_species(ora_sim* s, int ic, const double* part, int64_t ld, int64_t np) {
  if (ic < 0 || ic >= s->p.nsp || np > s->cap[ic]) return AGPU_E_ARG;
  for (int c = 0; c < s->ndv; ++c)
    memcpy(&s->part[ic][(size_t)c * s->cap[ic]], &part[(size_t)c * ld], sizeof(double) * (size_t)np);
  s->np[ic] = np;
  return 0;
}
int ora_get_species(const ora_sim* s, int ic, double* part, int64_t ld, int64_t* np) {
  if (ic < 0 || ic >= s->p.nsp) return AGPU_E_ARG;
  *np = s->np[ic];
  if (part)
    for (int c = 0; c < s->ndv; ++c)
      memcpy(&part[(size_t)c * ld], &s->part[ic][(size_t)c * s->cap[ic]], sizeof(double) * (size_t)s->np[ic]);
  return 0;
}
int64_t ora_count(const ora_sim* s, int ic) { return s->np[ic]; }
uint32_t ora_error_bits(const ora_sim* s) { return s->error_bits; }
double ora_xmn(const ora_sim* s) { return s->p.xmn; }

/* Window and injection state carried by a dump (dump_data / restart,
 * src/start/pic_dump.f90:35-380, 382-795): the window counter xlapse of
 * lp_window_xshift (window.f90:279-280; wi1 = nint(dx_inv*xlapse) follows
 * from it), the columns already injected nptx and the last target column
 * sptx_max (records 3-4 of Comm-data.bin), and the box origin (x(1), rdata(9)). */
void ora_get_window_state(const ora_sim* s, double* xlapse, int64_t* nptx, int64_t* sptx_max) {
  *xlapse = s->xlapse;
  for (int ic = 0; ic < 4; ++ic) {
    nptx[ic] = s->nptx[ic];
    sptx_max[ic] = s->sptx_max[ic];
  }
}
void ora_set_window_state(ora_sim* s, double xlapse, const int64_t* nptx) {
  s->xlapse = xlapse;
  s->wi1 = ora_nint(s->p.dx_inv * xlapse);
  for (int ic = 0; ic < 4; ++ic) s->nptx[ic] = nptx[ic];
}

/* ======================================================================== */
/* A1: field_xyzbd (src/parallel/mpi_field_interface.f90:53-198), ib = 0     */
/* ======================================================================== */
void ora_field_xyzbd(ora_sim* s, int nc) {
  int i1 = s->ix1, i2 = s->ix2, j1 = s->jy1, j2 = s->jy2, k1 = s->kz1, k2 = s->kz2;
  /* pex0, ibx < 2 */
  if (s->p.ibx < 2) {
    for (int ik = 1; ik <= nc; ++ik)
      for (int iz = k1; iz <= k2; ++iz)
        for (int iy = j1; iy <= j2; ++iy)
          EBF(s, s->ix1 - 1, iy, iz, ik) = 2. * EBF(s, s->ix1, iy, iz, ik) - EBF(s, s->ix1 + 1, iy, iz, ik);
  }
  i1 = i1 - 1;
  if (s->p.ibx == 0) {
    for (int ik = 1; ik <= nc; ++ik)
      for (int iz = k1; iz <= k2; ++iz)
        for (int iy = j1; iy <= j2; ++iy)
          EBF(s, s->ix2 + 1, iy, iz, ik) = 2. * EBF(s, s->ix2, iy, iz, ik) - EBF(s, s->ix2 - 1, iy, iz, ik);
  }
  i2 = i2 + 1;
  if (s->p.ndim < 2) return;
  if (s->p.iby == 0) {
    for (int ik = 1; ik <= nc; ++ik)
      for (int iz = k1; iz <= k2; ++iz)
        for (int ix = i1; ix <= i2; ++ix)
          EBF(s, ix, s->jy1 - 1, iz, ik) = 2. * EBF(s, ix, s->jy1, iz, ik) - EBF(s, ix, s->jy1 + 1, iz, ik);
  }
  j1 = j1 - 1;
  if (s->p.iby == 0) {
    for (int ik = 1; ik <= nc; ++ik)
      for (int iz = k1; iz <= k2; ++iz)
        for (int ix = i1; ix <= i2; ++ix)
          EBF(s, ix, s->jy2 + 1, iz, ik) = 2. * EBF(s, ix, s->jy2, iz, ik) - EBF(s, ix, s->jy2 - 1, iz, ik);
  }
  j2 = j2 + 1;
  if (s->p.ndim < 3) return;
  if (s->p.ibz == 0) {
    for (int ik = 1; ik <= nc; ++ik)
      for (int iy = j1; iy <= j2; ++iy)
        for (int ix = i1; ix <= i2; ++ix)
          EBF(s, ix, iy, s->kz1 - 1, ik) = 2 * EBF(s, ix, iy, s->kz1, ik) - EBF(s, ix, iy, s->kz1 + 1, ik);
    for (int ik = 1; ik <= nc; ++ik)
      for (int iy = j1; iy <= j2; ++iy)
        for (int ix = i1; ix <= i2; ++ix)
          EBF(s, ix, iy, s->kz2 + 1, ik) = 2 * EBF(s, ix, iy, s->kz2, ik) - EBF(s, ix, iy, s->kz2 - 1, ik);
  }
}

/* ======================================================================== */
/* A3 / A10 / qqh: spline shapes (src/particles/grid_part_lib.f90)          */
/* ======================================================================== */
/* qlh per dimension (qlh_2d_spline 110-143, qlh_3d_spline 212-259):
   quadratic weights on integer nodes, linear on half nodes; ix-1. */
static inline void ora_qlh_1d(double xp, double ax[3], double axh[2], int* ix) {
  double xx = shx + xp;
  int i = (int)(xx + 0.5);
  double sx = xx - (double)i;
  double sx2 = sx * sx;
  ax[1] = 0.75 - sx2;
  ax[2] = 0.5 * (0.25 + sx2 + sx);
  ax[0] = 1. - ax[1] - ax[2];
  axh[1] = sx + 0.5;
  axh[0] = 1. - axh[1];
  *ix = i - 1;
}
/* qqh per dimension (qqh_2d_spline 170-210, qqh_3d_spline 261-320). */
static inline void ora_qqh_1d(double xp, double ax[3], double axh[3], int* ix, int* ihx) {
  double xx = shx + xp;
  int i = (int)(xx + 0.5);
  double sx = xx - (double)i;
  double sx2 = sx * sx;
  ax[1] = 0.75 - sx2;
  ax[2] = 0.5 * (0.25 + sx2 + sx);
  ax[0] = 1. - ax[1] - ax[2];
  int ih = (int)(xx);
  sx = xx - (double)ih - 0.5;
  sx2 = sx * sx;
  axh[1] = 0.75 - sx2;
  axh[2] = 0.5 * (0.25 + sx2 + sx);
  axh[0] = 1. - axh[1] - axh[2];
  *ix = i - 1;
  *ihx = ih - 1;
}
/* qden per dimension (qden_2d_wgh 337-358, qden_3d_wgh 388-417): no ix-1. */
static inline void ora_qden_1d(double xp, double ax[3], int* ix) {
  double xx = shx + xp;
  int i = (int)(xx + 0.5);
  double sx = xx - (double)i;
  double sx2 = sx * sx;
  ax[1] = 0.75 - sx2;
  ax[2] = 0.5 * (0.25 + sx2 + sx);
  ax[0] = 1. - ax[1] - ax[2];
  *ix = i;
}

/* Exported for the shape invariant tests. */
void ora_shape_qlh(double xp, double* ax3, double* axh2, int* ix) { ora_qlh_1d(xp, ax3, axh2, ix); }
void ora_shape_qqh(double xp, double* ax3, double* axh3, int* ix, int* ih) { ora_qqh_1d(xp, ax3, axh3, ix, ih); }
void ora_shape_qden(double xp, double* ax3, int* ix) { ora_qden_1d(xp, ax3, ix); }

/* ======================================================================== */
/* A2 + A4/A5: gather (set_part2d_hcell_acc grid_part_connect.f90:89-185,    */
/* set_part3d_hcell_acc 187-285) with set_local_*_positions (lib 458-519)   */
/* ======================================================================== */
static void ora_gather(ora_sim* s, int ic, int64_t np) {
  const agpu_params* p = &s->p;
  if (p->ndim == 2) {
    #pragma omp parallel for schedule(static) num_threads(s->nthreads) if (s->nthreads > 1)
    for (int64_t n = 1; n <= np; ++n) {
      double xl = p->dx_inv * (PART(s, ic, n, 1) - p->xmn);
      double yl = ora_ly(s, PART(s, ic, n, 2));
      double ax1[3], axh[2], ay1[3], ayh[2];
      int i, j;
      ora_qlh_1d(xl, ax1, axh, &i);
      ora_qlh_1d(yl, ay1, ayh, &j);
      int ih = i, jh = j;
      double ap1 = 0., ap2 = 0., ap3 = 0.;
      for (int j1 = 0; j1 <= 2; ++j1) {
        int j2 = j + j1;
        double dvol = ay1[j1];
        for (int i1 = 0; i1 <= 1; ++i1) {
          int i2 = i1 + ih;
          double dvol1 = axh[i1] * dvol;
          ap1 = ap1 + dvol1 * EBF(s, i2, j2, 1, 1);
        }
      }
      for (int j1 = 0; j1 <= 1; ++j1) {
        int j2 = jh + j1;
        double dvol = ayh[j1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          int i2 = i + i1;
          double dvol1 = ax1[i1] * dvol;
          ap2 = ap2 + dvol1 * EBF(s, i2, j2, 1, 2);
        }
        for (int i1 = 0; i1 <= 1; ++i1) {
          int i2 = i1 + ih;
          double dvol1 = axh[i1] * dvol;
          ap3 = ap3 + dvol1 * EBF(s, i2, j2, 1, 3);
        }
      }
      PT(s, n, 1) = ap1;
      PT(s, n, 2) = ap2;
      PT(s, n, 3) = ap3;
    }
    return;
  }
  #pragma omp parallel for schedule(static) num_threads(s->nthreads) if (s->nthreads > 1)
  for (int64_t n = 1; n <= np; ++n) {
    double xl = p->dx_inv * (PART(s, ic, n, 1) - p->xmn);
    double yl = ora_ly(s, PART(s, ic, n, 2));
    double zl = ora_lz(s, PART(s, ic, n, 3));
    double ax1[3], axh[2], ay1[3], ayh[2], az1[3], azh[2];
    int i, j, k;
    ora_qlh_1d(xl, ax1, axh, &i);
    ora_qlh_1d(yl, ay1, ayh, &j);
    ora_qlh_1d(zl, az1, azh, &k);
    int ih = i, jh = j, kh = k;
    double ap[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int k1 = 0; k1 <= 2; ++k1) {
      int k2 = k + k1;
      for (int j1 = 0; j1 <= 2; ++j1) {
        int j2 = j + j1;
        double dvol = ay1[j1] * az1[k1];
        for (int i1 = 0; i1 <= 1; ++i1) {
          int i2 = i1 + ih;
          ap[1] = ap[1] + axh[i1] * dvol * EBF(s, i2, j2, k2, 1);
        }
      }
      for (int j1 = 0; j1 <= 1; ++j1) {
        int j2 = jh + j1;
        double dvol = ayh[j1] * az1[k1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          int i2 = i + i1;
          ap[2] = ap[2] + ax1[i1] * dvol * EBF(s, i2, j2, k2, 2);
        }
        for (int i1 = 0; i1 <= 1; ++i1) {
          int i2 = i1 + ih;
          ap[6] = ap[6] + axh[i1] * dvol * EBF(s, i2, j2, k2, 6);
        }
      }
    }
    for (int k1 = 0; k1 <= 1; ++k1) {
      int k2 = kh + k1;
      for (int j1 = 0; j1 <= 1; ++j1) {
        int j2 = jh + j1;
        double dvol = ayh[j1] * azh[k1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          int i2 = i1 + i;
          ap[4] = ap[4] + ax1[i1] * dvol * EBF(s, i2, j2, k2, 4);
        }
      }
      for (int j1 = 0; j1 <= 2; ++j1) {
        int j2 = j + j1;
        double dvol = ay1[j1] * azh[k1];
        for (int i1 = 0; i1 <= 1; ++i1) {
          int i2 = ih + i1;
          ap[5] = ap[5] + axh[i1] * dvol * EBF(s, i2, j2, k2, 5);
        }
        for (int i1 = 0; i1 <= 2; ++i1) {
          int i2 = i1 + i;
          ap[3] = ap[3] + ax1[i1] * dvol * EBF(s, i2, j2, k2, 3);
        }
      }
    }
    for (int c = 1; c <= 6; ++c) PT(s, n, c) = ap[c];
  }
}

/* A6: field_charge_multiply (src/dynamics/curr_and_fields_util.f90:58-72) */
static void ora_field_charge_multiply(ora_sim* s, int ic, int64_t np) {
  int ch = s->ndv;
  #pragma omp parallel for schedule(static) num_threads(s->nthreads) if (s->nthreads > 1)
  for (int64_t n = 1; n <= np; ++n) {
    ora_pack w = ora_unpack(PART(s, ic, n, ch));
    double q = (double)w.charge;
    for (int c = 1; c <= s->nf; ++c) PT(s, n, c) = q * PT(s, n, c);
  }
}

/* A7: init_lpf_momenta (src/dynamics/boris_push.f90:34-73) */
static void ora_init_lpf_momenta(ora_sim* s, int ic, int64_t np) {
  double dth_lp = 0.5 * s->p.dt;
  double alp = dth_lp * s->p.lorentz_fact[ic];
  if (s->p.curr_ndim == 2) {
    #pragma omp parallel for schedule(static) num_threads(s->nthreads) if (s->nthreads > 1)
    for (int64_t p = 1; p <= np; ++p) {
      double efp[3];
      for (int c = 0; c < 3; ++c) efp[c] = -alp * PT(s, p, c + 1);
      double pp1 = PART(s, ic, p, 3), pp2 = PART(s, ic, p, 4);
      double gam2 = 1. + (pp1 * pp1 + pp2 * pp2);
      double gam_inv = 1. / sqrt(gam2);
      double vp1 = pp1 * gam_inv, vp2 = pp2 * gam_inv;
      PART(s, ic, p, 3) = PART(s, ic, p, 3) + efp[0] + vp2 * efp[2];
      PART(s, ic, p, 4) = PART(s, ic, p, 4) + efp[1] - vp1 * efp[2];
    }
    return;
  }
  #pragma omp parallel for schedule(static) num_threads(s->nthreads) if (s->nthreads > 1)
  for (int64_t p = 1; p <= np; ++p) {
    double pp[3] = {PART(s, ic, p, 4), PART(s, ic, p, 5), PART(s, ic, p, 6)};
    double efp[6];
    for (int c = 0; c < 6; ++c) efp[c] = -alp * PT(s, p, c + 1);
    double gam2 = 1. + (pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2]);
    double gam_inv = 1. / sqrt(gam2);
    double vp[3] = {gam_inv * pp[0], gam_inv * pp[1], gam_inv * pp[2]};
    PART(s, ic, p, 4) = PART(s, ic, p, 4) + efp[0] + vp[1] * efp[5] - vp[2] * efp[4];
    PART(s, ic, p, 5) = PART(s, ic, p, 5) + efp[1] + vp[2] * efp[3] - vp[0] * efp[5];
    PART(s, ic, p, 6) = PART(s, ic, p, 6) + efp[2] + vp[0] * efp[4] - vp[1] * efp[3];
  }
}

/* A8: lpf_momenta_and_positions (src/dynamics/boris_push.f90:75-168) */
static void ora_push(ora_sim* s, int ic, int64_t np) {
  double dt_lp = s->p.dt;
  double dth_lp = 0.5 * dt_lp;
  double alp = dth_lp * s->p.lorentz_fact[ic];
  int ch;
  if (s->p.curr_ndim == 2) {
    ch = 5;
    #pragma omp parallel for schedule(static) num_threads(s->nthreads) if (s->nthreads > 1)
    for (int64_t p = 1; p <= np; ++p) {
      double pp1 = PART(s, ic, p, 3), pp2 = PART(s, ic, p, 4);
      double efp1 = alp * PT(s, p, 1), efp2 = alp * PT(s, p, 2), efp3 = alp * PT(s, p, 3);
      double vp1 = pp1 + efp1, vp2 = pp2 + efp2, vp3 = efp3;
      double gam02 = 1. + (vp1 * vp1 + vp2 * vp2);
      double b2 = vp3 * vp3;
      gam02 = gam02 - b2;
      double gam2 = 0.5 * (gam02 + sqrt(gam02 * gam02 + 4. * b2));
      double gam = sqrt(gam2);
      double vph1 = gam2 * vp1 + gam * vp2 * vp3;
      double vph2 = gam2 * vp2 - gam * vp1 * vp3;
      vph1 = vph1 / (gam2 + b2);
      vph2 = vph2 / (gam2 + b2);
      PART(s, ic, p, 3) = 2. * vph1 - pp1;
      PART(s, ic, p, 4) = 2. * vph2 - pp2;
      PT(s, p, 3) = PART(s, ic, p, 1);
      PT(s, p, 4) = PART(s, ic, p, 2);
      pp1 = PART(s, ic, p, 3);
      pp2 = PART(s, ic, p, 4);
      gam2 = 1. + (pp1 * pp1 + pp2 * pp2);
      PT(s, p, 5) = dt_lp / sqrt(gam2);
      vp1 = PT(s, p, 5) * pp1;
      vp2 = PT(s, p, 5) * pp2;
      PT(s, p, 1) = vp1;
      PT(s, p, 2) = vp2;
      PART(s, ic, p, 1) = PART(s, ic, p, 1) + vp1;
      PART(s, ic, p, 2) = PART(s, ic, p, 2) + vp2;
    }
  } else {
    ch = 7;
    #pragma omp parallel for schedule(static) num_threads(s->nthreads) if (s->nthreads > 1)
    for (int64_t p = 1; p <= np; ++p) {
      double pp[3] = {PART(s, ic, p, 4), PART(s, ic, p, 5), PART(s, ic, p, 6)};
      double efp[6];
      for (int c = 0; c < 6; ++c) efp[c] = alp * PT(s, p, c + 1);
      double vp[3] = {pp[0] + efp[0], pp[1] + efp[1], pp[2] + efp[2]};
      double bb[3] = {efp[3], efp[4], efp[5]};
      double gam02 = 1. + (vp[0] * vp[0] + vp[1] * vp[1] + vp[2] * vp[2]);
      double b2 = bb[0] * bb[0] + bb[1] * bb[1] + bb[2] * bb[2];
      double bv = bb[0] * vp[0] + bb[1] * vp[1] + bb[2] * vp[2];
      gam02 = gam02 - b2;
      double gam2 = 0.5 * (gam02 + sqrt(gam02 * gam02 + 4. * (b2 + bv * bv)));
      double gam = sqrt(gam2);
      double vph[3];
      for (int c = 0; c < 3; ++c) vph[c] = gam2 * vp[c] + bb[c] * bv;
      vph[0] = vph[0] + gam * (vp[1] * bb[2] - vp[2] * bb[1]);
      vph[1] = vph[1] + gam * (vp[2] * bb[0] - vp[0] * bb[2]);
      vph[2] = vph[2] + gam * (vp[0] * bb[1] - vp[1] * bb[0]);
      for (int c = 0; c < 3; ++c) vph[c] = vph[c] / (b2 + gam2);
      for (int c = 0; c < 3; ++c) PART(s, ic, p, 4 + c) = 2. * vph[c] - pp[c];
      for (int c = 0; c < 3; ++c) PT(s, p, 4 + c) = PART(s, ic, p, 1 + c);
      for (int c = 0; c < 3; ++c) pp[c] = PART(s, ic, p, 4 + c);
      gam2 = 1. + (pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2]);
      PT(s, p, 7) = dt_lp / sqrt(gam2);
      for (int c = 0; c < 3; ++c) vp[c] = PT(s, p, 7) * pp[c];
      for (int c = 0; c < 3; ++c) PT(s, p, 1 + c) = vp[c];
      for (int c = 0; c < 3; ++c) PART(s, ic, p, 1 + c) = PART(s, ic, p, 1 + c) + vp[c];
    }
  }
  if (s->p.iform < 2)
    for (int64_t p = 1; p <= np; ++p) PT(s, p, ch) = PART(s, ic, p, ch);
  /* comoving frame (vbeam = -w_speed > 0): x -= dt vbeam (boris_push.f90:161-166) */
  const double vbeam = s->p.w_speed < 0.0 ? -s->p.w_speed : 0.0;
  if (vbeam > 0.)
    for (int64_t p = 1; p <= np; ++p) {
      PART(s, ic, p, 1) = PART(s, ic, p, 1) - dt_lp * vbeam;
      PT(s, p, 1) = PT(s, p, 1) - dt_lp * vbeam;
    }
}

/* A9: cell_part_dist(.false.) single domain -> reset_all_part_dist
   (src/parallel/mpi_part_interface.f90:467-523, 525-753): stable removal of
   particles outside (gmin, gmax] along x, then y, then z; spec and ebfp
   compacted together. Returns the number removed. */
static int64_t ora_reset_dist(ora_sim* s, int ic, int cin, double xl, double xr, int with_pt) {
  int64_t np = s->np[ic], pout = 0;
  for (int64_t n = 1; n <= np; ++n) {
    double xp = PART(s, ic, n, cin);
    if (xp <= xl) pout++;
    if (xp > xr) pout++;
  }
  if (pout == 0) return 0;
  int64_t q = 0;
  for (int64_t n = 1; n <= np; ++n) {
    double xp = PART(s, ic, n, cin);
    if (xp > xl && xp <= xr) {
      q++;
      if (q != n) {
        for (int c = 1; c <= s->ndv; ++c) PART(s, ic, q, c) = PART(s, ic, n, c);
        if (with_pt)
          for (int c = 1; c <= s->ndv; ++c) PT(s, q, c) = PT(s, n, c);
      }
    }
  }
  s->np[ic] = q;
  return np - q;
}

static int64_t ora_cell_part_dist_step(ora_sim* s, int ic) {
  int64_t r = 0;
  r += ora_reset_dist(s, ic, 1, s->p.gxmin, s->p.gxmax, 1);
  r += ora_reset_dist(s, ic, 2, s->p.gymin, s->p.gymax, 1);
  if (s->p.ndim > 2) r += ora_reset_dist(s, ic, 3, s->p.gzmin, s->p.gzmax, 1);
  return r;
}

/* ======================================================================== */
/* A11/A12: Esirkepov deposit (grid_part_connect.f90:956-1334)              */
/* ======================================================================== */
static void ora_esirkepov_2d_one(ora_sim* s, double* jc, const double xp1[2], const double xp0[2],
                                 float wght) {
  double ax0[3], ay0[3], ax1[3], ay1[3];
  double axh[5], ayh[5], currx[5], curry[5];
  int i, j, ii0, jj0;
  ora_qden_1d(xp0[0], ax0, &ii0);
  ora_qden_1d(xp0[1], ay0, &jj0);
  ora_qden_1d(xp1[0], ax1, &i);
  ora_qden_1d(xp1[1], ay1, &j);
  /* a move of more than one node has no window slot: flagged, not deposited */
  if ((unsigned)(i - ii0 + 1) > 2u || (unsigned)(j - jj0 + 1) > 2u) {
    s->error_bits |= AGPU_EBIT_INDEX;
    return;
  }
  for (int q = 0; q < 5; ++q) axh[q] = 0.;
  int ih = i - ii0 + 1;
  for (int i1 = 0; i1 <= 2; ++i1) axh[ih + i1] = ax1[i1];
  currx[0] = -axh[0];
  for (int i1 = 1; i1 <= 3; ++i1) currx[i1] = currx[i1 - 1] + ax0[i1 - 1] - axh[i1];
  currx[4] = currx[3] - axh[4];
  for (int i1 = 1; i1 <= 3; ++i1) axh[i1] = axh[i1] + ax0[i1 - 1];
  for (int q = 0; q < 5; ++q) currx[q] = (double)wght * currx[q];
  int x0 = ih < 1 ? ih : 1;
  int x1 = (ih + 2) > 3 ? ih + 2 : 3;
  int jh = j - jj0 + 1;
  for (int q = 0; q < 5; ++q) ayh[q] = 0.;
  for (int i1 = 0; i1 <= 2; ++i1) ayh[jh + i1] = ay1[i1];
  curry[0] = -ayh[0];
  for (int i1 = 1; i1 <= 3; ++i1) curry[i1] = curry[i1 - 1] + ay0[i1 - 1] - ayh[i1];
  curry[4] = curry[3] - ayh[4];
  for (int q = 0; q < 5; ++q) curry[q] = (double)wght * curry[q];
  for (int i1 = 1; i1 <= 3; ++i1) ayh[i1] = ayh[i1] + ay0[i1 - 1];
  int y0 = jh < 1 ? jh : 1;
  int y1 = (jh + 2) > 3 ? jh + 2 : 3;
  jj0 = jj0 - 1;
  j = j - 1;
  jh = jj0 - 1;
  i = i - 1;
  ii0 = ii0 - 1;
  ih = ii0 - 1;
  size_t n1p = (size_t)s->n1p, n2p = (size_t)s->n2p;
  size_t comp = n1p * n2p * (size_t)s->n3p;
  for (int j1 = y0; j1 <= y1; ++j1) {
    int j2 = jh + j1;
    for (int i1 = x0; i1 <= x1; ++i1) {
      int i2 = ih + i1;
      size_t o = (size_t)(i2 - 1) + n1p * (size_t)(j2 - 1);
      jc[o] = jc[o] + ayh[j1] * currx[i1];
    }
  }
  for (int j1 = y0; j1 <= y1; ++j1) {
    int j2 = jh + j1;
    for (int i1 = x0; i1 <= x1; ++i1) {
      int i2 = ih + i1;
      size_t o = comp + (size_t)(i2 - 1) + n1p * (size_t)(j2 - 1);
      jc[o] = jc[o] + axh[i1] * curry[j1];
    }
  }
}

static void ora_esirkepov_3d_one(ora_sim* s, double* jc, const double xp1[3], const double xp0[3],
                                 float wght) {
  double ax0[3], ay0[3], az0[3], ax1[3], ay1[3], az1[3];
  double axh[5], ayh[5], azh[5], axh0[5], axh1[5], ayh0[5], ayh1[5];
  double currx[5], curry[5], currz[5];
  int i, j, k, ii0, jj0, kk0;
  ora_qden_1d(xp0[0], ax0, &ii0);
  ora_qden_1d(xp0[1], ay0, &jj0);
  ora_qden_1d(xp0[2], az0, &kk0);
  ora_qden_1d(xp1[0], ax1, &i);
  ora_qden_1d(xp1[1], ay1, &j);
  ora_qden_1d(xp1[2], az1, &k);
  /* a move of more than one node has no window slot: flagged, not deposited */
  if ((unsigned)(i - ii0 + 1) > 2u || (unsigned)(j - jj0 + 1) > 2u || (unsigned)(k - kk0 + 1) > 2u) {
    s->error_bits |= AGPU_EBIT_INDEX;
    return;
  }

  for (int q = 0; q < 5; ++q) axh[q] = 0.;
  int ih = i - ii0 + 1;
  for (int i1 = 0; i1 <= 2; ++i1) axh[ih + i1] = ax1[i1];
  currx[0] = -axh[0];
  for (int i1 = 1; i1 <= 3; ++i1) currx[i1] = currx[i1 - 1] + ax0[i1 - 1] - axh[i1];
  currx[4] = currx[3] - axh[4];
  for (int q = 0; q < 5; ++q) currx[q] = (double)wght * currx[q];
  for (int q = 0; q < 5; ++q) {
    axh0[q] = 0.5 * axh[q];
    axh1[q] = axh[q];
  }
  for (int i1 = 1; i1 <= 3; ++i1) {
    axh0[i1] = axh0[i1] + ax0[i1 - 1];
    axh1[i1] = axh1[i1] + 0.5 * ax0[i1 - 1];
  }
  int x0 = ih < 1 ? ih : 1;
  int x1 = (ih + 2) > 3 ? ih + 2 : 3;
  i = i - 1;
  ii0 = ii0 - 1;

  int jh = j - jj0 + 1;
  for (int q = 0; q < 5; ++q) ayh[q] = 0.;
  for (int i1 = 0; i1 <= 2; ++i1) ayh[jh + i1] = ay1[i1];
  curry[0] = -ayh[0];
  for (int i1 = 1; i1 <= 3; ++i1) curry[i1] = curry[i1 - 1] + ay0[i1 - 1] - ayh[i1];
  curry[4] = curry[3] - ayh[4];
  for (int q = 0; q < 5; ++q) curry[q] = (double)wght * curry[q];
  for (int q = 0; q < 5; ++q) {
    ayh0[q] = 0.5 * ayh[q];
    ayh1[q] = ayh[q];
  }
  for (int i1 = 1; i1 <= 3; ++i1) {
    ayh0[i1] = ayh0[i1] + ay0[i1 - 1];
    ayh1[i1] = ayh1[i1] + 0.5 * ay0[i1 - 1];
  }
  int y0 = jh < 1 ? jh : 1;
  int y1 = (jh + 2) > 3 ? jh + 2 : 3;
  jj0 = jj0 - 1;
  j = j - 1;

  int kh = k - kk0 + 1;
  for (int q = 0; q < 5; ++q) azh[q] = 0.;
  for (int i1 = 0; i1 <= 2; ++i1) azh[kh + i1] = az1[i1];
  currz[0] = -azh[0];
  for (int i1 = 1; i1 <= 3; ++i1) currz[i1] = currz[i1 - 1] + az0[i1 - 1] - azh[i1];
  currz[4] = currz[3] - azh[4];
  for (int q = 0; q < 5; ++q) currz[q] = (double)wght * currz[q];
  kk0 = kk0 - 1;
  k = k - 1;
  int z0 = kh < 1 ? kh : 1;
  int z1 = (kh + 2) > 3 ? kh + 2 : 3;

  size_t n1p = (size_t)s->n1p, n2p = (size_t)s->n2p, n3p = (size_t)s->n3p;
  size_t comp = n1p * n2p * n3p;
#define JIX(i2, j2, k2, c) ((size_t)((i2)-1) + n1p * ((size_t)((j2)-1) + n2p * (size_t)((k2)-1)) + comp * (size_t)(c))
  jh = jj0 - 1;
  ih = ii0 - 1;
  for (int k1 = 0; k1 <= 2; ++k1) {
    for (int j1 = y0; j1 <= y1; ++j1) {
      int j2 = jh + j1;
      double dvol = ayh0[j1] * az0[k1];
      double dvolh = ayh1[j1] * az1[k1];
      for (int i1 = x0; i1 <= x1; ++i1) {
        int i2 = ih + i1;
        size_t o0 = JIX(i2, j2, kk0 + k1, 0), o1 = JIX(i2, j2, k + k1, 0);
        jc[o0] = jc[o0] + dvol * currx[i1];
        jc[o1] = jc[o1] + dvolh * currx[i1];
      }
    }
  }
  for (int k1 = 0; k1 <= 2; ++k1) {
    for (int j1 = y0; j1 <= y1; ++j1) {
      int j2 = jh + j1;
      double dvol = curry[j1] * az0[k1];
      double dvolh = curry[j1] * az1[k1];
      for (int i1 = x0; i1 <= x1; ++i1) {
        int i2 = ih + i1;
        size_t o0 = JIX(i2, j2, kk0 + k1, 1), o1 = JIX(i2, j2, k + k1, 1);
        jc[o0] = jc[o0] + axh0[i1] * dvol;
        jc[o1] = jc[o1] + axh1[i1] * dvolh;
      }
    }
  }
  kh = kk0 - 1;
  for (int k1 = z0; k1 <= z1; ++k1) {
    int k2 = kh + k1;
    for (int j1 = 0; j1 <= 2; ++j1) {
      double dvol = ay0[j1] * currz[k1];
      double dvolh = ay1[j1] * currz[k1];
      for (int i1 = x0; i1 <= x1; ++i1) {
        int i2 = ih + i1;
        size_t o0 = JIX(i2, jj0 + j1, k2, 2), o1 = JIX(i2, j + j1, k2, 2);
        jc[o0] = jc[o0] + axh0[i1] * dvol;
        jc[o1] = jc[o1] + axh1[i1] * dvolh;
      }
    }
  }
#undef JIX
}

/* curr_accumulate -> esirkepov_{2,3}d_curr with the set_local_positions
   preamble (curr_and_fields_util.f90:74-102; grid_part_connect.f90:979-987,
   1201-1208): new positions from part, old positions from ebfp, weight
   wght = real(charge*wgh, sp). */
/* ======================================================================== */
/* Cubic shape extension (AGPU_SHAPE_CUBIC).  No counterpart in the         */
/* reference, which gathers and deposits with quadratic shapes only; the     */
/* cubic B-spline weights are those of its charge-density helper            */
/* cden_3d_wgh (grid_part_lib.f90:419-454), the half-node weights those of   */
/* qqh (170-210), and the deposit is Esirkepov's scheme with 4-point shapes  */
/* on 6-slot windows, written in the same regrouped form as the quadratic   */
/* one: J = curr(u) * (S0-plane term + S1-plane term).                      */
/* ======================================================================== */
static const double ora_one_sixth = 1.0 / 6.0, ora_two_third = 2.0 / 3.0;
/* cubic weights on integer nodes i-1..i+2, i = int(3 + x) */
static inline void ora_cden_1d(double xp, double a[4], int* ix) {
  double xx = shx + xp;
  int i = (int)xx;
  double sx = xx - (double)i;
  double sx2 = sx * sx;
  double sx3 = sx2 * sx;
  a[1] = ora_two_third - sx2 + 0.5 * sx3;
  a[2] = ora_one_sixth + 0.5 * (sx + sx2 - sx3);
  a[3] = ora_one_sixth * sx3;
  a[0] = 1. - a[1] - a[2] - a[3];
  *ix = i;
}
/* quadratic weights on half nodes h-1..h+1 (index m stands for m + 1/2) */
static inline void ora_qhalf_1d(double xp, double a[3], int* ih) {
  double xx = shx + xp;
  int h = (int)xx;
  double sx = xx - (double)h - 0.5;
  double sx2 = sx * sx;
  a[1] = 0.75 - sx2;
  a[2] = 0.5 * (0.25 + sx2 + sx);
  a[0] = 1. - a[1] - a[2];
  *ih = h;
}
void ora_shape_cubic(double xp, double* a4, double* ah3, int* ix, int* ih) {
  ora_cden_1d(xp, a4, ix);
  ora_qhalf_1d(xp, ah3, ih);
}

/* Gather with cubic (integer) x quadratic (half) weights; the staggering of
   set_part3d_hcell_acc / set_part2d_hcell_acc.  Product order per point:
   (w_x * (w_y * w_z)) * F. */
static void ora_gather_cubic(ora_sim* s, int ic, int64_t np) {
  const agpu_params* p = &s->p;
  #pragma omp parallel for schedule(static) num_threads(s->nthreads) if (s->nthreads > 1)
  for (int64_t n = 1; n <= np; ++n) {
    double xl = p->dx_inv * (PART(s, ic, n, 1) - p->xmn);
    double yl = p->dy_inv * (PART(s, ic, n, 2) - p->ymn);
    double ax[4], ay[4], az[4] = {0., 1., 0., 0.}, axh[3], ayh[3], azh[3] = {0., 1., 0.};
    int fx, fy, fz = 2, hx, hy, hz = 1;
    ora_cden_1d(xl, ax, &fx);
    ora_qhalf_1d(xl, axh, &hx);
    ora_cden_1d(yl, ay, &fy);
    ora_qhalf_1d(yl, ayh, &hy);
    int nzi = 1, nzh = 1, kz0 = 1, kh0 = 1;
    if (p->ndim == 3) {
      double zl = p->dz_inv * (PART(s, ic, n, 3) - p->zmn);
      ora_cden_1d(zl, az, &fz);
      ora_qhalf_1d(zl, azh, &hz);
      nzi = 4;
      nzh = 3;
      kz0 = fz - 1;
      kh0 = hz - 1;
    }
    const int ix0 = fx - 1, iy0 = fy - 1, hx0 = hx - 1, hy0 = hy - 1;
    const double* wzi = (p->ndim == 3) ? az : az + 1;
    const double* wzh = (p->ndim == 3) ? azh : azh + 1;
    double ap[6] = {0., 0., 0., 0., 0., 0.};
    /* Ex(i+1/2, j, k) */
    for (int k1 = 0; k1 < nzi; ++k1)
      for (int j1 = 0; j1 < 4; ++j1) {
        double dvol = ay[j1] * wzi[k1];
        for (int i1 = 0; i1 < 3; ++i1) ap[0] += (axh[i1] * dvol) * EBF(s, hx0 + i1, iy0 + j1, kz0 + k1, 1);
      }
    /* Ey(i, j+1/2, k) */
    for (int k1 = 0; k1 < nzi; ++k1)
      for (int j1 = 0; j1 < 3; ++j1) {
        double dvol = ayh[j1] * wzi[k1];
        for (int i1 = 0; i1 < 4; ++i1) ap[1] += (ax[i1] * dvol) * EBF(s, ix0 + i1, hy0 + j1, kz0 + k1, 2);
      }
    if (p->ndim == 2) {
      /* Bz(i+1/2, j+1/2) */
      for (int j1 = 0; j1 < 3; ++j1) {
        double dvol = ayh[j1];
        for (int i1 = 0; i1 < 3; ++i1) ap[2] += (axh[i1] * dvol) * EBF(s, hx0 + i1, hy0 + j1, 1, 3);
      }
      PT(s, n, 1) = ap[0];
      PT(s, n, 2) = ap[1];
      PT(s, n, 3) = ap[2];
      continue;
    }
    /* Ez(i, j, k+1/2) */
    for (int k1 = 0; k1 < 3; ++k1)
      for (int j1 = 0; j1 < 4; ++j1) {
        double dvol = ay[j1] * azh[k1];
        for (int i1 = 0; i1 < 4; ++i1) ap[2] += (ax[i1] * dvol) * EBF(s, ix0 + i1, iy0 + j1, kh0 + k1, 3);
      }
    /* Bx(i, j+1/2, k+1/2) */
    for (int k1 = 0; k1 < 3; ++k1)
      for (int j1 = 0; j1 < 3; ++j1) {
        double dvol = ayh[j1] * azh[k1];
        for (int i1 = 0; i1 < 4; ++i1) ap[3] += (ax[i1] * dvol) * EBF(s, ix0 + i1, hy0 + j1, kh0 + k1, 4);
      }
    /* By(i+1/2, j, k+1/2) */
    for (int k1 = 0; k1 < 3; ++k1)
      for (int j1 = 0; j1 < 4; ++j1) {
        double dvol = ay[j1] * azh[k1];
        for (int i1 = 0; i1 < 3; ++i1) ap[4] += (axh[i1] * dvol) * EBF(s, hx0 + i1, iy0 + j1, kh0 + k1, 5);
      }
    /* Bz(i+1/2, j+1/2, k) */
    for (int k1 = 0; k1 < 4; ++k1)
      for (int j1 = 0; j1 < 3; ++j1) {
        double dvol = ayh[j1] * az[k1];
        for (int i1 = 0; i1 < 3; ++i1) ap[5] += (axh[i1] * dvol) * EBF(s, hx0 + i1, hy0 + j1, kz0 + k1, 6);
      }
    for (int c = 0; c < 6; ++c) PT(s, n, 1 + c) = ap[c];
  }
}

/* 1-D part of the cubic Esirkepov deposit: old shape on slots 1..4 (slot 0
   = old floor node - 2), new shape on slots sh..sh+3 (sh = new floor - old
   floor + 1, in 0..2), the running current on the 6 slots, and the slot
   range lo..hi the particle touches. */
static void ora_cubic_window(double x0l, double x1l, double s0[6], double s1[6], double cur[6], int* base, int* lo,
                             int* hi) {
  double a0[4], a1[4];
  int f0, f1;
  ora_cden_1d(x0l, a0, &f0);
  ora_cden_1d(x1l, a1, &f1);
  int sh = f1 - f0 + 1;
  for (int q = 0; q < 6; ++q) {
    s0[q] = 0.;
    s1[q] = 0.;
  }
  for (int q = 0; q < 4; ++q) s0[q + 1] = a0[q];
  if (sh >= 0 && sh <= 2)
    for (int q = 0; q < 4; ++q) s1[q + sh] = a1[q];
  cur[0] = s0[0] - s1[0];
  for (int q = 1; q < 6; ++q) cur[q] = cur[q - 1] + s0[q] - s1[q];
  *base = f0 - 2;
  *lo = sh < 1 ? sh : 1;
  *hi = (sh + 3) > 4 ? sh + 3 : 4;
}

static inline int ora_in_box(const ora_sim* s, int i, int j, int k) {
  return i >= 1 && i <= s->n1p && j >= 1 && j <= s->n2p && k >= 1 && k <= s->n3p;
}

static void ora_esirkepov_cubic_2d_one(ora_sim* s, double* jc, const double xp1[2], const double xp0[2], float wght) {
  double sx0[6], sx1[6], cx[6], sy0[6], sy1[6], cy[6];
  int bx, x0, x1, by, y0, y1;
  ora_cubic_window(xp0[0], xp1[0], sx0, sx1, cx, &bx, &x0, &x1);
  ora_cubic_window(xp0[1], xp1[1], sy0, sy1, cy, &by, &y0, &y1);
  size_t n1p = (size_t)s->n1p, comp = n1p * (size_t)s->n2p * (size_t)s->n3p;
  for (int v = y0; v <= y1; ++v)
    for (int u = x0; u <= x1; ++u) {
      int i = bx + u, j = by + v;
      if (!ora_in_box(s, i, j, 1)) {
        s->error_bits |= AGPU_EBIT_INDEX;
        continue;
      }
      size_t o = (size_t)(i - 1) + n1p * (size_t)(j - 1);
      jc[o] = jc[o] + ((double)wght * cx[u]) * (sy0[v] + sy1[v]);
      jc[comp + o] = jc[comp + o] + (sx0[u] + sx1[u]) * ((double)wght * cy[v]);
    }
}

static void ora_esirkepov_cubic_3d_one(ora_sim* s, double* jc, const double xp1[3], const double xp0[3], float wght) {
  double sx0[6], sx1[6], cx[6], sy0[6], sy1[6], cy[6], sz0[6], sz1[6], cz[6];
  int bx, x0, x1, by, y0, y1, bz, z0, z1;
  ora_cubic_window(xp0[0], xp1[0], sx0, sx1, cx, &bx, &x0, &x1);
  ora_cubic_window(xp0[1], xp1[1], sy0, sy1, cy, &by, &y0, &y1);
  ora_cubic_window(xp0[2], xp1[2], sz0, sz1, cz, &bz, &z0, &z1);
  double wx0[6], wx1[6], wy0[6], wy1[6];
  for (int q = 0; q < 6; ++q) {
    wx0[q] = 0.5 * sx1[q] + sx0[q];
    wx1[q] = sx1[q] + 0.5 * sx0[q];
    wy0[q] = 0.5 * sy1[q] + sy0[q];
    wy1[q] = sy1[q] + 0.5 * sy0[q];
  }
  size_t n1p = (size_t)s->n1p, n2p = (size_t)s->n2p, comp = n1p * n2p * (size_t)s->n3p;
  for (int w = z0; w <= z1; ++w)
    for (int v = y0; v <= y1; ++v)
      for (int u = x0; u <= x1; ++u) {
        int i = bx + u, j = by + v, k = bz + w;
        if (!ora_in_box(s, i, j, k)) {
          s->error_bits |= AGPU_EBIT_INDEX;
          continue;
        }
        size_t o = (size_t)(i - 1) + n1p * ((size_t)(j - 1) + n2p * (size_t)(k - 1));
        jc[o] = jc[o] + ((double)wght * cx[u]) * (wy0[v] * sz0[w] + wy1[v] * sz1[w]);
        jc[comp + o] = jc[comp + o] + ((double)wght * cy[v]) * (wx0[u] * sz0[w] + wx1[u] * sz1[w]);
        jc[2 * comp + o] = jc[2 * comp + o] + ((double)wght * cz[w]) * (wx0[u] * sy0[v] + wx1[u] * sy1[v]);
      }
}

/* iform = 2: ncdef_2d_curr / ncdef_3d_curr (grid_part_connect.f90:1338-1512):
   half of q w dt v (dt / gamma = the push's ebfp(ch), kept when iform = 2) on
   the qlh shapes at the old and at the new position. */
static void ora_ncdef_3d_one(ora_sim* s, double* jc, const double xp1[3], const double xp0[3], const double pv[3],
                             float wght, double dtg) {
  double ax0[3], ay0[3], az0[3], axh0[2], ayh0[2], azh0[2];
  double ax1[3], ay1[3], az1[3], axh1[2], ayh1[2], azh1[2];
  int ii0, jj0, kk0, i, j, k;
  const double gam_inv = (double)wght * dtg;
  double vp[3];
  for (int c = 0; c < 3; ++c) vp[c] = 0.5 * gam_inv * pv[c];
  ora_qlh_1d(xp0[0], ax0, axh0, &ii0);
  ora_qlh_1d(xp0[1], ay0, ayh0, &jj0);
  ora_qlh_1d(xp0[2], az0, azh0, &kk0);
  ora_qlh_1d(xp1[0], ax1, axh1, &i);
  ora_qlh_1d(xp1[1], ay1, ayh1, &j);
  ora_qlh_1d(xp1[2], az1, azh1, &k);
  const size_t c3 = (size_t)s->n1p * s->n2p * s->n3p;
  double* jx = jc;
  double* jy = jc + c3;
  double* jz = jc + 2 * c3;
#define ORA_O(ii, jj, kk) (((size_t)(ii)-1) + (size_t)s->n1p * (((size_t)(jj)-1) + (size_t)s->n2p * ((size_t)(kk)-1)))
  for (int k1 = 0; k1 <= 2; ++k1) {
    for (int j1 = 0; j1 <= 2; ++j1) {
      double dvol = vp[0] * ay1[j1] * az1[k1];
      for (int i1 = 0; i1 <= 1; ++i1) jx[ORA_O(i + i1, j + j1, k + k1)] += dvol * axh1[i1];
    }
    for (int j1 = 0; j1 <= 2; ++j1) {
      double dvol = vp[0] * ay0[j1] * az0[k1];
      for (int i1 = 0; i1 <= 1; ++i1) jx[ORA_O(ii0 + i1, jj0 + j1, kk0 + k1)] += dvol * axh0[i1];
    }
  }
  for (int k1 = 0; k1 <= 2; ++k1) {
    for (int j1 = 0; j1 <= 1; ++j1) {
      double dvol = vp[1] * ayh0[j1] * az0[k1];
      for (int i1 = 0; i1 <= 2; ++i1) jy[ORA_O(ii0 + i1, jj0 + j1, kk0 + k1)] += dvol * ax0[i1];
    }
    for (int j1 = 0; j1 <= 1; ++j1) {
      double dvol = vp[1] * ayh1[j1] * az1[k1];
      for (int i1 = 0; i1 <= 2; ++i1) jy[ORA_O(i + i1, j + j1, k + k1)] += dvol * ax1[i1];
    }
  }
  for (int k1 = 0; k1 <= 1; ++k1) {
    for (int j1 = 0; j1 <= 2; ++j1) {
      double dvol = vp[2] * ay0[j1] * azh0[k1];
      for (int i1 = 0; i1 <= 2; ++i1) jz[ORA_O(ii0 + i1, jj0 + j1, kk0 + k1)] += dvol * ax0[i1];
    }
    for (int j1 = 0; j1 <= 2; ++j1) {
      double dvol = vp[2] * ay1[j1] * azh1[k1];
      for (int i1 = 0; i1 <= 2; ++i1) jz[ORA_O(i + i1, j + j1, k + k1)] += dvol * ax1[i1];
    }
  }
}
static void ora_ncdef_2d_one(ora_sim* s, double* jc, const double xp1[2], const double xp0[2], double p1, double p2,
                             float wght, double dtg) {
  double ax0[3], ay0[3], axh0[2], ayh0[2], ax1[3], ay1[3], axh1[2], ayh1[2];
  int ii0, jj0, i, j;
  double vp1 = (double)wght * dtg * p1, vp2 = (double)wght * dtg * p2;
  vp1 = 0.5 * vp1;
  vp2 = 0.5 * vp2;
  ora_qlh_1d(xp0[0], ax0, axh0, &ii0);
  ora_qlh_1d(xp0[1], ay0, ayh0, &jj0);
  ora_qlh_1d(xp1[0], ax1, axh1, &i);
  ora_qlh_1d(xp1[1], ay1, ayh1, &j);
  const size_t c3 = (size_t)s->n1p * s->n2p * s->n3p;
  double* jx = jc;
  double* jy = jc + c3;
  for (int j1 = 0; j1 <= 2; ++j1) {
    double dvol = vp1 * ay1[j1];
    for (int i1 = 0; i1 <= 1; ++i1) jx[ORA_O(i + i1, j + j1, 1)] += dvol * axh1[i1];
    dvol = vp1 * ay0[j1];
    for (int i1 = 0; i1 <= 1; ++i1) jx[ORA_O(ii0 + i1, jj0 + j1, 1)] += dvol * axh0[i1];
  }
  for (int j1 = 0; j1 <= 1; ++j1) {
    double dvol = vp2 * ayh0[j1];
    for (int i1 = 0; i1 <= 2; ++i1) jy[ORA_O(ii0 + i1, jj0 + j1, 1)] += dvol * ax0[i1];
    dvol = vp2 * ayh1[j1];
    for (int i1 = 0; i1 <= 2; ++i1) jy[ORA_O(i + i1, j + j1, 1)] += dvol * ax1[i1];
  }
#undef ORA_O
}

static void ora_curr_accumulate(ora_sim* s, int ic, int64_t np) {
  const agpu_params* p = &s->p;
  int nth = s->nthreads;
  size_t jsz = (size_t)s->n1p * s->n2p * s->n3p * s->nc;
  double** priv = NULL;
  if (nth > 1) {
    priv = (double**)calloc((size_t)nth, sizeof(double*));
    for (int t = 1; t < nth; ++t) priv[t] = (double*)calloc(jsz, sizeof(double));
    priv[0] = s->jc;
  }
#ifdef _OPENMP
#pragma omp parallel num_threads(nth) if (nth > 1)
#endif
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* jc = (nth > 1) ? priv[tid] : s->jc;
    int64_t lo = 1, hi = np;
    if (nth > 1) {
      int64_t chunk = (np + nth - 1) / nth;
      lo = 1 + (int64_t)tid * chunk;
      hi = lo + chunk - 1;
      if (hi > np) hi = np;
    }
    for (int64_t n = lo; n <= hi; ++n) {
      ora_pack w = ora_unpack(PART(s, ic, n, s->ndv));
      float wght = (float)w.charge * w.wgh;
      if (p->ndim == 2) {
        double xp1[2] = {p->dx_inv * (PART(s, ic, n, 1) - p->xmn), ora_ly(s, PART(s, ic, n, 2))};
        double xp0[2] = {p->dx_inv * (PT(s, n, 3) - p->xmn), ora_ly(s, PT(s, n, 4))};
        if (p->iform == 2)
          ora_ncdef_2d_one(s, jc, xp1, xp0, PART(s, ic, n, 3), PART(s, ic, n, 4), wght, PT(s, n, 5));
        else if (p->shape == AGPU_SHAPE_CUBIC)
          ora_esirkepov_cubic_2d_one(s, jc, xp1, xp0, wght);
        else
          ora_esirkepov_2d_one(s, jc, xp1, xp0, wght);
      } else {
        double xp1[3] = {p->dx_inv * (PART(s, ic, n, 1) - p->xmn), ora_ly(s, PART(s, ic, n, 2)),
                         ora_lz(s, PART(s, ic, n, 3))};
        double xp0[3] = {p->dx_inv * (PT(s, n, 4) - p->xmn), ora_ly(s, PT(s, n, 5)), ora_lz(s, PT(s, n, 6))};
        if (p->iform == 2) {
          const double pv[3] = {PART(s, ic, n, 4), PART(s, ic, n, 5), PART(s, ic, n, 6)};
          ora_ncdef_3d_one(s, jc, xp1, xp0, pv, wght, PT(s, n, 7));
        } else if (p->shape == AGPU_SHAPE_CUBIC)
          ora_esirkepov_cubic_3d_one(s, jc, xp1, xp0, wght);
        else
          ora_esirkepov_3d_one(s, jc, xp1, xp0, wght);
      }
    }
  }
  if (nth > 1) {
    for (int t = 1; t < nth; ++t) {
      for (size_t q = 0; q < jsz; ++q) s->jc[q] += priv[t][q];
      free(priv[t]);
    }
    free(priv);
  }
}

/* Deposit of one particle move for the continuity tests: positions in grid
   units (local, as set_local_positions returns them). */
void ora_deposit_move(ora_sim* s, const double* xnew, const double* xold, float wght) {
  const int cubic = s->p.shape == AGPU_SHAPE_CUBIC;
  if (s->p.ndim == 2) {
    if (cubic) ora_esirkepov_cubic_2d_one(s, s->jc, xnew, xold, wght);
    else ora_esirkepov_2d_one(s, s->jc, xnew, xold, wght);
  } else {
    if (cubic) ora_esirkepov_cubic_3d_one(s, s->jc, xnew, xold, wght);
    else ora_esirkepov_3d_one(s, s->jc, xnew, xold, wght);
  }
}
void ora_zero_currents(ora_sim* s) { memset(s->jc, 0, sizeof(double) * (size_t)s->n1p * s->n2p * s->n3p * s->nc); }

/* Charge density of one particle with the qden shapes into rho(n1p,n2p,n3p)
   (the density the Esirkepov scheme conserves; grid_part_lib.f90:337-417). */
void ora_rho_one(const ora_sim* s, double* rho, const double* xl, double wght) {
  if (s->p.shape == AGPU_SHAPE_CUBIC) {
    /* cubic density: nodes i-1..i+2 of the floor node i (cden_*_wgh) */
    double cx[4], cy[4], cz[4] = {1, 0, 0, 0};
    int i, j, k = 2, nzc = 1;
    ora_cden_1d(xl[0], cx, &i);
    ora_cden_1d(xl[1], cy, &j);
    if (s->p.ndim == 3) {
      ora_cden_1d(xl[2], cz, &k);
      nzc = 4;
    }
    size_t n1p = (size_t)s->n1p, n2p = (size_t)s->n2p;
    for (int k1 = 0; k1 < nzc; ++k1)
      for (int j1 = 0; j1 < 4; ++j1)
        for (int i1 = 0; i1 < 4; ++i1) {
          int i2 = i - 1 + i1, j2 = j - 1 + j1, k2 = (s->p.ndim == 3) ? k - 1 + k1 : 1;
          rho[(size_t)(i2 - 1) + n1p * ((size_t)(j2 - 1) + n2p * (size_t)(k2 - 1))] += wght * cx[i1] * cy[j1] * cz[k1];
        }
    return;
  }
  double ax[3], ay[3], az[3] = {1, 0, 0};
  int i, j, k = 1;
  ora_qden_1d(xl[0], ax, &i);
  ora_qden_1d(xl[1], ay, &j);
  int nz = 1;
  if (s->p.ndim == 3) {
    ora_qden_1d(xl[2], az, &k);
    nz = 3;
  }
  size_t n1p = (size_t)s->n1p, n2p = (size_t)s->n2p;
  for (int k1 = 0; k1 < nz; ++k1)
    for (int j1 = 0; j1 < 3; ++j1)
      for (int i1 = 0; i1 < 3; ++i1) {
        int i2 = i - 1 + i1, j2 = j - 1 + j1, k2 = (s->p.ndim == 3) ? k - 1 + k1 : 1;
        rho[(size_t)(i2 - 1) + n1p * ((size_t)(j2 - 1) + n2p * (size_t)(k2 - 1))] += wght * ax[i1] * ay[j1] * az[k1];
      }
}

/* ======================================================================== */
/* A13: curr_mpi_collect -> jc_xyzbd + djc (curr_and_fields_util.f90:104-152,*/
/* src/parallel/mpi_curr_interface.f90:551-643), ib = 0                      */
/* ======================================================================== */
static void ora_jc_xyzbd(ora_sim* s) {
  int i1 = s->ix1, n1 = s->ix2, j1 = s->jy1, n2 = s->jy2, k1 = s->kz1, n3 = s->kz2;
  int nc = s->nc;
  if (s->p.ibx == 0) {
    for (int ik = 1; ik <= nc; ++ik)
      for (int k = k1; k <= n3; ++k)
        for (int j = j1; j <= n2; ++j) {
          JC(s, i1, j, k, ik) = JC(s, i1, j, k, ik) + JC(s, i1 - 1, j, k, ik);
          JC(s, i1 - 1, j, k, ik) = 0.0;
          JC(s, n1, j, k, ik) = JC(s, n1, j, k, ik) + JC(s, n1 + 1, j, k, ik) + JC(s, n1 + 2, j, k, ik);
          JC(s, n1 + 1, j, k, ik) = 0.0;
          JC(s, n1 + 2, j, k, ik) = 0.0;
        }
  }
  if (s->p.ndim < 2) return;
  if (s->p.iby == 0) {
    for (int ik = 1; ik <= nc; ++ik)
      for (int iz = k1; iz <= n3; ++iz)
        for (int ix = i1; ix <= n1; ++ix) {
          JC(s, ix, j1, iz, ik) = JC(s, ix, j1, iz, ik) + JC(s, ix, j1 - 1, iz, ik) + JC(s, ix, j1 - 2, iz, ik);
          JC(s, ix, j1 - 2, iz, ik) = 0.0;
          JC(s, ix, j1 - 1, iz, ik) = 0.0;
        }
    for (int ik = 1; ik <= nc; ++ik)
      for (int iz = k1; iz <= n3; ++iz)
        for (int ix = i1; ix <= n1; ++ix) {
          JC(s, ix, n2, iz, ik) = JC(s, ix, n2, iz, ik) + JC(s, ix, n2 + 1, iz, ik) + JC(s, ix, n2 + 2, iz, ik);
          JC(s, ix, n2 + 1, iz, ik) = 0.0;
          JC(s, ix, n2 + 2, iz, ik) = 0.0;
        }
  }
  if (s->p.ndim < 3) return;
  if (s->p.ibz == 0) {
    for (int ik = 1; ik <= nc; ++ik)
      for (int iy = j1; iy <= n2; ++iy)
        for (int ix = i1; ix <= n1; ++ix) {
          JC(s, ix, iy, k1, ik) = JC(s, ix, iy, k1, ik) + JC(s, ix, iy, k1 - 1, ik);
          JC(s, ix, iy, k1 - 1, ik) = 0.0;
        }
    for (int ik = 1; ik <= nc; ++ik)
      for (int iy = j1; iy <= n2; ++iy)
        for (int ix = i1; ix <= n1; ++ix) {
          JC(s, ix, iy, n3, ik) = JC(s, ix, iy, n3, ik) + JC(s, ix, iy, n3 + 1, ik) + JC(s, ix, iy, n3 + 2, ik);
          JC(s, ix, iy, n3 + 1, ik) = 0.0;
          JC(s, ix, iy, n3 + 2, ik) = 0.0;
        }
  }
}

static void ora_curr_collect(ora_sim* s) {
  ora_jc_xyzbd(s);
  if (s->p.iform < 2) {
    size_t comp = (size_t)s->n1p * s->n2p * s->n3p;
    for (int i = 1; i <= s->p.ndim; ++i) {
      double d = s->p.djc[i - 1];
      double* c = s->jc + comp * (size_t)(i - 1);
      for (size_t q = 0; q < comp; ++q) c[q] = d * c[q];
    }
  }
  if (!s->str) return;
  /* stretched grid (curr_and_fields_util.f90:120-150): dery, derhy (2D);
     dery derz, derhy derz, dery derhz (3D) on the interior */
  if (s->nc == 2) {
    for (int k = s->kz1; k <= s->kz2; ++k)
      for (int j = s->jy1; j <= s->jy2; ++j) {
        const int jj = j - 2;
        const double dery = s->ym3[jj], derhy = s->ym4[jj];
        for (int i = s->ix1; i <= s->ix2; ++i) {
          JC(s, i, j, k, 1) = dery * JC(s, i, j, k, 1);
          JC(s, i, j, k, 2) = derhy * JC(s, i, j, k, 2);
        }
      }
    return;
  }
  for (int k = s->kz1; k <= s->kz2; ++k) {
    const int kk = k - 2;
    const double derz = s->zm3[kk], derhz = s->zm4[kk];
    for (int j = s->jy1; j <= s->jy2; ++j) {
      const int jj = j - 2;
      const double dery = s->ym3[jj], derhy = s->ym4[jj];
      for (int i = s->ix1; i <= s->ix2; ++i) {
        JC(s, i, j, k, 1) = dery * derz * JC(s, i, j, k, 1);
        JC(s, i, j, k, 2) = derhy * derz * JC(s, i, j, k, 2);
        JC(s, i, j, k, 3) = dery * derhz * JC(s, i, j, k, 3);
      }
    }
  }
}

/* ======================================================================== */
/* A14: advance_lpf_fields (curr_and_fields_util.f90:176-260) with ef_bds,   */
/* bf_bds, rote, rotb (src/fields/grid_fields.f90:1069-1552); loc_xg is 1  */
/* (x is never stretched), loc_yg/loc_zg are 1 unless the grid is stretched. */
/* ======================================================================== */
static void ora_ef_bds(ora_sim* s, double dtl, int imbd) {
  int nf = s->nf;
  int ix2 = s->ix2, jy2 = s->jy2, kz2 = s->kz2;
  double aphx, aphy, aphz;
  if (s->p.ibx < 2 && s->p.ibx == 0) {
    aphx = 1.0 * s->p.dx_inv * dtl;
    for (int k = s->kz1; k <= kz2; ++k)
      for (int j = s->jy1; j <= jy2; ++j)
        EBF(s, ix2 + 1, j, k, 2) = (2. * EBF(s, ix2, j, k, nf) - (1. - aphx) * EBF(s, ix2, j, k, 2)) / (1. + aphx);
    if (nf > 3)
      for (int k = s->kz1; k <= kz2; ++k)
        for (int j = s->jy1; j <= jy2; ++j)
          EBF(s, ix2 + 1, j, k, 3) = -(2. * EBF(s, ix2, j, k, 5) + (1. - aphx) * EBF(s, ix2, j, k, 3)) / (1. + aphx);
  }
  if (s->p.ndim < 2) return;
  if (s->p.iby < 2 && imbd == 0) {
    aphy = ora_my(s, jy2 - 2, 4) * s->p.dy_inv * dtl;
    for (int k = s->kz1; k <= kz2; ++k)
      for (int i = s->ix1; i <= ix2; ++i)
        EBF(s, i, jy2 + 1, k, 1) = -(2. * EBF(s, i, jy2, k, nf) + (1. - aphy) * EBF(s, i, jy2, k, 1)) / (1. + aphy);
    if (nf > 3)
      for (int k = s->kz1; k <= kz2; ++k)
        for (int i = s->ix1; i <= ix2; ++i)
          EBF(s, i, jy2 + 1, k, 3) = (2. * EBF(s, i, jy2, k, 4) - (1. - aphy) * EBF(s, i, jy2, k, 3)) / (1. + aphy);
  }
  if (s->p.ndim < 3) return;
  if (s->p.ibz < 2 && imbd == 0) {
    aphz = ora_mz(s, s->p.nz, 4) * s->p.dz_inv * dtl;
    for (int j = s->jy1; j <= jy2; ++j)
      for (int i = s->ix1; i <= ix2; ++i) {
        EBF(s, i, j, kz2 + 1, 1) = (2. * EBF(s, i, j, kz2, 5) - (1. - aphz) * EBF(s, i, j, kz2, 1)) / (1. + aphz);
        EBF(s, i, j, kz2 + 1, 2) = -(2. * EBF(s, i, j, kz2, 4) + (1. - aphz) * EBF(s, i, j, kz2, 2)) / (1. + aphz);
      }
  }
}

static void ora_bf_bds(ora_sim* s, double dtl, int imbd) {
  int nf = s->nf;
  int ix1 = s->ix1, jy1 = s->jy1, kz1 = s->kz1;
  double aphx, aphy, aphz;
  if (s->p.ibx < 2) {
    aphx = 1.0 * s->p.dx_inv * dtl;
    for (int k = s->kz1; k <= s->kz2; ++k)
      for (int j = s->jy1; j <= s->jy2; ++j)
        EBF(s, ix1 - 1, j, k, nf) = -(2. * EBF(s, ix1, j, k, 2) + (1. - aphx) * EBF(s, ix1, j, k, nf)) / (1. + aphx);
    if (nf > 3)
      for (int k = s->kz1; k <= s->kz2; ++k)
        for (int j = s->jy1; j <= s->jy2; ++j)
          EBF(s, ix1 - 1, j, k, 5) = (2. * EBF(s, ix1, j, k, 3) - (1. - aphx) * EBF(s, ix1, j, k, 5)) / (1. + aphx);
  }
  if (s->p.ndim < 2) return;
  if (s->p.iby < 2 && imbd == 0) {
    aphy = ora_my(s, 1, 3) * s->p.dy_inv * dtl;
    for (int k = s->kz1; k <= s->kz2; ++k)
      for (int i = s->ix1; i <= s->ix2; ++i) {
        EBF(s, i, jy1 - 1, k, nf) = 2. * EBF(s, i, jy1, k, 1) - (1. - aphy) * EBF(s, i, jy1, k, nf);
        EBF(s, i, jy1 - 1, k, nf) = EBF(s, i, jy1 - 1, k, nf) / (1. + aphy);
      }
    if (nf > 3)
      for (int k = s->kz1; k <= s->kz2; ++k)
        for (int i = s->ix1; i <= s->ix2; ++i) {
          EBF(s, i, jy1 - 1, k, 4) = -2. * EBF(s, i, jy1, k, 3) - (1. - aphy) * EBF(s, i, jy1, k, 4);
          EBF(s, i, jy1 - 1, k, 4) = EBF(s, i, jy1 - 1, k, 4) / (1. + aphy);
        }
  }
  if (s->p.ndim < 3) return;
  if (s->p.ibz < 2 && imbd == 0) {
    aphz = ora_mz(s, 1, 3) * s->p.dz_inv * dtl;
    for (int j = s->jy1; j <= s->jy2; ++j)
      for (int i = s->ix1; i <= s->ix2; ++i) {
        EBF(s, i, j, kz1 - 1, 4) = 2. * EBF(s, i, j, kz1, 2) - (1. - aphz) * EBF(s, i, j, kz1, 4);
        EBF(s, i, j, kz1 - 1, 4) = EBF(s, i, j, kz1 - 1, 4) / (1. + aphz);
        EBF(s, i, j, kz1 - 1, 5) = -2. * EBF(s, i, j, kz1, 1) - (1. - aphz) * EBF(s, i, j, kz1, 5);
        EBF(s, i, j, kz1 - 1, 5) = EBF(s, i, j, kz1 - 1, 5) / (1. + aphz);
      }
  }
}

static void ora_rote(ora_sim* s, double dtf) {
  int nf = s->nf;
  double aphx = dtf * s->p.dx_inv, aphy = dtf * s->p.dy_inv, aphz = dtf * s->p.dz_inv;
  double aph1 = aphx * s->p.se_coeff[0], aph2 = aphx * s->p.se_coeff[1];
  for (int k = s->kz1; k <= s->kz2; ++k)
    for (int j = s->jy1; j <= s->jy2; ++j) {
      double sdhy = ora_my(s, j - 2, 4) * aphy;
      for (int i = s->ix1; i <= s->ix2; ++i)
        EBF(s, i, j, k, nf) = EBF(s, i, j, k, nf) - aph1 * (EBF(s, i + 1, j, k, 2) - EBF(s, i, j, k, 2)) +
                              sdhy * (EBF(s, i, j + 1, k, 1) - EBF(s, i, j, k, 1)) -
                              aph2 * (EBF(s, i + 2, j, k, 2) - EBF(s, i - 1, j, k, 2));
    }
  if (nf < 6) return;
  for (int k = s->kz1; k <= s->kz2; ++k) {
    double sdhz = ora_mz(s, k - 2, 4) * aphz;
    for (int j = s->jy1; j <= s->jy2; ++j) {
      double sdhy = ora_my(s, j - 2, 4) * aphy;
      for (int i = s->ix1; i <= s->ix2; ++i) {
        EBF(s, i, j, k, 4) = EBF(s, i, j, k, 4) - sdhy * (EBF(s, i, j + 1, k, 3) - EBF(s, i, j, k, 3)) +
                             sdhz * (EBF(s, i, j, k + 1, 2) - EBF(s, i, j, k, 2));
        EBF(s, i, j, k, 5) = EBF(s, i, j, k, 5) + aph1 * (EBF(s, i + 1, j, k, 3) - EBF(s, i, j, k, 3)) -
                             sdhz * (EBF(s, i, j, k + 1, 1) - EBF(s, i, j, k, 1)) +
                             aph2 * (EBF(s, i + 2, j, k, 3) - EBF(s, i - 1, j, k, 3));
      }
    }
  }
}

static void ora_rotb(ora_sim* s, double dtf) {
  int nf = s->nf;
  double aphx = dtf * s->p.dx_inv, aphy = dtf * s->p.dy_inv, aphz = dtf * s->p.dz_inv;
  double aph1 = aphx * s->p.se_coeff[0], aph2 = aphx * s->p.se_coeff[1];
  for (int k = s->kz1; k <= s->kz2; ++k)
    for (int j = s->jy1; j <= s->jy2; ++j) {
      double sdy = ora_my(s, j - 2, 3) * aphy;
      for (int i = s->ix1; i <= s->ix2; ++i) {
        EBF(s, i, j, k, 1) = EBF(s, i, j, k, 1) + sdy * (EBF(s, i, j, k, nf) - EBF(s, i, j - 1, k, nf));
        EBF(s, i, j, k, 2) = EBF(s, i, j, k, 2) - aph1 * (EBF(s, i, j, k, nf) - EBF(s, i - 1, j, k, nf)) -
                             aph2 * (EBF(s, i + 1, j, k, nf) - EBF(s, i - 2, j, k, nf));
      }
    }
  if (nf < 6) return;
  for (int k = s->kz1; k <= s->kz2; ++k) {
    double sdz = aphz * ora_mz(s, k - 2, 3);
    for (int j = s->jy1; j <= s->jy2; ++j) {
      double sdy = aphy * ora_my(s, j - 2, 3);
      for (int i = s->ix1; i <= s->ix2; ++i) {
        EBF(s, i, j, k, 1) = EBF(s, i, j, k, 1) - sdz * (EBF(s, i, j, k, 5) - EBF(s, i, j, k - 1, 5));
        EBF(s, i, j, k, 2) = EBF(s, i, j, k, 2) + sdz * (EBF(s, i, j, k, 4) - EBF(s, i, j, k - 1, 4));
        EBF(s, i, j, k, 3) = EBF(s, i, j, k, 3) + aph1 * (EBF(s, i, j, k, 5) - EBF(s, i - 1, j, k, 5)) -
                             sdy * (EBF(s, i, j, k, 4) - EBF(s, i, j - 1, k, 4)) +
                             aph2 * (EBF(s, i + 1, j, k, 5) - EBF(s, i - 2, j, k, 5));
      }
    }
  }
}

/* field_xadvect (src/fields/grid_fields.f90:210-324), one rank: the x
   ghosts ix1-1 and ix2+1 copy ix1+1 and ix2, then along each row
   i = ix1..ix2 either the explicit step f_i - aphx_exp (f_{i+1} - f_{i-1})
   (isch 0) or the implicit one (isch 2), the tridiagonal solve of
   aphx_exp (f'_{i+1} - f'_{i-1}) + f'_i = f_i by trid_der1
   (grid_fields.f90:37-77) with b1 = bn = 1, c1 = an = 0;
   aphx_exp = v_adv dth dx_inv / 2. */
static void ora_field_xadvect(ora_sim* s, double dth, double v_adv, int ic1, int ic2, int isch) {
  const double aphx = dth * s->p.dx_inv;
  const double aphx_exp = 0.5 * v_adv * aphx;
  const int i1 = s->ix1, n1p = s->ix2, n = n1p - i1 + 1;
  for (int ic = ic1; ic <= ic2; ++ic)
    for (int k = s->kz1; k <= s->kz2; ++k)
      for (int j = s->jy1; j <= s->jy2; ++j) EBF(s, i1 - 1, j, k, ic) = EBF(s, i1 + 1, j, k, ic);
  for (int ic = ic1; ic <= ic2; ++ic)
    for (int k = s->kz1; k <= s->kz2; ++k)
      for (int j = s->jy1; j <= s->jy2; ++j) EBF(s, n1p + 1, j, k, ic) = EBF(s, n1p, j, k, ic);
  double* w0 = (double*)malloc(sizeof(double) * (size_t)(n + 2));
  double* w1 = (double*)malloc(sizeof(double) * (size_t)(n + 2));
  for (int ic = ic1; ic <= ic2; ++ic)
    for (int k = s->kz1; k <= s->kz2; ++k)
      for (int j = s->jy1; j <= s->jy2; ++j) {
        if (isch == 0) {
          for (int i = i1; i <= n1p; ++i)
            w0[i - 2] = EBF(s, i, j, k, ic) - aphx_exp * (EBF(s, i + 1, j, k, ic) - EBF(s, i - 1, j, k, ic));
        } else {
          const double a = -aphx_exp, b = 1., c = -a, b1 = 1., c1 = 0.0, an = 0.0, bn = 1.;
          for (int i = i1; i <= n1p; ++i) w0[i - 2] = EBF(s, i, j, k, ic);
          w1[1] = 0.0;
          double bet = b1;
          w0[1] = w0[1] / bet;
          int kk = 2;
          w1[kk] = c1 / bet;
          bet = b - a * w1[kk];
          w0[kk] = (w0[kk] - a * w0[kk - 1]) / bet;
          for (kk = 3; kk <= n - 1; ++kk) {
            w1[kk] = c / bet;
            bet = b - a * w1[kk];
            w0[kk] = (w0[kk] - a * w0[kk - 1]) / bet;
          }
          kk = n;
          w1[kk] = c / bet;
          bet = bn - an * w1[kk];
          w0[kk] = (w0[kk] - an * w0[kk - 1]) / bet;
          for (kk = n - 1; kk >= 1; --kk) w0[kk] = w0[kk] - w1[kk + 1] * w0[kk + 1];
        }
        for (int i = i1; i <= n1p; ++i) EBF(s, i, j, k, ic) = w0[i - 2];
      }
  free(w0);
  free(w1);
}

void ora_advance_fields(ora_sim* s) {
  double dt_lp = s->p.dt;
  double dth = 0.5 * dt_lp;
  /* comoving frame (vbeam = -w_speed > 0): the advection substeps of
     advance_lpf_fields (curr_and_fields_util.f90:200-258) */
  const int comoving = s->p.w_speed < 0.0;
  const double vbeam = comoving ? -s->p.w_speed : 0.0;
  ora_ef_bds(s, 0.0, 0);
  if (comoving) ora_field_xadvect(s, dth, -vbeam, s->nc + 1, s->nf, 0);
  ora_rote(s, dth);
  ora_bf_bds(s, dt_lp, 0);
  if (comoving) ora_field_xadvect(s, dth, -vbeam, 1, s->nc, 0);
  ora_rotb(s, dt_lp);
  for (int ik = 1; ik <= s->nc; ++ik)
    for (int k = s->kz1; k <= s->kz2; ++k)
      for (int j = s->jy1; j <= s->jy2; ++j)
        for (int i = s->ix1; i <= s->ix2; ++i)
          EBF(s, i, j, k, ik) = EBF(s, i, j, k, ik) - s->p.ompe * JC(s, i, j, k, ik);
  if (comoving) ora_field_xadvect(s, dth, -vbeam, 1, s->nc, 2);
  ora_ef_bds(s, dt_lp, 0);
  ora_rote(s, dth);
  if (comoving) ora_field_xadvect(s, dth, -vbeam, s->nc + 1, s->nf, 2);
}

/* Exposed for tests: field-only pieces. */
void ora_field_bd(ora_sim* s) { ora_field_xyzbd(s, s->nf); }
void ora_field_xadvect_once(ora_sim* s, double dth, double v_adv, int ic1, int ic2, int isch) {
  ora_field_xadvect(s, dth, v_adv, ic1, ic2, isch);
}
void ora_set_currents(ora_sim* s, const double* jc) {
  memcpy(s->jc, jc, sizeof(double) * (size_t)s->n1p * s->n2p * s->n3p * s->nc);
}
void ora_curr_fold(ora_sim* s) { ora_curr_collect(s); }

/* ======================================================================== */
/* A21 / window source: lattice plasma (the build's jittered stand-in for     */
/* the reference's regular (i-1/2)/n lattice, init_part_distrib.f90:152-203) */
/* ======================================================================== */
static void ora_lattice_particle(const ora_sim* s, int ic, int64_t ixl, int j, int k, double* x, double* y,
                                 double* z) {
  const agpu_plasma* src = &s->src[ic];
  double dxl = s->p.dx / (double)src->npx;
  double dyl = s->p.dy / (double)src->npy;
  double dzl = s->p.dz / (double)src->npz;
  uint32_t ctr[4] = {(uint32_t)ixl, (uint32_t)j, (uint32_t)k, (uint32_t)ic};
  uint32_t r[4];
  ora_philox4x32_10(ctr, (uint32_t)src->seed, (uint32_t)(src->seed >> 32), r);
  double jx = src->jitter * (ora_u32(r[0]) - 0.5);
  double jy = src->jitter * (ora_u32(r[1]) - 0.5);
  double jz = src->jitter * (ora_u32(r[2]) - 0.5);
  *x = src->x_start + ((double)ixl - 0.5 + jx) * dxl;
  *y = src->y_min + ((double)j - 0.5 + jy) * dyl;
  *z = (s->p.ndim == 3) ? src->z_min + ((double)k - 0.5 + jz) * dzl : 0.0;
}

int ora_set_plasma_source(ora_sim* s, const agpu_plasma* src) {
  int ic = src->ic;
  if (ic < 0 || ic >= s->p.nsp) return AGPU_E_ARG;
  s->src[ic] = *src;
  s->has_src[ic] = 1;
  s->nptx[ic] = 0;
  double dxl = s->p.dx / (double)src->npx;
  double dyl = s->p.dy / (double)src->npy;
  double dzl = s->p.dz / (double)src->npz;
  s->sptx_max[ic] = (int64_t)floor((src->x_end - src->x_start) / dxl + 1e-9);
  s->npty[ic] = (int)floor((src->y_max - src->y_min) / dyl + 1e-9);
  s->nptz[ic] = (s->p.ndim == 3) ? (int)floor((src->z_max - src->z_min) / dzl + 1e-9) : 1;
  return 0;
}

/* add_particles (src/dynamics/window.f90:39-104): k, j, ix order with x
   fastest; momenta zero; the packed slot carries charge, part_ind, wgh. */
static int ora_add_columns(ora_sim* s, int ic, int64_t i1, int64_t i2) {
  const agpu_plasma* src = &s->src[ic];
  int64_t n = s->np[ic];
  int64_t add = (i2 - i1 + 1) * (int64_t)s->npty[ic] * s->nptz[ic];
  if (n + add > s->cap[ic]) {
    s->error_bits |= AGPU_EBIT_CAPACITY;
    return AGPU_E_CAPACITY;
  }
  double slot = ora_pack_slot((int16_t)src->charge, (int16_t)src->part_ind, src->wgh);
  for (int k = 1; k <= s->nptz[ic]; ++k)
    for (int j = 1; j <= s->npty[ic]; ++j)
      for (int64_t ix = i1; ix <= i2; ++ix) {
        double x, y, z;
        ora_lattice_particle(s, ic, ix, j, k, &x, &y, &z);
        n = n + 1;
        PART(s, ic, n, 1) = x;
        PART(s, ic, n, 2) = y;
        if (s->p.ndim == 3) {
          PART(s, ic, n, 3) = z;
          PART(s, ic, n, 4) = 0.;
          PART(s, ic, n, 5) = 0.;
          PART(s, ic, n, 6) = 0.;
          PART(s, ic, n, 7) = slot;
        } else {
          PART(s, ic, n, 3) = 0.;
          PART(s, ic, n, 4) = 0.;
          PART(s, ic, n, 5) = slot;
        }
      }
  s->np[ic] = n;
  return 0;
}

/* Lattice column x centre, xpt(ix) (init_part_distrib.f90 (i-1/2)/n rule). */
static double ora_xpt(const ora_sim* s, int ic, int64_t ix) {
  double dxl = s->p.dx / (double)s->src[ic].npx;
  return s->src[ic].x_start + ((double)ix - 0.5) * dxl;
}

/* particles_inject (src/dynamics/window.f90:106-184) for one species. */
static int64_t ora_inject_species(ora_sim* s, int ic, double xmx) {
  int64_t i1 = 1 + s->nptx[ic], i2, ix;
  int64_t smax = s->sptx_max[ic];
  if (i1 <= smax) {
    for (ix = i1; ix <= smax; ++ix)
      if (ora_xpt(s, ic, ix) > xmx) break;
    i2 = ix - 1;
    if (ix == smax) i2 = ix;
  } else {
    i2 = i1 - 1;
  }
  s->nptx[ic] = i2;
  if (i2 > i1) {
    int64_t before = s->np[ic];
    if (ora_add_columns(s, ic, i1, i2) != 0) return -1;
    return s->np[ic] - before;
  }
  return 0;
}

/* Initial load: the same column rule from nptx = 0 against xmax. */
int ora_load_plasma(ora_sim* s, int ic) {
  if (!s->has_src[ic]) return AGPU_E_STATE;
  s->nptx[ic] = 0;
  int64_t i1 = 1, ix, i2;
  for (ix = i1; ix <= s->sptx_max[ic]; ++ix)
    if (ora_xpt(s, ic, ix) > s->p.xmax) break;
  i2 = ix - 1;
  s->nptx[ic] = i2;
  if (i2 >= i1) return ora_add_columns(s, ic, i1, i2);
  return 0;
}

/* ======================================================================== */
/* A19: lp_window_xshift (src/dynamics/window.f90:276-347) with              */
/* fields_left_xshift (mpi_field_interface.f90:299-359) and                  */
/* cell_part_dist(.true.) (mpi_part_interface.f90:549-597, non-prlx branch)  */
/* ======================================================================== */
static int ora_window_xshift(ora_sim* s, int witr, int init_iter, agpu_step_out* out) {
  agpu_params* p = &s->p;
  if (init_iter == 0) {
    s->xlapse = 0.0;
    s->wi1 = 0;
    return 0;
  }
  double dt_step = p->dt;
  s->xlapse = s->xlapse + p->w_speed * dt_step * (double)witr;
  int wi2 = ora_nint(p->dx_inv * s->xlapse);
  int nshx = wi2 - s->wi1;
  s->wi1 = wi2;
  double sh = p->dx * (double)nshx;
  p->xmax = p->xmax + sh;
  p->gxmin = p->gxmin + sh;
  p->gxmax = p->gxmax + sh;
  p->xmn = p->xmn + sh;
  if (out) out->nshx = nshx;
  wi2 = s->ix2 - nshx;
  if (wi2 <= 0) return AGPU_E_WINDOW;
  if (nshx != 0) {
    /* fields_left_xshift(ebf, i1 = ix1, wi2, 1, nfield, nshx) */
    for (int ic = 1; ic <= s->nf; ++ic)
      for (int iz = s->kz1; iz <= s->kz2; ++iz)
        for (int iy = s->jy1; iy <= s->jy2; ++iy) {
          for (int ix = s->ix1; ix <= wi2; ++ix) EBF(s, ix, iy, iz, ic) = EBF(s, ix + nshx, iy, iz, ic);
          for (int ix = wi2 + 1; ix <= wi2 + nshx; ++ix) EBF(s, ix, iy, iz, ic) = 0.0;
        }
    /* envelope: fields_left_xshift(env, i1, wi2, 1, nc_env = 4, nshx) (window.f90:326-330) */
    if (s->env) {
      const size_t c3 = (size_t)s->n1p * s->n2p * s->n3p;
      for (int ic = 0; ic < 4; ++ic)
        for (int iz = s->kz1; iz <= s->kz2; ++iz)
          for (int iy = s->jy1; iy <= s->jy2; ++iy) {
            double* row = s->env + c3 * ic + (size_t)s->n1p * ((size_t)(iy - 1) + (size_t)s->n2p * (size_t)(iz - 1)) - 1;
            for (int ix = s->ix1; ix <= wi2; ++ix) row[ix] = row[ix + nshx];
            for (int ix = wi2 + 1; ix <= wi2 + nshx; ++ix) row[ix] = 0.0;
          }
    }
  }
  /* cell_part_dist(.true.): x only, all species, spec compacted */
  for (int ic = 0; ic < p->nsp; ++ic) {
    if (s->np[ic] > 0) {
      int64_t r = ora_reset_dist(s, ic, 1, p->gxmin, p->gxmax, 0);
      if (out) out->removed[ic] += r;
    }
  }
  /* pex1: inject when targ_in <= xmax < targ_end */
  for (int ic = 0; ic < p->nsp; ++ic) {
    if (!s->has_src[ic]) continue;
    if (s->src[ic].x_start <= p->xmax && s->src[ic].x_end > p->xmax) {
      int64_t a = ora_inject_species(s, ic, p->xmax);
      if (a < 0) return AGPU_E_CAPACITY;
      if (out) out->injected[ic] += a;
    }
  }
  return 0;
}

/* comoving_coordinate (src/dynamics/window.f90:227-275), one rank: the
   target and the not-yet-injected lattice columns move by -vb w_nst dt (the
   plasma source's x range here), particles left of the box are dropped
   (cell_part_dist(.true.)) and the columns that entered are injected. */
static int ora_comoving_coordinate(ora_sim* s, double vb, int w_nst, int loc_it, agpu_step_out* out) {
  agpu_params* p = &s->p;
  if (loc_it == 0) return 0;
  const double dt_step = p->dt;
  double dt_tot = 0.0;
  for (int i = 1; i <= w_nst; ++i) dt_tot = dt_tot + dt_step;
  for (int ic = 0; ic < p->nsp; ++ic) {
    if (!s->has_src[ic]) continue;
    s->src[ic].x_start = s->src[ic].x_start - vb * dt_tot;
    s->src[ic].x_end = s->src[ic].x_end - vb * dt_tot;
  }
  for (int ic = 0; ic < p->nsp; ++ic) {
    if (s->np[ic] > 0) {
      int64_t r = ora_reset_dist(s, ic, 1, p->gxmin, p->gxmax, 0);
      if (out) out->removed[ic] += r;
    }
  }
  for (int ic = 0; ic < p->nsp; ++ic) {
    if (!s->has_src[ic]) continue;
    if (s->src[ic].x_start <= p->xmax && s->src[ic].x_end > p->xmax) {
      int64_t a = ora_inject_species(s, ic, p->xmax);
      if (a < 0) return AGPU_E_CAPACITY;
      if (out) out->injected[ic] += a;
    }
  }
  return 0;
}

/* ======================================================================== */
/* A15-A18: ionization                                                       */
/* ======================================================================== */
/* set_ionization_coeff for one species (src/ionization/ionz_data.f90:131-245,
   770-804): potentials V(i), l_fact and the ADK coefficients. Supported
   atomic numbers: 1 (H), 2 (He), 3 (Li), 6 (C), 7 (N). */
typedef struct {
  double v[8], v_norm[8], e_c[8], nstar[8], vfact[8], e_b[8], c_nstar[8];
  int l_fact[8];
  int an;
} ora_adk;

static int ora_adk_coeff(int an, ora_adk* a) {
  const double v_h = 13.5984, euler = 2.71828, pig = 3.141592653589793;
  memset(a, 0, sizeof(*a));
  for (int i = 0; i < 8; ++i) a->l_fact[i] = 1;
  a->an = an;
  switch (an) {
    case 1:
      a->v[1] = 13.5984;
      break;
    case 2:
      a->v[1] = 24.5874;
      a->v[2] = 54.41776;
      break;
    case 3:
      a->v[1] = 5.3917;
      a->v[2] = 75.6400;
      a->v[3] = 122.4543;
      break;
    case 6:
      a->v[1] = 11.2603;
      a->v[2] = 24.3833;
      a->l_fact[1] = a->l_fact[2] = 3;
      a->v[3] = 47.8878;
      a->v[4] = 64.4939;
      a->v[5] = 392.087;
      a->v[6] = 489.993;
      break;
    case 7:
      a->v[1] = 14.53;
      a->v[2] = 29.601;
      a->v[3] = 47.449;
      a->l_fact[1] = a->l_fact[2] = a->l_fact[3] = 3;
      a->v[4] = 77.473;
      a->v[5] = 97.89;
      a->v[6] = 552.07;
      a->v[7] = 667.046;
      break;
    default:
      return AGPU_E_ARG;
  }
  for (int i = 1; i <= an; ++i) {
    a->v_norm[i] = a->v[i] / v_h;
    a->e_c[i] = a->v_norm[i] * a->v_norm[i] / (16. * (double)i);
    a->nstar[i] = (double)i / sqrt(a->v_norm[i]);
    a->vfact[i] = (a->v_norm[i]) * sqrt(a->v_norm[i]);
    a->e_b[i] = 2. * a->vfact[i] / (3. * (2. * a->nstar[i] - 1.));
  }
  for (int i = 1; i <= an; ++i) {
    a->c_nstar[i] = pow(2. * euler / a->nstar[i], 2 * a->nstar[i]);
    a->c_nstar[i] = a->c_nstar[i] * (double)a->l_fact[i] / (2. * pig * a->nstar[i]);
    a->c_nstar[i] = 0.5 * a->v_norm[i] * a->c_nstar[i];
  }
  return 0;
}

/* set_field_ioniz_wfunction, one-level branch (src/ionization/ionize.f90:
   38-190): ADK rate tables for models 1-5 on n_ge bins of |E| in (0,e_max],
   w_one_lev = 1 - exp(-dt_fs * omega_a * W). Output table column-major
   (nk = 0..n_ge+1, z = 0..zm), rows never written by the reference are 0. */
int ora_build_ionization_table(int an, int z0, int model, double e_max, double dt, double* tab,
                               double* de_inv_out) {
  const double omega_a = 41.3, pig = 3.141592653589793, tiny = 1.e-10;
  const int n_ge = ORA_NGE;
  ora_adk a;
  if (ora_adk_coeff(an, &a) != 0) return AGPU_E_ARG;
  int zm = an;
  int nrow = n_ge + 2;
  double* wi = (double*)calloc((size_t)(n_ge + 1) * (zm + 1), sizeof(double));
  double dge = e_max / (double)n_ge;
  double de_inv = 1. / dge;
  for (int k = z0 + 1; k <= zm; ++k) {
    int j = k - z0;
    double ns = 2. * a.nstar[k] - 1.;
    for (int i = 1; i <= n_ge; ++i) {
      double ei = dge * (double)i;
      double fact2 = (2. * a.vfact[k] / ei);
      double fact1, w_adk, w_bsi, efact, avg_fact;
      double w = 0.0;
      switch (model) {
        case 1:
          fact1 = pow(fact2, ns);
          w_adk = a.c_nstar[k] * fact1 * exp(-fact2 / 3.);
          if (w_adk < tiny) w_adk = 0.0;
          w = w_adk;
          break;
        case 2:
          fact1 = pow(fact2, ns);
          fact1 = fact1 * sqrt(3. * ei / (pig * a.vfact[k]));
          w_adk = a.c_nstar[k] * fact1 * exp(-fact2 / 3.);
          if (w_adk < tiny) w_adk = 0.0;
          w = w_adk;
          break;
        case 3:
        case 5:
          if (model == 3) {
            fact1 = pow(fact2, ns);
            fact1 = fact1 * sqrt(3. * ei / (pig * a.vfact[k]));
          } else {
            fact1 = sqrt(3. * ei / (pig * a.vfact[k])) * pow(fact2, ns);
          }
          w_adk = a.c_nstar[k] * fact1 * exp(-fact2 / 3.);
          if (w_adk < tiny) w_adk = 0.0;
          w = w_adk;
          if (ei > a.e_c[k]) {
            fact2 = (2. * a.vfact[k] / a.e_c[k]);
            if (model == 3) {
              fact1 = pow(fact2, ns);
              fact1 = fact1 * sqrt(3. * a.e_c[k] / (pig * a.vfact[k]));
            } else {
              fact1 = sqrt(3. * a.e_c[k] / (pig * a.vfact[k])) * pow(fact2, ns);
            }
            w_adk = a.c_nstar[k] * fact1 * exp(-fact2 / 3.);
            w_bsi = a.vfact[k] * (1. - a.e_c[k] / ei) / (4. * pig * (double)k);
            w = w_bsi + w_adk;
          }
          break;
        case 4:
          fact1 = pow(fact2, ns);
          avg_fact = 1.0;
          if (a.l_fact[k] > 1) {
            for (int ll = 1; ll <= (a.l_fact[k] - 1) / 2; ++ll) avg_fact = avg_fact + 2. / pow(fact2, ll);
            avg_fact = avg_fact / a.l_fact[k];
            fact1 = fact1 * avg_fact;
          }
          fact1 = fact1 * sqrt(3. * ei / (pig * a.vfact[k]));
          w_adk = a.c_nstar[k] * fact1 * exp(-fact2 / 3.);
          if (w_adk < tiny) w_adk = 0.0;
          w = w_adk;
          efact = 1. - a.e_c[k] / ei;
          w_bsi = a.vfact[k] * efact / (4. * pig * (double)k);
          if (w_bsi < tiny) w_bsi = 0.;
          if (ei > a.e_c[k]) w = (w_bsi < w_adk) ? w_bsi : w_adk;
          if (ei > a.e_b[k]) w = w_bsi;
          break;
        default:
          free(wi);
          return AGPU_E_ARG;
      }
      wi[(size_t)i + (size_t)(n_ge + 1) * j] = w;
    }
  }
  double dt_fs = 10. * dt / 3.;
  for (size_t q = 0; q < (size_t)(n_ge + 1) * (zm + 1); ++q) wi[q] = omega_a * wi[q];
  memset(tab, 0, sizeof(double) * (size_t)nrow * (zm + 1));
  int zm_loc = zm - z0;
  for (int z = 0; z <= zm_loc - 1; ++z) {
    int zk = z + 1;
    int k = z + z0;
    for (int i = 1; i <= n_ge; ++i) tab[(size_t)i + (size_t)nrow * k] = 1. - exp(-dt_fs * wi[(size_t)i + (size_t)(n_ge + 1) * zk]);
  }
  free(wi);
  *de_inv_out = de_inv;
  return 0;
}

int ora_set_ionization_species(ora_sim* s, int ic, int an, int ion_min, int model, double lp_max) {
  if (ic < 1 || ic >= s->p.nsp) return AGPU_E_ARG;
  s->at_num[ic] = an;
  s->ion_min[ic] = ion_min;
  s->ionz_model[ic] = model;
  s->zmax[ic] = an;
  s->lp_max[ic] = lp_max;
  free(s->wtab[ic]);
  s->wtab[ic] = (double*)calloc((size_t)(ORA_NGE + 2) * (an + 1), sizeof(double));
  if (ic + 1 > s->nsp_ionz) s->nsp_ionz = ic + 1;
  return ora_build_ionization_table(an, ion_min, model, lp_max, s->p.dt, s->wtab[ic], &s->de_inv[ic]);
}

/* set_ion_efield (grid_part_connect.f90:288-410): |E|^2 on each ion with
   the qqh shapes, into ebfp(:, id_ch). */
static void ora_set_ion_efield(ora_sim* s, int ic, int64_t np) {
  const agpu_params* p = &s->p;
  int id_ch = s->ndv;
  #pragma omp parallel for schedule(static) num_threads(s->nthreads) if (s->nthreads > 1)
  for (int64_t n = 1; n <= np; ++n) {
    double ef_sqr = 0.;
    double xl = p->dx_inv * (PART(s, ic, n, 1) - p->xmn);
    double yl = p->dy_inv * (PART(s, ic, n, 2) - p->ymn);
    double ax1[3], axh[3], ay1[3], ayh[3], az1[3], azh[3];
    int i, ih, j, jh, k, kh;
    ora_qqh_1d(xl, ax1, axh, &i, &ih);
    ora_qqh_1d(yl, ay1, ayh, &j, &jh);
    if (p->ndim == 2) {
      for (int jp1 = 0; jp1 <= 2; ++jp1) {
        int jp2 = j + jp1;
        double dvol = ay1[jp1];
        for (int ip1 = 0; ip1 <= 2; ++ip1) {
          double ex = EBF(s, ih + ip1, jp2, 1, 1);
          ef_sqr = ef_sqr + axh[ip1] * dvol * ex * ex;
        }
      }
      for (int jp1 = 0; jp1 <= 2; ++jp1) {
        int jp2 = jh + jp1;
        double dvol = ayh[jp1];
        for (int ip1 = 0; ip1 <= 2; ++ip1) {
          double ey = EBF(s, i + ip1, jp2, 1, 2);
          ef_sqr = ef_sqr + ax1[ip1] * dvol * ey * ey;
        }
      }
    } else {
      double zl = p->dz_inv * (PART(s, ic, n, 3) - p->zmn);
      ora_qqh_1d(zl, az1, azh, &k, &kh);
      for (int kp1 = 0; kp1 <= 2; ++kp1) {
        int kp2 = k + kp1;
        for (int jp1 = 0; jp1 <= 2; ++jp1) {
          int jp2 = j + jp1;
          double dvol = ay1[jp1] * az1[kp1];
          for (int ip1 = 0; ip1 <= 2; ++ip1) {
            double ex = EBF(s, ip1 + ih, jp2, kp2, 1);
            ef_sqr = ef_sqr + axh[ip1] * dvol * ex * ex;
          }
        }
        for (int jp1 = 0; jp1 <= 2; ++jp1) {
          int jp2 = jh + jp1;
          double dvol = ayh[jp1] * az1[kp1];
          for (int ip1 = 0; ip1 <= 2; ++ip1) {
            double ey = EBF(s, i + ip1, jp2, kp2, 2);
            ef_sqr = ef_sqr + ax1[ip1] * dvol * ey * ey;
          }
        }
      }
      for (int kp1 = 0; kp1 <= 2; ++kp1) {
        int kp2 = kh + kp1;
        for (int jp1 = 0; jp1 <= 2; ++jp1) {
          int jp2 = j + jp1;
          double dvol = ay1[jp1] * azh[kp1];
          for (int ip1 = 0; ip1 <= 2; ++ip1) {
            double ez = EBF(s, ip1 + i, jp2, kp2, 3);
            ef_sqr = ef_sqr + ax1[ip1] * dvol * ez * ez;
          }
        }
      }
    }
    PT(s, n, id_ch) = ef_sqr;
  }
}

/* Ionization draw for ion n (0-based) of species ic at step iter. */
static inline double ora_ionz_draw(uint64_t seed, int64_t n, int iter, int ic) {
  uint32_t ctr[4] = {(uint32_t)n, (uint32_t)((uint64_t)n >> 32), (uint32_t)iter, 0x494f0000u | (uint32_t)ic};
  uint32_t r[4];
  ora_philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32), r);
  return ora_u53(r[0], r[1]);
}

/* ionization_cycle + part_ionize (ionz_lev = 1) + ionization_electrons_inject
   (src/ionization/ionize.f90:452-558, 390-450, 258-322).  Returns the number
   of new electrons. */
static int64_t ora_ionization_cycle(ora_sim* s, int ic, int64_t np, int iter) {
  int id_ch = s->ndv;
  int n_ge = ORA_NGE, nrow = n_ge + 2;
  double def_inv = s->de_inv[ic];
  int64_t kk = 0;
  int64_t ne = s->np[0];
  /* count first (capacity), then apply in ion order */
  for (int64_t n = 1; n <= np; ++n) {
    double ef2 = PT(s, n, id_ch);
    int nk = 0;
    if (ef2 > 0.) {
      double ef = sqrt(ef2);
      nk = ora_nint(def_inv * ef);
    }
    if (nk > n_ge + 1) {
      s->error_bits |= AGPU_EBIT_IONZ_INDEX;
      nk = n_ge + 1;
    }
    ora_pack w = ora_unpack(PART(s, ic, n, id_ch));
    int z0 = w.charge;
    double pr = ora_ionz_draw(s->p.seed, n - 1, iter, ic);
    double thr = (z0 >= 0 && z0 <= s->zmax[ic]) ? s->wtab[ic][(size_t)nk + (size_t)nrow * z0] : 0.0;
    if (pr < thr) {
      w.charge = (int16_t)(w.charge + 1);
      PART(s, ic, n, id_ch) = ora_pack_slot(w.charge, w.part_ind, w.wgh);
      kk++;
      if (ne + 1 > s->cap[0]) {
        s->error_bits |= AGPU_EBIT_CAPACITY;
        continue;
      }
      ne = ne + 1;
      float ewgh = w.wgh * (float)s->p.n_mol_atoms[ic];
      double slot = ora_pack_slot(-1, -1, ewgh);
      for (int c = 1; c <= s->p.curr_ndim; ++c) PART(s, 0, ne, c) = PART(s, ic, n, c);
      for (int c = s->p.curr_ndim + 1; c <= 2 * s->p.curr_ndim; ++c) PART(s, 0, ne, c) = 0.0;
      PART(s, 0, ne, id_ch) = slot;
    }
  }
  s->np[0] = ne;
  return kk;
}

/* ======================================================================== */
/* lpf2_evolve + lp_run (src/dynamics/pic_evolve_in_time.f90:37-144)         */
/* ======================================================================== */
int ora_step(ora_sim* s, int iter, double t, int initial_time, agpu_step_out* out) {
  agpu_params* p = &s->p;
  agpu_step_out dummy;
  if (!out) out = &dummy;
  memset(out, 0, sizeof(*out));
  out->ion_field_max = -1.0;
  ora_field_xyzbd(s, s->nf);
  if (p->ionz_lev > 0) {
    for (int ic = 1; ic < s->nsp_ionz; ++ic) {
      int64_t np = s->np[ic];
      if (np > 0 && s->wtab[ic]) {
        ora_set_ion_efield(s, ic, np);
        if (iter % 100 == 0) {
          double m = 0.0;
          for (int64_t n = 1; n <= np; ++n)
            if (PT(s, n, s->ndv) > m || n == 1) m = PT(s, n, s->ndv);
          m = sqrt(m);
          out->ion_field_max = m;
          if (m > s->lp_max[ic]) {
            s->lp_max[ic] = 1.1 * m;
            ora_build_ionization_table(s->at_num[ic], s->ion_min[ic], s->ionz_model[ic], s->lp_max[ic], p->dt,
                                       s->wtab[ic], &s->de_inv[ic]);
          }
        }
        out->new_electrons += ora_ionization_cycle(s, ic, np, iter);
      }
    }
  }
  ora_zero_currents(s);
  for (int ic = 0; ic < p->nsp_run; ++ic) {
    int64_t np = s->np[ic];
    if (s->p.shape == AGPU_SHAPE_CUBIC) ora_gather_cubic(s, ic, np); else ora_gather(s, ic, np);
    ora_field_charge_multiply(s, ic, np);
    if (initial_time) ora_init_lpf_momenta(s, ic, np);
    ora_push(s, ic, np);
    out->removed[ic] += ora_cell_part_dist_step(s, ic);
    np = s->np[ic];
    if (np > 0) ora_curr_accumulate(s, ic, np);
  }
  ora_curr_collect(s);
  ora_advance_fields(s);
  int rc = 0;
  if (p->w_speed > 0.0 && p->w_sh > 0) {
    if (t >= p->wi_time && t < p->wf_time) {
      if (iter % p->w_sh == 0) rc = ora_window_xshift(s, p->w_sh, iter, out);
    }
  }
  if (p->w_speed < 0.0 && p->w_sh > 0) { /* comoving = (w_speed < 0), vbeam = -w_speed */
    if (t >= p->wi_time && t < p->wf_time) {
      if (iter % p->w_sh == 0) rc = ora_comoving_coordinate(s, -p->w_speed, p->w_sh, iter, out);
    }
  }
  for (int ic = 0; ic < 4; ++ic) out->np[ic] = s->np[ic];
  out->xmn = p->xmn;
  out->error_bits = s->error_bits;
  return rc;
}

/* Individual phases for tests. */
void ora_phase_gather_push(ora_sim* s, int ic, int initial_time) {
  int64_t np = s->np[ic];
  if (s->p.shape == AGPU_SHAPE_CUBIC) ora_gather_cubic(s, ic, np); else ora_gather(s, ic, np);
  ora_field_charge_multiply(s, ic, np);
  if (initial_time) ora_init_lpf_momenta(s, ic, np);
  ora_push(s, ic, np);
}
int ora_get_scratch(const ora_sim* s, int col, double* out, int64_t n) {
  if (col < 1 || col > s->ndv || n > s->ebfp_cap) return AGPU_E_ARG;
  memcpy(out, &s->ebfp[(size_t)(col - 1) * s->ebfp_cap], sizeof(double) * (size_t)n);
  return 0;
}
int ora_get_ionization_table(const ora_sim* s, int ic, double* out) {
  if (!s->wtab[ic]) return AGPU_E_STATE;
  memcpy(out, s->wtab[ic], sizeof(double) * (size_t)(ORA_NGE + 2) * (s->zmax[ic] + 1));
  return 0;
}
double ora_ionz_de_inv(const ora_sim* s, int ic) { return s->de_inv[ic]; }
double ora_draw(uint64_t seed, int64_t n, int iter, int ic) { return ora_ionz_draw(seed, n, iter, ic); }
void ora_philox(const uint32_t* ctr, uint32_t k0, uint32_t k1, uint32_t* out) { ora_philox4x32_10(ctr, k0, k1, out); }

/* ======================================================================== */
/* A20: PWFA bunch set-up.  set_grid_charge (src/particles/grid_part_util.   */
/* f90:240-334), the sine-transform Poisson solve fft_3d_psolv /            */
/* fft_2d_psolv + beam_potential / beam_2d_potential (src/IO/psolve.f90:     */
/* 39-238) with the wavenumbers of set_grid_param.f90:967-987 and the r2r    */
/* transforms of src/fft/modern_fft_lib.F90:675-775, initial_beam_fields     */
/* (src/fields/init_grid_fields.f90:32-134), the box selection of            */
/* mpi_beam_distribute (src/IO/init_beam_part_distrib.f90:273-438) and       */
/* beam_inject (init_beam_part_distrib.f90:474-630, uniform-grid branch).    */
/* ======================================================================== */

/* FFTW_RODFT00 of length n by its published definition (FFTW is not
   vendored): Y_k = 2 sum_j x_j sin(pi (j+1)(k+1)/(n+1)), unnormalised.
   sint[m] = sin(pi m/(n+1)), m in [0, 2(n+1)). */
static void ora_rodft00(double* x, int n, double* work, const double* sint) {
  for (int k = 0; k < n; ++k) {
    double acc = 0.0;
    for (int j = 0; j < n; ++j) acc += x[j] * sint[(size_t)((j + 1) * (k + 1)) % (size_t)(2 * (n + 1))];
    work[k] = 2.0 * acc;
  }
  memcpy(x, work, sizeof(double) * (size_t)n);
}

static double* ora_sin_table(int n) {
  double* t = (double*)malloc(sizeof(double) * (size_t)(2 * (n + 1)));
  for (int m = 0; m < 2 * (n + 1); ++m) t[m] = sin(acos(-1.0) * (double)m / (double)(n + 1));
  return t;
}

/* ftw1d_sc (modern_fft_lib.F90:675-775), sine kind, on the compact array
   w(n1,n2,n3) along dir; is < 0 scales by 1/ndb with ndb = 2(n1+2) along x
   (logical_dimension(kind, n1+1)) and 2(n+1) along y and z. */
static void ora_ftw1d_sin(double* w, int n1, int n2, int n3, int is, int dir) {
  int n = dir == 1 ? n1 : (dir == 2 ? n2 : n3);
  double* line = (double*)malloc(sizeof(double) * (size_t)n);
  double* work = (double*)malloc(sizeof(double) * (size_t)n);
  double* sint = ora_sin_table(n);
  int ndb = dir == 1 ? 2 * (n1 + 1 + 1) : 2 * (n + 1);
  double sc = 1. / (double)ndb;
  size_t s1 = 1, s2 = (size_t)n1, s3 = (size_t)n1 * n2;
  size_t stride = dir == 1 ? s1 : (dir == 2 ? s2 : s3);
  int na = dir == 1 ? n2 : n1, nb = dir == 3 ? n2 : n3;
  size_t sa = dir == 1 ? s2 : s1, sb = dir == 3 ? s2 : s3;
  for (int b = 0; b < nb; ++b)
    for (int a = 0; a < na; ++a) {
      double* base = w + (size_t)a * sa + (size_t)b * sb;
      for (int i = 0; i < n; ++i) line[i] = base[(size_t)i * stride];
      ora_rodft00(line, n, work, sint);
      for (int i = 0; i < n; ++i) base[(size_t)i * stride] = is < 0 ? sc * line[i] : line[i];
    }
  free(line);
  free(work);
  free(sint);
}

/* Wavenumbers of the sine transform, case(2) of set_grid_param.f90:967-987:
   sk(i) = 2 sin(0.5 d ak(i))/d with ak(i) = (pi/l_box) i. */
static void ora_sine_k(double* sk, int n, double d, double l_box) {
  double wk = acos(-1.0) / l_box;
  for (int i = 1; i <= n; ++i) {
    double ak = wk * (double)i;
    sk[i - 1] = 2. * sin(0.5 * d * ak) / d;
  }
}

/* fft_3d_psolv / fft_2d_psolv with ft_mod = 2, sym = 1, s_ind = 0 on the
   field-layout array rho(n1p,n2p,n3p): the interior is replaced by the
   potential of Laplacian(pot) = -omp0 rho, x-derivative over gam2 in 3D. */
int ora_beam_potential(ora_sim* s, double* rho, double gam2) {
  const agpu_params* p = &s->p;
  int n1 = p->nx, n2 = p->ny, n3 = p->ndim == 3 ? p->nz : 1;
  size_t n1p = (size_t)s->n1p, n2p = (size_t)s->n2p;
  double* wb = (double*)malloc(sizeof(double) * (size_t)n1 * n2 * n3);
  double *skx = (double*)calloc((size_t)n1 + 2, sizeof(double)), *sky = (double*)calloc((size_t)n2 + 2, sizeof(double)),
         *skz = (double*)calloc((size_t)n3 + 2, sizeof(double));
  if (!wb || !skx || !sky || !skz) return 103;
  /* lx_box = x(n1) - x(1), ly_box = y(n2+1) - y(1), lz_box = z(n3+1) - z(1)
     (set_grid_param.f90:102-108, 168-170, 221-223) */
  ora_sine_k(skx, n1, p->dx, p->xmax - p->xmn);
  if (n2 > 1) ora_sine_k(sky, n2, p->dy, p->gymax - p->gymin);
  if (n3 > 1) ora_sine_k(skz, n3, p->dz, p->gzmax - p->gzmin);
  for (int k = 0; k < n3; ++k)
    for (int j = 0; j < n2; ++j)
      for (int i = 0; i < n1; ++i)
        wb[(size_t)i + (size_t)n1 * ((size_t)j + (size_t)n2 * k)] =
            rho[(size_t)(s->ix1 - 1 + i) + n1p * ((size_t)(s->jy1 - 1 + j) + n2p * (size_t)(s->kz1 - 1 + k))];
  double omp0 = p->ompe;
  size_t ncell = (size_t)n1 * n2 * n3;
  if (p->ndim == 3) {
    /* pftw3d_sc(-1): x, then pftw2d_sc: y (n2 > 2), z (n3 > 2) */
    ora_ftw1d_sin(wb, n1, n2, n3, -1, 1);
    if (n2 > 2) ora_ftw1d_sin(wb, n1, n2, n3, -1, 2);
    if (n2 > 2 && n3 > 2) ora_ftw1d_sin(wb, n1, n2, n3, -1, 3);
    for (size_t q = 0; q < ncell; ++q) wb[q] = omp0 * wb[q];
    /* beam_potential (psolve.f90:93-112) */
    for (int iz = 0; iz < n3; ++iz)
      for (int iy = 0; iy < n2; ++iy) {
        double ak2p = skz[iz] * skz[iz] + sky[iy] * sky[iy];
        double* row = wb + (size_t)n1 * ((size_t)iy + (size_t)n2 * iz);
        if (ak2p > 0.0) {
          for (int ix = 0; ix < n1; ++ix) {
            double ak2 = ak2p + skx[ix] * skx[ix] / gam2;
            row[ix] = row[ix] / ak2;
          }
        } else {
          for (int ix = 1; ix < n1; ++ix) {
            double ak2 = skx[ix] * skx[ix] / gam2;
            row[ix] = row[ix] / ak2;
          }
        }
      }
    /* pftw3d_sc(+1): pftw2d_sc (z if n3 > 1, y if n2 > 1), then x */
    if (n3 > 1) ora_ftw1d_sin(wb, n1, n2, n3, 1, 3);
    if (n2 > 1) ora_ftw1d_sin(wb, n1, n2, n3, 1, 2);
    ora_ftw1d_sin(wb, n1, n2, n3, 1, 1);
  } else {
    /* fft_2d_psolv: pftw2d_sc(-1) transforms y only (n3 = 1) */
    if (n2 > 2) ora_ftw1d_sin(wb, n1, n2, n3, -1, 2);
    for (size_t q = 0; q < ncell; ++q) wb[q] = omp0 * wb[q];
    /* beam_2d_potential (psolve.f90:39-64) */
    for (int iz = 0; iz < n3; ++iz)
      for (int iy = 0; iy < n2; ++iy) {
        double ak2p = skz[iz] * skz[iz] + sky[iy] * sky[iy];
        double* row = wb + (size_t)n1 * ((size_t)iy + (size_t)n2 * iz);
        if (ak2p > 0.0) {
          for (int ix = 0; ix < n1; ++ix) row[ix] = row[ix] / ak2p;
        } else {
          for (int ix = 0; ix < n1; ++ix) row[ix] = 0.0;
        }
      }
    if (n2 > 1) ora_ftw1d_sin(wb, n1, n2, n3, 1, 2);
  }
  for (int k = 0; k < n3; ++k)
    for (int j = 0; j < n2; ++j)
      for (int i = 0; i < n1; ++i)
        rho[(size_t)(s->ix1 - 1 + i) + n1p * ((size_t)(s->jy1 - 1 + j) + n2p * (size_t)(s->kz1 - 1 + k))] =
            wb[(size_t)i + (size_t)n1 * ((size_t)j + (size_t)n2 * k)];
  free(wb);
  free(skx);
  free(sky);
  free(skz);
  return 0;
}

/* set_grid_charge (grid_part_util.f90:240-334) of np records part(ld, ndv)
   into den(n1p,n2p,n3p): wght = real(charge*wgh, sp), qden shapes.  A record
   whose stencil leaves the array is skipped (the reference has no check). */
void ora_grid_charge(const ora_sim* s, const double* part, int64_t ld, int64_t np, double* den) {
  const agpu_params* p = &s->p;
  size_t n1p = (size_t)s->n1p, n2p = (size_t)s->n2p;
  int ch = p->ndim == 3 ? 7 : 5;
  for (int64_t n = 0; n < np; ++n) {
    ora_pack pk = ora_unpack(part[(size_t)(ch - 1) * (size_t)ld + (size_t)n]);
    float wght = (float)pk.charge * pk.wgh;
    double ax0[3], ay0[3], az0[3];
    int i, j, k;
    double xl = p->dx_inv * (part[(size_t)n] - p->xmn);
    double yl = p->dy_inv * (part[(size_t)ld + (size_t)n] - p->ymn);
    if (!(fabs(xl) < 1e9) || !(fabs(yl) < 1e9)) continue;
    ora_qden_1d(xl, ax0, &i);
    ora_qden_1d(yl, ay0, &j);
    for (int q = 0; q < 3; ++q) ax0[q] = (double)wght * ax0[q];
    i -= 1;
    j -= 1;
    /* stencil nodes i..i+2 must lie in 1..n1p */
    if (i < 1 || i > s->n1p - 2 || j < 1 || j > s->n2p - 2) continue;
    if (p->ndim == 2) {
      for (int j1 = 0; j1 <= 2; ++j1)
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol = ax0[i1] * ay0[j1];
          den[(size_t)(i + i1 - 1) + n1p * (size_t)(j + j1 - 1)] += dvol;
        }
    } else {
      double zl = p->dz_inv * (part[(size_t)2 * (size_t)ld + (size_t)n] - p->zmn);
      if (!(fabs(zl) < 1e9)) continue;
      ora_qden_1d(zl, az0, &k);
      k -= 1;
      if (k < 1 || k > s->n3p - 2) continue;
      for (int k1 = 0; k1 <= 2; ++k1)
        for (int j1 = 0; j1 <= 2; ++j1) {
          double dvol = az0[k1] * ay0[j1];
          for (int i1 = 0; i1 <= 2; ++i1)
            den[(size_t)(i + i1 - 1) + n1p * ((size_t)(j + j1 - 1) + n2p * (size_t)(k + k1 - 1))] += ax0[i1] * dvol;
        }
    }
  }
}

/* initial_beam_fields (init_grid_fields.f90:32-134) on poten = jc(:,:,:,1:2)
   into efb(n1p,n2p,n3p,6) (zero on entry), single domain: pe1x, pe1y, pe1z. */
static void ora_initial_beam_fields(ora_sim* s, double* efb, double g2, double bet) {
  const agpu_params* p = &s->p;
  int ix1 = s->ix1, ix2 = s->ix2, jy1 = s->jy1, jy2 = s->jy2, kz1 = s->kz1, kz2 = s->kz2;
  size_t n1p = (size_t)s->n1p, n2p = (size_t)s->n2p, n3p = (size_t)s->n3p, nc3 = n1p * n2p * n3p;
#define P1(i, j, k) s->jc[((size_t)(i)-1) + n1p * (((size_t)(j)-1) + n2p * ((size_t)(k)-1))]
#define P2(i, j, k) s->jc[nc3 + ((size_t)(i)-1) + n1p * (((size_t)(j)-1) + n2p * ((size_t)(k)-1))]
#define EF(i, j, k, c) efb[(size_t)((c)-1) * nc3 + ((size_t)(i)-1) + n1p * (((size_t)(j)-1) + n2p * ((size_t)(k)-1))]
  {
    int j = jy2;
    for (int k = kz1; k <= kz2; ++k)
      for (int i = ix1; i <= ix2; ++i) P1(i, j + 1, k) = 3. * (P1(i, j, k) - P1(i, j - 1, k)) + P1(i, j - 2, k);
  }
  for (int k = kz1; k <= kz2; ++k)
    for (int j = jy1; j <= jy2; ++j) {
      P1(ix2 + 1, j, k) = P1(ix2, j, k);
      P2(ix2 + 1, j, k) = 2. * P2(ix2, j, k) - P2(ix2 - 1, j, k);
    }
  for (int k = kz1; k <= kz2; ++k)
    for (int j = jy1; j <= jy2; ++j)
      for (int i = ix1; i <= ix2; ++i) EF(i, j, k, 4) = 0.5 * (P2(i, j, k) + P2(i + 1, j, k));
  for (int k = kz1; k <= kz2; ++k)
    for (int j = jy1; j <= jy2; ++j) {
      double sdhy = 1.0 * p->dy_inv; /* loc_yg(jj,3) = 1 on a uniform grid */
      for (int i = ix1; i <= ix2 + 1; ++i) EF(i, j, k, 2) = -sdhy * (P1(i, j + 1, k) - P1(i, j, k));
      for (int i = ix1; i <= ix2; ++i) EF(i, j, k, 1) = -p->dx_inv * (P1(i + 1, j, k) - P1(i, j, k)) / g2;
    }
  if (p->ndim == 2) {
    for (int k = kz1; k <= kz2; ++k)
      for (int j = jy1; j <= jy2; ++j)
        for (int i = ix1; i <= ix2; ++i) EF(i, j, k, 3) = 0.5 * bet * (EF(i, j, k, 2) + EF(i + 1, j, k, 2));
    return;
  }
  {
    int k = kz2;
    for (int j = jy1; j <= jy2; ++j)
      for (int i = ix1; i <= ix2; ++i) P1(i, j, k + 1) = 2. * P1(i, j, k) - P1(i, j, k - 1);
  }
  for (int k = kz1; k <= kz2; ++k)
    for (int j = jy1; j <= jy2; ++j)
      for (int i = ix1; i <= ix2; ++i) EF(i, j, k, 6) = 0.5 * bet * (EF(i, j, k, 2) + EF(i + 1, j, k, 2));
  for (int k = kz1; k <= kz2; ++k) {
    double sdhz = 1.0 * p->dz_inv;
    for (int j = jy1; j <= jy2; ++j)
      for (int i = ix1; i <= ix2; ++i) EF(i, j, k, 3) = -sdhz * (P1(i, j, k + 1) - P1(i, j, k));
  }
  for (int k = kz1; k <= kz2; ++k)
    for (int j = jy1; j <= jy2; ++j)
      for (int i = ix1; i <= ix2; ++i) {
        P2(i, j, k) = 0.5 * (EF(i, j, k, 3) + EF(i + 1, j, k, 3));
        EF(i, j, k, 5) = -bet * P2(i, j, k);
      }
#undef P1
#undef P2
#undef EF
}

/* beam_inject (init_beam_part_distrib.f90:474-630), uniform grid: append the
   bunch records inside the box to species ic, deposit their charge into
   jc(1), solve for the potential, jc(2) = bet0 jc(1), then
   ebf += initial_beam_fields with Bx = 0. */
int ora_beam_inject(ora_sim* s, int ic, const double* part, int64_t ld, int64_t nb_tot, double gam0) {
  if (ic < 0 || ic >= s->p.nsp || nb_tot < 0 || ld < nb_tot) return 101;
  const agpu_params* p = &s->p;
  /* mpi_beam_distribute (init_beam_part_distrib.f90:273-438): keep, in
     order, the records with x1 < x <= x2, y1 < y <= y2 (and z1 < z <= z2) */
  int64_t nb = 0;
  int64_t* keep = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nb_tot > 0 ? nb_tot : 1));
  if (!keep) return 103;
  for (int64_t n = 0; n < nb_tot; ++n) {
    double x = part[(size_t)n], y = part[(size_t)ld + (size_t)n];
    int in = y > p->gymin && y <= p->gymax && x > p->gxmin && x <= p->gxmax;
    if (p->ndim == 3) {
      double z = part[(size_t)2 * (size_t)ld + (size_t)n];
      in = in && z > p->gzmin && z <= p->gzmax;
    }
    if (in) keep[nb++] = n;
  }
  if (s->np[ic] + nb > s->cap[ic]) {
    free(keep);
    return 104;
  }
  double* sel = (double*)malloc(sizeof(double) * (size_t)(nb > 0 ? nb : 1) * (size_t)s->ndv);
  if (!sel) {
    free(keep);
    return 103;
  }
  for (int c = 1; c <= s->ndv; ++c)
    for (int64_t n = 0; n < nb; ++n) {
      double v = part[(size_t)(c - 1) * (size_t)ld + (size_t)keep[n]];
      sel[(size_t)(c - 1) * (size_t)nb + (size_t)n] = v;
      PART(s, ic, s->np[ic] + 1 + n, c) = v;
    }
  free(keep);
  s->np[ic] += nb;
  double gam2 = gam0 * gam0;
  double u0_b = sqrt(gam0 * gam0 - 1.); /* set_init_param.f90:353-354 */
  double bet0 = u0_b / gam0;
  size_t nc3 = (size_t)s->n1p * s->n2p * s->n3p;
  memset(s->jc, 0, sizeof(double) * nc3); /* jc(:,:,:,1) = 0.0 */
  ora_grid_charge(s, sel, nb, nb, s->jc);
  free(sel);
  int rc = ora_beam_potential(s, s->jc, gam2);
  if (rc) return rc;
  for (size_t q = 0; q < nc3; ++q) s->jc[nc3 + q] = bet0 * s->jc[q];
  double* efb = (double*)calloc(nc3 * 6, sizeof(double));
  if (!efb) return 103;
  ora_initial_beam_fields(s, efb, gam2, bet0);
  memset(efb + 3 * nc3, 0, sizeof(double) * nc3); /* ebf_bunch(:,:,:,4) = 0 */
  for (int c = 0; c < s->nf; ++c)
    for (size_t q = 0; q < nc3; ++q) s->ebf[(size_t)c * nc3 + q] = s->ebf[(size_t)c * nc3 + q] + efb[(size_t)c * nc3 + q];
  free(efb);
  return 0;
}

/* ======================================================================== */
/* A21: init_lp_inc0_fields (src/fields/init_grid_fields.f90:992-1386),     */
/* lp = 1 (P polarisation, normal incidence), with get_laser_gprof_fields_lp */
/* / get_laser_fields_lp (487-578) and the 2D forms (406-485).  Grid        */
/* coordinates of the interior nodes: x = xmn + (i-3) dx, xh = x + dx/2,    */
/* y and z alike (x(i) = dx*(i-1), xh = x + 0.5 dx, set_grid_param.f90:77-78,*/
/* 129-130, 187-188, with the box origin of the parameters).                */
/* ======================================================================== */
static void ora_lp_fields(int ndim, int g_prof, const double par_lp[7], const double coords[4], double fields[6]) {
  const double pi = acos(-1.0);
  double x1, y1, z1 = 0.0, t1, pih, r2, phi0, phi1, w2, phx, phig00, phig10, tshape, wshape, ampl, ampl_1;
  x1 = coords[0];
  y1 = coords[1] / par_lp[3];
  if (ndim == 3) z1 = coords[2] / par_lp[3];
  t1 = coords[3];
  pih = 0.5 * pi;
  r2 = (ndim == 3) ? y1 * y1 + z1 * z1 : y1 * y1;
  phi0 = par_lp[0] * (t1 - x1);
  if (g_prof) {
    phi1 = (t1 - x1) / par_lp[2];
  } else {
    phi1 = pi * (t1 - x1) / par_lp[2];
    if (fabs(phi1) > pih) phi1 = pih;
  }
  x1 = x1 / par_lp[4];
  w2 = 1. / (1. + x1 * x1);
  phx = (ndim == 3) ? atan(x1) : 0.5 * atan(x1);
  phig00 = phi0 + phx - x1 * r2 * w2;
  phig10 = phig00 + phx;
  tshape = g_prof ? exp(-phi1 * phi1) : cos(phi1) * cos(phi1);
  wshape = ((ndim == 3) ? sqrt(w2) : sqrt(sqrt(w2))) * exp(-w2 * r2);
  ampl = tshape * sin(phig00);
  fields[1] = wshape * ampl;
  if (g_prof && ndim == 3)
    ampl_1 = 2. * par_lp[5] * tshape * w2 * exp(-w2 * r2);
  else
    ampl_1 = tshape * 2. * par_lp[5] * w2 * exp(-w2 * r2);
  fields[0] = y1 * ampl_1 * cos(phig10);
  fields[3] = (ndim == 3) ? z1 * ampl_1 * cos(phig10) : 0.0;
  fields[5] = fields[1];
  fields[2] = 0.0;
  fields[4] = 0.0;
}

void ora_init_lp_fields(ora_sim* s, const agpu_lp_pulse* a) {
  const int ndim = s->p.ndim;
  double par_lp[7], coords[4], f[6];
  const double sigma = 1. / (a->om0 * a->wx);
  const double eps = 1. / (a->om0 * a->wy);
  const double zra = 0.5 * a->om0 * a->wy * a->wy;
  par_lp[0] = a->om0;
  par_lp[1] = a->xf0 - a->tf;
  par_lp[2] = a->wx;
  par_lp[3] = a->wy;
  par_lp[4] = zra;
  par_lp[5] = eps;
  par_lp[6] = sigma;
  coords[3] = a->t_loc - a->tf;
  const int k1 = (ndim == 3) ? s->kz1 : 1, k2 = (ndim == 3) ? s->kz2 : 1;
  for (int k = k1; k <= k2; ++k) {
    const double zz = (ndim == 3) ? s->p.zmn + s->p.dz * (double)(k - 3) : 0.0;
    const double zzh = zz + 0.5 * s->p.dz;
    for (int j = s->jy1; j <= s->jy2; ++j) {
      const double yy = s->p.ymn + s->p.dy * (double)(j - 3), yyh = yy + 0.5 * s->p.dy;
      for (int i = s->ix1; i <= s->ix2; ++i) {
        const double xx = s->p.xmn + s->p.dx * (double)(i - 3), xxh = xx + 0.5 * s->p.dx;
        if (ndim == 3) {
          coords[0] = xxh - a->xf0; coords[1] = yy - a->ycent; coords[2] = zz - a->zcent;
          ora_lp_fields(3, a->g_prof, par_lp, coords, f);
          EBF(s, i, j, k, 1) = EBF(s, i, j, k, 1) + a->ee0 * f[0];
          coords[0] = xx - a->xf0; coords[1] = yyh - a->ycent;
          ora_lp_fields(3, a->g_prof, par_lp, coords, f);
          EBF(s, i, j, k, 2) = EBF(s, i, j, k, 2) + a->ee0 * f[1];
          coords[0] = xx - a->xf0; coords[1] = yy - a->ycent; coords[2] = zzh - a->zcent;
          ora_lp_fields(3, a->g_prof, par_lp, coords, f);
          EBF(s, i, j, k, 3) = EBF(s, i, j, k, 3) + a->ee0 * f[2];
          coords[0] = xx - a->xf0; coords[1] = yyh - a->ycent; coords[2] = zzh - a->zcent;
          ora_lp_fields(3, a->g_prof, par_lp, coords, f);
          EBF(s, i, j, k, 4) = EBF(s, i, j, k, 4) + a->ee0 * f[3];
          coords[0] = xxh - a->xf0; coords[1] = yy - a->ycent; coords[2] = zzh - a->zcent;
          ora_lp_fields(3, a->g_prof, par_lp, coords, f);
          EBF(s, i, j, k, 5) = EBF(s, i, j, k, 5) + a->ee0 * f[4];
          coords[0] = xxh - a->xf0; coords[1] = yyh - a->ycent; coords[2] = zz - a->zcent;
          ora_lp_fields(3, a->g_prof, par_lp, coords, f);
          EBF(s, i, j, k, 6) = EBF(s, i, j, k, 6) + a->ee0 * f[5];
        } else {
          coords[2] = 0.0;
          coords[0] = xxh - a->xf0; coords[1] = yy - a->ycent;
          ora_lp_fields(2, a->g_prof, par_lp, coords, f);
          EBF(s, i, j, k, 1) = EBF(s, i, j, k, 1) + a->ee0 * f[0];
          coords[0] = xx - a->xf0; coords[1] = yyh - a->ycent;
          ora_lp_fields(2, a->g_prof, par_lp, coords, f);
          EBF(s, i, j, k, 2) = EBF(s, i, j, k, 2) + a->ee0 * f[1];
          coords[0] = xxh - a->xf0; coords[1] = yyh - a->ycent;
          ora_lp_fields(2, a->g_prof, par_lp, coords, f);
          EBF(s, i, j, k, 3) = EBF(s, i, j, k, 3) + a->ee0 * f[5];
        }
      }
    }
  }
}

/* ======================================================================== */
/* A22: Envar's reductions (src/diagnostics/diag_part_and_fields.f90:485-719)*/
/* with energy_momenta (172-220) and energy_spect (126-142), one rank.       */
/* out[0..6] = ek(1:7), out[7] = ekmax, out[8..10] = psig(1:3) (the sums    */
/* of (p - <p>)^2 of 594-604), out[16..16+ne) = nde(1:ne).                  */
/* ======================================================================== */
void ora_envar_species(const ora_sim* s, int ic, double pmass, double* out) {
  const int ne = AGPU_NE, nd = s->p.ndim, cnd = s->nc;
  const int64_t np = s->np[ic];
  memset(out, 0, sizeof(double) * (16 + ne));
  double ek[7] = {0, 0, 0, 0, 0, 0, 0}, ekmax = 0.0;
  for (int64_t ip = 1; ip <= np; ++ip) {
    double xp[3] = {0, 0, 0}, vp[3] = {0, 0, 0}, gamm, gam1;
    if (nd < 3) {
      vp[0] = PART(s, ic, ip, 3);
      vp[1] = PART(s, ic, ip, 4);
      gamm = sqrt(1. + vp[0] * vp[0] + vp[1] * vp[1]);
    } else {
      for (int c = 0; c < 3; ++c) {
        xp[c] = PART(s, ic, ip, 1 + c);
        vp[c] = PART(s, ic, ip, 4 + c);
      }
      gamm = sqrt(1. + vp[0] * vp[0] + vp[1] * vp[1] + vp[2] * vp[2]);
    }
    uint64_t b;
    double slot = PART(s, ic, ip, 2 * nd + 1);
    memcpy(&b, &slot, 8);
    const int16_t charge = (int16_t)(uint16_t)(b & 0xffffu);
    uint32_t wb = (uint32_t)(b >> 32);
    float wgh;
    memcpy(&wgh, &wb, 4);
    gam1 = gamm - 1.;
    if (nd < 3) {
      for (int ik = 0; ik < cnd; ++ik) ek[ik] = ek[ik] + (double)wgh * vp[ik];
    } else {
      for (int ik = 0; ik < cnd; ++ik) ek[ik] = ek[ik] + vp[ik];
      ek[3] = ek[3] + (double)wgh * (xp[1] * vp[2] - xp[2] * vp[1]);
    }
    ek[5] = ek[5] + (double)((float)charge * wgh);
    ek[6] = ek[6] + (double)wgh * gam1;
    ekmax = fmax(ekmax, gam1);
  }
  for (int c = 0; c < 7; ++c) out[c] = ek[c];
  out[7] = ekmax;
  /* <[p - <p>]^2> sums, <p> = ek(ik) * np_norm */
  const double np_norm = (np > 0) ? 1.0 / (double)np : 1.0;
  for (int ik = 0; ik < cnd; ++ik) {
    const double m = ek[ik] * np_norm;
    double acc = 0.0;
    for (int64_t ix = 1; ix <= np; ++ix) {
      const double sg = PART(s, ic, ix, ik + cnd + 1) - m;
      acc = acc + sg * sg;
    }
    out[8 + ik] = acc;
  }
  /* energy_spect(np, ek_max, gfield) with ek_max = pmass * ekmax */
  const double ekem = pmass * ekmax;
  const double de = ekem / (double)ne;
  if (ekem < 1.e-06) return;
  for (int64_t ip = 1; ip <= np; ++ip) {
    double gamm;
    if (nd < 3)
      gamm = sqrt(1. + PART(s, ic, ip, 3) * PART(s, ic, ip, 3) + PART(s, ic, ip, 4) * PART(s, ic, ip, 4));
    else
      gamm = sqrt(1. + PART(s, ic, ip, 4) * PART(s, ic, ip, 4) + PART(s, ic, ip, 5) * PART(s, ic, ip, 5) +
                  PART(s, ic, ip, 6) * PART(s, ic, ip, 6));
    uint64_t b;
    double slot = PART(s, ic, ip, 2 * nd + 1);
    memcpy(&b, &slot, 8);
    uint32_t wb = (uint32_t)(b >> 32);
    float wgh;
    memcpy(&wgh, &wb, 4);
    const double xx = pmass * (gamm - 1.) / de;
    int ix = (int)round(xx);
    ix = (ix + 1 < ne) ? ix + 1 : ne;
    out[16 + ix - 1] = out[16 + ix - 1] + (double)wgh;
  }
}

/* Envar's field section (uniform grid): out[0..5] = dgvol * sum F^2,
   out[6..11] = max |F_c|, out[12] = max over nodes of sum_{c<=curr_ndim} E_c^2. */
void ora_envar_fields(const ora_sim* s, double* out) {
  memset(out, 0, sizeof(double) * 16);
  const double dgvol = (s->p.ndim == 2) ? s->p.dx * s->p.dy * s->p.dy : s->p.dx * s->p.dy * s->p.dz;
  for (int ik = 1; ik <= s->nf; ++ik) {
    double ekt = 0.0, mx = 0.0;
    for (int iz = s->kz1; iz <= s->kz2; ++iz)
      for (int iy = s->jy1; iy <= s->jy2; ++iy)
        for (int ix = s->ix1; ix <= s->ix2; ++ix) {
          const double v = EBF(s, ix, iy, iz, ik);
          ekt = ekt + v * v;
          mx = fmax(mx, fabs(v));
        }
    out[ik - 1] = dgvol * ekt;
    out[6 + ik - 1] = (ekt > 0.0) ? mx : 0.0;
  }
  double e2 = 0.0;
  for (int iz = s->kz1; iz <= s->kz2; ++iz)
    for (int iy = s->jy1; iy <= s->jy2; ++iy)
      for (int ix = s->ix1; ix <= s->ix2; ++ix) {
        double ef2 = 0.0;
        for (int c = 1; c <= s->nc; ++c) ef2 = ef2 + EBF(s, ix, iy, iz, c) * EBF(s, ix, iy, iz, c);
        e2 = fmax(e2, ef2);
      }
  out[12] = e2;
}

/* ======================================================================== */
/* Envelope cycle: env_run -> env_lpf2_evolve (src/dynamics/                */
/* env_evolve_in_time.f90:196-361, 363-391) for species 0, one rank, fixed  */
/* frame (ib = 2: env_maxw_solve), der_ord 2 or 3, no ionization, no       */
/* second colour, no fluid.  env(:,:,:,1:2) = A^n (Re, Im), 3:4 = A^{n-1};  */
/* av(:,:,:,1:ndim+1) is the reference's jc during the envelope part of the */
/* step.  Uniform grid: the stretch factors loc_yg/loc_zg(:,3:4) are 1, so  */
/* the factors they multiply in are left out (x * 1 == x exactly).          */
/* ======================================================================== */
#define ORA_I4(s, i, j, k, c) \
  (((size_t)(i)-1) + (size_t)(s)->n1p * (((size_t)(j)-1) + (size_t)(s)->n2p * (((size_t)(k)-1) + (size_t)(s)->n3p * ((size_t)(c)-1))))
#define ENV(s, i, j, k, c) (s)->env[ORA_I4(s, i, j, k, c)]
#define AV(s, i, j, k, c) (s)->av[ORA_I4(s, i, j, k, c)]

int ora_env_enable(ora_sim* s, const agpu_env_params* ep) {
  if (!ep || (ep->der_ord != 2 && ep->der_ord != 3)) return AGPU_E_ARG;
  const size_t c3 = (size_t)s->n1p * s->n2p * s->n3p;
  free(s->env);
  free(s->av);
  s->nav = s->p.ndim + 1;
  s->env = (double*)calloc(c3 * 4, sizeof(double));
  s->av = (double*)calloc(c3 * (size_t)s->nav, sizeof(double));
  if (!s->env || !s->av) return AGPU_E_NOMEM;
  s->ep = *ep;
  return 0;
}
int ora_set_envelope(ora_sim* s, const double* env) {
  if (!s->env) return AGPU_E_STATE;
  memcpy(s->env, env, sizeof(double) * (size_t)s->n1p * s->n2p * s->n3p * 4);
  return 0;
}
int ora_get_envelope(const ora_sim* s, double* env) {
  if (!s->env) return AGPU_E_STATE;
  memcpy(env, s->env, sizeof(double) * (size_t)s->n1p * s->n2p * s->n3p * 4);
  return 0;
}
int ora_get_env_source(const ora_sim* s, double* av) {
  if (!s->av) return AGPU_E_STATE;
  memcpy(av, s->av, sizeof(double) * (size_t)s->n1p * s->n2p * s->n3p * (size_t)s->nav);
  return 0;
}

/* init_gprof_envelope_field (g_prof) / init_envelope_field
   (src/fields/init_grid_fields.f90:274-399 / 140-272) with the arguments of
   init_envelope (src/IO/init_laser_field.f90:150-200): adds A^n (t_loc) and
   A^{n-1} (t_loc - dt) on i = ix1..nxp, j = jy1..jy2, k = kz1..kz2. */
void ora_init_envelope(ora_sim* s, const agpu_lp_pulse* a, int plane_wave) {
  const double pi = acos(-1.0);
  const int ndim = s->p.ndim;
  const double t = a->t_loc - a->tf;
  const double tm = t - s->p.dt;
  const double zra = 0.5 * a->om0 * a->wy * a->wy;
  const double pih = 0.5 * acos(-1.0);
  const double ee0 = a->ee0, wx = a->wx, wy = a->wy;
  for (int k = s->kz1; k <= s->kz2; ++k) {
    const double zz = (ndim == 3) ? (s->p.zmn + s->p.dz * (double)(k - 3) - a->zcent) / wy : 0.0;
    for (int j = s->jy1; j <= s->jy2; ++j) {
      const double yy = (s->p.ymn + s->p.dy * (double)(j - 3) - a->ycent) / wy;
      const double r2 = (ndim == 3) ? (yy * yy + zz * zz) : yy * yy;
      for (int i = s->ix1; i <= s->ix2; ++i) {
        double xx = s->p.xmn + s->p.dx * (double)(i - 3);
        xx = xx - a->xf0;
        double phi0, phi1, phi, ar, ai, ampl1, ampl0;
        if (a->g_prof) {
          phi1 = (xx - t) / wx;
          phi0 = (xx - tm) / wx;
          if (plane_wave) {
            phi = atan(xx);
            ar = ee0 * cos(phi);
            ai = -ee0 * sin(phi);
          } else {
            xx = xx / zra;
            const double w2 = 1. / (1. + xx * xx);
            const double phx = atan(xx);
            phi = phx - xx * r2 * w2;
            const double ws = (ndim == 3) ? sqrt(w2) : sqrt(sqrt(w2));
            ar = ee0 * cos(phi) * ws * exp(-w2 * r2);
            ai = -ee0 * sin(phi) * ws * exp(-w2 * r2);
          }
          ampl1 = exp(-phi1 * phi1);
          ampl0 = exp(-phi0 * phi0);
        } else {
          if (plane_wave || ndim < 3) {
            phi1 = pi * (xx - t) / wx;
            phi0 = pi * (xx - tm) / wx;
          } else {
            phi1 = pi * (t - xx) / wx;
            phi0 = pi * (tm - xx) / wx;
          }
          if (fabs(phi1) > pih) phi1 = pih;
          if (fabs(phi0) > pih) phi0 = pih;
          if (plane_wave) {
            phi = 0.0;
            ar = ee0 * cos(phi);
            ai = -ee0 * sin(phi);
          } else {
            xx = xx / zra;
            const double w2 = 1. / (1. + xx * xx);
            const double phx = atan(xx);
            phi = phx - xx * r2 * w2;
            const double ws = (ndim == 3) ? sqrt(w2) : sqrt(sqrt(w2));
            ar = ee0 * cos(phi) * ws * exp(-w2 * r2);
            ai = -ee0 * sin(phi) * ws * exp(-w2 * r2);
          }
          ampl1 = cos(phi1) * cos(phi1);
          ampl0 = cos(phi0) * cos(phi0);
        }
        ENV(s, i, j, k, 1) = ENV(s, i, j, k, 1) + ampl1 * ar;
        ENV(s, i, j, k, 2) = ENV(s, i, j, k, 2) + ampl1 * ai;
        ENV(s, i, j, k, 3) = ENV(s, i, j, k, 3) + ampl0 * ar;
        ENV(s, i, j, k, 4) = ENV(s, i, j, k, 4) + ampl0 * ai;
      }
    }
  }
}

/* env_grad (src/fields/grid_fields.f90:426-586), der_ord < 4, one rank (all
   boundaries are domain edges): av(2) = D_x av(1) at i+1/2, av(3) = D_y at
   j+1/2, av(4) = D_z at k+1/2 (3D), one-sided at the edges; the 3D edge
   branches also write the ghost planes kz1-1 and kz2+1 of av(1). */
static void ora_env_grad(ora_sim* s) {
  const double dxi = s->p.dx_inv, dyi = s->p.dy_inv, dzi = s->p.dz_inv;
  const int ix1 = s->ix1, ix2 = s->ix2, jy1 = s->jy1, jy2 = s->jy2, kz1 = s->kz1, kz2 = s->kz2;
  for (int k = kz1; k <= kz2; ++k)
    for (int j = jy1; j <= jy2; ++j) {
      AV(s, ix1, j, k, 2) = dxi * (AV(s, ix1 + 1, j, k, 1) - AV(s, ix1, j, k, 1));
      int i = ix2 - 1;
      AV(s, i, j, k, 2) = dxi * (AV(s, i + 1, j, k, 1) - AV(s, i, j, k, 1));
      AV(s, i + 1, j, k, 2) = dxi * (2. * AV(s, i, j, k, 1) - 3. * AV(s, i - 1, j, k, 1) + AV(s, i - 2, j, k, 1));
      for (i = ix1 + 1; i <= ix2 - 2; ++i) AV(s, i, j, k, 2) = dxi * (AV(s, i + 1, j, k, 1) - AV(s, i, j, k, 1));
    }
  for (int k = kz1; k <= kz2; ++k) {
    for (int i = ix1; i <= ix2; ++i)
      AV(s, i, jy2, k, 3) = dyi * (2. * AV(s, i, jy2, k, 1) - 3. * AV(s, i, jy2 - 1, k, 1) + AV(s, i, jy2 - 2, k, 1));
    for (int i = ix1; i <= ix2; ++i) AV(s, i, jy2 - 1, k, 3) = dyi * (AV(s, i, jy2, k, 1) - AV(s, i, jy2 - 1, k, 1));
  }
  for (int k = kz1; k <= kz2; ++k)
    for (int i = ix1; i <= ix2; ++i) AV(s, i, jy1, k, 3) = dyi * (AV(s, i, jy1 + 1, k, 1) - AV(s, i, jy1, k, 1));
  for (int k = kz1; k <= kz2; ++k)
    for (int j = jy1 + 1; j <= jy2 - 2; ++j)
      for (int i = ix1; i <= ix2; ++i) AV(s, i, j, k, 3) = dyi * (AV(s, i, j + 1, k, 1) - AV(s, i, j, k, 1));
  if (s->p.ndim == 2) return;
  for (int j = jy1; j <= jy2; ++j)
    for (int i = ix1; i <= ix2; ++i) {
      AV(s, i, j, kz2 + 1, 1) = 2. * AV(s, i, j, kz2, 1) - AV(s, i, j, kz2 - 1, 1);
      AV(s, i, j, kz2, 4) = dzi * (AV(s, i, j, kz2 + 1, 1) - AV(s, i, j, kz2, 1));
    }
  for (int j = jy1; j <= jy2; ++j)
    for (int i = ix1; i <= ix2; ++i) {
      AV(s, i, j, kz1 - 1, 1) = 2. * AV(s, i, j, kz1, 1) - AV(s, i, j, kz1 + 1, 1);
      AV(s, i, j, kz1, 4) = dzi * (AV(s, i, j, kz1 + 1, 1) - AV(s, i, j, kz1, 1));
    }
  for (int k = kz1 + 1; k <= kz2 - 1; ++k)
    for (int j = jy1; j <= jy2; ++j)
      for (int i = ix1; i <= ix2; ++i) AV(s, i, j, k, 4) = dzi * (AV(s, i, j, k + 1, 1) - AV(s, i, j, k, 1));
}

/* env_amp_prepare (env_evolve_in_time.f90:129-158): av(1) = |A^n|^2/2 on the
   interior, then env_grad. */
static void ora_env_amp_prepare(ora_sim* s) {
  for (int k = s->kz1; k <= s->kz2; ++k)
    for (int j = s->jy1; j <= s->jy2; ++j)
      for (int i = s->ix1; i <= s->ix2; ++i)
        AV(s, i, j, k, 1) = 0.5 * (ENV(s, i, j, k, 1) * ENV(s, i, j, k, 1) + ENV(s, i, j, k, 2) * ENV(s, i, j, k, 2));
  ora_env_grad(s);
}

/* set_env_acc (src/particles/grid_part_connect.f90:414-615): qqh gather at
   x^n of (E, B), F = |A|^2/2 and grad F; the approximate gamma
   gam_new = (gam - (dth q E.p gam - dth q^2 gradF.p / 2) / gam^2) / gam^2;
   exit pt(1:3) = q E - q^2 gradF / (2 gam_new), pt(4:6) = q B / gam_new,
   pt(7) = wgh / gam_new (2D: pt(1:2), pt(3) = q Bz / gam_new, pt(5)). */
static void ora_env_acc(ora_sim* s, int64_t np) {
  const agpu_params* p = &s->p;
  const double dth = 0.5 * p->dt;
  for (int64_t n = 1; n <= np; ++n) {
    ora_pack w = ora_unpack(PART(s, 0, n, s->ndv));
    const double charge = (double)w.charge;
    double ax1[3], axh1[3], ay1[3], ayh1[3], az1[3], azh1[3];
    int i, ih, j, jh, k, kh;
    if (p->ndim == 2) {
      double ap[7] = {0, 0, 0, 0, 0, 0, 0};
      const double xp0 = p->dx_inv * (PART(s, 0, n, 1) - p->xmn);
      const double xp1 = p->dy_inv * (PART(s, 0, n, 2) - p->ymn);
      const double u1 = PART(s, 0, n, 3), u2 = PART(s, 0, n, 4);
      ora_qqh_1d(xp0, ax1, axh1, &i, &ih);
      ora_qqh_1d(xp1, ay1, ayh1, &j, &jh);
      for (int j1 = 0; j1 <= 2; ++j1) {
        int j2 = j + j1;
        double dvol = ay1[j1];
        for (int i1 = 0; i1 <= 2; ++i1) ap[6] = ap[6] + ax1[i1] * dvol * AV(s, i + i1, j2, 1, 1);
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol1 = dvol * axh1[i1];
          ap[1] = ap[1] + dvol1 * EBF(s, ih + i1, j2, 1, 1);
          ap[4] = ap[4] + dvol1 * AV(s, ih + i1, j2, 1, 2);
        }
      }
      for (int j1 = 0; j1 <= 2; ++j1) {
        int j2 = jh + j1;
        double dvol = ayh1[j1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol1 = dvol * ax1[i1];
          ap[2] = ap[2] + dvol1 * EBF(s, i + i1, j2, 1, 2);
          ap[5] = ap[5] + dvol1 * AV(s, i + i1, j2, 1, 3);
        }
        for (int i1 = 0; i1 <= 2; ++i1) ap[3] = ap[3] + axh1[i1] * dvol * EBF(s, ih + i1, j2, 1, 3);
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
      PT(s, n, 1) = ap[1] - ap[4];
      PT(s, n, 2) = ap[2] - ap[5];
      PT(s, n, 3) = ap[3];
      PT(s, n, 5) = (double)w.wgh * gam_inv;
      continue;
    }
    double ap[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double xp0 = p->dx_inv * (PART(s, 0, n, 1) - p->xmn);
    const double xp1 = p->dy_inv * (PART(s, 0, n, 2) - p->ymn);
    const double xp2 = p->dz_inv * (PART(s, 0, n, 3) - p->zmn);
    const double u1 = PART(s, 0, n, 4), u2 = PART(s, 0, n, 5), u3 = PART(s, 0, n, 6);
    ora_qqh_1d(xp0, ax1, axh1, &i, &ih);
    ora_qqh_1d(xp1, ay1, ayh1, &j, &jh);
    ora_qqh_1d(xp2, az1, azh1, &k, &kh);
    for (int k1 = 0; k1 <= 2; ++k1) {
      int k2 = k + k1;
      for (int j1 = 0; j1 <= 2; ++j1) {
        int j2 = j + j1;
        double dvol = ay1[j1] * az1[k1];
        for (int i1 = 0; i1 <= 2; ++i1) ap[10] = ap[10] + ax1[i1] * dvol * AV(s, i1 + i, j2, k2, 1);
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol1 = dvol * axh1[i1];
          ap[1] = ap[1] + dvol1 * EBF(s, i1 + ih, j2, k2, 1);
          ap[7] = ap[7] + dvol1 * AV(s, i1 + ih, j2, k2, 2);
        }
      }
      for (int j1 = 0; j1 <= 2; ++j1) {
        int j2 = jh + j1;
        double dvol = ayh1[j1] * az1[k1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol1 = dvol * ax1[i1];
          ap[2] = ap[2] + dvol1 * EBF(s, i + i1, j2, k2, 2);
          ap[8] = ap[8] + dvol1 * AV(s, i + i1, j2, k2, 3);
        }
        for (int i1 = 0; i1 <= 2; ++i1) ap[6] = ap[6] + axh1[i1] * dvol * EBF(s, i1 + ih, j2, k2, 6);
      }
    }
    for (int k1 = 0; k1 <= 2; ++k1) {
      int k2 = kh + k1;
      for (int j1 = 0; j1 <= 2; ++j1) {
        int j2 = jh + j1;
        double dvol = ayh1[j1] * azh1[k1];
        for (int i1 = 0; i1 <= 2; ++i1) ap[4] = ap[4] + ax1[i1] * dvol * EBF(s, i1 + i, j2, k2, 4);
      }
      for (int j1 = 0; j1 <= 2; ++j1) {
        int j2 = j + j1;
        double dvol = ay1[j1] * azh1[k1];
        for (int i1 = 0; i1 <= 2; ++i1) ap[5] = ap[5] + axh1[i1] * dvol * EBF(s, ih + i1, j2, k2, 5);
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol1 = dvol * ax1[i1];
          ap[3] = ap[3] + dvol1 * EBF(s, i1 + i, j2, k2, 3);
          ap[9] = ap[9] + dvol1 * AV(s, i1 + i, j2, k2, 4);
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
    for (int c = 1; c <= 3; ++c) PT(s, n, c) = ap[c] - ap[c + 6];
    for (int c = 4; c <= 6; ++c) PT(s, n, c) = ap[c];
    PT(s, n, 7) = (double)w.wgh * gam_inv;
  }
}

/* lpf_env_momenta (src/dynamics/boris_push.f90:170-223): Boris rotation
   with the force pt(1:3) and pt(4:6) = q B / gam (2D: pt(1:2), pt(3));
   p^{n-1/2} -> p^{n+1/2}; exit pt(1:3) = x^n. */
static void ora_env_momenta(ora_sim* s, int64_t np) {
  const double alp = 0.5 * s->p.dt * s->p.lorentz_fact[0];
  for (int64_t n = 1; n <= np; ++n) {
    if (s->p.curr_ndim == 2) {
      const double pp1 = PART(s, 0, n, 3), pp2 = PART(s, 0, n, 4);
      const double efp1 = alp * PT(s, n, 1), efp2 = alp * PT(s, n, 2), efp3 = alp * PT(s, n, 3);
      const double vp1 = pp1 + efp1, vp2 = pp2 + efp2;
      const double bb1 = efp3;
      const double b2 = 1. + bb1 * bb1;
      double vph1 = vp1 + vp2 * bb1;
      double vph2 = vp2 - vp1 * bb1;
      vph1 = vph1 / b2;
      vph2 = vph2 / b2;
      PART(s, 0, n, 3) = 2. * vph1 - pp1;
      PART(s, 0, n, 4) = 2. * vph2 - pp2;
      PT(s, n, 1) = PART(s, 0, n, 1);
      PT(s, n, 2) = PART(s, 0, n, 2);
      continue;
    }
    double pp[3], efp[6], vp[3], bb[3], vph[3];
    for (int c = 0; c < 3; ++c) pp[c] = PART(s, 0, n, 4 + c);
    for (int c = 0; c < 6; ++c) efp[c] = alp * PT(s, n, 1 + c);
    for (int c = 0; c < 3; ++c) vp[c] = efp[c] + pp[c];
    for (int c = 0; c < 3; ++c) bb[c] = efp[3 + c];
    const double b2 = 1. + (bb[0] * bb[0] + bb[1] * bb[1] + bb[2] * bb[2]);
    const double bv = bb[0] * vp[0] + bb[1] * vp[1] + bb[2] * vp[2];
    vph[0] = vp[0] + vp[1] * bb[2] - vp[2] * bb[1] + bb[0] * bv;
    vph[1] = vp[1] + vp[2] * bb[0] - vp[0] * bb[2] + bb[1] * bv;
    vph[2] = vp[2] + vp[0] * bb[1] - vp[1] * bb[0] + bb[2] * bv;
    for (int c = 0; c < 3; ++c) vph[c] = vph[c] / b2;
    for (int c = 0; c < 3; ++c) PART(s, 0, n, 4 + c) = 2. * vph[c] - pp[c];
    for (int c = 0; c < 3; ++c) PT(s, n, 1 + c) = PART(s, 0, n, 1 + c);
  }
}

/* set_env_density (grid_part_connect.f90:884-952): qden weights at x^n
   (pt(1:ndim), made local in place) times wgh/gam (pt(7), 2D pt(5)) summed
   into av(1) at nodes i-1..i+1. */
static void ora_env_density(ora_sim* s, int64_t np) {
  const agpu_params* p = &s->p;
  for (int64_t n = 1; n <= np; ++n) {
    double ax1[3], ay1[3], az1[3];
    int i, j, k;
    PT(s, n, 1) = p->dx_inv * (PT(s, n, 1) - p->xmn);
    PT(s, n, 2) = p->dy_inv * (PT(s, n, 2) - p->ymn);
    if (p->ndim == 2) {
      const double wghp = PT(s, n, 5);
      ora_qden_1d(PT(s, n, 1), ax1, &i);
      ora_qden_1d(PT(s, n, 2), ay1, &j);
      i = i - 1;
      j = j - 1;
      for (int j1 = 0; j1 <= 2; ++j1) {
        double dvol = ay1[j1] * wghp;
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol1 = dvol * ax1[i1];
          AV(s, i1 + i, j + j1, 1, 1) = AV(s, i1 + i, j + j1, 1, 1) + dvol1;
        }
      }
      continue;
    }
    PT(s, n, 3) = p->dz_inv * (PT(s, n, 3) - p->zmn);
    const double wghp = PT(s, n, 7);
    ora_qden_1d(PT(s, n, 1), ax1, &i);
    ora_qden_1d(PT(s, n, 2), ay1, &j);
    ora_qden_1d(PT(s, n, 3), az1, &k);
    i = i - 1;
    j = j - 1;
    k = k - 1;
    for (int k1 = 0; k1 <= 2; ++k1)
      for (int j1 = 0; j1 <= 2; ++j1) {
        double dvol = ay1[j1] * az1[k1] * wghp;
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol1 = dvol * ax1[i1];
          AV(s, i1 + i, j + j1, k + k1, 1) = AV(s, i1 + i, j + j1, k + k1, 1) + dvol1;
        }
      }
  }
}

/* den_zyxbd (src/parallel/mpi_curr_interface.f90, called by env_den_collect,
   env_evolve_in_time.f90:37-78), one rank: fold the first ghost layer of
   av(1) into the second interior layer and copy it onto the edge node, z
   then y then x; the ghosts keep their values. */
static void ora_den_zyxbd(ora_sim* s) {
  const int i1 = s->ix1, i2 = s->ix2, j1 = s->jy1, j2 = s->jy2, k1 = s->kz1, k2 = s->kz2;
  if (s->p.ndim > 2 && s->p.ibz == 0) {
    for (int iy = j1; iy <= j2; ++iy)
      for (int ix = i1; ix <= i2; ++ix) {
        AV(s, ix, iy, k1 + 1, 1) = AV(s, ix, iy, k1 + 1, 1) + AV(s, ix, iy, k1 - 1, 1);
        AV(s, ix, iy, k1, 1) = AV(s, ix, iy, k1 + 1, 1);
      }
    for (int iy = j1; iy <= j2; ++iy)
      for (int ix = i1; ix <= i2; ++ix) {
        AV(s, ix, iy, k2 - 1, 1) = AV(s, ix, iy, k2 - 1, 1) + AV(s, ix, iy, k2 + 1, 1);
        AV(s, ix, iy, k2, 1) = AV(s, ix, iy, k2 - 1, 1);
      }
  }
  if (s->p.iby == 0 || s->p.iby == 1) {
    for (int k = k1; k <= k2; ++k)
      for (int ix = i1; ix <= i2; ++ix) {
        AV(s, ix, j1 + 1, k, 1) = AV(s, ix, j1 + 1, k, 1) + AV(s, ix, j1 - 1, k, 1);
        if (s->p.iby == 0) AV(s, ix, j1, k, 1) = AV(s, ix, j1 + 1, k, 1);
        else AV(s, ix, j1 - 1, k, 1) = 0.0;
      }
  }
  if (s->p.iby < 2) {
    for (int k = k1; k <= k2; ++k)
      for (int ix = i1; ix <= i2; ++ix) {
        AV(s, ix, j2 - 1, k, 1) = AV(s, ix, j2 - 1, k, 1) + AV(s, ix, j2 + 1, k, 1);
        AV(s, ix, j2, k, 1) = AV(s, ix, j2 - 1, k, 1);
      }
  }
  if (s->p.ibx < 2) {
    for (int k = k1; k <= k2; ++k)
      for (int iy = j1; iy <= j2; ++iy) {
        AV(s, i1 + 1, iy, k, 1) = AV(s, i1 + 1, iy, k, 1) + AV(s, i1 - 1, iy, k, 1);
        AV(s, i1, iy, k, 1) = AV(s, i1 + 1, iy, k, 1);
      }
    for (int k = k1; k <= k2; ++k)
      for (int iy = j1; iy <= j2; ++iy) {
        AV(s, i2 - 1, iy, k, 1) = AV(s, i2 - 1, iy, k, 1) + AV(s, i2 + 1, iy, k, 1);
        AV(s, i2, iy, k, 1) = AV(s, i2 - 1, iy, k, 1);
      }
  }
}

/* env_bds(env, 2, 2) (src/fields/grid_fields.f90:864-1067) on env(1:2):
   x ghosts copy the edge node (COEFF_0, a one-term DOT_PRODUCT summed from
   zero), then the y ghosts over the widened x range and the z ghosts over
   the widened x, y ranges take the quadratic extrapolation
   alpha (e1 - e2) - 2 e1 + 3 e0 (alpha = 1 on a uniform grid); ib = 1 is
   the parity copy. */
static void ora_env_bds(ora_sim* s) {
  static const int xpar[2] = {-1, 1}, ypar[2] = {1, -1}, zpar[2] = {1, 1};
  int i1 = s->ix1, i2 = s->ix2, j1 = s->jy1, j2 = s->jy2, k1 = s->kz1, k2 = s->kz2;
  const int pl = 2, pr = 2;
  for (int c = 1; c <= 2; ++c)
    for (int k = k1; k <= k2; ++k)
      for (int j = j1; j <= j2; ++j) {
        for (int point = pl; point >= 1; --point) {
          const int i = i1 - point;
          ENV(s, i, j, k, c) = (s->p.ibx == 1) ? xpar[c - 1] * ENV(s, 2 * i1 - i, j, k, c) : 0.0 + 1.0 * ENV(s, i1, j, k, c);
        }
        for (int point = 1; point <= pr; ++point) {
          const int i = i2 + point;
          ENV(s, i, j, k, c) = (s->p.ibx == 1) ? xpar[c - 1] * ENV(s, 2 * i2 - i, j, k, c) : 0.0 + 1.0 * ENV(s, i2, j, k, c);
        }
      }
  i1 = i1 - pl;
  i2 = i2 + pr;
  for (int c = 1; c <= 2; ++c)
    for (int k = k1; k <= k2; ++k)
      for (int j = j1 - pl; j <= j1 - 1; ++j)
        for (int i = i1; i <= i2; ++i)
          ENV(s, i, j, k, c) = (s->p.iby == 1) ? ypar[c - 1] * ENV(s, i, 2 * j1 - j, k, c)
                                               : (ENV(s, i, j1 + 2, k, c) - ENV(s, i, j1 + 1, k, c)) -
                                                     2 * ENV(s, i, j1 + 1, k, c) + 3 * ENV(s, i, j1, k, c);
  j1 = j1 - pl;
  for (int c = 1; c <= 2; ++c)
    for (int k = k1; k <= k2; ++k)
      for (int j = j2 + 1; j <= j2 + pr; ++j)
        for (int i = i1; i <= i2; ++i)
          ENV(s, i, j, k, c) = (s->p.iby == 1) ? ypar[c - 1] * ENV(s, i, 2 * j2 - j, k, c)
                                               : (ENV(s, i, j2 - 2, k, c) - ENV(s, i, j2 - 1, k, c)) -
                                                     2 * ENV(s, i, j2 - 1, k, c) + 3 * ENV(s, i, j2, k, c);
  j2 = j2 + pr;
  if (s->p.ndim < 3) return;
  for (int c = 1; c <= 2; ++c)
    for (int k = k1 - pl; k <= k1 - 1; ++k)
      for (int j = j1; j <= j2; ++j)
        for (int i = i1; i <= i2; ++i)
          ENV(s, i, j, k, c) = (s->p.ibz == 1) ? zpar[c - 1] * ENV(s, i, j, 2 * k1 - k, c)
                                               : (ENV(s, i, j, k1 + 2, c) - ENV(s, i, j, k1 + 1, c)) -
                                                     2 * ENV(s, i, j, k1 + 1, c) + 3 * ENV(s, i, j, k1, c);
  for (int c = 1; c <= 2; ++c)
    for (int k = k2 + 1; k <= k2 + pr; ++k)
      for (int j = j1; j <= j2; ++j)
        for (int i = i1; i <= i2; ++i)
          ENV(s, i, j, k, c) = (s->p.ibz == 1) ? zpar[c - 1] * ENV(s, i, j, 2 * k2 - k, c)
                                               : (ENV(s, i, j, k2 - 2, c) - ENV(s, i, j, k2 - 1, c)) -
                                                     2 * ENV(s, i, j, k2 - 1, c) + 3 * ENV(s, i, j, k2, c);
}

/* advance_lpf_envelope (src/dynamics/curr_and_fields_util.f90:262-299) with
   ib = 2 -> env_maxw_solve (src/fields/grid_fields.f90:588-694), whose
   potential_lapl (1356-1403) and pp_lapl (326-424) build
   S(A) = [D^2 - omp^2 chi] A in av(1:2) and first_ader adds the centred
   x-derivative term; then A^{n+1} from the second-order time scheme. */
/* env_lpf_solve (src/fields/grid_fields.f90:696-858) with ib = 0, the
   comoving frame's reduced envelope solver: the transverse Laplacian
   (pp_lapl) added to the source, times -dt on the row j = jy1 only (the
   reference's loop `do j = jy1, jy1`), the centred x-derivative of
   first_der and the three-point inversion of explicit_mat_inv row by row,
   then A^{n+1} = A^{n-1} + the result. */
static void ora_env_lpf_solve(ora_sim* s) {
  const agpu_params* p = &s->p;
  const int ix1 = s->ix1, ix2 = s->ix2, jy1 = s->jy1, jy2 = s->jy2, kz1 = s->kz1, kz2 = s->kz2;
  const double om0 = s->ep.om0, dtl = p->dt;
  const double dhx = p->dx_inv;
  const double om2 = om0 * om0;
  const double dx1_inv = 0.5 * p->dx_inv;
  const double dx_norm = dhx / om0;
  const double dx2_norm = dx_norm * dx_norm;
  const double dy2 = p->dy_inv * p->dy_inv, dz2 = p->dz_inv * p->dz_inv;
  for (int c = 1; c <= 2; ++c)
    for (int k = kz1; k <= kz2; ++k)
      for (int j = jy1; j <= jy2; ++j)
        for (int i = ix1; i <= ix2; ++i)
          AV(s, i, j, k, c) = AV(s, i, j, k, c) + dy2 * ((ENV(s, i, j + 1, k, c) - ENV(s, i, j, k, c)) -
                                                        (ENV(s, i, j, k, c) - ENV(s, i, j - 1, k, c)));
  if (p->ndim == 3)
    for (int c = 1; c <= 2; ++c)
      for (int k = kz1; k <= kz2; ++k)
        for (int j = jy1; j <= jy2; ++j)
          for (int i = ix1; i <= ix2; ++i)
            AV(s, i, j, k, c) = AV(s, i, j, k, c) + dz2 * ((ENV(s, i, j, k + 1, c) - ENV(s, i, j, k, c)) -
                                                          (ENV(s, i, j, k, c) - ENV(s, i, j, k - 1, c)));
  for (int c = 1; c <= 2; ++c)
    for (int k = kz1; k <= kz2; ++k)
      for (int i = ix1; i <= ix2; ++i) AV(s, i, jy1, k, c) = -dtl * AV(s, i, jy1, k, c);
  const int n = ix2 - ix1 + 1;
  double* w1 = (double*)malloc(sizeof(double) * (size_t)(n + 2));
  double* w2 = (double*)malloc(sizeof(double) * (size_t)(n + 2));
  for (int k = kz1; k <= kz2; ++k)
    for (int j = jy1; j <= jy2; ++j) {
      for (int i = ix1; i <= ix2; ++i) {
        w1[i - 2] = om0 * AV(s, i, j, k, 2) + dx1_inv * (AV(s, i + 1, j, k, 1) - AV(s, i - 1, j, k, 1));
        w2[i - 2] = -om0 * AV(s, i, j, k, 1) + dx1_inv * (AV(s, i + 1, j, k, 2) - AV(s, i - 1, j, k, 2));
      }
      for (int i = ix1; i <= ix2; ++i) {
        AV(s, i, j, k, 1) = w1[i - 2];
        AV(s, i, j, k, 2) = w2[i - 2];
      }
    }
  for (int c = 1; c <= 2; ++c)
    for (int k = kz1; k <= kz2; ++k)
      for (int j = jy1; j <= jy2; ++j) {
        for (int i = ix1; i <= ix2; ++i)
          w1[i - 2] = dx2_norm * (AV(s, i + 1, j, k, c) - 2. * AV(s, i, j, k, c) + AV(s, i - 1, j, k, c));
        for (int i = ix1; i <= ix2; ++i) AV(s, i, j, k, c) = (AV(s, i, j, k, c) - w1[i - 2]) / om2;
      }
  free(w1);
  free(w2);
  for (int c = 1; c <= 2; ++c)
    for (int k = kz1; k <= kz2; ++k)
      for (int j = jy1; j <= jy2; ++j)
        for (int i = ix1; i <= ix2; ++i) {
          AV(s, i, j, k, c) = AV(s, i, j, k, c) + ENV(s, i, j, k, c + 2);
          ENV(s, i, j, k, c + 2) = ENV(s, i, j, k, c);
          ENV(s, i, j, k, c) = AV(s, i, j, k, c);
        }
}

static void ora_advance_lpf_envelope(ora_sim* s) {
  const agpu_params* p = &s->p;
  const int ix1 = s->ix1, ix2 = s->ix2, jy1 = s->jy1, jy2 = s->jy2, kz1 = s->kz1, kz2 = s->kz2;
  ora_env_bds(s);
  for (int k = kz1; k <= kz2; ++k)
    for (int j = jy1; j <= jy2; ++j)
      for (int i = ix1; i <= ix2; ++i) {
        AV(s, i, j, k, 1) = -p->ompe * AV(s, i, j, k, 3) * ENV(s, i, j, k, 1);
        AV(s, i, j, k, 2) = -p->ompe * AV(s, i, j, k, 3) * ENV(s, i, j, k, 2);
      }
  if (p->w_speed < 0.0) { /* comoving: ib = 0 (curr_and_fields_util.f90:276, 292-293) */
    ora_env_lpf_solve(s);
    return;
  }
  const double om0 = s->ep.om0, dtl = p->dt;
  const double dt2 = dtl * dtl;
  const double kfact = om0 * dtl;
  const double k2_fact = 1. / (1. + kfact * kfact);
  const double dx1_inv = om0 * p->dx_inv;
  double aph1 = 1., aph2 = 0.;
  if (s->ep.der_ord == 3) {
    aph1 = dx1_inv * s->ep.opt_der1;
    aph2 = dx1_inv * 0.5 * (1. - s->ep.opt_der1);
  }
  /* potential_lapl: x part */
  const double dx2 = p->dx_inv * p->dx_inv;
  double cf1 = 1., cf2 = 0.;
  if (s->ep.der_ord > 2) {
    cf1 = 1. - 4. * s->ep.hord_der2;
    cf2 = s->ep.hord_der2;
  }
  const double dx4_1 = cf1 * dx2, dx4_2 = cf2 * dx2;
  for (int c = 1; c <= 2; ++c)
    for (int k = kz1; k <= kz2; ++k)
      for (int j = jy1; j <= jy2; ++j)
        for (int i = ix1; i <= ix2; ++i)
          AV(s, i, j, k, c) =
              AV(s, i, j, k, c) + dx4_1 * (ENV(s, i + 1, j, k, c) + ENV(s, i - 1, j, k, c) - 2. * ENV(s, i, j, k, c));
  if (s->ep.der_ord > 2)
    for (int c = 1; c <= 2; ++c)
      for (int k = kz1; k <= kz2; ++k)
        for (int j = jy1; j <= jy2; ++j)
          for (int i = ix1; i <= ix2; ++i)
            AV(s, i, j, k, c) =
                AV(s, i, j, k, c) + dx4_2 * (ENV(s, i + 2, j, k, c) + ENV(s, i - 2, j, k, c) - 2. * ENV(s, i, j, k, c));
  /* pp_lapl (der_ord < 4: cf(1) = 1) */
  const double dy2 = p->dy_inv * p->dy_inv, dz2 = p->dz_inv * p->dz_inv;
  for (int c = 1; c <= 2; ++c)
    for (int k = kz1; k <= kz2; ++k)
      for (int j = jy1; j <= jy2; ++j)
        for (int i = ix1; i <= ix2; ++i)
          AV(s, i, j, k, c) = AV(s, i, j, k, c) + dy2 * ((ENV(s, i, j + 1, k, c) - ENV(s, i, j, k, c)) -
                                                        (ENV(s, i, j, k, c) - ENV(s, i, j - 1, k, c)));
  if (p->ndim == 3)
    for (int c = 1; c <= 2; ++c)
      for (int k = kz1; k <= kz2; ++k)
        for (int j = jy1; j <= jy2; ++j)
          for (int i = ix1; i <= ix2; ++i)
            AV(s, i, j, k, c) = AV(s, i, j, k, c) + dz2 * ((ENV(s, i, j, k + 1, c) - ENV(s, i, j, k, c)) -
                                                          (ENV(s, i, j, k, c) - ENV(s, i, j, k - 1, c)));
  /* first_ader */
  for (int k = kz1; k <= kz2; ++k)
    for (int j = jy1; j <= jy2; ++j)
      for (int i = ix1; i <= ix2; ++i) {
        if (s->ep.der_ord < 3) {
          AV(s, i, j, k, 1) = AV(s, i, j, k, 1) - dx1_inv * (ENV(s, i + 1, j, k, 2) - ENV(s, i - 1, j, k, 2));
          AV(s, i, j, k, 2) = AV(s, i, j, k, 2) + dx1_inv * (ENV(s, i + 1, j, k, 1) - ENV(s, i - 1, j, k, 1));
        } else {
          AV(s, i, j, k, 1) = AV(s, i, j, k, 1) - aph1 * (ENV(s, i + 1, j, k, 2) - ENV(s, i - 1, j, k, 2)) -
                              aph2 * (ENV(s, i + 2, j, k, 2) - ENV(s, i - 2, j, k, 2));
          AV(s, i, j, k, 2) = AV(s, i, j, k, 2) + aph1 * (ENV(s, i + 1, j, k, 1) - ENV(s, i - 1, j, k, 1)) +
                              aph2 * (ENV(s, i + 2, j, k, 1) - ENV(s, i - 2, j, k, 1));
        }
      }
  for (int k = kz1; k <= kz2; ++k)
    for (int j = jy1; j <= jy2; ++j)
      for (int i = ix1; i <= ix2; ++i) {
        AV(s, i, j, k, 1) = dt2 * AV(s, i, j, k, 1) + 2. * ENV(s, i, j, k, 1) - ENV(s, i, j, k, 3) + kfact * ENV(s, i, j, k, 4);
        AV(s, i, j, k, 2) = dt2 * AV(s, i, j, k, 2) + 2. * ENV(s, i, j, k, 2) - ENV(s, i, j, k, 4) - kfact * ENV(s, i, j, k, 3);
      }
  for (int k = kz1; k <= kz2; ++k)
    for (int j = jy1; j <= jy2; ++j)
      for (int i = ix1; i <= ix2; ++i) {
        ENV(s, i, j, k, 3) = ENV(s, i, j, k, 1);
        ENV(s, i, j, k, 4) = ENV(s, i, j, k, 2);
        ENV(s, i, j, k, 1) = k2_fact * (AV(s, i, j, k, 1) - kfact * AV(s, i, j, k, 2));
        ENV(s, i, j, k, 2) = k2_fact * (AV(s, i, j, k, 2) + kfact * AV(s, i, j, k, 1));
      }
}

/* env_fields_average (env_evolve_in_time.f90:103-127): av(1) =
   |(A^{n+1} + A^n)/2|^2 / 2 = (1/8)((e1+e3)^2 + (e2+e4)^2), then env_grad. */
static void ora_env_fields_average(ora_sim* s) {
  const double frac = 1.0 / 8.;
  for (int k = s->kz1; k <= s->kz2; ++k)
    for (int j = s->jy1; j <= s->jy2; ++j)
      for (int i = s->ix1; i <= s->ix2; ++i) {
        const double a = ENV(s, i, j, k, 1) + ENV(s, i, j, k, 3);
        const double b = ENV(s, i, j, k, 2) + ENV(s, i, j, k, 4);
        AV(s, i, j, k, 1) = frac * (a * a + b * b);
      }
  ora_env_grad(s);
}

/* set_env_grad_interp (grid_part_connect.f90:760-882): qqh gather at x^n of
   grad F (av(2:4)) and F (av(1)); exit pt(1:3) = grad F, pt(4) = F (2D:
   pt(1:2), pt(3)). */
static void ora_env_grad_interp(ora_sim* s, int64_t np) {
  const agpu_params* p = &s->p;
  for (int64_t n = 1; n <= np; ++n) {
    double ax1[3], axh1[3], ay1[3], ayh1[3], az1[3], azh1[3];
    int i, ih, j, jh, k, kh;
    const double xp0 = p->dx_inv * (PART(s, 0, n, 1) - p->xmn);
    const double xp1 = p->dy_inv * (PART(s, 0, n, 2) - p->ymn);
    ora_qqh_1d(xp0, ax1, axh1, &i, &ih);
    ora_qqh_1d(xp1, ay1, ayh1, &j, &jh);
    if (p->ndim == 2) {
      double ap[4] = {0, 0, 0, 0};
      for (int j1 = 0; j1 <= 2; ++j1) {
        int j2 = j + j1;
        double dvol = ay1[j1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol1 = dvol * axh1[i1];
          ap[1] = ap[1] + dvol1 * AV(s, i1 + ih, j2, 1, 2);
          ap[3] = ap[3] + ax1[i1] * dvol * AV(s, i1 + i, j2, 1, 1);
        }
      }
      for (int j1 = 0; j1 <= 2; ++j1) {
        int j2 = jh + j1;
        double dvol = ayh1[j1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol1 = dvol * ax1[i1];
          ap[2] = ap[2] + dvol1 * AV(s, i + i1, j2, 1, 3);
        }
      }
      for (int c = 1; c <= 3; ++c) PT(s, n, c) = ap[c];
      continue;
    }
    const double xp2 = p->dz_inv * (PART(s, 0, n, 3) - p->zmn);
    ora_qqh_1d(xp2, az1, azh1, &k, &kh);
    double ap[5] = {0, 0, 0, 0, 0};
    for (int k1 = 0; k1 <= 2; ++k1) {
      int k2 = k + k1;
      for (int j1 = 0; j1 <= 2; ++j1) {
        int j2 = j + j1;
        double dvol = ay1[j1] * az1[k1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol1 = dvol * axh1[i1];
          ap[1] = ap[1] + dvol1 * AV(s, i1 + ih, j2, k2, 2);
          ap[4] = ap[4] + ax1[i1] * dvol * AV(s, i1 + i, j2, k2, 1);
        }
      }
      for (int j1 = 0; j1 <= 2; ++j1) {
        int j2 = jh + j1;
        double dvol = ayh1[j1] * az1[k1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol1 = dvol * ax1[i1];
          ap[2] = ap[2] + dvol1 * AV(s, i + i1, j2, k2, 3);
        }
      }
      k2 = kh + k1;
      for (int j1 = 0; j1 <= 2; ++j1) {
        int j2 = j + j1;
        double dvol = ay1[j1] * azh1[k1];
        for (int i1 = 0; i1 <= 2; ++i1) {
          double dvol1 = dvol * ax1[i1];
          ap[3] = ap[3] + dvol1 * AV(s, i + i1, j2, k2, 4);
        }
      }
    }
    for (int c = 1; c <= 4; ++c) PT(s, n, c) = ap[c];
  }
}

/* lpf_env_positions (src/dynamics/boris_push.f90:225-295), vbeam = 0:
   gamma^{n+1/2} with the ponderomotive correction, x^{n+1} = x^n + dt v;
   exit pt(1:3) = dt v, pt(4:6) = x^n, pt(7) = wgh_cmp (iform < 2). */
static void ora_env_positions(ora_sim* s, int64_t np) {
  const double dt_lp = s->p.dt;
  const int ch = s->ndv;
  for (int64_t n = 1; n <= np; ++n) {
    if (s->p.curr_ndim == 2) {
      const double pp1 = PART(s, 0, n, 3), pp2 = PART(s, 0, n, 4);
      double vp1 = PT(s, n, 1), vp2 = PT(s, n, 2);
      const double gam2 = 1. + (pp1 * pp1 + pp2 * pp2) + PT(s, n, 3);
      const double gam = sqrt(gam2);
      const double gam3 = gam2 * gam;
      const double b2 = 0.25 * (pp1 * vp1 + pp2 * vp2);
      double gam_inv = 1. / gam;
      gam_inv = gam_inv * (1. - dt_lp * b2 / gam3);
      vp1 = dt_lp * gam_inv * pp1;
      vp2 = dt_lp * gam_inv * pp2;
      PT(s, n, 3) = PART(s, 0, n, 1);
      PT(s, n, 4) = PART(s, 0, n, 2);
      PT(s, n, 5) = dt_lp * gam_inv;
      PART(s, 0, n, 1) = PART(s, 0, n, 1) + vp1;
      PART(s, 0, n, 2) = PART(s, 0, n, 2) + vp2;
      PT(s, n, 1) = vp1;
      PT(s, n, 2) = vp2;
      continue;
    }
    double pp[3], vp[3];
    for (int c = 0; c < 3; ++c) pp[c] = PART(s, 0, n, 4 + c);
    for (int c = 0; c < 3; ++c) vp[c] = PT(s, n, 1 + c);
    const double gam2 = 1. + (pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2]) + PT(s, n, 4);
    const double gam = sqrt(gam2);
    const double gam3 = gam2 * gam;
    const double b2 = 0.25 * (pp[0] * vp[0] + pp[1] * vp[1] + pp[2] * vp[2]);
    double gam_inv = 1. / sqrt(gam2);
    gam_inv = gam_inv * (1. - dt_lp * b2 / gam3);
    for (int c = 0; c < 3; ++c) vp[c] = dt_lp * gam_inv * pp[c];
    for (int c = 0; c < 3; ++c) PT(s, n, 4 + c) = PART(s, 0, n, 1 + c);
    PT(s, n, 7) = dt_lp * gam_inv;
    for (int c = 0; c < 3; ++c) PART(s, 0, n, 1 + c) = PART(s, 0, n, 1 + c) + vp[c];
    for (int c = 0; c < 3; ++c) PT(s, n, 1 + c) = vp[c];
  }
  if (s->p.iform < 2)
    for (int64_t n = 1; n <= np; ++n) PT(s, n, ch) = PART(s, 0, n, ch);
  /* comoving frame: x -= dt vbeam (boris_push.f90:288-294) */
  const double vbeam = s->p.w_speed < 0.0 ? -s->p.w_speed : 0.0;
  if (vbeam > 0.0)
    for (int64_t n = 1; n <= np; ++n) {
      PART(s, 0, n, 1) = PART(s, 0, n, 1) - dt_lp * vbeam;
      PT(s, n, 1) = PT(s, n, 1) - dt_lp * vbeam;
    }
}

int ora_env_run(ora_sim* s, int iter, double t, agpu_step_out* out) {
  agpu_params* p = &s->p;
  agpu_step_out dummy;
  if (!out) out = &dummy;
  memset(out, 0, sizeof(*out));
  out->ion_field_max = -1.0;
  if (!s->env) return AGPU_E_STATE;
  const size_t c3 = (size_t)s->n1p * s->n2p * s->n3p;
  memset(s->av, 0, sizeof(double) * c3 * (size_t)s->nav); /* jc(:,:,:,:) = 0.0 */
  ora_env_amp_prepare(s);
  int64_t np = s->np[0];
  memset(s->ebfp, 0, sizeof(double) * (size_t)s->ebfp_cap * (size_t)s->ndv); /* ebfp(:,:) = 0.0 */
  ora_env_acc(s, np);
  ora_env_momenta(s, np);
  memset(s->av, 0, sizeof(double) * c3); /* jc(:,:,:,1) = 0.0 */
  ora_env_density(s, np);
  ora_den_zyxbd(s);
  memcpy(s->av + 2 * c3, s->av, sizeof(double) * c3); /* jc(:,:,:,3) = jc(:,:,:,1) */
  ora_advance_lpf_envelope(s);
  ora_env_fields_average(s);
  ora_env_grad_interp(s, np);
  ora_env_positions(s, np);
  out->removed[0] += ora_cell_part_dist_step(s, 0);
  np = s->np[0];
  ora_zero_currents(s);
  if (np > 0) ora_curr_accumulate(s, 0, np);
  ora_curr_collect(s);
  ora_advance_fields(s);
  int rc = 0;
  if (p->w_speed > 0.0 && p->w_sh > 0) {
    if (t >= p->wi_time && t < p->wf_time) {
      if (iter % p->w_sh == 0) rc = ora_window_xshift(s, p->w_sh, iter, out);
    }
  }
  if (p->w_speed < 0.0 && p->w_sh > 0) { /* comoving = (w_speed < 0), vbeam = -w_speed */
    if (t >= p->wi_time && t < p->wf_time) {
      if (iter % p->w_sh == 0) rc = ora_comoving_coordinate(s, -p->w_speed, p->w_sh, iter, out);
    }
  }
  for (int ic = 0; ic < 4; ++ic) out->np[ic] = s->np[ic];
  out->xmn = p->xmn;
  out->error_bits = s->error_bits;
  return rc;
}
