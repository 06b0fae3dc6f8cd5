/*
 * aladyn_gpu.h — C-ABI of the B200 (sm_100a) laser-plasma PIC step library.
 *
 * The library runs ALaDyn's per-timestep particle-in-cell cycle on one GPU:
 * field gather (staggered quadratic/linear shapes), the exact-gamma Boris
 * push, Esirkepov charge-conserving current deposition, the leapfrog Yee
 * update with first-order open boundaries, ADK field ionization and the
 * moving window.  Particle and field arrays stay resident in device memory
 * between calls; only the arrays the host asks for come back.
 *
 * Every entry point is plain C: pointers, sizes and POD structs.  Arrays use
 * the reference's Fortran layouts so that a Fortran host can pass its own
 * allocatables through ISO_C_BINDING without copies on its side:
 *
 *   ebf(n1p, n2p, n3p, nfield)  column-major FP64, n1p = nx+5, n2p = ny+5,
 *                               n3p = nz+5 (3D) or 1 (2D); interior nodes are
 *                               the Fortran indices 3..nx+2 (ix1..ix2) etc.
 *                               (src/work/array_alloc.f90:56-83,
 *                                src/grid/set_grid_param.f90:811-829)
 *   part(ld, ndv)               column-major FP64 particle records,
 *                               2D: x, y, px, py, wgh_cmp        (ndv = 5)
 *                               3D: x, y, z, px, py, pz, wgh_cmp (ndv = 7)
 *                               (src/work/pstruct_data.f90, array_alloc.f90)
 *   wgh_cmp                     the FP64 slot that packs, little-endian,
 *                               int16 charge | int16 part_ind | float32 wgh
 *                               (src/work/precision_def.F90:33-40)
 *
 * Every call returns an int status: 0 = success, the reference's own `ier`
 * codes where they apply (2 = window shift error, 99 = particle count
 * mismatch) and the AGPU_E* codes below otherwise.  No call exits or aborts.
 * One host thread drives one handle; each handle owns one CUDA stream.
 */
#ifndef ALADYN_GPU_H
#define ALADYN_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define AGPU_OK 0
#define AGPU_E_WINDOW 2          /* window shift larger than the box (window.f90:310-315) */
#define AGPU_E_COUNT 99          /* particle count mismatch (mpi_part_interface.f90:572)  */
#define AGPU_E_ARG 101           /* invalid argument / unsupported configuration           */
#define AGPU_E_CUDA 102          /* a CUDA runtime call failed                             */
#define AGPU_E_NOMEM 103         /* device allocation failed                               */
#define AGPU_E_CAPACITY 104      /* a species outgrew its particle capacity                */
#define AGPU_E_INDEX 105         /* a particle stencil left the field array                */
#define AGPU_E_IONZ_INDEX 106    /* ionization table index beyond n_ge + 1 (clamped)       */
#define AGPU_E_NONFINITE 107     /* non-finite momentum after the push                     */
#define AGPU_E_NODEVICE 108      /* no CUDA device / extension not usable                  */
#define AGPU_E_STATE 109         /* call out of order (e.g. step before fields are set)    */

/* ---- precision forms --------------------------------------------------- */
#define AGPU_FP64 0              /* plain FP64, the reference's arithmetic order          */
#define AGPU_FP32_SPLIT 1        /* FP32 bulk, positions = int cell + FP32 offset,
                                    compensated FP32 current accumulation                 */

/* ---- particle shapes --------------------------------------------------- */
#define AGPU_SHAPE_QUADRATIC 0   /* quadratic on integer nodes, linear on half nodes
                                    (qlh, grid_part_lib.f90:110-143, 212-259) and the
                                    quadratic Esirkepov deposit: the reference        */
#define AGPU_SHAPE_CUBIC 1       /* extension with no counterpart in the reference:
                                    cubic B-spline on integer nodes (the weights of
                                    cden_3d_wgh, grid_part_lib.f90:419-454), quadratic
                                    on half nodes, cubic Esirkepov deposit            */

/* ---- device error word bits (agpu_step_out.error_bits) ----------------- */
#define AGPU_EBIT_INDEX 1u
#define AGPU_EBIT_IONZ_INDEX 2u
#define AGPU_EBIT_NONFINITE 4u
#define AGPU_EBIT_CAPACITY 8u

/* Simulation parameters: the subset of the reference's common_param /
 * grid_param module variables that the PIC step reads
 * (src/work/common_param.f90, src/grid/grid_param.f90,
 *  derived in src/start/set_init_param.f90:25-414 and
 *  src/fields/grid_field_param.f90:36-99). Single-domain (one GPU) box. */
typedef struct agpu_params {
  int32_t ndim;            /* 2 or 3                                              */
  int32_t nx, ny, nz;      /* interior cells (nx_loc, ny_loc, nz_loc); nz=1 in 2D */
  int32_t nfield;          /* 3 in 2D (Ex,Ey,Bz), 6 in 3D (Ex,Ey,Ez,Bx,By,Bz)    */
  int32_t curr_ndim;       /* 2 in 2D, 3 in 3D                                    */
  int32_t ibx, iby, ibz;   /* boundary codes; 0 (open) is the supported value     */
  int32_t iform;           /* 0, 1: Esirkepov deposition; 2: the non-conserving
                              ncdef deposit (grid_part_connect.f90:1338-1512),
                              FP64 form with quadratic shapes only             */
  int32_t precision;       /* AGPU_FP64 or AGPU_FP32_SPLIT                        */
  int32_t nsp;             /* species count, 1..4; species 0 are electrons        */
  int32_t nsp_run;         /* species that move (1 in the wake regime)            */
  int32_t w_sh;            /* window shift period in steps (0 = no window)        */
  int32_t ionz_lev;        /* 0 = no ionization, 1 = one-level ADK                */
  int32_t n_mol_atoms[4];  /* atoms per molecule of each ion species (ionz_data) */
  int32_t shape;           /* AGPU_SHAPE_QUADRATIC (the reference's qlh gather and
                              quadratic Esirkepov) or AGPU_SHAPE_CUBIC           */
  int32_t reserved_i[3];
  double dx, dy, dz;       /* cell sizes (um)                                     */
  double dx_inv, dy_inv, dz_inv;
  double dt;               /* time step (um/c)                                    */
  double xmn, ymn, zmn;    /* coordinate of interior node ix1 / jy1 / kz1         */
  double gxmin, gxmax;     /* particle box in x: keep gxmin < x <= gxmax          */
  double gymin, gymax;
  double gzmin, gzmax;
  double xmax;             /* grid x(nx): right end used by window injection      */
  double se_coeff[2];      /* x-derivative coefficients (1,0) for der_ord = 2     */
  double djc[3];           /* current normalisation (dx/2,dy/2) or (dx/3,..)      */
  double ompe;             /* 4 pi r_c n0 1e-3                                    */
  double lorentz_fact[4];  /* 1/mass per species                                  */
  /* w_speed > 0: moving window (lp_window_xshift) every w_sh steps in
   * [wi_time, wf_time).  w_speed < 0: comoving frame with vbeam = -w_speed
   * (set_init_param.f90:239-245), FP64 form only: the pushers subtract
   * dt vbeam from x, the Yee step adds the field_xadvect substeps
   * (grid_fields.f90:210-324), the envelope uses env_lpf_solve with ib = 0
   * and every w_sh steps comoving_coordinate (window.f90:227-275) moves the
   * plasma source left by vbeam w_sh dt, drops x <= gxmin and injects.     */
  double w_speed, wi_time, wf_time;
  double reserved_d[4];
  uint64_t seed;           /* Philox key for ionization draws                     */
  int64_t capacity[4];     /* device particle capacity per species                */
} agpu_params;

/* Lattice plasma source: a species loaded on a (jittered) lattice of
 * npx*npy*npz particles per cell, as the reference's multi-layer gas target
 * loader places particles at (i-1/2)/n inside each cell
 * (src/IO/init_part_distrib.f90:152-203).  The same lattice feeds the
 * moving-window injection of new columns (src/dynamics/window.f90:106-184). */
typedef struct agpu_plasma {
  int32_t ic;              /* species index (0 = electrons)                       */
  int32_t npx, npy, npz;   /* particles per cell along x, y, z (npz=1 in 2D)      */
  int32_t charge;          /* int16 charge stored in the packed slot              */
  int32_t part_ind;        /* int16 tag stored in the packed slot                 */
  float wgh;               /* float32 macro weight stored in the packed slot      */
  float reserved_f;
  double x_start, x_end;   /* plasma slab in x (um)                               */
  double y_min, y_max;     /* transverse extent (um)                              */
  double z_min, z_max;
  double jitter;           /* jitter in units of the lattice spacing, in [0,1)    */
  uint64_t seed;           /* Philox key of the jitter                            */
} agpu_plasma;

/* Linearly polarised (along y) laser pulse with a Gaussian longitudinal
 * profile (g_prof), focused at x = xf: the namelist quantities from which
 * lp_pulse (src/IO/init_laser_field.f90:33-100) and set_initial_param
 * (src/start/set_init_param.f90:291-330) derive the arguments of
 * init_lp_inc0_fields; agpu_init_laser passes them on as an agpu_lp_pulse
 * with ee0 = a0 * 2 pi / lam0, om0 = 2 pi / lam0, wx = tau_fwhm / sqrt(2 ln 2),
 * wy = w0_y, xf0 = xf, tf = xf - xc, t_loc = 0, g_prof = 1. */
typedef struct agpu_laser {
  double a0;               /* normalised amplitude                                */
  double lam0;             /* wavelength (um)                                     */
  double w0_y;             /* waist (um)                                          */
  double tau_fwhm;         /* FWHM duration (um/c)                                */
  double xc;               /* pulse centre at t = 0 (um)                          */
  double xf;               /* focus position (um)                                 */
  double y0, z0;           /* transverse centre                                   */
} agpu_laser;

/* The arguments of init_lp_inc0_fields (src/fields/init_grid_fields.f90:
 * 992-1386) for one linearly polarised pulse at normal incidence (lp = 1,
 * P mode), whose fields come from get_laser_gprof_fields_lp (g_prof = 1)
 * or get_laser_fields_lp (g_prof = 0) in 3D (init_grid_fields.f90:487-578)
 * and their 2D forms (406-485). */
typedef struct agpu_lp_pulse {
  double ee0;              /* field amplitude lp_amp = a0 * oml                     */
  double t_loc;            /* time of the set-up (0)                                */
  double tf;               /* t0_lp: focus time, xf0 - pulse centre                 */
  double wx;               /* w0_x: longitudinal profile length                     */
  double wy;               /* w0_y: waist                                           */
  double xf0;              /* focus position xf                                     */
  double om0;              /* oml = 2 pi / lam0                                     */
  double ycent, zcent;     /* transverse centre                                     */
  int32_t g_prof;          /* 1: exp(-((t-x)/wx)^2); 0: cos^2(pi (t-x)/wx), |.| <= pi/2 */
  int32_t reserved;
} agpu_lp_pulse;

typedef struct agpu_step_out {
  int64_t np[4];           /* particles per species after the step                */
  int64_t removed[4];      /* particles dropped at the box edges this step        */
  int64_t injected[4];     /* particles added by the window this step             */
  int64_t new_electrons;   /* electrons born from ionization this step            */
  double ion_field_max;    /* max |E| on ions, when refreshed (else -1)           */
  double xmn;              /* local x origin after the step                       */
  int32_t nshx;            /* cells shifted by the window this step               */
  uint32_t error_bits;     /* sticky device error word (AGPU_EBIT_*)              */
} agpu_step_out;

typedef struct agpu_diag_out {
  double field_energy[6];  /* sum over interior cells of F^2 * dx*dy*dz           */
  double max_abs_e;        /* max |E| component over interior cells               */
  double kin_energy[4];    /* sum w*(gamma-1) per species                         */
  double charge[4];        /* sum charge*w per species                            */
  double momentum[4][3];   /* sum w*p per species                                 */
  int64_t np[4];
} agpu_diag_out;

/* Per-phase device time, in milliseconds, accumulated by CUDA events on the
 * handle's stream since the last agpu_reset_timers (enabled by
 * agpu_set_profiling).  The byte counts are the algorithmic bytes that the
 * library attributes to each phase (particle records read+written, cells). */
typedef struct agpu_timers {
  double ms_push_deposit;  /* fused gather + push + deposit                       */
  double ms_yee;           /* Yee update incl. boundaries and current fold        */
  double ms_sort;          /* particle tile sort / compaction                     */
  double ms_window;        /* window shift + injection                            */
  double ms_ionize;        /* ion field, ionization draws, electron append        */
  double ms_other;
  int64_t launches_push_deposit;
  int64_t launches_yee;
  int64_t launches_total;  /* every kernel launched by the library                */
  int64_t pushes;          /* particle pushes performed                           */
  int64_t yee_cells;       /* interior cells updated by the Yee kernels           */
} agpu_timers;

typedef struct agpu_handle agpu_handle;

/* ---- lifecycle --------------------------------------------------------- */
/* Replaces v_alloc (src/work/array_alloc.f90:56) + the module state that
 * lpf2_evolve reads (src/dynamics/pic_evolve_in_time.f90:37-109). */
int agpu_create(const agpu_params* params, agpu_handle** out);
int agpu_destroy(agpu_handle* h);
const char* agpu_error_string(int code);
int agpu_device_count(int* n);

/* ---- state transfer ---------------------------------------------------- */
/* ebf(n1p,n2p,n3p,nc): the module array ebf (src/work/fstruct_data.f90:27). */
int agpu_set_fields(agpu_handle* h, const double* ebf, int32_t n1p, int32_t n2p,
                    int32_t n3p, int32_t nc);
int agpu_get_fields(agpu_handle* h, double* ebf, int32_t n1p, int32_t n2p,
                    int32_t n3p, int32_t nc);
/* jc(n1p,n2p,n3p,curr_ndim) after the last step: the normalised currents
 * that entered the E update (src/work/fstruct_data.f90:28). */
int agpu_get_currents(agpu_handle* h, double* jc, int32_t n1p, int32_t n2p,
                      int32_t n3p, int32_t nc);
/* spec(ic)%part(1:np, 1:ndv) with leading dimension ld
 * (src/work/pstruct_data.f90:31). */
int agpu_set_species(agpu_handle* h, int32_t ic, const double* part, int64_t ld,
                     int64_t np, int32_t ndv);
int agpu_get_species(agpu_handle* h, int32_t ic, double* part, int64_t ld,
                     int64_t* np, int32_t ndv);
int agpu_get_count(agpu_handle* h, int32_t ic, int64_t* np);

/* ---- dump / restart state (dump_data / restart, src/start/pic_dump.f90) -- */
/* The state a dump carries besides fields and particles: the window counter
 * xlapse of lp_window_xshift (window.f90:279-280; wi1 = nint(dx_inv*xlapse)
 * follows from it), the lattice columns already injected nptx[4] and the
 * last target column sptx_max[4] (records 3-4 of Comm-data.bin), and the
 * current box origin xmn.  A restart creates the handle with agpu_params
 * whose xmn, gxmin, gxmax and xmax are shifted by the dumped origin shift
 * (restart, pic_dump.f90:515-526), sets the plasma source, fields and
 * particles, then xlapse and nptx here.  xlapse 0 (the reference's dumps
 * do not hold it) restarts the window counters as the reference's restart
 * does.  No device work. */
int agpu_get_window_state(agpu_handle* h, double* xlapse, int64_t* nptx, int64_t* sptx_max, double* xmn);
int agpu_set_window_state(agpu_handle* h, double xlapse, const int64_t* nptx);

/* ---- initial state generated on the device ------------------------------ */
/* Lattice loader (pspecies_distribute, src/IO/init_part_distrib.f90:152-203)
 * and the window injection source (particles_inject, window.f90:106-184). */
int agpu_set_plasma_source(agpu_handle* h, const agpu_plasma* src);
int agpu_load_plasma(agpu_handle* h, int32_t ic);
int agpu_init_laser(agpu_handle* h, const agpu_laser* laser);
/* init_lp_inc0_fields (src/fields/init_grid_fields.f90:992-1386), lp = 1:
 * adds the pulse to the fields on the interior nodes, each component
 * sampled at its staggered position (3D: Ex(xh,y,z), Ey(x,yh,z), Ez(x,y,zh),
 * Bx(x,yh,zh), By(xh,y,zh), Bz(xh,yh,z); 2D: Ex(xh,y), Ey(x,yh), Bz(xh,yh))
 * with x = xmn + (i-3) dx, xh = x + dx/2 and y, z alike, in FP64. */
int agpu_init_lp_fields(agpu_handle* h, const agpu_lp_pulse* pulse);

/* ---- ionization -------------------------------------------------------- */
/* Upload w_one_lev(0:n_ge+1, 0:zmax) for ion species ic (>= 1), as built by
 * set_field_ioniz_wfunction (src/ionization/ionize.f90:38-256), with
 * de_inv = n_ge / lp_max.  Column-major: index (nk, z) -> nk + (n_ge+2)*z. */
int agpu_set_ionization_table(agpu_handle* h, int32_t ic, const double* w_one_lev,
                              int32_t n_ge, int32_t zmax, double de_inv);
/* Host-only (no device needed): build w_one_lev(0:n_ge+1, 0:atomic_number)
 * with n_ge = 10000 for the one-level model, as set_field_ioniz_wfunction
 * (src/ionization/ionize.f90:38-190) with set_ionization_coeff
 * (src/ionization/ionz_data.f90:131-245) does; de_inv = n_ge / lp_max.
 * Supported atomic numbers 1, 2, 3, 6, 7; models 1-5. */
int agpu_build_ionization_table(int32_t atomic_number, int32_t ion_min, int32_t ionz_model, double lp_max, double dt,
                                double* w_one_lev, double* de_inv);
/* ADK parameters so the library can rebuild the table itself when the ion
 * field exceeds lp_max (pic_evolve_in_time.f90:53-62). */
int agpu_set_ionization_species(agpu_handle* h, int32_t ic, int32_t atomic_number,
                                int32_t ion_min, int32_t ion_max, int32_t ionz_model,
                                double lp_max);

/* ---- the step ---------------------------------------------------------- */
/* One call of lp_run (src/dynamics/pic_evolve_in_time.f90:113-144):
 * lpf2_evolve (field boundary extrapolation, ionization, gather, push,
 * box-edge removal, Esirkepov deposit, current fold, Yee update) and, when
 * mod(iter, w_sh) == 0 inside [wi_time, wf_time), lp_window_xshift.
 * out->error_bits is the sticky device error word; once a species has
 * outgrown its capacity (AGPU_EBIT_CAPACITY, set by any call that refused
 * records for that reason) every later step returns AGPU_E_CAPACITY (the
 * reference reallocates its particle arrays instead; the device arrays are
 * sized once, by agpu_params.capacity). */
int agpu_step(agpu_handle* h, int32_t iter, double t, int32_t initial_time,
              agpu_step_out* out);
/* Host-supplied window injection: append n records to species ic
 * (add_particles semantics, src/dynamics/window.f90:39-104). */
int agpu_window_inject(agpu_handle* h, int32_t ic, const double* part, int64_t ld,
                       int64_t n, int32_t ndv);

/* ---- envelope cycle ---------------------------------------------------- */
/* The reference's Env_cycle (src/ALaDyn.F90:111-130): the laser enters as
 * the complex envelope A of its vector potential (env(:,:,:,1:2) = Re, Im of
 * A^n, env(:,:,:,3:4) = A^{n-1}) advanced by the explicit Maxwell envelope
 * solver, and species 0 feels the wake fields plus the ponderomotive force
 * of |A|^2/2.  FP64 form, one running species, der_ord 2 or 3, no
 * ionization or second colour; in the comoving frame (w_speed < 0) the
 * reduced solver env_lpf_solve (ib = 0) replaces env_maxw_solve. */
typedef struct agpu_env_params {
  double om0;              /* oml = 2 pi / lam0, the envelope's carrier frequency   */
  double opt_der1;         /* der_ord 3: (4 - nu^2)/3, else 1
                              (set_field_param, src/fields/grid_field_param.f90:54-72) */
  double hord_der2;        /* der_ord 3: -(1 - nu^2)/12, else 0                       */
  int32_t der_ord;         /* 2 or 3                                                   */
  int32_t reserved;
} agpu_env_params;
/* Allocates env(n1p,n2p,n3p,4) (zeroed) and the step's source scratch: the
 * reference's jc(:,:,:,1:ndim+1) during env_lpf2_evolve. */
int agpu_env_enable(agpu_handle* h, const agpu_env_params* ep);
/* env(n1p, n2p, n3p, 4), column-major FP64 with ghosts, as the reference's
 * module array env (src/work/fstruct_data.f90:32, src/work/array_alloc.f90:
 * 107-112). */
int agpu_set_envelope(agpu_handle* h, const double* env, int32_t n1p, int32_t n2p, int32_t n3p, int32_t nc);
int agpu_get_envelope(agpu_handle* h, double* env, int32_t n1p, int32_t n2p, int32_t n3p, int32_t nc);
/* The source scratch after the last env step (nc = ndim + 1): component 1
 * holds |A|^2/2 at t^{n+1/2} on the interior, components 2..ndim+1 its
 * staggered gradient (env_fields_average + env_grad). */
int agpu_get_env_source(agpu_handle* h, double* av, int32_t n1p, int32_t n2p, int32_t n3p, int32_t nc);
/* init_gprof_envelope_field (g_prof = 1) or init_envelope_field (g_prof =
 * 0) (src/fields/init_grid_fields.f90:140-399), called from init_envelope
 * (src/IO/init_laser_field.f90:150-200) with ee0 = a0, tf = t0_lp,
 * wx = w0_x, wy = w0_y, xf0 = xf, om0 = oml: ADDS the pulse's A^n and
 * A^{n-1} = A(t - dt) on the interior nodes; plane_wave != 0 is the pw = 0
 * branch.  Coordinates x = xmn + (i-3) dx, y and z alike. */
int agpu_init_envelope(agpu_handle* h, const agpu_lp_pulse* pulse, int32_t plane_wave);
/* One call of env_run (src/dynamics/env_evolve_in_time.f90:363-391):
 * env_lpf2_evolve (196-361) for species 0 and, when mod(iter, w_sh) == 0
 * inside [wi_time, wf_time), lp_window_xshift, which shifts env as well.
 * Outside the deterministic mode the records of species 0 are moved in
 * memory along the tile order every agpu_set_sort_interval steps (every 8
 * calls when it is 0), which changes their order, not their values. */
int agpu_env_run(agpu_handle* h, int32_t iter, double t, agpu_step_out* out);

/* ---- PWFA bunch set-up ------------------------------------------------- */
/* beam_inject (src/IO/init_beam_part_distrib.f90:474-630, uniform-grid
 * branch), called once after the fields are set: of the nb bunch records
 * part(ld, ndv) (host-built by the caller, as the reference's beam_data /
 * bunch_gen build them on the host) those inside the box (gxmin < x <= gxmax,
 * and y, z alike: mpi_beam_distribute, init_beam_part_distrib.f90:273-438)
 * are appended, in order, to species ic; their charge density
 * (set_grid_charge, src/particles/grid_part_util.f90:240-334) is solved for
 * the potential with the FP64 sine-transform Poisson solver (fft_3d_psolv /
 * fft_2d_psolv, src/IO/psolve.f90:117-238, kx/gam0 in 3D); ebf += the bunch
 * fields of initial_beam_fields (src/fields/init_grid_fields.f90:32-134)
 * with Bx = 0.  FP64 form: jc(1) holds the potential afterwards and jc(2)
 * the reference's second component, as in the reference.  Allocates its
 * scratch and cuFFT plans for the call.  Returns AGPU_E_INDEX (fields still
 * added) when a record's stencil left the array; such records are skipped in
 * the charge density. */
int agpu_beam_inject(agpu_handle* h, int32_t ic, const double* part, int64_t ld,
                     int64_t nb, int32_t ndv, double gam0);
/* The Poisson solve alone (fft_3d_psolv / fft_2d_psolv with ft_mod = 2,
 * sym = 1): rho and pot are host arrays in the field layout (n1p, n2p, n3p);
 * pot = rho with the interior replaced by the potential of
 * Laplacian(pot) = -ompe rho (x-derivative over gam2 in 3D). */
int agpu_beam_potential(agpu_handle* h, const double* rho, double* pot, double gam2);

/* ---- batched instances (parameter scans) ------------------------------- */
/* N independent simulations on one GPU, each with its own parameters,
 * handle and stream (the reference runs a scan as N separate jobs).  No
 * counterpart call in the reference: agpu_batch_run replaces running the N
 * jobs' lp_run loops one after the other.  Set each instance up through its
 * handle (agpu_batch_handle + the calls above), then agpu_batch_run advances
 * every instance by nsteps steps from its own (iter, t), starting at
 * (0, 0.0): worker threads (nthreads, 0 = one per host core, at most N) each
 * drive a share of the instances in deferred-count mode and interleave their
 * steps, so kernels of different instances overlap on the GPU.  status[i]
 * (optional, N entries) receives each instance's first error; the return
 * value is the first non-zero status.  All instances are synchronised and
 * their counts refreshed when the call returns. */
typedef struct agpu_batch agpu_batch;
int agpu_batch_create(const agpu_params* params, int32_t n, agpu_batch** b);
int agpu_batch_destroy(agpu_batch* b);
int agpu_batch_size(const agpu_batch* b, int32_t* n);
int agpu_batch_handle(agpu_batch* b, int32_t i, agpu_handle** h);
int agpu_batch_run(agpu_batch* b, int32_t nsteps, int32_t nthreads, int32_t* status);
/* Multi-instance steps (on by default): the steps between window shifts of
 * all instances of the split form with one running species run as one
 * kernel per phase over every instance together (about 15 launches per batch
 * step whatever N); first steps, window shifts and other instances step one
 * by one on worker threads.  With it off, each worker steps its instances on
 * their own streams, from per-instance step graphs when
 * agpu_batch_set_graphs is on (the default). */
int agpu_batch_set_multi(agpu_batch* b, int32_t on);
int agpu_batch_set_graphs(agpu_batch* b, int32_t on);
/* Kernel launches issued by the multi-instance steps so far (the per-instance
 * launches are in each instance's agpu_timers). */
int agpu_batch_launches(const agpu_batch* b, int64_t* n);
/* The step counter and time of instance i after the steps run so far. */
int agpu_batch_clock(const agpu_batch* b, int32_t i, int32_t* iter, double* t);

/* ---- diagnostics ------------------------------------------------------- */
/* FP64 reductions of Envar / energy_momenta
 * (src/diagnostics/diag_part_and_fields.f90:172-220, 485-719). */
int agpu_diag(agpu_handle* h, agpu_diag_out* out);

/* The reductions of Envar (src/diagnostics/diag_part_and_fields.f90:485-719)
 * with energy_momenta (172-220) and energy_spect (126-142), in the
 * reference's definitions; the host applies pmass, np_per_cell and the unit
 * constants (mev_to_joule, field_energy, e0) as Envar does. */
#define AGPU_NE 100              /* energy spectrum bins (ne, diag_part_and_fields.f90:37) */
typedef struct agpu_envar_out {
  int64_t np;              /* alive particles of the species                       */
  double ek[7];            /* energy_momenta's ek(1:7): 3D ek(1:3) = sum p_k
                              (unweighted), 2D ek(1:2) = sum wgh p_k; ek(4) = sum
                              wgh (y pz - z py) (3D); ek(5) = 0; ek(6) = sum
                              real(charge wgh, sp); ek(7) = sum wgh (gamma - 1)  */
  double ekmax;            /* max (gamma - 1)                                      */
  double psig[3];          /* sum (p_k - ek(k)/np)^2, k <= curr_ndim (Envar 594-604) */
  double nde[AGPU_NE];     /* energy_spect: weights wgh in bins min(nint(pmass
                              (gamma-1) / de) + 1, ne), de = pmass ekmax / ne;
                              zero when pmass ekmax < 1e-6                        */
} agpu_envar_out;
typedef struct agpu_envar_fields_out {
  double energy[6];        /* dgvol * sum over interior nodes of F_c^2, dgvol =
                              dx dy dz (2D: dx dy dy), components past nfield 0  */
  double fmax[6];          /* max |F_c| over the interior nodes                     */
  double e2max;            /* max over nodes of sum_{c <= curr_ndim} E_c^2          */
} agpu_envar_fields_out;
/* Species ic with its pmass = electron_mass * mass(ic) (MeV). */
int agpu_envar_species(agpu_handle* h, int32_t ic, double pmass, agpu_envar_out* out);
int agpu_envar_fields(agpu_handle* h, agpu_envar_fields_out* out);

/* Field diagnostics for callers that cannot allocate device memory (a host
 * inside a CUDA stream capture, a host whose device memory comes from its
 * own pool, a host that must not grow the device footprint).  No counterpart
 * in the reference.  Computes, from a field array already on the device
 * (d_ebf in the ebf(n1p,n2p,n3p,nf) layout, n1p = nx+5 ...), the values
 * agpu_diag reports for the fields: d_out[c] = sum over interior cells of
 * F_c^2 * dx*dy*dz (c < nf, 0 beyond), d_out[6] = max |E| (device array of
 * 7 doubles, written on `stream`, a cudaStream_t or NULL).  Calls no
 * cudaMalloc/cudaFree: its scratch is a file-scope device array of 65536 x 8
 * doubles (4 MiB) that every GPU loading the library holds until exit, which
 * limits the interior to 2^28 cells (larger grids return AGPU_E_CAPACITY).
 * The array's address is looked up in the calling thread's current context
 * by every call made outside a stream capture (a device reset, or a host
 * driving the device through a context of its own, loads the library's
 * device code again at another address); a call inside a capture uses the
 * address that the last plain call found in the same context, so make one
 * plain call in each context before capturing.  All calls share the array:
 * calls that overlap on the GPU race and must be serialised by the caller. */
int agpu_field_diag_noalloc(const double* d_ebf, int32_t ndim, int32_t nx, int32_t ny, int32_t nz, double dx, double dy,
                            double dz, double* d_out, void* stream);

/* ---- profiling --------------------------------------------------------- */
int agpu_set_profiling(agpu_handle* h, int32_t on);
int agpu_get_timers(agpu_handle* h, agpu_timers* out);
int agpu_reset_timers(agpu_handle* h);
/* The handle's cudaStream_t, for callers that time on the launching stream. */
int agpu_get_stream(agpu_handle* h, void** stream);
int agpu_synchronize(agpu_handle* h);
/* Deterministic mode: the deposit runs its particles in order in one
 * thread, so every sum happens in the reference's order and the FP64 form
 * reproduces the reference arithmetic bit for bit (slow; for verification,
 * the race-free counterpart of the atomic deposit). */
int agpu_set_deterministic(agpu_handle* h, int32_t on);
/* Deferred counts (on != 0): steps of the tiled species leave the particle
 * counts, the push count and the error word on the device, so a step
 * between window shifts makes no host synchronisation and a host can queue
 * many steps ahead.  agpu_step_out.np and .error_bits then hold the values of
 * the last synchronisation point (a window shift, agpu_get_count,
 * agpu_get_species, agpu_diag, agpu_synchronize, or turning the mode off);
 * .removed is not filled.  Off by default (the reference's lp_run reports
 * the counts every step). */
int agpu_set_deferred_counts(agpu_handle* h, int32_t on);
/* Step graphs (on != 0, effective in deferred-count mode): a step between
 * window shifts (not the first step, no ionization, profiling off, every
 * running species binned) is captured once as a CUDA graph and replayed as
 * one graph launch while the particle counts, buffers and box stay the same;
 * the next window shift or any change of the species makes the following
 * plain step capture again.  Saves the per-kernel launch cost of small
 * grids; the work done is the same. */
int agpu_set_step_graphs(agpu_handle* h, int32_t on);
/* The leapfrog Yee update (with its Mur boundaries) as one z-streaming
 * kernel writing a second field array (on), or as the six separate sweeps
 * and face kernels (off, the default).  Same results (bit for bit in FP64);
 * the fused kernel moves each field word once, but with one column tile and
 * a few planes per CTA it is latency bound and on a B200 it is slower than
 * the separate kernels in 3D (faster in 2D).  Step graphs use the separate
 * kernels. */
int agpu_set_fused_yee(agpu_handle* h, int32_t on);
/* Sort interval (steps > 0): every `steps` steps the records of each tiled
 * species are moved in memory along the step's tile permutation (removed
 * records dropped), so that memory order follows the tiles again; window
 * steps are skipped (their compaction reorders anyway).  0 (the default):
 * records move only at window compactions.  No counterpart in the reference
 * (its particles are never sorted); the physics is unchanged. */
int agpu_set_sort_interval(agpu_handle* h, int32_t steps);
/* sizeof of agpu_params, agpu_plasma, agpu_laser, agpu_step_out,
 * agpu_diag_out, agpu_timers (in that order) into sizes[0..n-1], so that a
 * binding can check its struct layouts against the library's. */
int agpu_struct_sizes(int64_t* sizes, int32_t n);

/* ---- stretched transverse grids (str_flag 1, 2) --------------------------- */
/* The reference's stretched y and z axes (src/grid/set_grid_param.f90:52-226,
 * src/grid/stretched_grid.f90:45-160): ny_stretch cells at each end follow
 * y = smin + L tan(xi) (and smax + ...), the rest stays uniform.  One axis:
 * the particle-to-cell map of map2dy_part_sind / map2dz_part_sind and the
 * metric factors loc_yg(0:n+1, 3) (d1, integer nodes) and loc_yg(0:n+1, 4)
 * (d1h, half nodes) that scale the y (z) differences of rote / rotb, the Mur
 * faces of ef_bds / bf_bds and the currents in curr_mpi_collect. */
typedef struct agpu_stretch_axis {
  double cnst;        /* n d / 2                                               */
  double smin, smax;  /* ends of the uniform part                              */
  double xs;          /* n_stretch d                                           */
  double dl_inv;      /* 1 / d                                                 */
  double dli_inv;     /* 1 / dxi, dxi = 0.4 pi / n_stretch                     */
  double ratio;       /* dxi / d                                               */
  double nl_stretch;  /* n_stretch                                             */
  double init_cell;   /* loc_ygrid%min_cell (0 for one box)                    */
  int32_t n;          /* interior cells along the axis                         */
  int32_t reserved;
  const double* d1;   /* host array d1[0 .. n+1]                               */
  const double* d1h;  /* host array d1h[0 .. n+1]                              */
} agpu_stretch_axis;
typedef struct agpu_stretch {
  int32_t on;         /* 1: y (and z in 3D) stretched, 0: uniform              */
  int32_t reserved;
  agpu_stretch_axis y, z;
} agpu_stretch;
/* FP64 form, quadratic shapes, standard cycle (no envelope, no ionization,
 * no lattice plasma source: the reference loads stretched targets on the
 * host, so the host supplies the records); the handle then uses the
 * per-particle kernels.  The box bounds in agpu_params (ymn = gymin = y(1),
 * gymax = y(ny+1), z alike) are the stretched grid's. */
int agpu_set_stretch(agpu_handle* h, const agpu_stretch* s);

/* ---- domain decomposition in y (and z) ----------------------------------- */
/* One simulation split into slabs of rows along y (or blocks of rows and
 * planes along y and z), one handle per slab (one process per GPU, or
 * several handles of one process): the reference's nprocy x nprocz
 * decomposition (src/parallel/parallel.F90:75-140).  Each handle is created
 * with its slab's params: ny = the slab's interior rows, ymn = gymin = y of
 * its first row, gymax = y after its last row (the loc_ygrid bounds), z
 * alike, everything else global.  The exchanges the reference
 * makes by MPI inside the step are handed to the caller's hook, which moves
 * the packed rows between neighbours (NCCL, CUDA-aware MPI, device copies)
 * with the pack/unpack calls below, ordered on the handle's stream:
 *   AGPU_HALO_FIELDS    after field_xyzbd, before the gather: all nfield
 *                       components (pfields_prepare, fill_ebfield_yzxbdsdata
 *                       with 2 + 2 rows, curr_and_fields_util.f90:156-174);
 *   AGPU_HALO_PARTICLES after the push of species ic: particles that crossed
 *                       a shared side have deposited their current here and
 *                       leave (part_prl_exchange, mpi_part_interface.f90:
 *                       246-466); agpu_halo_emigrants / agpu_halo_immigrants;
 *   AGPU_HALO_CURRENTS  after the deposit, before jc_xyzbd: ghost rows of jc
 *                       summed into the neighbours' rows (fill_curr_yzxbdsdata,
 *                       mpi_curr_interface.f90:51-159, 2 rows down, 3 up);
 *   AGPU_HALO_E         in the Yee step after each ef_bds: E components
 *                       (1 row up, 2 rows down, curr_and_fields_util.f90:
 *                       186-193, 241-247);
 *   AGPU_HALO_B         after bf_bds: B components (2 rows up, 1 row down,
 *                       curr_and_fields_util.f90:209-215).
 * Rows move whole: every x and z node of the array, ghosts included, so a
 * slab sees its neighbour's boundary values exactly as one box would.  A
 * non-zero return from the hook ends the step with that code.  Supported in
 * the FP64 form with quadratic shapes and the fixed frame (no envelope);
 * the slab handle uses the per-particle kernels, no step graphs and no
 * fused Yee. */
#define AGPU_HALO_FIELDS 1
#define AGPU_HALO_PARTICLES 2
#define AGPU_HALO_CURRENTS 3
#define AGPU_HALO_E 4
#define AGPU_HALO_B 5
typedef int (*agpu_halo_fn)(void* user, agpu_handle* h, int32_t point, int32_t ic);
/* lo_shared / hi_shared: the slab's low / high y side borders another slab
 * (0: a physical boundary, handled as in one box). */
int agpu_set_subdomain(agpu_handle* h, int32_t lo_shared, int32_t hi_shared, agpu_halo_fn fn, void* user);
/* The y and z split (npe_y x npe_z blocks, 3D): shared[0..3] = low y, high
 * y, low z, high z side shared.  At every point the hook exchanges the y
 * rows first and then the z planes (every x and y node, y ghosts included,
 * agpu_halo_pack_z), so corner values pass through the y neighbour, as
 * fill_ebfield_yzxbdsdata extends its z exchange over the y ghosts; the
 * particles go through the y sides, then the z sides (emigrant sides 2,
 * 3). */
int agpu_set_subdomain_yz(agpu_handle* h, const int32_t* shared, agpu_halo_fn fn, void* user);
/* Elements of a block of nrows full rows of ncomp components:
 * ncomp * nrows * n1p * n3p doubles, ordered [component][z][row][x]. */
int agpu_halo_size(agpu_handle* h, int32_t ncomp, int32_t nrows, int64_t* n);
/* Copy rows j1 .. j1+nrows-1 (1-based local rows, ghosts included) of
 * components ic1..ic2 (1-based) of the fields (what = 0) or the currents
 * (what = 1) into the device buffer buf, on the handle's stream. */
int agpu_halo_pack(agpu_handle* h, int32_t what, int32_t ic1, int32_t ic2, int32_t j1, int32_t nrows, double* buf);
/* The reverse: mode 0 writes buf into the rows, 1 adds it, 2 zeroes the
 * rows (buf unused). */
int agpu_halo_unpack(agpu_handle* h, int32_t what, int32_t ic1, int32_t ic2, int32_t j1, int32_t nrows,
                     const double* buf, int32_t mode);
/* The same along z: planes k1 .. k1+nplanes-1, every x and y node,
 * ncomp * nplanes * n1p * n2p doubles ordered [component][plane][y][x]. */
int agpu_halo_size_z(agpu_handle* h, int32_t ncomp, int32_t nplanes, int64_t* n);
int agpu_halo_pack_z(agpu_handle* h, int32_t what, int32_t ic1, int32_t ic2, int32_t k1, int32_t nplanes, double* buf);
int agpu_halo_unpack_z(agpu_handle* h, int32_t what, int32_t ic1, int32_t ic2, int32_t k1, int32_t nplanes,
                       const double* buf, int32_t mode);
/* Copy the records of species ic that left through side `side` towards
 * that neighbour, in their order, into the device buffer buf (ndv columns
 * of leading dimension ld); *n = their count (at most ld, else
 * AGPU_E_CAPACITY).  Sides 0, 1: low, high y (x inside the box, z inside or
 * beyond a shared z side); 2, 3: low, high z (x and y inside the slab, for
 * after the y exchange).  Call it at AGPU_HALO_PARTICLES; the step drops
 * them afterwards. */
int agpu_halo_emigrants(agpu_handle* h, int32_t ic, int32_t side, double* buf, int64_t ld, int64_t* n);
/* Append n records from a device buffer (ndv columns, leading dimension ld)
 * to species ic. */
int agpu_halo_immigrants(agpu_handle* h, int32_t ic, const double* buf, int64_t ld, int64_t n);

#ifdef __cplusplus
}
#endif

#endif /* ALADYN_GPU_H */
