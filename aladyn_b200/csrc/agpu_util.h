// agpu_util.h — interface of agpu_util.cu (selection, window, injection,
// laser, diagnostics, format conversions).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "agpu_common.cuh"

namespace agpu {

constexpr int SEL_BLOCK = 256;
constexpr int SEL_ITEMS = 16;
constexpr int SEL_CHUNK = SEL_BLOCK * SEL_ITEMS;

struct Scratch {
  long long* blockcnt;  // >= ceil(max particles / SEL_CHUNK)
  long long* total;     // device scalar
  long long* h_total;   // pinned host scalar
};

struct BoxBounds {
  double x0, x1, y0, y1, z0, z1;
  int use_y, use_z;
};

// Device pointers of one species in the split form (oz/pz null in 2D).
struct Part32View {
  int* cell;
  float *ox, *oy, *oz;
  float *px, *py, *pz;
  uint64_t* slot;
};

struct LatticeArgs {
  int ndim, ic, npty, nptz;
  int j0;  // first lattice row generated (1 for the whole source; a y slab's first row)
  long long i1, i2;
  int charge, part_ind;
  float wgh;
  double x_start, y_min, z_min, dxl, dyl, dzl, jitter;
  uint64_t seed;
};

// init_lp_inc0_fields for one pulse (lp = 1): par_lp of the reference and
// the grid of the set-up
struct LaserArgs {
  int ndim, g_prof;
  double ee0, t1, xf0, om0, wx, wy, zra, eps, ycent, zcent;
  double xmn, ymn, zmn, dx, dy, dz;
};

long long compact64(double* part, double* tmp, long long cap, long long np, int ndv, const BoxBounds& b, Scratch& s,
                    cudaStream_t st);
// A y slab's halo rows: copy rows j1 .. j1+nrows-1 of components
// c0 .. c0+ncomp-1 (0-based) of f, every x and z node, to or from buf
// ([component][z][row][x]); mode 0 pack (f -> buf), 1 write, 2 add, 3 zero.
void halo_rows64(double* f, const Geo& g, int c0, int ncomp, int j1, int nrows, double* buf, int mode, cudaStream_t st,
                 int sms);
// The same for planes k1 .. k1+nplanes-1 along z (every x and y node;
// buf[component][plane][y][x]).
void halo_planes64(double* f, const Geo& g, int c0, int ncomp, int k1, int nplanes, double* buf, int mode,
                   cudaStream_t st, int sms);
// Records of a slab that left through side `side` (0, 1: low, high y; 2, 3:
// low, high z) towards that neighbour (zlo, zhi: the z sides shared), in
// order, into out (leading dimension ld; records beyond ld are counted, not
// written).  Returns the count.
long long emigrants64(const double* part, long long cap, long long np, int ndv, const BoxBounds& b, int side, int zlo,
                      int zhi, double* out, long long ld, Scratch& s, cudaStream_t st);
long long compact32(const Part32View& src, const Part32View& dst, long long np, int n1p, int n2p, int nx, int ny, int nz,
                    int use_y, int use_z, Scratch& s, cudaStream_t st);
long long compact_flag64(const int* key, int dead, double* part, double* tmp, long long cap, long long np, int ndv, Scratch& s,
                         cudaStream_t st);
long long compact_flag32(const int* key, int dead, const Part32View& src, const Part32View& dst, long long np, Scratch& s,
                         cudaStream_t st);
long long append_electrons64(const int* flag, long long nion, const double* ion, long long ion_ld, double* el, long long el_ld,
                             long long ne0, long long cap, int ndim, int n_mol, unsigned int* err, Scratch& s,
                             cudaStream_t st);
long long append_electrons32(const int* flag, long long nion, const Part32View& ion, const Part32View& el, long long ne0,
                             long long cap, int n_mol, unsigned int* err, Scratch& s, cudaStream_t st);
void xshift64(double* f, const Geo& g, int nc, int wi2, int nshx, cudaStream_t st, int sms);
void xshift32(float* f, const Geo& g, int nc, int wi2, int nshx, cudaStream_t st, int sms);
void lattice64(const LatticeArgs& a, double* part, long long ld, long long n0, cudaStream_t st, int sms);
void lattice32(const LatticeArgs& a, const Part32View& p, long long n0, const Geo& g, double xmn, double ymn, double zmn,
               double dx_inv, double dy_inv, double dz_inv, cudaStream_t st, int sms);
void rec_to_split(const double* rec, long long ld, long long n, const Part32View& p, long long n0, const Geo& g, double xmn,
                  double ymn, double zmn, double dx_inv, double dy_inv, double dz_inv, cudaStream_t st, int sms);
void split_to_rec(const Part32View& p, long long n, double* rec, long long ld, const Geo& g, double xmn, double ymn, double zmn,
                  double dx, double dy, double dz, cudaStream_t st, int sms);
void f64_to_f32(const double* a, float* b, long long n, cudaStream_t st, int sms);
void f32_to_f64(const float* a, double* b, long long n, cudaStream_t st, int sms);
void f32pair_to_f64(const float* hi, const float* lo, double* b, long long n, cudaStream_t st, int sms);
void laser64(const LaserArgs& a, double* ebf, const Geo& g, cudaStream_t st, int sms);
void field_diag64(const double* ebf, const Geo& g, double dvol, double* out_e, double* out_max, cudaStream_t st, int sms);
void field_diag32(const float* ebf, const Geo& g, double dvol, double* out_e, double* out_max, cudaStream_t st, int sms);
// perm: null (records 0..n-1) or the alive records perm[0..n-1]
void part_diag64(const double* part, long long ld, long long n, int nd, const int* perm, double* out, cudaStream_t st,
                 int sms);
// key: null (every record) or the binning keys, records keyed `dead` skipped
void part_diag32(const Part32View& p, long long n, int nd, const int* key, int dead, double* out, cudaStream_t st,
                 int sms);
// Envar reductions (agpu_envar.cu): per species into d_out[0..16+AGPU_NE)
// (ek(1:7), ekmax, psig(1:3), nde(1:ne) at 16..), fields into d_out[0..13)
void envar_species(const double* part, long long ld, const Part32View* sp, const int* perm, long long n, const Geo& g,
                   double ymn, double zmn, double dy, double dz, double pmass, double* d_out, cudaStream_t st, int sms);
void envar_fields64(const double* ebf, const Geo& g, double* d_out, cudaStream_t st, int sms);
void envar_fields32(const float* ebf, const Geo& g, double* d_out, cudaStream_t st, int sms);
void max_nonneg(const double* a, long long n, double* out, cudaStream_t st, int sms);

}  // namespace agpu
