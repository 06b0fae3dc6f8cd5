// agpu_util.cu — stable selection (compaction / append), the moving-window
// field shift, lattice injection, laser initialisation and FP64 diagnostics.
// Compiled with -fmad=false: positions generated here must match the
// oracle's arithmetic bit for bit.
#include "agpu_common.cuh"
#include "agpu_util.h"
#include "agpu_select.cuh"

namespace agpu {

// ---- predicates / movers ---------------------------------------------------
struct InBox64 {
  const double *x, *y, *z;
  double x0, x1, y0, y1, z0, z1;
  int use_y, use_z;
  __device__ bool operator()(long long i) const {
    double a = x[i];
    bool k = a > x0 && a <= x1;
    if (use_y) {
      double b = y[i];
      k = k && b > y0 && b <= y1;
    }
    if (use_z) {
      double c = z[i];
      k = k && c > z0 && c <= z1;
    }
    return k;
  }
};
struct MoveCols64 {
  const double* src;
  double* dst;
  long long ld;
  int ndv;
  __device__ void operator()(long long i, long long o) const {
    for (int c = 0; c < ndv; ++c) dst[(long long)c * ld + o] = src[(long long)c * ld + i];
  }
};

long long compact64(double* part, double* tmp, long long cap, long long np, int ndv, const BoxBounds& b, Scratch& s,
                    cudaStream_t st) {
  InBox64 pr{part, part + cap, part + 2 * cap, b.x0, b.x1, b.y0, b.y1, b.z0, b.z1, b.use_y, b.use_z};
  MoveCols64 mv{part, tmp, cap, ndv};
  long long kept = select_run(pr, mv, np, s, st);
  return kept;
}

__global__ void k_halo_rows64(double* f, Geo g, int c0, int ncomp, int j1, int nrows, double* buf, int mode) {
  const long long n1p = g.n1p, n3p = g.n3p;
  const long long total = (long long)ncomp * n3p * nrows * n1p;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const long long i = t % n1p;
    const long long r = (t / n1p) % nrows;
    const long long k = (t / (n1p * nrows)) % n3p;
    const long long c = t / (n1p * nrows * n3p);
    double* v = f + g.ncell * (c0 + c) + i + n1p * ((j1 - 1 + r) + (long long)g.n2p * k);
    if (mode == 0) buf[t] = *v;
    else if (mode == 1) *v = buf[t];
    else if (mode == 2) *v = *v + buf[t];
    else *v = 0.0;
  }
}
// planes k1 .. k1+nplanes-1 of components c0 .. c0+ncomp-1, every x and y
// node: buf[component][plane][y][x]
__global__ void k_halo_planes64(double* f, Geo g, int c0, int ncomp, int k1, int nplanes, double* buf, int mode) {
  const long long pl = (long long)g.n1p * g.n2p;
  const long long total = (long long)ncomp * nplanes * pl;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const long long q = t % pl;
    const long long r = (t / pl) % nplanes;
    const long long c = t / (pl * nplanes);
    double* v = f + g.ncell * (c0 + c) + pl * (k1 - 1 + r) + q;
    if (mode == 0) buf[t] = *v;
    else if (mode == 1) *v = buf[t];
    else if (mode == 2) *v = *v + buf[t];
    else *v = 0.0;
  }
}
void halo_planes64(double* f, const Geo& g, int c0, int ncomp, int k1, int nplanes, double* buf, int mode,
                   cudaStream_t st, int sms) {
  const long long total = (long long)ncomp * nplanes * g.n1p * g.n2p;
  if (total <= 0) return;
  k_halo_planes64<<<grid_for(total, 256, sms, 8), 256, 0, st>>>(f, g, c0, ncomp, k1, nplanes, buf, mode);
}

void halo_rows64(double* f, const Geo& g, int c0, int ncomp, int j1, int nrows, double* buf, int mode, cudaStream_t st,
                 int sms) {
  const long long total = (long long)ncomp * g.n3p * nrows * g.n1p;
  if (total <= 0) return;
  k_halo_rows64<<<grid_for(total, 256, sms, 8), 256, 0, st>>>(f, g, c0, ncomp, j1, nrows, buf, mode);
}

void halo_planes64(double* f, const Geo& g, int c0, int ncomp, int k1, int nplanes, double* buf, int mode,
                   cudaStream_t st, int sms);

// Records that left through side `side` (0, 1: low, high y; 2, 3: low, high
// z) of a slab and go to that neighbour: inside the x box, and, along the
// other transverse axis, inside the slab (y, for the z sides: the y
// exchange has run) or beyond a side that is shared too (z, for the y
// sides: a corner crosser travels on through the z exchange).
struct Emigrant64 {
  const double *x, *y, *z;
  BoxBounds b;
  int side;
  int zlo, zhi;  // z sides shared
  __device__ bool operator()(long long i) const {
    const double a = x[i], c = y[i];
    if (!(a > b.x0 && a <= b.x1)) return false;
    if (side < 2) {
      if (b.use_z) {
        const double d = z[i];
        const bool zin = (d > b.z0 && d <= b.z1) || (zlo && d <= b.z0) || (zhi && d > b.z1);
        if (!zin) return false;
      }
      return side == 0 ? c <= b.y0 : c > b.y1;
    }
    if (!(c > b.y0 && c <= b.y1)) return false;
    const double d = z[i];
    return side == 2 ? d <= b.z0 : d > b.z1;
  }
};
struct MoveColsOut64 {
  const double* src;
  long long src_ld;
  double* dst;
  long long dst_ld;
  int ndv;
  __device__ void operator()(long long i, long long o) const {
    if (o >= dst_ld) return;
    for (int c = 0; c < ndv; ++c) dst[(long long)c * dst_ld + o] = src[(long long)c * src_ld + i];
  }
};
long long emigrants64(const double* part, long long cap, long long np, int ndv, const BoxBounds& b, int side, int zlo,
                      int zhi, double* out, long long ld, Scratch& s, cudaStream_t st) {
  Emigrant64 pr{part, part + cap, part + 2 * cap, b, side, zlo, zhi};
  MoveColsOut64 mv{part, cap, out, ld, ndv};
  return select_run(pr, mv, np, s, st);
}

// Split form: x_loc = (ix - 3) + ox; keep 0 < x_loc <= nx along each axis,
// evaluated exactly from the integer node and the offset in [-0.5, 0.5).
struct InBox32 {
  const int* cell;
  const float *ox, *oy, *oz;
  int n1p, n2p, nx, ny, nz;
  int use_y, use_z;
  __device__ static bool inside(int i, float o, int n) {
    // 0 < (i-3) + o <= n
    int m = i - 3;
    bool gt0 = (m > 0) || (m == 0 && o > 0.f);
    bool le = (m < n) || (m == n && o <= 0.f);
    return gt0 && le;
  }
  __device__ bool operator()(long long q) const {
    int c = cell[q];
    int i = c % n1p + 1;
    int r = c / n1p;
    int j = r % n2p + 1;
    int k = r / n2p + 1;
    bool kp = inside(i, ox[q], nx);
    if (use_y) kp = kp && inside(j, oy[q], ny);
    if (use_z) kp = kp && inside(k, oz[q], nz);
    return kp;
  }
};
struct MoveSplit {
  Part32View src, dst;
  __device__ void operator()(long long i, long long o) const {
    dst.cell[o] = src.cell[i];
    dst.ox[o] = src.ox[i];
    dst.oy[o] = src.oy[i];
    dst.px[o] = src.px[i];
    dst.py[o] = src.py[i];
    dst.slot[o] = src.slot[i];
    if (src.oz) {
      dst.oz[o] = src.oz[i];
      dst.pz[o] = src.pz[i];
    }
  }
};

long long compact32(const Part32View& src, const Part32View& dst, long long np, int n1p, int n2p, int nx, int ny, int nz,
                    int use_y, int use_z, Scratch& s, cudaStream_t st) {
  InBox32 pr{src.cell, src.ox, src.oy, src.oz, n1p, n2p, nx, ny, nz, use_y, use_z};
  MoveSplit mv{src, dst};
  return select_run(pr, mv, np, s, st);
}

// ---- drop the records whose tile key marks them removed (memory order) ----
struct KeyLive {
  const int* key;
  int dead;
  __device__ bool operator()(long long i) const { return key[i] != dead; }
};
long long compact_flag64(const int* key, int dead, double* part, double* tmp, long long cap, long long np, int ndv, Scratch& s,
                         cudaStream_t st) {
  KeyLive pr{key, dead};
  MoveCols64 mv{part, tmp, cap, ndv};
  return select_run(pr, mv, np, s, st);
}
long long compact_flag32(const int* key, int dead, const Part32View& src, const Part32View& dst, long long np, Scratch& s,
                         cudaStream_t st) {
  KeyLive pr{key, dead};
  MoveSplit mv{src, dst};
  return select_run(pr, mv, np, s, st);
}

// ---- ionization electron append (ionization_electrons_inject,
// src/ionization/ionize.f90:258-322): for each ionized ion, in ion order, one
// electron at the ion position with zero momentum and
// wgh = ion wgh * n_mol_atoms, charge = part_ind = -1.
struct FlagPred {
  const int* flag;
  __device__ bool operator()(long long i) const { return flag[i] != 0; }
};
struct AppendElectron64 {
  const double* ion;
  long long ion_ld;
  double* el;
  long long el_ld;
  long long ne0, cap;
  int ndim, n_mol;
  unsigned int* err;
  __device__ void operator()(long long i, long long o) const {
    long long q = ne0 + o;
    if (q >= cap) {
      atomicOr(err, AGPU_EBIT_CAPACITY);
      return;
    }
    int nd = ndim;  // positions 0..nd-1, momenta nd..2nd-1, slot 2nd
    for (int c = 0; c < nd; ++c) el[(long long)c * el_ld + q] = ion[(long long)c * ion_ld + i];
    for (int c = nd; c < 2 * nd; ++c) el[(long long)c * el_ld + q] = 0.0;
    uint64_t sl = dbits(ion[(long long)(2 * nd) * ion_ld + i]);
    float w = slot_wgh(sl) * (float)n_mol;
    el[(long long)(2 * nd) * el_ld + q] = bitsd(make_slot(-1, -1, w));
  }
};
long long append_electrons64(const int* flag, long long nion, const double* ion, long long ion_ld, double* el, long long el_ld,
                             long long ne0, long long cap, int ndim, int n_mol, unsigned int* err, Scratch& s,
                             cudaStream_t st) {
  FlagPred pr{flag};
  AppendElectron64 mv{ion, ion_ld, el, el_ld, ne0, cap, ndim, n_mol, err};
  return select_run(pr, mv, nion, s, st);
}

struct AppendElectron32 {
  Part32View ion, el;
  long long ne0, cap;
  int n_mol;
  unsigned int* err;
  __device__ void operator()(long long i, long long o) const {
    long long q = ne0 + o;
    if (q >= cap) {
      atomicOr(err, AGPU_EBIT_CAPACITY);
      return;
    }
    el.cell[q] = ion.cell[i];
    el.ox[q] = ion.ox[i];
    el.oy[q] = ion.oy[i];
    el.px[q] = 0.f;
    el.py[q] = 0.f;
    if (el.oz) {
      el.oz[q] = ion.oz[i];
      el.pz[q] = 0.f;
    }
    uint64_t sl = ion.slot[i];
    el.slot[q] = make_slot(-1, -1, slot_wgh(sl) * (float)n_mol);
  }
};
long long append_electrons32(const int* flag, long long nion, const Part32View& ion, const Part32View& el, long long ne0,
                             long long cap, int n_mol, unsigned int* err, Scratch& s, cudaStream_t st) {
  FlagPred pr{flag};
  AppendElectron32 mv{ion, el, ne0, cap, n_mol, err};
  return select_run(pr, mv, nion, s, st);
}

// ============================================================================
// fields_left_xshift (src/parallel/mpi_field_interface.f90:299-359): for each
// (iy, iz, comp) row over the interior y/z range, f(ix) = f(ix + nshx) for
// ix = ix1..wi2, then f(wi2+1 : wi2+nshx) = 0.  One block per row; chunks
// move left in increasing order, every read of a chunk before its writes.
// ============================================================================
template <typename T>
__global__ void k_xshift(T* f, Geo g, int nc, int wi2, int nshx) {
  extern __shared__ unsigned char smem_raw[];
  T* buf = reinterpret_cast<T*>(smem_raw);
  int ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  long long rows = (long long)ny * nz * nc;
  for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
    int iy = g.jy1 + (int)(r % ny);
    int iz = g.kz1 + (int)((r / ny) % nz);
    int ic = (int)(r / ((long long)ny * nz));
    T* row = f + g.ncell * ic + goff(g, 1, iy, iz);  // row[ix-1] = f(ix)
    for (int c0 = g.ix1; c0 <= wi2; c0 += blockDim.x) {
      int ix = c0 + threadIdx.x;
      if (ix <= wi2) buf[threadIdx.x] = row[ix + nshx - 1];
      __syncthreads();
      if (ix <= wi2) row[ix - 1] = buf[threadIdx.x];
      __syncthreads();
    }
    for (int ix = wi2 + 1 + threadIdx.x; ix <= wi2 + nshx; ix += blockDim.x) row[ix - 1] = (T)0;
  }
}
void xshift64(double* f, const Geo& g, int nc, int wi2, int nshx, cudaStream_t st, int sms) {
  long long rows = (long long)(g.jy2 - g.jy1 + 1) * (g.kz2 - g.kz1 + 1) * nc;
  int grid = (int)(rows < (long long)sms * 16 ? rows : (long long)sms * 16);
  k_xshift<double><<<grid, 256, 256 * sizeof(double), st>>>(f, g, nc, wi2, nshx);
}
void xshift32(float* f, const Geo& g, int nc, int wi2, int nshx, cudaStream_t st, int sms) {
  long long rows = (long long)(g.jy2 - g.jy1 + 1) * (g.kz2 - g.kz1 + 1) * nc;
  int grid = (int)(rows < (long long)sms * 16 ? rows : (long long)sms * 16);
  k_xshift<float><<<grid, 256, 256 * sizeof(float), st>>>(f, g, nc, wi2, nshx);
}

// ============================================================================
// Lattice columns (add_particles, src/dynamics/window.f90:39-104): particle q
// of the block of columns i1..i2 is column i1 + q % ncol, row
// j = 1 + (q / ncol) % npty, k = 1 + q / (ncol*npty) (x fastest), with the
// jittered lattice position of the oracle's ora_lattice_particle.
// ============================================================================
__device__ __forceinline__ void lattice_pos(const LatticeArgs& a, long long ixl, int j, int k, double* x, double* y,
                                            double* z) {
  uint32_t r[4];
  philox4x32_10((uint32_t)ixl, (uint32_t)j, (uint32_t)k, (uint32_t)a.ic, (uint32_t)a.seed, (uint32_t)(a.seed >> 32), r);
  double jx = a.jitter * (u32d(r[0]) - 0.5);
  double jy = a.jitter * (u32d(r[1]) - 0.5);
  double jz = a.jitter * (u32d(r[2]) - 0.5);
  *x = a.x_start + ((double)ixl - 0.5 + jx) * a.dxl;
  *y = a.y_min + ((double)j - 0.5 + jy) * a.dyl;
  *z = (a.ndim == 3) ? a.z_min + ((double)k - 0.5 + jz) * a.dzl : 0.0;
}

__global__ void k_lattice64(LatticeArgs a, double* part, long long ld, long long n0) {
  long long ncol = a.i2 - a.i1 + 1;
  long long total = ncol * a.npty * a.nptz;
  uint64_t sl = make_slot(a.charge, a.part_ind, a.wgh);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    long long ix = a.i1 + q % ncol;
    int j = a.j0 + (int)((q / ncol) % a.npty);
    int k = 1 + (int)(q / (ncol * a.npty));
    double x, y, z;
    lattice_pos(a, ix, j, k, &x, &y, &z);
    long long n = n0 + q;
    part[n] = x;
    part[ld + n] = y;
    if (a.ndim == 3) {
      part[2 * ld + n] = z;
      part[3 * ld + n] = 0.;
      part[4 * ld + n] = 0.;
      part[5 * ld + n] = 0.;
      part[6 * ld + n] = bitsd(sl);
    } else {
      part[2 * ld + n] = 0.;
      part[3 * ld + n] = 0.;
      part[4 * ld + n] = bitsd(sl);
    }
  }
}
void lattice64(const LatticeArgs& a, double* part, long long ld, long long n0, cudaStream_t st, int sms) {
  long long total = (a.i2 - a.i1 + 1) * (long long)a.npty * a.nptz;
  if (total <= 0) return;
  k_lattice64<<<grid_for(total, 256, sms, 16), 256, 0, st>>>(a, part, ld, n0);
}

// FP64 absolute position -> split (node, offset) with the qden index rule.
__device__ __forceinline__ void to_split(double xabs, double mn, double dinv, int* node, float* off) {
  double xx = 3.0 + dinv * (xabs - mn);
  int i = (int)(xx + 0.5);
  *node = i;
  *off = (float)(xx - (double)i);
}

__global__ void k_lattice32(LatticeArgs a, Part32View p, long long n0, Geo g, double xmn, double ymn, double zmn,
                            double dx_inv, double dy_inv, double dz_inv) {
  long long ncol = a.i2 - a.i1 + 1;
  long long total = ncol * a.npty * a.nptz;
  uint64_t sl = make_slot(a.charge, a.part_ind, a.wgh);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    long long ix = a.i1 + q % ncol;
    int j = a.j0 + (int)((q / ncol) % a.npty);
    int k = 1 + (int)(q / (ncol * a.npty));
    double x, y, z;
    lattice_pos(a, ix, j, k, &x, &y, &z);
    long long n = n0 + q;
    int ni, nj, nk = 1;
    float fx, fy, fz = 0.f;
    to_split(x, xmn, dx_inv, &ni, &fx);
    to_split(y, ymn, dy_inv, &nj, &fy);
    if (a.ndim == 3) to_split(z, zmn, dz_inv, &nk, &fz);
    p.cell[n] = (int)goff(g, ni, nj, nk);
    p.ox[n] = fx;
    p.oy[n] = fy;
    p.px[n] = 0.f;
    p.py[n] = 0.f;
    if (p.oz) {
      p.oz[n] = fz;
      p.pz[n] = 0.f;
    }
    p.slot[n] = sl;
  }
}
void lattice32(const LatticeArgs& a, const Part32View& p, long long n0, const Geo& g, double xmn, double ymn, double zmn,
               double dx_inv, double dy_inv, double dz_inv, cudaStream_t st, int sms) {
  long long total = (a.i2 - a.i1 + 1) * (long long)a.npty * a.nptz;
  if (total <= 0) return;
  k_lattice32<<<grid_for(total, 256, sms, 16), 256, 0, st>>>(a, p, n0, g, xmn, ymn, zmn, dx_inv, dy_inv, dz_inv);
}

// ---- conversions between the FP64 Fortran records and the split form -----
__global__ void k_rec_to_split(const double* rec, long long ld, long long n, Part32View p, long long n0, Geo g, double xmn,
                               double ymn, double zmn, double dx_inv, double dy_inv, double dz_inv) {
  int nd = g.ndim;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int ni, nj, nk = 1;
    float fx, fy, fz = 0.f;
    to_split(rec[q], xmn, dx_inv, &ni, &fx);
    to_split(rec[ld + q], ymn, dy_inv, &nj, &fy);
    if (nd == 3) to_split(rec[2 * ld + q], zmn, dz_inv, &nk, &fz);
    long long o = n0 + q;
    p.cell[o] = (int)goff(g, ni, nj, nk);
    p.ox[o] = fx;
    p.oy[o] = fy;
    p.px[o] = (float)rec[nd * ld + q];
    p.py[o] = (float)rec[(nd + 1) * ld + q];
    if (nd == 3) {
      p.oz[o] = fz;
      p.pz[o] = (float)rec[5 * ld + q];
    }
    p.slot[o] = dbits(rec[2 * nd * ld + q]);
  }
}
void rec_to_split(const double* rec, long long ld, long long n, const Part32View& p, long long n0, const Geo& g, double xmn,
                  double ymn, double zmn, double dx_inv, double dy_inv, double dz_inv, cudaStream_t st, int sms) {
  if (n <= 0) return;
  k_rec_to_split<<<grid_for(n, 256, sms, 16), 256, 0, st>>>(rec, ld, n, p, n0, g, xmn, ymn, zmn, dx_inv, dy_inv, dz_inv);
}
__global__ void k_split_to_rec(Part32View p, long long n, double* rec, long long ld, Geo g, double xmn, double ymn, double zmn,
                               double dx, double dy, double dz) {
  int nd = g.ndim;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int c = p.cell[q];
    int i = c % g.n1p + 1;
    int r = c / g.n1p;
    int j = r % g.n2p + 1;
    int k = r / g.n2p + 1;
    rec[q] = xmn + ((double)(i - 3) + (double)p.ox[q]) * dx;
    rec[ld + q] = ymn + ((double)(j - 3) + (double)p.oy[q]) * dy;
    if (nd == 3) rec[2 * ld + q] = zmn + ((double)(k - 3) + (double)p.oz[q]) * dz;
    rec[nd * ld + q] = (double)p.px[q];
    rec[(nd + 1) * ld + q] = (double)p.py[q];
    if (nd == 3) rec[5 * ld + q] = (double)p.pz[q];
    rec[2 * nd * ld + q] = bitsd(p.slot[q]);
  }
}
void split_to_rec(const Part32View& p, long long n, double* rec, long long ld, const Geo& g, double xmn, double ymn, double zmn,
                  double dx, double dy, double dz, cudaStream_t st, int sms) {
  if (n <= 0) return;
  k_split_to_rec<<<grid_for(n, 256, sms, 16), 256, 0, st>>>(p, n, rec, ld, g, xmn, ymn, zmn, dx, dy, dz);
}
__global__ void k_f64_to_f32(const double* a, float* b, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    b[q] = (float)a[q];
}
__global__ void k_f32_to_f64(const float* a, double* b, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    b[q] = (double)a[q];
}
__global__ void k_f32pair_to_f64(const float* hi, const float* lo, double* b, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    b[q] = (double)hi[q] + (double)lo[q];
}
void f64_to_f32(const double* a, float* b, long long n, cudaStream_t st, int sms) {
  k_f64_to_f32<<<grid_for(n, 256, sms, 16), 256, 0, st>>>(a, b, n);
}
void f32_to_f64(const float* a, double* b, long long n, cudaStream_t st, int sms) {
  k_f32_to_f64<<<grid_for(n, 256, sms, 16), 256, 0, st>>>(a, b, n);
}
void f32pair_to_f64(const float* hi, const float* lo, double* b, long long n, cudaStream_t st, int sms) {
  k_f32pair_to_f64<<<grid_for(n, 256, sms, 16), 256, 0, st>>>(hi, lo, b, n);
}

// ============================================================================
// Laser: init_lp_inc0_fields (src/fields/init_grid_fields.f90:992-1386),
// lp = 1 (linear polarisation, normal incidence): every interior node gets
// ee0 times the pulse field of its component at the component's staggered
// position.  lp_fields is get_laser_gprof_fields_lp / get_laser_fields_lp
// (init_grid_fields.f90:487-578) in 3D and their 2D forms (406-485), in the
// reference's order of operations; (cx, cy, cz) = position - (xf0, yc, zc),
// a.t1 = t_loc - tf.  FP64 throughout (this file is built without FMA
// contraction).
// ============================================================================
__device__ void lp_fields(const LaserArgs& a, double cx, double cy, double cz, double f[6]) {
  const double pi = 3.141592653589793;
  double x1 = cx;
  const double y1 = cy / a.wy;
  const double z1 = (a.ndim == 3) ? cz / a.wy : 0.0;
  const double t1 = a.t1;
  const double r2 = (a.ndim == 3) ? y1 * y1 + z1 * z1 : y1 * y1;
  const double phi0 = a.om0 * (t1 - x1);
  double phi1;
  if (a.g_prof) {
    phi1 = (t1 - x1) / a.wx;
  } else {
    phi1 = pi * (t1 - x1) / a.wx;
    if (fabs(phi1) > 0.5 * pi) phi1 = 0.5 * pi;
  }
  x1 = x1 / a.zra;
  const double w2 = 1. / (1. + x1 * x1);
  const double phx = (a.ndim == 3) ? atan(x1) : 0.5 * atan(x1);
  const double phig00 = phi0 + phx - x1 * r2 * w2;
  const double phig10 = phig00 + phx;
  const double tshape = a.g_prof ? exp(-phi1 * phi1) : cos(phi1) * cos(phi1);
  const double wshape = ((a.ndim == 3) ? sqrt(w2) : sqrt(sqrt(w2))) * exp(-w2 * r2);
  const double ampl = tshape * sin(phig00);
  f[1] = wshape * ampl;
  // the 3D Gaussian form multiplies in another order (init_grid_fields.f90:570)
  const double ampl_1 = (a.g_prof && a.ndim == 3) ? 2. * a.eps * tshape * w2 * exp(-w2 * r2)
                                                  : tshape * 2. * a.eps * w2 * exp(-w2 * r2);
  f[0] = y1 * ampl_1 * cos(phig10);
  f[3] = (a.ndim == 3) ? z1 * ampl_1 * cos(phig10) : 0.0;
  f[5] = f[1];
  f[2] = 0.0;
  f[4] = 0.0;
}
__global__ void k_laser64(LaserArgs a, double* ebf, Geo g) {
  const int nx = g.ix2 - g.ix1 + 1, ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  const long long total = (long long)nx * ny * nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int i = g.ix1 + (int)(t % nx);
    const int j = g.jy1 + (int)((t / nx) % ny);
    const int k = g.kz1 + (int)(t / ((long long)nx * ny));
    const double xx = a.xmn + a.dx * (double)(i - 3), xxh = xx + 0.5 * a.dx;
    const double yy = a.ymn + a.dy * (double)(j - 3), yyh = yy + 0.5 * a.dy;
    const double zz = (g.ndim == 3) ? a.zmn + a.dz * (double)(k - 3) : 0.0, zzh = zz + 0.5 * a.dz;
    const long long o = goff(g, i, j, k);
    double f[6];
    if (g.ndim == 3) {
      lp_fields(a, xxh - a.xf0, yy - a.ycent, zz - a.zcent, f);  // Ex(xxh, yy, zz)
      ebf[o] += a.ee0 * f[0];
      lp_fields(a, xx - a.xf0, yyh - a.ycent, zz - a.zcent, f);  // Ey(xx, yyh, zz)
      ebf[g.ncell + o] += a.ee0 * f[1];
      lp_fields(a, xx - a.xf0, yy - a.ycent, zzh - a.zcent, f);  // Ez(xx, yy, zzh)
      ebf[2 * g.ncell + o] += a.ee0 * f[2];
      lp_fields(a, xx - a.xf0, yyh - a.ycent, zzh - a.zcent, f);  // Bx(xx, yyh, zzh)
      ebf[3 * g.ncell + o] += a.ee0 * f[3];
      lp_fields(a, xxh - a.xf0, yy - a.ycent, zzh - a.zcent, f);  // By(xxh, yy, zzh)
      ebf[4 * g.ncell + o] += a.ee0 * f[4];
      lp_fields(a, xxh - a.xf0, yyh - a.ycent, zz - a.zcent, f);  // Bz(xxh, yyh, zz)
      ebf[5 * g.ncell + o] += a.ee0 * f[5];
    } else {
      lp_fields(a, xxh - a.xf0, yy - a.ycent, 0.0, f);  // Ex(xxh, yy)
      ebf[o] += a.ee0 * f[0];
      lp_fields(a, xx - a.xf0, yyh - a.ycent, 0.0, f);  // Ey(xx, yyh)
      ebf[g.ncell + o] += a.ee0 * f[1];
      lp_fields(a, xxh - a.xf0, yyh - a.ycent, 0.0, f);  // Bz(xxh, yyh)
      ebf[2 * g.ncell + o] += a.ee0 * f[5];
    }
  }
}
void laser64(const LaserArgs& a, double* ebf, const Geo& g, cudaStream_t st, int sms) {
  long long cells = (long long)(g.ix2 - g.ix1 + 1) * (g.jy2 - g.jy1 + 1) * (g.kz2 - g.kz1 + 1);
  k_laser64<<<grid_for(cells, 256, sms, 16), 256, 0, st>>>(a, ebf, g);
}

// ============================================================================
// Diagnostics (Envar / energy_momenta, diag_part_and_fields.f90:172-220,
// 485-719), FP64 block reductions.
// ============================================================================
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ void atomic_max_nonneg(double* a, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(a), (unsigned long long)__double_as_longlong(v));
}

// One warp per interior x-row (j, k), the lanes along x: coalesced reads and
// no per-cell index division.
// NFC field components (3 in 2D, 6 in 3D) as a template argument, so the
// component loops unroll and the per-lane sums stay in registers.
template <typename T, int NFC>
__global__ void k_field_diag(const T* ebf, Geo g, double dvol, double* out_e, double* out_max) {
  constexpr int nf = NFC;
  const int nx = g.ix2 - g.ix1 + 1, ny = g.jy2 - g.jy1 + 1, nz = g.kz2 - g.kz1 + 1;
  const long long nrows = (long long)ny * nz;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  double mx = 0.0;
  const int ne = (nf == 6) ? 3 : 2;
  const int lane = threadIdx.x & 31;
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = warp; r < nrows; r += nwarps) {
    const int j = g.jy1 + (int)(r % ny), k = g.kz1 + (int)(r / ny);
    const long long o0 = goff(g, g.ix1, j, k);
    if (sizeof(T) == 8) {
#pragma unroll 4
      for (int i = lane; i < nx; i += 32) {
        const long long o = o0 + i;
#pragma unroll
        for (int c = 0; c < nf; ++c) {
          double v = (double)ebf[g.ncell * c + o];
          acc[c] += v * v;
          if (c < ne) mx = fmax(mx, fabs(v));
        }
      }
    } else {
      // split form: a lane's squares of one row summed in FP32 (the field
      // words are FP32), the row partial added in FP64
      float rs[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      float rm = 0.f;
#pragma unroll 4
      for (int i = lane; i < nx; i += 32) {
        const long long o = o0 + i;
#pragma unroll
        for (int c = 0; c < nf; ++c) {
          const float v = (float)ebf[g.ncell * c + o];
          rs[c] = fmaf(v, v, rs[c]);
          if (c < ne) rm = fmaxf(rm, fabsf(v));
        }
      }
#pragma unroll
      for (int c = 0; c < nf; ++c) acc[c] += (double)rs[c];
      mx = fmax(mx, (double)rm);
    }
  }
#pragma unroll
  for (int c = 0; c < nf; ++c) {
    double v = warp_sum(acc[c]);
    if ((threadIdx.x & 31) == 0) atomicAdd(&out_e[c], v * dvol);
  }
  double m = warp_max(mx);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out_max, m);
}
void field_diag64(const double* ebf, const Geo& g, double dvol, double* out_e, double* out_max, cudaStream_t st, int sms) {
  long long cells = (long long)(g.ix2 - g.ix1 + 1) * (g.jy2 - g.jy1 + 1) * (g.kz2 - g.kz1 + 1);
  if (g.nf == 6)
    k_field_diag<double, 6><<<grid_for(cells / 8, 256, sms, 16), 256, 0, st>>>(ebf, g, dvol, out_e, out_max);
  else
    k_field_diag<double, 3><<<grid_for(cells / 8, 256, sms, 16), 256, 0, st>>>(ebf, g, dvol, out_e, out_max);
}
void field_diag32(const float* ebf, const Geo& g, double dvol, double* out_e, double* out_max, cudaStream_t st, int sms) {
  long long cells = (long long)(g.ix2 - g.ix1 + 1) * (g.jy2 - g.jy1 + 1) * (g.kz2 - g.kz1 + 1);
  if (g.nf == 6)
    k_field_diag<float, 6><<<grid_for(cells / 8, 256, sms, 16), 256, 0, st>>>(ebf, g, dvol, out_e, out_max);
  else
    k_field_diag<float, 3><<<grid_for(cells / 8, 256, sms, 16), 256, 0, st>>>(ebf, g, dvol, out_e, out_max);
}

// out[0] = sum w (gamma-1), out[1] = sum charge*w, out[2..4] = sum w p over
// the records q < n, or over records perm[q], q < n, when perm is given (the
// alive records of a binned species, removed ones still stored)
__global__ void k_part_diag64(const double* part, long long ld, long long n, int nd, const int* perm, double* out) {
  double a[5] = {0, 0, 0, 0, 0};
  for (long long qq = blockIdx.x * (long long)blockDim.x + threadIdx.x; qq < n; qq += (long long)gridDim.x * blockDim.x) {
    const long long q = perm ? (long long)perm[qq] : qq;
    double p2 = 0.0, pv[3] = {0, 0, 0};
    for (int c = 0; c < nd; ++c) {
      pv[c] = part[(long long)(nd + c) * ld + q];
      p2 += pv[c] * pv[c];
    }
    uint64_t sl = dbits(part[(long long)(2 * nd) * ld + q]);
    double w = (double)slot_wgh(sl);
    double gm = sqrt(1.0 + p2);
    a[0] += w * (gm - 1.0);
    a[1] += (double)slot_charge(sl) * w;
    for (int c = 0; c < 3; ++c) a[2 + c] += w * pv[c];
  }
  for (int c = 0; c < 5; ++c) {
    double v = warp_sum(a[c]);
    if ((threadIdx.x & 31) == 0) atomicAdd(&out[c], v);
  }
}
void part_diag64(const double* part, long long ld, long long n, int nd, const int* perm, double* out, cudaStream_t st,
                 int sms) {
  if (n <= 0) return;
  k_part_diag64<<<grid_for(n, 256, sms, 16), 256, 0, st>>>(part, ld, n, nd, perm, out);
}
// Split form: each record's terms in FP32 (its momenta are FP32; gamma - 1 as
// p^2 / (1 + gamma), free of cancellation), summed in FP64; the charge term
// is exact.
__device__ __forceinline__ void diag_terms32(float px, float py, float pz, uint64_t sl, double a[5]) {
  const float p2 = fmaf(px, px, fmaf(py, py, pz * pz));
  const float g1 = p2 / (1.f + sqrtf(1.f + p2));
  const float w = slot_wgh(sl);
  a[0] += (double)(w * g1);
  a[1] += (double)slot_charge(sl) * (double)w;
  a[2] += (double)(w * px);
  a[3] += (double)(w * py);
  a[4] += (double)(w * pz);
}
// Records 0..n-1 in memory order, four at a time with 16-byte loads (the
// arrays are allocation-aligned), the last n % 4 one by one; with a key
// array, the records whose binning key is `dead` (removed at a box edge,
// still stored until the next compaction) are left out.
__global__ void k_part_diag32(Part32View p, long long n, int nd, const int* key, int dead, double* out) {
  double a[5] = {0, 0, 0, 0, 0};
  const long long n4 = n >> 2;
  const float4* px4 = reinterpret_cast<const float4*>(p.px);
  const float4* py4 = reinterpret_cast<const float4*>(p.py);
  const float4* pz4 = reinterpret_cast<const float4*>(p.pz);
  const ulonglong2* sl2 = reinterpret_cast<const ulonglong2*>(p.slot);
  const int4* key4 = reinterpret_cast<const int4*>(key);
  for (long long g4 = blockIdx.x * (long long)blockDim.x + threadIdx.x; g4 < n4; g4 += (long long)gridDim.x * blockDim.x) {
    const float4 x = px4[g4], y = py4[g4];
    const float4 z = (nd == 3) ? pz4[g4] : make_float4(0.f, 0.f, 0.f, 0.f);
    const ulonglong2 s0 = sl2[2 * g4], s1 = sl2[2 * g4 + 1];
    const int4 kk = key ? key4[g4] : make_int4(0, 0, 0, 0);
    if (!key || kk.x != dead) diag_terms32(x.x, y.x, z.x, s0.x, a);
    if (!key || kk.y != dead) diag_terms32(x.y, y.y, z.y, s0.y, a);
    if (!key || kk.z != dead) diag_terms32(x.z, y.z, z.z, s1.x, a);
    if (!key || kk.w != dead) diag_terms32(x.w, y.w, z.w, s1.y, a);
  }
  const long long q = 4 * n4 + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q < n && (!key || key[q] != dead)) diag_terms32(p.px[q], p.py[q], (nd == 3) ? p.pz[q] : 0.f, p.slot[q], a);
  for (int c = 0; c < 5; ++c) {
    double v = warp_sum(a[c]);
    if ((threadIdx.x & 31) == 0) atomicAdd(&out[c], v);
  }
}
void part_diag32(const Part32View& p, long long n, int nd, const int* key, int dead, double* out, cudaStream_t st,
                 int sms) {
  if (n <= 0) return;
  k_part_diag32<<<grid_for((n + 3) / 4, 256, sms, 16), 256, 0, st>>>(p, n, nd, key, dead, out);
}

// max of a non-negative FP64 array (ion |E|^2), for the lp_max refresh.
__global__ void k_max_nonneg(const double* a, long long n, double* out) {
  double m = 0.0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    m = fmax(m, a[q]);
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, m);
}
void max_nonneg(const double* a, long long n, double* out, cudaStream_t st, int sms) {
  cudaMemsetAsync(out, 0, sizeof(double), st);
  if (n > 0) k_max_nonneg<<<grid_for(n, 256, sms, 8), 256, 0, st>>>(a, n, out);
}

}  // namespace agpu
