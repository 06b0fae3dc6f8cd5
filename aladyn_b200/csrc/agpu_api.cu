// agpu_api.cu — the C-ABI of include/aladyn_gpu.h: handle lifetime, state
// transfer, the step driver (lpf2_evolve + lp_run), window, ionization and
// diagnostics.  Compiled with -fmad=false (host-side FP64 bookkeeping of the
// window origin follows the reference's arithmetic).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/aladyn_gpu.h"
#include "agpu_beam.h"
#include "agpu_bin.cuh"
#include "agpu_env.h"
#include "agpu_ionz.h"
#include "agpu_kernels.h"
#include "agpu_multi.h"
#include "agpu_tile.h"
#include "agpu_util.h"

using namespace agpu;

namespace {

struct Species32 {
  int* cell = nullptr;
  float *ox = nullptr, *oy = nullptr, *oz = nullptr;
  float *px = nullptr, *py = nullptr, *pz = nullptr;
  uint64_t* slot = nullptr;
  Part32View view() const { return Part32View{cell, ox, oy, oz, px, py, pz, slot}; }
};

enum Phase { PH_PUSH = 0, PH_YEE, PH_SORT, PH_WINDOW, PH_IONIZE, PH_OTHER, PH_N };

struct Counters {
  unsigned long long removed;
  unsigned int err;
  int alive;  // particles in tiles after the last binning
  double fmax;
  unsigned long long pushed;  // deferred mode: particles pushed since the last refresh
  int alive4[4];              // deferred mode: alive count per species at the refresh
};

}  // namespace

struct agpu_handle {
  agpu_params p;
  Geo g;
  int ndv = 0;
  int device = 0;
  int sms = 148;
  cudaStream_t st = nullptr;
  bool fp32 = false;
  // FP64 form
  double* ebf = nullptr;
  double* ebf_alt = nullptr;  // the fused Yee step's output, swapped with ebf
  float* ebf32_alt = nullptr;
  bool fused_yee = false;  // measured: the separate sweeps are faster in 3D
  double* jc = nullptr;
  double* part[4] = {nullptr, nullptr, nullptr, nullptr};
  double* tmp = nullptr;  // compaction target, cap_max * ndv
  // FP32 split form
  float* ebf32 = nullptr;
  float* jhi = nullptr;
  float* jlo = nullptr;
  Species32 sp[4];
  Species32 sptmp;
  long long np[4] = {0, 0, 0, 0};
  long long cap[4] = {0, 0, 0, 0};
  long long capmax = 0;
  // shared scratch
  int* flag = nullptr;       // per particle (max capacity)
  double* ef2 = nullptr;     // per ion |E|^2
  Counters* d_cnt = nullptr;
  Counters* h_cnt = nullptr;
  Scratch scr{};
  double* d_diag = nullptr;  // diagnostics accumulators
  double* d_envar = nullptr;  // Envar reductions (16 + AGPU_NE doubles)
  int* tile_work = nullptr;         // (tile, chunk) pairs of dense tiles, split form
  unsigned int* tile_work_n = nullptr;
  int tile_work_cap = 0;
  // envelope model (agpu_env_enable): env(n1p,n2p,n3p,4), the step's source
  // scratch (ndim+1 components) and the density before its copy
  double* env = nullptr;
  double* env_av = nullptr;
  double* env_den = nullptr;
  agpu_env_params ep{};
  long long env_steps = 0;  // env_run calls so far (the record sort period)
  // stretched y and z (agpu_set_stretch): the particle maps and the metric
  // factors loc_yg(:, 3), loc_yg(:, 4), loc_zg(:, 3), loc_zg(:, 4) on the device
  bool str = false;
  StrAxis sy{}, sz{};
  double* d_metric = nullptr;  // my3, my4 (ny+2 each), then mz3, mz4 (nz+2 each)
  std::vector<double> h_metric;  // the same on the host
  double by3 = 1.0, ty4 = 1.0, bz3 = 1.0, tz4 = 1.0;
  // a slab of a y decomposition (agpu_set_subdomain): shared sides and the
  // host's exchange hook
  bool dd = false;
  int dd_lo = 0, dd_hi = 0, dd_zlo = 0, dd_zhi = 0;
  agpu_halo_fn halo_fn = nullptr;
  void* halo_user = nullptr;
  // comoving frame (w_speed < 0): the field advection's scratch
  double* xadv_tmp = nullptr;
  double* xadv_coef = nullptr;  // bet[0..nx+1], then w1[0..nx+1]
  XAdv xadv{};
  // window state (lp_window_xshift saved variables)
  double xlapse = 0.0;
  int wi1 = 0;
  // plasma sources
  agpu_plasma src[4];
  bool has_src[4] = {false, false, false, false};
  long long nptx[4] = {0, 0, 0, 0}, sptx_max[4] = {0, 0, 0, 0};
  int npty[4] = {0, 0, 0, 0}, nptz[4] = {0, 0, 0, 0};
  // ionization
  double* d_wtab[4] = {nullptr, nullptr, nullptr, nullptr};
  int zmax[4] = {0, 0, 0, 0};
  double de_inv[4] = {0, 0, 0, 0};
  double lp_max[4] = {0, 0, 0, 0};
  int at_num[4] = {0, 0, 0, 0}, ion_min[4] = {0, 0, 0, 0}, model[4] = {0, 0, 0, 0};
  bool auto_table[4] = {false, false, false, false};
  int nsp_ionz = 1;
  // spatial tiles of the running species: key / perm per particle,
  // histogram (nkeys+1), key starts (nkeys+2), scatter cursors (nkeys+1) and
  // the scan's block sums
  TileGeo tg{};
  int* key[4] = {nullptr, nullptr, nullptr, nullptr};
  int* perm[4] = {nullptr, nullptr, nullptr, nullptr};
  int* hist[4] = {nullptr, nullptr, nullptr, nullptr};
  int* tstart[4] = {nullptr, nullptr, nullptr, nullptr};
  int* cursor = nullptr;
  int* scan_tmp = nullptr;
  // staging of window-injection records for the split form (kept between
  // calls: a per-call device allocation of hundreds of MB can take longer
  // than the step)
  double* inj_stage = nullptr;
  long long inj_stage_recs = 0;
  bool binned[4] = {false, false, false, false};
  long long nalive[4] = {0, 0, 0, 0};  // np minus removed records still stored
  // deferred counts: tiled steps leave the alive counts and the error word
  // on the device; refresh_counts reads them at the next synchronisation
  bool defer = false;
  bool stale[4] = {false, false, false, false};
  // step graph (deferred mode): the launches of a step between window
  // shifts, captured once and replayed while the signature holds
  bool use_graph = false;
  cudaGraphExec_t gexec = nullptr;
  unsigned char gsig[160] = {};
  long long g_launches = 0, g_push = 0, g_yee = 0, g_cells = 0;
  // flags
  bool fields_set = false;
  bool deterministic = false;
  bool profiling = false;
  int sort_interval = 0;
  uint32_t error_bits = 0;
  cudaEvent_t ev[2 * PH_N] = {};
  agpu_timers timers{};
};

namespace {

#define CK(call)                                                  \
  do {                                                            \
    cudaError_t e_ = (call);                                      \
    if (e_ != cudaSuccess) {                                      \
      std::fprintf(stderr, "aladyn_gpu: %s -> %s\n", #call, cudaGetErrorString(e_)); \
      return AGPU_E_CUDA;                                         \
    }                                                             \
  } while (0)

int dmalloc(void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return AGPU_E_NOMEM;
  }
  return 0;
}

// Comoving frame (w_speed < 0: vbeam = -w_speed, set_init_param.f90:239-245):
// the x displacement dt * vbeam subtracted after every push, 0 otherwise.
double comoving_vdt(const agpu_params& p) { return p.w_speed < 0.0 ? p.dt * (-p.w_speed) : 0.0; }

YeeC yee_coef(const agpu_params& p) {
  YeeC c;
  c.vbeam = p.w_speed < 0.0 ? -p.w_speed : 0.0;
  c.dx_inv = p.dx_inv;
  c.dy_inv = p.dy_inv;
  c.dz_inv = p.dz_inv;
  c.dt = p.dt;
  c.se1 = p.se_coeff[0];
  c.se2 = p.se_coeff[1];
  c.ompe = p.ompe;
  // curr_mpi_collect scales the currents by djc only when iform < 2
  c.djc1 = p.iform < 2 ? p.djc[0] : 1.0;
  c.djc2 = p.iform < 2 ? p.djc[1] : 1.0;
  c.djc3 = p.iform < 2 ? p.djc[2] : 1.0;
  return c;
}

void ph_begin(agpu_handle* h, int ph) {
  if (h->profiling) cudaEventRecord(h->ev[2 * ph], h->st);
}
void ph_end(agpu_handle* h, int ph) {
  if (!h->profiling) return;
  cudaEventRecord(h->ev[2 * ph + 1], h->st);
  cudaEventSynchronize(h->ev[2 * ph + 1]);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev[2 * ph], h->ev[2 * ph + 1]);
  double* slots[PH_N] = {&h->timers.ms_push_deposit, &h->timers.ms_yee, &h->timers.ms_sort,
                         &h->timers.ms_window, &h->timers.ms_ionize, &h->timers.ms_other};
  *slots[ph] += ms;
}

int free_all(agpu_handle* h) {
  cudaFree(h->ebf);
  cudaFree(h->jc);
  for (int i = 0; i < 4; ++i) cudaFree(h->part[i]);
  cudaFree(h->tmp);
  cudaFree(h->ebf32);
  cudaFree(h->ebf_alt);
  cudaFree(h->ebf32_alt);
  cudaFree(h->jhi);
  cudaFree(h->jlo);
  auto freesp = [](Species32& s) {
    cudaFree(s.cell);
    cudaFree(s.ox);
    cudaFree(s.oy);
    cudaFree(s.oz);
    cudaFree(s.px);
    cudaFree(s.py);
    cudaFree(s.pz);
    cudaFree(s.slot);
    s = Species32();
  };
  for (int i = 0; i < 4; ++i) freesp(h->sp[i]);
  freesp(h->sptmp);
  cudaFree(h->flag);
  cudaFree(h->ef2);
  cudaFree(h->d_cnt);
  cudaFreeHost(h->h_cnt);
  cudaFree(h->scr.blockcnt);
  cudaFree(h->scr.total);
  cudaFreeHost(h->scr.h_total);
  cudaFree(h->d_diag);
  cudaFree(h->d_envar);
  cudaFree(h->tile_work);
  cudaFree(h->tile_work_n);
  for (int i = 0; i < 4; ++i) cudaFree(h->d_wtab[i]);
  for (int i = 0; i < 4; ++i) {
    cudaFree(h->key[i]);
    cudaFree(h->perm[i]);
    cudaFree(h->hist[i]);
    cudaFree(h->tstart[i]);
  }
  cudaFree(h->cursor);
  cudaFree(h->scan_tmp);
  cudaFree(h->inj_stage);
  cudaFree(h->env);
  cudaFree(h->env_av);
  cudaFree(h->env_den);
  cudaFree(h->xadv_tmp);
  cudaFree(h->d_metric);
  cudaFree(h->xadv_coef);
  for (int i = 0; i < 2 * PH_N; ++i)
    if (h->ev[i]) cudaEventDestroy(h->ev[i]);
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->st) cudaStreamDestroy(h->st);
  return 0;
}

int alloc_species32(Species32& s, long long cap, int ndim) {
  int rc = 0;
  rc |= dmalloc((void**)&s.cell, sizeof(int) * cap);
  rc |= dmalloc((void**)&s.ox, sizeof(float) * cap);
  rc |= dmalloc((void**)&s.oy, sizeof(float) * cap);
  rc |= dmalloc((void**)&s.px, sizeof(float) * cap);
  rc |= dmalloc((void**)&s.py, sizeof(float) * cap);
  if (ndim == 3) {
    rc |= dmalloc((void**)&s.oz, sizeof(float) * cap);
    rc |= dmalloc((void**)&s.pz, sizeof(float) * cap);
  }
  rc |= dmalloc((void**)&s.slot, sizeof(uint64_t) * cap);
  return rc ? AGPU_E_NOMEM : 0;
}

// Particle-count sync point: removed count and the sticky error word.
int read_counters(agpu_handle* h) {
  CK(cudaMemcpyAsync(h->h_cnt, h->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->error_bits |= h->h_cnt->err;
  return 0;
}

// Deferred mode: bring the alive counts of the species binned since the last
// refresh, the pushed-particle count and the error word to the host, then
// restart the device accumulators.
int refresh_counts(agpu_handle* h) {
  bool any = false;
  for (int ic = 0; ic < 4; ++ic) any = any || h->stale[ic];
  if (!any) return 0;
  for (int ic = 0; ic < 4; ++ic)
    if (h->stale[ic])
      CK(cudaMemcpyAsync(&h->d_cnt->alive4[ic], h->tstart[ic] + h->tg.nkeys, sizeof(int), cudaMemcpyDeviceToDevice,
                         h->st));
  CK(cudaMemcpyAsync(h->h_cnt, h->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->error_bits |= h->h_cnt->err;
  h->timers.pushes += (long long)h->h_cnt->pushed;
  for (int ic = 0; ic < 4; ++ic)
    if (h->stale[ic]) {
      h->nalive[ic] = h->h_cnt->alive4[ic];
      h->stale[ic] = false;
    }
  CK(cudaMemsetAsync(h->d_cnt, 0, sizeof(Counters), h->st));
  return 0;
}

long long lattice_columns_end(const agpu_handle* h, int ic, long long i1, double xmx, bool reference_quirk) {
  // particles_inject (src/dynamics/window.f90:124-136): first column with
  // xpt > xmx ends the block; when that column is sptx_max itself, the
  // reference keeps it.
  const agpu_plasma& s = h->src[ic];
  double dxl = h->p.dx / (double)s.npx;
  long long smax = h->sptx_max[ic];
  long long ix;
  if (i1 > smax) return i1 - 1;
  for (ix = i1; ix <= smax; ++ix)
    if (s.x_start + ((double)ix - 0.5) * dxl > xmx) break;
  long long i2 = ix - 1;
  if (reference_quirk && ix == smax) i2 = ix;
  return i2;
}

int drop_removed(agpu_handle* h, int ic);
int compact_species(agpu_handle* h, int ic, bool window);

int add_lattice_columns(agpu_handle* h, int ic, long long i1, long long i2) {
  // lattice rows j1r .. j1r+nrow-1: all of them, or for a y slab those whose
  // jittered y, y_min + (j - 1/2 + u) dyl with |u| <= 1/2, can fall inside
  // (gymin, gymax], plus one row of margin on each side
  int j1r = 1, nrow = h->npty[ic];
  if (h->dd) {
    const double dyl = h->p.dy / (double)h->src[ic].npy;
    const double y_min = h->src[ic].y_min;
    long long lo = (long long)std::floor((h->p.gymin - y_min) / dyl);
    long long hi = (long long)std::ceil((h->p.gymax - y_min) / dyl) + 1;
    if (lo < 1) lo = 1;
    if (hi > h->npty[ic]) hi = h->npty[ic];
    j1r = (int)lo;
    nrow = hi >= lo ? (int)(hi - lo + 1) : 0;
  }
  long long n = (i2 - i1 + 1) * (long long)nrow * h->nptz[ic];
  if (n <= 0) return 0;
  if (int rc = drop_removed(h, ic)) return rc;
  if (h->np[ic] + n > h->cap[ic]) {
    h->error_bits |= AGPU_EBIT_CAPACITY;
    return AGPU_E_CAPACITY;
  }
  const agpu_plasma& s = h->src[ic];
  LatticeArgs a;
  a.ndim = h->p.ndim;
  a.ic = ic;
  a.npty = nrow;
  a.j0 = j1r;
  a.nptz = h->nptz[ic];
  a.i1 = i1;
  a.i2 = i2;
  a.charge = s.charge;
  a.part_ind = s.part_ind;
  a.wgh = s.wgh;
  a.x_start = s.x_start;
  a.y_min = s.y_min;
  a.z_min = s.z_min;
  a.dxl = h->p.dx / (double)s.npx;
  a.dyl = h->p.dy / (double)s.npy;
  a.dzl = h->p.dz / (double)s.npz;
  a.jitter = s.jitter;
  a.seed = s.seed;
  if (h->fp32)
    lattice32(a, h->sp[ic].view(), h->np[ic], h->g, h->p.xmn, h->p.ymn, h->p.zmn, h->p.dx_inv, h->p.dy_inv, h->p.dz_inv, h->st,
              h->sms);
  else
    lattice64(a, h->part[ic], h->cap[ic], h->np[ic], h->st, h->sms);
  CK(cudaGetLastError());
  h->timers.launches_total += 1;
  if (h->dd) {
    // a slab keeps the lattice particles of its own rows: the columns span
    // the whole source, as in one box, and the rest is dropped here
    h->np[ic] += n;
    h->nalive[ic] = h->np[ic];
    h->binned[ic] = false;
    return compact_species(h, ic, false);
  }
  h->np[ic] += n;
  h->nalive[ic] += n;
  h->binned[ic] = false;
  return 0;
}

// Stable removal of the particles of species ic outside the box; x only when
// window is set (cell_part_dist(.true.)), else x, y and z.
int drop_removed(agpu_handle* h, int ic);

int compact_species(agpu_handle* h, int ic, bool window) {
  if (int rc = refresh_counts(h)) return rc;
  if (h->np[ic] <= 0) return 0;
  long long kept;
  if (window && h->binned[ic]) {
    // the window compaction copies the alive records along the tile
    // permutation: the drop of x <= xmin and a physical sort by tile at once
    if (h->fp32) {
      kept = perm_compact32(h->perm[ic], h->nalive[ic], h->sp[ic].view(), h->sptmp.view(), true, h->g.n1p, h->p.nx, h->scr,
                            h->st);
      std::swap(h->sp[ic], h->sptmp);
    } else {
      kept = perm_compact64(h->perm[ic], h->nalive[ic], h->part[ic], h->tmp, h->cap[ic], h->ndv, true, h->p.gxmin,
                            h->p.gxmax, h->scr, h->st);
      std::swap(h->part[ic], h->tmp);
    }
    CK(cudaGetLastError());
    h->timers.launches_total += 3;
    h->np[ic] = kept;
    h->nalive[ic] = kept;
    h->binned[ic] = false;
    return 0;
  }
  if (int rc = drop_removed(h, ic)) return rc;
  if (h->fp32) {
    int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz;
    kept = compact32(h->sp[ic].view(), h->sptmp.view(), h->np[ic], h->g.n1p, h->g.n2p, nx, ny, nz, window ? 0 : 1,
                     (!window && h->p.ndim == 3) ? 1 : 0, h->scr, h->st);
    std::swap(h->sp[ic], h->sptmp);
  } else {
    BoxBounds b{h->p.gxmin, h->p.gxmax, h->p.gymin, h->p.gymax, h->p.gzmin, h->p.gzmax, window ? 0 : 1,
                (!window && h->p.ndim == 3) ? 1 : 0};
    kept = compact64(h->part[ic], h->tmp, h->cap[ic], h->np[ic], h->ndv, b, h->scr, h->st);
    // tmp has leading dimension cap[ic]; capacities are equal-size slots
    std::swap(h->part[ic], h->tmp);
  }
  CK(cudaGetLastError());
  h->timers.launches_total += 3;  // count, scan, scatter
  h->np[ic] = kept;
  h->nalive[ic] = kept;
  h->binned[ic] = false;
  return 0;
}

// ---- binning of the running species ---------------------------------------
// The FP64 tile kernel has the reference's quadratic shapes only; the cubic
// FP64 form runs the per-particle kernels.
bool tiled(const agpu_handle* h, int ic) {
  return !h->deterministic && !h->dd && !h->str && ic < h->p.nsp_run && h->key[ic] != nullptr &&
         (h->fp32 || (h->p.shape == AGPU_SHAPE_QUADRATIC && h->p.iform < 2));
}

// Keys from the current positions, histogram, scan and permutation.
int rebin(agpu_handle* h, int ic) {
  const TileGeo& t = h->tg;
  CK(cudaMemsetAsync(h->hist[ic], 0, sizeof(int) * (t.nkeys + 1), h->st));
  if (h->fp32)
    bin_keys_split(h->sp[ic].cell, h->sp[ic].ox, h->sp[ic].oy, h->sp[ic].oz, h->np[ic], h->g, t, h->key[ic], h->hist[ic],
                   &h->d_cnt->err, h->st, h->sms);
  else
    bin_keys_abs(h->part[ic], h->part[ic] + h->cap[ic], h->part[ic] + 2 * h->cap[ic], h->np[ic], h->g, t, h->p.xmn, h->p.ymn,
                 h->p.zmn, h->p.dx_inv, h->p.dy_inv, h->p.dz_inv, h->key[ic], h->hist[ic], &h->d_cnt->err, h->st, h->sms);
  const int nl = bin_finish(h->key[ic], h->np[ic], t, h->hist[ic], h->tstart[ic], h->cursor, h->perm[ic], h->scan_tmp,
                            h->st, h->sms);
  CK(cudaGetLastError());
  h->timers.launches_total += (h->np[ic] > 0 ? 1 : 0) + nl;  // keys, scan, scatter
  h->binned[ic] = true;
  if (h->defer) {
    h->stale[ic] = true;
    return 0;
  }
  CK(cudaMemcpyAsync(&h->d_cnt->alive, h->tstart[ic] + t.nkeys, sizeof(int), cudaMemcpyDeviceToDevice, h->st));
  if (int rc = read_counters(h)) return rc;
  h->nalive[ic] = h->h_cnt->alive;
  return 0;
}

// Drop the removed records (key == nkeys) keeping the memory order, so the
// stored arrays hold exactly the alive particles; the binning is then stale.
int drop_removed(agpu_handle* h, int ic) {
  if (int rc = refresh_counts(h)) return rc;
  if (!h->binned[ic] || h->nalive[ic] == h->np[ic]) return 0;
  long long kept;
  if (h->fp32) {
    kept = compact_flag32(h->key[ic], h->tg.nkeys, h->sp[ic].view(), h->sptmp.view(), h->np[ic], h->scr, h->st);
    std::swap(h->sp[ic], h->sptmp);
  } else {
    kept = compact_flag64(h->key[ic], h->tg.nkeys, h->part[ic], h->tmp, h->cap[ic], h->np[ic], h->ndv, h->scr, h->st);
    std::swap(h->part[ic], h->tmp);
  }
  CK(cudaGetLastError());
  h->timers.launches_total += 3;
  h->np[ic] = kept;
  h->nalive[ic] = kept;
  h->binned[ic] = false;
  return 0;
}

// agpu_set_sort_interval: every sort_interval steps (not on window steps,
// whose compaction reorders the records anyway) the records of a tiled
// species are moved along the step's tile permutation, so that memory order
// follows the tiles again where the particles have drifted (runs without a
// moving window never compact otherwise).  Removed records are dropped.
bool sort_step(const agpu_handle* h, int iter) {
  const agpu_params& p = h->p;
  if (h->sort_interval <= 0 || iter <= 0 || iter % h->sort_interval != 0) return false;
  return !(p.w_speed > 0.0 && p.w_sh > 0 && iter % p.w_sh == 0);
}

int reorder_records(agpu_handle* h, int ic) {
  if (!h->binned[ic]) return 0;
  if (int rc = refresh_counts(h)) return rc;
  long long kept;
  if (h->fp32) {
    kept = perm_compact32(h->perm[ic], h->nalive[ic], h->sp[ic].view(), h->sptmp.view(), false, h->g.n1p, h->p.nx, h->scr,
                          h->st);
    std::swap(h->sp[ic], h->sptmp);
  } else {
    kept = perm_compact64(h->perm[ic], h->nalive[ic], h->part[ic], h->tmp, h->cap[ic], h->ndv, false, h->p.gxmin,
                          h->p.gxmax, h->scr, h->st);
    std::swap(h->part[ic], h->tmp);
  }
  CK(cudaGetLastError());
  h->timers.launches_total += 3;
  h->np[ic] = kept;
  h->nalive[ic] = kept;
  h->binned[ic] = false;
  return 0;
}

// Tiled gather + push + deposit of species ic, then the next binning from
// the keys the kernel wrote.  Removed particles stay stored (key nkeys)
// until the next compaction.
int tiled_push(agpu_handle* h, int ic, int initial_time, agpu_step_out* out) {
  const agpu_params& p = h->p;
  if (!h->binned[ic]) {
    ph_begin(h, PH_SORT);
    int rc = rebin(h, ic);
    ph_end(h, PH_SORT);
    if (rc) return rc;
  }
  const long long alive0 = h->nalive[ic];
  hist_reset(h->hist[ic], h->tstart[ic], h->tg, h->np[ic], false, h->defer ? &h->d_cnt->pushed : nullptr, h->st);
  ph_begin(h, PH_PUSH);
  if (h->fp32) {
    TileArgs32 a;
    a.g = h->g;
    a.t = h->tg;
    a.ebf = h->ebf32;
    a.jhi = h->jhi;
    a.jlo = h->jlo;
    const Species32& s = h->sp[ic];
    a.p = Part32{s.cell, s.ox, s.oy, s.oz, s.px, s.py, s.pz, s.slot};
    a.perm = h->perm[ic];
    a.tstart = h->tstart[ic];
    a.key = h->key[ic];
    a.hist = h->hist[ic];
    a.dth = (float)(0.5 * p.dt);
    a.lfact = (float)p.lorentz_fact[ic];
    a.dtx = (float)(p.dt * p.dx_inv);
    a.dty = (float)(p.dt * p.dy_inv);
    a.dtz = (float)(p.dt * p.dz_inv);
    a.initial = initial_time ? 1 : 0;
    a.err = &h->d_cnt->err;
    a.work = h->tile_work;
    a.work_n = h->tile_work_n;
    a.work_cap = h->tile_work_cap;
    if (p.shape == AGPU_SHAPE_CUBIC)
      tile_push32_cubic(a, h->st);
    else
      h->timers.launches_total += tile_push32(a, h->st, h->sms) - 1;
  } else {
    TileArgs64 a;
    a.g = h->g;
    a.t = h->tg;
    a.ebf = h->ebf;
    a.jc = h->jc;
    double* b = h->part[ic];
    long long cp = h->cap[ic];
    a.x = b;
    a.y = b + cp;
    if (p.ndim == 3) {
      a.z = b + 2 * cp;
      a.px = b + 3 * cp;
      a.py = b + 4 * cp;
      a.pz = b + 5 * cp;
      a.slot = b + 6 * cp;
    } else {
      a.z = nullptr;
      a.px = b + 2 * cp;
      a.py = b + 3 * cp;
      a.pz = nullptr;
      a.slot = b + 4 * cp;
    }
    a.perm = h->perm[ic];
    a.tstart = h->tstart[ic];
    a.key = h->key[ic];
    a.hist = h->hist[ic];
    a.xmn = p.xmn;
    a.ymn = p.ymn;
    a.zmn = p.zmn;
    a.dx_inv = p.dx_inv;
    a.dy_inv = p.dy_inv;
    a.dz_inv = p.dz_inv;
    a.dt = p.dt;
    a.dth = 0.5 * p.dt;
    a.lfact = p.lorentz_fact[ic];
    a.gxmin = p.gxmin;
    a.gxmax = p.gxmax;
    a.gymin = p.gymin;
    a.gymax = p.gymax;
    a.gzmin = p.gzmin;
    a.gzmax = p.gzmax;
    a.vdt = comoving_vdt(p);
    a.initial = initial_time ? 1 : 0;
    a.err = &h->d_cnt->err;
    tile_push64(a, h->st);
  }
  CK(cudaGetLastError());
  ph_end(h, PH_PUSH);
  h->timers.launches_push_deposit += 1;
  h->timers.launches_total += 2;  // histogram reset + tile kernel
  if (!h->defer) h->timers.pushes += alive0;
  ph_begin(h, PH_SORT);
  const int nl = bin_finish(h->key[ic], h->np[ic], h->tg, h->hist[ic], h->tstart[ic], h->cursor, h->perm[ic], h->scan_tmp,
                            h->st, h->sms);
  CK(cudaGetLastError());
  h->timers.launches_total += nl;  // scan + scatter
  if (h->defer) {
    h->stale[ic] = true;
    ph_end(h, PH_SORT);
    return 0;
  }
  CK(cudaMemcpyAsync(&h->d_cnt->alive, h->tstart[ic] + h->tg.nkeys, sizeof(int), cudaMemcpyDeviceToDevice, h->st));
  if (int rc = read_counters(h)) return rc;
  ph_end(h, PH_SORT);
  h->nalive[ic] = h->h_cnt->alive;
  out->removed[ic] += alive0 - h->nalive[ic];
  return 0;
}

// Window shift of split positions: node index i -= nshx; a particle pushed
// past node 1 is parked on node 1 with offset -0.5 (x_loc < 0), so the
// compaction that follows removes it instead of wrapping into another row.
__global__ void k_shift_cells(int* cell, float* ox, long long n, int nshx, int n1p) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int c = cell[q];
    int i = c % n1p + 1;
    int rest = c - (i - 1);
    i -= nshx;
    if (i < 1) {
      i = 1;
      ox[q] = -0.5f;
    }
    cell[q] = rest + (i - 1);
  }
}

// lp_window_xshift (src/dynamics/window.f90:276-347).
int window_xshift(agpu_handle* h, int witr, int init_iter, agpu_step_out* out) {
  agpu_params& p = h->p;
  if (init_iter == 0) {
    h->xlapse = 0.0;
    h->wi1 = 0;
    return 0;
  }
  double dt_step = p.dt;
  h->xlapse = h->xlapse + p.w_speed * dt_step * (double)witr;
  int wi2 = (int)std::lround(p.dx_inv * h->xlapse);
  int nshx = wi2 - h->wi1;
  h->wi1 = wi2;
  double sh = p.dx * (double)nshx;
  p.xmax = p.xmax + sh;
  p.gxmin = p.gxmin + sh;
  p.gxmax = p.gxmax + sh;
  p.xmn = p.xmn + sh;
  out->nshx = nshx;
  wi2 = h->g.ix2 - nshx;
  if (wi2 <= 0) return AGPU_E_WINDOW;
  if (nshx != 0) {
    if (h->fp32)
      xshift32(h->ebf32, h->g, h->g.nf, wi2, nshx, h->st, h->sms);
    else
      xshift64(h->ebf, h->g, h->g.nf, wi2, nshx, h->st, h->sms);
    // envelope: fields_left_xshift(env, i1, wi2, 1, nc_env = 4, nshx) (window.f90:326-330)
    if (h->env) xshift64(h->env, h->g, 4, wi2, nshx, h->st, h->sms);
    CK(cudaGetLastError());
    h->timers.launches_total += h->env ? 2 : 1;
  }
  for (int ic = 0; ic < p.nsp; ++ic) {
    if (h->np[ic] <= 0) continue;
    if (h->fp32 && nshx != 0) {
      k_shift_cells<<<grid_for(h->np[ic], 256, h->sms, 16), 256, 0, h->st>>>(h->sp[ic].cell, h->sp[ic].ox, h->np[ic], nshx,
                                                                               h->g.n1p);
      CK(cudaGetLastError());
      h->timers.launches_total += 1;
    }
    long long before = h->np[ic];
    int rc = compact_species(h, ic, true);
    if (rc) return rc;
    out->removed[ic] += before - h->np[ic];
  }
  for (int ic = 0; ic < p.nsp; ++ic) {
    if (!h->has_src[ic]) continue;
    const agpu_plasma& s = h->src[ic];
    if (s.x_start <= p.xmax && s.x_end > p.xmax) {
      long long i1 = 1 + h->nptx[ic];
      long long i2 = lattice_columns_end(h, ic, i1, p.xmax, true);
      h->nptx[ic] = i2;
      if (i2 > i1) {
        long long before = h->np[ic];
        int rc = add_lattice_columns(h, ic, i1, i2);
        if (rc) return rc;
        out->injected[ic] += h->np[ic] - before;
      }
    }
  }
  return 0;
}

// comoving_coordinate (src/dynamics/window.f90:227-275) for the comoving
// frame (vb = -w_speed): the box stays put, the plasma source's x range (and
// so every lattice column not yet injected) moves by -vb w_nst dt, the
// particles at or left of gxmin (or past gxmax) are dropped along x only and
// the columns that entered the box are injected.
int comoving_coordinate(agpu_handle* h, double vb, int w_nst, int loc_it, agpu_step_out* out) {
  agpu_params& p = h->p;
  if (loc_it == 0) return 0;
  const double dt_step = p.dt;
  double dt_tot = 0.0;
  for (int i = 1; i <= w_nst; ++i) dt_tot = dt_tot + dt_step;
  for (int ic = 0; ic < p.nsp; ++ic) {
    if (!h->has_src[ic]) continue;
    h->src[ic].x_start = h->src[ic].x_start - vb * dt_tot;
    h->src[ic].x_end = h->src[ic].x_end - vb * dt_tot;
  }
  for (int ic = 0; ic < p.nsp; ++ic) {
    if (h->np[ic] <= 0) continue;
    long long before = h->np[ic];
    int rc = compact_species(h, ic, true);
    if (rc) return rc;
    out->removed[ic] += before - h->np[ic];
  }
  for (int ic = 0; ic < p.nsp; ++ic) {
    if (!h->has_src[ic]) continue;
    const agpu_plasma& s = h->src[ic];
    if (s.x_start <= p.xmax && s.x_end > p.xmax) {
      long long i1 = 1 + h->nptx[ic];
      long long i2 = lattice_columns_end(h, ic, i1, p.xmax, true);
      h->nptx[ic] = i2;
      if (i2 > i1) {
        long long before = h->np[ic];
        int rc = add_lattice_columns(h, ic, i1, i2);
        if (rc) return rc;
        out->injected[ic] += h->np[ic] - before;
      }
    }
  }
  return 0;
}

// field_xadvect launches of one Yee step in the comoving frame: four
// boundary-ghost kernels, two per component in the explicit substeps, two
// tridiagonal sweeps
long long xadv_launches(const agpu_handle* h) { return h->xadv.tmp ? 6 + 2LL * h->g.nf : 0; }

// lp_run (src/dynamics/pic_evolve_in_time.f90 callers): the moving window
// (w_speed > 0) or the comoving frame's coordinate step (w_speed < 0), every
// w_sh steps inside [wi_time, wf_time)
int window_or_comoving(agpu_handle* h, int iter, double t, agpu_step_out* out) {
  const agpu_params& p = h->p;
  if (p.w_sh <= 0 || !(t >= p.wi_time && t < p.wf_time) || iter % p.w_sh != 0) return 0;
  int rc = 0;
  if (p.w_speed > 0.0) {
    ph_begin(h, PH_WINDOW);
    rc = window_xshift(h, p.w_sh, iter, out);
    ph_end(h, PH_WINDOW);
  } else if (p.w_speed < 0.0) {
    ph_begin(h, PH_WINDOW);
    rc = comoving_coordinate(h, -p.w_speed, p.w_sh, iter, out);
    ph_end(h, PH_WINDOW);
  }
  return rc;
}

int upload_table(agpu_handle* h, int ic, const double* tab, int zmax) {
  size_t bytes = sizeof(double) * (size_t)(kNge + 2) * (zmax + 1);
  if (!h->d_wtab[ic] || h->zmax[ic] != zmax) {
    cudaFree(h->d_wtab[ic]);
    h->d_wtab[ic] = nullptr;
    if (dmalloc((void**)&h->d_wtab[ic], bytes)) return AGPU_E_NOMEM;
  }
  h->zmax[ic] = zmax;
  CK(cudaMemcpy(h->d_wtab[ic], tab, bytes, cudaMemcpyHostToDevice));
  if (ic + 1 > h->nsp_ionz) h->nsp_ionz = ic + 1;
  return 0;
}

// Ionization of the FP64 form (pic_evolve_in_time.f90:44-68).
int ionize64(agpu_handle* h, int iter, agpu_step_out* out) {
  for (int ic = 1; ic < h->nsp_ionz && ic < h->p.nsp; ++ic) {
    long long np = h->np[ic];
    if (np <= 0 || !h->d_wtab[ic]) continue;
    IonArgs64 a;
    a.g = h->g;
    a.ebf = h->ebf;
    a.x = h->part[ic];
    a.y = h->part[ic] + h->cap[ic];
    a.z = h->part[ic] + 2 * h->cap[ic];
    a.slot = h->part[ic] + (size_t)(h->ndv - 1) * h->cap[ic];
    a.ef2 = h->ef2;
    a.flag = h->flag;
    a.np = np;
    a.xmn = h->p.xmn;
    a.ymn = h->p.ymn;
    a.zmn = h->p.zmn;
    a.dx_inv = h->p.dx_inv;
    a.dy_inv = h->p.dy_inv;
    a.dz_inv = h->p.dz_inv;
    a.wtab = h->d_wtab[ic];
    a.n_ge = kNge;
    a.zmax = h->zmax[ic];
    a.iter = iter;
    a.ic = ic;
    a.de_inv = h->de_inv[ic];
    a.seed = h->p.seed;
    a.err = &h->d_cnt->err;
    int grid = grid_for(np, 256, h->sms, 8);
    k64_ion_efield<<<grid, 256, 0, h->st>>>(a);
    CK(cudaGetLastError());
    if (iter % 100 == 0) {
      max_nonneg(h->ef2, np, &h->d_cnt->fmax, h->st, h->sms);
      CK(cudaGetLastError());
      if (int rc_ = read_counters(h)) return rc_;
      double m = std::sqrt(h->h_cnt->fmax);
      out->ion_field_max = m;
      if (h->auto_table[ic] && m > h->lp_max[ic]) {
        h->lp_max[ic] = 1.1 * m;
        std::vector<double> tab((size_t)(kNge + 2) * (h->at_num[ic] + 1));
        double dinv = 0.0;
        if (build_ionization_table(h->at_num[ic], h->ion_min[ic], h->model[ic], h->lp_max[ic], h->p.dt, tab.data(), &dinv))
          return AGPU_E_ARG;
        h->de_inv[ic] = dinv;
        a.de_inv = dinv;
        int rc = upload_table(h, ic, tab.data(), h->at_num[ic]);
        if (rc) return rc;
      }
    }
    k64_ionize<<<grid, 256, 0, h->st>>>(a);
    CK(cudaGetLastError());
    h->timers.launches_total += 2 + 3 + ((iter % 100 == 0) ? 1 : 0);  // efield, ionize, append, [max]
    if (int rc = drop_removed(h, 0)) return rc;
    long long ne0 = h->np[0];
    long long added = append_electrons64(h->flag, np, h->part[ic], h->cap[ic], h->part[0], h->cap[0], ne0, h->cap[0],
                                         h->p.ndim, h->p.n_mol_atoms[ic], &h->d_cnt->err, h->scr, h->st);
    CK(cudaGetLastError());
    if (ne0 + added > h->cap[0]) {
      h->error_bits |= AGPU_EBIT_CAPACITY;
      added = h->cap[0] - ne0;
    }
    h->np[0] = ne0 + added;
    h->nalive[0] = h->np[0];
    if (added > 0) h->binned[0] = false;
    out->new_electrons += added;
  }
  return 0;
}

// Ionization of the FP32 split form: the same steps as ionize64 with the
// ion |E|^2 gathered in FP32 from the split positions.
int ionize32(agpu_handle* h, int iter, agpu_step_out* out) {
  for (int ic = 1; ic < h->nsp_ionz && ic < h->p.nsp; ++ic) {
    long long np = h->np[ic];
    if (np <= 0 || !h->d_wtab[ic]) continue;
    IonArgs32 a;
    a.g = h->g;
    a.ebf = h->ebf32;
    a.cell = h->sp[ic].cell;
    a.ox = h->sp[ic].ox;
    a.oy = h->sp[ic].oy;
    a.oz = h->sp[ic].oz;
    a.slot = h->sp[ic].slot;
    a.ef2 = h->ef2;
    a.flag = h->flag;
    a.np = np;
    a.wtab = h->d_wtab[ic];
    a.n_ge = kNge;
    a.zmax = h->zmax[ic];
    a.iter = iter;
    a.ic = ic;
    a.de_inv = h->de_inv[ic];
    a.seed = h->p.seed;
    a.err = &h->d_cnt->err;
    int grid = grid_for(np, 256, h->sms, 8);
    k32_ion_efield<<<grid, 256, 0, h->st>>>(a);
    CK(cudaGetLastError());
    if (iter % 100 == 0) {
      max_nonneg(h->ef2, np, &h->d_cnt->fmax, h->st, h->sms);
      CK(cudaGetLastError());
      if (int rc = read_counters(h)) return rc;
      double m = std::sqrt(h->h_cnt->fmax);
      out->ion_field_max = m;
      if (h->auto_table[ic] && m > h->lp_max[ic]) {
        h->lp_max[ic] = 1.1 * m;
        std::vector<double> tab((size_t)(kNge + 2) * (h->at_num[ic] + 1));
        double dinv = 0.0;
        if (build_ionization_table(h->at_num[ic], h->ion_min[ic], h->model[ic], h->lp_max[ic], h->p.dt, tab.data(), &dinv))
          return AGPU_E_ARG;
        h->de_inv[ic] = dinv;
        a.de_inv = dinv;
        if (int rc = upload_table(h, ic, tab.data(), h->at_num[ic])) return rc;
      }
    }
    k32_ionize<<<grid, 256, 0, h->st>>>(a);
    CK(cudaGetLastError());
    h->timers.launches_total += 2 + 3 + ((iter % 100 == 0) ? 1 : 0);
    if (int rc = drop_removed(h, 0)) return rc;
    long long ne0 = h->np[0];
    long long added = append_electrons32(h->flag, np, h->sp[ic].view(), h->sp[0].view(), ne0, h->cap[0],
                                         h->p.n_mol_atoms[ic], &h->d_cnt->err, h->scr, h->st);
    CK(cudaGetLastError());
    if (ne0 + added > h->cap[0]) {
      h->error_bits |= AGPU_EBIT_CAPACITY;
      added = h->cap[0] - ne0;
    }
    h->np[0] = ne0 + added;
    h->nalive[0] = h->np[0];
    if (added > 0) h->binned[0] = false;
    out->new_electrons += added;
  }
  return 0;
}

}  // namespace

// ============================================================================
// C-ABI
// ============================================================================
extern "C" {

const char* agpu_error_string(int code) {
  switch (code) {
    case AGPU_OK: return "ok";
    case AGPU_E_WINDOW: return "window shift larger than the box (ier = 2)";
    case AGPU_E_COUNT: return "particle count mismatch (ier = 99)";
    case AGPU_E_ARG: return "invalid argument or unsupported configuration";
    case AGPU_E_CUDA: return "CUDA runtime error";
    case AGPU_E_NOMEM: return "device allocation failed";
    case AGPU_E_CAPACITY: return "species capacity exceeded";
    case AGPU_E_INDEX: return "particle stencil outside the field array";
    case AGPU_E_IONZ_INDEX: return "ionization table index beyond n_ge+1";
    case AGPU_E_NONFINITE: return "non-finite particle momentum";
    case AGPU_E_NODEVICE: return "no usable CUDA device";
    case AGPU_E_STATE: return "call out of order";
    default: return "unknown status";
  }
}

int agpu_device_count(int* n) {
  if (!n) return AGPU_E_ARG;
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *n = 0;
    return AGPU_E_NODEVICE;
  }
  *n = c;
  return 0;
}

int agpu_struct_sizes(int64_t* sizes, int32_t n) {
  if (!sizes) return AGPU_E_ARG;
  int64_t s[6] = {(int64_t)sizeof(agpu_params), (int64_t)sizeof(agpu_plasma), (int64_t)sizeof(agpu_laser),
                  (int64_t)sizeof(agpu_step_out), (int64_t)sizeof(agpu_diag_out), (int64_t)sizeof(agpu_timers)};
  for (int i = 0; i < n && i < 6; ++i) sizes[i] = s[i];
  return 0;
}

int agpu_create(const agpu_params* params, agpu_handle** out) {
  if (!params || !out) return AGPU_E_ARG;
  *out = nullptr;
  const agpu_params& p = *params;
  if (!(p.ndim == 2 || p.ndim == 3)) return AGPU_E_ARG;
  if (p.nx < 4 || p.ny < 4 || (p.ndim == 3 && p.nz < 4)) return AGPU_E_ARG;
  if (p.nfield != (p.ndim == 3 ? 6 : 3) || p.curr_ndim != (p.ndim == 3 ? 3 : 2)) return AGPU_E_ARG;
  if (p.ibx != 0 || p.iby != 0 || p.ibz != 0 || p.iform < 0 || p.iform > 2) return AGPU_E_ARG;
  // iform = 2 (the non-conserving deposit) in the FP64 form, quadratic shapes
  if (p.iform == 2 && (p.precision != AGPU_FP64 || p.shape != AGPU_SHAPE_QUADRATIC)) return AGPU_E_ARG;
  // the comoving frame (w_speed < 0) in the FP64 form
  if (p.w_speed < 0.0 && p.precision != AGPU_FP64) return AGPU_E_ARG;
  if (p.nsp < 1 || p.nsp > 4 || p.nsp_run < 1 || p.nsp_run > p.nsp) return AGPU_E_ARG;
  if (p.precision != AGPU_FP64 && p.precision != AGPU_FP32_SPLIT) return AGPU_E_ARG;
  if (p.shape != AGPU_SHAPE_QUADRATIC && p.shape != AGPU_SHAPE_CUBIC) return AGPU_E_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    cudaGetLastError();
    return AGPU_E_NODEVICE;
  }
  agpu_handle* h = new (std::nothrow) agpu_handle();
  if (!h) return AGPU_E_NOMEM;
  h->p = p;
  cudaGetDevice(&h->device);
  cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device);
  h->fp32 = (p.precision == AGPU_FP32_SPLIT);
  Geo& g = h->g;
  g.ndim = p.ndim;
  g.n1p = p.nx + 5;
  g.n2p = p.ny + 5;
  g.n3p = (p.ndim == 3) ? p.nz + 5 : 1;
  g.ix1 = 3;
  g.ix2 = p.nx + 2;
  g.jy1 = 3;
  g.jy2 = p.ny + 2;
  g.kz1 = (p.ndim == 3) ? 3 : 1;
  g.kz2 = (p.ndim == 3) ? p.nz + 2 : 1;
  g.nf = p.nfield;
  g.nc = p.curr_ndim;
  g.ncell = (long long)g.n1p * g.n2p * g.n3p;
  geo_divisors(g);
  if (h->fp32 && g.ncell >= (1ll << 31)) {
    delete h;
    return AGPU_E_ARG;
  }
  h->ndv = (p.ndim == 3) ? 7 : 5;
  int rc = 0;
  if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) rc = AGPU_E_CUDA;
  for (int i = 0; i < 2 * PH_N && !rc; ++i)
    if (cudaEventCreate(&h->ev[i]) != cudaSuccess) rc = AGPU_E_CUDA;
  long long capmax = 16;
  for (int ic = 0; ic < 4; ++ic) {
    h->cap[ic] = (ic < p.nsp) ? std::max<long long>(p.capacity[ic], 16) : 0;
    capmax = std::max(capmax, h->cap[ic]);
  }
  // equal-size slots so that a compaction target can take any species
  for (int ic = 0; ic < p.nsp; ++ic) h->cap[ic] = capmax;
  h->capmax = capmax;
  if (!rc) {
    if (!h->fp32) {
      rc |= dmalloc((void**)&h->ebf, sizeof(double) * g.ncell * g.nf);
      rc |= dmalloc((void**)&h->ebf_alt, sizeof(double) * g.ncell * g.nf);
      rc |= dmalloc((void**)&h->jc, sizeof(double) * g.ncell * g.nc);
      for (int ic = 0; ic < p.nsp && !rc; ++ic) rc |= dmalloc((void**)&h->part[ic], sizeof(double) * capmax * h->ndv);
      if (!rc) rc |= dmalloc((void**)&h->tmp, sizeof(double) * capmax * h->ndv);
    } else {
      rc |= dmalloc((void**)&h->ebf32, sizeof(float) * g.ncell * g.nf);
      rc |= dmalloc((void**)&h->ebf32_alt, sizeof(float) * g.ncell * g.nf);
      rc |= dmalloc((void**)&h->jhi, sizeof(float) * g.ncell * g.nc);
      rc |= dmalloc((void**)&h->jlo, sizeof(float) * g.ncell * g.nc);
      for (int ic = 0; ic < p.nsp && !rc; ++ic) rc |= alloc_species32(h->sp[ic], capmax, p.ndim);
      if (!rc) rc |= alloc_species32(h->sptmp, capmax, p.ndim);
    }
  }
  if (!rc) {
    h->tg = make_tiles(g, p.nx, p.ny, p.nz);
    for (int ic = 0; ic < p.nsp_run && !rc; ++ic) {
      rc |= dmalloc((void**)&h->key[ic], sizeof(int) * capmax);
      rc |= dmalloc((void**)&h->perm[ic], sizeof(int) * capmax);
      rc |= dmalloc((void**)&h->hist[ic], sizeof(int) * (h->tg.nkeys + 1));
      rc |= dmalloc((void**)&h->tstart[ic], sizeof(int) * (h->tg.nkeys + 2));
    }
    if (!rc) rc |= dmalloc((void**)&h->cursor, sizeof(int) * (h->tg.nkeys + 1));
    if (!rc) rc |= dmalloc((void**)&h->scan_tmp, sizeof(int) * bin_scan_tmp_ints(h->tg));
    if (capmax >= (1ll << 31)) rc |= AGPU_E_NOMEM;  // int32 particle indices in the permutation
  }
  if (!rc) {
    rc |= dmalloc((void**)&h->flag, sizeof(int) * capmax);
    if (p.ionz_lev > 0) rc |= dmalloc((void**)&h->ef2, sizeof(double) * capmax);
    rc |= dmalloc((void**)&h->d_cnt, sizeof(Counters));
    long long nb = (capmax + SEL_CHUNK - 1) / SEL_CHUNK + 1;
    rc |= dmalloc((void**)&h->scr.blockcnt, sizeof(long long) * nb);
    rc |= dmalloc((void**)&h->scr.total, sizeof(long long));
    rc |= dmalloc((void**)&h->d_diag, sizeof(double) * 64);
    rc |= dmalloc((void**)&h->d_envar, sizeof(double) * (16 + AGPU_NE));
    if (h->fp32) {
      // every chunk beyond a tile's first holds LIST_CAP particles
      h->tile_work_cap = (int)(capmax / tile32_list_cap(p.ndim)) + 16;
      rc |= dmalloc((void**)&h->tile_work, sizeof(int) * 2 * (size_t)h->tile_work_cap);
      rc |= dmalloc((void**)&h->tile_work_n, 2 * sizeof(unsigned int));
    }
    if (cudaMallocHost((void**)&h->h_cnt, sizeof(Counters)) != cudaSuccess) rc |= AGPU_E_NOMEM;
    if (cudaMallocHost((void**)&h->scr.h_total, sizeof(long long)) != cudaSuccess) rc |= AGPU_E_NOMEM;
  }
  if (!rc && p.w_speed < 0.0) {
    // comoving frame: the advection's buffer and the tridiagonal coefficients
    // of trid_der1 for a = -aphx_exp, b = 1, c = aphx_exp, b1 = bn = 1,
    // c1 = an = 0 (grid_fields.f90:37-77, 210-324), computed once
    const int n = p.nx;
    const double vbeam = -p.w_speed, dth = 0.5 * p.dt;
    const double aphx = dth * p.dx_inv;
    const double aphx_exp = 0.5 * (-vbeam) * aphx;
    const double a = -aphx_exp, b = 1., c = -a, b1 = 1., c1 = 0.0, an = 0.0, bn = 1.;
    std::vector<double> coef(2 * (size_t)(n + 2), 0.0);
    double* bet = coef.data();
    double* w1 = coef.data() + (n + 2);
    w1[1] = 0.0;
    bet[1] = b1;
    w1[2] = c1 / bet[1];
    bet[2] = b - a * w1[2];
    for (int k = 3; k <= n - 1; ++k) {
      w1[k] = c / bet[k - 1];
      bet[k] = b - a * w1[k];
    }
    w1[n] = c / bet[n - 1];
    bet[n] = bn - an * w1[n];
    rc |= dmalloc((void**)&h->xadv_tmp, sizeof(double) * g.ncell);
    rc |= dmalloc((void**)&h->xadv_coef, sizeof(double) * coef.size());
    if (!rc && cudaMemcpy(h->xadv_coef, coef.data(), sizeof(double) * coef.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      rc |= AGPU_E_CUDA;
    h->xadv.tmp = h->xadv_tmp;
    h->xadv.bet = h->xadv_coef;
    h->xadv.w1 = h->xadv_coef + (n + 2);
    h->xadv.a = a;
    h->xadv.aphx_exp = aphx_exp;
  }
  if (!rc) {
    if (h->ebf) cudaMemsetAsync(h->ebf, 0, sizeof(double) * g.ncell * g.nf, h->st);
    if (h->jc) cudaMemsetAsync(h->jc, 0, sizeof(double) * g.ncell * g.nc, h->st);
    if (h->ebf32) cudaMemsetAsync(h->ebf32, 0, sizeof(float) * g.ncell * g.nf, h->st);
    if (h->jhi) cudaMemsetAsync(h->jhi, 0, sizeof(float) * g.ncell * g.nc, h->st);
    if (h->jlo) cudaMemsetAsync(h->jlo, 0, sizeof(float) * g.ncell * g.nc, h->st);
    cudaMemsetAsync(h->d_cnt, 0, sizeof(Counters), h->st);
    if (cudaStreamSynchronize(h->st) != cudaSuccess) rc = AGPU_E_CUDA;
  }
  if (rc) {
    free_all(h);
    delete h;
    return rc & AGPU_E_NOMEM ? AGPU_E_NOMEM : AGPU_E_CUDA;
  }
  *out = h;
  return 0;
}

int agpu_destroy(agpu_handle* h) {
  if (!h) return AGPU_E_ARG;
  cudaStreamSynchronize(h->st);
  free_all(h);
  delete h;
  return 0;
}

int agpu_set_fields(agpu_handle* h, const double* ebf, int32_t n1p, int32_t n2p, int32_t n3p, int32_t nc) {
  if (!h || !ebf) return AGPU_E_ARG;
  const Geo& g = h->g;
  if (n1p != g.n1p || n2p != g.n2p || n3p != g.n3p || nc != g.nf) return AGPU_E_ARG;
  size_t n = (size_t)g.ncell * g.nf;
  if (!h->fp32) {
    CK(cudaMemcpyAsync(h->ebf, ebf, sizeof(double) * n, cudaMemcpyHostToDevice, h->st));
  } else {
    double* stage = nullptr;
    if (dmalloc((void**)&stage, sizeof(double) * n)) return AGPU_E_NOMEM;
    cudaMemcpyAsync(stage, ebf, sizeof(double) * n, cudaMemcpyHostToDevice, h->st);
    f64_to_f32(stage, h->ebf32, (long long)n, h->st, h->sms);
    cudaStreamSynchronize(h->st);
    cudaFree(stage);
  }
  CK(cudaStreamSynchronize(h->st));
  h->fields_set = true;
  return 0;
}

int agpu_get_fields(agpu_handle* h, double* ebf, int32_t n1p, int32_t n2p, int32_t n3p, int32_t nc) {
  if (!h || !ebf) return AGPU_E_ARG;
  const Geo& g = h->g;
  if (n1p != g.n1p || n2p != g.n2p || n3p != g.n3p || nc != g.nf) return AGPU_E_ARG;
  size_t n = (size_t)g.ncell * g.nf;
  if (!h->fp32) {
    CK(cudaMemcpyAsync(ebf, h->ebf, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st));
  } else {
    double* stage = nullptr;
    if (dmalloc((void**)&stage, sizeof(double) * n)) return AGPU_E_NOMEM;
    f32_to_f64(h->ebf32, stage, (long long)n, h->st, h->sms);
    cudaMemcpyAsync(ebf, stage, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st);
    cudaStreamSynchronize(h->st);
    cudaFree(stage);
  }
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

int agpu_get_currents(agpu_handle* h, double* jc, int32_t n1p, int32_t n2p, int32_t n3p, int32_t nc) {
  if (!h || !jc) return AGPU_E_ARG;
  const Geo& g = h->g;
  if (n1p != g.n1p || n2p != g.n2p || n3p != g.n3p || nc != g.nc) return AGPU_E_ARG;
  size_t n = (size_t)g.ncell * g.nc;
  if (!h->fp32) {
    CK(cudaMemcpyAsync(jc, h->jc, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st));
  } else {
    double* stage = nullptr;
    if (dmalloc((void**)&stage, sizeof(double) * n)) return AGPU_E_NOMEM;
    f32pair_to_f64(h->jhi, h->jlo, stage, (long long)n, h->st, h->sms);
    cudaMemcpyAsync(jc, stage, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st);
    cudaStreamSynchronize(h->st);
    cudaFree(stage);
  }
  CK(cudaStreamSynchronize(h->st));
  // curr = djc(i) * curr (curr_and_fields_util.f90:111-115), whole array
  if (h->p.iform < 2)
    for (int i = 0; i < h->p.ndim; ++i) {
      double d = h->p.djc[i];
      double* c = jc + (size_t)g.ncell * i;
      for (size_t q = 0; q < (size_t)g.ncell; ++q) c[q] = d * c[q];
    }
  if (h->str) {
    // the stretched metric on the interior (curr_and_fields_util.f90:120-150)
    const int ny = h->p.ny;
    const double* my3 = h->h_metric.data();
    const double* my4 = my3 + (ny + 2);
    const double* mz3 = my3 + 2 * (ny + 2);
    const double* mz4 = mz3 + (h->p.ndim == 3 ? h->p.nz + 2 : 0);
    auto at = [&](int c, int i, int j, int k) -> double& {
      return jc[(size_t)g.ncell * c + (size_t)(i - 1) + (size_t)g.n1p * ((size_t)(j - 1) + (size_t)g.n2p * (k - 1))];
    };
    for (int k = g.kz1; k <= g.kz2; ++k)
      for (int j = g.jy1; j <= g.jy2; ++j)
        for (int i = g.ix1; i <= g.ix2; ++i) {
          const double dery = my3[j - 2], derhy = my4[j - 2];
          if (g.nc == 2) {
            at(0, i, j, k) = dery * at(0, i, j, k);
            at(1, i, j, k) = derhy * at(1, i, j, k);
          } else {
            const double derz = mz3[k - 2], derhz = mz4[k - 2];
            at(0, i, j, k) = dery * derz * at(0, i, j, k);
            at(1, i, j, k) = derhy * derz * at(1, i, j, k);
            at(2, i, j, k) = dery * derhz * at(2, i, j, k);
          }
        }
  }
  return 0;
}

int agpu_set_species(agpu_handle* h, int32_t ic, const double* part, int64_t ld, int64_t np, int32_t ndv) {
  if (!h || ic < 0 || ic >= h->p.nsp || ndv != h->ndv || np < 0 || (np > 0 && (!part || ld < np))) return AGPU_E_ARG;
  if (np > h->cap[ic]) return AGPU_E_CAPACITY;
  if (!h->fp32) {
    if (np > 0)
      CK(cudaMemcpy2DAsync(h->part[ic], sizeof(double) * h->cap[ic], part, sizeof(double) * ld, sizeof(double) * np, ndv,
                           cudaMemcpyHostToDevice, h->st));
  } else if (np > 0) {
    double* stage = nullptr;
    if (dmalloc((void**)&stage, sizeof(double) * np * ndv)) return AGPU_E_NOMEM;
    cudaMemcpy2DAsync(stage, sizeof(double) * np, part, sizeof(double) * ld, sizeof(double) * np, ndv, cudaMemcpyHostToDevice,
                      h->st);
    rec_to_split(stage, np, np, h->sp[ic].view(), 0, h->g, h->p.xmn, h->p.ymn, h->p.zmn, h->p.dx_inv, h->p.dy_inv, h->p.dz_inv,
                 h->st, h->sms);
    cudaStreamSynchronize(h->st);
    cudaFree(stage);
  }
  CK(cudaStreamSynchronize(h->st));
  h->np[ic] = np;
  h->nalive[ic] = np;
  h->binned[ic] = false;
  h->stale[ic] = false;
  return 0;
}

int agpu_get_species(agpu_handle* h, int32_t ic, double* part, int64_t ld, int64_t* np, int32_t ndv) {
  if (!h || ic < 0 || ic >= h->p.nsp || !np) return AGPU_E_ARG;
  if (int rc = refresh_counts(h)) return rc;
  if (h->binned[ic] && h->nalive[ic] != h->np[ic]) {
    if (int rc = drop_removed(h, ic)) return rc;
  }
  *np = h->np[ic];
  if (!part) return 0;
  if (ndv != h->ndv || ld < h->np[ic]) return AGPU_E_ARG;
  long long n = h->np[ic];
  if (n == 0) return 0;
  if (!h->fp32) {
    CK(cudaMemcpy2DAsync(part, sizeof(double) * ld, h->part[ic], sizeof(double) * h->cap[ic], sizeof(double) * n, ndv,
                         cudaMemcpyDeviceToHost, h->st));
  } else {
    double* stage = nullptr;
    if (dmalloc((void**)&stage, sizeof(double) * n * ndv)) return AGPU_E_NOMEM;
    split_to_rec(h->sp[ic].view(), n, stage, n, h->g, h->p.xmn, h->p.ymn, h->p.zmn, h->p.dx, h->p.dy, h->p.dz, h->st, h->sms);
    cudaMemcpy2DAsync(part, sizeof(double) * ld, stage, sizeof(double) * n, sizeof(double) * n, ndv, cudaMemcpyDeviceToHost,
                      h->st);
    cudaStreamSynchronize(h->st);
    cudaFree(stage);
  }
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

int agpu_get_count(agpu_handle* h, int32_t ic, int64_t* np) {
  if (!h || !np || ic < 0 || ic >= h->p.nsp) return AGPU_E_ARG;
  if (int rc = refresh_counts(h)) return rc;
  *np = h->binned[ic] ? h->nalive[ic] : h->np[ic];
  return 0;
}

int agpu_get_window_state(agpu_handle* h, double* xlapse, int64_t* nptx, int64_t* sptx_max, double* xmn) {
  if (!h || !xlapse || !nptx || !sptx_max || !xmn) return AGPU_E_ARG;
  *xlapse = h->xlapse;
  for (int ic = 0; ic < 4; ++ic) {
    nptx[ic] = h->nptx[ic];
    sptx_max[ic] = h->sptx_max[ic];
  }
  *xmn = h->p.xmn;
  return 0;
}
int agpu_set_window_state(agpu_handle* h, double xlapse, const int64_t* nptx) {
  if (!h || !nptx || !(xlapse >= 0.0)) return AGPU_E_ARG;
  for (int ic = 0; ic < 4; ++ic)
    if (nptx[ic] < 0) return AGPU_E_ARG;
  h->xlapse = xlapse;
  h->wi1 = (int)std::lround(h->p.dx_inv * xlapse);
  for (int ic = 0; ic < 4; ++ic) h->nptx[ic] = nptx[ic];
  return 0;
}

int agpu_set_plasma_source(agpu_handle* h, const agpu_plasma* src) {
  if (!h || !src) return AGPU_E_ARG;
  int ic = src->ic;
  if (ic < 0 || ic >= h->p.nsp || src->npx < 1 || src->npy < 1 || src->npz < 1) return AGPU_E_ARG;
  if (!(src->jitter >= 0.0 && src->jitter < 1.0)) return AGPU_E_ARG;
  if (h->str) return AGPU_E_STATE;  // stretched targets come from the host
  h->src[ic] = *src;
  h->has_src[ic] = true;
  h->nptx[ic] = 0;
  double dxl = h->p.dx / (double)src->npx;
  double dyl = h->p.dy / (double)src->npy;
  double dzl = h->p.dz / (double)src->npz;
  h->sptx_max[ic] = (long long)std::floor((src->x_end - src->x_start) / dxl + 1e-9);
  h->npty[ic] = (int)std::floor((src->y_max - src->y_min) / dyl + 1e-9);
  h->nptz[ic] = (h->p.ndim == 3) ? (int)std::floor((src->z_max - src->z_min) / dzl + 1e-9) : 1;
  return 0;
}

int agpu_load_plasma(agpu_handle* h, int32_t ic) {
  if (!h || ic < 0 || ic >= h->p.nsp) return AGPU_E_ARG;
  if (!h->has_src[ic]) return AGPU_E_STATE;
  h->nptx[ic] = 0;
  long long i2 = lattice_columns_end(h, ic, 1, h->p.xmax, false);
  h->nptx[ic] = i2;
  int rc = 0;
  if (i2 >= 1) rc = add_lattice_columns(h, ic, 1, i2);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

int agpu_init_lp_fields(agpu_handle* h, const agpu_lp_pulse* l) {
  if (!h || !l || !(l->wx > 0.0) || !(l->wy > 0.0) || !(l->om0 > 0.0)) return AGPU_E_ARG;
  LaserArgs a;
  a.ndim = h->p.ndim;
  a.g_prof = l->g_prof ? 1 : 0;
  a.ee0 = l->ee0;
  a.t1 = l->t_loc - l->tf;  // coords(4)
  a.xf0 = l->xf0;
  a.om0 = l->om0;
  a.wx = l->wx;
  a.wy = l->wy;
  a.zra = 0.5 * l->om0 * l->wy * l->wy;  // par_lp(5)
  a.eps = 1. / (l->om0 * l->wy);         // par_lp(6)
  a.ycent = l->ycent;
  a.zcent = l->zcent;
  a.xmn = h->p.xmn;
  a.ymn = h->p.ymn;
  a.zmn = h->p.zmn;
  a.dx = h->p.dx;
  a.dy = h->p.dy;
  a.dz = h->p.dz;
  size_t n = (size_t)h->g.ncell * h->g.nf;
  if (!h->fp32) {
    laser64(a, h->ebf, h->g, h->st, h->sms);
  } else {
    double* stage = nullptr;
    if (dmalloc((void**)&stage, sizeof(double) * n)) return AGPU_E_NOMEM;
    f32_to_f64(h->ebf32, stage, (long long)n, h->st, h->sms);
    laser64(a, stage, h->g, h->st, h->sms);
    f64_to_f32(stage, h->ebf32, (long long)n, h->st, h->sms);
    cudaStreamSynchronize(h->st);
    cudaFree(stage);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->st));
  h->fields_set = true;
  return 0;
}

int agpu_init_laser(agpu_handle* h, const agpu_laser* l) {
  if (!h || !l || !(l->lam0 > 0.0) || !(l->tau_fwhm > 0.0)) return AGPU_E_ARG;
  // lp_pulse (src/IO/init_laser_field.f90:33-100) with the set_initial_param
  // quantities (set_init_param.f90:291-330): Gaussian profile, aph_fwhm =
  // sqrt(2 ln 2), lx_fwhm = tau_fwhm (a length, um/c)
  const double pi2 = 2.0 * 3.141592653589793;
  agpu_lp_pulse a;
  a.om0 = pi2 / l->lam0;
  a.ee0 = l->a0 * a.om0;
  a.wx = l->tau_fwhm / std::sqrt(2. * std::log(2.));
  a.wy = l->w0_y;
  a.xf0 = l->xf;
  a.tf = l->xf - l->xc;
  a.t_loc = 0.0;
  a.ycent = l->y0;
  a.zcent = l->z0;
  a.g_prof = 1;
  a.reserved = 0;
  return agpu_init_lp_fields(h, &a);
}

int agpu_set_ionization_table(agpu_handle* h, int32_t ic, const double* w_one_lev, int32_t n_ge, int32_t zmax, double de_inv) {
  if (!h || !w_one_lev || ic < 1 || ic >= h->p.nsp || n_ge != kNge || zmax < 1 || zmax > 100) return AGPU_E_ARG;
  h->de_inv[ic] = de_inv;
  h->auto_table[ic] = false;
  return upload_table(h, ic, w_one_lev, zmax);
}

int agpu_build_ionization_table(int32_t atomic_number, int32_t ion_min, int32_t ionz_model, double lp_max, double dt,
                                double* w_one_lev, double* de_inv) {
  if (!w_one_lev || !de_inv) return AGPU_E_ARG;
  return build_ionization_table(atomic_number, ion_min, ionz_model, lp_max, dt, w_one_lev, de_inv) ? AGPU_E_ARG : 0;
}

int agpu_set_ionization_species(agpu_handle* h, int32_t ic, int32_t atomic_number, int32_t ion_min, int32_t ion_max,
                                int32_t ionz_model, double lp_max) {
  if (!h || ic < 1 || ic >= h->p.nsp || ion_min < 0 || ion_max > atomic_number || ion_min >= ion_max) return AGPU_E_ARG;
  std::vector<double> tab((size_t)(kNge + 2) * (atomic_number + 1));
  double dinv = 0.0;
  if (build_ionization_table(atomic_number, ion_min, ionz_model, lp_max, h->p.dt, tab.data(), &dinv)) return AGPU_E_ARG;
  h->at_num[ic] = atomic_number;
  h->ion_min[ic] = ion_min;
  h->model[ic] = ionz_model;
  h->lp_max[ic] = lp_max;
  h->de_inv[ic] = dinv;
  h->auto_table[ic] = true;
  return upload_table(h, ic, tab.data(), atomic_number);
}

static int step_impl(agpu_handle* h, int32_t iter, double t, int32_t initial_time, agpu_step_out* out);

// What a captured step's launches depend on: particle counts and array
// pointers (compactions swap buffers), binning state and the box.
static void step_signature(const agpu_handle* h, unsigned char* sig) {
  struct Sig {
    long long np[4];
    const void* ptr[4];
    int binned[4];
    double box[7];
    int det, nsp_run;
  } g;
  std::memset(&g, 0, sizeof(g));
  for (int ic = 0; ic < 4; ++ic) {
    g.np[ic] = h->np[ic];
    g.ptr[ic] = h->fp32 ? (const void*)h->sp[ic].cell : (const void*)h->part[ic];
    g.binned[ic] = h->binned[ic] ? 1 : 0;
  }
  const agpu_params& p = h->p;
  const double box[7] = {p.xmn, p.gxmin, p.gxmax, p.gymin, p.gymax, p.gzmin, p.gzmax};
  std::memcpy(g.box, box, sizeof(box));
  g.det = h->deterministic ? 1 : 0;
  g.nsp_run = p.nsp_run;
  static_assert(sizeof(Sig) <= sizeof(h->gsig), "signature buffer");
  std::memset(sig, 0, sizeof(h->gsig));
  std::memcpy(sig, &g, sizeof(g));
}

int agpu_step(agpu_handle* h, int32_t iter, double t, int32_t initial_time, agpu_step_out* out) {
  if (!h) return AGPU_E_ARG;
  const agpu_params& p = h->p;
  bool plain = h->use_graph && h->defer && !initial_time && p.ionz_lev == 0 && !h->profiling && !h->deterministic;
  if (plain && p.w_speed != 0.0 && p.w_sh > 0 && t >= p.wi_time && t < p.wf_time && iter % p.w_sh == 0) plain = false;
  if (plain && sort_step(h, iter)) plain = false;
  for (int ic = 0; ic < p.nsp_run && plain; ++ic)
    if (h->np[ic] > 0 && !(h->binned[ic] && h->key[ic])) plain = false;
  if (!plain) return step_impl(h, iter, t, initial_time, out);
  agpu_step_out dummy;
  if (!out) out = &dummy;
  unsigned char sig[sizeof(h->gsig)];
  step_signature(h, sig);
  if (!h->gexec || std::memcmp(sig, h->gsig, sizeof(sig)) != 0) {
    // capture this step's launches into a graph (nothing runs yet)
    const agpu_timers before = h->timers;
    cudaGraph_t gr = nullptr;
    CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    int rc = step_impl(h, iter, t, initial_time, out);
    cudaError_t ec = cudaStreamEndCapture(h->st, &gr);
    if (rc || ec != cudaSuccess || !gr) {
      if (gr) cudaGraphDestroy(gr);
      cudaGetLastError();
      h->timers = before;
      if (rc) return rc;
      h->use_graph = false;  // capture refused: plain launches from here on
      return step_impl(h, iter, t, initial_time, out);
    }
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    h->gexec = nullptr;
    cudaError_t ei = cudaGraphInstantiate(&h->gexec, gr, 0);
    cudaGraphDestroy(gr);
    if (ei != cudaSuccess) {
      cudaGetLastError();
      h->gexec = nullptr;
      h->timers = before;
      h->use_graph = false;
      return step_impl(h, iter, t, initial_time, out);
    }
    std::memcpy(h->gsig, sig, sizeof(sig));
    h->g_launches = h->timers.launches_total - before.launches_total;
    h->g_push = h->timers.launches_push_deposit - before.launches_push_deposit;
    h->g_yee = h->timers.launches_yee - before.launches_yee;
    h->g_cells = h->timers.yee_cells - before.yee_cells;
    h->timers = before;
  } else {
    std::memset(out, 0, sizeof(*out));
    out->ion_field_max = -1.0;
    for (int ic = 0; ic < 4; ++ic) out->np[ic] = h->binned[ic] ? h->nalive[ic] : h->np[ic];
    out->xmn = p.xmn;
    out->error_bits = h->error_bits;
  }
  CK(cudaGraphLaunch(h->gexec, h->st));
  h->timers.launches_total += h->g_launches;
  h->timers.launches_push_deposit += h->g_push;
  h->timers.launches_yee += h->g_yee;
  h->timers.yee_cells += h->g_cells;
  return 0;
}

// ---- multi-instance steps (used by the batch runner) -----------------------
// A step is "plain" when it is a deferred-count step between window shifts
// of the split form with one running species, binned, no ionization and no
// profiling: exactly the launches that one multi-instance step performs.
int agpu_x_plain(agpu_handle* h, int32_t iter, double t, int32_t initial_time) {
  if (!h) return 0;
  const agpu_params& p = h->p;
  if (!h->fp32 || !h->defer || initial_time || p.ionz_lev > 0 || h->profiling || h->deterministic || p.nsp_run != 1 ||
      p.shape != AGPU_SHAPE_QUADRATIC)
    return 0;
  if (p.w_speed > 0.0 && p.w_sh > 0 && t >= p.wi_time && t < p.wf_time && iter % p.w_sh == 0) return 0;
  if (h->np[0] <= 0 || !h->binned[0] || !h->key[0]) return 0;
  return 1;
}

struct agpu_x_ws {
  int maxn = 0;
  cudaStream_t st = nullptr;
  MultiInst* d_desc = nullptr;
  MultiInst* h_desc = nullptr;
  int* d_off = nullptr;
  int* h_off = nullptr;
  long long launches = 0;
};

int agpu_x_ws_create(int32_t maxn, agpu_x_ws** out) {
  if (!out || maxn < 1) return AGPU_E_ARG;
  agpu_x_ws* w = new (std::nothrow) agpu_x_ws();
  if (!w) return AGPU_E_NOMEM;
  w->maxn = maxn;
  int rc = 0;
  if (cudaStreamCreateWithFlags(&w->st, cudaStreamNonBlocking) != cudaSuccess) rc = AGPU_E_CUDA;
  if (!rc) rc |= dmalloc((void**)&w->d_desc, sizeof(MultiInst) * maxn);
  if (!rc) rc |= dmalloc((void**)&w->d_off, sizeof(int) * (maxn + 1));
  if (!rc && cudaMallocHost((void**)&w->h_desc, sizeof(MultiInst) * maxn) != cudaSuccess) rc = AGPU_E_NOMEM;
  if (!rc && cudaMallocHost((void**)&w->h_off, sizeof(int) * (maxn + 1)) != cudaSuccess) rc = AGPU_E_NOMEM;
  if (rc) {
    cudaGetLastError();
    cudaFree(w->d_desc);
    cudaFree(w->d_off);
    cudaFreeHost(w->h_desc);
    cudaFreeHost(w->h_off);
    if (w->st) cudaStreamDestroy(w->st);
    delete w;
    return rc;
  }
  *out = w;
  return 0;
}

int agpu_x_ws_destroy(agpu_x_ws* w) {
  if (!w) return AGPU_E_ARG;
  cudaStreamSynchronize(w->st);
  cudaFree(w->d_desc);
  cudaFree(w->d_off);
  cudaFreeHost(w->h_desc);
  cudaFreeHost(w->h_off);
  cudaStreamDestroy(w->st);
  delete w;
  return 0;
}

long long agpu_x_ws_launches(const agpu_x_ws* w) { return w ? w->launches : 0; }

// One plain step of n handles (all agpu_x_plain, same ndim, their streams
// idle) as one launch per phase on the workspace's stream; returns after the
// step has finished on the GPU.
int agpu_x_step_many(agpu_handle** hs, int32_t n, agpu_x_ws* w) {
  if (!hs || !w || n < 1 || n > w->maxn) return AGPU_E_ARG;
  const int ndim = hs[0]->p.ndim;
  long long max_cells = 1, max_faces = 1, max_np = 1;
  int total = 0;
  for (int i = 0; i < n; ++i) {
    agpu_handle* h = hs[i];
    if (h->p.ndim != ndim) return AGPU_E_ARG;
    const Geo& g = h->g;
    const agpu_params& p = h->p;
    MultiInst& m = w->h_desc[i];
    TileArgs32& a = m.ta;
    a.g = g;
    a.t = h->tg;
    a.ebf = h->ebf32;
    a.jhi = h->jhi;
    a.jlo = h->jlo;
    const Species32& sp = h->sp[0];
    a.p = Part32{sp.cell, sp.ox, sp.oy, sp.oz, sp.px, sp.py, sp.pz, sp.slot};
    a.perm = h->perm[0];
    a.tstart = h->tstart[0];
    a.key = h->key[0];
    a.hist = h->hist[0];
    a.dth = (float)(0.5 * p.dt);
    a.lfact = (float)p.lorentz_fact[0];
    a.dtx = (float)(p.dt * p.dx_inv);
    a.dty = (float)(p.dt * p.dy_inv);
    a.dtz = (float)(p.dt * p.dz_inv);
    a.initial = 0;
    a.err = &h->d_cnt->err;
    a.work = nullptr;  // the multi-instance tile kernel runs every chunk in the tile's CTA
    a.work_n = nullptr;
    a.work_cap = 0;
    m.ebf = h->ebf32;
    m.yc = yee_coef(p);
    m.cursor = h->cursor;
    m.pushed = &h->d_cnt->pushed;
    m.removed = &h->d_cnt->removed;
    m.fmax = &h->d_cnt->fmax;
    m.np = h->np[0];
    w->h_off[i] = total;
    total += h->tg.ntiles;
    long long cells = (long long)p.nx * p.ny * (ndim == 3 ? p.nz : 1);
    long long faces = (long long)(p.ny + 3) * (ndim == 3 ? p.nz + 3 : 1) + (long long)(p.nx + 3) * (ndim == 3 ? p.nz + 3 : 1) +
                      (ndim == 3 ? (long long)(p.nx + 3) * (p.ny + 3) : 0);
    max_cells = std::max(max_cells, std::max(cells, g.ncell * g.nc));
    max_faces = std::max(max_faces, faces * g.nf);
    max_np = std::max(max_np, h->np[0]);
  }
  w->h_off[n] = total;
  auto blocks = [](long long work, int cap) { return (int)std::max(1LL, std::min<long long>((work + 255) / 256, cap)); };
  MultiPlan pl;
  pl.n = n;
  pl.ndim = ndim;
  pl.total_tiles = total;
  pl.gx_cells = blocks(max_cells, 64);
  pl.gx_faces = blocks(max_faces, 16);
  pl.gx_parts = blocks(max_np, 128);
  cudaStream_t st = w->st;
  CK(cudaMemcpyAsync(w->d_desc, w->h_desc, sizeof(MultiInst) * n, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(w->d_off, w->h_off, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
  int launches = 0;
  multi_pre32(w->d_desc, pl, st, &launches);
  multi_field_bd32(w->d_desc, pl, st, &launches);
  multi_tile32(w->d_desc, w->d_off, pl, st, &launches);
  multi_bin32(w->d_desc, pl, st, &launches);
  multi_fields32(w->d_desc, pl, st, &launches);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  w->launches += launches;
  for (int i = 0; i < n; ++i) {
    agpu_handle* h = hs[i];
    h->stale[0] = true;
    h->timers.launches_push_deposit += 1;
    h->timers.launches_yee += 1;
    h->timers.yee_cells += (long long)h->p.nx * h->p.ny * (ndim == 3 ? h->p.nz : 1);
  }
  return 0;
}

int agpu_set_step_graphs(agpu_handle* h, int32_t on) {
  if (!h) return AGPU_E_ARG;
  if (on && (h->dd || h->str)) return AGPU_E_STATE;  // a slab's exchanges run between the kernels
  h->use_graph = on != 0;
  if (!h->use_graph && h->gexec) {
    cudaStreamSynchronize(h->st);
    cudaGraphExecDestroy(h->gexec);
    h->gexec = nullptr;
  }
  return 0;
}

// The stretched axes' metric in the Yee coefficients (no-op on a uniform grid).
static void stretch_coef(const agpu_handle* h, YeeC& c) {
  if (!h->str) return;
  const int ny = h->p.ny, nz = h->p.ndim == 3 ? h->p.nz : 0;
  c.my3 = h->d_metric;
  c.my4 = h->d_metric + (ny + 2);
  if (h->p.ndim == 3) {
    c.mz3 = h->d_metric + 2 * (ny + 2);
    c.mz4 = h->d_metric + 2 * (ny + 2) + (nz + 2);
  }
  c.by3 = h->by3;
  c.ty4 = h->ty4;
  c.bz3 = h->bz3;
  c.tz4 = h->tz4;
}

// The host's exchange at one point of a y slab's step (no-op otherwise).
static int halo_call(agpu_handle* h, int point, int ic) {
  if (!h->dd || !h->halo_fn) return 0;
  return h->halo_fn(h->halo_user, h, point, ic);
}
static int yee_halo(void* ctx, int point) { return halo_call((agpu_handle*)ctx, point, -1); }

static int step_impl(agpu_handle* h, int32_t iter, double t, int32_t initial_time, agpu_step_out* out) {
  if (!h) return AGPU_E_ARG;
  agpu_step_out dummy;
  if (!out) out = &dummy;
  std::memset(out, 0, sizeof(*out));
  out->ion_field_max = -1.0;
  agpu_params& p = h->p;
  int rc = 0;
  if (h->defer) {
    // keep the error word and the push count accumulating on the device
    CK(cudaMemsetAsync(&h->d_cnt->removed, 0, sizeof(unsigned long long), h->st));
    CK(cudaMemsetAsync(&h->d_cnt->fmax, 0, sizeof(double), h->st));
    if (p.ionz_lev > 0)
      if (int rc_ = refresh_counts(h)) return rc_;
  } else {
    CK(cudaMemsetAsync(h->d_cnt, 0, sizeof(Counters), h->st));
  }
  // pfields_prepare -> field_xyzbd
  ph_begin(h, PH_YEE);
  if (h->fp32) field_bd32(Dev32{h->g, h->ebf32, h->jhi, h->jlo}, h->st, h->sms);
  else field_bd64(Dev64{h->g, h->ebf, h->jc}, h->st, h->sms);
  CK(cudaGetLastError());
  h->timers.launches_total += (p.ndim == 3) ? 3 : 2;
  if (int rc_ = halo_call(h, AGPU_HALO_FIELDS, -1)) return rc_;
  ph_end(h, PH_YEE);
  // ionization
  if (p.ionz_lev > 0) {
    ph_begin(h, PH_IONIZE);
    rc = h->fp32 ? ionize32(h, iter, out) : ionize64(h, iter, out);
    ph_end(h, PH_IONIZE);
    if (rc) return rc;
  }
  // jc = 0, then each running species: gather/push/deposit
  if (h->fp32) {
    CK(cudaMemsetAsync(h->jhi, 0, sizeof(float) * h->g.ncell * h->g.nc, h->st));
    CK(cudaMemsetAsync(h->jlo, 0, sizeof(float) * h->g.ncell * h->g.nc, h->st));
  } else {
    CK(cudaMemsetAsync(h->jc, 0, sizeof(double) * h->g.ncell * h->g.nc, h->st));
  }
  for (int ic = 0; ic < p.nsp_run; ++ic) {
    long long np = h->np[ic];
    if (np <= 0) {
      // an empty slab still takes part in the particle exchange
      if (int rc_ = halo_call(h, AGPU_HALO_PARTICLES, ic)) return rc_;
      continue;
    }
    if (tiled(h, ic)) {
      if (int rc_ = tiled_push(h, ic, initial_time, out)) return rc_;
      if (sort_step(h, iter))
        if (int rc_ = reorder_records(h, ic)) return rc_;
      continue;
    }
    if (int rc_ = drop_removed(h, ic)) return rc_;
    np = h->np[ic];
    CK(cudaMemsetAsync(&h->d_cnt->removed, 0, sizeof(unsigned long long), h->st));
    ph_begin(h, PH_PUSH);
    if (h->fp32) {
      PushArgs32 a;
      a.g = h->g;
      a.ebf = h->ebf32;
      a.jhi = h->jhi;
      a.jlo = h->jlo;
      const Species32& s = h->sp[ic];
      a.p = Part32{s.cell, s.ox, s.oy, s.oz, s.px, s.py, s.pz, s.slot};
      a.flag = h->flag;
      a.np = np;
      a.dt = (float)p.dt;
      a.dth = (float)(0.5 * p.dt);
      a.lfact = (float)p.lorentz_fact[ic];
      a.dtx = (float)(p.dt * p.dx_inv);
      a.dty = (float)(p.dt * p.dy_inv);
      a.dtz = (float)(p.dt * p.dz_inv);
      a.initial = initial_time ? 1 : 0;
      a.removed = &h->d_cnt->removed;
      a.err = &h->d_cnt->err;
      push_deposit32(a, h->st, h->sms);
    } else {
      PushArgs64 a;
      a.g = h->g;
      a.ebf = h->ebf;
      a.jc = h->jc;
      double* b = h->part[ic];
      long long cp = h->cap[ic];
      a.x = b;
      a.y = b + cp;
      if (p.ndim == 3) {
        a.z = b + 2 * cp;
        a.px = b + 3 * cp;
        a.py = b + 4 * cp;
        a.pz = b + 5 * cp;
        a.slot = b + 6 * cp;
      } else {
        a.z = nullptr;
        a.px = b + 2 * cp;
        a.py = b + 3 * cp;
        a.pz = nullptr;
        a.slot = b + 4 * cp;
      }
      a.flag = h->flag;
      a.np = np;
      a.xmn = p.xmn;
      a.ymn = p.ymn;
      a.zmn = p.zmn;
      a.dx_inv = p.dx_inv;
      a.dy_inv = p.dy_inv;
      a.dz_inv = p.dz_inv;
      a.dt = p.dt;
      a.dth = 0.5 * p.dt;
      a.lfact = p.lorentz_fact[ic];
      a.gxmin = p.gxmin;
      a.gxmax = p.gxmax;
      a.gymin = p.gymin;
      a.gymax = p.gymax;
      a.gzmin = p.gzmin;
      a.gzmax = p.gzmax;
      a.vdt = comoving_vdt(p);
      a.initial = initial_time ? 1 : 0;
      a.shape = p.shape;
      a.iform = p.iform;
      a.dd_ylo = h->dd_lo;
      a.dd_yhi = h->dd_hi;
      a.dd_zlo = h->dd_zlo;
      a.dd_zhi = h->dd_zhi;
      a.str = h->str ? 1 : 0;
      a.sy = h->sy;
      a.sz = h->sz;
      a.removed = &h->d_cnt->removed;
      a.err = &h->d_cnt->err;
      push_deposit64(a, h->st, h->sms, h->deterministic);
    }
    CK(cudaGetLastError());
    ph_end(h, PH_PUSH);
    h->timers.launches_push_deposit += 1;
    h->timers.launches_total += 1;
    h->timers.pushes += np;
    if (int rc_ = read_counters(h)) return rc_;
    // a y slab: the particles that crossed a shared side go to the
    // neighbours (the host's hook), the ones that arrive are appended
    if (int rc_ = halo_call(h, AGPU_HALO_PARTICLES, ic)) return rc_;
    if (h->h_cnt->removed > 0) {
      ph_begin(h, PH_SORT);
      long long before = h->np[ic];
      rc = compact_species(h, ic, false);
      ph_end(h, PH_SORT);
      if (rc) return rc;
      out->removed[ic] += before - h->np[ic];
    }
  }
  // curr_mpi_collect -> jc_xyzbd (djc folded into the E update)
  ph_begin(h, PH_YEE);
  YeeC c = yee_coef(p);
  stretch_coef(h, c);
  // the fused step writes a second field array (its tiles read halos of the
  // input); not inside step graphs, whose launches keep their pointers
  // (the comoving frame's advection substeps and the stretched metric run
  // only in the plain sweeps)
  const bool fused = h->fused_yee && !h->use_graph && !h->xadv.tmp && !h->str;
  if (h->fp32) {
    Dev32 d{h->g, h->ebf32, h->jhi, h->jlo};
    jfold32(d, h->st, h->sms);
    if (fused) {
      yee32_fused(h->ebf32, h->ebf32_alt, h->jhi, h->jlo, h->g, c, h->st);
      std::swap(h->ebf32, h->ebf32_alt);
    } else {
      yee32(d, c, h->st, h->sms);
    }
  } else {
    Dev64 d{h->g, h->ebf, h->jc};
    if (int rc_ = halo_call(h, AGPU_HALO_CURRENTS, -1)) return rc_;
    jfold64(d, h->st, h->sms);
    if (fused) {
      yee64_fused(h->ebf, h->ebf_alt, h->jc, h->g, c, h->st);
      std::swap(h->ebf, h->ebf_alt);
    } else {
      YeeHook hk{yee_halo, h, 0};
      yee64(d, c, h->st, h->sms, h->xadv.tmp ? &h->xadv : nullptr, h->dd ? &hk : nullptr);
      if (hk.rc) return hk.rc;
    }
  }
  CK(cudaGetLastError());
  ph_end(h, PH_YEE);
  h->timers.launches_yee += 1;
  // current fold (x, y[, z] faces; hi and lo in the split form) + the Yee kernels
  h->timers.launches_total += ((p.ndim == 3) ? 3 : 2) * (h->fp32 ? 2 : 1) + (fused ? 1 : 6) + xadv_launches(h);
  h->timers.yee_cells += (long long)p.nx * p.ny * (p.ndim == 3 ? p.nz : 1);
  // lp_run: moving window, or the comoving frame's coordinate shift
  if (int rc_ = window_or_comoving(h, iter, t, out)) return rc_;
  if (!h->defer)
    if (int rc_ = read_counters(h)) return rc_;
  // deferred mode: the counts of the last synchronisation point
  for (int ic = 0; ic < 4; ++ic) out->np[ic] = h->binned[ic] ? h->nalive[ic] : h->np[ic];
  out->xmn = p.xmn;
  out->error_bits = h->error_bits;
  if (h->error_bits & AGPU_EBIT_CAPACITY) return AGPU_E_CAPACITY;
  return 0;
}

// ---- stretched transverse grids ------------------------------------------------
static StrAxis str_axis(const agpu_stretch_axis& a) {
  StrAxis s;
  s.cnst = a.cnst;
  s.smin = a.smin;
  s.smax = a.smax;
  s.xs = a.xs;
  s.dl_inv = a.dl_inv;
  s.dli_inv = a.dli_inv;
  s.ratio = a.ratio;
  s.nl_stretch = a.nl_stretch;
  s.init_cell = a.init_cell;
  s.n = (double)a.n;
  return s;
}

int agpu_set_stretch(agpu_handle* h, const agpu_stretch* st) {
  if (!h || !st) return AGPU_E_ARG;
  const agpu_params& p = h->p;
  if (int rc = agpu_synchronize(h)) return rc;
  if (!st->on) {
    h->str = false;
    return 0;
  }
  // FP64 form, quadratic shapes, the standard cycle; host-supplied records
  if (h->fp32 || p.ndim < 2 || p.shape != AGPU_SHAPE_QUADRATIC || p.iform == 2 || p.ionz_lev > 0 || h->env || h->dd ||
      p.w_speed < 0.0)
    return AGPU_E_ARG;
  for (int ic = 0; ic < 4; ++ic)
    if (h->has_src[ic]) return AGPU_E_STATE;
  if (st->y.n != p.ny || !st->y.d1 || !st->y.d1h) return AGPU_E_ARG;
  if (p.ndim == 3 && (st->z.n != p.nz || !st->z.d1 || !st->z.d1h)) return AGPU_E_ARG;
  const int ny = p.ny, nz = p.ndim == 3 ? p.nz : 0;
  const size_t nm = 2 * (size_t)(ny + 2) + (p.ndim == 3 ? 2 * (size_t)(nz + 2) : 0);
  if (!h->d_metric && dmalloc((void**)&h->d_metric, sizeof(double) * nm)) return AGPU_E_NOMEM;
  h->h_metric.assign(nm, 1.0);
  std::memcpy(h->h_metric.data(), st->y.d1, sizeof(double) * (ny + 2));
  std::memcpy(h->h_metric.data() + (ny + 2), st->y.d1h, sizeof(double) * (ny + 2));
  if (p.ndim == 3) {
    std::memcpy(h->h_metric.data() + 2 * (ny + 2), st->z.d1, sizeof(double) * (nz + 2));
    std::memcpy(h->h_metric.data() + 2 * (ny + 2) + (nz + 2), st->z.d1h, sizeof(double) * (nz + 2));
  }
  CK(cudaMemcpy(h->d_metric, st->y.d1, sizeof(double) * (ny + 2), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_metric + (ny + 2), st->y.d1h, sizeof(double) * (ny + 2), cudaMemcpyHostToDevice));
  if (p.ndim == 3) {
    CK(cudaMemcpy(h->d_metric + 2 * (ny + 2), st->z.d1, sizeof(double) * (nz + 2), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_metric + 2 * (ny + 2) + (nz + 2), st->z.d1h, sizeof(double) * (nz + 2), cudaMemcpyHostToDevice));
  }
  h->sy = str_axis(st->y);
  h->sz = p.ndim == 3 ? str_axis(st->z) : StrAxis{};
  // the Mur faces: loc_yg(1, 3), loc_yg(ny, 4), loc_zg(1, 3), loc_zg(nz, 4)
  h->by3 = st->y.d1[1];
  h->ty4 = st->y.d1h[ny];
  h->bz3 = p.ndim == 3 ? st->z.d1[1] : 1.0;
  h->tz4 = p.ndim == 3 ? st->z.d1h[nz] : 1.0;
  h->str = true;
  h->fused_yee = false;
  agpu_set_step_graphs(h, 0);
  for (int ic = 0; ic < 4; ++ic) h->binned[ic] = false;
  return 0;
}

// ---- domain decomposition in y ---------------------------------------------
int agpu_set_subdomain(agpu_handle* h, int32_t lo_shared, int32_t hi_shared, agpu_halo_fn fn, void* user) {
  const int32_t shared[4] = {lo_shared, hi_shared, 0, 0};
  return agpu_set_subdomain_yz(h, shared, fn, user);
}

int agpu_set_subdomain_yz(agpu_handle* h, const int32_t* shared, agpu_halo_fn fn, void* user) {
  if (!h || !shared) return AGPU_E_ARG;
  const agpu_params& p = h->p;
  const bool zs = shared[2] || shared[3];
  const bool any = shared[0] || shared[1] || zs;
  if (any) {
    // FP64 form, quadratic shapes, fixed frame, no envelope
    if (h->fp32 || p.shape != AGPU_SHAPE_QUADRATIC || p.w_speed < 0.0 || h->env || h->str) return AGPU_E_ARG;
    if (!fn) return AGPU_E_ARG;
    if ((shared[0] || shared[1]) && p.ny < 3) return AGPU_E_ARG;  // the exchanges move up to 3 rows
    if (zs && (p.ndim < 3 || p.nz < 3)) return AGPU_E_ARG;
  }
  if (int rc = agpu_synchronize(h)) return rc;
  h->dd = any;
  h->dd_lo = shared[0] ? 1 : 0;
  h->dd_hi = shared[1] ? 1 : 0;
  h->dd_zlo = shared[2] ? 1 : 0;
  h->dd_zhi = shared[3] ? 1 : 0;
  h->halo_fn = any ? fn : nullptr;
  h->halo_user = any ? user : nullptr;
  if (any) {
    // the exchanges run between the kernels of a step: plain launches only
    agpu_set_step_graphs(h, 0);
    h->fused_yee = false;
    for (int ic = 0; ic < 4; ++ic) h->binned[ic] = false;
  }
  return 0;
}

int agpu_halo_size(agpu_handle* h, int32_t ncomp, int32_t nrows, int64_t* n) {
  if (!h || !n || ncomp < 0 || nrows < 0) return AGPU_E_ARG;
  *n = (int64_t)ncomp * nrows * h->g.n1p * h->g.n3p;
  return 0;
}

static int halo_args(agpu_handle* h, int32_t what, int32_t ic1, int32_t ic2, int32_t j1, int32_t nrows, double** f) {
  if (!h || h->fp32 || (what != 0 && what != 1)) return AGPU_E_ARG;
  const int nmax = what == 0 ? h->g.nf : h->g.nc;
  if (ic1 < 1 || ic2 < ic1 || ic2 > nmax || nrows < 0 || j1 < 1 || j1 + nrows - 1 > h->g.n2p) return AGPU_E_ARG;
  *f = what == 0 ? h->ebf : h->jc;
  return 0;
}

static int halo_args_z(agpu_handle* h, int32_t what, int32_t ic1, int32_t ic2, int32_t k1, int32_t n, double** f) {
  if (!h || h->fp32 || h->p.ndim < 3 || (what != 0 && what != 1)) return AGPU_E_ARG;
  const int nmax = what == 0 ? h->g.nf : h->g.nc;
  if (ic1 < 1 || ic2 < ic1 || ic2 > nmax || n < 0 || k1 < 1 || k1 + n - 1 > h->g.n3p) return AGPU_E_ARG;
  *f = what == 0 ? h->ebf : h->jc;
  return 0;
}

int agpu_halo_size_z(agpu_handle* h, int32_t ncomp, int32_t nplanes, int64_t* n) {
  if (!h || !n || ncomp < 0 || nplanes < 0) return AGPU_E_ARG;
  *n = (int64_t)ncomp * nplanes * h->g.n1p * h->g.n2p;
  return 0;
}

int agpu_halo_pack_z(agpu_handle* h, int32_t what, int32_t ic1, int32_t ic2, int32_t k1, int32_t nplanes, double* buf) {
  double* f = nullptr;
  if (int rc = halo_args_z(h, what, ic1, ic2, k1, nplanes, &f)) return rc;
  if (!buf) return AGPU_E_ARG;
  halo_planes64(f, h->g, ic1 - 1, ic2 - ic1 + 1, k1, nplanes, buf, 0, h->st, h->sms);
  CK(cudaGetLastError());
  h->timers.launches_total += 1;
  return 0;
}

int agpu_halo_unpack_z(agpu_handle* h, int32_t what, int32_t ic1, int32_t ic2, int32_t k1, int32_t nplanes,
                       const double* buf, int32_t mode) {
  double* f = nullptr;
  if (int rc = halo_args_z(h, what, ic1, ic2, k1, nplanes, &f)) return rc;
  if (mode < 0 || mode > 2 || (mode < 2 && !buf)) return AGPU_E_ARG;
  halo_planes64(f, h->g, ic1 - 1, ic2 - ic1 + 1, k1, nplanes, const_cast<double*>(buf), mode + 1, h->st, h->sms);
  CK(cudaGetLastError());
  h->timers.launches_total += 1;
  return 0;
}

int agpu_halo_pack(agpu_handle* h, int32_t what, int32_t ic1, int32_t ic2, int32_t j1, int32_t nrows, double* buf) {
  double* f = nullptr;
  if (int rc = halo_args(h, what, ic1, ic2, j1, nrows, &f)) return rc;
  if (!buf) return AGPU_E_ARG;
  halo_rows64(f, h->g, ic1 - 1, ic2 - ic1 + 1, j1, nrows, buf, 0, h->st, h->sms);
  CK(cudaGetLastError());
  h->timers.launches_total += 1;
  return 0;
}

int agpu_halo_unpack(agpu_handle* h, int32_t what, int32_t ic1, int32_t ic2, int32_t j1, int32_t nrows,
                     const double* buf, int32_t mode) {
  double* f = nullptr;
  if (int rc = halo_args(h, what, ic1, ic2, j1, nrows, &f)) return rc;
  if (mode < 0 || mode > 2 || (mode < 2 && !buf)) return AGPU_E_ARG;
  halo_rows64(f, h->g, ic1 - 1, ic2 - ic1 + 1, j1, nrows, const_cast<double*>(buf), mode + 1, h->st, h->sms);
  CK(cudaGetLastError());
  h->timers.launches_total += 1;
  return 0;
}

int agpu_halo_emigrants(agpu_handle* h, int32_t ic, int32_t side, double* buf, int64_t ld, int64_t* n) {
  if (!h || h->fp32 || ic < 0 || ic >= h->p.nsp || side < 0 || side > 3 || (side > 1 && h->p.ndim < 3) || !n ||
      ld < 0 || (ld > 0 && !buf))
    return AGPU_E_ARG;
  *n = 0;
  if (h->np[ic] <= 0) return 0;
  const agpu_params& p = h->p;
  BoxBounds b{p.gxmin, p.gxmax, p.gymin, p.gymax, p.gzmin, p.gzmax, 1, p.ndim == 3 ? 1 : 0};
  long long cnt =
      emigrants64(h->part[ic], h->cap[ic], h->np[ic], h->ndv, b, side, h->dd_zlo, h->dd_zhi, buf, ld, h->scr, h->st);
  CK(cudaGetLastError());
  h->timers.launches_total += 3;
  *n = cnt;
  return cnt > ld ? AGPU_E_CAPACITY : 0;
}

int agpu_halo_immigrants(agpu_handle* h, int32_t ic, const double* buf, int64_t ld, int64_t n) {
  if (!h || h->fp32 || ic < 0 || ic >= h->p.nsp || n < 0 || (n > 0 && (!buf || ld < n))) return AGPU_E_ARG;
  if (n == 0) return 0;
  if (int rc = drop_removed(h, ic)) return rc;
  if (h->np[ic] + n > h->cap[ic]) {
    h->error_bits |= AGPU_EBIT_CAPACITY;
    return AGPU_E_CAPACITY;
  }
  CK(cudaMemcpy2DAsync(h->part[ic] + h->np[ic], sizeof(double) * h->cap[ic], buf, sizeof(double) * ld, sizeof(double) * n,
                       h->ndv, cudaMemcpyDeviceToDevice, h->st));
  h->np[ic] += n;
  h->nalive[ic] = h->np[ic];
  h->binned[ic] = false;
  return 0;
}

int agpu_window_inject(agpu_handle* h, int32_t ic, const double* part, int64_t ld, int64_t n, int32_t ndv) {
  if (!h || ic < 0 || ic >= h->p.nsp || ndv != h->ndv || n < 0 || (n > 0 && (!part || ld < n))) return AGPU_E_ARG;
  if (int rc = drop_removed(h, ic)) return rc;
  if (h->np[ic] + n > h->cap[ic]) return AGPU_E_CAPACITY;
  if (n == 0) return 0;
  if (!h->fp32) {
    CK(cudaMemcpy2DAsync(h->part[ic] + h->np[ic], sizeof(double) * h->cap[ic], part, sizeof(double) * ld, sizeof(double) * n,
                         ndv, cudaMemcpyHostToDevice, h->st));
  } else {
    // chunks of at most 2^20 records through a staging buffer kept in the
    // handle (allocated on the first call, grown up to the chunk size)
    const long long chunk_max = 1ll << 20;
    const long long chunk = n < chunk_max ? n : chunk_max;
    if (h->inj_stage_recs < chunk) {
      CK(cudaStreamSynchronize(h->st));
      cudaFree(h->inj_stage);
      h->inj_stage = nullptr;
      h->inj_stage_recs = 0;
      if (dmalloc((void**)&h->inj_stage, sizeof(double) * chunk * ndv)) return AGPU_E_NOMEM;
      h->inj_stage_recs = chunk;
    }
    for (long long q0 = 0; q0 < n; q0 += chunk) {
      const long long m = (n - q0) < chunk ? (n - q0) : chunk;
      CK(cudaMemcpy2DAsync(h->inj_stage, sizeof(double) * m, part + q0, sizeof(double) * ld, sizeof(double) * m, ndv,
                           cudaMemcpyHostToDevice, h->st));
      rec_to_split(h->inj_stage, m, m, h->sp[ic].view(), h->np[ic] + q0, h->g, h->p.xmn, h->p.ymn, h->p.zmn, h->p.dx_inv,
                   h->p.dy_inv, h->p.dz_inv, h->st, h->sms);
      CK(cudaGetLastError());
    }
  }
  CK(cudaStreamSynchronize(h->st));
  h->np[ic] += n;
  h->nalive[ic] = h->np[ic];
  h->binned[ic] = false;
  return 0;
}

// ---- envelope cycle (Env_cycle, src/ALaDyn.F90:111-130) -------------------
int agpu_env_enable(agpu_handle* h, const agpu_env_params* ep) {
  if (!h || !ep || h->fp32 || (ep->der_ord != 2 && ep->der_ord != 3) || !(ep->om0 > 0.0)) return AGPU_E_ARG;
  if (h->dd || h->str) return AGPU_E_STATE;  // the envelope cycle runs on one uniform box
  const Geo& g = h->g;
  if (g.ix2 - g.ix1 < 3 || g.jy2 - g.jy1 < 2 || (g.ndim == 3 && g.kz2 - g.kz1 < 2)) return AGPU_E_ARG;
  CK(cudaStreamSynchronize(h->st));
  cudaFree(h->env);
  cudaFree(h->env_av);
  cudaFree(h->env_den);
  h->env = h->env_av = h->env_den = nullptr;
  const size_t c3 = (size_t)g.ncell;
  int rc = dmalloc((void**)&h->env, sizeof(double) * c3 * 4);
  rc |= dmalloc((void**)&h->env_av, sizeof(double) * c3 * (g.ndim + 1));
  rc |= dmalloc((void**)&h->env_den, sizeof(double) * c3);
  if (rc) return AGPU_E_NOMEM;
  CK(cudaMemsetAsync(h->env, 0, sizeof(double) * c3 * 4, h->st));
  CK(cudaMemsetAsync(h->env_av, 0, sizeof(double) * c3 * (g.ndim + 1), h->st));
  CK(cudaStreamSynchronize(h->st));
  h->ep = *ep;
  return 0;
}

static int env_copy(agpu_handle* h, double* dev, const double* src_h, double* dst_h, int32_t n1p, int32_t n2p,
                    int32_t n3p, int32_t nc, int32_t want) {
  if (!h || !dev) return h ? AGPU_E_STATE : AGPU_E_ARG;
  const Geo& g = h->g;
  if (n1p != g.n1p || n2p != g.n2p || n3p != g.n3p || nc != want) return AGPU_E_ARG;
  const size_t bytes = sizeof(double) * (size_t)g.ncell * nc;
  if (src_h) CK(cudaMemcpyAsync(dev, src_h, bytes, cudaMemcpyHostToDevice, h->st));
  if (dst_h) CK(cudaMemcpyAsync(dst_h, dev, bytes, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return 0;
}
int agpu_set_envelope(agpu_handle* h, const double* env, int32_t n1p, int32_t n2p, int32_t n3p, int32_t nc) {
  if (!env) return AGPU_E_ARG;
  return env_copy(h, h ? h->env : nullptr, env, nullptr, n1p, n2p, n3p, nc, 4);
}
int agpu_get_envelope(agpu_handle* h, double* env, int32_t n1p, int32_t n2p, int32_t n3p, int32_t nc) {
  if (!env) return AGPU_E_ARG;
  return env_copy(h, h ? h->env : nullptr, nullptr, env, n1p, n2p, n3p, nc, 4);
}
int agpu_get_env_source(agpu_handle* h, double* av, int32_t n1p, int32_t n2p, int32_t n3p, int32_t nc) {
  if (!av) return AGPU_E_ARG;
  return env_copy(h, h ? h->env_av : nullptr, nullptr, av, n1p, n2p, n3p, nc, h ? h->p.ndim + 1 : 0);
}

int agpu_init_envelope(agpu_handle* h, const agpu_lp_pulse* l, int32_t plane_wave) {
  if (!h || !l || !(l->wx > 0.0) || !(l->wy > 0.0) || !(l->om0 > 0.0)) return AGPU_E_ARG;
  if (!h->env) return AGPU_E_STATE;
  EnvPulseArgs a;
  a.ndim = h->p.ndim;
  a.g_prof = l->g_prof ? 1 : 0;
  a.plane_wave = plane_wave ? 1 : 0;
  a.ee0 = l->ee0;
  a.t = l->t_loc - l->tf;
  a.tm = a.t - h->p.dt;
  a.xf0 = l->xf0;
  a.wx = l->wx;
  a.wy = l->wy;
  a.zra = 0.5 * l->om0 * l->wy * l->wy;
  a.ycent = l->ycent;
  a.zcent = l->zcent;
  a.xmn = h->p.xmn;
  a.ymn = h->p.ymn;
  a.zmn = h->p.zmn;
  a.dx = h->p.dx;
  a.dy = h->p.dy;
  a.dz = h->p.dz;
  env_init_pulse(a, h->env, h->g, h->st, h->sms);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

// env_run (src/dynamics/env_evolve_in_time.f90:363-391): env_lpf2_evolve
// (196-361) for species 0, then the moving window.
int agpu_env_run(agpu_handle* h, int32_t iter, double t, agpu_step_out* out) {
  if (!h) return AGPU_E_ARG;
  agpu_step_out dummy;
  if (!out) out = &dummy;
  std::memset(out, 0, sizeof(*out));
  out->ion_field_max = -1.0;
  if (!h->env) return AGPU_E_STATE;
  agpu_params& p = h->p;
  const Geo& g = h->g;
  const int ic = 0;
  if (int rc = drop_removed(h, ic)) return rc;
  CK(cudaMemsetAsync(h->d_cnt, 0, sizeof(Counters), h->st));
  // Every `every` calls the records move in memory along the tile
  // permutation (tile, row inside the tile, offset octant): a warp then
  // covers consecutive x cells of one tile row, so its stencil loads share
  // cache lines and its FP64 atomics mostly hit different addresses.  Not in
  // the deterministic mode, whose serial sums follow the particle order.
  const int every = h->sort_interval > 0 ? h->sort_interval : 8;
  if (!h->deterministic && h->key[ic] && h->np[ic] > 0 && h->env_steps % every == 0) {
    ph_begin(h, PH_SORT);
    if (int rc = rebin(h, ic)) return rc;
    if (int rc = reorder_records(h, ic)) return rc;
    ph_end(h, PH_SORT);
  }
  h->env_steps++;
  EnvArgs a;
  a.g = g;
  a.ebf = h->ebf;
  a.env = h->env;
  a.av = h->env_av;
  a.den = h->env_den;
  a.jc = h->jc;
  double* b = h->part[ic];
  const long long cp = h->cap[ic];
  a.x = b;
  a.y = b + cp;
  if (p.ndim == 3) {
    a.z = b + 2 * cp;
    a.px = b + 3 * cp;
    a.py = b + 4 * cp;
    a.pz = b + 5 * cp;
    a.slot = b + 6 * cp;
  } else {
    a.z = nullptr;
    a.px = b + 2 * cp;
    a.py = b + 3 * cp;
    a.pz = nullptr;
    a.slot = b + 4 * cp;
  }
  a.flag = h->flag;
  a.np = h->np[ic];
  a.xmn = p.xmn;
  a.ymn = p.ymn;
  a.zmn = p.zmn;
  a.dx_inv = p.dx_inv;
  a.dy_inv = p.dy_inv;
  a.dz_inv = p.dz_inv;
  a.dt = p.dt;
  a.lfact = p.lorentz_fact[ic];
  a.ompe = p.ompe;
  a.gxmin = p.gxmin;
  a.gxmax = p.gxmax;
  a.gymin = p.gymin;
  a.gymax = p.gymax;
  a.gzmin = p.gzmin;
  a.gzmax = p.gzmax;
  a.vdt = comoving_vdt(p);
  a.xtmp = h->xadv_tmp;
  a.om0 = h->ep.om0;
  a.opt_der1 = h->ep.opt_der1;
  a.hord_der2 = h->ep.hord_der2;
  a.der_ord = h->ep.der_ord;
  a.ibx = p.ibx;
  a.iby = p.iby;
  a.ibz = p.ibz;
  a.iform = p.iform;
  a.removed = &h->d_cnt->removed;
  a.err = &h->d_cnt->err;
  const size_t c3 = (size_t)g.ncell;
  ph_begin(h, PH_PUSH);
  // jc(:,:,:,:) = 0; env_amp_prepare
  CK(cudaMemsetAsync(h->env_av, 0, sizeof(double) * c3 * (g.ndim + 1), h->st));
  env_amp_grad(a, h->st, h->sms);
  // set_env_acc, lpf_env_momenta, set_env_density (jc(:,:,:,1) = 0 first)
  CK(cudaMemsetAsync(h->env_den, 0, sizeof(double) * c3, h->st));
  env_acc_momenta(a, h->st, h->sms, h->deterministic);
  // env_den_collect; jc(3) = jc(1)
  env_den_collect(a, h->st, h->sms);
  // advance_lpf_envelope, env_fields_average
  env_advance(a, h->st, h->sms);
  // set_env_grad_interp, lpf_env_positions, cell_part_dist, curr_accumulate
  CK(cudaMemsetAsync(h->jc, 0, sizeof(double) * c3 * g.nc, h->st));
  env_positions_deposit(a, h->st, h->sms, h->deterministic);
  CK(cudaGetLastError());
  ph_end(h, PH_PUSH);
  h->timers.launches_push_deposit += 2;
  h->timers.launches_total += 12 + (g.ndim == 3 ? 2 : 0) + (a.vdt > 0. ? 1 : 0);
  h->timers.pushes += a.np;
  if (int rc = read_counters(h)) return rc;
  int rc = 0;
  if (h->h_cnt->removed > 0) {
    ph_begin(h, PH_SORT);
    const long long before = h->np[ic];
    rc = compact_species(h, ic, false);
    ph_end(h, PH_SORT);
    if (rc) return rc;
    out->removed[ic] += before - h->np[ic];
  }
  // curr_mpi_collect (djc folded into the E update), advance_lpf_fields
  ph_begin(h, PH_YEE);
  Dev64 d{g, h->ebf, h->jc};
  jfold64(d, h->st, h->sms);
  yee64(d, yee_coef(p), h->st, h->sms, h->xadv.tmp ? &h->xadv : nullptr);
  CK(cudaGetLastError());
  ph_end(h, PH_YEE);
  h->timers.launches_yee += 1;
  h->timers.launches_total += ((p.ndim == 3) ? 3 : 2) + 6 + xadv_launches(h);
  h->timers.yee_cells += (long long)p.nx * p.ny * (p.ndim == 3 ? p.nz : 1);
  if ((rc = window_or_comoving(h, iter, t, out))) return rc;
  if (int rc_ = read_counters(h)) return rc_;
  for (int q = 0; q < 4; ++q) out->np[q] = h->binned[q] ? h->nalive[q] : h->np[q];
  out->xmn = p.xmn;
  out->error_bits = h->error_bits;
  if (h->error_bits & AGPU_EBIT_CAPACITY) return AGPU_E_CAPACITY;
  return 0;
}

// Geometry and constants of the bunch set-up; box lengths as set_grid
// computes them (set_grid_param.f90:102-108, 168-170, 221-223).
static BeamArgs beam_args(const agpu_handle* h, double gam2, double bet0) {
  const agpu_params& p = h->p;
  BeamArgs a;
  a.g = h->g;
  a.nx = p.nx;
  a.ny = p.ny;
  a.nz = p.ndim == 3 ? p.nz : 1;
  a.dx = p.dx;
  a.dy = p.dy;
  a.dz = p.dz;
  a.dx_inv = p.dx_inv;
  a.dy_inv = p.dy_inv;
  a.dz_inv = p.dz_inv;
  a.xmn = p.xmn;
  a.ymn = p.ymn;
  a.zmn = p.zmn;
  a.lx_box = p.xmax - p.xmn;
  a.ly_box = p.gymax - p.gymin;
  a.lz_box = p.gzmax - p.gzmin;
  a.ompe = p.ompe;
  a.gam2 = gam2;
  a.bet0 = bet0;
  return a;
}

int agpu_beam_potential(agpu_handle* h, const double* rho, double* pot, double gam2) {
  if (!h || !rho || !pot || !(gam2 >= 1.0) || !std::isfinite(gam2)) return AGPU_E_ARG;
  double* d = nullptr;
  const size_t n = (size_t)h->g.ncell;
  if (dmalloc((void**)&d, sizeof(double) * n)) return AGPU_E_NOMEM;
  int rc = 0;
  if (cudaMemcpyAsync(d, rho, sizeof(double) * n, cudaMemcpyHostToDevice, h->st) != cudaSuccess) rc = AGPU_E_CUDA;
  int launches = 0;
  if (!rc) rc = beam_potential(beam_args(h, gam2, 0.0), d, h->st, h->sms, &launches);
  if (!rc && cudaMemcpyAsync(pot, d, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st) != cudaSuccess) rc = AGPU_E_CUDA;
  if (cudaStreamSynchronize(h->st) != cudaSuccess && !rc) rc = AGPU_E_CUDA;
  cudaFree(d);
  h->timers.launches_total += launches;
  return rc;
}

int agpu_beam_inject(agpu_handle* h, int32_t ic, const double* part, int64_t ld, int64_t nb_tot, int32_t ndv,
                     double gam0) {
  if (!h || ic < 0 || ic >= h->p.nsp || ndv != h->ndv || nb_tot < 0 || (nb_tot > 0 && (!part || ld < nb_tot)) ||
      !(gam0 >= 1.0) || !std::isfinite(gam0))
    return AGPU_E_ARG;
  if (int rc = drop_removed(h, ic)) return rc;
  const Geo& g = h->g;
  const agpu_params& p = h->p;
  const long long ldb = nb_tot > 0 ? nb_tot : 1;
  double* stage = nullptr;  // the records as passed
  double* sel = nullptr;    // the records inside the box, in order
  double* pot = nullptr;    // split form: FP64 potential pair (the FP64 form uses jc(1:2))
  int rc = 0;
  if (dmalloc((void**)&stage, sizeof(double) * (size_t)ldb * ndv) ||
      dmalloc((void**)&sel, sizeof(double) * (size_t)ldb * ndv) ||
      (h->fp32 && dmalloc((void**)&pot, sizeof(double) * (size_t)g.ncell * 2)))
    rc = AGPU_E_NOMEM;
  int launches = 0;
  long long nb = 0;
  if (!rc && cudaMemsetAsync(h->d_cnt, 0, sizeof(Counters), h->st) != cudaSuccess) rc = AGPU_E_CUDA;
  if (!rc && nb_tot > 0) {
    if (cudaMemcpy2DAsync(stage, sizeof(double) * ldb, part, sizeof(double) * ld, sizeof(double) * nb_tot, ndv,
                          cudaMemcpyHostToDevice, h->st) != cudaSuccess)
      rc = AGPU_E_CUDA;
    // mpi_beam_distribute (init_beam_part_distrib.f90:273-438): the records
    // with x1 < x <= x2, y1 < y <= y2 (and z1 < z <= z2), in order
    if (!rc) {
      BoxBounds b{p.gxmin, p.gxmax, p.gymin, p.gymax, p.gzmin, p.gzmax, 1, p.ndim == 3 ? 1 : 0};
      nb = compact64(stage, sel, ldb, nb_tot, ndv, b, h->scr, h->st);
      launches += 3;
      if (cudaGetLastError() != cudaSuccess) rc = AGPU_E_CUDA;
    }
  }
  if (!rc && h->np[ic] + nb > h->cap[ic]) rc = AGPU_E_CAPACITY;
  // spec(1)%part grows by the bunch records (beam_inject 508-535)
  if (!rc && nb > 0) {
    if (!h->fp32) {
      if (cudaMemcpy2DAsync(h->part[ic] + h->np[ic], sizeof(double) * h->cap[ic], sel, sizeof(double) * ldb,
                            sizeof(double) * nb, ndv, cudaMemcpyDeviceToDevice, h->st) != cudaSuccess)
        rc = AGPU_E_CUDA;
    } else {
      rec_to_split(sel, ldb, nb, h->sp[ic].view(), h->np[ic], g, p.xmn, p.ymn, p.zmn, p.dx_inv, p.dy_inv, p.dz_inv, h->st,
                   h->sms);
      launches += 1;
    }
  }
  // jc(:,:,:,1) = 0; set_grid_charge; fft_3d_psolv / fft_2d_psolv;
  // jc(:,:,:,2) = bet0 jc(:,:,:,1); initial_beam_fields; ebf += ebf_bunch
  const double gam2 = gam0 * gam0;
  const double u0_b = std::sqrt(gam0 * gam0 - 1.);  // set_init_param.f90:353-354
  const double bet0 = u0_b / gam0;
  const BeamArgs a = beam_args(h, gam2, bet0);
  double* p1 = h->fp32 ? pot : h->jc;
  double* p2 = p1 ? p1 + g.ncell : nullptr;
  if (!rc && cudaMemsetAsync(p1, 0, sizeof(double) * g.ncell, h->st) != cudaSuccess) rc = AGPU_E_CUDA;
  if (!rc) {
    beam_charge(a, sel, ldb, nb, p1, &h->d_cnt->err, h->st, h->sms);
    launches += nb > 0 ? 1 : 0;
    if (cudaGetLastError() != cudaSuccess) rc = AGPU_E_CUDA;
  }
  if (!rc) rc = beam_potential(a, p1, h->st, h->sms, &launches);
  if (!rc) {
    beam_fields(a, p1, p2, h->fp32 ? nullptr : h->ebf, h->fp32 ? h->ebf32 : nullptr, h->st, h->sms, &launches);
    if (cudaGetLastError() != cudaSuccess) rc = AGPU_E_CUDA;
  }
  if (cudaStreamSynchronize(h->st) != cudaSuccess && !rc) rc = AGPU_E_CUDA;
  cudaFree(stage);
  cudaFree(sel);
  cudaFree(pot);
  h->timers.launches_total += launches;
  if (rc) return rc;
  if (int rc_ = read_counters(h)) return rc_;
  h->np[ic] += nb;
  h->nalive[ic] = h->np[ic];
  h->binned[ic] = false;
  h->fields_set = true;
  if (h->h_cnt->err & AGPU_EBIT_INDEX) return AGPU_E_INDEX;
  return 0;
}

int agpu_diag(agpu_handle* h, agpu_diag_out* out) {
  if (!h || !out) return AGPU_E_ARG;
  std::memset(out, 0, sizeof(*out));
  // removed records of a binned species stay stored until the next
  // compaction: the particle sums leave them out (by their binning key in the
  // split form, in memory order; along the tile permutation in the FP64
  // form) instead of compacting (a full copy and a rebinning)
  if (int rc = refresh_counts(h)) return rc;
  CK(cudaMemsetAsync(h->d_diag, 0, sizeof(double) * 64, h->st));
  double dvol = h->p.dx * h->p.dy * (h->p.ndim == 3 ? h->p.dz : 1.0);
  if (h->fp32)
    field_diag32(h->ebf32, h->g, dvol, h->d_diag, h->d_diag + 6, h->st, h->sms);
  else
    field_diag64(h->ebf, h->g, dvol, h->d_diag, h->d_diag + 6, h->st, h->sms);
  long long nd_alive[4] = {0, 0, 0, 0};
  for (int ic = 0; ic < h->p.nsp; ++ic) {
    double* o = h->d_diag + 8 + 5 * ic;
    const bool along = h->binned[ic] && h->nalive[ic] < h->np[ic];
    const int* perm = along ? h->perm[ic] : nullptr;
    const long long n = along ? h->nalive[ic] : h->np[ic];
    nd_alive[ic] = n;
    if (h->fp32)
      part_diag32(h->sp[ic].view(), along ? h->np[ic] : n, h->p.ndim, along ? h->key[ic] : nullptr, h->tg.nkeys, o,
                  h->st, h->sms);
    else
      part_diag64(h->part[ic], h->cap[ic], n, h->p.ndim, perm, o, h->st, h->sms);
  }
  CK(cudaGetLastError());
  double hd[64];
  CK(cudaMemcpyAsync(hd, h->d_diag, sizeof(hd), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  for (int c = 0; c < 6; ++c) out->field_energy[c] = hd[c];
  out->max_abs_e = hd[6];
  for (int ic = 0; ic < 4; ++ic) {
    const double* o = hd + 8 + 5 * ic;
    out->kin_energy[ic] = o[0];
    out->charge[ic] = o[1];
    for (int c = 0; c < 3; ++c) out->momentum[ic][c] = o[2 + c];
    out->np[ic] = nd_alive[ic];
  }
  return 0;
}

int agpu_envar_species(agpu_handle* h, int32_t ic, double pmass, agpu_envar_out* out) {
  if (!h || !out || ic < 0 || ic >= h->p.nsp) return AGPU_E_ARG;
  std::memset(out, 0, sizeof(*out));
  if (int rc = refresh_counts(h)) return rc;
  CK(cudaMemsetAsync(h->d_envar, 0, sizeof(double) * (16 + AGPU_NE), h->st));
  const bool along = h->binned[ic] && h->nalive[ic] < h->np[ic];
  const int* perm = along ? h->perm[ic] : nullptr;
  const long long n = along ? h->nalive[ic] : h->np[ic];
  if (h->fp32) {
    const Part32View v = h->sp[ic].view();
    envar_species(nullptr, 0, &v, perm, n, h->g, h->p.ymn, h->p.zmn, h->p.dy, h->p.dz, pmass, h->d_envar, h->st, h->sms);
  } else {
    envar_species(h->part[ic], h->cap[ic], nullptr, perm, n, h->g, h->p.ymn, h->p.zmn, h->p.dy, h->p.dz, pmass,
                  h->d_envar, h->st, h->sms);
  }
  CK(cudaGetLastError());
  double hd[16 + AGPU_NE];
  CK(cudaMemcpyAsync(hd, h->d_envar, sizeof(hd), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  out->np = n;
  for (int c = 0; c < 7; ++c) out->ek[c] = hd[c];
  out->ekmax = hd[7];
  for (int c = 0; c < 3; ++c) out->psig[c] = hd[8 + c];
  for (int b = 0; b < AGPU_NE; ++b) out->nde[b] = hd[16 + b];
  return 0;
}

int agpu_envar_fields(agpu_handle* h, agpu_envar_fields_out* out) {
  if (!h || !out) return AGPU_E_ARG;
  std::memset(out, 0, sizeof(*out));
  CK(cudaMemsetAsync(h->d_envar, 0, sizeof(double) * 16, h->st));
  if (h->fp32)
    envar_fields32(h->ebf32, h->g, h->d_envar, h->st, h->sms);
  else
    envar_fields64(h->ebf, h->g, h->d_envar, h->st, h->sms);
  CK(cudaGetLastError());
  double hd[16];
  CK(cudaMemcpyAsync(hd, h->d_envar, sizeof(hd), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  // Envar: ekt(1:nfield) = dgvol * sum, dgvol = dx dy dz (2D dx dy dy)
  const double dgvol = (h->p.ndim == 2) ? h->p.dx * h->p.dy * h->p.dy : h->p.dx * h->p.dy * h->p.dz;
  for (int c = 0; c < h->g.nf; ++c) {
    out->energy[c] = dgvol * hd[c];
    out->fmax[c] = hd[6 + c];
  }
  out->e2max = hd[12];
  return 0;
}

int agpu_set_profiling(agpu_handle* h, int32_t on) {
  if (!h) return AGPU_E_ARG;
  h->profiling = on != 0;
  return 0;
}
int agpu_get_timers(agpu_handle* h, agpu_timers* out) {
  if (!h || !out) return AGPU_E_ARG;
  *out = h->timers;
  return 0;
}
int agpu_reset_timers(agpu_handle* h) {
  if (!h) return AGPU_E_ARG;
  std::memset(&h->timers, 0, sizeof(h->timers));
  return 0;
}
int agpu_get_stream(agpu_handle* h, void** stream) {
  if (!h || !stream) return AGPU_E_ARG;
  *stream = (void*)h->st;
  return 0;
}
int agpu_synchronize(agpu_handle* h) {
  if (!h) return AGPU_E_ARG;
  if (int rc = refresh_counts(h)) return rc;
  CK(cudaStreamSynchronize(h->st));
  return 0;
}
int agpu_set_deferred_counts(agpu_handle* h, int32_t on) {
  if (!h) return AGPU_E_ARG;
  if (!on)
    if (int rc = refresh_counts(h)) return rc;
  h->defer = on != 0;
  return 0;
}
int agpu_set_sort_interval(agpu_handle* h, int32_t steps) {
  if (!h || steps < 0) return AGPU_E_ARG;
  h->sort_interval = steps;
  return 0;
}
int agpu_set_fused_yee(agpu_handle* h, int32_t on) {
  if (!h) return AGPU_E_ARG;
  if (on && (h->dd || h->str)) return AGPU_E_STATE;
  h->fused_yee = on != 0;
  return 0;
}

int agpu_set_deterministic(agpu_handle* h, int32_t on) {
  if (!h) return AGPU_E_ARG;
  // the per-particle FP32 kernel has the quadratic shapes only
  if (on && h->fp32 && h->p.shape == AGPU_SHAPE_CUBIC) return AGPU_E_ARG;
  h->deterministic = on != 0;
  return 0;
}

}  // extern "C"
