// agpu_noalloc.cu — field-energy diagnostics that allocate no device memory.
//
// Some hosts cannot call cudaMalloc: a host that runs inside a CUDA stream
// capture (allocation is not a capturable operation), a host whose device
// memory is handed out by an external pool (a Fortran driver that owns one
// big arena, a framework with its own caching allocator), or a host that must
// not change the device's memory footprint while it runs.  This entry point
// computes what agpu_diag reports for the fields -- sum of F^2 dV per
// component over the interior and max |E| -- from a field array the caller
// already has on the device, into an output the caller provides, with its
// scratch (one partial sum per block) in a file-scope device array.
//
// The scratch array is shared by every call in the process and keeps the
// last call's contents: each call overwrites the partials it later reads,
// so nothing has to start at zero.  Calls that overlap on the GPU (two
// streams, two host threads) race on it; serialise them.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/aladyn_gpu.h"
#include "agpu_common.cuh"

namespace {

constexpr int NA_BLOCK = 256;
constexpr int NA_ITEMS = 16;                          // cells per thread
constexpr long long NA_CELLS_PER_BLOCK = NA_BLOCK * NA_ITEMS;
constexpr int NA_MAX_BLOCKS = 65536;                  // 2^28 interior cells at most
constexpr int NA_SLOTS = 8;                           // 6 energies, max |E|, pad

// 65536 blocks x 8 doubles = 4 MiB, held by every GPU that loads the library
static __device__ __align__(256) double g_na_partials[NA_MAX_BLOCKS * NA_SLOTS];

// The array's device address belongs to the module instance loaded into one
// CUDA context: a device reset, or a host that drives the device through a
// context of its own, loads the module again at another address.  The cache
// is therefore keyed on (device, context), and every call made outside a
// stream capture looks the address up again (cheap), so a stale entry can
// only be used by a capture that starts before any plain call in a new
// context.  The driver's cuCtxGetCurrent is reached through the runtime's
// entry-point query, so the library does not link libcuda itself.
constexpr int NA_CACHE = 64;
struct NaEntry {
  int dev;
  void* ctx;
  double* ptr;
};
std::mutex g_na_mu;
NaEntry g_na_cache[NA_CACHE] = {};
int g_na_used = 0;
typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn g_ctx_get = nullptr;
bool g_ctx_tried = false;

void* na_current_context() {
  if (!g_ctx_tried) {
    g_ctx_tried = true;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get = reinterpret_cast<CtxGetCurrentFn>(fn);
    else
      cudaGetLastError();
  }
  void* ctx = nullptr;
  if (!g_ctx_get || g_ctx_get(&ctx) != 0) return nullptr;
  return ctx;
}

// Device address of the scratch array in the current context.
int na_scratch(cudaStream_t st, double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return AGPU_E_NODEVICE;
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
    cudaGetLastError();
    return AGPU_E_CUDA;
  }
  std::lock_guard<std::mutex> lk(g_na_mu);
  void* ctx = na_current_context();
  int slot = -1;
  for (int i = 0; i < g_na_used; ++i)
    if (g_na_cache[i].dev == dev && g_na_cache[i].ctx == ctx) slot = i;
  if (slot >= 0 && cap != cudaStreamCaptureStatusNone) {
    *out = g_na_cache[slot].ptr;
    return 0;
  }
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_na_partials);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    return AGPU_E_CUDA;
  }
  if (!ctx) ctx = na_current_context();  // the lookup made the primary context current
  if (slot < 0) {
    for (int i = 0; i < g_na_used; ++i)
      if (g_na_cache[i].dev == dev && g_na_cache[i].ctx == ctx) slot = i;
  }
  if (slot < 0) {
    slot = (g_na_used < NA_CACHE) ? g_na_used++ : (int)(((uintptr_t)ctx >> 4) % NA_CACHE);
    g_na_cache[slot].dev = dev;
    g_na_cache[slot].ctx = ctx;
  }
  g_na_cache[slot].ptr = static_cast<double*>(p);
  *out = g_na_cache[slot].ptr;
  return 0;
}

// One partial per block: sum of F_c^2 over the block's interior cells for
// every component c and max |E_c| over the electric components.
__global__ void __launch_bounds__(NA_BLOCK) k_na_partial(const double* __restrict__ ebf, Geo g, long long ncells,
                                                         double* partials) {
  __shared__ double red[NA_SLOTS][NA_BLOCK / 32];
  const int nx = g.ix2 - g.ix1 + 1, ny = g.jy2 - g.jy1 + 1;
  const int ne = (g.nf == 6) ? 3 : 2;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  long long base = (long long)blockIdx.x * NA_CELLS_PER_BLOCK;
  for (int it = 0; it < NA_ITEMS; ++it) {
    long long t = base + (long long)it * NA_BLOCK + threadIdx.x;
    if (t >= ncells) break;
    int i = g.ix1 + (int)(t % nx);
    int j = g.jy1 + (int)((t / nx) % ny);
    int k = g.kz1 + (int)(t / ((long long)nx * ny));
    long long o = goff(g, i, j, k);
    for (int c = 0; c < g.nf; ++c) {
      double v = ebf[g.ncell * c + o];
      acc[c] += v * v;
      if (c < ne) acc[6] = fmax(acc[6], fabs(v));
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int s = 0; s < 7; ++s) {
    double v = acc[s];
    for (int off = 16; off > 0; off >>= 1) {
      double w = __shfl_down_sync(0xffffffffu, v, off);
      v = (s == 6) ? fmax(v, w) : v + w;
    }
    if (lane == 0) red[s][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    int s = threadIdx.x;
    double v = red[s][0];
    for (int w = 1; w < NA_BLOCK / 32; ++w) v = (s == 6) ? fmax(v, red[s][w]) : v + red[s][w];
    partials[(long long)blockIdx.x * NA_SLOTS + s] = v;
  }
}

// Fixed-order reduction of the nb partials into out[0..6].
__global__ void __launch_bounds__(NA_BLOCK) k_na_final(const double* partials, int nb, int nf, double dvol, double* out) {
  __shared__ double red[NA_BLOCK];
  for (int s = 0; s < 7; ++s) {
    double v = 0.0;
    for (int b = threadIdx.x; b < nb; b += NA_BLOCK) {
      double w = partials[(long long)b * NA_SLOTS + s];
      v = (s == 6) ? fmax(v, w) : v + w;
    }
    red[threadIdx.x] = v;
    __syncthreads();
    for (int h = NA_BLOCK / 2; h > 0; h >>= 1) {
      if (threadIdx.x < h) red[threadIdx.x] = (s == 6) ? fmax(red[threadIdx.x], red[threadIdx.x + h])
                                                         : red[threadIdx.x] + red[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[s] = (s == 6) ? red[0] : ((s < nf) ? red[0] * dvol : 0.0);
    __syncthreads();
  }
}

}  // namespace

extern "C" int agpu_field_diag_noalloc(const double* d_ebf, int32_t ndim, int32_t nx, int32_t ny, int32_t nz, double dx,
                                       double dy, double dz, double* d_out, void* stream) {
  if (!d_ebf || !d_out) return AGPU_E_ARG;
  if (!(ndim == 2 || ndim == 3) || nx < 1 || ny < 1 || (ndim == 3 && nz < 1)) return AGPU_E_ARG;
  Geo g;
  g.ndim = ndim;
  g.n1p = nx + 5;
  g.n2p = ny + 5;
  g.n3p = (ndim == 3) ? nz + 5 : 1;
  g.ix1 = 3;
  g.ix2 = nx + 2;
  g.jy1 = 3;
  g.jy2 = ny + 2;
  g.kz1 = (ndim == 3) ? 3 : 1;
  g.kz2 = (ndim == 3) ? nz + 2 : 1;
  g.nf = (ndim == 3) ? 6 : 3;
  g.nc = (ndim == 3) ? 3 : 2;
  g.ncell = (long long)g.n1p * g.n2p * g.n3p;
  geo_divisors(g);
  const long long ncells = (long long)nx * ny * (ndim == 3 ? nz : 1);
  const long long nb = (ncells + NA_CELLS_PER_BLOCK - 1) / NA_CELLS_PER_BLOCK;
  if (nb > NA_MAX_BLOCKS) return AGPU_E_CAPACITY;  // more than 2^28 interior cells
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* partials = nullptr;
  if (int rc = na_scratch(st, &partials)) return rc;
  const double dvol = dx * dy * (ndim == 3 ? dz : 1.0);
  k_na_partial<<<(unsigned)nb, NA_BLOCK, 0, st>>>(d_ebf, g, ncells, partials);
  k_na_final<<<1, NA_BLOCK, 0, st>>>(partials, (int)nb, g.nf, dvol, d_out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? AGPU_OK : AGPU_E_CUDA;
}
