// agpu_batch.cpp — batched instances for parameter scans: N independent
// simulations (their own grids, lasers and plasmas) advanced together on one
// GPU.  The reference runs a scan as N separate jobs, one after the other;
// here every instance keeps its own handle and CUDA stream, worker threads
// each drive a share of the instances, and the steps between window shifts
// run in deferred-count mode, so each worker queues the next instance's step
// without waiting for the GPU and the kernels of different instances overlap
// on the SMs.
//
// Only the public C-ABI of include/aladyn_gpu.h is used (plus cudaSetDevice
// so that the workers use the device the batch was created on).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <new>
#include <thread>
#include <vector>

#include "../../include/aladyn_gpu.h"

struct agpu_batch {
  int device = 0;
  std::vector<agpu_handle*> h;
  std::vector<agpu_params> p;
  std::vector<int32_t> iter;
  std::vector<double> t;
  std::vector<int32_t> status;
};

extern "C" {

int agpu_batch_create(const agpu_params* params, int32_t n, agpu_batch** out) {
  if (!params || !out || n < 1) return AGPU_E_ARG;
  *out = nullptr;
  agpu_batch* b = new (std::nothrow) agpu_batch();
  if (!b) return AGPU_E_NOMEM;
  cudaGetDevice(&b->device);
  b->h.assign(n, nullptr);
  b->p.assign(params, params + n);
  b->iter.assign(n, 0);
  b->t.assign(n, 0.0);
  b->status.assign(n, 0);
  for (int i = 0; i < n; ++i) {
    int rc = agpu_create(&params[i], &b->h[i]);
    if (rc) {
      for (int j = 0; j < i; ++j) agpu_destroy(b->h[j]);
      delete b;
      return rc;
    }
  }
  *out = b;
  return 0;
}

int agpu_batch_destroy(agpu_batch* b) {
  if (!b) return AGPU_E_ARG;
  for (agpu_handle* h : b->h)
    if (h) agpu_destroy(h);
  delete b;
  return 0;
}

int agpu_batch_size(const agpu_batch* b, int32_t* n) {
  if (!b || !n) return AGPU_E_ARG;
  *n = (int32_t)b->h.size();
  return 0;
}

int agpu_batch_handle(agpu_batch* b, int32_t i, agpu_handle** h) {
  if (!b || !h || i < 0 || i >= (int32_t)b->h.size()) return AGPU_E_ARG;
  *h = b->h[i];
  return 0;
}

int agpu_batch_clock(const agpu_batch* b, int32_t i, int32_t* iter, double* t) {
  if (!b || i < 0 || i >= (int32_t)b->h.size()) return AGPU_E_ARG;
  if (iter) *iter = b->iter[i];
  if (t) *t = b->t[i];
  return 0;
}

int agpu_batch_run(agpu_batch* b, int32_t nsteps, int32_t nthreads, int32_t* status) {
  if (!b || nsteps < 0) return AGPU_E_ARG;
  const int n = (int)b->h.size();
  int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
  nt = std::min(nt, n);
  auto work = [b, n, nt, nsteps](int w) {
    cudaSetDevice(b->device);
    std::vector<int> mine;
    for (int i = w; i < n; i += nt) mine.push_back(i);
    for (int i : mine)
      if (!b->status[i]) b->status[i] = agpu_set_deferred_counts(b->h[i], 1);
    // step s of every instance of this worker, then step s+1: the instances
    // interleave on the GPU; only window shifts wait for their own stream
    for (int s = 0; s < nsteps; ++s)
      for (int i : mine) {
        if (b->status[i]) continue;
        agpu_step_out out;
        int rc = agpu_step(b->h[i], b->iter[i], b->t[i], b->iter[i] == 0 ? 1 : 0, &out);
        if (rc) {
          b->status[i] = rc;
          continue;
        }
        b->t[i] += b->p[i].dt;
        b->iter[i] += 1;
      }
    for (int i : mine) {
      int rc = agpu_synchronize(b->h[i]);
      if (!b->status[i]) b->status[i] = rc;
    }
  };
  std::vector<std::thread> pool;
  pool.reserve(nt);
  for (int w = 0; w < nt; ++w) pool.emplace_back(work, w);
  for (auto& th : pool) th.join();
  int first = 0;
  for (int i = 0; i < n; ++i) {
    if (status) status[i] = b->status[i];
    if (!first && b->status[i]) first = b->status[i];
  }
  return first;
}

}  // extern "C"
