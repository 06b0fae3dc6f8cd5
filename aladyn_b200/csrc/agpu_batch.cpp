// agpu_batch.cpp — batched instances for parameter scans: N independent
// simulations (their own grids, lasers and plasmas) advanced together on one
// GPU.  The reference runs a scan as N separate jobs, one after the other;
// here every instance keeps its own handle and CUDA stream, worker threads
// each drive a share of the instances, and the steps between window shifts
// run in deferred-count mode, so each worker queues the next instance's step
// without waiting for the GPU and the kernels of different instances overlap
// on the SMs.
//
// By default the steps between window shifts of all instances run as one
// multi-instance step: one kernel per phase for every instance together
// (agpu_x_step_many), about 15 launches per batch step instead of ~17 per
// instance; first steps and window shifts run per instance on the workers.
// With that off, each worker steps its instances on their own streams
// (optionally from per-instance CUDA graphs).
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

// Multi-instance steps (agpu_api.cu, not part of the public header): the
// plain steps of many instances as one launch per phase.
struct agpu_x_ws;
extern "C" {
int agpu_x_plain(agpu_handle* h, int32_t iter, double t, int32_t initial_time);
int agpu_x_ws_create(int32_t maxn, agpu_x_ws** out);
int agpu_x_ws_destroy(agpu_x_ws* w);
long long agpu_x_ws_launches(const agpu_x_ws* w);
int agpu_x_step_many(agpu_handle** hs, int32_t n, agpu_x_ws* w);
}

struct agpu_batch {
  int device = 0;
  std::vector<agpu_handle*> h;
  std::vector<agpu_params> p;
  std::vector<int32_t> iter;
  std::vector<double> t;
  std::vector<int32_t> status;
  bool graphs = true;
  bool multi = true;
  agpu_x_ws* ws = nullptr;
};

// Runs fn(i) for every i of idx on up to nt worker threads (each on the
// batch's device).
template <typename F>
static void parallel_for(const std::vector<int>& idx, int nt, int device, F fn) {
  if (idx.empty()) return;
  nt = std::max(1, std::min<int>(nt, (int)idx.size()));
  std::atomic<size_t> next{0};
  auto work = [&]() {
    cudaSetDevice(device);
    for (size_t k = next++; k < idx.size(); k = next++) fn(idx[k]);
  };
  std::vector<std::thread> pool;
  for (int w = 1; w < nt; ++w) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
}

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
  if (b->ws) agpu_x_ws_destroy(b->ws);
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

int agpu_batch_set_graphs(agpu_batch* b, int32_t on) {
  if (!b) return AGPU_E_ARG;
  b->graphs = on != 0;
  for (agpu_handle* h : b->h) agpu_set_step_graphs(h, b->graphs ? 1 : 0);
  return 0;
}

int agpu_batch_set_multi(agpu_batch* b, int32_t on) {
  if (!b) return AGPU_E_ARG;
  b->multi = on != 0;
  return 0;
}

int agpu_batch_launches(const agpu_batch* b, int64_t* n) {
  if (!b || !n) return AGPU_E_ARG;
  *n = agpu_x_ws_launches(b->ws);
  return 0;
}

int agpu_batch_run(agpu_batch* b, int32_t nsteps, int32_t nthreads, int32_t* status) {
  if (!b || nsteps < 0) return AGPU_E_ARG;
  cudaSetDevice(b->device);
  const int n = (int)b->h.size();
  int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
  nt = std::min(nt, n);
  for (int i = 0; i < n; ++i) {
    if (!b->status[i]) b->status[i] = agpu_set_deferred_counts(b->h[i], 1);
    if (!b->status[i]) b->status[i] = agpu_set_step_graphs(b->h[i], (b->graphs && !b->multi) ? 1 : 0);
  }
  if (b->multi && !b->ws && agpu_x_ws_create(n, &b->ws) != 0) b->multi = false;
  if (b->multi) {
    // the multi-instance steps run on the workspace's stream and read every
    // instance's buffers: let work the host queued on the instances' own
    // streams before this call (set-up, injection, diagnostics) finish first
    for (int i = 0; i < n; ++i) {
      int rc = agpu_synchronize(b->h[i]);
      if (rc && !b->status[i]) b->status[i] = rc;
    }
  }
  auto step_one = [b](int i) {
    int rc = agpu_step(b->h[i], b->iter[i], b->t[i], b->iter[i] == 0 ? 1 : 0, nullptr);
    if (rc) {
      b->status[i] = rc;
      return;
    }
    b->t[i] += b->p[i].dt;
    b->iter[i] += 1;
  };
  std::vector<int> all;
  for (int i = 0; i < n; ++i) all.push_back(i);
  if (!b->multi) {
    // every instance on its own stream: each worker queues step s of its
    // instances, then step s+1, so the instances interleave on the GPU
    std::vector<std::thread> pool;
    for (int w = 0; w < nt; ++w)
      pool.emplace_back([&, w]() {
        cudaSetDevice(b->device);
        for (int s = 0; s < nsteps; ++s)
          for (int i = w; i < n; i += nt)
            if (!b->status[i]) step_one(i);
      });
    for (auto& th : pool) th.join();
  } else {
    std::vector<int> special;
    std::vector<agpu_handle*> plain_h;
    std::vector<int> plain_i;
    for (int s = 0; s < nsteps; ++s) {
      special.clear();
      plain_h.clear();
      plain_i.clear();
      for (int i = 0; i < n; ++i) {
        if (b->status[i]) continue;
        if (agpu_x_plain(b->h[i], b->iter[i], b->t[i], b->iter[i] == 0 ? 1 : 0) && b->p[i].ndim == b->p[0].ndim) {
          plain_h.push_back(b->h[i]);
          plain_i.push_back(i);
        } else {
          special.push_back(i);
        }
      }
      // first steps, window shifts and other non-plain steps: one instance
      // per worker at a time, each left idle for the multi-instance step
      parallel_for(special, nt, b->device, [&](int i) {
        step_one(i);
        int rc = agpu_synchronize(b->h[i]);
        if (rc && !b->status[i]) b->status[i] = rc;
      });
      if (!plain_h.empty()) {
        int rc = agpu_x_step_many(plain_h.data(), (int32_t)plain_h.size(), b->ws);
        for (int i : plain_i) {
          if (rc) {
            b->status[i] = rc;
            continue;
          }
          b->t[i] += b->p[i].dt;
          b->iter[i] += 1;
        }
      }
    }
  }
  parallel_for(all, nt, b->device, [&](int i) {
    int rc = agpu_synchronize(b->h[i]);
    if (!b->status[i]) b->status[i] = rc;
  });
  int first = 0;
  for (int i = 0; i < n; ++i) {
    if (status) status[i] = b->status[i];
    if (!first && b->status[i]) first = b->status[i];
  }
  return first;
}

}  // extern "C"
