// Batches of independent boxes (a batch of contexts stepped together).
//
// The reference runs one box per process (test.cpp:16-80) and has no batched entry
// point.  A batch is one context per box, each with its own CUDA stream.  apc_batch_step
// hands the boxes to host worker threads through a shared queue ordered largest box
// first (longest-processing-time order), and each worker runs the box's ordinary
// apc_step.  The boxes' kernels then run concurrently on the GPU: the many small grids
// of a 16^3 box leave most SMs idle, and other boxes fill them.  Every box runs the
// single-context code path, so its results are exactly those of a lone context.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <new>
#include <thread>
#include <vector>

#include "apc_internal.cuh"

struct apc_batch {
  std::vector<apc_context *> ctx;
  std::vector<int> order;  // boxes by decreasing particle count
  int workers = 1;
};

extern "C" {

int apc_batch_create(const apc_config *cfgs, int n_boxes, int n_workers, apc_batch **out) {
  if (!out) return APC_ERR_INVALID_ARG;
  *out = nullptr;
  if (!cfgs || n_boxes <= 0 || n_workers < 0) return APC_ERR_INVALID_ARG;
  apc_batch *b = new (std::nothrow) apc_batch();
  if (!b) return APC_ERR_OUT_OF_MEMORY;
  b->ctx.assign(n_boxes, nullptr);
  for (int i = 0; i < n_boxes; ++i) {
    const int rc = apc_create(&cfgs[i], &b->ctx[i]);
    if (rc != APC_OK) {
      apc_batch_destroy(b);
      return rc;
    }
  }
  b->order.resize(n_boxes);
  for (int i = 0; i < n_boxes; ++i) b->order[i] = i;
  std::stable_sort(b->order.begin(), b->order.end(),
                   [&](int a, int c) { return cfgs[a].n_particles > cfgs[c].n_particles; });
  b->workers = n_workers > 0 ? std::min(n_workers, n_boxes) : std::min(n_boxes, 8);
  *out = b;
  return APC_OK;
}

int apc_batch_destroy(apc_batch *b) {
  if (!b) return APC_ERR_INVALID_ARG;
  for (apc_context *c : b->ctx)
    if (c) apc_destroy(c);
  delete b;
  return APC_OK;
}

int apc_batch_size(const apc_batch *b) { return b ? (int)b->ctx.size() : 0; }

apc_context *apc_batch_context(apc_batch *b, int box) {
  if (!b || box < 0 || box >= (int)b->ctx.size()) return nullptr;
  return b->ctx[box];
}

int apc_batch_step(apc_batch *b, const apc_step_params *params, int *status, double *max_dv, double *max_dx) {
  if (!b || !params) return APC_ERR_INVALID_ARG;
  const int n = (int)b->ctx.size();
  std::vector<int> st(n, APC_OK);
  std::atomic<int> next{0};
  auto work = [&]() {
    for (;;) {
      const int k = next.fetch_add(1);
      if (k >= n) return;
      const int i = b->order[k];
      double dv = 0.0, dx = 0.0;
      st[i] = apc_step(b->ctx[i], &params[i], nullptr, &dv, &dx);
      if (max_dv) max_dv[i] = dv;
      if (max_dx) max_dx[i] = dx;
    }
  };
  if (b->workers <= 1) {
    work();
  } else {
    std::vector<std::thread> pool;
    pool.reserve(b->workers - 1);
    for (int w = 1; w < b->workers; ++w) pool.emplace_back(work);
    work();
    for (std::thread &t : pool) t.join();
  }
  int first = APC_OK;
  for (int i = 0; i < n; ++i) {
    if (status) status[i] = st[i];
    if (first == APC_OK && st[i] != APC_OK) first = st[i];
  }
  return first;
}

}  // extern "C"
