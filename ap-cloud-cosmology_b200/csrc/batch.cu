// Batches of independent boxes (a batch of contexts stepped together).
//
// The reference runs one box per process (test.cpp:16-80) and has no batched entry
// point.  A batch is one context per box, each with its own CUDA stream, and every box
// runs the single-context code path, so its results are exactly those of a lone context.
//
// Scheduling.  A small box's step is a chain of short kernels broken by host round trips
// (level sizes of the selection, hierarchy sizes of the multigrid, solver statistics).
// Driven one box per blocking host thread, the GPU idles through each round trip and the
// threads contend for the driver.  Here every box runs as a fiber (a user-space stack
// switched with swapcontext) on a few host threads.  A host wait inside the library
// (apc_stream_wait / apc_event_wait) records an event and yields to the next box instead
// of blocking, so one thread keeps the kernels of many boxes in flight and the boxes'
// small grids fill the SMs together.  Boxes are dealt to the threads in
// longest-processing-time order (largest first, round robin).
#include <cuda_runtime.h>
#include <sys/mman.h>
#include <ucontext.h>

#include <algorithm>
#include <new>
#include <thread>
#include <vector>

#include "apc_internal.cuh"

namespace {

constexpr size_t kStackBytes = 8u << 20;  // per box; pages are committed only when touched
constexpr size_t kGuardBytes = 64u << 10; // no-access guard below each stack

struct Fiber;
using FiberFn = int (*)(Fiber *);

struct Fiber {
  ucontext_t uc;
  bool done = false;
  apc_context *ctx = nullptr;
  const apc_step_params *params = nullptr;
  FiberFn fn = nullptr;  // the work this fiber runs (a whole step, or one part of it)
  int status = APC_OK;
  int n_cells = 0;
  double dv = 0.0, dx = 0.0;
};

int whole_step(Fiber *f) { return apc_step(f->ctx, f->params, &f->n_cells, &f->dv, &f->dx); }

// the three parts of a step around the two batched solve launches
int part_select_density(Fiber *f) {
  f->ctx->defer_solve = true;
  APC_TRY(apc_select(f->ctx, &f->n_cells));
  APC_TRY(apc_solve_part_density(f->ctx, f->params->c_dens));
  return cudaEventRecord(f->ctx->batch_ev, f->ctx->s) == cudaSuccess ? APC_OK : APC_ERR_CUDA;
}
int part_potential(Fiber *f) {
  APC_TRY(apc_solve_part_potential(f->ctx, f->params->c_pot));
  return cudaEventRecord(f->ctx->batch_ev, f->ctx->s) == cudaSuccess ? APC_OK : APC_ERR_CUDA;
}
int part_fields_move(Fiber *f) {
  APC_TRY(apc_solve_part_fields(f->ctx, f->params->c_field));
  f->ctx->defer_solve = false;
  return apc_step_move(f->ctx, f->params, &f->dv, &f->dx);
}

struct Sched {
  ucontext_t main;
  Fiber *cur = nullptr;
};

thread_local Sched *t_sched = nullptr;

void fiber_main() {
  Fiber *f = t_sched->cur;
  f->status = f->fn(f);
  f->done = true;
}  // returning resumes uc_link, the scheduler

inline bool in_fiber() { return t_sched && t_sched->cur; }

inline void yield() {
  Fiber *f = t_sched->cur;
  swapcontext(&f->uc, &t_sched->main);
}

// Run the fibers of one host thread until all have finished: each is resumed in turn and
// runs until it waits on the GPU (yield) or its step ends.
void run_fibers(std::vector<Fiber *> &fibers, std::vector<char *> &stacks) {
  Sched sch;
  t_sched = &sch;
  for (size_t k = 0; k < fibers.size(); ++k) {
    Fiber *f = fibers[k];
    getcontext(&f->uc);
    f->uc.uc_stack.ss_sp = stacks[k] + kGuardBytes;
    f->uc.uc_stack.ss_size = kStackBytes - kGuardBytes;
    f->uc.uc_link = &sch.main;
    makecontext(&f->uc, fiber_main, 0);
  }
  size_t live = fibers.size();
  while (live) {
    for (Fiber *f : fibers) {
      if (f->done) continue;
      sch.cur = f;
      swapcontext(&sch.main, &f->uc);
      sch.cur = nullptr;
      if (f->done) --live;
    }
  }
  t_sched = nullptr;
}

}  // namespace

cudaError_t apc_event_wait(cudaEvent_t e) {
  if (!in_fiber()) return cudaEventSynchronize(e);
  // every fiber leaves through here with no launch error pending, so the thread's last
  // error can be cleared after each not-ready poll without losing another box's error
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess) return pending;
  for (;;) {
    const cudaError_t q = cudaEventQuery(e);
    if (q != cudaErrorNotReady) return q;
    cudaGetLastError();
    yield();
  }
}

cudaError_t apc_stream_wait(apc_context *c) {
  if (!in_fiber()) return cudaStreamSynchronize(c->s);
  const cudaError_t e = cudaEventRecord(c->wait_ev, c->s);
  if (e != cudaSuccess) return e;
  return apc_event_wait(c->wait_ev);
}

struct apc_batch {
  std::vector<apc_context *> ctx;
  std::vector<int> order;  // boxes by decreasing particle count
  int threads = 1;
  char *stack_base = nullptr;  // n_boxes stacks of kStackBytes, guard page first
  size_t stack_bytes = 0;
  int solve_mode = APC_BATCH_SOLVE_PER_BOX;
  BatchSolveBuf *sbuf = nullptr;  // the batched solves' queue, barriers and partial sums
  cudaStream_t bstream = nullptr;
  float last_solve_ms = 0.f;      // device time of the last step's two batched launches
};

namespace {

// every box runs fn as a fiber, boxes dealt to the host threads largest first
void run_all(apc_batch *b, std::vector<Fiber> &fib, FiberFn fn) {
  const int n = (int)b->ctx.size();
  for (int i = 0; i < n; ++i) {
    fib[i].done = false;
    fib[i].fn = fn;
  }
  const int T = b->threads;
  auto work = [&](int t) {
    std::vector<Fiber *> mine;
    std::vector<char *> stacks;
    for (int k = t; k < n; k += T) {
      const int i = b->order[k];
      if (fib[i].status != APC_OK) continue;  // a box that failed sits out the rest of the step
      mine.push_back(&fib[i]);
      stacks.push_back(b->stack_base + kStackBytes * (size_t)i);
    }
    run_fibers(mine, stacks);
  };
  if (T <= 1) {
    work(0);
  } else {
    std::vector<std::thread> pool;
    pool.reserve(T - 1);
    for (int t = 1; t < T; ++t) pool.emplace_back(work, t);
    work(0);
    for (std::thread &th : pool) th.join();
  }
}

// one launch for the prepared solves of every box still running
void batched_solve(apc_batch *b, std::vector<Fiber> &fib, float *ms) {
  std::vector<apc_context *> live;
  for (size_t i = 0; i < fib.size(); ++i)
    if (fib[i].status == APC_OK) live.push_back(b->ctx[i]);
  if (live.empty()) return;
  cudaSetDevice(live[0]->dev);
  float t = 0.f;
  const int rc = apc_mg_batched_solve(live.data(), (int)live.size(), b->sbuf, b->bstream, &t);
  *ms += t;
  if (rc != APC_OK)
    for (size_t i = 0; i < fib.size(); ++i)
      if (fib[i].status == APC_OK) {
        fib[i].status = rc;
        b->ctx[i]->defer_solve = false;
        b->ctx[i]->err = "batched solve launch failed";
      }
}

}  // namespace

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
  b->stack_bytes = kStackBytes * (size_t)n_boxes;
  void *m = mmap(nullptr, b->stack_bytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE,
                 -1, 0);
  if (m == MAP_FAILED) {
    b->stack_bytes = 0;
    apc_batch_destroy(b);
    return APC_ERR_OUT_OF_MEMORY;
  }
  b->stack_base = static_cast<char *>(m);
  for (int i = 0; i < n_boxes; ++i) mprotect(b->stack_base + kStackBytes * (size_t)i, kGuardBytes, PROT_NONE);
  b->order.resize(n_boxes);
  for (int i = 0; i < n_boxes; ++i) b->order[i] = i;
  std::stable_sort(b->order.begin(), b->order.end(),
                   [&](int a, int c) { return cfgs[a].n_particles > cfgs[c].n_particles; });
  b->threads = n_workers > 0 ? std::min(n_workers, n_boxes) : std::min(n_boxes, 16);
  for (apc_context *c : b->ctx)
    if (cudaEventCreateWithFlags(&c->batch_ev, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      apc_batch_destroy(b);
      return APC_ERR_CUDA;
    }
  *out = b;
  return APC_OK;
}

int apc_batch_destroy(apc_batch *b) {
  if (!b) return APC_ERR_INVALID_ARG;
  for (apc_context *c : b->ctx)
    if (c) apc_destroy(c);
  if (b->bstream) cudaStreamDestroy(b->bstream);
  apc_batch_solve_buf_free(b->sbuf);
  if (b->stack_base) munmap(b->stack_base, b->stack_bytes);
  delete b;
  return APC_OK;
}

int apc_batch_size(const apc_batch *b) { return b ? (int)b->ctx.size() : 0; }

apc_context *apc_batch_context(apc_batch *b, int box) {
  if (!b || box < 0 || box >= (int)b->ctx.size()) return nullptr;
  return b->ctx[box];
}

int apc_batch_set_solve_mode(apc_batch *b, int mode) {
  if (!b || (mode != APC_BATCH_SOLVE_PER_BOX && mode != APC_BATCH_SOLVE_QUEUED)) return APC_ERR_INVALID_ARG;
  if (mode == APC_BATCH_SOLVE_QUEUED && !b->sbuf) {
    const int dev = b->ctx[0]->dev;
    cudaSetDevice(dev);
    b->sbuf = apc_batch_solve_buf_create(dev);
    if (!b->sbuf) return APC_ERR_OUT_OF_MEMORY;
    if (cudaStreamCreateWithFlags(&b->bstream, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      return APC_ERR_CUDA;
    }
  }
  b->solve_mode = mode;
  return APC_OK;
}

float apc_batch_solve_ms(const apc_batch *b) { return b ? b->last_solve_ms : 0.f; }

int apc_batch_step(apc_batch *b, const apc_step_params *params, int *status, double *max_dv, double *max_dx) {
  if (!b || !params) return APC_ERR_INVALID_ARG;
  const int n = (int)b->ctx.size();
  std::vector<Fiber> fib(n);
  for (int i = 0; i < n; ++i) {
    fib[i].ctx = b->ctx[i];
    fib[i].params = &params[i];
  }
  if (b->solve_mode == APC_BATCH_SOLVE_QUEUED) {
    // select + assembly + density solve prepared; one launch; potential rhs + potential
    // solve prepared; one launch; differentiation + kick + drift
    float ms = 0.f;
    run_all(b, fib, part_select_density);
    batched_solve(b, fib, &ms);
    run_all(b, fib, part_potential);
    batched_solve(b, fib, &ms);
    run_all(b, fib, part_fields_move);
    b->last_solve_ms = ms;
    for (int i = 0; i < n; ++i) b->ctx[i]->defer_solve = false;
  } else {
    run_all(b, fib, whole_step);
  }
  int first = APC_OK;
  for (int i = 0; i < n; ++i) {
    if (status) status[i] = fib[i].status;
    if (max_dv) max_dv[i] = fib[i].dv;
    if (max_dx) max_dx[i] = fib[i].dx;
    if (first == APC_OK && fib[i].status != APC_OK) first = fib[i].status;
  }
  return first;
}

}  // extern "C"
