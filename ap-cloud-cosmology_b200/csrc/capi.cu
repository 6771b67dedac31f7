// C ABI of libapcloud_gpu.so: context lifetime, particle I/O, the four phases of
// Controller::solve (controller.cpp:133-197) and the result accessors.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "apc_internal.cuh"

// --------------------------------------------------------------- allocation

// Device buffers come from one stream-ordered memory pool per device: allocation and
// release are ordered on the context's stream, so growing a buffer between steps never
// synchronises the device (cudaFree would wait for every stream, stalling the other
// boxes of a batch).  Freed blocks stay in the pool for reuse until a context is
// destroyed, which trims the pool's unused memory.  Reuse across streams waits for the
// free to complete instead of adding a cross-stream dependency.
// live contexts per device: the pool keeps its freed blocks while any context of the device
// is alive (a new context reuses them instead of mapping fresh memory), and is trimmed when
// the last one goes
static std::atomic<int> g_live[64];

cudaMemPool_t apc_device_pool(int dev) {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  if (dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!pools[dev]) {
    cudaMemPoolProps pr{};
    pr.allocType = cudaMemAllocationTypePinned;
    pr.location.type = cudaMemLocationTypeDevice;
    pr.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &pr) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    uint64_t keep = UINT64_MAX;
    int no = 0;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    cudaMemPoolSetAttribute(p, cudaMemPoolReuseAllowInternalDependencies, &no);
    pools[dev] = p;
  }
  return pools[dev];
}

int apc_alloc(apc_context *c, void **p, size_t bytes) {
  *p = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(p, std::max<size_t>(bytes, 16), c->pool, c->s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    c->err = std::string("device allocation of ") + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? APC_ERR_OUT_OF_MEMORY : APC_ERR_CUDA;
  }
  return APC_OK;
}

void apc_free(apc_context *c, void *p) {
  if (p) cudaFreeAsync(p, c->s);
}

template <class T>
int apc_ensure(apc_context *c, T **p, size_t count, size_t *) {
  size_t &cap = c->caps[(const void *)p];
  if (*p && cap >= count) return APC_OK;
  if (*p) {
    apc_free(c, *p);  // ordered after the work already queued on the stream
    *p = nullptr;
  }
  size_t want = std::max<size_t>(count + count / 4, 64);
  APC_TRY(apc_alloc(c, (void **)p, want * sizeof(T)));
  cap = want;
  return APC_OK;
}
template int apc_ensure<double>(apc_context *, double **, size_t, size_t *);
template int apc_ensure<float>(apc_context *, float **, size_t, size_t *);
template int apc_ensure<int>(apc_context *, int **, size_t, size_t *);
template int apc_ensure<uint32_t>(apc_context *, uint32_t **, size_t, size_t *);
template int apc_ensure<uint64_t>(apc_context *, uint64_t **, size_t, size_t *);

int apc_read_errors(apc_context *c, int *flags) {
  APC_CUDA_TRY(c, cudaMemcpyAsync(c->h_pinned + 1, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, apc_stream_wait(c));
  *flags = c->h_pinned[1];
  if (*flags & DERR_SORT) {
    c->err = "radix sort: a tile's look-back wait ran past its bound";
    return APC_ERR_TIMEOUT;
  }
  return APC_OK;
}

int apc_sm_count(apc_context *c) {
  static std::atomic<int> cached[64];
  int d = c->dev;
  if (d >= 0 && d < 64) {
    const int v = cached[d].load(std::memory_order_relaxed);
    if (v) return v;
  }
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
  if (v <= 0) v = 1;
  if (d >= 0 && d < 64) cached[d].store(v, std::memory_order_relaxed);
  return v;
}

namespace {

__global__ void iota_int(int n, int *p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = i;
}

// up to 6 arrays from the sorted order to the caller's: dst_k[pid[s]] = src_k[s]
struct Arrays6 {
  const double *src[6];
  double *dst[6];
  int count;
};

__global__ void unpermute6(int n, const int *__restrict__ pid, Arrays6 a) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int p = pid[s];
    for (int k = 0; k < a.count; ++k) a.dst[k][p] = a.src[k][s];
  }
}

// dst_k[s] = src_k[pid[s]]: the caller-order velocities of a fresh upload, in sorted order
__global__ void gather3(int n, const int *__restrict__ pid, const double *__restrict__ x, const double *__restrict__ y,
                        const double *__restrict__ z, double *__restrict__ ox, double *__restrict__ oy,
                        double *__restrict__ oz) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int p = pid[s];
    ox[s] = x[p];
    oy[s] = y[p];
    oz[s] = z[p];
  }
}

void free_all(apc_context *c) {
  if (c->cs) cudaStreamSynchronize(c->cs);  // a velocity upload still writing the buffers
  apc_krylov_free(c);
  apc_mg_free(c);
  void *ptrs[] = {c->px, c->py, c->pz, c->pvx, c->pvy, c->pvz, c->pax, c->pay, c->paz, c->pid,
                  c->qx, c->qy, c->qz, c->qvx, c->qvy, c->qvz, c->qid, c->keys, c->keys_alt, c->perm,
                  c->perm_alt, c->sort_hist, c->reduce_buf, c->h_keys, c->h_vals, c->r_keys, c->r_vals,
                  c->l_keys, c->l_vals, c->op_code, c->op_base, c->op_first, c->op_count, c->req_key,
                  c->req_key_alt, c->req_idx, c->req_idx_alt, c->req_code, c->req_pos, c->counters,
                  c->d_err, c->scan_tmp, c->flags, c->cx, c->cy, c->cz, c->ch, c->cfirst, c->ccount,
                  c->ctype, c->ccode, c->nb24, c->nnb, c->cell_of, c->st_idx, c->st_dist, c->gfd_x,
                  c->ell_col, c->a1, c->a2, c->a1f, c->a2f, c->a1d, c->a2d, c->rhs, c->bcrhs, c->density, c->potential,
                  c->deriv, c->adj_ckpt, c->adj_tape, c->gfd_scr_d, c->gfd_scr_i, c->gfd_qr, c->full_keys, c->full_keys_alt, c->full_ids, c->full_ids_alt, c->warm_keys, c->warm_rho,
                  c->warm_phi, c->tr_cnt, c->tr_off, c->tr_cur, c->tr_tmp,
                  c->tp_col, c->tp_src, c->ta_col, c->ta_src, c->ta_val, c->vjp_c, c->vjp_phi, c->vjp_r2,
                  c->vjp_rho};
  if (c->s) {
    for (void *p : ptrs) apc_free(c, p);
    cudaStreamSynchronize(c->s);
  }
  if (c->pool && g_live[c->dev].fetch_sub(1) == 1) cudaMemPoolTrimTo(c->pool, 0);
  if (c->h_pinned) cudaFreeHost(c->h_pinned);
  for (auto &e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto &e : c->kev)
    if (e) cudaEventDestroy(e);
  if (c->wait_ev) cudaEventDestroy(c->wait_ev);
  if (c->batch_ev) cudaEventDestroy(c->batch_ev);
  for (auto &e : c->gev)
    if (e) cudaEventDestroy(e);
  for (auto &e : c->sev)
    if (e) cudaEventDestroy(e);
  if (c->cs) cudaStreamDestroy(c->cs);
  if (c->cs_ev) cudaEventDestroy(c->cs_ev);
  if (c->vel_ev) cudaEventDestroy(c->vel_ev);
  if (c->s) cudaStreamDestroy(c->s);
}

int check_ready(apc_context *c, bool particles, bool cells, bool fields) {
  if (!c) return APC_ERR_INVALID_ARG;
  if ((particles && !c->have_particles) || (cells && !c->have_cells) || (fields && !c->have_fields)) {
    c->err = "phase called before its inputs exist";
    return APC_ERR_ORDER;
  }
  return APC_OK;
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
    cudaGetLastError();  // a timing query must not leave a sticky error behind
    ms = 0.f;
  }
  return ms;
}

}  // namespace

// ------------------------------------------------------------------- API

extern "C" {

void apc_config_default(apc_config *cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->n_particles = 0;
  cfg->depth = 21;
  cfg->bc = 1;
  cfg->box[0] = 0.0; cfg->box[1] = 1.0;
  cfg->box[2] = 0.0; cfg->box[3] = 1.0;
  cfg->box[4] = 0.0; cfg->box[5] = 1.0;
  cfg->gfd_c = 5e-3;
  cfg->lm = 17;
  cfg->maxnc = 10000;
  cfg->nmax_cap = 0;
  cfg->gmres_restart = 30;
  cfg->gmres_rtol = 1e-10;
  cfg->gmres_atol = 1e-50;
  cfg->gmres_dtol = 1e5;
  cfg->gmres_max_it = 10000;
  cfg->precision = APC_PREC_FP64;
  cfg->mixed_restart = 0;
  cfg->mixed_inner_rtol = 0.0;
  cfg->device = 0;
  cfg->mixed_precond = APC_PRECOND_MULTIGRID;
  cfg->mg_sweeps = 0;
  cfg->mg_omega = 0.0;
  cfg->mg_alpha = 0.0;
  cfg->mg_reorth = 0;
  cfg->warm_start = 0;
  cfg->mixed_solve_graphs = 1;
}

const char *apc_status_string(int s) {
  switch (s) {
    case APC_OK: return "ok";
    case APC_ERR_INVALID_ARG: return "invalid argument";
    case APC_ERR_CUDA: return "CUDA error";
    case APC_ERR_OUT_OF_MEMORY: return "out of device memory";
    case APC_ERR_ORDER: return "phase called out of order";
    case APC_ERR_NMAX: return "temp-node budget exceeded";
    case APC_ERR_STENCIL: return "GFD neighbour search failed";
    case APC_ERR_RANK: return "rank-deficient GFD least squares";
    case APC_ERR_NOT_FINITE: return "non-finite particle coordinates";
    case APC_ERR_UNSUPPORTED: return "unsupported configuration";
    case APC_ERR_TIMEOUT: return "device wait timed out";
    default: return "unknown status";
  }
}

const char *apc_last_error(const apc_context *ctx) { return ctx ? ctx->err.c_str() : ""; }

int apc_create(const apc_config *cfg, apc_context **out) {
  if (!cfg || !out) return APC_ERR_INVALID_ARG;
  *out = nullptr;
  if (cfg->n_particles < 1 || cfg->depth < 1 || cfg->depth > 21 || cfg->lm < 9 || cfg->lm > 32 ||
      (cfg->bc != 0 && cfg->bc != 1) || !(cfg->gfd_c >= 0.0) || cfg->gmres_restart < 1 ||
      cfg->gmres_restart > 255 || cfg->mixed_restart < 0 || cfg->mixed_restart > 31 || cfg->mg_sweeps < 0 ||
      (cfg->mixed_precond != APC_PRECOND_JACOBI && cfg->mixed_precond != APC_PRECOND_MULTIGRID) ||
      (cfg->precision != APC_PREC_FP64 && cfg->precision != APC_PREC_MIXED &&
       cfg->precision != APC_PREC_FP64_MULTIGRID && cfg->precision != APC_PREC_MIXED_VCYCLE))
    return APC_ERR_INVALID_ARG;
  for (int d = 0; d < 3; ++d)
    if (!(cfg->box[2 * d + 1] > cfg->box[2 * d])) return APC_ERR_INVALID_ARG;
  if (cfg->bc != 1) return APC_ERR_UNSUPPORTED;
  apc_context *c = new apc_context();
  c->cfg = *cfg;
  c->dev = cfg->device;
  c->n = cfg->n_particles;
  c->lm = cfg->lm;
  c->maxnc_state = cfg->maxnc > 0 ? cfg->maxnc : 10000;
  auto fail = [&](int rc) {
    free_all(c);
    delete c;
    return rc;
  };
  if (cudaSetDevice(c->dev) != cudaSuccess) {
    cudaGetLastError();
    return fail(APC_ERR_CUDA);
  }
  if (cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking) != cudaSuccess) return fail(APC_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&c->cs, cudaStreamNonBlocking) != cudaSuccess) return fail(APC_ERR_CUDA);
  if (cudaEventCreateWithFlags(&c->cs_ev, cudaEventDisableTiming) != cudaSuccess) return fail(APC_ERR_CUDA);
  if (cudaEventCreateWithFlags(&c->vel_ev, cudaEventDisableTiming) != cudaSuccess) return fail(APC_ERR_CUDA);
  c->pool = apc_device_pool(c->dev);
  if (!c->pool) return fail(APC_ERR_CUDA);
  g_live[c->dev].fetch_add(1);
  for (auto &e : c->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return fail(APC_ERR_CUDA);
  for (auto &e : c->kev)
    if (cudaEventCreate(&e) != cudaSuccess) return fail(APC_ERR_CUDA);
  for (auto &e : c->gev)
    if (cudaEventCreate(&e) != cudaSuccess) return fail(APC_ERR_CUDA);
  for (auto &e : c->sev)
    if (cudaEventCreate(&e) != cudaSuccess) return fail(APC_ERR_CUDA);
  if (cudaEventCreateWithFlags(&c->wait_ev, cudaEventDisableTiming) != cudaSuccess) return fail(APC_ERR_CUDA);
  if (cudaMallocHost((void **)&c->h_pinned, 64 * sizeof(int)) != cudaSuccess) return fail(APC_ERR_CUDA);
  const size_t n = (size_t)c->n;
  double **dbl[] = {&c->px, &c->py, &c->pz, &c->pvx, &c->pvy, &c->pvz, &c->pax, &c->pay, &c->paz,
                    &c->qx, &c->qy, &c->qz, &c->qvx, &c->qvy, &c->qvz};
  for (double **p : dbl) {
    int rc = apc_alloc(c, (void **)p, n * sizeof(double));
    if (rc) return fail(rc);
  }
  int rc;
  if ((rc = apc_alloc(c, (void **)&c->pid, n * sizeof(int)))) return fail(rc);
  if ((rc = apc_alloc(c, (void **)&c->qid, n * sizeof(int)))) return fail(rc);
  if ((rc = apc_alloc(c, (void **)&c->keys, n * sizeof(uint64_t)))) return fail(rc);
  if ((rc = apc_alloc(c, (void **)&c->keys_alt, n * sizeof(uint64_t)))) return fail(rc);
  if ((rc = apc_alloc(c, (void **)&c->perm, n * sizeof(uint32_t)))) return fail(rc);
  if ((rc = apc_alloc(c, (void **)&c->perm_alt, n * sizeof(uint32_t)))) return fail(rc);
  if ((rc = apc_alloc(c, (void **)&c->counters, 256 * sizeof(int)))) return fail(rc);
  if ((rc = apc_alloc(c, (void **)&c->d_err, 4 * sizeof(int)))) return fail(rc);
  cudaMemsetAsync(c->d_err, 0, 4 * sizeof(int), c->s);
  cudaMemsetAsync(c->pax, 0, n * sizeof(double), c->s);
  cudaMemsetAsync(c->pay, 0, n * sizeof(double), c->s);
  cudaMemsetAsync(c->paz, 0, n * sizeof(double), c->s);
  // root cell geometry (octree.cpp:1117-1131): centre from the box, h0 = volume^(1/3)
  const double *b = cfg->box;
  c->hx0 = b[1] - b[0];
  c->hy0 = b[3] - b[2];
  c->hz0 = b[5] - b[4];
  c->h0 = std::pow(c->hx0 * c->hy0 * c->hz0, 1.0 / 3);
  c->cx0 = (b[1] + b[0]) / 2;
  c->cy0 = (b[3] + b[2]) / 2;
  c->cz0 = (b[5] + b[4]) / 2;
  // octant rotation of the neighbour search (solver.cpp:464-475), evaluated once on the host
  const double al = 0.01, be = 0.001, ga = 0.0001;
  double *A = c->rot;
  A[0] = std::cos(al) * std::cos(ga) - std::sin(al) * std::sin(be) * std::sin(ga);
  A[1] = -std::sin(al) * std::cos(be);
  A[2] = -std::cos(al) * std::sin(ga) - std::sin(al) * std::sin(be) * std::cos(ga);
  A[3] = std::cos(al) * std::sin(be) * std::sin(ga) + std::sin(al) * std::cos(ga);
  A[4] = std::cos(al) * std::cos(be);
  A[5] = std::cos(al) * std::sin(be) * std::cos(ga) - std::sin(al) * std::sin(ga);
  A[6] = std::cos(be) * std::sin(ga);
  A[7] = -std::sin(be);
  A[8] = std::cos(be) * std::cos(ga);
  if (cudaStreamSynchronize(c->s) != cudaSuccess) return fail(APC_ERR_CUDA);
  *out = c;
  return APC_OK;
}

int apc_destroy(apc_context *c) {
  if (!c) return APC_ERR_INVALID_ARG;
  cudaSetDevice(c->dev);
  cudaStreamSynchronize(c->s);
  free_all(c);
  delete c;
  return APC_OK;
}

static int set_particles_impl(apc_context *c, const double *const *src, cudaMemcpyKind kind) {
  if (!c) return APC_ERR_INVALID_ARG;
  for (int k = 0; k < 6; ++k)
    if (!src[k]) return APC_ERR_INVALID_ARG;
  cudaSetDevice(c->dev);
  const size_t bytes = sizeof(double) * (size_t)c->n;
  double *dst[6] = {c->px, c->py, c->pz, c->pvx, c->pvy, c->pvz};
  for (int k = 0; k < 3; ++k) APC_CUDA_TRY(c, cudaMemcpyAsync(dst[k], src[k], bytes, kind, c->s));
  // the velocities in the caller's order, on the copy stream after the work already queued
  // (which may still read them); the kick gathers them into the sorted order
  APC_CUDA_TRY(c, cudaEventRecord(c->cs_ev, c->s));
  APC_CUDA_TRY(c, cudaStreamWaitEvent(c->cs, c->cs_ev, 0));
  for (int k = 3; k < 6; ++k) APC_CUDA_TRY(c, cudaMemcpyAsync(dst[k], src[k], bytes, kind, c->cs));
  APC_CUDA_TRY(c, cudaEventRecord(c->vel_ev, c->cs));
  c->vel_caller_order = true;
  iota_int<<<std::max(1, std::min((c->n + 255) / 256, apc_sm_count(c) * 8)), 256, 0, c->s>>>(c->n, c->pid);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaGetLastError());
  c->have_particles = true;
  c->have_cells = false;
  c->have_fields = false;
  c->warm_cap = 0;  // a new particle set: no guess from the previous one
  // levels_hint stays: a selection deeper than the hint redoes the sort over every bit
  return APC_OK;
}

int apc_set_particles(apc_context *c, const double *x, const double *y, const double *z, const double *vx,
                      const double *vy, const double *vz) {
  const double *s[6] = {x, y, z, vx, vy, vz};
  return set_particles_impl(c, s, cudaMemcpyHostToDevice);
}

int apc_set_particles_device(apc_context *c, const double *x, const double *y, const double *z,
                             const double *vx, const double *vy, const double *vz) {
  const double *s[6] = {x, y, z, vx, vy, vz};
  return set_particles_impl(c, s, cudaMemcpyDeviceToDevice);
}

static int get_particles_impl(apc_context *c, double *const *dst, int count, cudaMemcpyKind kind) {
  APC_TRY(check_ready(c, true, false, false));
  cudaSetDevice(c->dev);
  APC_TRY(apc_velocities_sorted(c));
  const double *src[9] = {c->px, c->py, c->pz, c->pvx, c->pvy, c->pvz, c->pax, c->pay, c->paz};
  double *spare[6] = {c->qx, c->qy, c->qz, c->qvx, c->qvy, c->qvz};
  const size_t bytes = sizeof(double) * (size_t)c->n;
  const int G = std::max(1, std::min((c->n + 255) / 256, apc_sm_count(c) * 8));
  // caller order: up to six arrays at a time are scattered through the particle ids into
  // the spare buffers by one kernel, then copied out back to back
  for (int k0 = 0; k0 < count; k0 += 6) {
    Arrays6 a{};
    int which[6];
    for (int k = k0; k < count && k < k0 + 6; ++k) {
      if (!dst[k]) continue;
      a.src[a.count] = src[k];
      a.dst[a.count] = spare[a.count];
      which[a.count++] = k;
    }
    if (a.count == 0) continue;
    unpermute6<<<G, 256, 0, c->s>>>(c->n, c->pid, a);
    apc_count_launch(c);
    for (int j = 0; j < a.count; ++j) APC_CUDA_TRY(c, cudaMemcpyAsync(dst[which[j]], a.dst[j], bytes, kind, c->s));
  }
  APC_CUDA_TRY(c, apc_stream_wait(c));
  return APC_OK;
}

}  // extern "C"

int apc_velocities_sorted(apc_context *c) {
  if (!c->vel_caller_order) return APC_OK;
  APC_CUDA_TRY(c, cudaStreamWaitEvent(c->s, c->vel_ev, 0));
  const int G = std::max(1, std::min((c->n + 255) / 256, apc_sm_count(c) * 8));
  gather3<<<G, 256, 0, c->s>>>(c->n, c->pid, c->pvx, c->pvy, c->pvz, c->qvx, c->qvy, c->qvz);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaGetLastError());
  std::swap(c->pvx, c->qvx);
  std::swap(c->pvy, c->qvy);
  std::swap(c->pvz, c->qvz);
  c->vel_caller_order = false;
  return APC_OK;
}

extern "C" {

int apc_get_particles(apc_context *c, double *x, double *y, double *z, double *vx, double *vy, double *vz,
                      double *ax, double *ay, double *az) {
  double *d[9] = {x, y, z, vx, vy, vz, ax, ay, az};
  return get_particles_impl(c, d, 9, cudaMemcpyDeviceToHost);
}

int apc_get_particles_device(apc_context *c, double *x, double *y, double *z, double *vx, double *vy,
                             double *vz) {
  double *d[6] = {x, y, z, vx, vy, vz};
  return get_particles_impl(c, d, 6, cudaMemcpyDeviceToDevice);
}

int apc_select(apc_context *c, int *n_cells) {
  APC_TRY(check_ready(c, true, false, false));
  cudaSetDevice(c->dev);
  c->err.clear();
  c->have_cells = false;
  c->have_fields = false;
  APC_CUDA_TRY(c, cudaEventRecord(c->ev[0], c->s));
  c->step_open = true;
  APC_CUDA_TRY(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->s));
  APC_TRY(apc_octree_build(c));
  int derr = 0;
  APC_TRY(apc_read_errors(c, &derr));
  if (derr & DERR_NOT_FINITE) {
    c->err = "non-finite particle coordinates";
    return APC_ERR_NOT_FINITE;
  }
  int rc = apc_selection(c);
  if (rc == APC_RETRY_FULL_SORT) {
    // the tree went deeper than the sort: sort by every bit and select again
    c->levels_hint = 0;
    c->prof.sort_retries++;
    APC_TRY(apc_octree_build(c));
    rc = apc_selection(c);
  }
  APC_TRY(rc);
  APC_CUDA_TRY(c, cudaEventRecord(c->ev[1], c->s));
  APC_CUDA_TRY(c, apc_event_wait(c->ev[1]));
  // the velocity upload ran beside the selection: once a phase call returns, the caller's
  // arrays are no longer read, as with the positions
  if (c->vel_caller_order) APC_CUDA_TRY(c, apc_event_wait(c->vel_ev));
  c->t_select_ms = elapsed(c->ev[0], c->ev[1]);
  c->prof.select_ms += c->t_select_ms;
  c->numnodes.clear();
  c->have_cells = true;
  if (++c->select_gen == 0) c->select_gen = 1;
  if (n_cells) *n_cells = c->nc + c->nv + c->nb;
  return APC_OK;
}

}  // extern "C"

// The solve phase in three parts, so that a batch can run every box's density solve, and
// then every potential solve, in one launch (batch.cu).  With ctx->defer_solve the mixed
// solves are only prepared by apc_krylov_solve, and the next part reads their outcome.
int apc_solve_part_density(apc_context *c, double c_dens) {
  APC_TRY(check_ready(c, true, true, false));
  cudaSetDevice(c->dev);
  c->err.clear();
  APC_CUDA_TRY(c, cudaEventRecord(c->ev[2], c->s));
  // multigrid paths: the hierarchy's aggregation is built while the assembly runs, its
  // operators while the density solve runs
  const bool overlap = c->cfg.precision != APC_PREC_FP64 && c->cfg.mixed_precond == APC_PRECOND_MULTIGRID;
  APC_TRY(apc_gfd_assemble(c, c_dens, overlap ? apc_mg_structure_during_assembly : nullptr));
  if (c->cfg.precision == APC_PREC_MIXED) {
    APC_TRY(apc_ensure(c, &c->a1f, (size_t)c->m_cap * c->ell_w, nullptr));
    APC_TRY(apc_ensure(c, &c->a2f, (size_t)c->m_cap * c->ell_w, nullptr));
  } else if (c->cfg.precision == APC_PREC_FP64_MULTIGRID) {
    APC_TRY(apc_ensure(c, &c->a1d, (size_t)c->m_cap * c->ell_w, nullptr));
    APC_TRY(apc_ensure(c, &c->a2d, (size_t)c->m_cap * c->ell_w, nullptr));
  } else if (c->cfg.precision == APC_PREC_MIXED_VCYCLE) {
    // FP32 density corrections; FP64 potential FGMRES over the FP32 V-cycle
    APC_TRY(apc_ensure(c, &c->a1f, (size_t)c->m_cap * c->ell_w, nullptr));
    APC_TRY(apc_ensure(c, &c->a2f, (size_t)c->m_cap * c->ell_w, nullptr));
    APC_TRY(apc_ensure(c, &c->a2d, (size_t)c->m_cap * c->ell_w, nullptr));
  }
  apc_solve_stats &st = c->stats;
  if (overlap) APC_TRY(apc_mg_mark_assembled(c));
  APC_CUDA_TRY(c, cudaEventRecord(c->sev[0], c->s));
  APC_TRY(apc_krylov_solve(c, 0, c->rhs, c->density, &st.density_its, &st.density_rnorm, &st.density_reason,
                           &st.density_refinements, overlap ? apc_mg_prebuild : nullptr));
  return APC_OK;
}

int apc_solve_part_potential(apc_context *c, double c_pot) {
  apc_solve_stats &st = c->stats;
  if (c->defer_solve)
    APC_TRY(apc_ir_finish(c, &st.density_its, &st.density_rnorm, &st.density_reason, &st.density_refinements));
  APC_CUDA_TRY(c, cudaEventRecord(c->sev[1], c->s));
  APC_TRY(apc_potential_rhs(c, c_pot));
  APC_CUDA_TRY(c, cudaEventRecord(c->sev[2], c->s));
  APC_TRY(apc_krylov_solve(c, 1, c->rhs, c->potential, &st.potential_its, &st.potential_rnorm,
                           &st.potential_reason, &st.potential_refinements));
  c->last_c_pot = c_pot;
  return APC_OK;
}

int apc_solve_part_fields(apc_context *c, double c_field) {
  apc_solve_stats &st = c->stats;
  if (c->defer_solve)
    APC_TRY(apc_ir_finish(c, &st.potential_its, &st.potential_rnorm, &st.potential_reason,
                          &st.potential_refinements));
  APC_CUDA_TRY(c, cudaEventRecord(c->ev[7], c->s));
  APC_TRY(apc_differentiate(c, c_field));
  if (c->cfg.precision != APC_PREC_FP64 && c->cfg.warm_start) APC_TRY(apc_warm_save(c));
  c->last_c_field = c_field;
  APC_CUDA_TRY(c, cudaEventRecord(c->ev[3], c->s));
  APC_CUDA_TRY(c, apc_event_wait(c->ev[3]));
  c->t_solve_ms = elapsed(c->ev[2], c->ev[3]);
  c->prof.assemble_ms += elapsed(c->ev[2], c->sev[0]);
  c->prof.density_ms += elapsed(c->sev[0], c->sev[1]);
  c->prof.potential_ms += elapsed(c->sev[2], c->ev[7]);
  c->prof.solve_ms += c->t_solve_ms;
  c->prof.steps += 1;
  c->have_fields = true;
  return APC_OK;
}

// move_velocity + move_position (mover.cpp:51-121) as one fused pass over the particles
int apc_step_move(apc_context *c, const apc_step_params *p, double *max_dv, double *max_dx) {
  APC_CUDA_TRY(c, cudaEventRecord(c->ev[4], c->s));
  APC_TRY(apc_mover_kick_drift(c, p->dt, p->c_vel, p->c_pos, max_dv, max_dx));
  APC_CUDA_TRY(c, cudaEventRecord(c->ev[6], c->s));
  APC_CUDA_TRY(c, apc_event_wait(c->ev[6]));
  c->t_move_ms = elapsed(c->ev[4], c->ev[6]);
  c->prof.move_ms += c->t_move_ms;
  c->kick_recorded = false;
  if (c->step_open) {
    c->prof.step_ms += elapsed(c->ev[0], c->ev[6]);
    c->step_open = false;
  }
  return APC_OK;
}

extern "C" {

int apc_solve(apc_context *c, double c_dens, double c_pot, double c_field) {
  APC_TRY(apc_solve_part_density(c, c_dens));
  APC_TRY(apc_solve_part_potential(c, c_pot));
  return apc_solve_part_fields(c, c_field);
}

int apc_move_velocity(apc_context *c, double dt, double c_vel, double *max_dv) {
  APC_TRY(check_ready(c, true, true, true));
  cudaSetDevice(c->dev);
  APC_CUDA_TRY(c, cudaEventRecord(c->ev[4], c->s));
  c->kick_recorded = true;
  APC_TRY(apc_mover_velocity(c, dt, c_vel, max_dv));
  APC_CUDA_TRY(c, cudaEventRecord(c->ev[5], c->s));
  return APC_OK;
}

int apc_move_position(apc_context *c, double dt, double c_pos, double *max_dx) {
  APC_TRY(check_ready(c, true, false, false));
  cudaSetDevice(c->dev);
  APC_TRY(apc_mover_position(c, dt, c_pos, max_dx));
  APC_CUDA_TRY(c, cudaEventRecord(c->ev[6], c->s));
  APC_CUDA_TRY(c, apc_event_wait(c->ev[6]));
  if (c->kick_recorded) {
    c->t_move_ms = elapsed(c->ev[4], c->ev[6]);
    c->prof.move_ms += c->t_move_ms;
    c->kick_recorded = false;
  }
  if (c->step_open) {
    c->prof.step_ms += elapsed(c->ev[0], c->ev[6]);
    c->step_open = false;
  }
  return APC_OK;
}

int apc_step(apc_context *c, const apc_step_params *p, int *n_cells, double *max_dv, double *max_dx) {
  if (!p) return APC_ERR_INVALID_ARG;
  APC_TRY(apc_select(c, n_cells));
  APC_TRY(apc_solve(c, p->c_dens, p->c_pot, p->c_field));
  return apc_step_move(c, p, max_dv, max_dx);
}

int apc_synchronize(apc_context *c) {
  if (!c) return APC_ERR_INVALID_ARG;
  APC_CUDA_TRY(c, apc_stream_wait(c));
  return APC_OK;
}

int apc_get_cell_counts(apc_context *c, int *nc, int *nv, int *nb, int *n_neigh24) {
  APC_TRY(check_ready(c, true, true, false));
  if (nc) *nc = c->nc;
  if (nv) *nv = c->nv;
  if (nb) *nb = c->nb;
  if (n_neigh24) {
    const int M = c->nc + c->nv;
    std::vector<int> nn(M);
    APC_CUDA_TRY(c, cudaMemcpy(nn.data(), c->nnb, sizeof(int) * M, cudaMemcpyDeviceToHost));
    long long s = 0;
    for (int v : nn) s += v;
    *n_neigh24 = (int)s;
  }
  return APC_OK;
}

int apc_get_cells(apc_context *c, double *x, double *y, double *z, double *cell_length, int *first, int *count,
                  int *type, int *first_neigh, int *number_neigh, int *neigh24) {
  APC_TRY(check_ready(c, true, true, false));
  cudaSetDevice(c->dev);
  const int M = c->nc + c->nv;
  const size_t db = sizeof(double) * M, ib = sizeof(int) * M;
  if (x) APC_CUDA_TRY(c, cudaMemcpy(x, c->cx, db, cudaMemcpyDeviceToHost));
  if (y) APC_CUDA_TRY(c, cudaMemcpy(y, c->cy, db, cudaMemcpyDeviceToHost));
  if (z) APC_CUDA_TRY(c, cudaMemcpy(z, c->cz, db, cudaMemcpyDeviceToHost));
  if (cell_length) APC_CUDA_TRY(c, cudaMemcpy(cell_length, c->ch, db, cudaMemcpyDeviceToHost));
  if (first) APC_CUDA_TRY(c, cudaMemcpy(first, c->cfirst, ib, cudaMemcpyDeviceToHost));
  if (count) APC_CUDA_TRY(c, cudaMemcpy(count, c->ccount, ib, cudaMemcpyDeviceToHost));
  if (type) APC_CUDA_TRY(c, cudaMemcpy(type, c->ctype, ib, cudaMemcpyDeviceToHost));
  if (first_neigh || number_neigh || neigh24) {
    std::vector<int> nn(M), nb((size_t)M * 24);
    APC_CUDA_TRY(c, cudaMemcpy(nn.data(), c->nnb, ib, cudaMemcpyDeviceToHost));
    APC_CUDA_TRY(c, cudaMemcpy(nb.data(), c->nb24, ib * 24, cudaMemcpyDeviceToHost));
    int tot = 0;
    for (int i = 0; i < M; ++i) {
      if (first_neigh) first_neigh[i] = tot;
      if (number_neigh) number_neigh[i] = nn[i];
      if (neigh24)
        for (int k = 0; k < nn[i]; ++k) neigh24[tot + k] = nb[(size_t)i * 24 + k];
      tot += nn[i];
    }
  }
  return APC_OK;
}

int apc_get_cell_codes(apc_context *c, uint64_t *codes) {
  APC_TRY(check_ready(c, true, true, false));
  if (!codes) return APC_ERR_INVALID_ARG;
  APC_CUDA_TRY(c, cudaMemcpy(codes, c->ccode, sizeof(uint64_t) * (c->nc + c->nv), cudaMemcpyDeviceToHost));
  return APC_OK;
}

int apc_get_keys(apc_context *c, uint64_t *keys, int *index) {
  APC_TRY(check_ready(c, true, true, false));
  uint64_t *k = nullptr;
  uint32_t *id = nullptr;
  APC_TRY(apc_sorted_keys_copy(c, &k, &id));
  if (keys) APC_CUDA_TRY(c, cudaMemcpy(keys, k, sizeof(uint64_t) * c->n, cudaMemcpyDeviceToHost));
  if (index) APC_CUDA_TRY(c, cudaMemcpy(index, id, sizeof(int) * c->n, cudaMemcpyDeviceToHost));
  return APC_OK;
}

int apc_get_octree_levels(apc_context *c, int *numnodes) {
  APC_TRY(check_ready(c, true, true, false));
  if (!numnodes) return APC_ERR_INVALID_ARG;
  if (c->numnodes.empty()) APC_TRY(apc_octree_levels_count(c));
  for (int k = 0; k <= c->cfg.depth; ++k) numnodes[k] = c->numnodes[k];
  return APC_OK;
}

int apc_get_fields(apc_context *c, double *density, double *potential, double *deriv9) {
  APC_TRY(check_ready(c, true, true, true));
  const int M = c->nc + c->nv;
  if (density) APC_CUDA_TRY(c, cudaMemcpy(density, c->density, sizeof(double) * M, cudaMemcpyDeviceToHost));
  if (potential) APC_CUDA_TRY(c, cudaMemcpy(potential, c->potential, sizeof(double) * M, cudaMemcpyDeviceToHost));
  if (deriv9) APC_CUDA_TRY(c, cudaMemcpy(deriv9, c->deriv, sizeof(double) * 9 * M, cudaMemcpyDeviceToHost));
  return APC_OK;
}

int apc_get_stencils(apc_context *c, int *idx, double *dist) {
  APC_TRY(check_ready(c, true, true, true));
  const size_t k = (size_t)(c->nc + c->nv) * c->lm;
  if (idx) APC_CUDA_TRY(c, cudaMemcpy(idx, c->st_idx, sizeof(int) * k, cudaMemcpyDeviceToHost));
  if (dist) {
    APC_TRY(apc_gfd_stencil_dist(c));
    APC_CUDA_TRY(c, cudaMemcpy(dist, c->st_dist, sizeof(double) * k, cudaMemcpyDeviceToHost));
  }
  return APC_OK;
}

int apc_get_solve_stats(apc_context *c, apc_solve_stats *st) {
  APC_TRY(check_ready(c, true, true, true));
  if (!st) return APC_ERR_INVALID_ARG;
  *st = c->stats;
  return APC_OK;
}

int apc_get_matrix(apc_context *c, int which, int *n, int *nnz, int *rowptr, int *col, double *val) {
  APC_TRY(check_ready(c, true, true, true));
  if (which != 0 && which != 1) return APC_ERR_INVALID_ARG;
  const int M = c->nc + c->nv, W = c->ell_w;
  const size_t ld = (size_t)c->m_cap;
  std::vector<int> ec(ld * W);
  std::vector<double> ev(ld * W);
  APC_CUDA_TRY(c, cudaMemcpy(ec.data(), c->ell_col, sizeof(int) * ld * W, cudaMemcpyDeviceToHost));
  APC_CUDA_TRY(c, cudaMemcpy(ev.data(), which == 0 ? c->a1 : c->a2, sizeof(double) * ld * W,
                             cudaMemcpyDeviceToHost));
  std::vector<std::vector<std::pair<int, double>>> rows(M);
  for (int i = 0; i < M; ++i) {
    const bool pin = which == 1 && c->cfg.bc == 1 && i == 0;
    for (int s = 0; s < W; ++s) {
      const int cj = ec[(size_t)s * ld + i];
      if (s > 0 && (cj == i || pin)) continue;  // dropped slot
      bool dup = false;
      for (auto &e : rows[i])
        if (e.first == cj) { e.second = ev[(size_t)s * ld + i]; dup = true; }
      if (!dup) rows[i].push_back({cj, ev[(size_t)s * ld + i]});
    }
    std::sort(rows[i].begin(), rows[i].end());
  }
  int total = 0;
  for (auto &r : rows) total += (int)r.size();
  if (n) *n = M;
  if (nnz) *nnz = total;
  if (!rowptr) return APC_OK;
  int k = 0;
  for (int i = 0; i < M; ++i) {
    rowptr[i] = k;
    for (auto &e : rows[i]) {
      if (col) col[k] = e.first;
      if (val) val[k] = e.second;
      ++k;
    }
  }
  rowptr[M] = k;
  return APC_OK;
}

int64_t apc_kernel_launches(const apc_context *c) { return c ? c->launches : 0; }

int apc_get_profile(apc_context *c, apc_profile *out) {
  if (!c || !out) return APC_ERR_INVALID_ARG;
  *out = c->prof;
  return APC_OK;
}

int apc_reset_profile(apc_context *c) {
  if (!c) return APC_ERR_INVALID_ARG;
  c->prof = apc_profile{};
  return APC_OK;
}

int apc_config_from_options(apc_config *cfg, int argc, const char *const *argv) {
  // the KSP options of the reference's run lines (Makefile:30-32) reach both solves
  // through KSPSetFromOptions (solver.cpp:202, 275)
  if (!cfg || argc < 0 || (argc > 0 && !argv)) return APC_ERR_INVALID_ARG;
  for (int i = 0; i < argc; ++i) {
    const char *a = argv[i];
    if (!a || a[0] != '-') continue;
    const bool has = i + 1 < argc && argv[i + 1];
    auto num = [&](double *out) {
      if (!has) return false;
      char *end = nullptr;
      const double v = strtod(argv[i + 1], &end);
      if (!end || *end != '\0') return false;
      *out = v;
      ++i;
      return true;
    };
    double v = 0.0;
    if (!strcmp(a, "-ksp_gmres_restart")) {
      if (!num(&v) || v != (int)v) return APC_ERR_INVALID_ARG;
      if (v < 1 || v > 255) return APC_ERR_UNSUPPORTED;  // the FP64 GMRES kernel holds <= 255 basis vectors
      cfg->gmres_restart = (int)v;
    } else if (!strcmp(a, "-ksp_rtol")) {
      if (!num(&v)) return APC_ERR_INVALID_ARG;
      cfg->gmres_rtol = v;
    } else if (!strcmp(a, "-ksp_atol")) {
      if (!num(&v)) return APC_ERR_INVALID_ARG;
      cfg->gmres_atol = v;
    } else if (!strcmp(a, "-ksp_divtol")) {
      if (!num(&v)) return APC_ERR_INVALID_ARG;
      cfg->gmres_dtol = v;
    } else if (!strcmp(a, "-ksp_max_it")) {
      if (!num(&v) || v != (int)v || v < 1) return APC_ERR_INVALID_ARG;
      cfg->gmres_max_it = (int)v;
    }
  }
  return APC_OK;
}

int apc_max_cell_density(apc_context *c, double *max_density) {
  APC_TRY(check_ready(c, true, true, false));
  if (!max_density) return APC_ERR_INVALID_ARG;
  cudaSetDevice(c->dev);
  return apc_mover_max_density(c, max_density);
}

int apc_adaptive_dt(apc_context *c, double delta_a, double *dt) {
  if (!dt) return APC_ERR_INVALID_ARG;
  double rho = 0.0;
  APC_TRY(apc_max_cell_density(c, &rho));
  // controller.cpp:157-162: dt = 0.05 Delta_A / max_density^(1/2), at most Delta_A
  const double step = 0.05 * delta_a;
  const double d = 1.0 / pow(rho, 1.0 / 2);
  double v = step * d;
  if (v > delta_a) v = delta_a;
  *dt = v;
  return APC_OK;
}

int apc_device_code_version(int device, int *binary_version, int *ptx_version) {
  if (!binary_version && !ptx_version) return APC_ERR_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return APC_ERR_CUDA;
  }
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, (const void *)iota_int) != cudaSuccess) {
    cudaGetLastError();
    return APC_ERR_CUDA;
  }
  if (binary_version) *binary_version = fa.binaryVersion;
  if (ptx_version) *ptx_version = fa.ptxVersion;
  return APC_OK;
}

int apc_get_phase_times(apc_context *c, double *a, double *b, double *d) {
  if (!c) return APC_ERR_INVALID_ARG;
  if (a) *a = c->t_select_ms;
  if (b) *b = c->t_solve_ms;
  if (d) *d = c->t_move_ms;
  return APC_OK;
}

}  // extern "C"
