// Internal declarations shared by the CUDA translation units of libapcloud_gpu.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/apcloud_gpu.h"

// ------------------------------------------------------------------ errors

// device-side error flags (bit set), read back by the host after each phase
enum : int {
  DERR_HASH_FULL = 1,      // a hash table probe ran past its bound
  DERR_STENCIL_FEW = 2,    // < lm candidates after 5 expansions
  DERR_STENCIL_MANY = 4,   // candidate buffers overflowed
  DERR_RANK = 8,           // zero diagonal in R of a GFD least-squares system
  DERR_NEIGH = 16,         // a face neighbour required by 2:1 balance was not found
  DERR_NOT_FINITE = 32,
  DERR_KRYLOV = 64,
  DERR_SORT = 128,         // a radix-sort tile's look-back wait ran past its bound
};

#define APC_CUDA_TRY(ctx, call)                                                      \
  do {                                                                               \
    cudaError_t e__ = (call);                                                        \
    if (e__ != cudaSuccess) {                                                        \
      (ctx)->err = std::string(#call) + ": " + cudaGetErrorString(e__);              \
      return APC_ERR_CUDA;                                                           \
    }                                                                                \
  } while (0)

#define APC_TRY(...)                  \
  do {                                \
    int rc__ = (__VA_ARGS__);         \
    if (rc__ != APC_OK) return rc__;  \
  } while (0)

// ----------------------------------------------------------------- context

struct KrylovWork;  // krylov.cu
struct MgWork;      // mg.cu

struct apc_context {
  apc_config cfg{};
  int dev = 0;
  // capacity (elements) of every buffer grown by apc_ensure, keyed by the address of the
  // owning pointer; per context, so contexts can be driven from different host threads
  std::unordered_map<const void *, size_t> caps;
  cudaStream_t s = nullptr;
  // host uploads of the velocities run on a copy stream beside the step's kernels: they are
  // needed only at the kick, so the upload overlaps the selection, assembly and solves
  cudaStream_t cs = nullptr;
  cudaEvent_t cs_ev = nullptr, vel_ev = nullptr;  // c->s before the upload; upload done
  bool vel_caller_order = false;  // pvx.. hold the caller's order (a fresh upload), not the sorted one
  cudaMemPool_t pool = nullptr;  // the device's stream-ordered pool (all device buffers)
  std::string err;
  int64_t launches = 0;
  bool have_particles = false, have_cells = false, have_fields = false;

  // ---- particles, kept in Morton (sorted) order on the device ----
  int n = 0;
  double *px = nullptr, *py = nullptr, *pz = nullptr, *pvx = nullptr, *pvy = nullptr, *pvz = nullptr;
  double *pax = nullptr, *pay = nullptr, *paz = nullptr;
  int *pid = nullptr;  // caller index of each sorted particle
  // particles are sorted by the top 3 * sorted_levels bits of their keys (the selection
  // needs no more than its deepest level); levels_hint = the last selection's deepest
  // level, 0 = unknown (then the sort takes every bit)
  int sorted_levels = 0, levels_hint = 0;
  double *qx = nullptr, *qy = nullptr, *qz = nullptr, *qvx = nullptr, *qvy = nullptr, *qvz = nullptr;
  int *qid = nullptr;
  uint64_t *keys = nullptr, *keys_alt = nullptr;
  uint32_t *perm = nullptr, *perm_alt = nullptr;
  uint32_t *sort_hist = nullptr;
  int sort_blocks = 0;
  double *reduce_buf = nullptr;  // per-block partial maxima of the mover

  // ---- selection ----
  double h0 = 1.0, hx0 = 1.0, hy0 = 1.0, hz0 = 1.0;  // root cell sizes (octree.cpp:1127-1131)
  double cx0 = 0.5, cy0 = 0.5, cz0 = 0.5;              // root centre (octree.cpp:1117-1119)
  int hcap = 0;                  // opened-node hash capacity (power of two)
  uint64_t *h_keys = nullptr;    // opened-node hash: location code
  int *h_vals = nullptr;         //                   index into the opened list
  int rcap = 0;                  // request hash capacity
  uint64_t *r_keys = nullptr, *r_vals = nullptr;
  int lcap = 0;                  // leaf hash capacity
  uint64_t *l_keys = nullptr;
  int *l_vals = nullptr;
  int op_cap = 0;                // opened list capacity
  uint64_t *op_code = nullptr;   // opened nodes: td in BFS order, then balance events in order
  int *op_base = nullptr;        // temp index of the node's first child
  int *op_first = nullptr, *op_count = nullptr;  // particle range (all opened nodes)
  int n_open_td = 0, n_open = 0;
  std::vector<int> td_level_off;  // [level] -> offset of level's td-opened nodes; size depth+2
  uint64_t *req_key = nullptr, *req_key_alt = nullptr;  // balance requests: first-requester key
  uint32_t *req_idx = nullptr, *req_idx_alt = nullptr;  //                   sort payload
  uint64_t *req_code = nullptr;                         //                   requested cell
  int *req_pos = nullptr;        // scan output of per-(node, octant) flags
  long long maxnc_state = 10000; // temp-node budget, doubled like Mover::maxnc (mover.cpp:36-41)
  int *counters = nullptr;       // small device counters
  int *d_err = nullptr;          // device error flags
  int *h_pinned = nullptr;       // pinned host mirror for small readbacks
  int *scan_tmp = nullptr;
  int scan_tmp_cap = 0;
  int *flags = nullptr;          // per-(opened node, octant) flags / scan
  int flags_cap = 0;
  std::vector<int> numnodes;     // octree level sizes of the last build

  // ---- cells (Computational_particle) in the reference's output order ----
  int nc = 0, nv = 0, nb = 0, m_cap = 0;
  double *cx = nullptr, *cy = nullptr, *cz = nullptr, *ch = nullptr;
  int *cfirst = nullptr, *ccount = nullptr, *ctype = nullptr;
  uint64_t *ccode = nullptr;
  int *nb24 = nullptr;   // 24 per cell
  int *nnb = nullptr;    // Neigh24 count per cell
  int *cell_of = nullptr;  // sorted particle -> cell
  uint64_t *full_keys = nullptr, *full_keys_alt = nullptr;  // fully sorted key copies (diagnostics)
  uint32_t *full_ids = nullptr, *full_ids_alt = nullptr;
  double *gfd_scr_d = nullptr;  // GFD search: per-warp sort lists longer than a warp
  int *gfd_scr_i = nullptr;
  int *gfd_qr = nullptr;         // GFD: cells queued for the Householder pass
  double *adj_ckpt = nullptr, *adj_tape = nullptr;  // trajectory VJP: checkpoints, Hessian tape
  double last_c_pot = 0.0, last_c_field = 0.0;       // constants of the last apc_solve
  uint64_t *warm_keys = nullptr;      // warm start: codes of the previous step's cells (hash)
  double *warm_rho = nullptr, *warm_phi = nullptr;
  int warm_cap = 0;
  // solve VJP: transposed stencil pattern and matrices (ELL, leading dimension M)
  int *tr_cnt = nullptr, *tr_off = nullptr, *tr_cur = nullptr, *tr_tmp = nullptr;
  int *tp_col = nullptr, *tp_src = nullptr, *ta_col = nullptr, *ta_src = nullptr;
  double *ta_val = nullptr, *vjp_c = nullptr, *vjp_phi = nullptr, *vjp_r2 = nullptr, *vjp_rho = nullptr;

  // ---- GFD / solver ----
  int lm = 17;
  int *st_idx = nullptr;     // lm per cell
  double *st_dist = nullptr; // lm per cell, filled on request (apc_get_stencils)
  double *gfd_x = nullptr;   // 9 x lm least-squares operator per cell
  int ell_w = 18;            // ELL width lm + 1
  int *ell_col = nullptr;    // [slot][row]
  double *a1 = nullptr, *a2 = nullptr;  // [slot][row]
  float *a1f = nullptr, *a2f = nullptr;    // D^-1 A1, D^-1 A2 in FP32 (mixed path)
  double *a1d = nullptr, *a2d = nullptr;   // the same in FP64 (FP64 multigrid path)
  double *rhs = nullptr, *bcrhs = nullptr;
  double *density = nullptr, *potential = nullptr, *deriv = nullptr;
  double rot[9] = {0};       // octant rotation (solver.cpp:464-475), host-computed
  KrylovWork *kw = nullptr;
  MgWork *mg = nullptr;
  // batched solves (apc_batch_step): the mixed solves are prepared here and run in one
  // launch with the other boxes' (defer_solve); batch_ev marks the prepared state
  bool defer_solve = false;
  cudaEvent_t batch_ev = nullptr;
  apc_solve_stats stats{};

  // ---- timing ----
  cudaEvent_t ev[8] = {};
  cudaEvent_t kev[2] = {};   // around each GMRES launch
  cudaEvent_t gev[2] = {};   // around the GFD stencil kernel
  cudaEvent_t sev[3] = {};   // solve phase: after assembly, after the density solve, after the potential rhs
  cudaEvent_t wait_ev = nullptr;  // host waits of a context driven by a batch fiber
  double t_select_ms = 0, t_solve_ms = 0, t_move_ms = 0;
  apc_profile prof{};
  bool step_open = false;    // a select has started a step that move_position will close
  unsigned select_gen = 0;   // completed selections (keys the multigrid aggregation to its cells)
  bool kick_recorded = false;  // ev[4] holds the start of a move_velocity
};

// ----------------------------------------------------------- helpers (host)

int apc_alloc(apc_context *c, void **p, size_t bytes);
void apc_free(apc_context *c, void *p);  // stream-ordered release of an apc_alloc buffer
cudaMemPool_t apc_device_pool(int dev);
template <class T>
int apc_ensure(apc_context *c, T **p, size_t count, size_t *cap_elems_io = nullptr);
int apc_read_errors(apc_context *c, int *flags);
// the velocities in the particles' sorted order on c->s (waits for a pending upload and
// gathers a fresh one through the particle ids); every kernel that reads them calls it first
int apc_velocities_sorted(apc_context *c);

// Host waits for the context's stream (or one of its events).  On an ordinary thread they
// block like cudaStreamSynchronize / cudaEventSynchronize.  Inside a batch fiber
// (batch.cu) they poll the event and yield to the other boxes' fibers until it completes,
// so one host thread keeps many boxes' GPU work in flight.
cudaError_t apc_stream_wait(apc_context *c);
cudaError_t apc_event_wait(cudaEvent_t e);

// launch accounting
inline void apc_count_launch(apc_context *c, int k = 1) { c->launches += k; }

// subsystem entry points (each in its own .cu)
int apc_octree_build(apc_context *c);        // keys, sort, permute (octree_build.cu)
int apc_octree_levels_count(apc_context *c); // numnodes per level (octree_build.cu)
int apc_selection(apc_context *c);           // top-down + balance + cells (selection.cu)
constexpr int APC_RETRY_FULL_SORT = -100;    // internal: the selection went deeper than the sort
int apc_sorted_keys_copy(apc_context *c, uint64_t **keys, uint32_t **ids);  // octree_build.cu
// gfd.cu; `during` runs on the host after the assembly's kernels are queued
int apc_gfd_assemble(apc_context *c, double c_dens, int (*during)(apc_context *) = nullptr);
// during (optional): host work run while the mixed solve's graph runs on the GPU, before
// the host waits for its outcome
int apc_krylov_solve(apc_context *c, int which, const double *b, double *x, int *its,
                     double *rnorm, int *reason, int *refinements,
                     int (*during)(apc_context *) = nullptr);  // krylov.cu
// the potential operator Jacobi-scaled in the inner precision of the configured path
// (c->a2 -> c->a2f, or c->a2d for the FP64 multigrid path), on stream s
void apc_potential_scaled(apc_context *c, cudaStream_t s);  // krylov.cu
void apc_krylov_free(apc_context *c);
int apc_gmres_fp64_ell(apc_context *c, int n, int w, size_t ld, const int *col, const double *val,
                       const double *b, double *x, int *its, double *rnorm, int *reason);  // krylov.cu
void apc_mg_free(apc_context *c);
// One solve of the mixed or FP64 multigrid path (mg.cu): FP64 refinement with (F)GMRES
// corrections on the Jacobi-scaled operator (c->a1f/a2f in FP32, c->a1d/a2d in FP64), run
// on the device as one CUDA graph; with use_mg the corrections are right-preconditioned by
// the octree-aggregation V-cycle, whose hierarchy is rebuilt from the scaled operator
int apc_ir_solve(apc_context *c, int which, bool use_mg, const double *val, const double *b, double *x, double *r,
                 int restart, double rtol_in, int *its, double *rnorm, int *reason, int *refinements, int *levels,
                 int (*during)(apc_context *) = nullptr);
// Overlap of the potential solve's set-up with the density solve (mg.cu).  After the
// assembly, apc_mg_mark_assembled records where the potential operator is ready;
// apc_mg_prebuild, run while the density graph executes, converts that operator to FP32
// and builds the multigrid hierarchy on a second stream, and makes the context's stream
// wait for it; the potential solve then uses the prebuilt hierarchy (apc_mg_prebuilt)
// instead of building its own.
// Solves of many contexts in one persistent launch (mg.cu): each context, with
// defer_solve set, prepares its solve in apc_krylov_solve and records batch_ev; one
// cooperative kernel then runs every prepared solve, its block groups pulling boxes from a
// device work queue, largest first; apc_ir_finish reads each context's outcome.
struct BatchSolveBuf;
BatchSolveBuf *apc_batch_solve_buf_create(int device);
void apc_batch_solve_buf_free(BatchSolveBuf *b);
int apc_mg_batched_solve(apc_context *const *ctx, int n, BatchSolveBuf *buf, cudaStream_t s, float *ms);
int apc_ir_finish(apc_context *c, int *its, double *rnorm, int *reason, int *refinements);
// apc_solve in three parts (capi.cu): assembly + density solve; potential rhs + potential
// solve; differentiation + bookkeeping.  With defer_solve the solves are only prepared and
// each following part starts by reading the prepared solve's outcome.
int apc_solve_part_density(apc_context *c, double c_dens);
int apc_solve_part_potential(apc_context *c, double c_pot);
int apc_solve_part_fields(apc_context *c, double c_field);
int apc_step_move(apc_context *c, const apc_step_params *p, double *max_dv, double *max_dx);
int apc_mg_mark_assembled(apc_context *c);
int apc_mg_prebuild(apc_context *c);
// the aggregation of the hierarchy (cell codes only) on the second stream while the GFD
// assembly runs
int apc_mg_structure_during_assembly(apc_context *c);
bool apc_mg_prebuilt(const apc_context *c);
void apc_mg_clear_prebuilt(apc_context *c);  // a new assembly invalidates a prebuilt hierarchy
int apc_warm_save(apc_context *c);                       // warmstart.cu
int apc_warm_guess(apc_context *c, int which, double *x);
int apc_potential_rhs(apc_context *c, double c_pot);    // gfd.cu
int apc_differentiate(apc_context *c, double c_field);  // gfd.cu
int apc_gfd_stencil_dist(apc_context *c);  // gfd.cu: stencil distances into st_dist
int apc_mover_velocity(apc_context *c, double dt, double c_vel, double *max_dv);  // mover.cu
int apc_mover_position(apc_context *c, double dt, double c_pos, double *max_dx);  // mover.cu
int apc_mover_kick_drift(apc_context *c, double dt, double c_vel, double c_pos, double *max_dv,
                         double *max_dx);                                          // mover.cu
int apc_mover_max_density(apc_context *c, double *out);                           // mover.cu
int apc_exclusive_scan(apc_context *c, const int *in, int *out, int n, int *total_dev);  // scan.cu
int apc_radix_sort_u64(apc_context *c, uint64_t *keys, uint32_t *vals, uint64_t *keys_alt,
                       uint32_t *vals_alt, int n, int lo_bit, int hi_bit, bool *result_in_alt);

// grid sizing: a multiple of the SM count
int apc_sm_count(apc_context *c);

// ------------------------------------------------------- grid barrier (persistent kernels)

// Generation barrier of a cooperative (persistent) kernel, in device memory zeroed before
// the launch.
struct GridBar {
  unsigned count;
  unsigned gen;
  int abort;
  int pad;
};

#ifdef __CUDACC__
constexpr long long kSpinLimit = 1ll << 24;  // ~1-2 s of __nanosleep(64)

// bounded sense-free generation barrier; returns false when the grid must abort.  A block
// that waits more than `limit` polls raises DERR_KRYLOV and the abort flag, which every
// other waiting block sees at its next poll
__device__ __forceinline__ bool grid_sync(GridBar *bar, unsigned nblocks, int *err, long long limit = kSpinLimit) {
  __syncthreads();
  __shared__ int s_abort;
  if (threadIdx.x == 0) {
    volatile unsigned *vgen = &bar->gen;
    volatile int *vab = &bar->abort;
    const unsigned g = *vgen;
    __threadfence();
    const unsigned a = atomicAdd(&bar->count, 1u);
    if (a == nblocks - 1) {
      atomicExch(&bar->count, 0u);
      __threadfence();
      atomicAdd(&bar->gen, 1u);
    } else {
      long long spins = 0;
      while (*vgen == g && !*vab) {
        if (++spins > limit) {
          atomicOr(err, DERR_KRYLOV);
          atomicExch(&bar->abort, 1);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_abort = *vab;
  }
  __syncthreads();
  return s_abort == 0;
}
#endif

// ------------------------------------------------------- device helpers

#ifdef __CUDACC__
__device__ __forceinline__ int code_level(uint64_t code) {
  // code = (1 << 3L) | prefix: L = (63 - clz) / 3
  return (63 - __clzll((long long)code)) / 3;
}

__device__ __forceinline__ uint64_t hash_mix(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

// open-addressing hash set/map over location codes (0 = empty slot); bounded probing
constexpr int kMaxProbe = 4096;

__device__ __forceinline__ int hash_find(const uint64_t *keys, int cap, uint64_t code) {
  uint32_t m = (uint32_t)cap - 1u;
  uint32_t h = (uint32_t)hash_mix(code) & m;
  for (int p = 0; p < kMaxProbe; ++p) {
    uint64_t k = keys[h];
    if (k == code) return (int)h;
    if (k == 0) return -1;
    h = (h + 1) & m;
  }
  return -1;
}

// insert; returns slot, sets *fresh when this call created the entry; -1 on overflow
__device__ __forceinline__ int hash_insert(uint64_t *keys, int cap, uint64_t code, bool *fresh) {
  uint32_t m = (uint32_t)cap - 1u;
  uint32_t h = (uint32_t)hash_mix(code) & m;
  *fresh = false;
  for (int p = 0; p < kMaxProbe; ++p) {
    unsigned long long prev =
        atomicCAS((unsigned long long *)&keys[h], 0ULL, (unsigned long long)code);
    if (prev == 0ULL) {
      *fresh = true;
      return (int)h;
    }
    if (prev == code) return (int)h;
    h = (h + 1) & m;
  }
  return -1;
}

// Morton helpers: spread / compact 21-bit integers over every third bit
__device__ __forceinline__ uint64_t spread3(uint64_t v) {
  v &= 0x1fffffULL;
  v = (v | v << 32) & 0x1f00000000ffffULL;
  v = (v | v << 16) & 0x1f0000ff0000ffULL;
  v = (v | v << 8) & 0x100f00f00f00f00fULL;
  v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
  v = (v | v << 2) & 0x1249249249249249ULL;
  return v;
}
__device__ __forceinline__ uint64_t compact3(uint64_t v) {
  v &= 0x1249249249249249ULL;
  v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ULL;
  v = (v ^ (v >> 4)) & 0x100f00f00f00f00fULL;
  v = (v ^ (v >> 8)) & 0x1f0000ff0000ffULL;
  v = (v ^ (v >> 16)) & 0x1f00000000ffffULL;
  v = (v ^ (v >> 32)) & 0x1fffffULL;
  return v;
}
#endif
