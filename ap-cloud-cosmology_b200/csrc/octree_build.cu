// Octree build on the device: Morton keys, radix sort, particle permutation, and the
// per-level node counts of the reference octree.
//
// Reference: Octree::buildOctree (octree.cpp:111-494) and Octree::computeKey64
// (octree.cpp:676-852).  The reference materialises every level of the octree as node
// arrays (about 28M nodes at 2M particles, depth 21).  Selection here only needs the
// sorted keys, so the node arrays are not built on the step path:
//   - the particle range of any node is two binary searches in the sorted keys;
//   - numnodes[] (octree.cpp:174-191) comes from one longest-common-prefix histogram.
// Particles are kept physically in sorted order, so every later per-particle pass
// reads coalesced SoA arrays.
#include <cuda_runtime.h>

#include <algorithm>

#include "apc_internal.cuh"

namespace {

// computeKey64 by repeated bisection in FP64, exactly as octree.cpp:691-849 (the
// midpoint (l + r) / 2.0 and the < / >= tests round identically on the GPU).  Bits
// per level: x -> 4, y -> 2, z -> 1, level 1 most significant.
__global__ void morton_keys(const double *__restrict__ x, const double *__restrict__ y,
                            const double *__restrict__ z, int n, int depth, double bx0, double bx1,
                            double by0, double by1, double bz0, double bz1, uint64_t *__restrict__ keys,
                            uint32_t *__restrict__ perm, int *err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double px = x[i], py = y[i], pz = z[i];
  if (!(isfinite(px) && isfinite(py) && isfinite(pz))) atomicOr(err, DERR_NOT_FINITE);
  double lx = bx0, rx = bx1, ly = by0, ry = by1, lz = bz0, rz = bz1;
  uint64_t key = 0;
  for (int l = 1; l <= depth; ++l) {
    const double mx = __dmul_rn(__dadd_rn(lx, rx), 0.5);
    const double my = __dmul_rn(__dadd_rn(ly, ry), 0.5);
    const double mz = __dmul_rn(__dadd_rn(lz, rz), 0.5);
    const bool hx = px >= mx, hy = py >= my, hz = pz >= mz;
    key = (key << 3) | (uint64_t)((hx ? 4 : 0) | (hy ? 2 : 0) | (hz ? 1 : 0));
    if (hx) lx = mx; else rx = mx;
    if (hy) ly = my; else ry = my;
    if (hz) lz = mz; else rz = mz;
  }
  keys[i] = key;
  perm[i] = (uint32_t)i;
}

__global__ void permute_particles(const uint32_t *__restrict__ perm, int n,
                                  const double *__restrict__ x, const double *__restrict__ y,
                                  const double *__restrict__ z, const double *__restrict__ vx,
                                  const double *__restrict__ vy, const double *__restrict__ vz,
                                  const int *__restrict__ id, double *__restrict__ ox,
                                  double *__restrict__ oy, double *__restrict__ oz,
                                  double *__restrict__ ovx, double *__restrict__ ovy,
                                  double *__restrict__ ovz, int *__restrict__ oid) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t p = perm[s];
  ox[s] = x[p];
  oy[s] = y[p];
  oz[s] = z[p];
  if (vx) {  // velocities still in the caller's order are gathered at the kick instead
    ovx[s] = vx[p];
    ovy[s] = vy[p];
    ovz[s] = vz[p];
  }
  oid[s] = id[p];
}

// histogram of the level at which consecutive sorted keys first differ:
// numnodes[k] = 1 + #{i >= 1 : keys differ within the top k levels}
__global__ void lcp_histogram(const uint64_t *__restrict__ keys, int n, int depth, int *hist) {
  __shared__ int h[24];
  if (threadIdx.x < 24) h[threadIdx.x] = 0;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x + 1; i < n; i += gridDim.x * blockDim.x) {
    uint64_t d = keys[i] ^ keys[i - 1];
    if (d) {
      int lead = __clzll((long long)d) - (64 - 3 * depth);  // leading equal bits
      atomicAdd(&h[lead / 3], 1);                            // first differing level - 1
    }
  }
  __syncthreads();
  if (threadIdx.x < 24 && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

}  // namespace

int apc_octree_build(apc_context *c) {
  const int n = c->n;
  if (n <= 0) return APC_OK;
  const int T = 256, G = (n + T - 1) / T;
  morton_keys<<<G, T, 0, c->s>>>(c->px, c->py, c->pz, n, c->cfg.depth, c->cfg.box[0], c->cfg.box[1],
                                 c->cfg.box[2], c->cfg.box[3], c->cfg.box[4], c->cfg.box[5], c->keys,
                                 c->perm, c->d_err);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaGetLastError());
  bool in_alt = false;
  // Sort by the top bits the selection will read: two levels below the last selection's
  // deepest, or all of them.  A selection that goes deeper asks for a full sort.
  const int D = c->cfg.depth;
  const int ls = c->levels_hint > 0 ? std::min(D, c->levels_hint + 2) : D;
  APC_TRY(apc_radix_sort_u64(c, c->keys, c->perm, c->keys_alt, c->perm_alt, n, 3 * (D - ls), 3 * D, &in_alt));
  c->sorted_levels = ls;
  if (in_alt) {
    uint64_t *tk = c->keys; c->keys = c->keys_alt; c->keys_alt = tk;
    uint32_t *tp = c->perm; c->perm = c->perm_alt; c->perm_alt = tp;
  }
  const bool vel = !c->vel_caller_order;
  permute_particles<<<G, T, 0, c->s>>>(c->perm, n, c->px, c->py, c->pz, vel ? c->pvx : nullptr, c->pvy, c->pvz,
                                       c->pid, c->qx, c->qy, c->qz, c->qvx, c->qvy, c->qvz, c->qid);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaGetLastError());
  std::swap(c->px, c->qx);
  std::swap(c->py, c->qy);
  std::swap(c->pz, c->qz);
  if (vel) {
    std::swap(c->pvx, c->qvx);
    std::swap(c->pvy, c->qvy);
    std::swap(c->pvz, c->qvz);
  }
  std::swap(c->pid, c->qid);
  return APC_OK;
}

// Copies of the keys and caller ids sorted by every key bit (the context's particles may
// be sorted by the top bits only); for the key and octree-level accessors.
int apc_sorted_keys_copy(apc_context *c, uint64_t **keys, uint32_t **ids) {
  const int n = c->n;
  APC_TRY(apc_ensure(c, &c->full_keys, (size_t)n + 1, nullptr));
  APC_TRY(apc_ensure(c, &c->full_keys_alt, (size_t)n + 1, nullptr));
  APC_TRY(apc_ensure(c, &c->full_ids, (size_t)n + 1, nullptr));
  APC_TRY(apc_ensure(c, &c->full_ids_alt, (size_t)n + 1, nullptr));
  APC_CUDA_TRY(c, cudaMemcpyAsync(c->full_keys, c->keys, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, c->s));
  APC_CUDA_TRY(c, cudaMemcpyAsync(c->full_ids, c->pid, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, c->s));
  bool alt = false;
  // an LSD sort orders by its last digits, so the copy is sorted by every bit again
  if (c->sorted_levels < c->cfg.depth)
    APC_TRY(apc_radix_sort_u64(c, c->full_keys, c->full_ids, c->full_keys_alt, c->full_ids_alt, n, 0,
                               3 * c->cfg.depth, &alt));
  *keys = alt ? c->full_keys_alt : c->full_keys;
  *ids = alt ? c->full_ids_alt : c->full_ids;
  // callers read the copies with plain cudaMemcpy, which does not wait for this stream
  APC_CUDA_TRY(c, apc_stream_wait(c));
  return APC_OK;
}

int apc_octree_levels_count(apc_context *c) {
  const int D = c->cfg.depth, n = c->n;
  c->numnodes.assign(D + 1, 0);
  if (n <= 0) return APC_OK;
  uint64_t *sorted = nullptr;
  uint32_t *ids = nullptr;
  APC_TRY(apc_sorted_keys_copy(c, &sorted, &ids));
  int *hist = c->counters + 64;  // 24 ints reserved
  APC_CUDA_TRY(c, cudaMemsetAsync(hist, 0, 24 * sizeof(int), c->s));
  int G = std::min((n + 255) / 256, apc_sm_count(c) * 8);
  lcp_histogram<<<G, 256, 0, c->s>>>(sorted, n, D, hist);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaGetLastError());
  int h[24];
  APC_CUDA_TRY(c, cudaMemcpyAsync(h, hist, sizeof(h), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, apc_stream_wait(c));
  // keys first differing at level lev+1 create a new node on every level >= lev+1
  c->numnodes[0] = 1;
  for (int k = 1; k <= D; ++k) {
    int cnt = 1;
    for (int lev = 0; lev < k; ++lev) cnt += h[lev];
    c->numnodes[k] = cnt;
  }
  return APC_OK;
}
