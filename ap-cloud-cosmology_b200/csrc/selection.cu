// Computational-particle selection on the device.
//
// Reference: Octree::select_computational_particles_2to1_3d (octree.cpp:1050-3001), a
// serial breadth-first refinement followed by a serial bottom-up 2:1 balance.  This
// file computes the same cell set in the same output order with level-parallel passes.
//
// Top-down (octree.cpp:1161-1790).  A node is opened when n*h^2 > c and level < depth.
// n and h both shrink with depth, so the opened set is every octree node that passes
// the test.  Each level is one parallel pass over the opened nodes of the level above.
// The child particle ranges come from binary searches in the sorted keys.  The
// reference's temp-node order is breadth-first, octants in Morton order, so the
// opened list built level by level (stable compaction) is in that same order.  The
// temp index of child c of the r-th opened node is 1 + 8r + c.
//
// Bottom-up 2:1 balance (octree.cpp:1793-2718).  At sweep ln every node of level ln
// looks at its six same-level face neighbours.  If the leaf containing a neighbour is
// coarser than ln-1, the leaf and its descendants down to level ln-2 along that
// position are opened.  Requests within a sweep do not interact, so a sweep is one
// parallel pass.  The reference creates those cells in the order of its first
// requester: temp index of the requesting node, then direction, then level.  That
// order is rebuilt exactly by keeping, per requested cell, the minimum of
// (temp index << 8 | direction << 5 | level) and sorting on it.
//
// Output (octree.cpp:2720-3000).  Cells are the unopened children of opened nodes, in
// temp-index order: top-down leaves (Type 0) first, then balance leaves (Type -1).
// Neigh24 is rebuilt from location codes in the reference's direction order
// x+, x-, y+, y-, z+, z-.  A neighbour is one same-or-coarser cell or the 4 finer
// cells on the shared face.
//
// Location code of a cell at level L with Morton prefix P: (1 << 3L) | P.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "apc_internal.cuh"

namespace {

constexpr int kT = 256;

__device__ __forceinline__ int lower_digit(const uint64_t *keys, int lo, int hi, int shift, int d) {
  // first index in [lo, hi) whose digit ((key >> shift) & 7) >= d; digits ascend in range
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if ((int)((keys[mid] >> shift) & 7ull) < d) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int lower_key(const uint64_t *keys, int n, uint64_t v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (keys[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// particle range [first, first+count) of the cell with location code `code`
__device__ __forceinline__ void cell_range(const uint64_t *keys, int n, int depth, uint64_t code,
                                           int *first, int *count) {
  const int L = code_level(code);
  const uint64_t prefix = code ^ (1ull << (3 * L));
  const int s = 3 * (depth - L);
  const uint64_t lo = prefix << s;
  const uint64_t hi = (s >= 63 && L == 0) ? (1ull << 63) : ((prefix + 1) << s);
  int a = lower_key(keys, n, lo);
  int b = (L == 0) ? n : lower_key(keys, n, hi);
  *first = a;
  *count = b - a;
}

// ------------------------------------------------------------------ top-down

__global__ void td_root(uint64_t *op_code, int *op_base, int *op_first, int *op_count, int n,
                        uint64_t *hkeys, int *hvals, int hcap, int *err) {
  op_code[0] = 1ull;
  op_base[0] = 1;
  op_first[0] = 0;
  op_count[0] = n;
  bool fresh;
  int s = hash_insert(hkeys, hcap, 1ull, &fresh);
  if (s < 0) atomicOr(err, DERR_HASH_FULL);
  else hvals[s] = 0;
}

// children of the opened nodes [off, off+cnt) of level L: particle ranges and the
// refinement test n*h^2 > c (octree.cpp:1165-1183)
__global__ void td_expand(const uint64_t *__restrict__ keys, int depth, int L, int off, int cnt,
                          const int *__restrict__ op_first, const int *__restrict__ op_count,
                          double hchild, double c, int maxdepth, int *__restrict__ flags,
                          int *__restrict__ cfirst, int *__restrict__ ccount) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 8 * cnt) return;
  const int o = off + (t >> 3), ch = t & 7;
  const int lo = op_first[o], hi = lo + op_count[o];
  const int shift = 3 * (depth - L - 1);
  const int a = lower_digit(keys, lo, hi, shift, ch);
  const int b = lower_digit(keys, a, hi, shift, ch + 1);
  const int np = b - a;
  double temp = 1.0 * np;
  temp = __dmul_rn(temp, hchild);
  temp = __dmul_rn(temp, hchild);
  flags[t] = (temp > c) && (L + 1 < maxdepth);
  cfirst[t] = a;
  ccount[t] = np;
}

__global__ void td_compact(int off, int cnt, int off_next, const int *__restrict__ flags,
                           const int *__restrict__ pos, const int *__restrict__ cfirst,
                           const int *__restrict__ ccount, uint64_t *op_code, int *op_base,
                           int *op_first, int *op_count, uint64_t *hkeys, int *hvals, int hcap,
                           int *err) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 8 * cnt || !flags[t]) return;
  const int o = off + (t >> 3);
  const int q = off_next + pos[t];
  const uint64_t code = (op_code[o] << 3) | (uint64_t)(t & 7);
  op_code[q] = code;
  op_base[q] = 1 + 8 * q;
  op_first[q] = cfirst[t];
  op_count[q] = ccount[t];
  bool fresh;
  int s = hash_insert(hkeys, hcap, code, &fresh);
  if (s < 0) atomicOr(err, DERR_HASH_FULL);
  else hvals[s] = q;
}

// ------------------------------------------------------------------ balance

__device__ __forceinline__ bool neighbour_code(uint64_t code, int L, int di, int bc, uint64_t *out) {
  const uint64_t prefix = code ^ (1ull << (3 * L));
  long long ix = (long long)compact3(prefix >> 2), iy = (long long)compact3(prefix >> 1),
            iz = (long long)compact3(prefix);
  // direction numbering of the reference's temp links: 0 x+, 1 x-, 2 y-, 3 y+, 4 z+, 5 z-
  switch (di) {
    case 0: ++ix; break;
    case 1: --ix; break;
    case 2: --iy; break;
    case 3: ++iy; break;
    case 4: ++iz; break;
    default: --iz; break;
  }
  const long long side = 1ll << L;
  if (ix < 0 || ix >= side || iy < 0 || iy >= side || iz < 0 || iz >= side) {
    if (bc != 1) return false;
    ix = (ix + side) & (side - 1);
    iy = (iy + side) & (side - 1);
    iz = (iz + side) & (side - 1);
  }
  *out = (1ull << (3 * L)) | (spread3((uint64_t)ix) << 2) | (spread3((uint64_t)iy) << 1) |
         spread3((uint64_t)iz);
  return true;
}

// sweep ln: every node of level ln (children of opened nodes of level ln-1) requests the
// opening of the coarse cells that break 2:1 across its six faces
__global__ void bal_requests(int ln, int td_a, int td_b, int bal_a, int bal_b, int bc,
                             const uint64_t *__restrict__ op_code, const int *__restrict__ op_base,
                             const uint64_t *__restrict__ hkeys, int hcap, uint64_t *rkeys,
                             unsigned long long *rvals, int rcap, int *err) {
  const int ntd = td_b - td_a, nbal = bal_b - bal_a;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 8 * (ntd + nbal)) return;
  const int r = t >> 3, ch = t & 7;
  const int o = r < ntd ? td_a + r : bal_a + (r - ntd);
  const uint64_t pcode = op_code[o];
  if (code_level(pcode) != ln - 1) return;
  const uint64_t code = (pcode << 3) | (uint64_t)ch;
  const unsigned long long tidx = (unsigned long long)(op_base[o] + ch);
  for (int di = 0; di < 6; ++di) {
    uint64_t nc;
    if (!neighbour_code(code, ln, di, bc, &nc)) continue;
    if (ln >= 2 && hash_find(hkeys, hcap, nc >> 6) >= 0) continue;  // leaf at level >= ln-1
    int lstar = 0;
    for (int l = ln - 3; l >= 0; --l)
      if (hash_find(hkeys, hcap, nc >> (3 * (ln - l))) >= 0) { lstar = l; break; }
    for (int l = lstar + 1; l <= ln - 2; ++l) {
      const uint64_t target = nc >> (3 * (ln - l));
      const unsigned long long key = (tidx << 8) | ((unsigned long long)di << 5) | (unsigned long long)l;
      bool fresh;
      int s = hash_insert(rkeys, rcap, target, &fresh);
      if (s < 0) { atomicOr(err, DERR_HASH_FULL); continue; }
      atomicMin(&rvals[s], key);
    }
  }
}

__global__ void bal_collect(const uint64_t *__restrict__ rkeys, const unsigned long long *__restrict__ rvals,
                            int rcap, int *count, uint64_t *out_key, uint32_t *out_idx,
                            uint64_t *out_code) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= rcap) return;
  uint64_t k = rkeys[s];
  if (!k) return;
  int q = atomicAdd(count, 1);
  out_key[q] = rvals[s];
  out_idx[q] = (uint32_t)q;
  out_code[q] = k;
}

__global__ void bal_commit(int nreq, int n_open, int child_base0, const uint32_t *__restrict__ order,
                           const uint64_t *__restrict__ codes, const uint64_t *__restrict__ keys,
                           int n, int depth, uint64_t *op_code, int *op_base, int *op_first,
                           int *op_count, uint64_t *hkeys, int *hvals, int hcap, int *err) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nreq) return;
  const int q = n_open + r;
  const uint64_t code = codes[order[r]];
  op_code[q] = code;
  op_base[q] = child_base0 + 8 * r;
  int f, cnt;
  cell_range(keys, n, depth, code, &f, &cnt);
  op_first[q] = f;
  op_count[q] = cnt;
  bool fresh;
  int s = hash_insert(hkeys, hcap, code, &fresh);
  if (s < 0) atomicOr(err, DERR_HASH_FULL);
  else hvals[s] = q;
}

// ------------------------------------------------------------------ output

__global__ void leaf_flags(int n_open, const uint64_t *__restrict__ op_code,
                           const uint64_t *__restrict__ hkeys, int hcap, int *flags) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 8 * n_open) return;
  const uint64_t child = (op_code[t >> 3] << 3) | (uint64_t)(t & 7);
  flags[t] = hash_find(hkeys, hcap, child) < 0;
}

// cell centre by replaying the reference's parent-centre +- h/4 recursion from the root
// (octree.cpp:1233-1235 and siblings), so that every rounding step is the same
__global__ void leaf_emit(int n_open, int n_open_td, const int *__restrict__ flags,
                          const int *__restrict__ pos, const uint64_t *__restrict__ op_code,
                          const uint64_t *__restrict__ keys, int n, int depth, double cx0,
                          double cy0, double cz0, double hx0, double hy0, double hz0, double h0,
                          double *cx, double *cy, double *cz, double *ch, int *cfirst, int *ccount,
                          int *ctype, uint64_t *ccode, uint64_t *lkeys, int *lvals, int lcap,
                          int *err) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 8 * n_open || !flags[t]) return;
  const int i = pos[t];
  const uint64_t code = (op_code[t >> 3] << 3) | (uint64_t)(t & 7);
  const int L = code_level(code);
  double x = cx0, y = cy0, z = cz0;
  for (int l = 0; l < L; ++l) {
    const unsigned dgt = (unsigned)((code >> (3 * (L - 1 - l))) & 7ull);
    const double qx = 0.25 * ldexp(hx0, -l), qy = 0.25 * ldexp(hy0, -l), qz = 0.25 * ldexp(hz0, -l);
    x = (dgt & 4) ? __dadd_rn(x, qx) : __dsub_rn(x, qx);
    y = (dgt & 2) ? __dadd_rn(y, qy) : __dsub_rn(y, qy);
    z = (dgt & 1) ? __dadd_rn(z, qz) : __dsub_rn(z, qz);
  }
  cx[i] = x;
  cy[i] = y;
  cz[i] = z;
  ch[i] = ldexp(h0, -L);
  int f, c;
  cell_range(keys, n, depth, code, &f, &c);
  cfirst[i] = f;
  ccount[i] = c;
  ctype[i] = (t >> 3) < n_open_td ? 0 : -1;
  ccode[i] = code;
  bool fresh;
  int s = hash_insert(lkeys, lcap, code, &fresh);
  if (s < 0) atomicOr(err, DERR_HASH_FULL);
  else lvals[s] = i;
}

// Neigh24 of every cell (octree.cpp:2764-2975): direction order x+, x-, y+, y-, z+, z-;
// a finer neighbour contributes the 4 cells on the shared face in the reference's order
__global__ void neigh24_build(int m, int bc, const uint64_t *__restrict__ ccode,
                              const uint64_t *__restrict__ hkeys, int hcap,
                              const uint64_t *__restrict__ lkeys, const int *__restrict__ lvals,
                              int lcap, int *nb24, int *nnb, int *err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const uint64_t code = ccode[i];
  const int L = code_level(code);
  const int order[6] = {0, 1, 3, 2, 4, 5};
  // faces of a finer neighbour adjacent to this cell, indexed by link direction
  const int quad[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {2, 3, 6, 7}, {0, 1, 4, 5}, {0, 2, 4, 6}, {1, 3, 5, 7}};
  int k = 0;
  for (int dd = 0; dd < 6; ++dd) {
    const int di = order[dd];
    uint64_t nc;
    if (!neighbour_code(code, L, di, bc, &nc)) {
      atomicOr(err, DERR_NEIGH);  // non-periodic boundary cells are not produced here
      continue;
    }
    const bool exists = (L == 0) || hash_find(hkeys, hcap, nc >> 3) >= 0;
    if (exists) {
      int s = hash_find(lkeys, lcap, nc);
      if (s >= 0) {
        nb24[24 * (size_t)i + k++] = lvals[s];
      } else {
        for (int a = 0; a < 4; ++a) {
          int s2 = hash_find(lkeys, lcap, (nc << 3) | (uint64_t)quad[di][a]);
          if (s2 < 0) { atomicOr(err, DERR_NEIGH); continue; }
          nb24[24 * (size_t)i + k++] = lvals[s2];
        }
      }
    } else {
      int s = hash_find(lkeys, lcap, nc >> 3);
      if (s < 0) { atomicOr(err, DERR_NEIGH); continue; }
      nb24[24 * (size_t)i + k++] = lvals[s];
    }
  }
  nnb[i] = k;
}

int next_pow2(long long v) {
  long long p = 1;
  while (p < v) p <<= 1;
  return (int)std::min<long long>(p, 1ll << 30);
}

int grid_for(long long n) { return (int)std::max<long long>(1, (n + kT - 1) / kT); }

}  // namespace

static int read_int(apc_context *c, const int *dev, int *host) {
  APC_CUDA_TRY(c, cudaMemcpyAsync(c->h_pinned, dev, sizeof(int), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, apc_stream_wait(c));
  *host = c->h_pinned[0];
  return APC_OK;
}

static int ensure_open_cap(apc_context *c, long long need) {
  if (need <= c->op_cap) return APC_OK;
  long long cap = std::max<long long>(need, 2ll * c->op_cap);
  // grow preserving contents
  uint64_t *nc = nullptr;
  int *nb = nullptr, *nf = nullptr, *nn = nullptr;
  APC_TRY(apc_alloc(c, (void **)&nc, sizeof(uint64_t) * cap));
  APC_TRY(apc_alloc(c, (void **)&nb, sizeof(int) * cap));
  APC_TRY(apc_alloc(c, (void **)&nf, sizeof(int) * cap));
  APC_TRY(apc_alloc(c, (void **)&nn, sizeof(int) * cap));
  if (c->op_cap > 0) {
    APC_CUDA_TRY(c, cudaMemcpyAsync(nc, c->op_code, sizeof(uint64_t) * c->op_cap, cudaMemcpyDeviceToDevice, c->s));
    APC_CUDA_TRY(c, cudaMemcpyAsync(nb, c->op_base, sizeof(int) * c->op_cap, cudaMemcpyDeviceToDevice, c->s));
    APC_CUDA_TRY(c, cudaMemcpyAsync(nf, c->op_first, sizeof(int) * c->op_cap, cudaMemcpyDeviceToDevice, c->s));
    APC_CUDA_TRY(c, cudaMemcpyAsync(nn, c->op_count, sizeof(int) * c->op_cap, cudaMemcpyDeviceToDevice, c->s));
    apc_free(c, c->op_code);
    apc_free(c, c->op_base);
    apc_free(c, c->op_first);
    apc_free(c, c->op_count);
  }
  c->op_code = nc;
  c->op_base = nb;
  c->op_first = nf;
  c->op_count = nn;
  c->op_cap = (int)cap;
  return APC_OK;
}

static int ensure_hash(apc_context *c, uint64_t **keys, void **vals, size_t val_size, int *cap, int want) {
  if (want > *cap) {
    apc_free(c, *keys);
    apc_free(c, *vals);
    *keys = nullptr;
    *vals = nullptr;
    APC_TRY(apc_alloc(c, (void **)keys, sizeof(uint64_t) * (size_t)want));
    APC_TRY(apc_alloc(c, vals, val_size * (size_t)want));
    *cap = want;
  }
  return APC_OK;
}

// One attempt at the whole selection with the current hash capacities.
static int select_once(apc_context *c, int *hash_full) {
  const int n = c->n, D = c->cfg.depth;
  const double cc = c->cfg.gfd_c;
  *hash_full = 0;
  APC_CUDA_TRY(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->s));
  APC_CUDA_TRY(c, cudaMemsetAsync(c->h_keys, 0, sizeof(uint64_t) * c->hcap, c->s));

  // ---- level 0 (octree.cpp:1114-1160, 1165-1183) ----
  double temp = 1.0 * n;
  temp = temp * c->h0;
  temp = temp * c->h0;
  const bool root_open = n > 0 && temp > cc && 0 < D;
  c->td_level_off.assign(1, 0);
  APC_TRY(ensure_open_cap(c, 1024));
  int n_open = 0;
  if (root_open) {
    td_root<<<1, 1, 0, c->s>>>(c->op_code, c->op_base, c->op_first, c->op_count, n, c->h_keys,
                               c->h_vals, c->hcap, c->d_err);
    apc_count_launch(c);
    n_open = 1;
  }
  c->td_level_off.push_back(n_open);

  // ---- top-down, level by level ----
  int maxlev = 0;  // level of the last temp node (octree.cpp:1792 ml)
  for (int L = 0; L < D; ++L) {
    const int off = c->td_level_off[L], cnt = c->td_level_off[L + 1] - off;
    if (cnt == 0) break;
    // children at level L + 1 need the particles sorted by that many levels of key bits
    if (L + 1 > c->sorted_levels) return APC_RETRY_FULL_SORT;
    maxlev = L + 1;
    const long long m8 = 8ll * cnt;
    APC_TRY(apc_ensure(c, &c->flags, (size_t)(3 * m8 + 1), nullptr));
    int *flg = c->flags, *cf = c->flags + m8, *cn = c->flags + 2 * m8;
    APC_TRY(apc_ensure(c, &c->scan_tmp, 16, nullptr));
    const double hchild = ldexp(c->h0, -(L + 1));
    td_expand<<<grid_for(m8), kT, 0, c->s>>>(c->keys, D, L, off, cnt, c->op_first, c->op_count,
                                              hchild, cc, D, flg, cf, cn);
    apc_count_launch(c);
    APC_CUDA_TRY(c, cudaGetLastError());
    int *pos = nullptr;
    APC_TRY(apc_ensure(c, &c->req_pos, (size_t)m8 + 1, nullptr));
    pos = c->req_pos;
    APC_TRY(apc_exclusive_scan(c, flg, pos, (int)m8, c->counters));
    int total = 0;
    APC_TRY(read_int(c, c->counters, &total));
    const int off_next = off + cnt;
    APC_TRY(ensure_open_cap(c, (long long)off_next + total + 1));
    if (total > 0) {
      td_compact<<<grid_for(m8), kT, 0, c->s>>>(off, cnt, off_next, flg, pos, cf, cn, c->op_code,
                                                 c->op_base, c->op_first, c->op_count, c->h_keys,
                                                 c->h_vals, c->hcap, c->d_err);
      apc_count_launch(c);
    }
    c->td_level_off.push_back(off_next + total);
  }
  const int n_open_td = c->td_level_off.back();
  c->n_open_td = n_open_td;
  c->levels_hint = maxlev;
  n_open = n_open_td;
  const int child_base_bal = 1 + 8 * n_open_td;  // j after the top-down sweep

  // ---- bottom-up 2:1 balance, sweeps ln = maxlev .. 2 ----
  int n_events = 0;
  for (int ln = maxlev; ln > 1; --ln) {
    const int lv = ln - 1;
    const int td_a = lv < (int)c->td_level_off.size() - 1 ? c->td_level_off[lv] : n_open_td;
    const int td_b = lv < (int)c->td_level_off.size() - 1 ? c->td_level_off[lv + 1] : n_open_td;
    const int bal_a = n_open_td, bal_b = n_open;
    const long long nthreads = 8ll * ((td_b - td_a) + (bal_b - bal_a));
    if (nthreads == 0) continue;
    APC_CUDA_TRY(c, cudaMemsetAsync(c->r_keys, 0, sizeof(uint64_t) * c->rcap, c->s));
    APC_CUDA_TRY(c, cudaMemsetAsync(c->r_vals, 0xff, sizeof(uint64_t) * c->rcap, c->s));
    bal_requests<<<grid_for(nthreads), kT, 0, c->s>>>(ln, td_a, td_b, bal_a, bal_b, c->cfg.bc, c->op_code,
                                                      c->op_base, c->h_keys, c->hcap, c->r_keys,
                                                      (unsigned long long *)c->r_vals, c->rcap, c->d_err);
    apc_count_launch(c);
    APC_CUDA_TRY(c, cudaGetLastError());
    APC_CUDA_TRY(c, cudaMemsetAsync(c->counters, 0, sizeof(int), c->s));
    APC_TRY(apc_ensure(c, &c->req_key, (size_t)c->rcap, nullptr));
    APC_TRY(apc_ensure(c, &c->req_key_alt, (size_t)c->rcap, nullptr));
    APC_TRY(apc_ensure(c, &c->req_idx, (size_t)c->rcap, nullptr));
    APC_TRY(apc_ensure(c, &c->req_idx_alt, (size_t)c->rcap, nullptr));
    APC_TRY(apc_ensure(c, &c->req_code, (size_t)c->rcap, nullptr));
    bal_collect<<<grid_for(c->rcap), kT, 0, c->s>>>(c->r_keys, (const unsigned long long *)c->r_vals,
                                                     c->rcap, c->counters, c->req_key, c->req_idx,
                                                     c->req_code);
    apc_count_launch(c);
    int nreq = 0;
    APC_TRY(read_int(c, c->counters, &nreq));
    if (nreq == 0) continue;
    bool alt = false;
    APC_TRY(apc_radix_sort_u64(c, c->req_key, c->req_idx, c->req_key_alt, c->req_idx_alt, nreq, 0, 40, &alt));
    const uint32_t *order = alt ? c->req_idx_alt : c->req_idx;
    APC_TRY(ensure_open_cap(c, (long long)n_open + nreq + 1));
    bal_commit<<<grid_for(nreq), kT, 0, c->s>>>(nreq, n_open, child_base_bal + 8 * n_events, order,
                                                c->req_code, c->keys, n, D, c->op_code, c->op_base,
                                                c->op_first, c->op_count, c->h_keys, c->h_vals,
                                                c->hcap, c->d_err);
    apc_count_launch(c);
    APC_CUDA_TRY(c, cudaGetLastError());
    n_open += nreq;
    n_events += nreq;
    if (2ll * n_open > c->hcap) { *hash_full = 1; return APC_OK; }
  }
  c->n_open = n_open;
  // a full hash table is read with the output's errors below: every probe is bounded, so
  // the output pass runs safely on an incomplete table, and the selection is then redone
  int derr = 0;

  // ---- output cells ----
  if (n_open == 0) {
    // the root is the only cell (octree.cpp:1785-1788 leaf[0] = 1)
    APC_TRY(apc_ensure(c, &c->cx, 1, nullptr));
    c->nc = 1;
    c->nv = 0;
    c->nb = 0;
    return APC_ERR_UNSUPPORTED;
  }
  const long long m8 = 8ll * n_open;
  APC_TRY(apc_ensure(c, &c->flags, (size_t)m8 + 1, nullptr));
  APC_TRY(apc_ensure(c, &c->req_pos, (size_t)m8 + 1, nullptr));
  leaf_flags<<<grid_for(m8), kT, 0, c->s>>>(n_open, c->op_code, c->h_keys, c->hcap, c->flags);
  apc_count_launch(c);
  APC_TRY(apc_exclusive_scan(c, c->flags, c->req_pos, (int)m8, c->counters));
  int M = 0, nc = 0;
  // the cell count and the computational-cell count in one round trip
  APC_CUDA_TRY(c, cudaMemcpyAsync(c->h_pinned, c->counters, sizeof(int), cudaMemcpyDeviceToHost, c->s));
  if (8ll * n_open_td < m8)
    APC_CUDA_TRY(c, cudaMemcpyAsync(c->h_pinned + 3, c->req_pos + 8ll * n_open_td, sizeof(int),
                                    cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, apc_stream_wait(c));
  M = c->h_pinned[0];
  nc = (8ll * n_open_td < m8) ? c->h_pinned[3] : M;
  c->nc = nc;
  c->nv = M - nc;
  c->nb = 0;
  // capacities for cells
  const size_t mc = (size_t)M + 1;
  APC_TRY(apc_ensure(c, &c->cx, mc, nullptr));
  APC_TRY(apc_ensure(c, &c->cy, mc, nullptr));
  APC_TRY(apc_ensure(c, &c->cz, mc, nullptr));
  APC_TRY(apc_ensure(c, &c->ch, mc, nullptr));
  APC_TRY(apc_ensure(c, &c->cfirst, mc, nullptr));
  APC_TRY(apc_ensure(c, &c->ccount, mc, nullptr));
  APC_TRY(apc_ensure(c, &c->ctype, mc, nullptr));
  APC_TRY(apc_ensure(c, &c->ccode, mc, nullptr));
  APC_TRY(apc_ensure(c, &c->nnb, mc, nullptr));
  APC_TRY(apc_ensure(c, &c->nb24, 24 * mc, nullptr));
  const int want_l = next_pow2(2ll * M + 1024);
  APC_TRY(ensure_hash(c, &c->l_keys, (void **)&c->l_vals, sizeof(int), &c->lcap, want_l));
  APC_CUDA_TRY(c, cudaMemsetAsync(c->l_keys, 0, sizeof(uint64_t) * c->lcap, c->s));
  leaf_emit<<<grid_for(m8), kT, 0, c->s>>>(n_open, n_open_td, c->flags, c->req_pos, c->op_code, c->keys, n,
                                            D, c->cx0, c->cy0, c->cz0, c->hx0, c->hy0, c->hz0, c->h0,
                                            c->cx, c->cy, c->cz, c->ch, c->cfirst, c->ccount, c->ctype,
                                            c->ccode, c->l_keys, c->l_vals, c->lcap, c->d_err);
  neigh24_build<<<grid_for(M), kT, 0, c->s>>>(M, c->cfg.bc, c->ccode, c->h_keys, c->hcap, c->l_keys,
                                               c->l_vals, c->lcap, c->nb24, c->nnb, c->d_err);
  apc_count_launch(c, 2);
  APC_CUDA_TRY(c, cudaGetLastError());
  APC_TRY(apc_read_errors(c, &derr));
  if (derr & DERR_HASH_FULL) { *hash_full = 1; return APC_OK; }
  if (derr & DERR_NOT_FINITE) {
    c->err = "non-finite particle coordinates";
    return APC_ERR_NOT_FINITE;
  }
  if (derr & DERR_NEIGH) {
    c->err = c->cfg.bc == 1 ? "2:1 face neighbour missing in the selected cell set"
                             : "non-periodic boundary cells are not supported";
    return c->cfg.bc == 1 ? APC_ERR_CUDA : APC_ERR_UNSUPPORTED;
  }
  return APC_OK;
}

int apc_selection(apc_context *c) {
  // hash capacities: opened nodes are ~1/7 of the cells; start generously and double
  // on overflow (the device reports a full table instead of probing without bound)
  int want_h = next_pow2(std::max<long long>(1 << 16, (long long)c->n / 2));
  for (int attempt = 0; attempt < 8; ++attempt) {
    APC_TRY(ensure_hash(c, &c->h_keys, (void **)&c->h_vals, sizeof(int), &c->hcap, want_h));
    APC_TRY(ensure_hash(c, &c->r_keys, (void **)&c->r_vals, sizeof(uint64_t), &c->rcap, want_h));
    int full = 0;
    int rc = select_once(c, &full);
    if (rc != APC_OK) return rc;
    if (!full) {
      // temp-node budget of the reference (mover.cpp:20,36-41, octree.cpp:1781-1782):
      // the run fails when 1 + 8 * opened + 8 exceeds the budget, which doubles while
      // below the cap
      if (c->cfg.nmax_cap > 0 && c->n_open > 0) {
        const long long need = 1ll + 8ll * c->n_open + 8;
        int ok = 0;
        while (!ok && c->maxnc_state < c->cfg.nmax_cap) {
          if (need <= c->maxnc_state) ok = 1;
          else c->maxnc_state *= 2;
        }
        if (!ok) {
          c->err = "selection needs more temp nodes than the budget cap allows";
          return APC_ERR_NMAX;
        }
      }
      return APC_OK;
    }
    want_h *= 2;
  }
  c->err = "selection hash tables kept overflowing";
  return APC_ERR_OUT_OF_MEMORY;
}
