// GFD stencils, density / Poisson system assembly and differentiation on the device.
//
// Reference: Solver::Build_Linear_System (solver.cpp:24-180), Solver::searchneighboroctant
// (solver.cpp:456-570), Solver::Solve_Potential's right-hand side (solver.cpp:236-259)
// and Solver::Differentiate (solver.cpp:295-362).
//
// One warp per cell (computational or vacuum particle), except where noted:
//  * Neighbour search.  The cell's Neigh24 entries are bucketed into 8 octants of a
//    slightly rotated frame, then grown ring by ring through the neighbours' Neigh24
//    lists until at least lm candidates exist.  Discovery order is kept exactly: one
//    warp-wide batch per candidate, ordered appends by ballot, duplicates removed
//    against the buckets and within the batch.  The rotation and distance products
//    are evaluated without FMA contraction, in the reference's operand order, so the
//    octant signs and distance ties are bit-identical.  A warp takes 12 consecutive
//    cells this way and stages their lists in shared memory; then one lane per cell
//    runs the reference's sort sequentially, exactly:
//      - quicksort of octant 0 only (solver.cpp:557 passes the running offset);
//      - 1e4^rank penalties within each octant;
//      - a global quicksort with the same partition scheme, so ties break identically.
//  * Least squares.  The lm x 9 weighted monomial matrix B (rows b_j) is solved through
//    the Cholesky factor of its Gram matrix G = B^T B; a cell whose pivots show cond(B)
//    over ~100 is solved by FP64 Householder QR instead
//    (one row per lane, warp-shuffle reductions).  Either way the full operator
//    X = G^-1 B^T W (9 x lm) is formed, i.e. the dgels solution for the lm right-hand
//    sides of solver.cpp:101-106, and kept for the differentiation step.  The second
//    neighbour search and QR of Solver::Differentiate (solver.cpp:307-342) repeat the
//    same computation, so they are not redone.
//  * Assembly.  A1 = I + (h^2/24) Lap and A2 = Lap go to slot-major ELL of width lm+1:
//    slot 0 is the diagonal, slot 1+j neighbour j.  Row 0 of A2 is the Dirichlet pin of
//    periodic boxes (solver.cpp:147-152).
#include <cuda_runtime.h>

#include <cmath>

#include "apc_internal.cuh"

namespace {

constexpr int kWarps = 4;         // warps per block of the least-squares phase
constexpr int kSearchWarps = 4;   // warps per block of the search phase
constexpr int kBucketCap = 48;    // entries per octant bucket
constexpr int kListCap = 256;     // candidates entering the final sort
constexpr int kMaxLm = 32;

struct GfdParams {
  int m, lm, bc, nc_nv, sort_cap;
  double L[3], halfL[3];
  double rot[9];
  double e4;       // exp(-4)
  double inv_1me4;  // 1 / (1 - exp(-4))
  double c_dens;
  const double *cx, *cy, *cz, *ch;
  const int *count, *type, *nb24, *nnb;
  int *st_idx;
  double *gx;  // per cell the 9 x lm least-squares operator X
  double *scr_d;  // per search warp: kListCap sort keys and indices (lists over 32)
  int *scr_i;
  int *qr_list, *qr_count;  // cells for the Householder pass
  int *chunk_next;          // the search's next unclaimed cell (zeroed before its launch)
  int *ell_col;
  double *a1, *a2, *rhs;
  size_t ld;  // ELL leading dimension (row capacity)
  int *err;
};

__device__ __forceinline__ double pwrap(double x, double L, double halfL) {
  // Solver::periodic_wrap (solver.cpp:574-594); |x| < L for points inside the box
  for (int k = 0; k < 4 && x >= halfL; ++k) x = __dsub_rn(x, L);
  for (int k = 0; k < 4 && x < -halfL; ++k) x = __dadd_rn(x, L);
  return x;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// apartition / aquickSort (solver.cpp:600-632) with an explicit stack.  Sub-ranges are
// disjoint, so processing order does not change the result; the smaller side is taken
// first, which bounds the stack by log2(n).  Only positions below `limit` are wanted:
// a sub-range starting at or beyond it only permutes unwanted positions, so it is not
// entered, and positions below the limit end exactly as in the full sort.
__device__ void aquicksort(double *a, int *b, int l, int r, int limit) {
  int stack[64];
  int sp = 0;
  for (;;) {
    if (l >= r || l >= limit) {
      if (sp == 0) break;
      r = stack[--sp];
      l = stack[--sp];
      continue;
    }
    double pivot = a[l], t;
    int i = l, j = r + 1, ti;
    for (;;) {
      do ++i; while (i <= r && a[i] <= pivot);
      do --j; while (a[j] > pivot);
      if (i >= j) break;
      t = a[i]; a[i] = a[j]; a[j] = t;
      ti = b[i]; b[i] = b[j]; b[j] = ti;
    }
    t = a[l]; a[l] = a[j]; a[j] = t;
    ti = b[l]; b[l] = b[j]; b[j] = ti;
    if (j - l < r - j) {
      stack[sp++] = j + 1;
      stack[sp++] = r;
      r = j - 1;
    } else {
      stack[sp++] = l;
      stack[sp++] = j - 1;
      l = j + 1;
    }
  }
}

// neighbour search, per warp: the candidates of the cell in hand, by octant bucket
// 16-byte aligned so that bucket rows (kBucketCap ints, a multiple of 4) can be read as int4
static_assert(kBucketCap % 4 == 0, "bucket rows are scanned four entries at a time");
struct __align__(16) WarpSmem {
  int soff[32], sp[32];  // expansion ring: item offset and cell of each candidate
  int bidx[8][kBucketCap];
};

// The search handles kChunk consecutive cells per warp: their lists (at most 32
// candidates each, the usual case) are staged here, then lane q sorts cell q's list
// sequentially.  Rows are padded to 33 entries so that lanes at the same position fall
// in different banks.  12 cells per warp keep a block's shared memory at 28 KB, so 8
// blocks (32 warps) fit on an SM; at 128^3 this measured faster than 8 or 16 cells.
constexpr int kChunk = 12;
constexpr int kStageLd = 33;
struct SortStage {
  double key[kChunk][kStageLd];
  int idx[kChunk][kStageLd];
  int nn[kChunk][8];
  int staged[kChunk];
};

// Least squares, per warp: a slice of the dynamic shared memory laid out as
//   [0, A)            the Gram products b_r b_c (r <= c) of each row, 45 x lm (fast path),
//                     or the QR's column reductions red (9 x 32), sums (9) and R (9 x 9);
//   G (45), L (9 x 9), inv (9), the pivot flag.
// A = max(45 lm, 378) doubles, so the slice is only as large as lm needs.
struct LsqView {
  double *g45, *red, *sums, *R, *G, *L, *inv;
  int *chol_ok;
};

__host__ __device__ constexpr int lsq_area(int lm) { return 45 * lm > 378 ? 45 * lm : 378; }
__host__ __device__ constexpr int lsq_doubles(int lm) { return (lsq_area(lm) + 45 + 81 + 9 + 1 + 1) & ~1; }

__device__ __forceinline__ LsqView lsq_view(double *base, int lm) {
  LsqView v;
  v.g45 = base;
  v.red = base;
  v.sums = base + 9 * 32;
  v.R = base + 9 * 32 + 9;
  v.G = base + lsq_area(lm);
  v.L = v.G + 45;
  v.inv = v.L + 81;
  v.chol_ok = reinterpret_cast<int *>(v.inv + 9);
  return v;
}

// position of (r, c), r <= c, in the row-major upper triangle of a 9 x 9 matrix
__host__ __device__ constexpr int tri(int r, int c) { return r * 9 - r * (r - 1) / 2 + (c - r); }

__device__ __forceinline__ void offset_of(const GfdParams &P, int m, int i0, double &wx, double &wy,
                                          double &wz) {
  wx = pwrap(__dsub_rn(P.cx[m], P.cx[i0]), P.L[0], P.halfL[0]);
  wy = pwrap(__dsub_rn(P.cy[m], P.cy[i0]), P.L[1], P.halfL[1]);
  wz = pwrap(__dsub_rn(P.cz[m], P.cz[i0]), P.L[2], P.halfL[2]);
}

__device__ __forceinline__ int octant_of(const GfdParams &P, double wx, double wy, double wz) {
  const double *A = P.rot;
  double xt = __dadd_rn(__dadd_rn(__dmul_rn(A[0], wx), __dmul_rn(A[1], wy)), __dmul_rn(A[2], wz));
  double yt = __dadd_rn(__dadd_rn(__dmul_rn(A[3], wx), __dmul_rn(A[4], wy)), __dmul_rn(A[5], wz));
  double zt = __dadd_rn(__dadd_rn(__dmul_rn(A[6], wx), __dmul_rn(A[7], wy)), __dmul_rn(A[8], wz));
  return (xt > 0) + 2 * (yt > 0) + 4 * (zt > 0);
}

__device__ __forceinline__ double sq3(double wx, double wy, double wz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(wx, wx), __dmul_rn(wy, wy)), __dmul_rn(wz, wz));
}

// ordered append of the valid lanes' candidates to their octant buckets: a lane's slot is
// its bucket's fill plus the number of lower valid lanes of the same octant
__device__ __forceinline__ bool append(WarpSmem &S, int (&nn)[8], bool valid, int m, int oct, int lane) {
  bool ok = true;
  const unsigned lt = (1u << lane) - 1u;
  // invalid lanes get keys no octant has, so they match only themselves
  const unsigned peers = __match_any_sync(0xffffffffu, valid ? oct : 8 + lane);
  if (valid) {
    int base = 0;
#pragma unroll
    for (int o = 0; o < 8; ++o) base = (oct == o) ? nn[o] : base;
    const int p = base + __popc(peers & lt);
    if (p < kBucketCap) S.bidx[oct][p] = m;
  }
#pragma unroll
  for (int o = 0; o < 8; ++o) {
    nn[o] += __popc(__ballot_sync(0xffffffffu, valid && oct == o));
    if (nn[o] > kBucketCap) ok = false;
  }
  __syncwarp();
  return ok;
}

// sums[c] = sum over the lanes of val[c], c in [c0, 9).  Every lane stores its values;
// then g lanes per column (4 for up to 8 columns, 2 for 9) each add a chunk of rows in
// row order, and the chunks are combined by a fixed shuffle tree.  Fewer instructions
// than one 5-step butterfly per column; the order is fixed, so results are reproducible.
__device__ __forceinline__ void col_sums(const LsqView &S, const double (&val)[9], int c0, int lane) {
#pragma unroll
  for (int c = 0; c < 9; ++c)
    if (c >= c0) S.red[c * 32 + lane] = val[c];
  __syncwarp();
  const int ncol = 9 - c0;
  const int g = ncol <= 8 ? 4 : 2;
  const int rows = 32 / g;
  const int col = c0 + lane / g, chunk = lane % g;
  double t = 0.0;
  if (col < 9) {
    const double *r = &S.red[col * 32 + chunk * rows];
    for (int q = 0; q < rows; ++q) t += r[q];
  }
  for (int o = 1; o < g; o <<= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if (col < 9 && chunk == 0) S.sums[col] = t;
  __syncwarp();
}

// Solver::searchneighboroctant's sort (solver.cpp:553-569) of one cell's candidate list,
// given in bucket order (octant 0's entries, then octant 1's, ...) with raw squared
// distances as keys, sequentially as the reference runs it: the quicksort of octant 0
// (solver.cpp:557 passes the running offset, so only octant 0's run is sorted), the
// 1e4^rank penalties within each octant, then the quicksort of the whole list.  Positions
// below lm end as in the reference; the rest are not needed.
__device__ void reference_sort(double *key, int *idx, const int *nn, int l, int lm) {
  aquicksort(key, idx, 0, nn[0] - 1, nn[0]);
  int k = 0;
  for (int b = 0; b < 8; ++b) {
    double penalty = 1.0;
    for (int e = 0; e < nn[b]; ++e) {
      key[k] = __dmul_rn(penalty, key[k]);
      penalty = __dmul_rn(penalty, 10000.0);
      ++k;
    }
  }
  aquicksort(key, idx, 0, l - 1, lm);
}

// Phase 1: the neighbour search and the reference's sort; the first lm candidates go to
// st_idx.  A warp takes kChunk consecutive cells.  For each in turn the whole warp finds
// the candidates (rings of Neigh24 lists, discovery order kept per octant); a list of at
// most 32 candidates is staged in shared memory.  Then lane q runs cell q's sort
// (reference_sort), and the warp writes the chunk's stencils with coalesced stores.
// Longer lists are sorted at once by lane 0 in a global scratch slice.  A cell whose
// search fails raises its flag and gets its own index in every slot, so that phase 2
// stays in bounds (the step then fails).
__global__ void __launch_bounds__(32 * kSearchWarps, 8) gfd_search(GfdParams P) {
  __shared__ WarpSmem smem[kSearchWarps];
  __shared__ SortStage stage[kSearchWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  WarpSmem &S = smem[w];
  SortStage &T = stage[w];
  const int lm = P.lm;
  const int gw = blockIdx.x * kSearchWarps + w;
  // chunks are claimed from a counter: late in a run the cost per cell varies widely along
  // the Morton order, and a fixed assignment left warps with runs of costly cells
  for (;;) {
    int c0 = 0;
    if (lane == 0) c0 = atomicAdd(P.chunk_next, kChunk);
    c0 = __shfl_sync(0xffffffffu, c0, 0);
    if (c0 >= P.m) break;
    const int nq = min(kChunk, P.m - c0);
    // the next cell's Neigh24 row is loaded while the current cell is searched
    int cnt_next = P.nnb[c0];
    int m_next = lane < cnt_next ? P.nb24[24 * (size_t)c0 + lane] : -1;
    for (int q = 0; q < nq; ++q) {
      const int i0 = c0 + q;
      int nn[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      bool ok = true;   // false once a bucket overflowed
      bool few = false; // true when 5 expansions did not reach lm candidates
      // ---- first ring: Neigh24 of i0 (solver.cpp:479-492), no de-duplication ----
      {
        const int cnt = cnt_next;
        const bool v = lane < cnt;
        const int m = m_next;
        if (q + 1 < nq) {
          cnt_next = P.nnb[i0 + 1];
          m_next = lane < cnt_next ? P.nb24[24 * (size_t)(i0 + 1) + lane] : -1;
        }
        int oct = 0;
        if (v) {
          double wx, wy, wz;
          offset_of(P, m, i0, wx, wy, wz);
          oct = octant_of(P, wx, wy, wz);
        }
        ok &= append(S, nn, v, m, oct, lane);
      }
      int l = 0;
#pragma unroll
      for (int o = 0; o < 8; ++o) l += nn[o];
      // ---- expansion rings (solver.cpp:494-552) ----
      int ite = 0;
      while (ok && l < lm) {
        // the reference exits on its sixth expansion whatever it finds (solver.cpp:544-550)
        if (ite == 5) {
          few = true;
          break;
        }
        // the ring's (candidate, Neigh24 entry) items in the reference's order, processed
        // 32 at a time: candidates of the snapshot are < lm <= 32, so one lane holds each
        int pre[9];
        pre[0] = 0;
#pragma unroll
        for (int o = 0; o < 8; ++o) pre[o + 1] = pre[o] + nn[o];
        const int lsnap = pre[8];
        int pc = 0, cc = 0;
        if (lane < lsnap) {
          int b = 0;
#pragma unroll
          for (int o = 1; o < 8; ++o) b += (lane >= pre[o]) ? 1 : 0;
          pc = S.bidx[b][lane - pre[b]];
          cc = P.nnb[pc];
        }
        int incl = cc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += t;
        }
        S.soff[lane] = incl - cc;
        S.sp[lane] = pc;
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        __syncwarp();
        for (int f0 = 0; f0 < total && ok; f0 += 32) {
          const int f = f0 + lane;
          bool v = f < total;
          int m = -1, oct = 0;
          if (v) {
            // the snapshot candidate whose Neigh24 list holds item f: the last q with
            // soff[q] <= f (soff is a non-decreasing exclusive scan, soff[0] = 0 <= f), by
            // binary search
            int c = 0;
            for (int step = 16; step > 0; step >>= 1)
              if (c + step < lsnap && S.soff[c + step] <= f) c += step;
            m = P.nb24[24 * (size_t)S.sp[c] + (f - S.soff[c])];
            double wx, wy, wz;
            offset_of(P, m, i0, wx, wy, wz);
            oct = octant_of(P, wx, wy, wz);
            bool dup = (m == i0);
            const int cap = min(nn[oct], kBucketCap);
            // membership among the bucket's first cap entries, four per shared-memory load
            for (int t = 0; t < cap && !dup; t += 4) {
              const int4 e = *reinterpret_cast<const int4 *>(&S.bidx[oct][t]);
              dup = (e.x == m) | ((t + 1 < cap) & (e.y == m)) | ((t + 2 < cap) & (e.z == m)) |
                    ((t + 3 < cap) & (e.w == m));
            }
            v = !dup;
          }
          // only the first lane holding a given index survives within the chunk
          const unsigned peers = __match_any_sync(0xffffffffu, v ? m : -1 - lane);
          if (v && lane != __ffs(peers) - 1) v = false;
          ok &= append(S, nn, v, m, oct, lane);
        }
        if (!ok) break;
        ++ite;
        l = 0;
#pragma unroll
        for (int o = 0; o < 8; ++o) l += nn[o];
      }
      if (few || !ok || l > P.sort_cap) {
        if (lane == 0) {
          atomicOr(P.err, few ? DERR_STENCIL_FEW : DERR_STENCIL_MANY);
          T.staged[q] = 0;
        }
        if (lane < lm) P.st_idx[(size_t)i0 * lm + lane] = i0;
        __syncwarp();
        continue;
      }
      // ---- the list in bucket order, keyed by the squared distances (recomputed from
      //      the indices by the same operations as at discovery) ----
      {
        int v = 0;
#pragma unroll
        for (int o = 0; o < 8; ++o)
          if (lane == o) v = nn[o];
        if (lane < 8) T.nn[q][lane] = v;
        __syncwarp();
      }
      if (l <= 32) {
        int e = lane, m = i0;
        double d2 = 0.0;
        if (lane < l) {
          int b = 0;
#pragma unroll
          for (int o = 0; o < 8; ++o) {
            if (b == o && e >= nn[o]) {
              e -= nn[o];
              b = o + 1;
            }
          }
          m = S.bidx[b][e];
          double wx, wy, wz;
          offset_of(P, m, i0, wx, wy, wz);
          d2 = sq3(wx, wy, wz);
          T.key[q][lane] = d2;
          T.idx[q][lane] = m;
        }
        if (lane == 0) T.staged[q] = l;
      } else {
        // a longer list: the warp writes it in bucket order to this warp's slice of a global
        // scratch list, 32 entries at a time; lane 0 sorts it now
        double *ldist = P.scr_d + (size_t)gw * kListCap;
        int *lidx = P.scr_i + (size_t)gw * kListCap;
        int pre[9];
        pre[0] = 0;
#pragma unroll
        for (int o = 0; o < 8; ++o) pre[o + 1] = pre[o] + nn[o];
        for (int p = lane; p < l; p += 32) {
          int b = 0, base = 0;
#pragma unroll
          for (int o = 1; o < 8; ++o)
            if (p >= pre[o]) {
              b = o;
              base = pre[o];
            }
          const int m = S.bidx[b][p - base];
          double wx, wy, wz;
          offset_of(P, m, i0, wx, wy, wz);
          ldist[p] = sq3(wx, wy, wz);
          lidx[p] = m;
        }
        __threadfence_block();
        __syncwarp();
        if (lane == 0) {
          reference_sort(ldist, lidx, T.nn[q], l, lm);
          T.staged[q] = 0;
        }
        __threadfence_block();
        __syncwarp();
        if (lane < lm) P.st_idx[(size_t)i0 * lm + lane] = lidx[lane];
      }
      __syncwarp();
    }
    // ---- the staged lists: lane q sorts cell q's, then coalesced stores of the chunk ----
    if (lane < nq && T.staged[lane] > 0) reference_sort(T.key[lane], T.idx[lane], T.nn[lane], T.staged[lane], lm);
    __syncwarp();
    for (int t = lane; t < nq * lm; t += 32) {
      const int q = t / lm;
      if (T.staged[q] > 0) P.st_idx[(size_t)c0 * lm + t] = T.idx[q][t - q * lm];
    }
    __syncwarp();
  }
}

// Phase 2, one warp per cell: weights, the weighted monomial system, its FP64 Householder
// QR, the operator X and the matrix rows, from the stencil of phase 1.
// QR = false: every cell by the Cholesky fast path; a cell that fails its pivot check is
// queued.  QR = true: the queued cells by Householder QR.  The two instantiations keep
// their register budgets apart, so the fast path runs at higher occupancy.
template <bool QR>
__global__ void __launch_bounds__(32 * kWarps, QR ? 4 : 7) gfd_lsq(GfdParams P) {
  extern __shared__ __align__(16) double lsq_smem[];  // kWarps slices of lsq_doubles(lm)
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int lm = P.lm;
  const LsqView S = lsq_view(lsq_smem + (size_t)w * lsq_doubles(lm), lm);
  const int ncell = QR ? *P.qr_count : P.m;
  for (int it = blockIdx.x * kWarps + w; it < ncell; it += gridDim.x * kWarps) {
    const int i0 = QR ? P.qr_list[it] : it;
    // ---- weights and weighted monomials (solver.cpp:75-103) ----
    const bool act = lane < lm;
    const int mj = act ? P.st_idx[(size_t)i0 * lm + lane] : i0;
    double wx, wy, wz;
    offset_of(P, mj, i0, wx, wy, wz);
    const double dist = act ? sqrt(sq3(wx, wy, wz)) : 0.0;
    const double maxdis = warp_max(dist) * 0.7;
    double weight = 0.0;
    // the reference's divisions (solver.cpp:75-103) as products with reciprocals taken once
    // per cell: the same values to a few ulp, far inside the least squares' own rounding
    const double inv_m2 = 1.0 / (maxdis * maxdis);
    if (act) weight = (exp(-dist * dist * inv_m2) - P.e4) * P.inv_1me4;
    const double h = P.ch[i0];
    const double ih = 1.0 / h;
    const double p1 = wx * ih, p2 = wy * ih, p3 = wz * ih;
    double b[9];
    b[0] = p1; b[1] = p2; b[2] = p3;
    b[3] = p1 * p1 / 2.0; b[4] = p2 * p2 / 2.0; b[5] = p3 * p3 / 2.0;
    b[6] = p1 * p2; b[7] = p1 * p3; b[8] = p2 * p3;
#pragma unroll
    for (int k = 0; k < 9; ++k) b[k] = act ? b[k] * weight : 0.0;
    // ---- least squares, fast path: Cholesky factor of the Gram matrix B^T B.  The weighted
    //      monomial systems are well conditioned (cond(B) ~ 5-30 for lattice and octree
    //      stencils), so X = G^-1 B^T W agrees with the Householder solution to ~1e-14; a
    //      cell whose Cholesky pivots fall below 1e-4 of the diagonal (cond(B) over ~100)
    //      takes the Householder path below. ----
    double y[9];
    if (!QR) {
      int pidx = 0;
#pragma unroll
      for (int r = 0; r < 9; ++r)
#pragma unroll
        for (int c = r; c < 9; ++c) S.g45[(pidx++) * lm + lane] = b[r] * b[c];
      __syncwarp();
      for (int t = lane; t < 45; t += 32) {
        double sacc = 0.0;
        for (int q = 0; q < lm; ++q) sacc += S.g45[t * lm + q];
        S.G[t] = sacc;
      }
      if (lane == 0) *S.chol_ok = 1;
      __syncwarp();
      for (int k = 0; k < 9; ++k) {
        if (lane == 0) {
          double d = S.G[tri(k, k)];
          for (int j = 0; j < k; ++j) d -= S.L[k * 9 + j] * S.L[k * 9 + j];
          if (!(d > 1e-4 * S.G[tri(k, k)])) *S.chol_ok = 0;
          // 1 / L_kk by one reciprocal square root, L_kk = d / sqrt(d)
          const double dd = fmax(d, 1e-300);
          const double inv = rsqrt(dd);
          S.L[k * 9 + k] = dd * inv;
          S.inv[k] = inv;
        }
        __syncwarp();
        if (lane > k && lane < 9) {
          double t = S.G[tri(k, lane)];
          for (int j = 0; j < k; ++j) t -= S.L[lane * 9 + j] * S.L[k * 9 + j];
          S.L[lane * 9 + k] = t * S.inv[k];
        }
        __syncwarp();
      }
    }
    if (!QR && *S.chol_ok == 0) {
      if (lane == 0) P.qr_list[atomicAdd(P.qr_count, 1)] = i0;
      __syncwarp();
      continue;
    }
    if (!QR) {
      // lane j: y = G^-1 b_j by the two triangular solves.  The factor is read where it is
      // used (volatile): hoisting its 45 broadcast loads ahead of the dependent chain of
      // multiply-adds gains nothing and made the kernel spill its registers.
      double t9[9];
      const volatile double *VL = S.L, *VI = S.inv;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        double t = b[k];
#pragma unroll
        for (int j = 0; j < k; ++j) t -= VL[k * 9 + j] * t9[j];
        t9[k] = t * VI[k];
      }
#pragma unroll
      for (int k = 8; k >= 0; --k) {
        double t = t9[k];
#pragma unroll
        for (int j = k + 1; j < 9; ++j) t -= VL[j * 9 + k] * y[j];
        y[k] = t * VI[k];
      }
    } else {
    // ---- Householder QR, one row per lane ----
    double v[9], tau[9];
    bool rank_ok = true;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const double x = b[k];
      const double xn2 = warp_sum(lane > k ? x * x : 0.0);
      const double alpha = __shfl_sync(0xffffffffu, x, k);
      const double xnorm = sqrt(xn2);
      double beta = alpha, tk = 0.0, vr = (lane == k) ? 1.0 : 0.0;
      if (xnorm != 0.0) {
        beta = -copysign(hypot(alpha, xnorm), alpha);
        tk = (beta - alpha) / beta;
        const double scal = 1.0 / (alpha - beta);
        if (lane > k) vr = x * scal;
      }
      tau[k] = tk;
      v[k] = lane >= k ? vr : 0.0;
      if (lane == k) b[k] = beta;
      if (beta == 0.0) rank_ok = false;
      if (k < 8) {
        double pv[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) pv[c] = c > k ? v[k] * b[c] : 0.0;
        col_sums(S, pv, k + 1, lane);
#pragma unroll
        for (int c = k + 1; c < 9; ++c)
          if (lane >= k) b[c] = b[c] + v[k] * (-tk * S.sums[c]);
        __syncwarp();
      }
    }
    if (!rank_ok) {
      if (lane == 0) atomicOr(P.err, DERR_RANK);
      continue;
    }
    if (lane < 9) {
#pragma unroll
      for (int c = 0; c < 9; ++c) S.R[lane * 9 + c] = c >= lane ? b[c] : 0.0;
    }
    // ---- thin Q rows: Q1 = H0 H1 ... H8 [I; 0] (backward accumulation) ----
    double q[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) q[c] = (lane == c) ? 1.0 : 0.0;
#pragma unroll
    for (int k = 8; k >= 0; --k) {
      double pv[9];
#pragma unroll
      for (int c = 0; c < 9; ++c) pv[c] = c >= k ? v[k] * q[c] : 0.0;
      col_sums(S, pv, k, lane);
#pragma unroll
      for (int c = k; c < 9; ++c) q[c] = q[c] - tau[k] * v[k] * S.sums[c];
      __syncwarp();
    }
    __syncwarp();
    // ---- y = R^-1 Q1(j, :)^T, lane j ----
#pragma unroll
    for (int k = 8; k >= 0; --k) {
      double t = q[k];
#pragma unroll
      for (int c = k + 1; c < 9; ++c) t -= S.R[k * 9 + c] * y[c];
      y[k] = t / S.R[k * 9 + k];
    }
    }
    // ---- X(:, j) = w_j y ----
    double *X = P.gx + (size_t)i0 * 9 * lm;
    if (act) {
#pragma unroll
      for (int k = 0; k < 9; ++k) X[k * lm + lane] = weight * y[k];
    }
    // ---- rows of A1, A2 and the density rhs (solver.cpp:116-172) ----
    const double lap = act ? (weight * y[3] + weight * y[4]) + weight * y[5] : 0.0;
    const double l24 = lap * (1.0 / 24.0);
    const double lh2 = lap * (ih * ih);
    const bool in1 = act && mj < P.nc_nv;
    const bool in2 = act && P.type[mj] < 1;
    const bool pin = (i0 == 0) && (P.bc == 1);
    if (act) {
      const size_t at = (size_t)(1 + lane) * P.ld + i0;
      P.ell_col[at] = in1 ? mj : i0;
      P.a1[at] = in1 ? l24 : 0.0;
      P.a2[at] = (in2 && !pin) ? lh2 : 0.0;
    }
    // diagonal sums in the reference's sequential order
    double s1 = 0.0, s2 = 0.0;
    for (int j = 0; j < lm; ++j) {
      const double a = __shfl_sync(0xffffffffu, l24, j);
      const double c = __shfl_sync(0xffffffffu, lh2, j);
      s1 = s1 - a;
      s2 = s2 - c;
    }
    if (lane == 0) {
      const size_t at = (size_t)i0;
      P.ell_col[at] = i0;
      P.a1[at] = s1 + 1;
      P.a2[at] = pin ? 1.0 : s2;
      P.rhs[i0] = P.count[i0] * (ih * ih * ih) * P.c_dens;
    }
    __syncwarp();
  }
}

// -------------------------------------------------------------- potential rhs

__global__ void mass_partials(const double *__restrict__ rho, const double *__restrict__ h, int m,
                              double *partial) {
  __shared__ double s1[256], s2[256];
  double a = 0.0, b = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const double v = h[i] * h[i] * h[i];
    a += rho[i] * h[i] * h[i] * h[i];
    b += v;
  }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = b;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      s1[threadIdx.x] += s1[threadIdx.x + o];
      s2[threadIdx.x] += s2[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = s1[0];
    partial[2 * blockIdx.x + 1] = s2[0];
  }
}

// the volume-weighted mean density sum(rho h^3) / sum(h^3) (solver.cpp:244-251) from the
// blocks' partial sums, by one block in a fixed tree order (one thread summing them in
// sequence, in every block of the next kernel, took longer than the kernel's own work)
__global__ void mass_mean(const double *__restrict__ partial, int nparts, double *mean) {
  __shared__ double s1[256], s2[256];
  double a = 0.0, b = 0.0;
  for (int k = threadIdx.x; k < nparts; k += blockDim.x) {
    a += partial[2 * k];
    b += partial[2 * k + 1];
  }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = b;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      s1[threadIdx.x] += s1[threadIdx.x + o];
      s2[threadIdx.x] += s2[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *mean = s1[0] / s2[0];
}

// rhs = (rho - mean_volume_weighted(rho)) * c_pot (solver.cpp:244-259)
__global__ void potential_rhs_kernel(const double *__restrict__ rho, int m, const double *__restrict__ mean_p,
                                     double c_pot, double *rhs) {
  const double mean = *mean_p;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    rhs[i] = (rho[i] - mean) * c_pot;
}

__global__ void potential_rhs_dirichlet(const double *__restrict__ rho, const double *__restrict__ bc,
                                        int m, double c_pot, double *rhs) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    rhs[i] = (rho[i] + bc[i]) * c_pot;
}

// -------------------------------------------------------------- differentiate

// gradient / Hessian of phi: y = X (phi_j - phi_i) c_field (solver.cpp:315-358), one warp
// per cell.  X is stored by the least squares: rebuilding its columns here from a stored
// Cholesky factor (360 B per cell instead of 1,224) was measured slower, since the
// rows' weights and the per-lane solves cost more than the bytes they save.  Lane j forms
// the products X_kj (phi_j - phi_i) c_field in shared memory; lane k < 9 then sums row k in
// stencil order (one short chain instead of nine five-level shuffle trees).
constexpr int kDiffWarps = 8;
__global__ void __launch_bounds__(32 * kDiffWarps) differentiate_kernel(GfdParams P, const double *__restrict__ phi,
                                                                       double c_field, double *deriv) {
  __shared__ double prod[kDiffWarps][9][33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int lm = P.lm;
  for (int i = blockIdx.x * kDiffWarps + w; i < P.m; i += gridDim.x * kDiffWarps) {
    const double p4 = phi[i];
    double r = 0.0;
    if (lane < lm) {
      const int k = P.st_idx[(size_t)i * lm + lane];
      const double p1 = k < P.nc_nv ? phi[k] : 0.0;
      r = (p1 - p4) * c_field;
    }
    const double *X = P.gx + (size_t)i * 9 * lm;
    if (lane < lm) {
#pragma unroll
      for (int k = 0; k < 9; ++k) prod[w][k][lane] = X[k * lm + lane] * r;
    }
    __syncwarp();
    if (lane < 9) {
      double t = 0.0;
      for (int j = 0; j < lm; ++j) t += prod[w][lane][j];
      const double hi = P.ch[i];
      deriv[(size_t)i * 9 + lane] = lane < 3 ? t / hi : t / hi / hi;
    }
    __syncwarp();
  }
}

// the stencil distances |x_mj - x_i| (solver.cpp:567-569), as the least squares compute them
__global__ void stencil_dist_kernel(GfdParams P, double *__restrict__ dist) {
  const long long total = (long long)P.m * P.lm;
  for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < total;
       f += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(f / P.lm);
    double wx, wy, wz;
    offset_of(P, P.st_idx[f], i, wx, wy, wz);
    dist[f] = sqrt(sq3(wx, wy, wz));
  }
}

// the geometry, stencil and operator fields of GfdParams for context c
GfdParams gfd_params(apc_context *c) {
  GfdParams P{};
  const int M = c->nc + c->nv;
  P.m = M;
  P.lm = c->lm;
  P.bc = c->cfg.bc;
  P.nc_nv = M;
  P.sort_cap = std::min(kListCap, 10 * c->lm);
  for (int d = 0; d < 3; ++d) {
    P.L[d] = c->cfg.box[2 * d + 1] - c->cfg.box[2 * d];
    P.halfL[d] = c->cfg.bc == 1 ? 0.5 * P.L[d] : 1e308;
  }
  for (int k = 0; k < 9; ++k) P.rot[k] = c->rot[k];
  P.e4 = std::exp(-4.0);
  P.inv_1me4 = 1.0 / (1.0 - P.e4);
  P.cx = c->cx; P.cy = c->cy; P.cz = c->cz; P.ch = c->ch;
  P.count = c->ccount; P.type = c->ctype; P.nb24 = c->nb24; P.nnb = c->nnb;
  P.st_idx = c->st_idx; P.gx = c->gfd_x;
  return P;
}

}  // namespace

int apc_gfd_assemble(apc_context *c, double c_dens, int (*during)(apc_context *)) {
  const int M = c->nc + c->nv;
  const int lm = c->lm;
  if (lm > kMaxLm || lm < 9) {
    c->err = "lm must be in [9, 32]";
    return APC_ERR_INVALID_ARG;
  }
  const size_t mc = (size_t)M + 1;
  // a hierarchy built beside an earlier density solve belongs to the old operator
  apc_mg_clear_prebuilt(c);
  APC_TRY(apc_ensure(c, &c->st_idx, mc * lm, nullptr));
  APC_TRY(apc_ensure(c, &c->gfd_x, mc * 9 * lm, nullptr));
  c->ell_w = lm + 1;
  if ((size_t)c->m_cap < mc) {
    c->m_cap = (int)(mc + mc / 4 + 1024);
  }
  const size_t ld = (size_t)c->m_cap;
  APC_TRY(apc_ensure(c, &c->ell_col, ld * c->ell_w, nullptr));
  APC_TRY(apc_ensure(c, &c->a1, ld * c->ell_w, nullptr));
  APC_TRY(apc_ensure(c, &c->a2, ld * c->ell_w, nullptr));
  APC_TRY(apc_ensure(c, &c->rhs, ld, nullptr));
  APC_TRY(apc_ensure(c, &c->bcrhs, ld, nullptr));
  APC_TRY(apc_ensure(c, &c->density, ld, nullptr));
  APC_TRY(apc_ensure(c, &c->potential, ld, nullptr));
  APC_TRY(apc_ensure(c, &c->deriv, ld * 9, nullptr));
  APC_CUDA_TRY(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->s));
  APC_CUDA_TRY(c, cudaMemsetAsync(c->bcrhs, 0, sizeof(double) * M, c->s));
  GfdParams P = gfd_params(c);
  P.c_dens = c_dens;
  P.ell_col = c->ell_col; P.a1 = c->a1; P.a2 = c->a2; P.rhs = c->rhs;
  P.ld = ld;
  P.err = c->d_err;
  const int sblocks =
      std::max(1, std::min((M + kSearchWarps * kChunk - 1) / (kSearchWarps * kChunk), apc_sm_count(c) * 8));
  APC_TRY(apc_ensure(c, &c->gfd_scr_d, (size_t)sblocks * kSearchWarps * kListCap, nullptr));
  APC_TRY(apc_ensure(c, &c->gfd_scr_i, (size_t)sblocks * kSearchWarps * kListCap, nullptr));
  P.scr_d = c->gfd_scr_d;
  P.scr_i = c->gfd_scr_i;
  APC_TRY(apc_ensure(c, &c->gfd_qr, (size_t)M + 1, nullptr));
  P.qr_list = c->gfd_qr;
  P.qr_count = c->counters + 112;
  P.chunk_next = c->counters + 114;
  const int blocks = std::max(1, std::min((M + kWarps - 1) / kWarps, apc_sm_count(c) * 16));
  APC_CUDA_TRY(c, cudaMemsetAsync(P.chunk_next, 0, sizeof(int), c->s));
  APC_CUDA_TRY(c, cudaEventRecord(c->gev[0], c->s));
  gfd_search<<<sblocks, 32 * kSearchWarps, 0, c->s>>>(P);
  const size_t lsq_bytes = sizeof(double) * lsq_doubles(lm) * kWarps;
  APC_CUDA_TRY(c, cudaFuncSetAttribute(gfd_lsq<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)lsq_bytes));
  APC_CUDA_TRY(c, cudaFuncSetAttribute(gfd_lsq<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)lsq_bytes));
  APC_CUDA_TRY(c, cudaMemsetAsync(P.qr_count, 0, sizeof(int), c->s));
  gfd_lsq<false><<<blocks, 32 * kWarps, lsq_bytes, c->s>>>(P);
  // the queued cells, whatever their number: the kernel reads the count itself
  gfd_lsq<true><<<apc_sm_count(c) * 4, 32 * kWarps, lsq_bytes, c->s>>>(P);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaEventRecord(c->gev[1], c->s));
  apc_count_launch(c, 2);
  APC_CUDA_TRY(c, cudaGetLastError());
  if (during) APC_TRY(during(c));
  int derr = 0;
  APC_TRY(apc_read_errors(c, &derr));
  float gms = 0.f;
  APC_CUDA_TRY(c, cudaEventElapsedTime(&gms, c->gev[0], c->gev[1]));
  c->prof.gfd_ms += gms;
  if (derr & (DERR_STENCIL_FEW | DERR_STENCIL_MANY)) {
    c->err = (derr & DERR_STENCIL_FEW) ? "GFD neighbour search: not enough neighbours after 5 expansions"
                                       : "GFD neighbour search: candidate buffers exceeded";
    return APC_ERR_STENCIL;
  }
  if (derr & DERR_RANK) {
    c->err = "GFD least-squares system is rank deficient";
    return APC_ERR_RANK;
  }
  return APC_OK;
}

int apc_potential_rhs(apc_context *c, double c_pot) {
  const int M = c->nc + c->nv;
  const int G = std::max(1, std::min((M + 255) / 256, apc_sm_count(c) * 4));
  if (c->cfg.bc == 1) {
    APC_TRY(apc_ensure(c, &c->reduce_buf, (size_t)2 * G + 2, nullptr));
    mass_partials<<<G, 256, 0, c->s>>>(c->density, c->ch, M, c->reduce_buf);
    mass_mean<<<1, 256, 0, c->s>>>(c->reduce_buf, G, c->reduce_buf + 2 * G);
    potential_rhs_kernel<<<G, 256, 0, c->s>>>(c->density, M, c->reduce_buf + 2 * G, c_pot, c->rhs);
    apc_count_launch(c, 3);
  } else {
    potential_rhs_dirichlet<<<G, 256, 0, c->s>>>(c->density, c->bcrhs, M, c_pot, c->rhs);
    apc_count_launch(c);
  }
  APC_CUDA_TRY(c, cudaGetLastError());
  return APC_OK;
}

int apc_differentiate(apc_context *c, double c_field) {
  const int M = c->nc + c->nv;
  const int G = std::max(1, std::min((M + kDiffWarps - 1) / kDiffWarps, apc_sm_count(c) * 16));
  differentiate_kernel<<<G, 32 * kDiffWarps, 0, c->s>>>(gfd_params(c), c->potential, c_field, c->deriv);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaGetLastError());
  return APC_OK;
}

int apc_gfd_stencil_dist(apc_context *c) {
  const int M = c->nc + c->nv;
  APC_TRY(apc_ensure(c, &c->st_dist, (size_t)M * c->lm + 1, nullptr));
  const long long total = (long long)M * c->lm;
  const int G = (int)std::max<long long>(1, std::min<long long>((total + 255) / 256, apc_sm_count(c) * 6));
  stencil_dist_kernel<<<G, 256, 0, c->s>>>(gfd_params(c), c->st_dist);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaGetLastError());
  APC_CUDA_TRY(c, cudaStreamSynchronize(c->s));
  return APC_OK;
}
