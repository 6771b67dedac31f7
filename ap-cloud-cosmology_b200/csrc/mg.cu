// The mixed-precision solves: FP64 iterative refinement with FP32 Krylov corrections,
// run on the device as one CUDA graph per solve, and the multigrid preconditioner of the
// potential solve.
//
// The reference solves the Poisson system with GMRES + Jacobi (solver.cpp:267-276).  At
// 262k cells that reaches max_it before rtol (KSP_DIVERGED_ITS), in the reference and on
// the GPU alike.  The mixed path keeps the reference's stopping test on the FP64 residual
// ||D^-1 (b - A x)|| <= max(rtol ||D^-1 b||, atol), with dtol and max_it.  Each
// correction solves the Jacobi-scaled system (D^-1 A) d = D^-1 r / ||D^-1 r|| in FP32:
//   * Loops on the device.  The refinement loop and the (F)GMRES cycle are nested
//     conditional WHILE nodes of one graph; kernels hold every scalar (Hessenberg
//     column, Givens rotations, stopping tests) in device memory and set the loop
//     conditions, so a solve costs the host one launch and one readback.
//   * Aggregation by the octree.  A node of the next coarser level is the parent cell
//     (location code >> 3); its aggregate is the set of its children present on the
//     finer level.  Coarse node order is sorted location code, so Morton order.
//   * Galerkin coarse operators A_c = P^T A P, P piecewise constant, one warp per
//     coarse row: the members' (J, a_ij) contributions are sorted in shared memory by a
//     bitonic network and summed in sorted order, so the hierarchy is deterministic.
//     Rows sum to zero except the Dirichlet pin's aggregate, so the constant mode is
//     reproduced exactly on every level.
//   * Damped Jacobi smoothing on ELL operators, over-scaled coarse corrections; the
//     levels of <= 1024 nodes in one single-block kernel; an explicit dense inverse (FP64,
//     formed on the host) on the coarsest level of <= 64 nodes.
//   * Flexible GMRES with classical Gram-Schmidt (optionally a second, re-orthogonalising
//     sweep), right preconditioned, so the residual it monitors is the true residual of
//     the correction equation.  The SpMV is fused with the first dot-product pass.  The
//     density solve runs the same loop without a preconditioner.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <type_traits>
#include <vector>

#include "apc_internal.cuh"

namespace {

constexpr int kT = 256;
constexpr int kMaxLevels = 24;
constexpr int kCoarsest = 64;

int grid_for(long long n, int cap = 4096) {
  return (int)std::max<long long>(1, std::min<long long>((n + kT - 1) / kT, cap));
}

// ------------------------------------------------------------ hierarchy build

__global__ void parent_codes(int n, const uint64_t *__restrict__ code, uint64_t *__restrict__ key,
                             uint32_t *__restrict__ idx) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint64_t c = code[i];
    key[i] = c > 1ull ? (c >> 3) : 1ull;
    idx[i] = (uint32_t)i;
  }
}

__global__ void change_flags_u64(int n, const uint64_t *__restrict__ key, int *__restrict__ flag) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    flag[k] = (k == 0 || key[k] != key[k - 1]) ? 1 : 0;
}

// after the scan: aggregate map, coarse codes, member CSR of the coarse nodes
__global__ void aggregate_map(int n, const uint64_t *__restrict__ key, const uint32_t *__restrict__ idx,
                              const int *__restrict__ flag, const int *__restrict__ pos, int *__restrict__ agg,
                              uint64_t *__restrict__ ccode, int *__restrict__ mptr, int *__restrict__ mem) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int I = pos[k] + flag[k] - 1;  // inclusive count - 1
    agg[idx[k]] = I;
    mem[k] = (int)idx[k];
    if (flag[k]) {
      ccode[I] = key[k];
      mptr[I] = k;
    }
  }
}

template <class V>
__global__ void ell_dinv(int n, size_t ld, const V *__restrict__ val, V *__restrict__ dinv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const V d = val[i];
    dinv[i] = d != V(0) ? V(1) / d : V(1);
  }
}

// Galerkin row I of A_c = P^T A P, one warp per coarse row.  The (J, a) contributions of
// the members' rows are taken 32 at a time in member-then-slot order; lanes with equal J
// are merged by their lowest lane, which adds the values in lane order into a shared-
// memory hash table keyed by J (one writer per J per round, so every coarse entry is
// summed in contribution order).  The distinct entries are then written sorted by J.
// The result does not depend on scheduling, so the hierarchy is deterministic.
constexpr int kGalWarps = 4;
constexpr int kGalTab = 512;   // hash slots per warp
constexpr int kGalRows = 256;  // distinct coarse columns per row

template <class V>
__global__ void __launch_bounds__(32 * kGalWarps) galerkin_rows(int nc, const int *__restrict__ mptr, int nf,
                                                              const int *__restrict__ mem, int wf_host,
                                                              const int *__restrict__ wf_dev, int wf_cap, size_t ldf,
                                                              const int *__restrict__ colf,
                                                              const V *__restrict__ valf,
                                                              const int *__restrict__ agg, int wcap,
                                                              int *__restrict__ rowlen, int *__restrict__ tcol,
                                                              V *__restrict__ tval, int *__restrict__ err) {
  __shared__ int tkey[kGalWarps][kGalTab];
  __shared__ double tsum[kGalWarps][kGalTab];
  __shared__ double stage[kGalWarps][32];
  __shared__ int dkey[kGalWarps][kGalRows];
  __shared__ double dval[kGalWarps][kGalRows];
  // the fine level's width: from the device when that level was built just before (capped by
  // its ELL's slots: a wider level is flagged and the build repeated)
  const int wf = wf_dev ? min(*wf_dev, wf_cap) : wf_host;
  const int lane = threadIdx.x & 31, wv = threadIdx.x >> 5;
  int *K = tkey[wv];
  double *T = tsum[wv];
  for (int I = blockIdx.x * kGalWarps + wv; I < nc; I += gridDim.x * kGalWarps) {
    const int a = mptr[I], e = (I + 1 < nc) ? mptr[I + 1] : nf;
    const int cnt = (e - a) * wf;
    for (int t = lane; t < kGalTab; t += 32) K[t] = -1;
    __syncwarp();
    bool bad = false;
    for (int t0 = 0; t0 < cnt; t0 += 32) {
      const int t = t0 + lane;
      int J = -1;
      double v = 0.0;
      if (t < cnt) {
        const int i = mem[a + t / wf], sl = t % wf;
        const size_t at = (size_t)sl * ldf + i;
        J = agg[colf[at]];
        v = (double)valf[at];
      }
      stage[wv][lane] = v;
      __syncwarp();
      const unsigned peers = __match_any_sync(0xffffffffu, J);
      if (J >= 0 && lane == __ffs(peers) - 1) {
        double sum = 0.0;
        for (unsigned q = peers; q; q &= q - 1) sum += stage[wv][__ffs(q) - 1];
        unsigned h = ((unsigned)J * 2654435761u) >> (32 - 9);
        bool placed = false;
        for (int probe = 0; probe < kGalTab && !placed; ++probe, h = (h + 1) & (kGalTab - 1)) {
          const int cur = atomicCAS(&K[h], -1, J);
          if (cur == -1) {
            T[h] = sum;
            placed = true;
          } else if (cur == J) {
            T[h] += sum;
            placed = true;
          }
        }
        if (!placed) bad = true;
      }
      __syncwarp();
    }
    // compact the occupied slots, then place each by its rank in J
    int nd = 0;
    for (int t0 = 0; t0 < kGalTab; t0 += 32) {
      const int key = K[t0 + lane];
      const unsigned occ = __ballot_sync(0xffffffffu, key >= 0);
      const int pos = nd + __popc(occ & ((1u << lane) - 1u));
      if (key >= 0 && pos < kGalRows) {
        dkey[wv][pos] = key;
        dval[wv][pos] = T[t0 + lane];
      }
      nd += __popc(occ);
    }
    __syncwarp();
    const int len = min(nd, kGalRows);
    for (int q = lane; q < len; q += 32) {
      const int key = dkey[wv][q];
      int rank = 0;
      for (int u = 0; u < len; ++u) rank += dkey[wv][u] < key ? 1 : 0;
      if (rank < wcap) {
        tcol[(size_t)I * wcap + rank] = key;
        tval[(size_t)I * wcap + rank] = (V)dval[wv][q];
      }
    }
    bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) {
      rowlen[I] = nd;
      if (bad || nd > wcap || nd > kGalRows) atomicOr(err, DERR_STENCIL_MANY);
    }
    __syncwarp();
  }
}

template <class V>
__global__ void rows_to_ell(int n, const int *__restrict__ w_dev, int wslots, size_t ld, int wcap,
                            const int *__restrict__ rowlen, const int *__restrict__ tcol,
                            const V *__restrict__ tval, int *__restrict__ col, V *__restrict__ val,
                            V *__restrict__ dinv, int *__restrict__ overflow) {
  // the level's width (max_int, just before); the ELL holds wslots slots, and a wider level
  // is flagged (the build then runs again with room for it)
  const int wd = *w_dev;
  const int w = min(wd, wslots);
  if (wd > wslots && blockIdx.x == 0 && threadIdx.x == 0) atomicExch(overflow, 1);
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < n; I += gridDim.x * blockDim.x) {
    const int len = rowlen[I];
    V d = V(0);
    for (int s = 0; s < w; ++s) {
      const bool in = s < len;
      const int c = in ? tcol[(size_t)I * wcap + s] : I;
      const V v = in ? tval[(size_t)I * wcap + s] : V(0);
      col[(size_t)s * ld + I] = c;
      val[(size_t)s * ld + I] = v;
      if (in && c == I) d += v;
    }
    dinv[I] = d != V(0) ? V(1) / d : V(1);
  }
}

__global__ void max_int(int n, const int *__restrict__ a, int *out) {
  int m = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = max(m, a[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// The coarsest level's explicit inverse: Gauss-Jordan elimination on [A | I] in FP64
// with partial pivoting (the first row of largest |a_ik| at or below the diagonal), in one
// block with the augmented matrix in shared memory.  Every element sees the operations of
// a serial elimination in the same order, each rounded on its own (no contraction), and
// rows whose multiplier is zero are skipped, so the inverse is the serial one bit for bit.
// A zero pivot sets *status = 1 and leaves inv unwritten.
constexpr int kCoarseInvMax = 96;  // [A | I] of 96 rows is 147 KB of shared memory

template <class T>
__global__ void __launch_bounds__(256) coarse_inverse(int n, int w, size_t ld, const int *__restrict__ col,
                                                      const T *__restrict__ val, T *__restrict__ inv,
                                                      int *status) {
  extern __shared__ double aug[];
  __shared__ double fk[kCoarseInvMax];
  __shared__ int piv, singular;
  const int n2 = 2 * n;
  for (int e = threadIdx.x; e < n * n2; e += blockDim.x) {
    const int i = e / n2, j = e - i * n2;
    aug[e] = (j == n + i) ? 1.0 : 0.0;
  }
  if (threadIdx.x == 0) singular = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    for (int q = 0; q < w; ++q) {
      const size_t at = (size_t)q * ld + i;
      double &d = aug[(size_t)i * n2 + col[at]];
      d = __dadd_rn(d, (double)val[at]);
    }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    if (threadIdx.x < 32) {
      double best = -1.0;
      int bi = n;
      for (int i = k + threadIdx.x; i < n; i += 32) {
        const double v = fabs(aug[(size_t)i * n2 + k]);
        if (v > best) {
          best = v;
          bi = i;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (threadIdx.x == 0) {
        piv = bi < n ? bi : k;
        if (!(aug[(size_t)piv * n2 + k] != 0.0)) singular = 1;
      }
    }
    __syncthreads();
    if (singular) {
      if (threadIdx.x == 0) *status = 1;
      return;
    }
    const int p = piv;
    if (p != k)
      for (int j = threadIdx.x; j < n2; j += blockDim.x) {
        const double t = aug[(size_t)p * n2 + j];
        aug[(size_t)p * n2 + j] = aug[(size_t)k * n2 + j];
        aug[(size_t)k * n2 + j] = t;
      }
    __syncthreads();
    const double d = 1.0 / aug[(size_t)k * n2 + k];
    __syncthreads();
    for (int j = threadIdx.x; j < n2; j += blockDim.x) aug[(size_t)k * n2 + j] = __dmul_rn(aug[(size_t)k * n2 + j], d);
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      if (i != k) fk[i] = aug[(size_t)i * n2 + k];
    __syncthreads();
    for (int e = threadIdx.x; e < n * n2; e += blockDim.x) {
      const int i = e / n2, j = e - i * n2;
      const double f = fk[i];
      if (i == k || f == 0.0) continue;
      aug[e] = __dsub_rn(aug[e], __dmul_rn(f, aug[(size_t)k * n2 + j]));
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e - i * n;
    inv[e] = (T)aug[(size_t)i * n2 + n + j];
  }
  if (threadIdx.x == 0) *status = 0;
}

// ------------------------------------------------------------------ V-cycle

template <class V>
__global__ void jacobi_first(int n, const V *__restrict__ dinv, const V *__restrict__ b, V omega,
                             V *__restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = omega * dinv[i] * b[i];
}

// x += alpha P xc (piecewise-constant prolongation), in place
template <class V>
__global__ void prolong_add(int n, const int *__restrict__ agg, const V *__restrict__ xc, V alpha,
                            V *__restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] += alpha * xc[agg[i]];
}

// levels with more rows than this apply the coarse correction in its own pass and then
// sweep, instead of inside the sweep: the fused form gathers three arrays per slot
// (x, the aggregate map and the coarse x), which on the levels with many rows costs more
// than the extra pass (measured at 128^3 on levels of 262k and 33k rows)
constexpr int kSplitProlongRows = 1 << 14;

// b_c[I] = sum of r over the members of I, in member order
template <class V>
__global__ void restrict_sum(int nc, const int *__restrict__ mptr, int nf, const int *__restrict__ mem,
                             const V *__restrict__ r, V *__restrict__ bc) {
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nc; I += gridDim.x * blockDim.x) {
    const int a = mptr[I], e = (I + 1 < nc) ? mptr[I + 1] : nf;
    V s = V(0);
    for (int k = a; k < e; ++k) s += r[mem[k]];
    bc[I] = s;
  }
}

// sum over this lane's slots k = sub, sub + g, ... < w of val[k][i] * xj(col[k][i]), added in
// slot order.  The loads of up to kRowBatch slots are issued before the first product, so
// a short row costs two dependent round trips to L2 (columns, then the gathered values)
// rather than two per slot: the coarse levels have few rows per SM, and their time is
// load latency, not bandwidth.
template <class V>
struct RowBatch {
  static constexpr int n = sizeof(V) == 4 ? 12 : 6;  // registers: 1024-thread blocks have 64
};

// STREAM: the matrix values are read with the evict-first hint (a pass over data too large
// to stay in L2, which should not push out the data that can).
template <class V, int B = RowBatch<V>::n, bool STREAM = false, class XJ>
__device__ __forceinline__ V row_sum(int w, size_t ld, long long i, int sub, int g, const int *__restrict__ col,
                                     const V *__restrict__ val, XJ xj) {
  V sacc = V(0);
  for (int k0 = sub; k0 < w; k0 += g * B) {
    int c[B];
    V a[B], x[B];
#pragma unroll
    for (int u = 0; u < B; ++u) {
      const int k = k0 + u * g;
      if (k < w) {
        const size_t at = (size_t)k * ld + i;
        c[u] = col[at];  // the columns are shared with the V-cycle's fine level
        a[u] = STREAM ? __ldcs(val + at) : val[at];
      }
    }
#pragma unroll
    for (int u = 0; u < B; ++u)
      if (k0 + u * g < w) x[u] = xj(c[u]);
#pragma unroll
    for (int u = 0; u < B; ++u)
      if (k0 + u * g < w) sacc += a[u] * x[u];
  }
  return sacc;
}

// The row operations of the grid levels, with G lanes per row: the lanes of a group take
// slots sub, sub + G, ... (the slot-major ELL keeps each slot's rows adjacent, so a warp
// still reads whole sectors) and add their sums by a fixed shuffle tree.  Levels with few
// rows get more lanes per row (vcycle), so that each lane's loads fit one batch.
enum RowOp { kOpFirst2, kOpSweep, kOpResidual, kOpProlongSweep };

template <int G, int OP, class V>
__global__ void __launch_bounds__(kT) row_op(int n, int w, size_t ld, const int *__restrict__ col,
                                             const V *__restrict__ val, const V *__restrict__ dinv,
                                             const V *__restrict__ b, const V *__restrict__ xin,
                                             const int *__restrict__ agg, const V *__restrict__ xc, V alpha,
                                             V omega, V *__restrict__ out) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int sub = (int)(tid % G);
  const long long groups = ((long long)gridDim.x * blockDim.x) / G;
  const long long rounds = (n + groups - 1) / groups;  // the same for every lane
  for (long long rd = 0; rd < rounds; ++rd) {
    const long long i = tid / G + rd * groups;
    const bool act = i < n;
    V sacc = V(0);
    if (act)
      // one lane per row only on levels with many rows: there occupancy hides the latency,
      // and a short batch keeps the registers (and so the occupancy) of the old loop
      sacc = row_sum<V, G == 1 ? 4 : RowBatch<V>::n>(w, ld, i, sub, G, col, val, [&](int j) {
        if (OP == kOpFirst2) return omega * dinv[j] * b[j];
        if (OP == kOpProlongSweep) return xin[j] + alpha * xc[agg[j]];
        return xin[j];
      });
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) sacc += __shfl_xor_sync(0xffffffffu, sacc, o);
    if (act && sub == 0) {
      if (OP == kOpFirst2) {
        const V x1 = omega * dinv[i] * b[i];
        out[i] = x1 + omega * dinv[i] * (b[i] - sacc);
      } else if (OP == kOpSweep) {
        out[i] = xin[i] + omega * dinv[i] * (b[i] - sacc);
      } else if (OP == kOpResidual) {
        out[i] = b[i] - sacc;
      } else {
        const V y = xin[i] + alpha * xc[agg[i]];
        out[i] = y + omega * dinv[i] * (b[i] - sacc);
      }
    }
  }
}

// b_c[I] = sum over the members q of I (in member order) of r_q = b_q - (A x)_q: the
// residual and the restriction in one pass, 8 lanes per coarse row, one member row each
// (more members go round in turns).  For the coarse levels, whose rows are in code order,
// so that a coarse row's members are adjacent rows and a warp's loads stay coalesced.
template <class V>
__global__ void __launch_bounds__(kT) residual_restrict(int nc, const int *__restrict__ mptr,
                                                        const int *__restrict__ mem, int nf, int w, size_t ld,
                                                        const int *__restrict__ col, const V *__restrict__ val,
                                                        const V *__restrict__ b, const V *__restrict__ x,
                                                        V *__restrict__ bc) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane8 = (int)(tid & 7), lane = threadIdx.x & 31;
  const long long groups = ((long long)gridDim.x * blockDim.x) / 8;
  const long long rounds = (nc + groups - 1) / groups;  // the same for every lane
  for (long long rd = 0; rd < rounds; ++rd) {
    const long long I = tid / 8 + rd * groups;
    const bool act = I < nc;
    const int q0 = act ? mptr[I] : 0, q1 = act ? ((I + 1 < nc) ? mptr[I + 1] : nf) : 0;
    const int turns = __reduce_max_sync(0xffffffffu, (unsigned)((q1 - q0 + 7) / 8));
    V total = V(0);
    for (int tn = 0; tn < turns; ++tn) {
      const int qb = q0 + 8 * tn, q = qb + lane8;
      V r = V(0);
      if (q < q1) {
        const int i = mem[q];
        r = b[i] - row_sum<V>(w, ld, i, 0, 1, col, val, [&](int j) { return x[j]; });
      }
      const int cnt = min(8, q1 - qb);
      for (int m = 0; m < 8; ++m) {
        const V t = __shfl_sync(0xffffffffu, r, (lane & ~7) + m);
        if (m < cnt) total += t;
      }
    }
    if (act && lane8 == 0) bc[I] = total;
  }
}

// ------------------------------------------------------------------ FGMRES

// State of the device-resident mixed solve: the FP64 refinement loop and the FP32
// FGMRES cycle both run as conditional WHILE nodes of one CUDA graph, so every
// scalar of the iteration lives here.  The leading fields are read back by the host
// once the graph has run.
constexpr int kMaxM = 31;

struct IrState {
  int outer;      // corrections applied (refinements)
  int total_its;  // FGMRES iterations over all corrections
  int reason;     // KSP convergence reason of the refinement loop
  int it;         // iteration of the current FGMRES cycle
  double rn;      // ||D^-1 (b - A x)|| of the current iterate
  double rn0, ttol;
  double bnorm;   // ||D^-1 b||: the stopping test's scale, whatever the initial guess
  double rtol, atol, dtol, rtol_in;
  double rtol_in_base;  // the configured inner tolerance; rtol_in adapts per correction
  int max_it, max_outer, M, inner_max;
  int exact_inner;  // FP64 corrections: each cycle aims straight at the outer tolerance
  double beta;    // ||v_0|| of the current cycle
  double scale;   // factor that normalises the newest basis vector
  double H[(kMaxM + 1) * kMaxM];  // column j at H[j * (M + 1)]
  double cs[kMaxM], sn[kMaxM], g[kMaxM + 1], y[kMaxM];
};

// KSPConvergedReason values of the stopping test (petsc 3.5 kspconvergedreason)
constexpr int kConvergedRtol = 2, kConvergedAtol = 3, kDivergedIts = -3, kDivergedDtol = -4,
              kDivergedNanOrInf = -9;

// Every reduction finishes in the last block to arrive, which adds the per-block
// partials in a fixed order (deterministic).
constexpr int kRedBlocks = 444;  // grid of the reduction kernels (3 per SM)

__device__ __forceinline__ bool last_block_arrived(unsigned *counter) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  return last;
}

// the last block: out[j] = sum_b partial[j * G + b] for j < nv, then re-arm the counter
__device__ __forceinline__ void finish_sums(int nv, const double *partial, unsigned *counter, double *out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, G = gridDim.x;
  for (int j = warp; j < nv; j += blockDim.x / 32) {
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < (kRedBlocks + 31) / 32; ++k) {
      const int b = lane + 32 * k;
      if (b < G) v += __ldcg(partial + (size_t)j * G + b);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) out[j] = v;
  }
  if (threadIdx.x == 0) atomicExch(counter, 0u);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// block partials of nv per-lane accumulators: reduced across each warp once, then
// across the block's warps in warp order
template <int NV>
__device__ __forceinline__ void block_partials(const double (&acc)[NV], int nv, double *partial) {
  __shared__ double sm[kT / 32][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double mine = 0.0;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    if (j < nv) {
      const double p = warp_sum(acc[j]);
      if (lane == j) mine = p;
    }
  }
  sm[warp][lane] = mine;
  __syncthreads();
  if ((int)threadIdx.x < nv) {
    double v = 0.0;
    for (int k = 0; k < nw; ++k) v += sm[k][threadIdx.x];
    partial[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = v;
  }
}

__device__ __forceinline__ void block_partial1(double acc, double *partial) {
  __shared__ double sm1[kT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  acc = warp_sum(acc);
  if (lane == 0) sm1[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int k = 0; k < nw; ++k) v += sm1[k];
    partial[blockIdx.x] = v;
  }
}

// One Arnoldi step's scalar work, by the first warp of a block: Hessenberg column (h1 + h2,
// h2 the re-orthogonalisation pass or null), Givens rotations, residual estimate, and
// whether the cycle goes on (sets the inner loop's condition).  The lanes load the column
// and the previous rotations into shared memory at once; lane 0 then runs the serial
// recurrences there (the same operations in the same order), so the step costs one round
// trip to memory instead of one per rotation.
__device__ void arnoldi_step(IrState *S, const double *h1, const double *h2, double nr,
                             cudaGraphConditionalHandle cond) {
  __shared__ double hs[kMaxM + 2], css[kMaxM], sns[kMaxM];
  const int lane = threadIdx.x;
  const int it = S->it, M1 = S->M + 1;
  if (lane <= it) hs[lane] = __ldcg(h1 + lane) + (h2 ? __ldcg(h2 + lane) : 0.0);
  if (lane < it) {
    css[lane] = S->cs[lane];
    sns[lane] = S->sn[lane];
  }
  __syncwarp();
  if (lane == 0) {
    const double tt = sqrt(nr);
    hs[it + 1] = tt;
    for (int j = 1; j <= it; ++j) {
      const double t0 = hs[j - 1];
      hs[j - 1] = css[j - 1] * t0 + sns[j - 1] * hs[j];
      hs[j] = css[j - 1] * hs[j] - sns[j - 1] * t0;
    }
    const double t = sqrt(hs[it] * hs[it] + hs[it + 1] * hs[it + 1]);
    bool more = false;
    if (t != 0.0 && t == t) {
      const double cs = hs[it] / t, sn = hs[it + 1] / t;
      S->cs[it] = cs;
      S->sn[it] = sn;
      const double g = S->g[it];
      S->g[it + 1] = -sn * g;
      S->g[it] = cs * g;
      hs[it] = cs * hs[it] + sn * hs[it + 1];
      more = !(fabs(S->g[it + 1]) <= S->rtol_in * S->beta) && tt != 0.0;
    }
    S->it = it + 1;
    more = more && S->it < S->inner_max;
    S->scale = tt > 0.0 ? 1.0 / tt : 0.0;
    cudaGraphSetConditional(cond, more ? 1u : 0u);
  }
  __syncwarp();
  double *hc = S->H + (size_t)it * M1;
  if (lane <= it + 1) hc[lane] = hs[lane];
}

// a basis-vector load of the Krylov passes (evict-first in FP64, see kKrylovStream)
template <class T>
__device__ __forceinline__ T ld_krylov(const T *p) {
  if constexpr (sizeof(T) == 8) return __ldcs(p);
  else return *p;
}

// Basis vectors V_0..V_it are rows of V (stride vn); the vector being orthogonalised is
// V_{it+1}, with it read from the state.  Each warp takes tiles of 32 consecutive rows
// (one per lane); a row's basis values stay in registers for the update and the dots.
//   MODE 1: w -= V h_in; h = V^T w.   MODE 2: w -= V h_in; out[0] = ||w||^2.
// MODE 2 also finishes the Arnoldi step in its last block (h1, h2 as arnoldi_step).
template <int MODE, class T, int NV>
__global__ void __launch_bounds__(kT) cgs_pass(int n, IrState *S, T *V, size_t vn,
                                                const double *__restrict__ h_in, double *partial, unsigned *counter,
                                                double *out, const double *h1, const double *h2,
                                                cudaGraphConditionalHandle cond) {
  __shared__ double hsh[32];
  const int nv = S->it + 1;
  T *w = V + (size_t)nv * vn;
  if ((int)threadIdx.x < nv) hsh[threadIdx.x] = h_in[threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double acc[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) acc[j] = 0.0;
  double acc1 = 0.0;
  const int ntiles = (n + 31) / 32;
  for (int tile = blockIdx.x * nw + warp; tile < ntiles; tile += gridDim.x * nw) {
    const int i = tile * 32 + lane;
    const bool ok = i < n;
    if (MODE == 1) {
      T vj[NV];
#pragma unroll
      for (int j = 0; j < NV; ++j) vj[j] = (j < nv && ok) ? ld_krylov(V + (size_t)j * vn + i) : T(0);
      double wi = ok ? (double)w[i] : 0.0;
#pragma unroll
      for (int j = 0; j < NV; ++j)
        if (j < nv) wi -= hsh[j] * (double)vj[j];
      if (ok) w[i] = (T)wi;
      wi = (double)(T)wi;
#pragma unroll
      for (int j = 0; j < NV; ++j)
        if (j < nv) acc[j] += wi * (double)vj[j];
    } else if (ok) {
      double wi = (double)w[i];
#pragma unroll
      for (int j = 0; j < NV; ++j)
        if (j < nv) wi -= hsh[j] * (double)ld_krylov(V + (size_t)j * vn + i);
      w[i] = (T)wi;
      wi = (double)(T)wi;
      acc1 += wi * wi;
    }
  }
  if (MODE == 1) {
    block_partials(acc, nv, partial);
    if (last_block_arrived(counter)) finish_sums(nv, partial, counter, out);
  } else {
    block_partial1(acc1, partial);
    if (last_block_arrived(counter)) {
      finish_sums(1, partial, counter, out);
      __syncthreads();
      if (threadIdx.x < 32) arnoldi_step(S, h1, h2, __ldcg(out), cond);
    }
  }
}

// slots per batch of the Krylov SpMV: with 16 basis vectors three 256-thread blocks fit
// an SM (85 registers, the dot accumulators taking 32), with 32 two
template <class T>
constexpr int kSpmvBatch = sizeof(T) == 4 ? 8 : 4;
// FP64 Krylov passes (the operator and the basis, ~130 MB at 128^3) stream with the
// evict-first hint so that the FP32 V-cycle's levels (~50 MB) stay in the 126 MB L2
// between iterations; the FP32 passes fit beside them
template <class T>
constexpr bool kKrylovStream = sizeof(T) == 8;

// V_{it+1} = A z and the dots <V_{it+1}, V_j>, j <= it, in the same warp-tile pass.
// With a preconditioner z is its output, kept as Z_it for the solution; without one
// (Z == nullptr) z is V_it itself.
template <class T, class TZ, int NV>
__global__ void __launch_bounds__(kT, NV <= 16 ? 3 : 2) spmv_dots(int n, int ew, size_t ld, const int *__restrict__ col,
                                                 const T *__restrict__ val, const TZ *zin, T *Z,
                                                 T *V, size_t vn, const IrState *__restrict__ S, double *partial,
                                                 unsigned *counter, double *out) {
  const int it = S->it, nv = it + 1;
  // the preconditioner's output (of type TZ), or the basis vector itself
  const TZ *zp = zin;
  const T *zv = V + (size_t)it * vn;
  T *zk = Z ? Z + (size_t)it * vn : nullptr;
  T *w = V + (size_t)nv * vn;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double acc[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) acc[j] = 0.0;
  const int ntiles = (n + 31) / 32;
  for (int tile = blockIdx.x * nw + warp; tile < ntiles; tile += gridDim.x * nw) {
    const int i = tile * 32 + lane;
    if (i >= n) continue;
    T sacc;
    if (Z) {
      sacc = row_sum<T, kSpmvBatch<T>, kKrylovStream<T>>(ew, ld, i, 0, 1, col, val,
                                                          [&](int j) { return (T)zp[j]; });
      zk[i] = (T)zp[i];
    } else {
      sacc = row_sum<T, kSpmvBatch<T>, kKrylovStream<T>>(ew, ld, i, 0, 1, col, val,
                                                          [&](int j) { return zv[j]; });
    }
    w[i] = sacc;
    const double wi = (double)sacc;
#pragma unroll
    for (int j = 0; j < NV; ++j)
      if (j < nv) acc[j] += wi * (double)ld_krylov(V + (size_t)j * vn + i);
  }
  block_partials(acc, nv, partial);
  if (last_block_arrived(counter)) finish_sums(nv, partial, counter, out);
}

// V_it *= scale (the newest basis vector), and the same into the V-cycle's input if any
template <class T, class TV = T>
__global__ void scale_next(int n, const IrState *__restrict__ S, T *__restrict__ V, size_t vn,
                           TV *__restrict__ vin) {
  const T f = (T)S->scale;
  T *v = V + (size_t)S->it * vn;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const T u = v[i] * f;
    v[i] = u;
    if (vin) vin[i] = (TV)u;
  }
}

// y = H^-1 g (upper triangular) for the cycle's iterations
// (one warp: the triangle and g are staged in shared memory, lane 0 solves)
__global__ void fg_finish(IrState *S) {
  __shared__ double Hs[(kMaxM + 1) * kMaxM], gs[kMaxM + 1], ys[kMaxM];
  const int it = S->it, M1 = S->M + 1;
  for (int e = threadIdx.x; e < it * M1; e += blockDim.x) Hs[e] = S->H[e];
  for (int k = threadIdx.x; k < it; k += blockDim.x) gs[k] = S->g[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = it - 1; k >= 0; --k) {
      double s = gs[k];
      for (int j = k + 1; j < it; ++j) s -= Hs[(size_t)j * M1 + k] * ys[j];
      const double hkk = Hs[(size_t)k * M1 + k];
      ys[k] = hkk != 0.0 ? s / hkk : 0.0;
    }
    S->total_its += it;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < it; k += blockDim.x) S->y[k] = ys[k];
}

// d = Z y
template <class T>
__global__ void combine(int n, const T *__restrict__ Z, size_t vn, const IrState *__restrict__ S,
                        T *__restrict__ d) {
  const int nv = S->it;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int j = 0; j < nv; ++j) t += S->y[j] * (double)Z[(size_t)j * vn + i];
    d[i] = (T)t;
  }
}

// ---- the FP64 refinement loop ----

__global__ void ir_init(IrState *S, double rtol, double atol, double dtol, double rtol_in, int max_it, int max_outer,
                        int M, int exact_inner) {
  S->outer = 0;
  S->total_its = 0;
  S->reason = 0;
  S->it = 0;
  S->rn = S->rn0 = S->ttol = 0.0;
  S->rtol = rtol;
  S->atol = atol;
  S->dtol = dtol;
  S->rtol_in = rtol_in;
  S->rtol_in_base = rtol_in;
  S->max_it = max_it;
  S->max_outer = max_outer;
  S->M = M;
  S->exact_inner = exact_inner;
}

// r = b - A x in FP64 and ||D^-1 r||; the last block applies the stopping test of the
// reference's KSP (rtol on the first residual, atol, dtol, max_it) and sets the
// refinement loop's condition
__global__ void __launch_bounds__(kT) ir_residual(int n, int w, size_t ld, const int *__restrict__ col,
                                                   const double *__restrict__ val, const double *__restrict__ b,
                                                   const double *__restrict__ x, double *__restrict__ r,
                                                   IrState *S, double *partial, unsigned *counter, double *tmp,
                                                   cudaGraphConditionalHandle cond) {
  double nrm = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < w; ++k) {
      const size_t at = (size_t)k * ld + i;
      s += val[at] * x[col[at]];
    }
    const double ri = b[i] - s;
    r[i] = ri;
    const double d = val[i];
    const double pr = (d == 0.0 ? 1.0 : 1.0 / d) * ri;
    nrm += pr * pr;
  }
  block_partial1(nrm, partial);
  if (!last_block_arrived(counter)) return;
  finish_sums(1, partial, counter, tmp);
  __syncthreads();
  if (threadIdx.x != 0) return;
  const double rn = sqrt(__ldcg(tmp));
  if (S->outer == 0) {
    S->ttol = fmax(S->rtol * S->bnorm, S->atol);
    S->rn0 = S->bnorm;
  }
  int reason = 0;
  bool stop = true;
  if (S->outer == 0 && S->bnorm == 0.0) reason = kConvergedAtol;
  else if (!(rn == rn)) reason = kDivergedNanOrInf;
  else if (rn <= S->ttol) reason = rn < S->atol ? kConvergedAtol : kConvergedRtol;
  else if (rn >= S->dtol * S->rn0) reason = kDivergedDtol;
  else if (S->total_its >= S->max_it) reason = kDivergedIts;
  else if (S->outer >= S->max_outer) reason = 0;
  else stop = false;
  // A correction cannot reduce the FP64 residual by more than the FP32 operator allows
  // (~cond(A) 6e-8, which grows as the tree deepens); solving the next correction much
  // further than the last one's achieved reduction is wasted.  So the next inner
  // tolerance is half the last reduction, never tighter than the configured one.
  if (S->exact_inner) {
    // FP64 corrections carry no operator rounding to stop at: each cycle is asked for
    // the whole remaining reduction, with a factor 2 of margin
    if (rn > 0.0) S->rtol_in = fmin(0.1, fmax(0.5 * S->ttol / rn, 1e-15));
  } else if (S->outer >= 1 && S->rn > 0.0) {
    S->rtol_in = fmin(0.1, fmax(S->rtol_in_base, 0.5 * (rn / S->rn)));
  }
  S->rn = rn;
  S->reason = reason;
  cudaGraphSetConditional(cond, stop ? 0u : 1u);
}

// ||D^-1 b|| into the state (last block)
__global__ void __launch_bounds__(kT) ir_bnorm(int n, const double *__restrict__ val, const double *__restrict__ b,
                                                IrState *S, double *partial, unsigned *counter, double *tmp) {
  double nrm = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double d = val[i];
    const double pb = (d == 0.0 ? 1.0 : 1.0 / d) * b[i];
    nrm += pb * pb;
  }
  block_partial1(nrm, partial);
  if (!last_block_arrived(counter)) return;
  finish_sums(1, partial, counter, tmp);
  __syncthreads();
  if (threadIdx.x == 0) S->bnorm = sqrt(__ldcg(tmp));
}

// v_0 = D^-1 r / ||D^-1 r|| rounded to the inner precision, and beta = ||v_0||; the last
// block opens the (F)GMRES cycle (sets the inner loop's condition)
template <class T>
__global__ void __launch_bounds__(kT) ir_to_inner(int n, const double *__restrict__ r, const double *__restrict__ diag,
                                                   IrState *S, T *__restrict__ v0, double *partial,
                                                   unsigned *counter, double *tmp, cudaGraphConditionalHandle cond) {
  const double inv_s = 1.0 / S->rn;
  double nrm = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double d = diag[i];
    const T v = (T)((d == 0.0 ? r[i] : r[i] / d) * inv_s);
    v0[i] = v;
    nrm += (double)v * (double)v;
  }
  block_partial1(nrm, partial);
  if (!last_block_arrived(counter)) return;
  finish_sums(1, partial, counter, tmp);
  __syncthreads();
  if (threadIdx.x != 0) return;
  const double beta = sqrt(__ldcg(tmp));
  S->beta = beta;
  S->it = 0;
  S->g[0] = beta;
  S->scale = beta > 0.0 ? 1.0 / beta : 0.0;
  S->inner_max = min(S->M, max(1, S->max_it - S->total_its));
  cudaGraphSetConditional(cond, beta > 0.0 ? 1u : 0u);
}

// x += ||D^-1 r|| d: apply the correction of the scaled system
template <class T>
__global__ void ir_axpy(int n, IrState *S, const T *__restrict__ d, double *__restrict__ x) {
  const double s = S->rn;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] += s * (double)d[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) S->outer += 1;
}


// ---- the coarse end of the V-cycle in one block: every level with <= kTail nodes,
//      down (smooth, residual, restrict), the dense coarsest solve, and up (prolong,
//      smooth), separated by block barriers instead of kernel launches ----
constexpr int kTail = 1024;
constexpr int kTailLevels = 12;

template <class V>
struct TailLevel {
  int n, w, g;  // g: lanes per row (power of two)
  size_t ld;
  const int *col;
  const V *val, *dinv;
  const int *agg;             // node -> next coarser node
  const int *mptr, *mem;      // members of this level's nodes on the finer level
  V *x, *x2, *b, *r;
};
template <class V>
struct TailArgs {
  int nl;                     // levels in the tail, the last one solved densely
  TailLevel<V> L[kTailLevels];
  const V *inv;
  int sweeps;
  V omega, alpha;
};

// lanes per row of a tail level run by `threads` threads: as many as keep the level in one
// round, at most 16 and no more than the row's slots
static inline int tail_lanes(int n, int w, int threads) {
  int g = 1;
  while (g < 16 && g < w && 2 * g * n <= threads) g *= 2;
  return g;
}

// the graph path's tail kernel: 512 threads leave 128 registers a thread for the batched
// row loads (a 1024-thread block has 64)
constexpr int kTailThreads = 512;
// the staged tail: its loads hit shared memory, so short batches suffice and the block can
// take 1024 threads (64 registers), one round for levels of up to 1024 rows
constexpr int kTailSmemThreads = 1024;
template <class V>
constexpr int kTailSmemBatch = 4;

// sum_j a_ij xj(j) for every row of a tail level, L.g lanes per row; emit(i, sum) runs on
// the group's first lane.  The trip count is the same for the whole block (shuffles).
template <class V, int B, class XJ, class F>
__device__ __forceinline__ void tail_rows(const TailLevel<V> L, XJ xj, F emit) {
  const int g = L.g, sub = threadIdx.x & (g - 1);
  const int per = blockDim.x / g;
  const int rounds = (L.n + per - 1) / per;
  for (int rd = 0; rd < rounds; ++rd) {
    const int i = (int)threadIdx.x / g + rd * per;
    V sacc = V(0);
    if (i < L.n) sacc = row_sum<V, B>(L.w, L.ld, i, sub, g, L.col, L.val, xj);
    for (int o = g >> 1; o > 0; o >>= 1) sacc += __shfl_xor_sync(0xffffffffu, sacc, o);
    if (i < L.n && sub == 0) emit(i, sacc);
  }
}

// The tail's levels in one block (every thread of the block takes part; the block
// barriers separate the phases).  Per level: pre-smoothing (the first two sweeps from
// zero in one pass), residual and restriction in one pass, and on the way up the coarse
// correction inside the first post-sweep, so a level costs four barriers.  The
// pre-smoothed iterate is placed so that the post-sweeps end in L.x.  B: slots per lane whose
// loads are issued together (registers).
template <class V, int B>
__device__ __forceinline__ void tail_body(const TailArgs<V> &A) {
  const V om = A.omega, al = A.alpha;
  const int sw = A.sweeps;
  V *cur[kTailLevels];  // each level's pre-smoothed iterate
  for (int l = 0; l < A.nl - 1; ++l) {
    const TailLevel<V> L = A.L[l];  // by value: the stores below cannot alias it
    V *c;
    if (sw >= 2) {
      tail_rows<V, B>(L, [&](int j) { return om * L.dinv[j] * L.b[j]; }, [&](int i, V sacc) {
        const V x1 = om * L.dinv[i] * L.b[i];
        L.x[i] = x1 + om * L.dinv[i] * (L.b[i] - sacc);
      });
      __syncthreads();
      c = L.x;
      V *o = L.x2;
      for (int k = 2; k < sw; ++k) {
        tail_rows<V, B>(L, [&](int j) { return c[j]; },
                  [&](int i, V sacc) { o[i] = c[i] + om * L.dinv[i] * (L.b[i] - sacc); });
        __syncthreads();
        V *t = c; c = o; o = t;
      }
    } else {
      for (int i = threadIdx.x; i < L.n; i += blockDim.x) L.x2[i] = om * L.dinv[i] * L.b[i];
      __syncthreads();
      c = L.x2;
    }
    cur[l] = c;
    // residual of every member row and the coarse row's sum, in member order: 8 lanes per
    // coarse row, one member row each (more members go round in turns)
    const TailLevel<V> C = A.L[l + 1];
    const int lane8 = threadIdx.x & 7, per = blockDim.x / 8;
    const int rounds = (C.n + per - 1) / per;
    for (int rd = 0; rd < rounds; ++rd) {
      const int I = (int)threadIdx.x / 8 + rd * per;
      const bool act = I < C.n;
      const int q0 = act ? C.mptr[I] : 0, q1 = act ? ((I + 1 < C.n) ? C.mptr[I + 1] : L.n) : 0;
      // turns of 8 members: the same count across the warp, for the shuffles
      const int turns = __reduce_max_sync(0xffffffffu, (unsigned)((q1 - q0 + 7) / 8));
      V total = V(0);
      for (int tn = 0; tn < turns; ++tn) {
        const int qb = q0 + 8 * tn;
        const int q = qb + lane8;
        V r = V(0);
        if (q < q1) {
          const int i = C.mem[q];
          r = L.b[i] - row_sum<V, B>(L.w, L.ld, i, 0, 1, L.col, L.val, [&](int j) { return c[j]; });
        }
        const int cnt = min(8, q1 - qb);
        for (int m = 0; m < 8; ++m) {
          const V t = __shfl_sync(0xffffffffu, r, (threadIdx.x & 31 & ~7) + m, 32);
          if (m < cnt) total += t;
        }
      }
      if (act && lane8 == 0) C.b[I] = total;
    }
    __syncthreads();
  }
  {
    // the coarsest level: x = K^-1 b, g lanes per row (a row is up to 96 entries)
    const TailLevel<V> K = A.L[A.nl - 1];
    const V *inv = A.inv;
    const int nk = K.n;
    int g = 32;
    while (g > 1 && g * nk > (int)blockDim.x) g >>= 1;
    const int sub = threadIdx.x & (g - 1), per = blockDim.x / g;
    const int rounds = (nk + per - 1) / per;
    for (int rd = 0; rd < rounds; ++rd) {
      const int i = (int)threadIdx.x / g + rd * per;
      V sacc = V(0);
      if (i < nk)
#pragma unroll 4
        for (int j = sub; j < nk; j += g) sacc += inv[(size_t)i * nk + j] * K.b[j];
      for (int o = g >> 1; o > 0; o >>= 1) sacc += __shfl_xor_sync(0xffffffffu, sacc, o);
      if (i < nk && sub == 0) K.x[i] = sacc;
    }
    __syncthreads();
  }
  for (int l = A.nl - 2; l >= 0; --l) {
    const TailLevel<V> L = A.L[l];  // by value: the stores below cannot alias it
    const V *xc = A.L[l + 1].x;
    V *c = cur[l];
    V *o = (c == L.x) ? L.x2 : L.x;
    tail_rows<V, B>(L, [&](int j) { return c[j] + al * xc[L.agg[j]]; }, [&](int i, V sacc) {
      const V y = c[i] + al * xc[L.agg[i]];
      o[i] = y + om * L.dinv[i] * (L.b[i] - sacc);
    });
    __syncthreads();
    { V *t = c; c = o; o = t; }
    for (int k = 1; k < sw; ++k) {
      tail_rows<V, B>(L, [&](int j) { return c[j]; },
                [&](int i, V sacc) { o[i] = c[i] + om * L.dinv[i] * (L.b[i] - sacc); });
      __syncthreads();
      V *t = c; c = o; o = t;
    }
  }
}

template <class V>
__global__ void __launch_bounds__(kTailThreads) vcycle_tail(TailArgs<V> A) {
  tail_body<V, RowBatch<V>::n>(A);
}

constexpr size_t kTailSmemMax = 227 * 1024;  // dynamic shared memory a block may opt into

// The tail with every level staged in shared memory (the levels are constant for a solve
// and, at a few hundred rows, take tens of KB): each launch copies the tail's matrices,
// maps and the first level's right-hand side in, runs the same body on the copies, and
// writes the first level's solution back.  Staging turns each phase's gathers from L2
// round trips into shared-memory loads.  The layout is tail_smem_bytes's.
__host__ __device__ inline size_t tail_align(size_t b) { return (b + 15) & ~(size_t)15; }

template <class V>
__host__ __device__ inline size_t tail_smem_bytes(const TailArgs<V> &A) {
  size_t b = tail_align(sizeof(TailArgs<V>));
  for (int k = 0; k < A.nl; ++k) {
    const size_t n = (size_t)A.L[k].n, nw = n * (size_t)A.L[k].w;
    b += tail_align(nw * sizeof(int)) + tail_align(nw * sizeof(V)) + tail_align(n * sizeof(V));  // col, val, dinv
    if (k + 1 < A.nl) b += tail_align(n * sizeof(int));                                          // agg
    if (k > 0) b += tail_align(n * sizeof(int)) + tail_align((size_t)A.L[k - 1].n * sizeof(int)); // mptr, mem
    b += 4 * tail_align(n * sizeof(V));                                                          // x, x2, b, r
  }
  const size_t nk = (size_t)A.L[A.nl - 1].n;
  return b + tail_align(nk * nk * sizeof(V));  // the coarsest inverse
}

// Block-wide asynchronous copy of `bytes` (a multiple of 4) from global to shared memory:
// 16-byte cp.async where both addresses allow it, 4-byte otherwise.  Completion is waited
// for by stage_wait.
__device__ __forceinline__ void stage_copy(void *dst, const void *src, size_t bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const char *sp = static_cast<const char *>(src);
  size_t done = 0;
  if (((reinterpret_cast<uintptr_t>(src) | d) & 15) == 0) {
    const size_t n16 = bytes / 16;
    for (size_t k = threadIdx.x; k < n16; k += blockDim.x)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d + (unsigned)(16 * k)), "l"(sp + 16 * k)
                   : "memory");
    done = n16 * 16;
  }
  for (size_t k = done / 4 + threadIdx.x; k < bytes / 4; k += blockDim.x)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d + (unsigned)(4 * k)), "l"(sp + 4 * k)
                 : "memory");
}

__device__ __forceinline__ void stage_wait() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
}

template <class V>
__global__ void __launch_bounds__(kTailSmemThreads) vcycle_tail_smem(TailArgs<V> A) {
  extern __shared__ __align__(16) unsigned char tsm[];
  TailArgs<V> &S = *reinterpret_cast<TailArgs<V> *>(tsm);
  unsigned char *p = tsm + tail_align(sizeof(TailArgs<V>));
  auto take = [&](size_t bytes) {
    unsigned char *q = p;
    p += tail_align(bytes);
    return q;
  };
  const int t = threadIdx.x, T = blockDim.x;
  if (t == 0) S = A;
  __syncthreads();
  for (int k = 0; k < A.nl; ++k) {
    const TailLevel<V> &G = A.L[k];
    const int n = G.n, w = G.w;
    int *col = (int *)take((size_t)n * w * sizeof(int));
    V *val = (V *)take((size_t)n * w * sizeof(V));
    V *dinv = (V *)take((size_t)n * sizeof(V));
    if (G.ld == (size_t)n) {
      // coarse levels: the slot-major arrays are contiguous
      stage_copy(col, G.col, (size_t)n * w * sizeof(int));
      stage_copy(val, G.val, (size_t)n * w * sizeof(V));
    } else {
      for (int e = t; e < n * w; e += T) {
        const int slot = e / n, i = e - slot * n;
        const size_t at = (size_t)slot * G.ld + i;
        col[e] = G.col[at];
        val[e] = G.val[at];
      }
    }
    stage_copy(dinv, G.dinv, (size_t)n * sizeof(V));
    int *agg = nullptr, *mptr = nullptr, *mem = nullptr;
    if (k + 1 < A.nl) {
      agg = (int *)take((size_t)n * sizeof(int));
      stage_copy(agg, G.agg, (size_t)n * sizeof(int));
    }
    if (k > 0) {
      const int nf = A.L[k - 1].n;
      mptr = (int *)take((size_t)n * sizeof(int));
      mem = (int *)take((size_t)nf * sizeof(int));
      stage_copy(mptr, G.mptr, (size_t)n * sizeof(int));
      stage_copy(mem, G.mem, (size_t)nf * sizeof(int));
    }
    V *x = (V *)take((size_t)n * sizeof(V));
    V *x2 = (V *)take((size_t)n * sizeof(V));
    V *b = (V *)take((size_t)n * sizeof(V));
    V *r = (V *)take((size_t)n * sizeof(V));
    if (k == 0) stage_copy(b, G.b, (size_t)n * sizeof(V));
    if (t == 0) {
      TailLevel<V> &D = S.L[k];
      D.ld = (size_t)n;
      D.col = col;
      D.val = val;
      D.dinv = dinv;
      D.agg = agg;
      D.mptr = mptr;
      D.mem = mem;
      D.x = x;
      D.x2 = x2;
      D.b = b;
      D.r = r;
    }
  }
  {
    const int nk = A.L[A.nl - 1].n;
    V *inv = (V *)take((size_t)nk * nk * sizeof(V));
    stage_copy(inv, A.inv, (size_t)nk * nk * sizeof(V));
    if (t == 0) S.inv = inv;
  }
  stage_wait();
  tail_body<V, kTailSmemBatch<V>>(S);
  __syncthreads();
  for (int i = t; i < A.L[0].n; i += T) A.L[0].x[i] = S.L[0].x[i];
}
// ---------------------------------------------- the whole solve as one persistent kernel
//
// One cooperative launch runs a complete solve: the FP64 refinement loop, each
// correction's (F)GMRES cycle and, for the potential, the V-cycle of every iteration.
// The phases are separated by the bounded grid barrier instead of kernel launches: per
// iteration 4 barriers per grid level of the V-cycle plus one after the single-block
// tail, one after the SpMV + dot products and one after the Gram-Schmidt update.
//   * Reductions are deterministic: each block publishes its partial sums, and after the
//     barrier every block adds all partials in block order, so every block holds the
//     same Hessenberg column, Givens rotations and stopping decisions without another
//     barrier, and takes the same branches.
//   * Krylov vectors are kept un-normalised with a per-vector scale in shared memory, so
//     normalisation costs no pass.
//   * The V-cycle's residual and restriction are one phase: each coarse row sums its
//     members' residuals directly.
//   * Levels of <= kTail nodes run in block 0 (the same code as the graph path's tail
//     kernel) while the other blocks wait at the next barrier.
constexpr int kPT = 1024;         // threads per block, one block per SM
constexpr int kPMaxBlocks = 256;  // partial sums are laid out [slot][block]
constexpr int kPSlots = kMaxM + 2;

template <class T>
struct PLevel {
  int n, w, g;                // rows, ELL width, lanes per row (power of two <= 8)
  size_t ld;
  const int *col;
  const T *val, *dinv;
  const int *agg;             // node -> next coarser node
  const int *mptr, *mem;      // members (on the finer level) of this level's nodes
  T *x, *x2, *b, *r;
};

struct PResult {
  int outer, total_its, reason, pad;
  double rn;
};

template <class T>
struct PSolveArgs {
  int n, w;
  size_t ld;
  const int *col;
  const T *valf;              // D^-1 A in the inner precision
  const double *val, *b;      // FP64 operator (diagonal in slot 0) and rhs
  double *x, *r;
  T *V, *Z;                   // basis (M + 1 vectors), preconditioned vectors (M)
  size_t vn;
  int M, use_mg;
  int nlev, tail;             // levels; first level of the single-block tail
  PLevel<T> L[kMaxLevels];
  TailArgs<T> ta;             // the tail levels (first = L[tail])
  int sweeps;
  T omega, alpha;
  double rtol, atol, dtol, rtol_in;
  int max_it, max_outer, exact_inner;
  double *part;
  GridBar *bar;
  int *err;
  PResult *out;
};

struct PShared {
  double H[(kMaxM + 1) * kMaxM];  // column j at H[j * (M + 1)]
  double cs[kMaxM], sn[kMaxM], g[kMaxM + 1], y[kMaxM], scale[kMaxM + 1], h[kPSlots];
  double red[32];
  double wdots[32][kPSlots];      // per-warp dot products of one Arnoldi step
  double rn, rn0, ttol, bnorm, rtol_in, beta;
  int outer, total_its, reason, it, inner_max, more;
};

// The blocks that run one solve together: the whole grid for a single solve, or one group
// of a batched launch.  Every phase indexes blocks by rank / size.
struct Grp {
  int rank, size;
  GridBar *bar;
  int *err;
};

__device__ __forceinline__ bool gsync(const Grp &g) { return grid_sync(g.bar, (unsigned)g.size, g.err); }

__device__ __forceinline__ double p_block_sum(double v, double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) r = warp_sum(lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0);
  return r;  // valid in warp 0
}

// all blocks: out[j] = sum over blocks of part[j][b], b in block order, for j < nv
__device__ __forceinline__ void p_gather(const Grp &g, const double *part, int nv, double *out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5, nb = g.size;
  for (int j = warp; j < nv; j += nw) {
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < kPMaxBlocks / 32; ++k) {
      const int b = lane + 32 * k;
      if (b < nb) v += __ldcg(part + (size_t)j * kPMaxBlocks + b);
    }
    v = warp_sum(v);
    if (lane == 0) out[j] = v;
  }
  __syncthreads();
}

__device__ __forceinline__ void p_put(const Grp &g, double *part, int j, double v) {
  if (threadIdx.x == 0) part[(size_t)j * kPMaxBlocks + g.rank] = v;
}

template <class T>
__device__ __forceinline__ T group_sum(T s, int G) {
  for (int o = G >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// f(i, sub, G, active) for every row of L, G lanes per row, over the whole grid; the trip
// count is the same for every lane (the group sums shuffle)
template <class T, class F>
__device__ __forceinline__ void grid_rows(const Grp &g, const PLevel<T> &L, F f) {
  const int G = L.g;
  const long long tid = (long long)g.rank * blockDim.x + threadIdx.x;
  const int sub = (int)(tid & (G - 1));
  const long long groups = ((long long)g.size * blockDim.x) / G;
  const long long rounds = (L.n + groups - 1) / groups;
  for (long long rd = 0; rd < rounds; ++rd) {
    const long long i = tid / G + rd * groups;
    f((int)i, sub, G, i < L.n);
  }
}

// two damped Jacobi sweeps from x = 0 in one pass: x1 = w D^-1 b, out = x1 + w D^-1 (b - A x1);
// b = bs * bsrc
template <class T>
__device__ void p_first2(const Grp &g, const PLevel<T> &L, const T *bsrc, T bs, T omega, T *out) {
  grid_rows(g, L, [&](int i, int sub, int G, bool act) {
    T s = T(0);
    if (act)
#pragma unroll 8
      for (int k = sub; k < L.w; k += G) {
        const size_t at = (size_t)k * L.ld + i;
        const int j = L.col[at];
        s += L.val[at] * (omega * L.dinv[j] * (bs * bsrc[j]));
      }
    s = group_sum(s, G);
    if (act && sub == 0) {
      const T bi = bs * bsrc[i];
      const T x1 = omega * L.dinv[i] * bi;
      out[i] = x1 + omega * L.dinv[i] * (bi - s);
    }
  });
}

// x = w D^-1 b (one sweep from zero)
template <class T>
__device__ void p_first1(const Grp &g, const PLevel<T> &L, const T *bsrc, T bs, T omega, T *out) {
  for (int i = g.rank * blockDim.x + threadIdx.x; i < L.n; i += g.size * blockDim.x)
    out[i] = omega * L.dinv[i] * (bs * bsrc[i]);
}

// out = y + w D^-1 (b - A y), y = xin (+ alpha xc[agg] when xc is given)
template <class T>
__device__ void p_sweep(const Grp &g, const PLevel<T> &L, const T *bsrc, T bs, T omega, const T *xin, const T *xc, T alpha,
                        T *out) {
  grid_rows(g, L, [&](int i, int sub, int G, bool act) {
    T s = T(0);
    if (act)
#pragma unroll 8
      for (int k = sub; k < L.w; k += G) {
        const size_t at = (size_t)k * L.ld + i;
        const int j = L.col[at];
        const T yj = xc ? xin[j] + alpha * xc[L.agg[j]] : xin[j];
        s += L.val[at] * yj;
      }
    s = group_sum(s, G);
    if (act && sub == 0) {
      const T yi = xc ? xin[i] + alpha * xc[L.agg[i]] : xin[i];
      out[i] = yi + omega * L.dinv[i] * (bs * bsrc[i] - s);
    }
  });
}

// r = b - A x over the rows of L (G lanes per row, coalesced slot-major reads)
template <class T>
__device__ void p_residual(const Grp &g, const PLevel<T> &L, const T *bsrc, T bs, const T *x, T *r) {
  grid_rows(g, L, [&](int i, int sub, int G, bool act) {
    T s = T(0);
    if (act)
#pragma unroll 8
      for (int k = sub; k < L.w; k += G) {
        const size_t at = (size_t)k * L.ld + i;
        s += L.val[at] * x[L.col[at]];
      }
    s = group_sum(s, G);
    if (act && sub == 0) r[i] = bs * bsrc[i] - s;
  });
}

// the coarse right-hand side: bc[I] = sum of r over the members of I, in member order
template <class T>
__device__ void p_restrict(const Grp &g, int nf, const T *r, const PLevel<T> &C) {
  for (int I = g.rank * blockDim.x + threadIdx.x; I < C.n; I += g.size * blockDim.x) {
    const int a = C.mptr[I], e = (I + 1 < C.n) ? C.mptr[I + 1] : nf;
    T s = T(0);
    for (int q = a; q < e; ++q) s += r[C.mem[q]];
    C.b[I] = s;
  }
}

// z = V-cycle(bs * bsrc) into zout.  Every block calls it; all barriers are common.
template <class T>
__device__ bool p_vcycle(const Grp &g, const PSolveArgs<T> &A, const T *bsrc, T bs, T *zout) {
  const int S = A.sweeps;
  T *pre[kMaxLevels];
  // ---- down: pre-smoothing, then the coarse rhs from the residual ----
  for (int l = 0; l < A.tail; ++l) {
    const PLevel<T> &L = A.L[l];
    const T *bl = l == 0 ? bsrc : L.b;
    const T bsl = l == 0 ? bs : T(1);
    // the post-smoothing's S sweeps alternate between two buffers and must end in the
    // level's output (zout on level 0, L.x above it); so the pre-smoothing result, which
    // the first post sweep reads, lies in the output buffer when S is even
    T *outb = l == 0 ? zout : L.x;
    T *altb = L.x2;
    T *cur = (S % 2 == 0) ? outb : altb;
    T *oth = cur == outb ? altb : outb;
    // pre-smoothing: S sweeps from zero; the result must land in cur
    if (S >= 2) {
      T *tgt = (S % 2 == 0) ? cur : oth;  // S - 2 more sweeps each flip the buffer
      p_first2(g, L, bl, bsl, A.omega, tgt);
      if (!gsync(g)) return false;
      for (int k = 2; k < S; ++k) {
        T *nx = tgt == cur ? oth : cur;
        p_sweep(g, L, bl, bsl, A.omega, tgt, (const T *)nullptr, A.alpha, nx);
        if (!gsync(g)) return false;
        tgt = nx;
      }
    } else {
      p_first1(g, L, bl, bsl, A.omega, cur);
      if (!gsync(g)) return false;
    }
    pre[l] = cur;
    p_residual(g, L, bl, bsl, cur, L.r);
    if (!gsync(g)) return false;
    p_restrict(g, L.n, (const T *)L.r, A.L[l + 1]);
    if (!gsync(g)) return false;
  }
  // ---- the tail in block 0 ----
  if (g.rank == 0) {
    if (A.tail == 0) {  // the whole cycle is the tail: its rhs is the scaled input
      const PLevel<T> &L = A.L[0];
      for (int i = threadIdx.x; i < L.n; i += blockDim.x) L.b[i] = bs * bsrc[i];
      __syncthreads();
    }
    tail_body<T, 4>(A.ta);
    if (A.tail == 0) {
      const PLevel<T> &L = A.L[0];
      for (int i = threadIdx.x; i < L.n; i += blockDim.x) zout[i] = L.x[i];
    }
  }
  if (!gsync(g)) return false;
  // ---- up: coarse correction inside the first post sweep, then plain sweeps ----
  for (int l = A.tail - 1; l >= 0; --l) {
    const PLevel<T> &L = A.L[l];
    const T *bl = l == 0 ? bsrc : L.b;
    const T bsl = l == 0 ? bs : T(1);
    T *outb = l == 0 ? zout : L.x;
    T *altb = L.x2;
    T *cur = pre[l];
    T *nx = cur == outb ? altb : outb;
    p_sweep(g, L, bl, bsl, A.omega, cur, (const T *)A.L[l + 1].x, A.alpha, nx);
    if (!gsync(g)) return false;
    for (int k = 1; k < S; ++k) {
      cur = nx;
      nx = cur == outb ? altb : outb;
      p_sweep(g, L, bl, bsl, A.omega, cur, (const T *)nullptr, A.alpha, nx);
      if (!gsync(g)) return false;
    }
  }
  return true;
}

// One whole solve by the group g (all of its blocks call it); part holds the group's
// [slot][block] partial sums.  Returns false when a barrier gave up.
template <class T>
__device__ bool solve_body(const PSolveArgs<T> &A, const Grp &g, PShared &sh, double *part) {
  const int nb = g.size, n = A.n, M1 = A.M + 1;
  const int rpb = (n + nb - 1) / nb;
  const int r0 = min(n, g.rank * rpb), r1 = min(n, r0 + rpb);
  // ---- ||D^-1 b||: the stopping test's scale ----
  {
    double s = 0.0;
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      const double d = A.val[i];
      const double pb = (d == 0.0 ? 1.0 : 1.0 / d) * A.b[i];
      s += pb * pb;
    }
    s = p_block_sum(s, sh.red);
    p_put(g, part, 0, s);
  }
  if (threadIdx.x == 0) {
    sh.outer = 0;
    sh.total_its = 0;
    sh.reason = 0;
    sh.rn = 0.0;
    sh.rtol_in = A.rtol_in;
  }
  if (!gsync(g)) return false;
  p_gather(g, part, 1, sh.h);
  if (threadIdx.x == 0) sh.bnorm = sqrt(sh.h[0]);
  __syncthreads();
  for (;;) {
    // ---- r = b - A x in FP64 and ||D^-1 r||; the reference's stopping test ----
    if (!gsync(g)) return false;  // x is complete
    {
      double s = 0.0;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        double ax = 0.0;
        for (int k = 0; k < A.w; ++k) {
          const size_t at = (size_t)k * A.ld + i;
          ax += A.val[at] * __ldcg(A.x + A.col[at]);
        }
        const double ri = A.b[i] - ax;
        A.r[i] = ri;
        const double d = A.val[i];
        const double pr = (d == 0.0 ? 1.0 : 1.0 / d) * ri;
        s += pr * pr;
      }
      s = p_block_sum(s, sh.red);
      p_put(g, part, 0, s);
    }
    if (!gsync(g)) return false;
    p_gather(g, part, 1, sh.h);
    if (threadIdx.x == 0) {
      const double rn = sqrt(sh.h[0]);
      if (sh.outer == 0) {
        sh.ttol = fmax(A.rtol * sh.bnorm, A.atol);
        sh.rn0 = sh.bnorm;
      }
      int reason = 0;
      bool stop = true;
      if (sh.outer == 0 && sh.bnorm == 0.0) reason = kConvergedAtol;
      else if (!(rn == rn)) reason = kDivergedNanOrInf;
      else if (rn <= sh.ttol) reason = rn < A.atol ? kConvergedAtol : kConvergedRtol;
      else if (rn >= A.dtol * sh.rn0) reason = kDivergedDtol;
      else if (sh.total_its >= A.max_it) reason = kDivergedIts;
      else if (sh.outer >= A.max_outer) reason = 0;
      else stop = false;
      if (A.exact_inner) {
        if (rn > 0.0) sh.rtol_in = fmin(0.1, fmax(0.5 * sh.ttol / rn, 1e-15));
      } else if (sh.outer >= 1 && sh.rn > 0.0) {
        sh.rtol_in = fmin(0.1, fmax(A.rtol_in, 0.5 * (rn / sh.rn)));
      }
      sh.rn = rn;
      sh.reason = reason;
      sh.more = stop ? 0 : 1;
    }
    __syncthreads();
    if (!sh.more) break;
    // ---- v_0 = D^-1 r / ||D^-1 r|| in the inner precision, beta = ||v_0|| ----
    {
      const double inv_s = 1.0 / sh.rn;
      double s = 0.0;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        const double d = A.val[i];
        const T v = (T)((d == 0.0 ? A.r[i] : A.r[i] / d) * inv_s);
        A.V[i] = v;
        s += (double)v * (double)v;
      }
      s = p_block_sum(s, sh.red);
      p_put(g, part, 0, s);
    }
    if (!gsync(g)) return false;
    p_gather(g, part, 1, sh.h);
    if (threadIdx.x == 0) {
      const double beta = sqrt(sh.h[0]);
      sh.beta = beta;
      sh.it = 0;
      sh.g[0] = beta;
      sh.scale[0] = beta > 0.0 ? 1.0 / beta : 0.0;
      sh.inner_max = min(A.M, max(1, A.max_it - sh.total_its));
      sh.more = beta > 0.0 ? 1 : 0;
    }
    __syncthreads();
    // ---- the (F)GMRES cycle ----
    while (sh.more) {
      const int it = sh.it;
      const T s_it = (T)sh.scale[it];
      const T *vit = A.V + (size_t)it * A.vn;
      T *zit = A.use_mg ? A.Z + (size_t)it * A.vn : nullptr;
      if (A.use_mg && !p_vcycle(g, A, vit, s_it, zit)) return false;
      // w = A z; V_{it+1} = w; partial dots <w, V_j>, j <= it
      T *w = A.V + (size_t)(it + 1) * A.vn;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        T acc = T(0);
#pragma unroll 6
        for (int k = 0; k < A.w; ++k) {
          const size_t at = (size_t)k * A.ld + i;
          const int j = A.col[at];
          acc += A.valf[at] * (A.use_mg ? __ldcg(zit + j) : s_it * __ldcg(vit + j));
        }
        w[i] = acc;
      }
      __syncthreads();
      {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        for (int j = 0; j <= it; ++j) {
          const T *vj = A.V + (size_t)j * A.vn;
          double s = 0.0;
          for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) s += (double)w[i] * (double)vj[i];
          s = warp_sum(s);
          if (lane == 0) sh.wdots[warp][j] = s;
        }
        __syncthreads();
        if ((int)threadIdx.x <= it) {
          double s = 0.0;
          for (int q = 0; q < nw; ++q) s += sh.wdots[q][threadIdx.x];
          part[(size_t)threadIdx.x * kPMaxBlocks + g.rank] = s;
        }
      }
      if (!gsync(g)) return false;
      p_gather(g, part, it + 1, sh.h);
      // w -= sum_j h_j v_j with v_j = scale_j V_j (h_j = scale_j <w, V_j>); ||w||^2
      {
        double s = 0.0;
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
          double wi = (double)w[i];
          for (int j = 0; j <= it; ++j) {
            const double sj = sh.scale[j];
            wi -= (sh.h[j] * sj) * (sj * (double)A.V[(size_t)j * A.vn + i]);
          }
          const T wt = (T)wi;
          w[i] = wt;
          s += (double)wt * (double)wt;
        }
        s = p_block_sum(s, sh.red);
        p_put(g, part, kPSlots - 1, s);
      }
      if (!gsync(g)) return false;
      p_gather(g, part + (size_t)(kPSlots - 1) * kPMaxBlocks, 1, sh.h + kPSlots - 1);
      // Arnoldi scalars, the same in every block
      if (threadIdx.x == 0) {
        const double tt = sqrt(sh.h[kPSlots - 1]);
        double *hc = sh.H + (size_t)it * M1;
        for (int j = 0; j <= it; ++j) hc[j] = sh.h[j] * sh.scale[j];
        hc[it + 1] = tt;
        for (int j = 1; j <= it; ++j) {
          const double t0 = hc[j - 1];
          hc[j - 1] = sh.cs[j - 1] * t0 + sh.sn[j - 1] * hc[j];
          hc[j] = sh.cs[j - 1] * hc[j] - sh.sn[j - 1] * t0;
        }
        const double t = sqrt(hc[it] * hc[it] + hc[it + 1] * hc[it + 1]);
        bool more = false;
        if (t != 0.0 && t == t) {
          const double cs = hc[it] / t, sn = hc[it + 1] / t;
          sh.cs[it] = cs;
          sh.sn[it] = sn;
          sh.g[it + 1] = -sn * sh.g[it];
          sh.g[it] = cs * sh.g[it];
          hc[it] = cs * hc[it] + sn * hc[it + 1];
          more = !(fabs(sh.g[it + 1]) <= sh.rtol_in * sh.beta) && tt != 0.0;
        }
        sh.it = it + 1;
        sh.more = (more && sh.it < sh.inner_max) ? 1 : 0;
        sh.scale[it + 1] = tt > 0.0 ? 1.0 / tt : 0.0;
      }
      __syncthreads();
    }
    // ---- y = H^-1 g; x += ||D^-1 r|| sum_j y_j z_j ----
    if (threadIdx.x == 0) {
      const int it = sh.it;
      for (int k = it - 1; k >= 0; --k) {
        double s = sh.g[k];
        for (int j = k + 1; j < it; ++j) s -= sh.H[(size_t)j * M1 + k] * sh.y[j];
        const double hkk = sh.H[(size_t)k * M1 + k];
        sh.y[k] = hkk != 0.0 ? s / hkk : 0.0;
      }
      sh.total_its += it;
      sh.outer += 1;
    }
    __syncthreads();
    {
      const int nv = sh.it;
      const double rn = sh.rn;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        double t = 0.0;
        if (A.use_mg)
          for (int j = 0; j < nv; ++j) t += sh.y[j] * (double)A.Z[(size_t)j * A.vn + i];
        else
          for (int j = 0; j < nv; ++j) t += sh.y[j] * (sh.scale[j] * (double)A.V[(size_t)j * A.vn + i]);
        A.x[i] += rn * (double)(T)t;
      }
    }
  }
  if (g.rank == 0 && threadIdx.x == 0) {
    A.out->outer = sh.outer;
    A.out->total_its = sh.total_its;
    A.out->reason = sh.reason;
    A.out->rn = sh.rn;
  }
  return true;
}

template <class T>
__global__ void __launch_bounds__(kPT, 1) ir_solve_persistent(PSolveArgs<T> A) {
  __shared__ PShared sh;
  const Grp g{(int)blockIdx.x, (int)gridDim.x, A.bar, A.err};
  solve_body(A, g, sh, A.part);
}

// The solves of a batch of boxes in one cooperative launch.  The blocks form groups of
// gsize blocks; each group takes the next box from a device work queue (the boxes are
// queued largest first), copies its arguments to shared memory, runs its whole solve with
// the group's own barrier and partial sums, and takes the next box until none is left.
template <class T>
__global__ void __launch_bounds__(kPT, 1) ir_solve_batched(const PSolveArgs<T> *__restrict__ boxes, int nbox,
                                                          int gsize, int *queue, int *slot, GridBar *bars,
                                                          double *parts, int *err) {
  __shared__ PShared sh;
  __shared__ PSolveArgs<T> A;
  const int grp = blockIdx.x / gsize;
  const Grp g{(int)(blockIdx.x % gsize), gsize, bars + grp, err};
  double *part = parts + (size_t)grp * kPSlots * kPMaxBlocks;
  for (;;) {
    if (g.rank == 0 && threadIdx.x == 0) slot[grp] = atomicAdd(queue, 1);
    if (!gsync(g)) return;  // publishes the slot to the group
    const int b = __ldcg(slot + grp);
    if (b >= nbox) return;
    static_assert(sizeof(PSolveArgs<T>) % sizeof(int) == 0, "argument block copied as words");
    const int *src = reinterpret_cast<const int *>(boxes + b);
    int *dst = reinterpret_cast<int *>(&A);
    for (int k = threadIdx.x; k < (int)(sizeof(PSolveArgs<T>) / sizeof(int)); k += blockDim.x) dst[k] = src[k];
    __syncthreads();
    if (!solve_body(A, g, sh, part)) return;
    __syncthreads();  // the next box's arguments overwrite A
  }
}

}  // namespace

// The hierarchy and Krylov vectors of one inner precision T: float for the mixed path,
// double for the FP64 multigrid path.
template <class T>
struct MgLevel {
  int n = 0, w = 0;
  size_t ld = 0;
  int *col = nullptr;
  T *val = nullptr, *dinv = nullptr;
  // the aggregation (MgStruct's arrays, not owned)
  const int *agg = nullptr;                         // node -> coarser node
  const int *mptr = nullptr, *mem = nullptr;        // members on the finer level (levels >= 1)
  T *x = nullptr, *x2 = nullptr, *b = nullptr, *r = nullptr;
  bool owns_matrix = true;
};

// The aggregation of the current cells, level by level: octree-parent codes, the
// node -> aggregate map and each aggregate's members.  Only the cell codes go in, so it is
// built while the GFD assembly runs (apc_mg_structure_during_assembly); the operators
// (Galerkin products) follow the assembly, in the precision of the solve.
struct MgStructLevel {
  int n = 0;
  const uint64_t *code = nullptr;       // level 0: the context's cell codes
  uint64_t *own_code = nullptr;         // levels >= 1
  int *agg = nullptr;                   // node -> coarser node (every level but the last)
  int *mptr = nullptr, *mem = nullptr;  // members on the finer level (levels >= 1)
};

struct MgStruct {
  MgStructLevel lv[kMaxLevels];
  int nlev = 0;
  unsigned gen = 0;      // the selection it belongs to (apc_context::select_gen; 0: none)
  bool on_side = false;  // built on the side stream, after which side_ev[2] was recorded
};

template <class T>
struct MgHier {
  MgLevel<T> lv[kMaxLevels];
  int nlev = 0;
  T *coarse_inv = nullptr;
  int coarse_n = 0;
  T *uval = nullptr;  // coarse rows before the ELL transpose
  // FGMRES: basis V, preconditioned vectors Z, V-cycle in/out, correction
  T *V = nullptr, *Z = nullptr, *vin = nullptr, *vout = nullptr, *dvec = nullptr;
};

struct MgWork {
  MgStruct st;
  MgHier<float> h32;
  MgHier<double> h64;
  // hierarchy temporaries: parent-code sort, flags, coarse rows before the ELL transpose
  uint64_t *pkey = nullptr, *pkey_alt = nullptr;
  uint32_t *pidx = nullptr, *pidx_alt = nullptr;
  int *eflag = nullptr, *epos = nullptr, *ucol = nullptr, *rowstart = nullptr;
  size_t vn = 0;
  double *partial = nullptr, *dots = nullptr;
  unsigned *counter = nullptr;
  IrState *state = nullptr;
  void *host = nullptr;  // pinned readback of the state
  int *total = nullptr;
  // each mixed solve of the step as one graph, captured on c->s with the loop bodies on
  // two side streams
  cudaStream_t cap[2] = {nullptr, nullptr};
  cudaGraph_t solve_graph[2] = {nullptr, nullptr};  // density, potential
  cudaGraphExec_t solve_exec[2] = {nullptr, nullptr};
  int64_t vcycle_nodes[2] = {0, 0};
  // the hierarchy built while the density solve runs (apc_mg_prebuild)
  cudaStream_t side = nullptr;
  // operator assembled (main), hierarchy built (side), aggregation built (side)
  cudaEvent_t side_ev[3] = {nullptr, nullptr, nullptr};
  bool prebuilt = false;
  // the persistent solve kernel: partial sums, grid barrier, outcome (+ its pinned copy)
  double *ppart = nullptr;
  GridBar *pbar = nullptr;
  PResult *pres = nullptr;
  PResult *pres_host = nullptr;
  // the device-side coarse inverse's outcome (0 or 1 = singular) and its pinned copy,
  // checked after the next solve's readback
  int *cstat = nullptr;
  int *cstat_host = nullptr;
  bool tail_smem_set = false;  // the staged tail kernels may take kTailSmemMax
  // the numeric build's per-level widths (device, and its pinned readback; [kMaxLevels + 1]
  // is the ELL overflow flag) and the ELL slots allocated per level (host, the widest seen)
  int *wdev = nullptr;
  int *whost = nullptr;
  int wslots[kMaxLevels] = {};
  // a solve prepared for a batched launch (apc_mg_batched_solve): its arguments, which
  // solve it is, and whether it is multigrid-preconditioned
  PSolveArgs<float> deferred32{};
  PSolveArgs<double> deferred64{};
  int deferred_which = -1;
  bool deferred_mg = false;
};

static MgWork *mg(apc_context *c) {
  if (!c->mg) c->mg = new MgWork();
  return c->mg;
}

template <class T>
MgHier<T> &hier(MgWork *m);
template <>
MgHier<float> &hier<float>(MgWork *m) {
  return m->h32;
}
template <>
MgHier<double> &hier<double>(MgWork *m) {
  return m->h64;
}

template <class T>
PSolveArgs<T> &deferred(MgWork *m);
template <>
PSolveArgs<float> &deferred<float>(MgWork *m) {
  return m->deferred32;
}
template <>
PSolveArgs<double> &deferred<double>(MgWork *m) {
  return m->deferred64;
}

template <class T>
static void free_hier(apc_context *c, MgHier<T> &H) {
  for (auto &L : H.lv) {
    if (L.owns_matrix) {
      apc_free(c, L.col);
      apc_free(c, L.val);
    }
    apc_free(c, L.dinv);
    apc_free(c, L.x);
    apc_free(c, L.x2);
    apc_free(c, L.b);
    apc_free(c, L.r);
  }
  void *p[] = {H.coarse_inv, H.uval, H.V, H.Z, H.vin, H.vout, H.dvec};
  for (void *q : p) apc_free(c, q);
}

void apc_mg_free(apc_context *c) {
  MgWork *m = c->mg;
  if (!m) return;
  free_hier(c, m->h32);
  free_hier(c, m->h64);
  for (auto &L : m->st.lv) {
    apc_free(c, L.own_code);
    apc_free(c, L.agg);
    apc_free(c, L.mptr);
    apc_free(c, L.mem);
  }
  void *p[] = {m->pkey, m->pkey_alt, m->pidx, m->pidx_alt, m->eflag, m->epos, m->ucol,
               m->rowstart, m->partial, m->dots, m->counter, m->state, m->total, m->ppart, m->pbar, m->pres,
               m->cstat, m->wdev};
  for (void *q : p) apc_free(c, q);
  if (m->host) cudaFreeHost(m->host);
  if (m->pres_host) cudaFreeHost(m->pres_host);
  if (m->cstat_host) cudaFreeHost(m->cstat_host);
  if (m->whost) cudaFreeHost(m->whost);
  for (int k = 0; k < 2; ++k) {
    if (m->solve_exec[k]) cudaGraphExecDestroy(m->solve_exec[k]);
    if (m->solve_graph[k]) cudaGraphDestroy(m->solve_graph[k]);
  }
  for (cudaStream_t q : m->cap)
    if (q) cudaStreamDestroy(q);
  if (m->side) cudaStreamDestroy(m->side);
  for (cudaEvent_t e : m->side_ev)
    if (e) cudaEventDestroy(e);
  delete m;
  c->mg = nullptr;
}

static int read_int(apc_context *c, const int *dev, int *host) {
  // through the context's pinned word: a pageable destination would be staged
  APC_CUDA_TRY(c, cudaMemcpyAsync(c->h_pinned + 10, dev, sizeof(int), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, apc_stream_wait(c));
  *host = c->h_pinned[10];
  return APC_OK;
}

// Build the hierarchy over the current Jacobi-scaled potential operator in precision T
// (c->a2f or c->a2d) and the cell codes.
template <class T>
static const T *scaled_potential(const apc_context *c);
template <>
const float *scaled_potential<float>(const apc_context *c) {
  return c->a2f;
}
template <>
const double *scaled_potential<double>(const apc_context *c) {
  return c->a2d;
}

// The aggregation on c->s: level l + 1's nodes are the distinct parents (code >> 3) of
// level l's, in code order, down to kCoarsest nodes or until nothing coarsens.
static int mg_structure(apc_context *c) {
  MgWork *m = mg(c);
  MgStruct &S = m->st;
  S.gen = 0;
  S.on_side = false;
  S.lv[0].n = c->nc + c->nv;
  S.lv[0].code = c->ccode;
  if (!m->total) APC_TRY(apc_alloc(c, (void **)&m->total, 4 * sizeof(int)));
  int lev = 0;
  while (S.lv[lev].n > kCoarsest && lev + 1 < kMaxLevels) {
    MgStructLevel &F = S.lv[lev];
    MgStructLevel &C = S.lv[lev + 1];
    const int nf = F.n;
    APC_TRY(apc_ensure(c, &m->pkey, (size_t)nf));
    APC_TRY(apc_ensure(c, &m->pkey_alt, (size_t)nf));
    APC_TRY(apc_ensure(c, &m->pidx, (size_t)nf));
    APC_TRY(apc_ensure(c, &m->pidx_alt, (size_t)nf));
    APC_TRY(apc_ensure(c, &F.agg, (size_t)nf));
    parent_codes<<<grid_for(nf), kT, 0, c->s>>>(nf, F.code, m->pkey, m->pidx);
    apc_count_launch(c);
    bool alt = false;
    // level 0 is in the reference's cell order; coarser levels are already sorted by
    // code, and so are their parents' codes
    if (lev == 0) {
      // parent codes of cells at level <= D have at most 3 D - 2 significant bits; the
      // deepest cell level is one below the deepest top-down opened level
      const int deepest = (int)c->td_level_off.size();
      const int bits = std::min(64, 3 * deepest + 1);
      APC_TRY(apc_radix_sort_u64(c, m->pkey, m->pidx, m->pkey_alt, m->pidx_alt, nf, 0, bits, &alt));
    }
    uint64_t *pk = alt ? m->pkey_alt : m->pkey;
    uint32_t *pi = alt ? m->pidx_alt : m->pidx;
    APC_TRY(apc_ensure(c, &m->eflag, (size_t)nf + 1));
    APC_TRY(apc_ensure(c, &m->epos, (size_t)nf + 1));
    change_flags_u64<<<grid_for(nf), kT, 0, c->s>>>(nf, pk, m->eflag);
    apc_count_launch(c);
    APC_TRY(apc_exclusive_scan(c, m->eflag, m->epos, nf, m->total));
    int nc = 0;
    APC_TRY(read_int(c, m->total, &nc));
    if (nc >= nf) break;  // no coarsening left
    C.n = nc;
    APC_TRY(apc_ensure(c, &C.own_code, (size_t)nc + 1));
    APC_TRY(apc_ensure(c, &C.mptr, (size_t)nc + 1));
    APC_TRY(apc_ensure(c, &C.mem, (size_t)nf + 1));
    C.code = C.own_code;
    aggregate_map<<<grid_for(nf), kT, 0, c->s>>>(nf, pk, pi, m->eflag, m->epos, F.agg, C.own_code, C.mptr, C.mem);
    apc_count_launch(c);
    APC_CUDA_TRY(c, cudaGetLastError());
    ++lev;
  }
  S.nlev = lev + 1;
  S.gen = c->select_gen;
  return APC_OK;
}

// The operators over the aggregation, on c->s: the Jacobi-scaled potential operator in
// precision T on level 0, Galerkin products below it, the coarsest level's inverse.
template <class T>
static int mg_build(apc_context *c) {
  MgWork *m = mg(c);
  MgStruct &S = m->st;
  if (S.gen == 0 || S.gen != c->select_gen) {
    APC_TRY(mg_structure(c));
  } else if (S.on_side && c->s != m->side) {
    APC_CUDA_TRY(c, cudaStreamWaitEvent(c->s, m->side_ev[2], 0));
  }
  MgHier<T> &H = hier<T>(m);
  const int n0 = c->nc + c->nv;
  MgLevel<T> &L0 = H.lv[0];
  L0.n = n0;
  L0.w = c->ell_w;
  L0.ld = (size_t)c->m_cap;
  L0.col = c->ell_col;
  L0.val = const_cast<T *>(scaled_potential<T>(c));
  L0.owns_matrix = false;
  APC_TRY(apc_ensure(c, &L0.dinv, (size_t)n0 + 1));
  APC_TRY(apc_ensure(c, &L0.x, (size_t)n0 + 1));
  APC_TRY(apc_ensure(c, &L0.x2, (size_t)n0 + 1));
  APC_TRY(apc_ensure(c, &L0.b, (size_t)n0 + 1));
  APC_TRY(apc_ensure(c, &L0.r, (size_t)n0 + 1));
  ell_dinv<T><<<grid_for(n0), kT, 0, c->s>>>(n0, L0.ld, L0.val, L0.dinv);
  apc_count_launch(c);
  // Every level's Galerkin product and ELL are queued without a host round trip: the
  // kernels read each level's width from wdev, and the ELL is allocated for the widths of
  // the last build (at least 32 slots).  One readback at the end gives the widths; when a
  // level is wider than its allocation, the build runs again with room for it (the levels
  // below it were built from its truncated rows, so each repeat settles at least one more
  // level).
  if (!m->wdev) {
    APC_TRY(apc_alloc(c, (void **)&m->wdev, (kMaxLevels + 2) * sizeof(int)));
    APC_CUDA_TRY(c, cudaMallocHost((void **)&m->whost, (kMaxLevels + 2) * sizeof(int)));
  }
  int lev = 0;
  for (int attempt = 0; attempt <= S.nlev; ++attempt) {
  APC_CUDA_TRY(c, cudaMemsetAsync(m->wdev, 0, (kMaxLevels + 2) * sizeof(int), c->s));
  APC_CUDA_TRY(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->s));
  int *overflow = m->wdev + kMaxLevels + 1;
  lev = 0;
  for (; lev + 1 < S.nlev; ++lev) {
    MgLevel<T> &F = H.lv[lev];
    MgLevel<T> &C = H.lv[lev + 1];
    const int nf = F.n;
    const int nc = S.lv[lev + 1].n;
    F.agg = S.lv[lev].agg;
    C.n = nc;
    C.mptr = S.lv[lev + 1].mptr;
    C.mem = S.lv[lev + 1].mem;
    // ---- Galerkin product, one warp per coarse row ----
    const int wcap = 256;
    APC_TRY(apc_ensure(c, &m->rowstart, (size_t)nc + 1));
    APC_TRY(apc_ensure(c, &m->ucol, (size_t)nc * wcap));
    APC_TRY(apc_ensure(c, &H.uval, (size_t)nc * wcap));
    galerkin_rows<<<std::max(1, std::min((nc + kGalWarps - 1) / kGalWarps, apc_sm_count(c) * 8)), 32 * kGalWarps, 0,
                    c->s>>>(nc, C.mptr, nf, C.mem, F.w, lev == 0 ? nullptr : m->wdev + lev, F.w, F.ld, F.col,
                            F.val, F.agg, wcap, m->rowstart, m->ucol, H.uval, c->d_err);
    max_int<<<grid_for(nc, 256), kT, 0, c->s>>>(nc, m->rowstart, m->wdev + lev + 1);
    apc_count_launch(c, 2);
    const int wslots = std::max(32, m->wslots[lev + 1]);
    C.w = wslots;  // until the readback below
    C.ld = (size_t)nc;
    APC_TRY(apc_ensure(c, &C.col, C.ld * wslots));
    APC_TRY(apc_ensure(c, &C.val, C.ld * wslots));
    APC_TRY(apc_ensure(c, &C.dinv, (size_t)nc + 1));
    APC_TRY(apc_ensure(c, &C.x, (size_t)nc + 1));
    APC_TRY(apc_ensure(c, &C.x2, (size_t)nc + 1));
    APC_TRY(apc_ensure(c, &C.b, (size_t)nc + 1));
    APC_TRY(apc_ensure(c, &C.r, (size_t)nc + 1));
    rows_to_ell<T><<<grid_for(nc), kT, 0, c->s>>>(nc, m->wdev + lev + 1, wslots, C.ld, wcap, m->rowstart, m->ucol,
                                                 H.uval, C.col, C.val, C.dinv, overflow);
    apc_count_launch(c);
    APC_CUDA_TRY(c, cudaGetLastError());
  }
  // the widths and the error flags in one round trip
  APC_CUDA_TRY(c, cudaMemcpyAsync(m->whost, m->wdev, (kMaxLevels + 2) * sizeof(int), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, cudaMemcpyAsync(c->h_pinned + 9, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, apc_stream_wait(c));
  if (c->h_pinned[9] & DERR_STENCIL_MANY) {
    c->err = "multigrid coarse row exceeds its buffers";
    return APC_ERR_UNSUPPORTED;
  }
  bool wider = false;
  for (int k = 1; k < S.nlev; ++k) {
    const int wk = m->whost[k];
    if (wk > std::max(32, m->wslots[k])) wider = true;
    m->wslots[k] = std::max(m->wslots[k], wk);
    H.lv[k].w = wk;
  }
  if (!wider) break;
  if (attempt == S.nlev) {
    c->err = "multigrid coarse level wider than its rebuilt allocation";
    return APC_ERR_UNSUPPORTED;
  }
  }
  H.lv[lev].agg = S.lv[lev].agg;
  H.nlev = lev + 1;
  {
    int first_tail = 0;
    while (first_tail < H.nlev - 1 && H.lv[first_tail].n > kTail) ++first_tail;
    if (H.nlev - first_tail > kTailLevels) {
      c->err = "multigrid hierarchy deeper than the single-block tail supports";
      return APC_ERR_UNSUPPORTED;
    }
  }
  // ---- coarsest level: explicit inverse in FP64 ----
  MgLevel<T> &K = H.lv[lev];
  const int n = K.n;
  if (n > 4 * kCoarsest) {
    c->err = "multigrid coarsening stalled";
    return APC_ERR_UNSUPPORTED;
  }
  APC_TRY(apc_ensure(c, &H.coarse_inv, (size_t)n * n + 1));
  H.coarse_n = n;
  if (!m->tail_smem_set) {
    APC_CUDA_TRY(c, cudaFuncSetAttribute(vcycle_tail_smem<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTailSmemMax));
    APC_CUDA_TRY(c, cudaFuncSetAttribute(vcycle_tail_smem<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTailSmemMax));
    m->tail_smem_set = true;
  }
  if (n <= kCoarseInvMax) {
    // on the device, in stream order: no host round trip; a singular operator is reported
    // by the solve that follows (check_coarse)
    if (!m->cstat) {
      APC_TRY(apc_alloc(c, (void **)&m->cstat, sizeof(int)));
      APC_CUDA_TRY(c, cudaMallocHost((void **)&m->cstat_host, sizeof(int)));
      APC_CUDA_TRY(c, cudaFuncSetAttribute(coarse_inverse<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           kCoarseInvMax * 2 * kCoarseInvMax * (int)sizeof(double)));
      APC_CUDA_TRY(c, cudaFuncSetAttribute(coarse_inverse<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           kCoarseInvMax * 2 * kCoarseInvMax * (int)sizeof(double)));
    }
    const size_t smem = (size_t)n * 2 * n * sizeof(double);
    coarse_inverse<T><<<1, 256, smem, c->s>>>(n, K.w, K.ld, K.col, K.val, H.coarse_inv, m->cstat);
    apc_count_launch(c);
    APC_CUDA_TRY(c, cudaGetLastError());
    APC_CUDA_TRY(c, cudaMemcpyAsync(m->cstat_host, m->cstat, sizeof(int), cudaMemcpyDeviceToHost, c->s));
    return APC_OK;
  }
  // a stalled coarsening leaves more rows: on the host
  std::vector<int> col(K.ld * K.w);
  std::vector<T> val(K.ld * K.w);
  APC_CUDA_TRY(c, cudaMemcpyAsync(col.data(), K.col, sizeof(int) * col.size(), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, cudaMemcpyAsync(val.data(), K.val, sizeof(T) * val.size(), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, apc_stream_wait(c));
  std::vector<double> a((size_t)n * n, 0.0), inv((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) {
    for (int s = 0; s < K.w; ++s) a[(size_t)i * n + col[(size_t)s * K.ld + i]] += val[(size_t)s * K.ld + i];
    inv[(size_t)i * n + i] = 1.0;
  }
  for (int k = 0; k < n; ++k) {  // Gauss-Jordan with partial pivoting
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(a[(size_t)i * n + k]) > std::fabs(a[(size_t)p * n + k])) p = i;
    if (a[(size_t)p * n + k] == 0.0) {
      c->err = "singular coarsest multigrid operator";
      return APC_ERR_RANK;
    }
    if (p != k)
      for (int j = 0; j < n; ++j) {
        std::swap(a[(size_t)p * n + j], a[(size_t)k * n + j]);
        std::swap(inv[(size_t)p * n + j], inv[(size_t)k * n + j]);
      }
    const double d = 1.0 / a[(size_t)k * n + k];
    for (int j = 0; j < n; ++j) {
      a[(size_t)k * n + j] *= d;
      inv[(size_t)k * n + j] *= d;
    }
    for (int i = 0; i < n; ++i) {
      if (i == k) continue;
      const double f = a[(size_t)i * n + k];
      if (f == 0.0) continue;
      for (int j = 0; j < n; ++j) {
        a[(size_t)i * n + j] -= f * a[(size_t)k * n + j];
        inv[(size_t)i * n + j] -= f * inv[(size_t)k * n + j];
      }
    }
  }
  std::vector<T> invf(inv.begin(), inv.end());
  APC_CUDA_TRY(c, cudaMemcpyAsync(H.coarse_inv, invf.data(), sizeof(T) * invf.size(), cudaMemcpyHostToDevice,
                                  c->s));
  APC_CUDA_TRY(c, apc_stream_wait(c));
  if (m->cstat_host) *m->cstat_host = 0;
  return APC_OK;
}

// After a host wait that follows the hierarchy build in stream order: the device-side
// coarse inverse's outcome.
static int check_coarse(apc_context *c) {
  MgWork *m = c->mg;
  if (m && m->cstat_host && *m->cstat_host) {
    c->err = "singular coarsest multigrid operator";
    return APC_ERR_RANK;
  }
  return APC_OK;
}

// x = V-cycle(b) on level l, launched on stream s; b and x are that level's buffers
template <class T>
static void vcycle(apc_context *c, cudaStream_t s, int l, const T *b, T *x) {
  MgHier<T> &H = hier<T>(c->mg);
  MgLevel<T> &L = H.lv[l];
  const int n = L.n;
  const int sweeps = c->cfg.mg_sweeps > 0 ? c->cfg.mg_sweeps : 2;
  // piecewise-constant prolongation under-corrects smooth errors; over-scaling the
  // coarse correction (1.8) with lightly damped Jacobi (0.95) took the 128^3 potential
  // solve from 48 to 29 FGMRES iterations
  const T omega = (T)(c->cfg.mg_omega > 0 ? c->cfg.mg_omega : 0.95);
  const T alpha = (T)(c->cfg.mg_alpha > 0 ? c->cfg.mg_alpha : 1.8);
  if (n <= kTail || l == H.nlev - 1) {
    // this level and every coarser one in a single block
    TailArgs<T> A{};
    A.nl = std::min(H.nlev - l, kTailLevels);
    A.inv = H.coarse_inv;
    A.sweeps = sweeps;
    A.omega = omega;
    A.alpha = alpha;
    for (int k = 0; k < A.nl; ++k) {
      MgLevel<T> &Q = H.lv[l + k];
      TailLevel<T> &D = A.L[k];
      D.n = Q.n;
      D.w = Q.w;
      D.ld = Q.ld;
      D.col = Q.col;
      D.val = Q.val;
      D.dinv = Q.dinv;
      D.agg = Q.agg;
      D.mptr = Q.mptr;
      D.mem = Q.mem;
      D.x = k == 0 ? x : Q.x;
      D.b = k == 0 ? const_cast<T *>(b) : Q.b;
      D.x2 = Q.x2;
      D.r = Q.r;
    }
    // staged in shared memory when the tail's levels fit (they do at 128^3: ~90 KB in FP32)
    const size_t tb = tail_smem_bytes(A);
    const bool staged = tb <= kTailSmemMax;
    const int threads = staged ? kTailSmemThreads : kTailThreads;
    // wide rows get several lanes while the block has lanes to spare
    for (int k = 0; k < A.nl; ++k) A.L[k].g = tail_lanes(A.L[k].n, A.L[k].w, threads);
    if (staged)
      vcycle_tail_smem<T><<<1, threads, tb, s>>>(A);
    else
      vcycle_tail<T><<<1, threads, 0, s>>>(A);
    apc_count_launch(c);
    return;
  }
  MgLevel<T> &C = H.lv[l + 1];
  // lanes per row: wide rows get several, and so do levels with few rows (up to one
  // resident lane-group per SM thread slot), whose time is load latency
  int g = L.w <= 24 ? 1 : (L.w <= 48 ? 4 : 8);
  const long long budget = (long long)apc_sm_count(c) * 1024;
  while (g < 16 && g < L.w && 2LL * g * n <= budget) g *= 2;
  const int G = grid_for((long long)n * g);
  auto op = [&](int kind, const T *xin, T *out) {
#define APC_ROW_OP(GG)                                                                                            \
  switch (kind) {                                                                                                 \
    case kOpFirst2:                                                                                               \
      row_op<GG, kOpFirst2, T><<<G, kT, 0, s>>>(n, L.w, L.ld, L.col, L.val, L.dinv, b, xin, L.agg, C.x, alpha,       \
                                            omega, out);                                                         \
      break;                                                                                                      \
    case kOpSweep:                                                                                                \
      row_op<GG, kOpSweep, T><<<G, kT, 0, s>>>(n, L.w, L.ld, L.col, L.val, L.dinv, b, xin, L.agg, C.x, alpha,        \
                                           omega, out);                                                          \
      break;                                                                                                      \
    case kOpResidual:                                                                                             \
      row_op<GG, kOpResidual, T><<<G, kT, 0, s>>>(n, L.w, L.ld, L.col, L.val, L.dinv, b, xin, L.agg, C.x, alpha,     \
                                              omega, out);                                                       \
      break;                                                                                                      \
    default:                                                                                                      \
      row_op<GG, kOpProlongSweep, T><<<G, kT, 0, s>>>(n, L.w, L.ld, L.col, L.val, L.dinv, b, xin, L.agg, C.x, alpha, \
                                                  omega, out);                                                   \
  }
    if (g == 1) {
      APC_ROW_OP(1)
    } else if (g == 2) {
      APC_ROW_OP(2)
    } else if (g == 4) {
      APC_ROW_OP(4)
    } else if (g == 8) {
      APC_ROW_OP(8)
    } else {
      APC_ROW_OP(16)
    }
#undef APC_ROW_OP
    apc_count_launch(c);
  };
  // Buffers alternate between x and L.x2.  The pre-smoothing result is placed so that the
  // `sweeps` post-smoothing sweeps, each flipping buffers, end in x.
  T *cur, *nxt;
  if (sweeps >= 2) {
    op(kOpFirst2, nullptr, x);
    cur = x;
    nxt = L.x2;
    for (int k = 2; k < sweeps; ++k) {
      op(kOpSweep, cur, nxt);
      std::swap(cur, nxt);
    }
  } else {
    jacobi_first<T><<<grid_for(n), kT, 0, s>>>(n, L.dinv, b, omega, L.x2);
    cur = L.x2;
    nxt = x;
    apc_count_launch(c);
  }
  if (l > 0) {
    // coarse levels are in code order: residual and restriction in one pass
    residual_restrict<T><<<grid_for((long long)C.n * 8), kT, 0, s>>>(C.n, C.mptr, C.mem, n, L.w, L.ld, L.col,
                                                                     L.val, b, cur, C.b);
    apc_count_launch(c);
  } else {
    op(kOpResidual, cur, L.r);
    restrict_sum<T><<<grid_for(C.n), kT, 0, s>>>(C.n, C.mptr, n, C.mem, L.r, C.b);
    apc_count_launch(c);
  }
  vcycle<T>(c, s, l + 1, C.b, C.x);
  if (n > kSplitProlongRows) {
    prolong_add<T><<<grid_for(n), kT, 0, s>>>(n, L.agg, C.x, alpha, cur);
    apc_count_launch(c);
    op(kOpSweep, cur, nxt);
  } else {
    op(kOpProlongSweep, cur, nxt);
  }
  std::swap(cur, nxt);
  for (int k = 1; k < sweeps; ++k) {
    op(kOpSweep, cur, nxt);
    std::swap(cur, nxt);
  }
}

// Add a conditional WHILE node after the current capture dependencies of stream s and
// make it the new dependency; *body receives the node's body graph.
static cudaError_t add_while(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraph_t *body) {
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd);
  if (e != cudaSuccess) return e;
  if (st != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureInvalidated;
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  e = cudaGraphAddNode(&node, g, deps, nd, &p);
  if (e != cudaSuccess) return e;
  *body = p.conditional.phGraph_out[0];
  return cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
}

template <class T>
struct IrSolveArgs {
  int which;               // 0 density, 1 potential
  bool mg;                 // V-cycle preconditioner (else none: GMRES on the scaled system)
  bool mg32;               // the V-cycle runs on the FP32 hierarchy (T = double only)
  int n, w;
  size_t ld;
  const int *col;          // ELL columns shared by both operators
  const T *valf;           // Jacobi-scaled operator D^-1 A in the inner precision
  const double *val, *b;   // FP64 operator (diagonal in slot 0) and rhs
  double *x, *r;           // solution, FP64 residual
  double rtol, atol, dtol, rtol_in;
  int max_it, max_outer, M;
};

// Capture one mixed solve:
//   init; residual (sets cond_outer)
//   while (cond_outer) {                       -- FP64 iterative refinement
//     v0 = D^-1 r / ||D^-1 r|| (sets cond_inner); normalise v0
//     while (cond_inner) {                     -- FP32 (F)GMRES cycle, right preconditioned
//       z = V-cycle(v_it) or v_it; v_it+1 = A z; CGS; Arnoldi scalars (sets cond_inner);
//       normalise
//     }
//     y = H^-1 g; d = Z y; x += ||D^-1 r|| d; residual (sets cond_outer)
//   }
// Both loops end by counters the kernels advance: at most max_outer corrections, M
// iterations per cycle, max_it iterations in all.
template <class T>
static int capture_solve(apc_context *c, const IrSolveArgs<T> &a) {
  MgWork *m = c->mg;
  MgHier<T> &H = hier<T>(m);
  const int n = a.n, slot = a.which;
  const size_t vn = m->vn;
  const int G = std::min(kRedBlocks, grid_for(n));
  const int Gs = grid_for(n, 1184);
  const bool reorth = c->cfg.mg_reorth != 0;
  double *h1 = m->dots, *h2 = m->dots + 34, *nr = m->dots + 68, *tmp = m->dots + 70;
  T *Z = a.mg ? H.Z : nullptr;
  // the V-cycle's input and output: this precision's, or the FP32 hierarchy's
  MgHier<float> &H32 = m->h32;
  const bool v32 = a.mg && a.mg32;
  T *vin = a.mg && !v32 ? H.vin : nullptr;
  float *vin32 = v32 ? H32.vin : nullptr;
  const int64_t l0 = c->launches;
  cudaStream_t s = c->s, s1 = m->cap[0], s2 = m->cap[1];
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    c->err = std::string("solve capture: ") + cudaGetErrorString(e);
    return APC_ERR_CUDA;
  }
  auto ok = [&](cudaError_t r) {
    if (e == cudaSuccess && r != cudaSuccess) e = r;
    return e == cudaSuccess;
  };
  cudaStreamCaptureStatus st;
  cudaGraph_t top = nullptr, body_out = nullptr, body_in = nullptr;
  cudaGraphConditionalHandle cond_out = 0, cond_in = 0;
  bool cap1 = false, cap2 = false;
  if (ok(cudaStreamGetCaptureInfo(s, &st, nullptr, &top, nullptr, nullptr)) &&
      ok(cudaGraphConditionalHandleCreate(&cond_out, top, 0, 0))) {
    ir_init<<<1, 1, 0, s>>>(m->state, a.rtol, a.atol, a.dtol, a.rtol_in, a.max_it, a.max_outer, a.M,
                            sizeof(T) == sizeof(double) ? 1 : 0);
    ir_bnorm<<<G, kT, 0, s>>>(n, a.val, a.b, m->state, m->partial, m->counter, tmp);
    ir_residual<<<G, kT, 0, s>>>(n, a.w, a.ld, a.col, a.val, a.b, a.x, a.r, m->state, m->partial, m->counter, tmp,
                                 cond_out);
    if (ok(cudaGetLastError()) && ok(add_while(s, cond_out, &body_out)) &&
        ok(cudaStreamBeginCaptureToGraph(s1, body_out, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal))) {
      cap1 = true;
      if (ok(cudaGraphConditionalHandleCreate(&cond_in, body_out, 0, 0))) {
        ir_to_inner<T><<<G, kT, 0, s1>>>(n, a.r, a.val, m->state, H.V, m->partial, m->counter, tmp, cond_in);
        if (v32)
          scale_next<T, float><<<Gs, kT, 0, s1>>>(n, m->state, H.V, vn, vin32);
        else
          scale_next<T><<<Gs, kT, 0, s1>>>(n, m->state, H.V, vn, vin);
        if (ok(cudaGetLastError()) && ok(add_while(s1, cond_in, &body_in)) &&
            ok(cudaStreamBeginCaptureToGraph(s2, body_in, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal))) {
          cap2 = true;
          const int64_t v0 = c->launches;
          if (v32)
            vcycle<float>(c, s2, 0, H32.vin, H32.vout);
          else if (a.mg)
            vcycle<T>(c, s2, 0, H.vin, H.vout);
          m->vcycle_nodes[slot] = c->launches - v0;
          // basis vectors per cycle: 16 (the potential's FGMRES(16)) or up to 32; the dot
          // accumulators are registers
          auto krylov = [&](auto nvt) {
            constexpr int NV = decltype(nvt)::value;
            if (v32)
              spmv_dots<T, float, NV><<<G, kT, 0, s2>>>(n, a.w, a.ld, a.col, a.valf, H32.vout, Z, H.V, vn,
                                                        m->state, m->partial, m->counter, h1);
            else
              spmv_dots<T, T, NV><<<G, kT, 0, s2>>>(n, a.w, a.ld, a.col, a.valf, a.mg ? H.vout : nullptr, Z, H.V,
                                                    vn, m->state, m->partial, m->counter, h1);
            if (reorth) {
              cgs_pass<1, T, NV><<<G, kT, 0, s2>>>(n, m->state, H.V, vn, h1, m->partial, m->counter, h2, nullptr,
                                                   nullptr, cond_in);
              cgs_pass<2, T, NV><<<G, kT, 0, s2>>>(n, m->state, H.V, vn, h2, m->partial, m->counter, nr, h1, h2,
                                                   cond_in);
            } else {
              cgs_pass<2, T, NV><<<G, kT, 0, s2>>>(n, m->state, H.V, vn, h1, m->partial, m->counter, nr, h1,
                                                   nullptr, cond_in);
            }
          };
          if (a.M <= 16)
            krylov(std::integral_constant<int, 16>{});
          else
            krylov(std::integral_constant<int, 32>{});
          if (v32)
            scale_next<T, float><<<Gs, kT, 0, s2>>>(n, m->state, H.V, vn, vin32);
          else
            scale_next<T><<<Gs, kT, 0, s2>>>(n, m->state, H.V, vn, vin);
          ok(cudaGetLastError());
        }
        if (cap2) {
          cudaGraph_t g2 = nullptr;
          ok(cudaStreamEndCapture(s2, &g2));
        }
        fg_finish<<<1, 32, 0, s1>>>(m->state);
        combine<T><<<Gs, kT, 0, s1>>>(n, a.mg ? H.Z : H.V, vn, m->state, H.dvec);
        ir_axpy<T><<<Gs, kT, 0, s1>>>(n, m->state, H.dvec, a.x);
        ir_residual<<<G, kT, 0, s1>>>(n, a.w, a.ld, a.col, a.val, a.b, a.x, a.r, m->state, m->partial, m->counter,
                                      tmp, cond_out);
        ok(cudaGetLastError());
      }
    }
    if (cap1) {
      cudaGraph_t g1 = nullptr;
      ok(cudaStreamEndCapture(s1, &g1));
    }
  }
  cudaGraph_t g = nullptr;
  ok(cudaStreamEndCapture(s, &g));
  c->launches = l0;
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    c->err = std::string("solve capture: ") + cudaGetErrorString(e);
    return APC_ERR_CUDA;
  }
  // the graph of the previous step usually differs only in kernel parameters: update
  // the executable in place, and instantiate only when the topology changed
  if (m->solve_exec[slot]) {
    cudaGraphExecUpdateResultInfo info{};
    if (cudaGraphExecUpdate(m->solve_exec[slot], g, &info) == cudaSuccess) {
      if (m->solve_graph[slot]) cudaGraphDestroy(m->solve_graph[slot]);
      m->solve_graph[slot] = g;
      c->prof.graph_updates += 1;
      return APC_OK;
    }
    cudaGetLastError();
    cudaGraphExecDestroy(m->solve_exec[slot]);
    m->solve_exec[slot] = nullptr;
  }
  if (m->solve_graph[slot]) cudaGraphDestroy(m->solve_graph[slot]);
  m->solve_graph[slot] = g;
  APC_CUDA_TRY(c, cudaGraphInstantiate(&m->solve_exec[slot], g, 0));
  c->prof.graph_instantiations += 1;
  return APC_OK;
}

// One solve of the mixed path: FP64 iterative refinement on the true Jacobi-
// preconditioned residual, each correction an FP32 (F)GMRES cycle on the Jacobi-scaled
// system.  For the potential with the multigrid option, builds the hierarchy over the
// current operator and right-preconditions with its V-cycle.  The solve is captured as
// one graph and run; the host reads the outcome once.
// Run one solve as the persistent kernel (ir_solve_persistent): the arguments carry the
// hierarchy's levels and the tail; `blocks` blocks of kPT threads, co-resident by the
// cooperative launch.  Returns APC_ERR_UNSUPPORTED when the kernel cannot be launched
// co-resident (the caller then uses the graph path).
// The persistent kernel's arguments for one prepared solve (buffers of the context).
template <class T>
static int fill_psolve(apc_context *c, const IrSolveArgs<T> &a, PSolveArgs<T> &P) {
  MgWork *m = c->mg;
  MgHier<T> &H = hier<T>(m);
  if (!m->ppart) {
    APC_TRY(apc_alloc(c, (void **)&m->ppart, sizeof(double) * (size_t)kPSlots * kPMaxBlocks));
    APC_TRY(apc_alloc(c, (void **)&m->pbar, sizeof(GridBar)));
    APC_TRY(apc_alloc(c, (void **)&m->pres, sizeof(PResult)));
  }
  if (!m->pres_host) APC_CUDA_TRY(c, cudaMallocHost((void **)&m->pres_host, sizeof(PResult)));
  P = PSolveArgs<T>{};
  P.n = a.n;
  P.w = a.w;
  P.ld = a.ld;
  P.col = a.col;
  P.valf = a.valf;
  P.val = a.val;
  P.b = a.b;
  P.x = a.x;
  P.r = a.r;
  P.V = H.V;
  P.Z = H.Z;
  P.vn = m->vn;
  P.M = a.M;
  P.use_mg = a.mg ? 1 : 0;
  P.sweeps = c->cfg.mg_sweeps > 0 ? c->cfg.mg_sweeps : 2;
  P.omega = (T)(c->cfg.mg_omega > 0 ? c->cfg.mg_omega : 0.95);
  P.alpha = (T)(c->cfg.mg_alpha > 0 ? c->cfg.mg_alpha : 1.8);
  if (a.mg) {
    P.nlev = H.nlev;
    P.tail = 0;
    while (P.tail < H.nlev - 1 && H.lv[P.tail].n > kTail) ++P.tail;
    for (int l = 0; l < H.nlev; ++l) {
      const MgLevel<T> &Q = H.lv[l];
      PLevel<T> &D = P.L[l];
      D.n = Q.n;
      D.w = Q.w;
      D.g = Q.w <= 24 ? 1 : (Q.w <= 48 ? 4 : 8);
      D.ld = Q.ld;
      D.col = Q.col;
      D.val = Q.val;
      D.dinv = Q.dinv;
      D.agg = Q.agg;
      D.mptr = Q.mptr;
      D.mem = Q.mem;
      D.x = Q.x;
      D.x2 = Q.x2;
      D.b = Q.b;
      D.r = Q.r;
    }
    TailArgs<T> &TA = P.ta;
    TA.nl = std::min(H.nlev - P.tail, kTailLevels);
    TA.inv = H.coarse_inv;
    TA.sweeps = P.sweeps;
    TA.omega = P.omega;
    TA.alpha = P.alpha;
    for (int k = 0; k < TA.nl; ++k) {
      const MgLevel<T> &Q = H.lv[P.tail + k];
      TailLevel<T> &D = TA.L[k];
      D.n = Q.n;
      D.w = Q.w;
      // lanes per row: each lane takes at most 8 of the row's slots (a row's slots are a
      // chain of dependent gathers per lane), the block's rows then run in rounds
      D.g = tail_lanes(Q.n, Q.w, kPT);
      D.ld = Q.ld;
      D.col = Q.col;
      D.val = Q.val;
      D.dinv = Q.dinv;
      D.agg = Q.agg;
      D.mptr = Q.mptr;
      D.mem = Q.mem;
      D.x = Q.x;
      D.b = Q.b;
      D.x2 = Q.x2;
      D.r = Q.r;
    }
  }
  P.rtol = a.rtol;
  P.atol = a.atol;
  P.dtol = a.dtol;
  P.rtol_in = a.rtol_in;
  P.max_it = a.max_it;
  P.max_outer = a.max_outer;
  P.exact_inner = sizeof(T) == sizeof(double) ? 1 : 0;
  P.part = m->ppart;
  P.bar = m->pbar;
  P.err = c->d_err;
  P.out = m->pres;
  return APC_OK;
}

template <class T>
static int persistent_solve(apc_context *c, const IrSolveArgs<T> &a, int blocks) {
  MgWork *m = c->mg;
  const void *kern = (const void *)ir_solve_persistent<T>;
  int occ = 0;
  APC_CUDA_TRY(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kPT, 0));
  if (occ < 1) return APC_ERR_UNSUPPORTED;
  blocks = std::max(1, std::min(blocks, std::min(kPMaxBlocks, apc_sm_count(c) * occ)));
  PSolveArgs<T> P;
  APC_TRY(fill_psolve<T>(c, a, P));
  APC_CUDA_TRY(c, cudaMemsetAsync(m->pbar, 0, sizeof(GridBar), c->s));
  APC_CUDA_TRY(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->s));
  void *args[] = {&P};
  APC_CUDA_TRY(c, cudaLaunchCooperativeKernel(kern, dim3(blocks), dim3(kPT), args, 0, c->s));
  apc_count_launch(c);
  return APC_OK;
}

// Algorithmic bytes of one multigrid solve (apc_profile.mg_bytes): every array a phase
// reads or writes, counted once per phase; S = sizeof(T), ELL rows cost w (S + 4).
//   refinement step: FP64 residual (w 12 + b, x, r), v_0 (r, D, v_0), solution update
//     (the cycle's basis vectors + x read and written);
//   Arnoldi step with j earlier basis vectors (j averaged over the cycles): SpMV (ELL, z,
//     w written), dots (w + j + 1 vectors), Gram-Schmidt update (w, j + 1 vectors, w);
//   V-cycle, per grid level of n rows: two-sweep pre-smoothing (ELL, b, D^-1, x written),
//     residual + restriction (ELL, x, b, coarse b written), prolongation + sweep (ELL, x,
//     b, D^-1, aggregate map, coarse x, out), each further sweep (ELL, x, b, D^-1, out);
//   the single-block tail: the same per level, from L2.
template <class TV>
static double solve_bytes(const MgHier<TV> &H, bool use_mg, int n, int w, int sweeps, int total_its, int outer,
                          double S_krylov = sizeof(TV)) {
  const double S = S_krylov, N = n;
  const double cyc = outer > 0 ? (double)total_its / outer : 0.0;
  const double jbar = cyc > 0 ? 0.5 * (cyc - 1.0) : 0.0;
  const double per_outer = N * (w * 12.0 + 24.0) + N * (16.0 + S) + N * (cyc * S + 16.0);
  double per_it = N * (w * (S + 4) + 2 * S) + N * (jbar + 2) * S + N * (jbar + 3) * S;
  if (use_mg) {
    const double S = sizeof(TV);  // the V-cycle's element size
    for (int l = 0; l < H.nlev; ++l) {
      const MgLevel<TV> &L = H.lv[l];
      const double nl = L.n, ell = L.w * (S + 4);
      const double nc = l + 1 < H.nlev ? H.lv[l + 1].n : 0.0;
      if (l + 1 < H.nlev) {
        per_it += nl * (ell + 3 * S);                   // pre-smoothing
        per_it += nl * (ell + 2 * S) + nc * S;          // residual + restriction
        per_it += nl * (ell + 4 * S + 4) + nc * S;      // prolongation + sweep
        per_it += (sweeps - 1) * nl * (ell + 3 * S);    // further sweeps
      } else {
        per_it += 2.0 * nl * nl * S;                    // dense coarsest solve (inverse, b, x)
      }
    }
  }
  return outer * per_outer + total_its * per_it;
}

template <class T>
static int ir_solve(apc_context *c, int which, bool use_mg, const double *val, const T *valf, const double *b,
                    double *x, double *r, int restart, double rtol_in, int *its, double *rnorm, int *reason,
                    int *refinements, int *levels, int (*during)(apc_context *)) {
  MgWork *m = mg(c);
  MgHier<T> &H = hier<T>(m);
  const int n = c->nc + c->nv;
  const size_t vn = ((size_t)n + 31) & ~(size_t)31;
  const int M = std::max(1, std::min(restart, kMaxM));
  // FP64 Krylov vectors with the V-cycle on the FP32 hierarchy
  const bool mg32 = use_mg && sizeof(T) == sizeof(double) && c->cfg.precision == APC_PREC_MIXED_VCYCLE;
  APC_TRY(apc_ensure(c, &H.V, vn * (M + 1)));
  if (use_mg) {
    APC_TRY(apc_ensure(c, &H.Z, vn * M));
    if (mg32) {
      APC_TRY(apc_ensure(c, &m->h32.vin, vn));
      APC_TRY(apc_ensure(c, &m->h32.vout, vn));
    } else {
      APC_TRY(apc_ensure(c, &H.vin, vn));
      APC_TRY(apc_ensure(c, &H.vout, vn));
    }
  }
  APC_TRY(apc_ensure(c, &H.dvec, vn));
  APC_TRY(apc_ensure(c, &m->partial, (size_t)kRedBlocks * 34));
  APC_TRY(apc_ensure(c, &m->dots, (size_t)4 * 34));
  m->vn = vn;
  if (!m->counter) {
    APC_TRY(apc_alloc(c, (void **)&m->counter, 4 * sizeof(unsigned)));
    APC_CUDA_TRY(c, cudaMemsetAsync(m->counter, 0, 4 * sizeof(unsigned), c->s));
  }
  if (!m->state) APC_TRY(apc_alloc(c, (void **)&m->state, sizeof(IrState)));
  if (!m->host) APC_CUDA_TRY(c, cudaMallocHost((void **)&m->host, sizeof(IrState)));
  for (int k = 0; k < 2; ++k)
    if (!m->cap[k]) APC_CUDA_TRY(c, cudaStreamCreateWithFlags(&m->cap[k], cudaStreamNonBlocking));
  const apc_config &cfg = c->cfg;
  const auto t0 = std::chrono::steady_clock::now();
  const bool prebuilt = use_mg && m->prebuilt;  // built during the density solve
  m->prebuilt = false;
  if (use_mg && !prebuilt) {
    APC_CUDA_TRY(c, apc_stream_wait(c));
    APC_TRY(mg32 ? mg_build<float>(c) : mg_build<T>(c));
  }
  const int nlev = mg32 ? m->h32.nlev : H.nlev;
  const int sweeps = c->cfg.mg_sweeps > 0 ? c->cfg.mg_sweeps : 2;
  auto bytes = [&](int its_, int outer_) {
    return mg32 ? solve_bytes<float>(m->h32, true, n, c->ell_w, sweeps, its_, outer_, sizeof(T))
                : solve_bytes<T>(H, true, n, c->ell_w, sweeps, its_, outer_);
  };
  IrSolveArgs<T> a{};
  a.which = which;
  a.mg = use_mg;
  a.mg32 = mg32;
  a.n = n;
  a.w = c->ell_w;
  a.ld = (size_t)c->m_cap;
  a.col = c->ell_col;
  a.valf = valf;
  a.val = val;
  a.b = b;
  a.x = x;
  a.r = r;
  a.rtol = cfg.gmres_rtol;
  a.atol = cfg.gmres_atol;
  a.dtol = cfg.gmres_dtol;
  a.rtol_in = rtol_in;
  a.max_it = cfg.gmres_max_it;
  // the FP32 multigrid corrections gain ~5 digits each; an FP64 correction is one
  // restart cycle of FGMRES; without a preconditioner a correction may gain little.  max_it
  // bounds the loop in every case
  a.max_outer = use_mg && sizeof(T) == sizeof(float) ? 40 : std::max(40, cfg.gmres_max_it);
  a.M = M;
  // one persistent kernel per solve unless the graph path is asked for (or needed: the
  // re-orthogonalising Gram-Schmidt and the FP32 V-cycle under FP64 vectors run only there)
  const bool can_persist = !cfg.mg_reorth && !mg32;
  bool persistent = can_persist && !cfg.mixed_solve_graphs;
  if (can_persist && c->defer_solve) {
    // prepared for a batched launch with other boxes' solves (apc_mg_batched_solve);
    // apc_ir_finish reads the outcome
    if (use_mg)
      c->prof.mg_build_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    APC_TRY(fill_psolve<T>(c, a, deferred<T>(m)));
    m->deferred_which = which;
    m->deferred_mg = use_mg;
    if (during) APC_TRY(during(c));
    *its = 0;
    *rnorm = 0.0;
    *reason = 0;
    *refinements = 0;
    *levels = use_mg ? nlev : 0;
    return APC_OK;
  }
  if (persistent) {
    // a density solve overlapped with the potential's hierarchy build keeps half of the
    // SMs free for it
    const int sms = apc_sm_count(c);
    const int want = std::max(1, (n + kPT - 1) / kPT);
    const int blocks = during ? std::max(1, std::min(want, sms / 2)) : want;
    if (use_mg)
      c->prof.mg_build_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    APC_CUDA_TRY(c, cudaEventRecord(c->kev[0], c->s));
    const int rc = persistent_solve<T>(c, a, blocks);
    if (rc == APC_ERR_UNSUPPORTED) {
      persistent = false;
    } else {
      APC_TRY(rc);
      APC_CUDA_TRY(c, cudaEventRecord(c->kev[1], c->s));
      APC_CUDA_TRY(c, cudaMemcpyAsync(m->pres_host, m->pres, sizeof(PResult), cudaMemcpyDeviceToHost, c->s));
      APC_CUDA_TRY(c, cudaMemcpyAsync(c->h_pinned + 2, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->s));
      if (during) APC_TRY(during(c));
      APC_CUDA_TRY(c, apc_stream_wait(c));
      APC_CUDA_TRY(c, cudaGetLastError());
      if (c->h_pinned[2] & DERR_KRYLOV) {
        c->err = "solve kernel grid barrier timed out";
        return APC_ERR_TIMEOUT;
      }
      if (use_mg) APC_TRY(check_coarse(c));
      const PResult &R = *m->pres_host;
      float ms = 0.f;
      APC_CUDA_TRY(c, cudaEventElapsedTime(&ms, c->kev[0], c->kev[1]));
      *its = R.total_its;
      *rnorm = R.rn;
      *reason = R.reason;
      *refinements = R.outer;
      *levels = use_mg ? nlev : 0;
      if (use_mg) {
        c->prof.mg_solve_ms += ms;
        c->prof.mg_iterations += R.total_its;
        c->prof.mg_bytes += bytes(R.total_its, R.outer);
      }
      return APC_OK;
    }
  }
  APC_TRY(capture_solve(c, a));
  if (use_mg)
    c->prof.mg_build_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  APC_CUDA_TRY(c, cudaEventRecord(c->kev[0], c->s));
  APC_CUDA_TRY(c, cudaGraphLaunch(m->solve_exec[which], c->s));
  APC_CUDA_TRY(c, cudaEventRecord(c->kev[1], c->s));
  APC_CUDA_TRY(c, cudaMemcpyAsync(m->host, m->state, sizeof(IrState), cudaMemcpyDeviceToHost, c->s));
  if (during) APC_TRY(during(c));
  APC_CUDA_TRY(c, apc_stream_wait(c));
  APC_CUDA_TRY(c, cudaGetLastError());
  if (use_mg) APC_TRY(check_coarse(c));
  const IrState &S = *reinterpret_cast<const IrState *>(m->host);
  float ms = 0.f;
  APC_CUDA_TRY(c, cudaEventElapsedTime(&ms, c->kev[0], c->kev[1]));
  *its = S.total_its;
  *rnorm = S.rn;
  *reason = S.reason;
  *refinements = S.outer;
  *levels = use_mg ? nlev : 0;
  const int per_it = (int)m->vcycle_nodes[which] + 3 + (cfg.mg_reorth != 0 ? 1 : 0);
  apc_count_launch(c, 3 + 6 * S.outer + per_it * S.total_its);
  if (use_mg) {
    c->prof.mg_solve_ms += ms;
    c->prof.mg_iterations += S.total_its;
    c->prof.mg_bytes += bytes(S.total_its, S.outer);
  }
  return APC_OK;
}

int apc_ir_solve(apc_context *c, int which, bool use_mg, const double *val, const double *b, double *x, double *r,
                 int restart, double rtol_in, int *its, double *rnorm, int *reason, int *refinements, int *levels,
                 int (*during)(apc_context *)) {
  // FP64 Krylov: the FP64 path, and MIXED_VCYCLE's potential; FP32 corrections otherwise
  if (c->cfg.precision == APC_PREC_FP64_MULTIGRID || (c->cfg.precision == APC_PREC_MIXED_VCYCLE && which == 1))
    return ir_solve<double>(c, which, use_mg, val, which == 0 ? c->a1d : c->a2d, b, x, r, restart, rtol_in, its,
                            rnorm, reason, refinements, levels, during);
  return ir_solve<float>(c, which, use_mg, val, which == 0 ? c->a1f : c->a2f, b, x, r, restart, rtol_in, its, rnorm,
                         reason, refinements, levels, during);
}

static int ensure_side(apc_context *c, MgWork *m) {
  if (!m->side) {
    // the highest priority: the hierarchy's kernels and round trips are the critical path
    // while the GFD kernels (or the density solve) fill the SMs beside them
    int least = 0, greatest = 0;
    APC_CUDA_TRY(c, cudaDeviceGetStreamPriorityRange(&least, &greatest));
    APC_CUDA_TRY(c, cudaStreamCreateWithPriority(&m->side, cudaStreamNonBlocking, greatest));
    for (cudaEvent_t &e : m->side_ev) APC_CUDA_TRY(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  return APC_OK;
}

// Runs while the GFD assembly's kernels execute on the context's stream: the aggregation
// of the new cells is built on the side stream.  It reads only the cell codes, which were
// complete when the selection returned to the host.
int apc_mg_structure_during_assembly(apc_context *c) {
  MgWork *m = mg(c);
  APC_TRY(ensure_side(c, m));
  const auto t0 = std::chrono::steady_clock::now();
  cudaStream_t main = c->s;
  c->s = m->side;
  int rc = mg_structure(c);
  if (rc == APC_OK && cudaEventRecord(m->side_ev[2], c->s) != cudaSuccess) rc = APC_ERR_CUDA;
  c->s = main;
  APC_TRY(rc);
  m->st.on_side = true;
  c->prof.mg_build_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return APC_OK;
}

int apc_mg_mark_assembled(apc_context *c) {
  MgWork *m = mg(c);
  APC_TRY(ensure_side(c, m));
  m->prebuilt = false;
  APC_CUDA_TRY(c, cudaEventRecord(m->side_ev[0], c->s));
  return APC_OK;
}

// Runs while the density solve's graph executes on the context's stream: the potential
// operator's FP32 copy and the multigrid hierarchy are built on the side stream, after
// the assembly recorded by apc_mg_mark_assembled.  The buffers they touch are not used by
// the density solve.  The library's helpers all work on c->s, so c->s names the side
// stream for the duration; allocations and releases are then ordered on it.
int apc_mg_prebuild(apc_context *c) {
  MgWork *m = c->mg;
  if (!m || !m->side) return APC_ERR_INVALID_ARG;
  const auto t0 = std::chrono::steady_clock::now();
  cudaStream_t main = c->s;
  APC_CUDA_TRY(c, cudaStreamWaitEvent(m->side, m->side_ev[0], 0));
  c->s = m->side;
  apc_potential_scaled(c, c->s);
  // the FP64 path's hierarchy is FP64; the mixed paths' V-cycles run on an FP32 one
  int rc = c->cfg.precision == APC_PREC_FP64_MULTIGRID ? mg_build<double>(c) : mg_build<float>(c);
  if (rc == APC_OK && cudaEventRecord(m->side_ev[1], c->s) != cudaSuccess) rc = APC_ERR_CUDA;
  c->s = main;
  APC_TRY(rc);
  APC_CUDA_TRY(c, cudaStreamWaitEvent(c->s, m->side_ev[1], 0));
  m->prebuilt = true;
  c->prof.mg_build_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return APC_OK;
}

bool apc_mg_prebuilt(const apc_context *c) { return c->mg && c->mg->prebuilt; }

void apc_mg_clear_prebuilt(apc_context *c) {
  if (c->mg) c->mg->prebuilt = false;
}

// ------------------------------------------------ batched solves across boxes (C4)

struct BatchSolveBuf {
  int dev = 0;
  void *args = nullptr;        // device copy of the boxes' PSolveArgs, queue order
  void *args_host = nullptr;   // pinned staging
  size_t args_bytes = 0;
  int *queue = nullptr;        // [0] next box; [1..] the groups' current slots
  GridBar *bars = nullptr;     // one barrier per group
  double *parts = nullptr;     // one [slot][block] partial-sum area per group
  int *err = nullptr;          // barrier time-out flag of the launch
  int *err_host = nullptr;
  int max_groups = 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};  // around the launch (timing)
};

BatchSolveBuf *apc_batch_solve_buf_create(int device) {
  BatchSolveBuf *b = new BatchSolveBuf();
  b->dev = device;
  int sms = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  b->max_groups = std::max(1, sms);
  bool ok = cudaMalloc((void **)&b->queue, sizeof(int) * (b->max_groups + 1)) == cudaSuccess &&
            cudaMalloc((void **)&b->bars, sizeof(GridBar) * b->max_groups) == cudaSuccess &&
            cudaMalloc((void **)&b->parts, sizeof(double) * (size_t)kPSlots * kPMaxBlocks * b->max_groups) ==
                cudaSuccess &&
            cudaMalloc((void **)&b->err, sizeof(int)) == cudaSuccess &&
            cudaMallocHost((void **)&b->err_host, sizeof(int)) == cudaSuccess &&
            cudaEventCreate(&b->ev[0]) == cudaSuccess && cudaEventCreate(&b->ev[1]) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    apc_batch_solve_buf_free(b);
    return nullptr;
  }
  return b;
}

void apc_batch_solve_buf_free(BatchSolveBuf *b) {
  if (!b) return;
  cudaFree(b->args);
  cudaFreeHost(b->args_host);
  cudaFree(b->queue);
  cudaFree(b->bars);
  cudaFree(b->parts);
  cudaFree(b->err);
  cudaFreeHost(b->err_host);
  for (cudaEvent_t e : b->ev)
    if (e) cudaEventDestroy(e);
  delete b;
}

// One cooperative launch for the prepared solves of the given contexts (all of the same
// inner precision T), on stream s after each context's ready event; boxes are queued
// largest first.  Group size: the share of the SMs the largest box would get if every
// block worked on rows in proportion, at least one block.
template <class T>
static int batched_launch(apc_context *const *ctx, int n, BatchSolveBuf *B, cudaStream_t s, float *ms) {
  std::vector<int> order(n);
  long long total = 0, nmax = 1;
  for (int i = 0; i < n; ++i) {
    order[i] = i;
    const long long rows = deferred<T>(ctx[i]->mg).n;
    total += rows;
    nmax = std::max(nmax, rows);
  }
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return deferred<T>(ctx[a]->mg).n > deferred<T>(ctx[b]->mg).n; });
  const void *kern = (const void *)ir_solve_batched<T>;
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kPT, 0) != cudaSuccess || occ < 1) {
    cudaGetLastError();
    return APC_ERR_UNSUPPORTED;
  }
  int sms = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, B->dev);
  const int blocks_all = sms * occ;
  int gsize = (int)std::min<long long>(blocks_all, (blocks_all * nmax + total - 1) / std::max(1ll, total));
  gsize = std::max(1, std::min(gsize, std::min(kPMaxBlocks, (int)((nmax + kPT - 1) / kPT))));
  const int groups = std::max(1, std::min(B->max_groups, blocks_all / gsize));
  const size_t bytes = sizeof(PSolveArgs<T>) * (size_t)n;
  if (bytes > B->args_bytes) {
    cudaFree(B->args);
    cudaFreeHost(B->args_host);
    B->args = B->args_host = nullptr;
    B->args_bytes = 0;
    if (cudaMalloc(&B->args, bytes) != cudaSuccess || cudaMallocHost(&B->args_host, bytes) != cudaSuccess) {
      cudaGetLastError();
      return APC_ERR_OUT_OF_MEMORY;
    }
    B->args_bytes = bytes;
  }
  PSolveArgs<T> *h = static_cast<PSolveArgs<T> *>(B->args_host);
  for (int k = 0; k < n; ++k) h[k] = deferred<T>(ctx[order[k]]->mg);
  for (int i = 0; i < n; ++i)
    if (cudaStreamWaitEvent(s, ctx[i]->batch_ev, 0) != cudaSuccess) return APC_ERR_CUDA;
  bool ok = cudaMemcpyAsync(B->args, B->args_host, bytes, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemsetAsync(B->queue, 0, sizeof(int) * (groups + 1), s) == cudaSuccess &&
            cudaMemsetAsync(B->bars, 0, sizeof(GridBar) * groups, s) == cudaSuccess &&
            cudaMemsetAsync(B->err, 0, sizeof(int), s) == cudaSuccess && cudaEventRecord(B->ev[0], s) == cudaSuccess;
  if (!ok) return APC_ERR_CUDA;
  const PSolveArgs<T> *dargs = static_cast<const PSolveArgs<T> *>(B->args);
  int *queue = B->queue, *slot = B->queue + 1;
  GridBar *bars = B->bars;
  double *parts = B->parts;
  int *err = B->err;
  int nbox = n;
  void *kargs[] = {(void *)&dargs, &nbox, &gsize, &queue, &slot, &bars, &parts, &err};
  if (cudaLaunchCooperativeKernel(kern, dim3(groups * gsize), dim3(kPT), kargs, 0, s) != cudaSuccess) {
    cudaGetLastError();
    return APC_ERR_CUDA;
  }
  if (cudaEventRecord(B->ev[1], s) != cudaSuccess ||
      cudaMemcpyAsync(B->err_host, B->err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return APC_ERR_CUDA;
  float t = 0.f;
  cudaEventElapsedTime(&t, B->ev[0], B->ev[1]);
  if (ms) *ms = t;
  for (int i = 0; i < n; ++i) ctx[i]->launches += 1;
  return (*B->err_host & DERR_KRYLOV) ? APC_ERR_TIMEOUT : APC_OK;
}

int apc_mg_batched_solve(apc_context *const *ctx, int n, BatchSolveBuf *B, cudaStream_t s, float *ms) {
  if (!B || n <= 0) return APC_ERR_INVALID_ARG;
  std::vector<apc_context *> f32, f64;
  for (int i = 0; i < n; ++i) {
    if (!ctx[i]->mg || ctx[i]->mg->deferred_which < 0) continue;
    (ctx[i]->cfg.precision == APC_PREC_FP64_MULTIGRID ? f64 : f32).push_back(ctx[i]);
  }
  float t = 0.f, total = 0.f;
  if (!f32.empty()) {
    APC_TRY(batched_launch<float>(f32.data(), (int)f32.size(), B, s, &t));
    total += t;
  }
  if (!f64.empty()) {
    APC_TRY(batched_launch<double>(f64.data(), (int)f64.size(), B, s, &t));
    total += t;
  }
  if (ms) *ms = total;
  return APC_OK;
}

// The outcome of the solve this context prepared for a batched launch, once the launch has
// completed: its iteration count, residual, reason and refinements; the profile counts its
// iterations and algorithmic bytes.  A no-op when no solve is pending.
int apc_ir_finish(apc_context *c, int *its, double *rnorm, int *reason, int *refinements) {
  MgWork *m = c->mg;
  if (!m || m->deferred_which < 0) return APC_OK;  // the solve ran at once (FP64 GMRES path)
  APC_CUDA_TRY(c, cudaMemcpyAsync(m->pres_host, m->pres, sizeof(PResult), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, apc_stream_wait(c));
  if (m->deferred_mg) APC_TRY(check_coarse(c));
  const PResult &R = *m->pres_host;
  *its = R.total_its;
  *rnorm = R.rn;
  *reason = R.reason;
  *refinements = R.outer;
  if (m->deferred_mg) {
    c->prof.mg_iterations += R.total_its;
    if (c->cfg.precision == APC_PREC_FP64_MULTIGRID) {
      const PSolveArgs<double> &P = m->deferred64;
      c->prof.mg_bytes += solve_bytes<double>(m->h64, true, P.n, P.w, P.sweeps, R.total_its, R.outer);
    } else {
      const PSolveArgs<float> &P = m->deferred32;
      c->prof.mg_bytes += solve_bytes<float>(m->h32, true, P.n, P.w, P.sweeps, R.total_its, R.outer);
    }
  }
  m->deferred_which = -1;
  return APC_OK;
}
