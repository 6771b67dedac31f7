// Restarted GMRES with left Jacobi preconditioning on the device (the FP64 path), and
// the solve entry point, which hands the mixed-precision path to mg.cu.
//
// Reference: Solver::Solve_Density / Solve_Potential (solver.cpp:182-293) call PETSc
// KSPGMRES + PCJACOBI (solver.cpp:196-204, 267-276).  The FP64 kernel follows PETSc
// 3.5's GMRES control flow:
//   - zero initial guess; left preconditioning r = D^-1 (b - A x);
//   - classical Gram-Schmidt, refinement "never";
//   - Givens rotations; happy-breakdown tolerance 1e-30;
//   - convergence on the preconditioned residual estimate against
//     max(rtol ||D^-1 b||, atol), divergence at dtol * ||D^-1 b||, DIVERGED_ITS at max_it.
//
// Design (B200): one persistent cooperative kernel per solve.  Every block owns a
// strided set of rows.
//   - Per Arnoldi step, one pass fuses SpMV + Jacobi + all dot products with the
//     basis, and a second pass fuses the Gram-Schmidt update + norm.  That is two grid
//     barriers per iteration.  With re-orthogonalisation (CGS2) it is three.
//   - Basis vectors are stored un-normalised with a separate scale, so normalisation
//     costs no pass.
//   - Each block reduces the per-block partial sums itself in a fixed order, so all
//     blocks hold identical Hessenberg / Givens state without another barrier.
//   - Data other blocks write is read through L2 (ld.cg).
//   - The grid barrier's spin is bounded.  On timeout it raises an error flag and an
//     abort flag, and every block leaves.
// At the problem sizes of interest the basis (M x (restart+1) words) and the ELL matrix
// sit in the 126 MB L2, so an iteration runs at L2 bandwidth plus barrier latency.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "apc_internal.cuh"

namespace {

constexpr int kThreads = 1024;              // one block per SM
constexpr int kWarpsPB = kThreads / 32;
constexpr int kMaxBlocks = 256;             // partial sums are laid out [slot][block]
constexpr int kMaxRestart = 255;            // basis vectors of the large instantiation, minus one
constexpr int kSlots = kMaxRestart + 2;     // slots per partial-sum buffer: the dots, and one norm
constexpr int kNormSlot = kSlots - 1;


enum {
  KSP_CONVERGED_RTOL = 2,
  KSP_CONVERGED_ATOL = 3,
  KSP_DIVERGED_NULL = -2,
  KSP_DIVERGED_ITS = -3,
  KSP_DIVERGED_DTOL = -4,
  KSP_DIVERGED_BREAKDOWN = -5,
  KSP_DIVERGED_NANORINF = -9,
};

template <class T>
struct GmresArgs {
  int n;                // rows
  int w;                // ELL width
  size_t ld;            // ELL leading dimension
  const int *col;       // [slot][row]
  const T *val;         // [slot][row], slot 0 = diagonal
  const T *b;           // rhs
  T *x;                 // solution (out)
  T *U;                 // (restart+1) x n basis, un-normalised
  size_t un;            // basis leading dimension
  double *hh;           // per-block Hessenberg, (restart+1) x restart, when it exceeds shared memory
  double *part;         // 2 x kSlots x kMaxBlocks partial sums
  GridBar *bar;
  int *err;
  int restart;
  double rtol, atol, dtol;
  int max_it;
  int *out_its;
  int *out_reason;
  double *out_rnorm;
};

template <class T>
__device__ __forceinline__ T ldcg(const T *p) {
  return __ldcg(p);
}

// sum of slot j over all blocks' partials, identical in every block: each lane adds a
// fixed strided subset with independent loads (one L2 round trip), then a shuffle tree
__device__ __forceinline__ void gather_partials(const double *part, int nblocks, int nv, double *out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j = warp; j < nv; j += kWarpsPB) {
    const double *row = part + (size_t)j * kMaxBlocks;
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < kMaxBlocks / 32; ++k) {
      const int b = lane + 32 * k;
      if (b < nblocks) v += __ldcg(row + b);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) out[j] = v;
  }
}

__device__ __forceinline__ void put_partial(double *part, int j, double v) {
  part[(size_t)j * kMaxBlocks + blockIdx.x] = v;
}

__device__ __forceinline__ int converged_default(int n_its, double rnorm, double rtol, double atol,
                                                 double dtol, double &ttol, double &rnorm0) {
  if (n_its == 0) {
    ttol = fmax(rtol * rnorm, atol);
    rnorm0 = rnorm;
  }
  if (rnorm != rnorm) return KSP_DIVERGED_NANORINF;
  if (rnorm <= ttol) return rnorm < atol ? KSP_CONVERGED_ATOL : KSP_CONVERGED_RTOL;
  if (rnorm >= dtol * rnorm0) return KSP_DIVERGED_DTOL;
  return 0;
}

// sum of one value per thread over the block; the result is valid in warp 0
__device__ __forceinline__ double block_sum(double v, double *sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) sm[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    r = lane < kWarpsPB ? sm[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;
}

// The block's partial dot products <a, u_j>, j < nv, over its row range [r0, r1):
// every warp covers a contiguous sub-range with coalesced loads, four basis vectors per
// sweep, then the warps' sums are added in a fixed order and published as partials.
template <class T>
__device__ __forceinline__ void block_dots(const T *a, const T *U, size_t un, int r0, int r1, int nv,
                                           double *sm_red, double *part) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int per = (r1 - r0 + kWarpsPB - 1) / kWarpsPB;
  const int ws = r0 + warp * per, we = min(r1, ws + per);
  // 32 basis vectors at a time through the [warp][32] staging array
  for (int c0 = 0; c0 < nv; c0 += 32) {
    const int cn = min(32, nv - c0);
    for (int j0 = 0; j0 < cn; j0 += 4) {
      double v[4] = {0.0, 0.0, 0.0, 0.0};
      for (int r = ws + lane; r < we; r += 32) {
        const double ar = (double)ldcg(a + r);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (j0 + q < cn) v[q] += ar * (double)ldcg(U + (size_t)(c0 + j0 + q) * un + r);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double t = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0 && j0 + q < cn) sm_red[warp * 33 + j0 + q] = t;
      }
    }
    __syncthreads();
    if ((int)threadIdx.x < cn) {
      double t = 0.0;
      for (int wv = 0; wv < kWarpsPB; ++wv) t += sm_red[wv * 33 + threadIdx.x];
      put_partial(part, c0 + threadIdx.x, t);
    }
    if (c0 + 32 < nv) __syncthreads();
  }
}

// t -/+= sum_{j <= last} coef[j] u_j[i], one term at a time in j order.  Up to 32 vectors
// the loop is unrolled with predicates (independent loads); above, a plain loop.
template <int MAXV, bool SUB, class T>
__device__ __forceinline__ double basis_axpy(double t, const T *U, size_t un, int i, const double *coef,
                                             int last) {
  if constexpr (MAXV <= 32) {
#pragma unroll
    for (int j = 0; j < MAXV; ++j)
      if (j <= last) {
        const double u = (double)ldcg(U + (size_t)j * un + i);
        t = SUB ? t - coef[j] * u : t + coef[j] * u;
      }
  } else {
#pragma unroll 8
    for (int j = 0; j <= last; ++j) {
      const double u = (double)ldcg(U + (size_t)j * un + i);
      t = SUB ? t - coef[j] * u : t + coef[j] * u;
    }
  }
  return t;
}

// Each block owns the contiguous rows [r0, r1); within a pass every thread takes rows
// r0 + threadIdx.x + k * blockDim.x.
//
// MAXV bounds the basis (restart <= MAXV - 1).  Up to 32 vectors the Hessenberg matrix
// lives in shared memory; above (PETSc production runs use restart 200), in the block's
// own slice of global memory, written and read by thread 0 of that block only.
template <class T, bool REORTH, int MAXV>
__global__ void __launch_bounds__(kThreads, 1) gmres_kernel(GmresArgs<T> A) {
  constexpr bool kSmemH = MAXV <= 32;
  __shared__ double sm_red[kWarpsPB * 33];
  __shared__ double sh[MAXV + 1];      // reduced dots / norms of this step
  __shared__ double HHs[kSmemH ? (MAXV + 1) * MAXV : 1];
  __shared__ double cc[MAXV], ss[MAXV], grs[MAXV + 1], scale[MAXV + 1], coef[MAXV + 1];
  __shared__ int s_flow[4];
  __shared__ double s_res;

  const int nb = gridDim.x;
  const int m = A.restart;
  const int hld = kSmemH ? MAXV + 1 : m + 1;  // Hessenberg column stride
  double *HH = kSmemH ? HHs : A.hh + (size_t)blockIdx.x * (size_t)hld * m;
  const int rpb = (A.n + nb - 1) / nb;
  const int r0 = min(A.n, (int)blockIdx.x * rpb), r1 = min(A.n, r0 + rpb);
  double *partA = A.part;
  double *partB = A.part + (size_t)kSlots * kMaxBlocks;

  for (int i = r0 + threadIdx.x; i < r1; i += kThreads) A.x[i] = T(0);
  int its = 0, reason = 0, itcount = 0;
  bool guess_zero = true;
  double ttol = 0.0, rnorm0 = 0.0, res = 0.0;
  if (threadIdx.x == 0) s_res = 0.0;
  if (!grid_sync(A.bar, nb, A.err)) return;

  while (!reason) {
    // ---- initial residual: u0 = D^-1 (b - A x) ----
    double nrm = 0.0;
    for (int i = r0 + threadIdx.x; i < r1; i += kThreads) {
      const T d = A.val[i];
      const double di = d == T(0) ? 1.0 : 1.0 / (double)d;
      double r = (double)A.b[i];
      if (!guess_zero) {
        double sacc = 0.0;
        for (int k = 0; k < A.w; ++k) {
          const size_t at = (size_t)k * A.ld + i;
          sacc += (double)A.val[at] * (double)ldcg(A.x + A.col[at]);
        }
        r -= sacc;
      }
      const double u = di * r;
      A.U[i] = T(u);
      nrm += u * u;
    }
    {
      const double v = block_sum(nrm, sm_red);
      if (threadIdx.x == 0) put_partial(partB, 0, v);
    }
    if (!grid_sync(A.bar, nb, A.err)) return;
    gather_partials(partB, nb, 1, sh);
    __syncthreads();
    const double beta = sqrt(sh[0]);
    if (threadIdx.x == 0) {
      scale[0] = beta != 0.0 ? 1.0 / beta : 1.0;
      grs[0] = beta;
    }
    res = beta;
    if (res == 0.0) {
      reason = KSP_CONVERGED_ATOL;
      break;
    }
    reason = converged_default(its, res, A.rtol, A.atol, A.dtol, ttol, rnorm0);
    int it = 0;
    __syncthreads();
    while (!reason && it < m && its < A.max_it) {
      const T *uk = A.U + (size_t)it * A.un;
      T *w = A.U + (size_t)(it + 1) * A.un;
      const double sk = scale[it];
      // ---- pass A: w = D^-1 A v_it, then the block's dots with u_0..u_it ----
      for (int i = r0 + threadIdx.x; i < r1; i += kThreads) {
        const T d = A.val[i];
        const double di = d == T(0) ? 1.0 : 1.0 / (double)d;
        double sacc = 0.0;
        for (int k = 0; k < A.w; ++k) {
          const size_t at = (size_t)k * A.ld + i;
          sacc += (double)A.val[at] * (double)ldcg(uk + A.col[at]);
        }
        w[i] = T(di * sk * sacc);
      }
      __syncthreads();
      block_dots(w, A.U, A.un, r0, r1, it + 1, sm_red, partA);
      if (!grid_sync(A.bar, nb, A.err)) return;
      gather_partials(partA, nb, it + 1, sh);
      __syncthreads();
      if ((int)threadIdx.x <= it) {
        const double h = sh[threadIdx.x] * scale[threadIdx.x];  // <v_j, w>
        HH[it * hld + threadIdx.x] = h;
        coef[threadIdx.x] = h * scale[threadIdx.x];              // weight on u_j
      }
      __syncthreads();
      // ---- pass B: w -= sum_j h_j v_j, then its norm (CGS) or a second sweep (CGS2) ----
      double nr = 0.0;
      for (int i = r0 + threadIdx.x; i < r1; i += kThreads) {
        const double t = basis_axpy<MAXV, true>((double)ldcg(w + i), A.U, A.un, i, coef, it);
        const T tv = T(t);
        w[i] = tv;
        nr += (double)tv * (double)tv;
      }
      if (REORTH) {
        __syncthreads();
        block_dots(w, A.U, A.un, r0, r1, it + 1, sm_red, partB);
        if (!grid_sync(A.bar, nb, A.err)) return;
        gather_partials(partB, nb, it + 1, sh);
        __syncthreads();
        if ((int)threadIdx.x <= it) {
          const double h2 = sh[threadIdx.x] * scale[threadIdx.x];
          HH[it * hld + threadIdx.x] += h2;
          coef[threadIdx.x] = h2 * scale[threadIdx.x];
        }
        __syncthreads();
        nr = 0.0;
        for (int i = r0 + threadIdx.x; i < r1; i += kThreads) {
          const double t = basis_axpy<MAXV, true>((double)ldcg(w + i), A.U, A.un, i, coef, it);
          const T tv = T(t);
          w[i] = tv;
          nr += (double)tv * (double)tv;
        }
        const double v = block_sum(nr, sm_red);
        if (threadIdx.x == 0) put_partial(partA, kNormSlot, v);
        if (!grid_sync(A.bar, nb, A.err)) return;
        gather_partials(partA + (size_t)kNormSlot * kMaxBlocks, nb, 1, sh);
        __syncthreads();
      } else {
        const double v = block_sum(nr, sm_red);
        if (threadIdx.x == 0) put_partial(partB, 0, v);
        if (!grid_sync(A.bar, nb, A.err)) return;
        gather_partials(partB, nb, 1, sh);
        __syncthreads();
      }
      // ---- Hessenberg / Givens (KSPGMRESUpdateHessenberg), every block alike ----
      if (threadIdx.x == 0) {
        const double tt = sqrt(sh[0]);
        scale[it + 1] = tt != 0.0 ? 1.0 / tt : 1.0;
        double *hh = HH + it * hld;
        hh[it + 1] = tt;
        double hapbnd = fabs(tt / grs[it]);
        if (hapbnd > 1e-30) hapbnd = 1e-30;
        const int hapend = tt < hapbnd;
        for (int j = 1; j <= it; ++j) {
          const double t0 = hh[j - 1];
          hh[j - 1] = cc[j - 1] * t0 + ss[j - 1] * hh[j];
          hh[j] = cc[j - 1] * hh[j] - ss[j - 1] * t0;
        }
        int rs = 0;
        double rr = s_res;
        if (!hapend) {
          const double t = sqrt(hh[it] * hh[it] + hh[it + 1] * hh[it + 1]);
          if (t == 0.0) {
            rs = KSP_DIVERGED_NULL;
          } else {
            cc[it] = hh[it] / t;
            ss[it] = hh[it + 1] / t;
            grs[it + 1] = -(ss[it] * grs[it]);
            grs[it] = cc[it] * grs[it];
            hh[it] = cc[it] * hh[it] + ss[it] * hh[it + 1];
            rr = fabs(grs[it + 1]);
          }
        } else {
          rr = 0.0;
        }
        s_flow[0] = rs;
        s_flow[2] = hapend;
        s_res = rr;
      }
      __syncthreads();
      const int rs = s_flow[0], hapend = s_flow[2];
      if (!rs) res = s_res;
      ++it;
      ++its;
      if (rs) {
        reason = rs;
        break;
      }
      reason = converged_default(its, res, A.rtol, A.atol, A.dtol, ttol, rnorm0);
      if (hapend) {
        if (!reason) reason = KSP_DIVERGED_BREAKDOWN;
        break;
      }
    }
    // ---- KSPGMRESBuildSoln: back substitution, x += sum_j y_j v_j ----
    const int last = it - 1;
    if (last >= 0) {
      if (threadIdx.x == 0) {
        double *y = sh;
        const double hl = HH[last * hld + last];
        y[last] = hl != 0.0 ? grs[last] / hl : 0.0;
        for (int ii = 1; ii <= last; ++ii) {
          const int k = last - ii;
          double t = grs[k];
          for (int j = k + 1; j <= last; ++j) t -= HH[j * hld + k] * y[j];
          const double hkk = HH[k * hld + k];
          y[k] = hkk != 0.0 ? t / hkk : 0.0;
        }
        for (int j = 0; j <= last; ++j) coef[j] = y[j] * scale[j];
      }
      __syncthreads();
      for (int i = r0 + threadIdx.x; i < r1; i += kThreads) {
        const double t = basis_axpy<MAXV, false>(0.0, A.U, A.un, i, coef, last);
        A.x[i] = T((double)A.x[i] + t);
      }
    }
    itcount += it;
    if (itcount >= A.max_it) {
      if (!reason) reason = KSP_DIVERGED_ITS;
      break;
    }
    guess_zero = false;
    if (!grid_sync(A.bar, nb, A.err)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *A.out_its = its;
    *A.out_reason = reason;
    *A.out_rnorm = res;
  }
}

// ------------------------------------------------------------ mixed-path helpers

// D^-1 A in the inner precision T (rows past n zeroed)
template <class T>
__global__ void ell_to_scaled(size_t ld, int w, int n, const double *__restrict__ a, T *__restrict__ f) {
  const size_t count = ld * (size_t)w;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x) {
    const size_t i = e % ld;
    if ((int)i >= n) {
      f[e] = T(0);
      continue;
    }
    const double d = a[i];
    f[e] = (T)(d == 0.0 ? a[e] : a[e] / d);
  }
}

__global__ void zero_f64(int n, double *x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = 0.0;
}

// Self-check of the bounded wait: block 0 waits at the barrier for block 1, which
// leaves without arriving (a flag that nothing sets), so the wait must run out.
__global__ void bounded_wait_probe(GridBar *bar, int *err, long long limit) {
  if (blockIdx.x == 1) return;
  grid_sync(bar, 2u, err, limit);
}

}  // namespace

struct KrylovWork {
  size_t u_bytes = 0;
  void *U = nullptr;
  double *part = nullptr;
  int part_blocks = 0;
  GridBar *bar = nullptr;
  int *ires = nullptr;     // its, reason
  double *dres = nullptr;  // rnorm
  double *r = nullptr;  // FP64 residual of the mixed path
  float *a32 = nullptr;
  double *hh = nullptr;  // per-block Hessenberg slices of the large-restart kernel
  size_t hh_bytes = 0;
  int cap_n = 0;
  int occ64[2] = {0, 0}, occ32[2] = {0, 0};
};

void apc_krylov_free(apc_context *c) {
  KrylovWork *k = c->kw;
  if (!k) return;
  apc_free(c, k->U);
  apc_free(c, k->part);
  apc_free(c, k->bar);
  apc_free(c, k->ires);
  apc_free(c, k->dres);
  apc_free(c, k->r);
  apc_free(c, k->a32);
  apc_free(c, k->hh);
  delete k;
  c->kw = nullptr;
}

template <class T, bool RE>
static int launch_gmres(apc_context *c, int n, const T *val, const T *b, T *x, int restart, double rtol,
                        double atol, double dtol, int max_it, int *its, double *rnorm, int *reason,
                        const int *col = nullptr, int w = 0, size_t ld = 0) {
  KrylovWork *k = c->kw;
  if (restart < 1 || restart > kMaxRestart) {
    c->err = "GMRES restart must be in [1, 255]";
    return APC_ERR_INVALID_ARG;
  }
  const bool large = restart > 31;
  const void *kern = large ? (const void *)gmres_kernel<T, RE, kMaxRestart + 1>
                           : (const void *)gmres_kernel<T, RE, 32>;
  const size_t un = ((size_t)n + 31) & ~(size_t)31;
  const size_t need = un * (restart + 1) * sizeof(T);
  if (need > k->u_bytes) {
    apc_free(c, k->U);
    k->U = nullptr;
    APC_TRY(apc_alloc(c, &k->U, need));
    k->u_bytes = need;
  }
  int occ = 0;
  APC_CUDA_TRY(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, 0));
  if (occ < 1) {
    c->err = "GMRES kernel does not fit on an SM";
    return APC_ERR_CUDA;
  }
  int blocks = std::min(std::min(apc_sm_count(c), kMaxBlocks), std::max(1, (n + kThreads - 1) / kThreads));
  if (!k->part) {
    APC_TRY(apc_alloc(c, (void **)&k->part, sizeof(double) * 2 * kSlots * (size_t)kMaxBlocks));
    k->part_blocks = kMaxBlocks;
  }
  if (large) {
    const size_t hb = sizeof(double) * (size_t)blocks * (restart + 1) * restart;
    if (hb > k->hh_bytes) {
      apc_free(c, k->hh);
      k->hh = nullptr;
      APC_TRY(apc_alloc(c, (void **)&k->hh, hb));
      k->hh_bytes = hb;
    }
  }
  APC_CUDA_TRY(c, cudaMemsetAsync(k->bar, 0, sizeof(GridBar), c->s));
  GmresArgs<T> a;
  a.n = n;
  a.w = col ? w : c->ell_w;
  a.ld = col ? ld : (size_t)c->m_cap;
  a.col = col ? col : c->ell_col;
  a.val = val;
  a.b = b;
  a.x = x;
  a.U = (T *)k->U;
  a.un = un;
  a.hh = large ? k->hh : nullptr;
  a.part = k->part;
  a.bar = k->bar;
  a.err = c->d_err;
  a.restart = restart;
  a.rtol = rtol;
  a.atol = atol;
  a.dtol = dtol;
  a.max_it = max_it;
  a.out_its = k->ires;
  a.out_reason = k->ires + 1;
  a.out_rnorm = k->dres;
  void *args[] = {&a};
  APC_CUDA_TRY(c, cudaEventRecord(c->kev[0], c->s));
  APC_CUDA_TRY(c, cudaLaunchCooperativeKernel(kern, dim3(blocks), dim3(kThreads), args, 0, c->s));
  APC_CUDA_TRY(c, cudaEventRecord(c->kev[1], c->s));
  apc_count_launch(c);
  int hi[2];
  double hd;
  APC_CUDA_TRY(c, cudaMemcpyAsync(hi, k->ires, sizeof(hi), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, cudaMemcpyAsync(&hd, k->dres, sizeof(hd), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, apc_stream_wait(c));
  int derr = 0;
  APC_TRY(apc_read_errors(c, &derr));
  if (derr & DERR_KRYLOV) {
    c->err = "GMRES grid barrier timed out";
    return APC_ERR_TIMEOUT;
  }
  *its = hi[0];
  *reason = hi[1];
  *rnorm = hd;
  float ms = 0.f;
  APC_CUDA_TRY(c, cudaEventElapsedTime(&ms, c->kev[0], c->kev[1]));
  // algorithmic bytes of this launch (model documented in apcloud_gpu.h)
  const double S = sizeof(T), W = c->ell_w, rows = n;
  double per_row = 0.0;
  int left = hi[0], cycles = 0;
  while (left > 0 || cycles == 0) {
    const int in_cycle = std::min(left, restart);
    per_row += W * (S + 4) + 3 * S;  // restart residual
    for (int j = 0; j < in_cycle; ++j) per_row += W * (S + 4) + (2.0 * j + 6) * S + (RE ? (j + 3) * S : 0.0);
    per_row += (in_cycle + 1) * S;  // solution update
    left -= in_cycle;
    ++cycles;
    if (in_cycle == 0) break;
  }
  c->prof.krylov_launches += 1;
  c->prof.krylov_iterations += hi[0];
  c->prof.krylov_ms += ms;
  c->prof.krylov_bytes += per_row * rows;
  return APC_OK;
}

static int ensure_work(apc_context *c, int n) {
  if (!c->kw) {
    c->kw = new KrylovWork();
    APC_TRY(apc_alloc(c, (void **)&c->kw->bar, sizeof(GridBar)));
    APC_TRY(apc_alloc(c, (void **)&c->kw->ires, 4 * sizeof(int)));
    APC_TRY(apc_alloc(c, (void **)&c->kw->dres, 2 * sizeof(double)));
  }
  KrylovWork *k = c->kw;
  if (n > k->cap_n) {
    apc_free(c, k->r);
    k->r = nullptr;
    const int cap = n + n / 4 + 1024;
    APC_TRY(apc_alloc(c, (void **)&k->r, sizeof(double) * cap));
    k->cap_n = cap;
  }
  return APC_OK;
}

// FP64 GMRES (the FP64 path's kernel and stopping test) on an ELL matrix of the caller's:
// slot-major, leading dimension ld, width w, diagonal in slot 0; x starts from zero.
int apc_gmres_fp64_ell(apc_context *c, int n, int w, size_t ld, const int *col, const double *val,
                       const double *b, double *x, int *its, double *rnorm, int *reason) {
  APC_TRY(ensure_work(c, n));
  const int G = std::max(1, std::min((n + 255) / 256, 4096));
  zero_f64<<<G, 256, 0, c->s>>>(n, x);
  apc_count_launch(c);
  const apc_config &cfg = c->cfg;
  return launch_gmres<double, false>(c, n, val, b, x, cfg.gmres_restart, cfg.gmres_rtol, cfg.gmres_atol,
                                     cfg.gmres_dtol, cfg.gmres_max_it, its, rnorm, reason, col, w, ld);
}

// Solve A_which x = b.  FP64: one PETSc-semantics GMRES.  Mixed: FP64 iterative
// refinement on the true preconditioned residual, stopping at the same test
// ||D^-1 (b - A x)|| <= max(rtol ||D^-1 b||, atol); each correction solves the
// Jacobi-scaled system (D^-1 A) d = D^-1 r / ||D^-1 r|| in FP32 to the inner tolerance,
// by GMRES(CGS2) or, for the potential with the multigrid option, by FGMRES with the
// octree-aggregation V-cycle.
static void to_scaled(apc_context *c, cudaStream_t s, int which) {
  const int n = c->nc + c->nv;
  const size_t ell_count = (size_t)c->m_cap * c->ell_w;
  const int G = (int)std::min<size_t>((ell_count + 255) / 256, 8192);
  const double *a = which == 0 ? c->a1 : c->a2;
  const int prec = c->cfg.precision;
  // FP64: the FP64 path's operators, and MIXED_VCYCLE's potential (its FGMRES is FP64)
  if (prec == APC_PREC_FP64_MULTIGRID || (prec == APC_PREC_MIXED_VCYCLE && which == 1)) {
    ell_to_scaled<double><<<G, 256, 0, s>>>((size_t)c->m_cap, c->ell_w, n, a, which == 0 ? c->a1d : c->a2d);
    apc_count_launch(c);
  }
  // FP32: the mixed paths' operators (MIXED_VCYCLE: the density's FP32 corrections and the
  // potential's V-cycle hierarchy)
  if (prec == APC_PREC_MIXED || prec == APC_PREC_MIXED_VCYCLE) {
    ell_to_scaled<float><<<G, 256, 0, s>>>((size_t)c->m_cap, c->ell_w, n, a, which == 0 ? c->a1f : c->a2f);
    apc_count_launch(c);
  }
}

void apc_potential_scaled(apc_context *c, cudaStream_t s) { to_scaled(c, s, 1); }

int apc_krylov_solve(apc_context *c, int which, const double *b, double *x, int *its, double *rnorm,
                     int *reason, int *refinements, int (*during)(apc_context *)) {
  const int n = c->nc + c->nv;
  APC_TRY(ensure_work(c, n));
  KrylovWork *k = c->kw;
  const double *val = which == 0 ? c->a1 : c->a2;
  const apc_config &cfg = c->cfg;
  *refinements = 0;
  if (cfg.precision == APC_PREC_FP64) {
    return launch_gmres<double, false>(c, n, val, b, x, cfg.gmres_restart, cfg.gmres_rtol, cfg.gmres_atol,
                                       cfg.gmres_dtol, cfg.gmres_max_it, its, rnorm, reason);
  }
  // ---- mixed precision or FP64 multigrid: the refinement loop and its corrections run on
  //      the device as one graph per solve (mg.cu) ----
  const int G = std::max(1, std::min((n + 255) / 256, std::min(apc_sm_count(c) * 8, 4096)));
  // a prebuilt potential hierarchy (apc_mg_prebuild) came with its scaled operator
  const bool prebuilt = which == 1 && apc_mg_prebuilt(c);
  if (!prebuilt) to_scaled(c, c->s, which);
  if (cfg.warm_start) {
    APC_TRY(apc_warm_guess(c, which, x));
  } else {
    zero_f64<<<G, 256, 0, c->s>>>(n, x);
    apc_count_launch(c);
  }
  // inner restart: 16 for the multigrid FGMRES (a V-cycle per iteration makes short
  // cycles cheapest at 128^3) and for the density solve (it converges in about 10
  // iterations, and a 16-vector basis keeps the Krylov kernels' accumulators in half the
  // registers); 30 for the potential without a preconditioner
  const bool use_mg = which == 1 && cfg.mixed_precond == APC_PRECOND_MULTIGRID;
  const int m32 = cfg.mixed_restart > 0 ? cfg.mixed_restart : ((use_mg || which == 0) ? 16 : 30);
  // inner tolerance: a correction gains only ~2-3 digits of the FP64 residual whatever its
  // inner accuracy (the FP32 operator's rounding, ~cond(A) 6e-8, bounds it), so the
  // multigrid cycles stop at 1e-3; the density solve keeps 1e-5
  const double rtol_in = cfg.mixed_inner_rtol > 0 ? cfg.mixed_inner_rtol : (use_mg ? 1e-3 : 1e-5);
  int levels = 0;
  APC_TRY(apc_ir_solve(c, which, use_mg, val, b, x, k->r, m32, rtol_in, its, rnorm, reason, refinements, &levels,
                       during));
  if (use_mg) c->stats.mg_levels = levels;
  return APC_OK;
}

extern "C" int apc_check_bounded_wait(int device, int spin_limit) {
  if (spin_limit < 1 || spin_limit > (1 << 24)) return APC_ERR_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return APC_ERR_CUDA;
  }
  // the barrier word and the error flag
  void *buf = nullptr;
  if (cudaMalloc(&buf, sizeof(GridBar) + 16) != cudaSuccess) {
    cudaGetLastError();
    return APC_ERR_OUT_OF_MEMORY;
  }
  GridBar *bar = (GridBar *)buf;
  int *err = (int *)((char *)buf + sizeof(GridBar));
  int flag = 0;
  cudaError_t e = cudaMemset(buf, 0, sizeof(GridBar) + 16);
  if (e == cudaSuccess) {
    bounded_wait_probe<<<2, 32>>>(bar, err, spin_limit);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(&flag, err, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(buf);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return APC_ERR_CUDA;
  }
  return (flag & DERR_KRYLOV) ? APC_ERR_TIMEOUT : APC_OK;
}
