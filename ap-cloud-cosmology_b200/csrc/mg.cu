// Multigrid-preconditioned FP32 Krylov solve of the potential system (mixed path).
//
// The reference solves the Poisson system with GMRES + Jacobi (solver.cpp:267-276).  At
// 262k cells that reaches max_it before rtol (KSP_DIVERGED_ITS), in the reference and on
// the GPU alike.  The mixed path keeps the reference's stopping test on the FP64 residual
// (krylov.cu).  Its FP32 correction solves use this preconditioner:
//   * Aggregation by the octree.  A node of the next coarser level is the parent cell
//     (location code >> 3); its aggregate is the set of its children present on the
//     finer level.  Coarse node order is sorted location code, so Morton order.
//   * Galerkin coarse operators A_c = P^T A P, P piecewise constant, one warp per
//     coarse row: the members' (J, a_ij) contributions are sorted in shared memory by a
//     bitonic network and summed in sorted order, so the hierarchy is deterministic.
//     Rows sum to zero except the Dirichlet pin's aggregate, so the constant mode is
//     reproduced exactly on every level.
//   * Damped Jacobi smoothing on ELL operators; an explicit dense inverse (FP64, formed
//     on the host) on the coarsest level of <= 128 nodes.
//   * Flexible GMRES with classical Gram-Schmidt (optionally a second, re-orthogonalising
//     sweep), right preconditioned, so the residual it monitors is the true residual of
//     the correction equation.  The SpMV is fused with the first dot-product pass.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
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

__global__ void ell_f32_dinv(int n, size_t ld, const float *__restrict__ val, float *__restrict__ dinv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float d = val[i];
    dinv[i] = d != 0.f ? 1.f / d : 1.f;
  }
}

// Galerkin row I of A_c = P^T A P, one warp per coarse row: the (J, a) contributions of
// the members' rows are gathered in shared memory, sorted by J with a bitonic network
// (data-independent, so deterministic), and equal-J runs summed in sorted order.
constexpr int kGalWarps = 2;
constexpr int kGalCap = 2048;  // contributions per coarse row

__global__ void __launch_bounds__(32 * kGalWarps) galerkin_rows(int nc, const int *__restrict__ mptr, int nf,
                                                              const int *__restrict__ mem, int wf, size_t ldf,
                                                              const int *__restrict__ colf,
                                                              const float *__restrict__ valf,
                                                              const int *__restrict__ agg, int wcap,
                                                              int *__restrict__ rowlen, int *__restrict__ tcol,
                                                              float *__restrict__ tval, int *__restrict__ err) {
  __shared__ unsigned long long buf[kGalWarps][kGalCap];  // (J << 32) | float bits
  const int lane = threadIdx.x & 31, wv = threadIdx.x >> 5;
  unsigned long long *B = buf[wv];
  for (int I = blockIdx.x * kGalWarps + wv; I < nc; I += gridDim.x * kGalWarps) {
    const int a = mptr[I], e = (I + 1 < nc) ? mptr[I + 1] : nf;
    const int cnt = (e - a) * wf;
    if (cnt > kGalCap) {
      if (lane == 0) atomicOr(err, DERR_STENCIL_MANY);
      continue;
    }
    int P = 1;
    while (P < cnt) P <<= 1;
    for (int t = lane; t < P; t += 32) {
      unsigned long long v = ~0ull;  // padding sorts last
      if (t < cnt) {
        const int i = mem[a + t / wf], sl = t % wf;
        const size_t at = (size_t)sl * ldf + i;
        const unsigned J = (unsigned)agg[colf[at]];
        v = ((unsigned long long)J << 32) | (unsigned long long)__float_as_uint(valf[at]);
      }
      B[t] = v;
    }
    __syncwarp();
    for (int k = 2; k <= P; k <<= 1) {
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int t = lane; t < P; t += 32) {
          const int u = t ^ j;
          if (u > t) {
            const unsigned long long x = B[t], y = B[u];
            const bool up = (t & k) == 0;
            // order by J only (upper 32 bits), ties by the raw word, so the network is total
            if ((x > y) == up) {
              B[t] = y;
              B[u] = x;
            }
          }
        }
        __syncwarp();
      }
    }
    // segmented sums in sorted order by lane 0 (rows are short)
    if (lane == 0) {
      int len = 0;
      int curJ = -1;
      double acc = 0.0;
      for (int t = 0; t < cnt; ++t) {
        const int J = (int)(B[t] >> 32);
        const float v = __uint_as_float((unsigned)(B[t] & 0xffffffffull));
        if (J != curJ) {
          if (curJ >= 0) {
            if (len < wcap) {
              tcol[(size_t)I * wcap + len] = curJ;
              tval[(size_t)I * wcap + len] = (float)acc;
            }
            ++len;
          }
          curJ = J;
          acc = 0.0;
        }
        acc += (double)v;
      }
      if (curJ >= 0) {
        if (len < wcap) {
          tcol[(size_t)I * wcap + len] = curJ;
          tval[(size_t)I * wcap + len] = (float)acc;
        }
        ++len;
      }
      rowlen[I] = len;
      if (len > wcap) atomicOr(err, DERR_STENCIL_MANY);
    }
    __syncwarp();
  }
}

__global__ void rows_to_ell(int n, int w, size_t ld, int wcap, const int *__restrict__ rowlen,
                            const int *__restrict__ tcol, const float *__restrict__ tval, int *__restrict__ col,
                            float *__restrict__ val, float *__restrict__ dinv) {
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < n; I += gridDim.x * blockDim.x) {
    const int len = rowlen[I];
    float d = 0.f;
    for (int s = 0; s < w; ++s) {
      const bool in = s < len;
      const int c = in ? tcol[(size_t)I * wcap + s] : I;
      const float v = in ? tval[(size_t)I * wcap + s] : 0.f;
      col[(size_t)s * ld + I] = c;
      val[(size_t)s * ld + I] = v;
      if (in && c == I) d += v;
    }
    dinv[I] = d != 0.f ? 1.f / d : 1.f;
  }
}

__global__ void max_int(int n, const int *__restrict__ a, int *out) {
  int m = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = max(m, a[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// ------------------------------------------------------------------ V-cycle

__global__ void jacobi_first(int n, const float *__restrict__ dinv, const float *__restrict__ b, float omega,
                             float *__restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = omega * dinv[i] * b[i];
}

__global__ void jacobi_sweep(int n, int w, size_t ld, const int *__restrict__ col, const float *__restrict__ val,
                             const float *__restrict__ dinv, const float *__restrict__ b,
                             const float *__restrict__ xin, float omega, float *__restrict__ xout) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int k = 0; k < w; ++k) {
      const size_t at = (size_t)k * ld + i;
      s += val[at] * xin[col[at]];
    }
    xout[i] = xin[i] + omega * dinv[i] * (b[i] - s);
  }
}

// r = b - A x, one thread per row
__global__ void residual_f32(int n, int w, size_t ld, const int *__restrict__ col, const float *__restrict__ val,
                             const float *__restrict__ b, const float *__restrict__ x, float *__restrict__ r) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int k = 0; k < w; ++k) {
      const size_t at = (size_t)k * ld + i;
      s += val[at] * x[col[at]];
    }
    r[i] = b[i] - s;
  }
}

// b_c[I] = sum of r over the members of I, in member order
__global__ void restrict_sum(int nc, const int *__restrict__ mptr, int nf, const int *__restrict__ mem,
                             const float *__restrict__ r, float *__restrict__ bc) {
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nc; I += gridDim.x * blockDim.x) {
    const int a = mptr[I], e = (I + 1 < nc) ? mptr[I + 1] : nf;
    float s = 0.f;
    for (int k = a; k < e; ++k) s += r[mem[k]];
    bc[I] = s;
  }
}

__global__ void prolong_add(int n, const int *__restrict__ agg, const float *__restrict__ xc, float alpha,
                            float *__restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] += alpha * xc[agg[i]];
}

// ------------------------------------------------------------------ FGMRES

__global__ void combine(int n, int nv, const float *__restrict__ Z, size_t vn, const double *__restrict__ y,
                        float *__restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int j = 0; j < nv; ++j) t += y[j] * (double)Z[(size_t)j * vn + i];
    x[i] = (float)t;
  }
}

// ---- fused FGMRES kernels: every reduction finishes in the last block to arrive, which
//      adds the per-block partials in a fixed order (deterministic) ----

constexpr int kRedBlocks = 296;  // grid of the reduction kernels (2 per SM)

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

// mode 0: h = V^T w.  mode 1: w -= V h_in; h = V^T w.  mode 2: w -= V h_in; h[0] = ||w||^2.
// Each warp takes tiles of 32 consecutive rows (one per lane); the basis values of a row
// stay in registers for the update and the dots; every dot is reduced across the warp at
// once and kept by lane j, so one accumulator per lane covers all basis vectors.
template <int MODE>
__global__ void __launch_bounds__(kT) cgs_pass(int n, int nv, const float *__restrict__ V, size_t vn, float *w,
                                                const double *__restrict__ h_in, double *partial, unsigned *counter,
                                                double *out) {
  __shared__ double hsh[32];
  __shared__ double sm[kT / 32][32];
  if (MODE > 0 && (int)threadIdx.x < nv) hsh[threadIdx.x] = h_in[threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double acc = 0.0;
  const int ntiles = (n + 31) / 32;
  for (int tile = blockIdx.x * nw + warp; tile < ntiles; tile += gridDim.x * nw) {
    const int i = tile * 32 + lane;
    const bool ok = i < n;
    float vj[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) vj[j] = (j < nv && ok) ? V[(size_t)j * vn + i] : 0.f;
    double wi = ok ? (double)w[i] : 0.0;
    if (MODE > 0) {
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (j < nv) wi -= hsh[j] * (double)vj[j];
      if (ok) w[i] = (float)wi;
      wi = (double)(float)wi;
    }
    if (MODE < 2) {
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        if (j < nv) {
          double p = wi * (double)vj[j];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
          if (lane == j) acc += p;
        }
      }
    } else {
      double p = wi * wi;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
      if (lane == 0) acc += p;
    }
  }
  sm[warp][lane] = acc;
  __syncthreads();
  const int nout = MODE < 2 ? nv : 1;
  if ((int)threadIdx.x < nout) {
    double v = 0.0;
    for (int k = 0; k < nw; ++k) v += sm[k][threadIdx.x];
    partial[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = v;
  }
  if (last_block_arrived(counter)) finish_sums(nout, partial, counter, out);
}

// w = A z (z kept for the solution), then the block's dots <w, V_j>, j < nv, in the same
// warp-tile pass as cgs_pass<0>
__global__ void __launch_bounds__(kT) spmv_dots(int n, int ew, size_t ld, const int *__restrict__ col,
                                                 const float *__restrict__ val, const float *__restrict__ z,
                                                 float *__restrict__ zkeep, float *__restrict__ w, int nv,
                                                 const float *__restrict__ V, size_t vn, double *partial,
                                                 unsigned *counter, double *out) {
  __shared__ double sm[kT / 32][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double acc = 0.0;
  const int ntiles = (n + 31) / 32;
  for (int tile = blockIdx.x * nw + warp; tile < ntiles; tile += gridDim.x * nw) {
    const int i = tile * 32 + lane;
    const bool ok = i < n;
    float vj[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) vj[j] = (j < nv && ok) ? V[(size_t)j * vn + i] : 0.f;
    float sacc = 0.f;
    if (ok) {
      for (int k = 0; k < ew; ++k) {
        const size_t at = (size_t)k * ld + i;
        sacc += val[at] * z[col[at]];
      }
      zkeep[i] = z[i];
      w[i] = sacc;
    }
    const double wi = (double)sacc;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      if (j < nv) {
        double p = wi * (double)vj[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
        if (lane == j) acc += p;
      }
    }
  }
  sm[warp][lane] = acc;
  __syncthreads();
  if ((int)threadIdx.x < nv) {
    double v = 0.0;
    for (int k = 0; k < nw; ++k) v += sm[k][threadIdx.x];
    partial[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = v;
  }
  if (last_block_arrived(counter)) finish_sums(nv, partial, counter, out);
}

// v_next = f w, and the same into the V-cycle's fixed input buffer
__global__ void scale2(int n, const float *__restrict__ w, float f, float *__restrict__ v, float *__restrict__ vin) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float u = w[i] * f;
    v[i] = u;
    vin[i] = u;
  }
}


// ---- the coarse end of the V-cycle in one block: every level with <= kTail nodes,
//      down (smooth, residual, restrict), the dense coarsest solve, and up (prolong,
//      smooth), separated by block barriers instead of kernel launches ----
constexpr int kTail = 512;
constexpr int kTailLevels = 12;

struct TailLevel {
  int n, w;
  size_t ld;
  const int *col;
  const float *val, *dinv;
  const int *agg;             // node -> next coarser node
  const int *mptr, *mem;      // members of this level's nodes on the finer level
  float *x, *x2, *b, *r;
};
struct TailArgs {
  int nl;                     // levels in the tail, the last one solved densely
  TailLevel L[kTailLevels];
  const float *inv;
  int sweeps;
  float omega, alpha;
};

__device__ __forceinline__ void tail_sweep(const TailLevel &L, const float *xin, float *xout, float omega) {
  for (int i = threadIdx.x; i < L.n; i += blockDim.x) {
    float sacc = 0.f;
    for (int k = 0; k < L.w; ++k) {
      const size_t at = (size_t)k * L.ld + i;
      sacc += L.val[at] * xin[L.col[at]];
    }
    xout[i] = xin[i] + omega * L.dinv[i] * (L.b[i] - sacc);
  }
  __syncthreads();
}

__global__ void __launch_bounds__(1024) vcycle_tail(TailArgs A) {
  float *cur[kTailLevels];
  for (int l = 0; l < A.nl - 1; ++l) {
    const TailLevel &L = A.L[l];
    for (int i = threadIdx.x; i < L.n; i += blockDim.x) L.x[i] = A.omega * L.dinv[i] * L.b[i];
    __syncthreads();
    float *c = L.x, *o = L.x2;
    for (int k = 1; k < A.sweeps; ++k) {
      tail_sweep(L, c, o, A.omega);
      float *t = c; c = o; o = t;
    }
    cur[l] = c;
    for (int i = threadIdx.x; i < L.n; i += blockDim.x) {
      float sacc = 0.f;
      for (int k = 0; k < L.w; ++k) {
        const size_t at = (size_t)k * L.ld + i;
        sacc += L.val[at] * c[L.col[at]];
      }
      L.r[i] = L.b[i] - sacc;
    }
    __syncthreads();
    const TailLevel &C = A.L[l + 1];
    for (int I = threadIdx.x; I < C.n; I += blockDim.x) {
      const int a = C.mptr[I], e = (I + 1 < C.n) ? C.mptr[I + 1] : L.n;
      float sacc = 0.f;
      for (int q = a; q < e; ++q) sacc += L.r[C.mem[q]];
      C.b[I] = sacc;
    }
    __syncthreads();
  }
  {
    const TailLevel &K = A.L[A.nl - 1];
    for (int i = threadIdx.x; i < K.n; i += blockDim.x) {
      float sacc = 0.f;
      for (int j = 0; j < K.n; ++j) sacc += A.inv[(size_t)i * K.n + j] * K.b[j];
      K.x[i] = sacc;
    }
    __syncthreads();
    cur[A.nl - 1] = K.x;
  }
  for (int l = A.nl - 2; l >= 0; --l) {
    const TailLevel &L = A.L[l];
    float *c = cur[l];
    float *o = (c == L.x) ? L.x2 : L.x;
    const float *xc = cur[l + 1];
    for (int i = threadIdx.x; i < L.n; i += blockDim.x) c[i] += A.alpha * xc[L.agg[i]];
    __syncthreads();
    for (int k = 0; k < A.sweeps; ++k) {
      tail_sweep(L, c, o, A.omega);
      float *t = c; c = o; o = t;
    }
    if (c != L.x) {
      for (int i = threadIdx.x; i < L.n; i += blockDim.x) L.x[i] = c[i];
      __syncthreads();
    }
    cur[l] = L.x;
  }
}

}  // namespace

struct MgLevel {
  int n = 0, w = 0;
  size_t ld = 0;
  int *col = nullptr;
  float *val = nullptr, *dinv = nullptr;
  uint64_t *code = nullptr;
  int *agg = nullptr;                   // node -> coarser node
  int *mptr = nullptr, *mem = nullptr;  // members on the finer level (levels >= 1)
  float *x = nullptr, *x2 = nullptr, *b = nullptr, *r = nullptr;
  bool owns_matrix = true;
};

struct MgWork {
  MgLevel lv[kMaxLevels];
  int nlev = 0;
  float *coarse_inv = nullptr;
  int coarse_n = 0;
  // hierarchy temporaries: parent-code sort, flags, coarse rows before the ELL transpose
  uint64_t *pkey = nullptr, *pkey_alt = nullptr;
  uint32_t *pidx = nullptr, *pidx_alt = nullptr;
  int *eflag = nullptr, *epos = nullptr, *ucol = nullptr, *rowstart = nullptr;
  float *uval = nullptr;
  // FGMRES
  float *V = nullptr, *Z = nullptr, *w = nullptr, *vin = nullptr, *vout = nullptr;
  double *partial = nullptr, *dots = nullptr;
  unsigned *counter = nullptr;
  double *host = nullptr;  // pinned readback buffer
  int *total = nullptr;
  // the V-cycle of the current hierarchy as a CUDA graph (vin -> vout)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  int64_t graph_nodes = 0;
};

static MgWork *mg(apc_context *c) {
  if (!c->mg) c->mg = new MgWork();
  return c->mg;
}

void apc_mg_free(apc_context *c) {
  MgWork *m = c->mg;
  if (!m) return;
  for (auto &L : m->lv) {
    if (L.owns_matrix) {
      cudaFree(L.col);
      cudaFree(L.val);
    }
    cudaFree(L.dinv);
    cudaFree(L.code);
    cudaFree(L.agg);
    cudaFree(L.mptr);
    cudaFree(L.mem);
    cudaFree(L.x);
    cudaFree(L.x2);
    cudaFree(L.b);
    cudaFree(L.r);
  }
  void *p[] = {m->coarse_inv, m->pkey, m->pkey_alt, m->pidx, m->pidx_alt, m->eflag, m->epos, m->ucol,
               m->rowstart, m->uval, m->V, m->Z, m->w,
               m->vin, m->vout, m->partial, m->dots, m->counter, m->total};
  for (void *q : p) cudaFree(q);
  if (m->host) cudaFreeHost(m->host);
  if (m->graph_exec) cudaGraphExecDestroy(m->graph_exec);
  if (m->graph) cudaGraphDestroy(m->graph);
  delete m;
  c->mg = nullptr;
}

static int read_int(apc_context *c, const int *dev, int *host) {
  APC_CUDA_TRY(c, cudaMemcpyAsync(host, dev, sizeof(int), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, cudaStreamSynchronize(c->s));
  return APC_OK;
}

// Build the hierarchy over the current f32 potential operator (c->a2f) and cell codes.
static int mg_build(apc_context *c) {
  MgWork *m = mg(c);
  const int n0 = c->nc + c->nv;
  MgLevel &L0 = m->lv[0];
  L0.n = n0;
  L0.w = c->ell_w;
  L0.ld = (size_t)c->m_cap;
  L0.col = c->ell_col;
  L0.val = c->a2f;
  L0.owns_matrix = false;
  APC_TRY(apc_ensure(c, &L0.dinv, (size_t)n0 + 1));
  APC_TRY(apc_ensure(c, &L0.code, (size_t)n0 + 1));
  APC_TRY(apc_ensure(c, &L0.x, (size_t)n0 + 1));
  APC_TRY(apc_ensure(c, &L0.x2, (size_t)n0 + 1));
  APC_TRY(apc_ensure(c, &L0.b, (size_t)n0 + 1));
  APC_TRY(apc_ensure(c, &L0.r, (size_t)n0 + 1));
  APC_CUDA_TRY(c, cudaMemcpyAsync(L0.code, c->ccode, sizeof(uint64_t) * n0, cudaMemcpyDeviceToDevice, c->s));
  ell_f32_dinv<<<grid_for(n0), kT, 0, c->s>>>(n0, L0.ld, L0.val, L0.dinv);
  apc_count_launch(c);
  if (!m->total) APC_TRY(apc_alloc(c, (void **)&m->total, 4 * sizeof(int)));
  int lev = 0;
  while (m->lv[lev].n > kCoarsest && lev + 1 < kMaxLevels) {
    MgLevel &F = m->lv[lev];
    MgLevel &C = m->lv[lev + 1];
    const int nf = F.n;
    // ---- aggregates: parents of this level's nodes ----
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
    if (lev == 0) APC_TRY(apc_radix_sort_u64(c, m->pkey, m->pidx, m->pkey_alt, m->pidx_alt, nf, 0, 64, &alt));
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
    APC_TRY(apc_ensure(c, &C.code, (size_t)nc + 1));
    APC_TRY(apc_ensure(c, &C.mptr, (size_t)nc + 1));
    APC_TRY(apc_ensure(c, &C.mem, (size_t)nf + 1));
    aggregate_map<<<grid_for(nf), kT, 0, c->s>>>(nf, pk, pi, m->eflag, m->epos, F.agg, C.code, C.mptr, C.mem);
    apc_count_launch(c);
    // ---- Galerkin product, one warp per coarse row ----
    const int wcap = 256;
    APC_TRY(apc_ensure(c, &m->rowstart, (size_t)nc + 1));
    APC_TRY(apc_ensure(c, &m->ucol, (size_t)nc * wcap));
    APC_TRY(apc_ensure(c, &m->uval, (size_t)nc * wcap));
    APC_CUDA_TRY(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->s));
    APC_CUDA_TRY(c, cudaMemsetAsync(m->total, 0, sizeof(int), c->s));
    galerkin_rows<<<std::max(1, std::min((nc + kGalWarps - 1) / kGalWarps, apc_sm_count(c) * 8)), 32 * kGalWarps, 0,
                    c->s>>>(nc, C.mptr, nf, C.mem, F.w, F.ld, F.col, F.val, F.agg, wcap, m->rowstart, m->ucol,
                            m->uval, c->d_err);
    max_int<<<grid_for(nc, 256), kT, 0, c->s>>>(nc, m->rowstart, m->total);
    apc_count_launch(c, 2);
    int wc = 0, derr = 0;
    APC_TRY(read_int(c, m->total, &wc));
    APC_TRY(apc_read_errors(c, &derr));
    if (derr & DERR_STENCIL_MANY) {
      c->err = "multigrid coarse row exceeds its buffers";
      return APC_ERR_UNSUPPORTED;
    }
    C.w = wc;
    C.ld = (size_t)nc;
    APC_TRY(apc_ensure(c, &C.col, C.ld * wc));
    APC_TRY(apc_ensure(c, &C.val, C.ld * wc));
    APC_TRY(apc_ensure(c, &C.dinv, (size_t)nc + 1));
    APC_TRY(apc_ensure(c, &C.x, (size_t)nc + 1));
    APC_TRY(apc_ensure(c, &C.x2, (size_t)nc + 1));
    APC_TRY(apc_ensure(c, &C.b, (size_t)nc + 1));
    APC_TRY(apc_ensure(c, &C.r, (size_t)nc + 1));
    rows_to_ell<<<grid_for(nc), kT, 0, c->s>>>(nc, wc, C.ld, wcap, m->rowstart, m->ucol, m->uval, C.col, C.val,
                                              C.dinv);
    apc_count_launch(c);
    APC_CUDA_TRY(c, cudaGetLastError());
    ++lev;
  }
  m->nlev = lev + 1;
  {
    int first_tail = 0;
    while (first_tail < m->nlev - 1 && m->lv[first_tail].n > kTail) ++first_tail;
    if (m->nlev - first_tail > kTailLevels) {
      c->err = "multigrid hierarchy deeper than the single-block tail supports";
      return APC_ERR_UNSUPPORTED;
    }
  }
  // ---- coarsest level: explicit inverse in FP64 on the host ----
  MgLevel &K = m->lv[lev];
  const int n = K.n;
  if (n > 4 * kCoarsest) {
    c->err = "multigrid coarsening stalled";
    return APC_ERR_UNSUPPORTED;
  }
  std::vector<int> col(K.ld * K.w);
  std::vector<float> val(K.ld * K.w);
  APC_CUDA_TRY(c, cudaMemcpyAsync(col.data(), K.col, sizeof(int) * col.size(), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, cudaMemcpyAsync(val.data(), K.val, sizeof(float) * val.size(), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, cudaStreamSynchronize(c->s));
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
  std::vector<float> invf(inv.begin(), inv.end());
  APC_TRY(apc_ensure(c, &m->coarse_inv, (size_t)n * n + 1));
  APC_CUDA_TRY(c, cudaMemcpyAsync(m->coarse_inv, invf.data(), sizeof(float) * invf.size(), cudaMemcpyHostToDevice,
                                  c->s));
  APC_CUDA_TRY(c, cudaStreamSynchronize(c->s));
  m->coarse_n = n;
  return APC_OK;
}

// x = V-cycle(b) on level l; b and x are that level's buffers
static void vcycle(apc_context *c, int l, const float *b, float *x) {
  MgWork *m = c->mg;
  MgLevel &L = m->lv[l];
  const int n = L.n;
  const int sweeps = c->cfg.mg_sweeps > 0 ? c->cfg.mg_sweeps : 2;
  const float omega = (float)(c->cfg.mg_omega > 0 ? c->cfg.mg_omega : 0.7);
  const float alpha = (float)(c->cfg.mg_alpha > 0 ? c->cfg.mg_alpha : 1.0);
  if (n <= kTail || l == m->nlev - 1) {
    // this level and every coarser one in a single block
    TailArgs A{};
    A.nl = std::min(m->nlev - l, kTailLevels);
    A.inv = m->coarse_inv;
    A.sweeps = sweeps;
    A.omega = omega;
    A.alpha = alpha;
    for (int k = 0; k < A.nl; ++k) {
      MgLevel &T = m->lv[l + k];
      TailLevel &D = A.L[k];
      D.n = T.n;
      D.w = T.w;
      D.ld = T.ld;
      D.col = T.col;
      D.val = T.val;
      D.dinv = T.dinv;
      D.agg = T.agg;
      D.mptr = T.mptr;
      D.mem = T.mem;
      D.x = k == 0 ? x : T.x;
      D.b = k == 0 ? const_cast<float *>(b) : T.b;
      D.x2 = T.x2;
      D.r = T.r;
    }
    vcycle_tail<<<1, 1024, 0, c->s>>>(A);
    apc_count_launch(c);
    return;
  }
  MgLevel &C = m->lv[l + 1];
  const int G = grid_for(n);
  jacobi_first<<<G, kT, 0, c->s>>>(n, L.dinv, b, omega, x);
  float *cur = x, *nxt = L.x2;
  for (int k = 1; k < sweeps; ++k) {
    jacobi_sweep<<<G, kT, 0, c->s>>>(n, L.w, L.ld, L.col, L.val, L.dinv, b, cur, omega, nxt);
    std::swap(cur, nxt);
  }
  residual_f32<<<G, kT, 0, c->s>>>(n, L.w, L.ld, L.col, L.val, b, cur, L.r);
  restrict_sum<<<grid_for(C.n), kT, 0, c->s>>>(C.n, C.mptr, n, C.mem, L.r, C.b);
  apc_count_launch(c, sweeps + 2);
  vcycle(c, l + 1, C.b, C.x);
  prolong_add<<<G, kT, 0, c->s>>>(n, L.agg, C.x, alpha, cur);
  apc_count_launch(c);
  for (int k = 0; k < sweeps; ++k) {
    jacobi_sweep<<<G, kT, 0, c->s>>>(n, L.w, L.ld, L.col, L.val, L.dinv, b, cur, omega, nxt);
    std::swap(cur, nxt);
  }
  apc_count_launch(c, sweeps);
  if (cur != x) {
    cudaMemcpyAsync(x, cur, sizeof(float) * n, cudaMemcpyDeviceToDevice, c->s);
  }
}

// Capture the V-cycle of the freshly built hierarchy (fixed buffers vin -> vout).
static int capture_vcycle(apc_context *c) {
  MgWork *m = c->mg;
  if (m->graph_exec) {
    cudaGraphExecDestroy(m->graph_exec);
    m->graph_exec = nullptr;
  }
  if (m->graph) {
    cudaGraphDestroy(m->graph);
    m->graph = nullptr;
  }
  const int64_t l0 = c->launches;
  APC_CUDA_TRY(c, cudaStreamBeginCapture(c->s, cudaStreamCaptureModeThreadLocal));
  vcycle(c, 0, m->vin, m->vout);
  cudaError_t e = cudaStreamEndCapture(c->s, &m->graph);
  m->graph_nodes = c->launches - l0;
  c->launches = l0;
  if (e != cudaSuccess) {
    c->err = std::string("V-cycle capture: ") + cudaGetErrorString(e);
    cudaGetLastError();
    return APC_ERR_CUDA;
  }
  APC_CUDA_TRY(c, cudaGraphInstantiate(&m->graph_exec, m->graph, 0));
  return APC_OK;
}

// FP32 FGMRES(m) with the V-cycle as right preconditioner: solve A d = r to rtol_in.
// r is Jacobi-scaled to unit norm by the caller.
int apc_mg_fgmres(apc_context *c, bool rebuild, const float *r, float *d, int restart, double rtol_in, int max_it,
                  int *its, int *levels) {
  MgWork *m = mg(c);
  const int n = c->nc + c->nv;
  const size_t vn = ((size_t)n + 31) & ~(size_t)31;
  const int M = std::max(1, std::min(restart, 31));
  APC_TRY(apc_ensure(c, &m->V, vn * (M + 1)));
  APC_TRY(apc_ensure(c, &m->Z, vn * M));
  APC_TRY(apc_ensure(c, &m->vin, vn));
  APC_TRY(apc_ensure(c, &m->vout, vn));
  APC_TRY(apc_ensure(c, &m->partial, (size_t)kRedBlocks * 34));
  APC_TRY(apc_ensure(c, &m->dots, (size_t)4 * 34));
  if (!m->counter) {
    APC_TRY(apc_alloc(c, (void **)&m->counter, 4 * sizeof(unsigned)));
    APC_CUDA_TRY(c, cudaMemsetAsync(m->counter, 0, 4 * sizeof(unsigned), c->s));
  }
  if (!m->host) APC_CUDA_TRY(c, cudaMallocHost((void **)&m->host, sizeof(double) * 4 * 34));
  if (rebuild || m->nlev == 0 || !m->graph_exec) {
    APC_CUDA_TRY(c, cudaStreamSynchronize(c->s));
    const auto t0 = std::chrono::steady_clock::now();
    APC_TRY(mg_build(c));
    APC_TRY(capture_vcycle(c));
    APC_CUDA_TRY(c, cudaStreamSynchronize(c->s));
    c->prof.mg_build_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  const auto ts = std::chrono::steady_clock::now();
  *levels = m->nlev;
  MgLevel &L0 = m->lv[0];
  const bool reorth = c->cfg.mg_reorth != 0;
  const int G = std::min(kRedBlocks, grid_for(n));
  const int Gs = grid_for(n, 1184);
  double *h1 = m->dots, *h2 = m->dots + 34, *nr = m->dots + 68;
  // beta = ||r||, v0 = r / beta
  cgs_pass<0><<<G, kT, 0, c->s>>>(n, 1, r, vn, const_cast<float *>(r), nullptr, m->partial, m->counter, nr);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaMemcpyAsync(m->host, nr, sizeof(double), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, cudaStreamSynchronize(c->s));
  const double beta = std::sqrt(m->host[0]);
  *its = 0;
  if (beta == 0.0) {
    APC_CUDA_TRY(c, cudaMemsetAsync(d, 0, sizeof(float) * n, c->s));
    return APC_OK;
  }
  scale2<<<Gs, kT, 0, c->s>>>(n, r, (float)(1.0 / beta), m->V, m->vin);
  apc_count_launch(c);
  std::vector<double> H((size_t)(M + 1) * M, 0.0), cs(M), sn(M), g(M + 1, 0.0);
  g[0] = beta;
  int it = 0;
  for (; it < M && it < max_it; ++it) {
    float *zk = m->Z + (size_t)it * vn, *w = m->V + (size_t)(it + 1) * vn;
    APC_CUDA_TRY(c, cudaGraphLaunch(m->graph_exec, c->s));  // vout = V-cycle(vin)
    apc_count_launch(c, (int)m->graph_nodes);
    spmv_dots<<<G, kT, 0, c->s>>>(n, L0.w, L0.ld, L0.col, L0.val, m->vout, zk, w, it + 1, m->V, vn, m->partial,
                                  m->counter, h1);
    if (reorth) {
      cgs_pass<1><<<G, kT, 0, c->s>>>(n, it + 1, m->V, vn, w, h1, m->partial, m->counter, h2);
      cgs_pass<2><<<G, kT, 0, c->s>>>(n, it + 1, m->V, vn, w, h2, m->partial, m->counter, nr);
    } else {
      cgs_pass<2><<<G, kT, 0, c->s>>>(n, it + 1, m->V, vn, w, h1, m->partial, m->counter, nr);
    }
    apc_count_launch(c, reorth ? 3 : 2);
    if (!reorth) APC_CUDA_TRY(c, cudaMemsetAsync(h2, 0, sizeof(double) * (it + 1), c->s));
    APC_CUDA_TRY(c, cudaMemcpyAsync(m->host, m->dots, sizeof(double) * 69, cudaMemcpyDeviceToHost, c->s));
    APC_CUDA_TRY(c, cudaStreamSynchronize(c->s));
    const double tt = std::sqrt(m->host[68]);
    double *hc = H.data() + (size_t)it * (M + 1);
    for (int j = 0; j <= it; ++j) hc[j] = m->host[j] + m->host[34 + j];
    hc[it + 1] = tt;
    for (int j = 1; j <= it; ++j) {
      const double t0 = hc[j - 1];
      hc[j - 1] = cs[j - 1] * t0 + sn[j - 1] * hc[j];
      hc[j] = cs[j - 1] * hc[j] - sn[j - 1] * t0;
    }
    const double t = std::sqrt(hc[it] * hc[it] + hc[it + 1] * hc[it + 1]);
    if (t == 0.0) {
      ++it;
      break;
    }
    cs[it] = hc[it] / t;
    sn[it] = hc[it + 1] / t;
    g[it + 1] = -sn[it] * g[it];
    g[it] = cs[it] * g[it];
    hc[it] = cs[it] * hc[it] + sn[it] * hc[it + 1];
    if (std::fabs(g[it + 1]) <= rtol_in * beta || tt == 0.0) {
      ++it;
      break;
    }
    scale2<<<Gs, kT, 0, c->s>>>(n, w, (float)(1.0 / tt), w, m->vin);
    apc_count_launch(c);
  }
  *its = it;
  // y = H^-1 g (upper triangular), d = Z y
  std::vector<double> y(std::max(it, 1), 0.0);
  for (int k = it - 1; k >= 0; --k) {
    double sacc = g[k];
    for (int j = k + 1; j < it; ++j) sacc -= H[(size_t)j * (M + 1) + k] * y[j];
    const double hkk = H[(size_t)k * (M + 1) + k];
    y[k] = hkk != 0.0 ? sacc / hkk : 0.0;
  }
  for (int j = 0; j < it; ++j) m->host[j] = y[j];
  APC_CUDA_TRY(c, cudaMemcpyAsync(m->dots, m->host, sizeof(double) * std::max(it, 1), cudaMemcpyHostToDevice, c->s));
  combine<<<Gs, kT, 0, c->s>>>(n, it, m->Z, vn, m->dots, d);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaStreamSynchronize(c->s));
  APC_CUDA_TRY(c, cudaGetLastError());
  c->prof.mg_solve_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ts).count();
  c->prof.mg_iterations += it;
  return APC_OK;
}
