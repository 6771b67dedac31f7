// Adjoint (vector-Jacobian product) of the Controller step sequence.
//
// The reference has no derivatives; this is the reverse mode of the forward path of
// controller.cpp:88-208 with the octree, the selected cells and their particle counts
// held fixed (piecewise constant in the particle positions).  Under that assumption:
//   * the density right-hand side n_p / h^3 (solver.cpp:116-172) does not change with the
//     positions, so the potential, its gradient and its Hessian per cell are constants
//     of each step, and the adjoint of the two solves receives no source;
//   * the only position dependence is the interpolation a = g + H (x - x_c)
//     (octree.cpp:3003-3031), whose Jacobian is the cell's Hessian H.
// One step is kick v' = v + c_vel dt a(x), drift x' = wrap(x + c_pos dt v'); its
// reverse, given the cotangents (lx, lv) of (x', v'), is
//     lv <- lv + c_pos dt lx,     lx <- lx + c_vel dt H lv      (H symmetric).
// A trajectory VJP runs the steps forward keeping the state every k steps, then for
// each segment from the last: restores the state, reruns the segment recording the
// per-particle Hessians, and applies the reverse steps backwards.  The rerun is bit-
// identical to the forward run: every per-particle and per-cell result depends only
// on the particle's position and its cell.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "apc_internal.cuh"

namespace {

// per-particle Hessian of the cell the particle was kicked in, scattered to caller order
__global__ void gather_hessians(int n, int m, const int *__restrict__ cell_of, const int *__restrict__ pid,
                                const double *__restrict__ deriv, double *__restrict__ hxx,
                                double *__restrict__ hyy, double *__restrict__ hzz, double *__restrict__ hxy,
                                double *__restrict__ hxz, double *__restrict__ hyz) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int i = cell_of[s], p = pid[s];
    if (i < 0 || i >= m || p < 0 || p >= n) continue;
    const double *d = deriv + (size_t)i * 9;
    hxx[p] = d[3];
    hyy[p] = d[4];
    hzz[p] = d[5];
    hxy[p] = d[6];
    hxz[p] = d[7];
    hyz[p] = d[8];
  }
}

__global__ void reverse_kick_drift(int n, const double *__restrict__ hxx, const double *__restrict__ hyy,
                                   const double *__restrict__ hzz, const double *__restrict__ hxy,
                                   const double *__restrict__ hxz, const double *__restrict__ hyz, double kdt,
                                   double ddt, double *__restrict__ lx, double *__restrict__ ly,
                                   double *__restrict__ lz, double *__restrict__ lvx, double *__restrict__ lvy,
                                   double *__restrict__ lvz) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const double ax = lx[p], ay = ly[p], az = lz[p];
    const double bx = lvx[p] + ddt * ax, by = lvy[p] + ddt * ay, bz = lvz[p] + ddt * az;
    lvx[p] = bx;
    lvy[p] = by;
    lvz[p] = bz;
    lx[p] = ax + kdt * (hxx[p] * bx + hxy[p] * by + hxz[p] * bz);
    ly[p] = ay + kdt * (hxy[p] * bx + hyy[p] * by + hyz[p] * bz);
    lz[p] = az + kdt * (hxz[p] * bx + hyz[p] * by + hzz[p] * bz);
  }
}

__global__ void reverse_drift(int n, double ddt, const double *__restrict__ lx, const double *__restrict__ ly,
                              const double *__restrict__ lz, double *__restrict__ lvx, double *__restrict__ lvy,
                              double *__restrict__ lvz) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    lvx[p] += ddt * lx[p];
    lvy[p] += ddt * ly[p];
    lvz[p] += ddt * lz[p];
  }
}

int grid_of(int n) { return std::max(1, std::min((n + 255) / 256, 4096)); }

// ---- transposition of a sparsity pattern ----
// Source entries (i, s), i < n, s in [s0, w): column col[s * ss + i * si].  Entries whose
// column is i itself or outside [0, n) are skipped (ELL padding and the diagonal slot).
// The transposed pattern has, per row t, the flat sources i * w + s with column t, sorted
// ascending, so every sum over it runs in a fixed order.

__global__ void tr_count(int n, int w, int s0, size_t ss, size_t si, const int *__restrict__ col,
                         int *__restrict__ cnt) {
  const long long total = (long long)n * w;
  for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < total;
       f += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(f / w), sl = (int)(f % w);
    if (sl < s0) continue;
    const int t = col[sl * ss + i * si];
    if (t >= 0 && t < n && t != i) atomicAdd(&cnt[t], 1);
  }
}

__global__ void tr_fill(int n, int w, int s0, size_t ss, size_t si, const int *__restrict__ col,
                        int *__restrict__ cur, int *__restrict__ tmp) {
  const long long total = (long long)n * w;
  for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < total;
       f += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(f / w), sl = (int)(f % w);
    if (sl < s0) continue;
    const int t = col[sl * ss + i * si];
    if (t >= 0 && t < n && t != i) tmp[atomicAdd(&cur[t], 1)] = (int)f;
  }
}

__global__ void max_count(int n, const int *__restrict__ cnt, int *out) {
  int m = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = max(m, cnt[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// sort each row's sources and write the transposed ELL (slot-major, leading dimension n):
// slot 0 = the row's own diagonal source (diag_w > 0: flat t * diag_w) or none, slots
// 1.. = the sorted sources, padding = (column t, source -1)
__global__ void tr_emit(int n, int w, int wt, int diag_w, const int *__restrict__ off, const int *__restrict__ cnt,
                        int *__restrict__ tmp, int *__restrict__ tcol, int *__restrict__ tsrc) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    int *seg = tmp + off[t];
    const int k = cnt[t];
    for (int a = 1; a < k; ++a) {  // insertion sort: rows are short
      const int v = seg[a];
      int b = a - 1;
      while (b >= 0 && seg[b] > v) {
        seg[b + 1] = seg[b];
        --b;
      }
      seg[b + 1] = v;
    }
    tcol[t] = t;
    tsrc[t] = diag_w > 0 ? t * diag_w : -1;
    for (int q = 0; q < wt - 1; ++q) {
      const size_t at = (size_t)(q + 1) * n + t;
      if (q < k) {
        tcol[at] = seg[q] / w;
        tsrc[at] = seg[q];
      } else {
        tcol[at] = t;
        tsrc[at] = -1;
      }
    }
  }
}

// values of the transposed ELL matrix: source flat i * w + s is entry (i, slot s) of the
// slot-major source with leading dimension ld
__global__ void tr_values(size_t count, int w, size_t ld, const int *__restrict__ tsrc, const double *__restrict__ val,
                          double *__restrict__ tval) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x) {
    const int f = tsrc[e];
    tval[e] = f < 0 ? 0.0 : val[(size_t)(f % w) * ld + f / w];
  }
}

// C[i, j] = c_field sum_k g[i, k] X_i[k, j] / h_i^(1 or 2): the cotangents of the
// differences (phi_nbr - phi_i) of cell i's stencil (solver.cpp:315-358 transposed)
__global__ void stencil_cot(int m, int lm, const double *__restrict__ gx, const double *__restrict__ h,
                            const double *__restrict__ g, double c_field, double *__restrict__ cmat) {
  const long long total = (long long)m * lm;
  for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < total;
       f += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(f / lm), j = (int)(f % lm);
    const double *X = gx + (size_t)i * 9 * lm;
    const double hi = h[i];
    double s = 0.0;
    for (int k = 0; k < 9; ++k) s += g[(size_t)i * 9 + k] * X[k * lm + j] / (k < 3 ? hi : hi * hi);
    cmat[f] = c_field * s;
  }
}

// phi_bar[t] = sum of C over the stencil entries naming t (sorted) - sum_j C[t, j]
__global__ void stencil_gather(int m, int lm, int wt, const int *__restrict__ tsrc, const double *__restrict__ cmat,
                               double *__restrict__ phib) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int q = 1; q < wt; ++q) {
      const int f = tsrc[(size_t)q * m + t];
      if (f >= 0) s += cmat[f];
    }
    double own = 0.0;
    for (int j = 0; j < lm; ++j) own += cmat[(size_t)t * lm + j];
    phib[t] = s - own;
  }
}

// rho_bar = c_pot (r - w sum(r) / sum(w)), w = h^3: the transpose of rhs = c_pot (rho -
// sum(rho h^3) / sum(h^3)) (solver.cpp:244-259)
__global__ void mean_transpose(int m, const double *__restrict__ h, const double *__restrict__ r, double c_pot,
                               double *__restrict__ out) {
  __shared__ double sr[256], sw[256];
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    a += r[i];
    b += h[i] * h[i] * h[i];
  }
  sr[threadIdx.x] = a;
  sw[threadIdx.x] = b;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      sr[threadIdx.x] += sr[threadIdx.x + o];
      sw[threadIdx.x] += sw[threadIdx.x + o];
    }
    __syncthreads();
  }
  const double f = sr[0] / sw[0];
  for (int i = threadIdx.x; i < m; i += blockDim.x) out[i] = c_pot * (r[i] - h[i] * h[i] * h[i] * f);
}

}  // namespace

// Transpose the pattern of (n rows, w slots from s0) into c->tr_* / (tcol, tsrc); returns
// the transposed width (1 + the largest column count).
static int transpose_pattern(apc_context *c, int n, int w, int s0, size_t ss, size_t si, const int *col, int diag_w,
                             int **tcol, int **tsrc, int *wt_out) {
  APC_TRY(apc_ensure(c, &c->tr_cnt, (size_t)n + 1, nullptr));
  APC_TRY(apc_ensure(c, &c->tr_off, (size_t)n + 1, nullptr));
  APC_TRY(apc_ensure(c, &c->tr_cur, (size_t)n + 1, nullptr));
  APC_TRY(apc_ensure(c, &c->tr_tmp, (size_t)n * w + 1, nullptr));
  APC_CUDA_TRY(c, cudaMemsetAsync(c->tr_cnt, 0, sizeof(int) * (size_t)n, c->s));
  const int G = grid_of((int)std::min<long long>((long long)n * w, 1 << 30));
  tr_count<<<G, 256, 0, c->s>>>(n, w, s0, ss, si, col, c->tr_cnt);
  APC_TRY(apc_exclusive_scan(c, c->tr_cnt, c->tr_off, n, nullptr));
  APC_CUDA_TRY(c, cudaMemcpyAsync(c->tr_cur, c->tr_off, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, c->s));
  tr_fill<<<G, 256, 0, c->s>>>(n, w, s0, ss, si, col, c->tr_cur, c->tr_tmp);
  int *mx = c->counters + 110;
  APC_CUDA_TRY(c, cudaMemsetAsync(mx, 0, sizeof(int), c->s));
  max_count<<<grid_of(n), 256, 0, c->s>>>(n, c->tr_cnt, mx);
  int h = 0;
  APC_CUDA_TRY(c, cudaMemcpyAsync(&h, mx, sizeof(int), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, apc_stream_wait(c));
  const int wt = h + 1;
  APC_TRY(apc_ensure(c, tcol, (size_t)n * wt, nullptr));
  APC_TRY(apc_ensure(c, tsrc, (size_t)n * wt, nullptr));
  tr_emit<<<grid_of(n), 256, 0, c->s>>>(n, w, wt, diag_w, c->tr_off, c->tr_cnt, c->tr_tmp, *tcol, *tsrc);
  apc_count_launch(c, 4);
  APC_CUDA_TRY(c, cudaGetLastError());
  *wt_out = wt;
  return APC_OK;
}

extern "C" {

int apc_get_hessians_device(apc_context *c, double *hxx, double *hyy, double *hzz, double *hxy, double *hxz,
                            double *hyz) {
  if (!c || !hxx || !hyy || !hzz || !hxy || !hxz || !hyz) return APC_ERR_INVALID_ARG;
  if (!c->have_fields || !c->cell_of) {
    c->err = "no kick since the last solve";
    return APC_ERR_INVALID_ARG;
  }
  cudaSetDevice(c->dev);
  const int n = c->n, m = c->nc + c->nv;
  gather_hessians<<<grid_of(n), 256, 0, c->s>>>(n, m, c->cell_of, c->pid, c->deriv, hxx, hyy, hzz, hxy, hxz, hyz);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaGetLastError());
  APC_CUDA_TRY(c, apc_stream_wait(c));
  return APC_OK;
}

int apc_vjp_kick_drift(int n, const double *const hess[6], double kdt, double ddt, double *const cot[6],
                       void *stream) {
  if (n <= 0 || !hess || !cot) return APC_ERR_INVALID_ARG;
  for (int k = 0; k < 6; ++k)
    if (!hess[k] || !cot[k]) return APC_ERR_INVALID_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  reverse_kick_drift<<<grid_of(n), 256, 0, s>>>(n, hess[0], hess[1], hess[2], hess[3], hess[4], hess[5], kdt, ddt,
                                                cot[0], cot[1], cot[2], cot[3], cot[4], cot[5]);
  if (cudaGetLastError() != cudaSuccess) return APC_ERR_CUDA;
  return cudaStreamSynchronize(s) == cudaSuccess ? APC_OK : APC_ERR_CUDA;
}

int apc_fields_from_rhs(apc_context *c, const double *rhs_dev) {
  if (!c || !rhs_dev) return APC_ERR_INVALID_ARG;
  if (!c->have_fields) {
    c->err = "no solve on the current cells";
    return APC_ERR_INVALID_ARG;
  }
  cudaSetDevice(c->dev);
  const int M = c->nc + c->nv;
  APC_CUDA_TRY(c, cudaMemcpyAsync(c->rhs, rhs_dev, sizeof(double) * M, cudaMemcpyDeviceToDevice, c->s));
  apc_solve_stats &st = c->stats;
  APC_TRY(apc_krylov_solve(c, 0, c->rhs, c->density, &st.density_its, &st.density_rnorm, &st.density_reason,
                           &st.density_refinements));
  APC_TRY(apc_potential_rhs(c, c->last_c_pot));
  APC_TRY(apc_krylov_solve(c, 1, c->rhs, c->potential, &st.potential_its, &st.potential_rnorm,
                           &st.potential_reason, &st.potential_refinements));
  APC_TRY(apc_differentiate(c, c->last_c_field));
  APC_CUDA_TRY(c, apc_stream_wait(c));
  return APC_OK;
}

int apc_solve_vjp(apc_context *c, const double *g_deriv, double *g_rhs, double *g_rho, double *g_phi) {
  if (!c || !g_deriv || !g_rhs) return APC_ERR_INVALID_ARG;
  if (!c->have_fields) {
    c->err = "no solve on the current cells";
    return APC_ERR_INVALID_ARG;
  }
  if (c->cfg.bc != 1) return APC_ERR_UNSUPPORTED;
  cudaSetDevice(c->dev);
  const int M = c->nc + c->nv, lm = c->lm, w = c->ell_w;
  const size_t ld = (size_t)c->m_cap;
  APC_TRY(apc_ensure(c, &c->vjp_c, (size_t)M * lm + 1, nullptr));
  APC_TRY(apc_ensure(c, &c->vjp_phi, (size_t)M + 1, nullptr));
  APC_TRY(apc_ensure(c, &c->vjp_r2, (size_t)M + 1, nullptr));
  APC_TRY(apc_ensure(c, &c->vjp_rho, (size_t)M + 1, nullptr));
  // 1. the transposed differentiation stencil
  int wtp = 0;
  APC_TRY(transpose_pattern(c, M, lm, 0, 1, (size_t)lm, c->st_idx, 0, &c->tp_col, &c->tp_src, &wtp));
  const int G = grid_of((int)std::min<long long>((long long)M * lm, 1 << 30));
  stencil_cot<<<G, 256, 0, c->s>>>(M, lm, c->gfd_x, c->ch, g_deriv, c->last_c_field, c->vjp_c);
  stencil_gather<<<grid_of(M), 256, 0, c->s>>>(M, lm, wtp, c->tp_src, c->vjp_c, c->vjp_phi);
  apc_count_launch(c, 2);
  // 2. A2^T r2 = phi_bar
  int wt = 0, its = 0, reason = 0;
  double rn = 0.0;
  APC_TRY(transpose_pattern(c, M, w, 1, ld, 1, c->ell_col, w, &c->ta_col, &c->ta_src, &wt));
  APC_TRY(apc_ensure(c, &c->ta_val, (size_t)M * wt, nullptr));
  tr_values<<<grid_of(M * wt), 256, 0, c->s>>>((size_t)M * wt, w, ld, c->ta_src, c->a2, c->ta_val);
  apc_count_launch(c);
  APC_TRY(apc_gmres_fp64_ell(c, M, wt, (size_t)M, c->ta_col, c->ta_val, c->vjp_phi, c->vjp_r2, &its, &rn, &reason));
  c->stats.adjoint_potential_its = its;
  c->stats.adjoint_potential_reason = reason;
  // 3. the mean subtraction, transposed
  mean_transpose<<<1, 256, 0, c->s>>>(M, c->ch, c->vjp_r2, c->last_c_pot, c->vjp_rho);
  apc_count_launch(c);
  // 4. A1^T r1 = rho_bar (same pattern as A2)
  tr_values<<<grid_of(M * wt), 256, 0, c->s>>>((size_t)M * wt, w, ld, c->ta_src, c->a1, c->ta_val);
  apc_count_launch(c);
  APC_TRY(apc_gmres_fp64_ell(c, M, wt, (size_t)M, c->ta_col, c->ta_val, c->vjp_rho, g_rhs, &its, &rn, &reason));
  c->stats.adjoint_density_its = its;
  c->stats.adjoint_density_reason = reason;
  if (g_rho)
    APC_CUDA_TRY(c, cudaMemcpyAsync(g_rho, c->vjp_rho, sizeof(double) * M, cudaMemcpyDeviceToDevice, c->s));
  if (g_phi)
    APC_CUDA_TRY(c, cudaMemcpyAsync(g_phi, c->vjp_phi, sizeof(double) * M, cudaMemcpyDeviceToDevice, c->s));
  APC_CUDA_TRY(c, cudaGetLastError());
  APC_CUDA_TRY(c, apc_stream_wait(c));
  return APC_OK;
}

int apc_trajectory_vjp(apc_context *c, const apc_trajectory *t, const double *const state0[6],
                       double *const cot[6], double *const statef[6]) {
  if (!c || !t || !state0 || !cot || t->n_steps < 0 || t->checkpoint_every < 1 || (t->n_steps > 0 && !t->steps))
    return APC_ERR_INVALID_ARG;
  for (int k = 0; k < 6; ++k)
    if (!state0[k] || !cot[k]) return APC_ERR_INVALID_ARG;
  cudaSetDevice(c->dev);
  // cold starts in both passes: a warm start would make each segment's rerun depend on
  // the solve that ran before it, and the rerun must repeat the forward run exactly
  struct WarmOff {
    apc_context *c;
    int saved;
    ~WarmOff() { c->cfg.warm_start = saved; }
  } warm_off{c, c->cfg.warm_start};
  c->cfg.warm_start = 0;
  const int n = c->n, K = t->n_steps, every = std::min(std::max(1, t->checkpoint_every), std::max(1, K));
  const int nseg = K > 0 ? (K + every - 1) / every : 0;
  const size_t nn = (size_t)n;
  // checkpoints: 6 n doubles per segment start; tape: 6 n doubles per step of a segment
  APC_TRY(apc_ensure(c, &c->adj_ckpt, 6 * nn * std::max(nseg, 1), nullptr));
  APC_TRY(apc_ensure(c, &c->adj_tape, 6 * nn * every, nullptr));
  auto slot = [&](double *base, int j, int k) { return base + ((size_t)j * 6 + k) * nn; };
  // ---- forward ----
  APC_TRY(apc_set_particles_device(c, state0[0], state0[1], state0[2], state0[3], state0[4], state0[5]));
  APC_TRY(apc_select(c, nullptr));
  APC_TRY(apc_move_position(c, t->start_dt, t->start_c_pos, nullptr));
  for (int k = 0; k < K; ++k) {
    if (k % every == 0) {
      double *ck = c->adj_ckpt;
      APC_TRY(apc_get_particles_device(c, slot(ck, k / every, 0), slot(ck, k / every, 1), slot(ck, k / every, 2),
                                       slot(ck, k / every, 3), slot(ck, k / every, 4), slot(ck, k / every, 5)));
    }
    APC_TRY(apc_step(c, &t->steps[k], nullptr, nullptr, nullptr));
  }
  if (statef) {
    for (int k = 0; k < 6; ++k)
      if (!statef[k]) return APC_ERR_INVALID_ARG;
    APC_TRY(apc_get_particles_device(c, statef[0], statef[1], statef[2], statef[3], statef[4], statef[5]));
  }
  // ---- backward ----
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int k0 = seg * every, k1 = std::min(k0 + every, K);
    double *ck = c->adj_ckpt;
    APC_TRY(apc_set_particles_device(c, slot(ck, seg, 0), slot(ck, seg, 1), slot(ck, seg, 2), slot(ck, seg, 3),
                                     slot(ck, seg, 4), slot(ck, seg, 5)));
    for (int k = k0; k < k1; ++k) {
      APC_TRY(apc_step(c, &t->steps[k], nullptr, nullptr, nullptr));
      double *tp = c->adj_tape;
      const int j = k - k0;
      APC_TRY(apc_get_hessians_device(c, slot(tp, j, 0), slot(tp, j, 1), slot(tp, j, 2), slot(tp, j, 3),
                                      slot(tp, j, 4), slot(tp, j, 5)));
    }
    for (int k = k1 - 1; k >= k0; --k) {
      const apc_step_params &p = t->steps[k];
      double *tp = c->adj_tape;
      const int j = k - k0;
      reverse_kick_drift<<<grid_of(n), 256, 0, c->s>>>(n, slot(tp, j, 0), slot(tp, j, 1), slot(tp, j, 2),
                                                       slot(tp, j, 3), slot(tp, j, 4), slot(tp, j, 5),
                                                       p.c_vel * p.dt, p.c_pos * p.dt, cot[0], cot[1], cot[2],
                                                       cot[3], cot[4], cot[5]);
      apc_count_launch(c);
    }
    APC_CUDA_TRY(c, cudaGetLastError());
  }
  // the initial half drift x_1/2 = x_0 + C_pos(start) dt/2 v_0
  reverse_drift<<<grid_of(n), 256, 0, c->s>>>(n, t->start_c_pos * t->start_dt, cot[0], cot[1], cot[2], cot[3],
                                              cot[4], cot[5]);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaGetLastError());
  APC_CUDA_TRY(c, apc_stream_wait(c));
  return APC_OK;
}

}  // extern "C"
