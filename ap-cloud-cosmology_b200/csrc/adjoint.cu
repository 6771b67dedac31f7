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

}  // namespace

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
  APC_CUDA_TRY(c, cudaStreamSynchronize(c->s));
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

int apc_trajectory_vjp(apc_context *c, const apc_trajectory *t, const double *const state0[6],
                       double *const cot[6], double *const statef[6]) {
  if (!c || !t || !state0 || !cot || t->n_steps < 0 || t->checkpoint_every < 1 || (t->n_steps > 0 && !t->steps))
    return APC_ERR_INVALID_ARG;
  for (int k = 0; k < 6; ++k)
    if (!state0[k] || !cot[k]) return APC_ERR_INVALID_ARG;
  cudaSetDevice(c->dev);
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
  APC_CUDA_TRY(c, cudaStreamSynchronize(c->s));
  return APC_OK;
}

}  // extern "C"
