// Warm start of the mixed-path solves from the previous step's solution.
//
// The cells of consecutive steps are mostly the same octree cells (location codes): at
// 128^3 98-100 % of them survive a step.  After a solve the (code -> density, potential)
// pairs are kept in an open-addressing hash table; before the next step's solves each
// cell takes the previous value of its own code, or of its nearest ancestor that was a
// cell (a cell refined since), or zero.  In the linear regime the EdS potential does not
// change in time, so the guess already carries several digits.  The stopping test is
// unchanged: the iteration ends when ||D^-1 (b - A x)|| <= max(rtol ||D^-1 b||, atol),
// as from a zero guess, so the accuracy of the result does not depend on the guess.
#include <cuda_runtime.h>

#include <algorithm>

#include "apc_internal.cuh"

namespace {

int grid_of(int n) { return std::max(1, std::min((n + 255) / 256, 4096)); }

__global__ void warm_insert(int m, const uint64_t *__restrict__ code, const double *__restrict__ rho,
                            const double *__restrict__ phi, uint64_t *keys, double *vrho, double *vphi, int cap,
                            int *err) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    bool fresh = false;
    const int h = hash_insert(keys, cap, code[i], &fresh);
    if (h < 0) {
      atomicOr(err, DERR_HASH_FULL);
      continue;
    }
    vrho[h] = rho[i];
    vphi[h] = phi[i];
  }
}

__global__ void warm_lookup(int m, const uint64_t *__restrict__ code, const uint64_t *__restrict__ keys,
                            const double *__restrict__ vals, int cap, double *__restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    uint64_t c = code[i];
    double v = 0.0;
    for (int up = 0; up < 3 && c > 1ull; ++up, c >>= 3) {
      const int h = hash_find(keys, cap, c);
      if (h >= 0) {
        v = vals[h];
        break;
      }
    }
    x[i] = v;
  }
}

}  // namespace

// keep this step's solution for the next step's guess
int apc_warm_save(apc_context *c) {
  const int m = c->nc + c->nv;
  int cap = 1024;
  while (cap < 2 * m) cap <<= 1;
  APC_TRY(apc_ensure(c, &c->warm_keys, (size_t)cap, nullptr));
  APC_TRY(apc_ensure(c, &c->warm_rho, (size_t)cap, nullptr));
  APC_TRY(apc_ensure(c, &c->warm_phi, (size_t)cap, nullptr));
  APC_CUDA_TRY(c, cudaMemsetAsync(c->warm_keys, 0, sizeof(uint64_t) * cap, c->s));
  warm_insert<<<grid_of(m), 256, 0, c->s>>>(m, c->ccode, c->density, c->potential, c->warm_keys, c->warm_rho,
                                            c->warm_phi, cap, c->d_err);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaGetLastError());
  c->warm_cap = cap;
  return APC_OK;
}

// x = the previous solution of solve `which` (0 density, 1 potential) at the current
// cells, or zeros when there is none
int apc_warm_guess(apc_context *c, int which, double *x) {
  const int m = c->nc + c->nv;
  if (c->warm_cap == 0) {
    APC_CUDA_TRY(c, cudaMemsetAsync(x, 0, sizeof(double) * m, c->s));
    return APC_OK;
  }
  warm_lookup<<<grid_of(m), 256, 0, c->s>>>(m, c->ccode, c->warm_keys, which == 0 ? c->warm_rho : c->warm_phi,
                                            c->warm_cap, x);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaGetLastError());
  return APC_OK;
}
