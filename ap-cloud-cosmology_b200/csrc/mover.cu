// Interpolation to physical particles, kick and drift.
//
// Reference: Octree::interpolation_from_node_to_particle_2to1_3d (octree.cpp:3003-3031),
// Mover::move_velocity (mover.cpp:51-89), Mover::move_position (mover.cpp:91-121) and
// Mover::periodic_wrap (mover.cpp:123-153).
//
// Particles are stored in Morton order.  Each cell's particles are a contiguous range,
// so the interpolation is one coalesced pass: one thread per particle, the cell index
// from a particle->cell map, the 9 field values of the cell from one 72-byte row.
// Products and sums use explicit round-to-nearest operations in the reference's
// operand order.  Given the same fields and particles the results are bit-identical
// to the reference's.  The max-change reductions use atomicMax on the IEEE bit
// pattern; the values are non-negative, so this is exact and order-independent.
#include <cuda_runtime.h>

#include "apc_internal.cuh"

namespace {

__global__ void cell_of_particles(int m, const int *__restrict__ first, const int *__restrict__ count,
                                  int *__restrict__ cell_of) {
  // one warp per cell writes its particle range
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  for (int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < m; i += gridDim.x * wpb) {
    const int f = first[i], c = count[i];
    for (int k = lane; k < c; k += 32) cell_of[f + k] = i;
  }
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *addr, double v) {
  atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

__device__ __forceinline__ double block_max(double v) {
  __shared__ double sm[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  return v;
}

// a = g + H (x - x_c);  v += a c_vel dt;  max |a|^2 c_vel^2 dt^2
__global__ void __launch_bounds__(256) kick(int n, int m, const int *__restrict__ cell_of,
                                            const double *__restrict__ deriv, const double *__restrict__ cx,
                                            const double *__restrict__ cy, const double *__restrict__ cz,
                                            const double *__restrict__ x, const double *__restrict__ y,
                                            const double *__restrict__ z, double *__restrict__ vx,
                                            double *__restrict__ vy, double *__restrict__ vz,
                                            double *__restrict__ ax, double *__restrict__ ay,
                                            double *__restrict__ az, double cv, double dt,
                                            unsigned long long *maxbits, int *err) {
  double mx = 0.0;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int i = cell_of[s];
    if (i < 0 || i >= m) {  // every particle lies in exactly one cell; guard regardless
      atomicOr(err, DERR_NEIGH);
      continue;
    }
    const double *d = deriv + (size_t)i * 9;
    const double dx = __dsub_rn(x[s], cx[i]), dy = __dsub_rn(y[s], cy[i]), dz = __dsub_rn(z[s], cz[i]);
    const double a1 = __dadd_rn(__dadd_rn(__dadd_rn(d[0], __dmul_rn(dx, d[3])), __dmul_rn(dy, d[6])), __dmul_rn(dz, d[7]));
    const double a2 = __dadd_rn(__dadd_rn(__dadd_rn(d[1], __dmul_rn(dx, d[6])), __dmul_rn(dy, d[4])), __dmul_rn(dz, d[8]));
    const double a3 = __dadd_rn(__dadd_rn(__dadd_rn(d[2], __dmul_rn(dx, d[7])), __dmul_rn(dy, d[8])), __dmul_rn(dz, d[5]));
    ax[s] = a1;
    ay[s] = a2;
    az[s] = a3;
    vx[s] = __dadd_rn(vx[s], __dmul_rn(__dmul_rn(a1, cv), dt));
    vy[s] = __dadd_rn(vy[s], __dmul_rn(__dmul_rn(a2, cv), dt));
    vz[s] = __dadd_rn(vz[s], __dmul_rn(__dmul_rn(a3, cv), dt));
    const double sq = __dadd_rn(__dadd_rn(__dmul_rn(a1, a1), __dmul_rn(a2, a2)), __dmul_rn(a3, a3));
    const double ch = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(sq, cv), cv), dt), dt);
    mx = fmax(mx, ch);
  }
  mx = block_max(mx);
  if (threadIdx.x == 0) atomic_max_nonneg(maxbits, mx);
}

__device__ __forceinline__ double mwrap(double v, double lo, double hi, int bc) {
  if (bc == 1) {
    const double len = __dsub_rn(hi, lo);
    for (int k = 0; k < 64 && v >= hi; ++k) v = __dsub_rn(v, len);
    for (int k = 0; k < 64 && v < lo; ++k) v = __dadd_rn(v, len);
  }
  return v;
}

// x = wrap(x + v c_pos dt);  max |v|^2 c_pos^2 dt^2
__global__ void __launch_bounds__(256) drift(int n, double *__restrict__ x, double *__restrict__ y,
                                             double *__restrict__ z, const double *__restrict__ vx,
                                             const double *__restrict__ vy, const double *__restrict__ vz,
                                             double cp, double dt, double x0, double x1, double y0, double y1,
                                             double z0, double z1, int bc, unsigned long long *maxbits) {
  double mx = 0.0;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const double u = vx[s], v = vy[s], w = vz[s];
    x[s] = mwrap(__dadd_rn(x[s], __dmul_rn(__dmul_rn(u, cp), dt)), x0, x1, bc);
    y[s] = mwrap(__dadd_rn(y[s], __dmul_rn(__dmul_rn(v, cp), dt)), y0, y1, bc);
    z[s] = mwrap(__dadd_rn(z[s], __dmul_rn(__dmul_rn(w, cp), dt)), z0, z1, bc);
    const double sq = __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w));
    const double ch = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(sq, cp), cp), dt), dt);
    mx = fmax(mx, ch);
  }
  mx = block_max(mx);
  if (threadIdx.x == 0) atomic_max_nonneg(maxbits, mx);
}

// Kick then drift in one pass (apc_step): the same operations as `kick` followed by
// `drift`, so the results are bit-identical, with x and v read once and written once.
__global__ void __launch_bounds__(256) kick_drift(int n, int m, const int *__restrict__ cell_of,
                                                  const double *__restrict__ deriv, const double *__restrict__ cx,
                                                  const double *__restrict__ cy, const double *__restrict__ cz,
                                                  double *__restrict__ x, double *__restrict__ y,
                                                  double *__restrict__ z, double *__restrict__ vx,
                                                  double *__restrict__ vy, double *__restrict__ vz,
                                                  double *__restrict__ ax, double *__restrict__ ay,
                                                  double *__restrict__ az, double cv, double cp, double dt,
                                                  double x0, double x1, double y0, double y1, double z0, double z1,
                                                  int bc, unsigned long long *maxbits_v,
                                                  unsigned long long *maxbits_x, int *err) {
  double mv = 0.0, mxx = 0.0;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int i = cell_of[s];
    if (i < 0 || i >= m) {
      atomicOr(err, DERR_NEIGH);
      continue;
    }
    const double *d = deriv + (size_t)i * 9;
    const double px = x[s], py = y[s], pz = z[s];
    const double dx = __dsub_rn(px, cx[i]), dy = __dsub_rn(py, cy[i]), dz = __dsub_rn(pz, cz[i]);
    const double a1 = __dadd_rn(__dadd_rn(__dadd_rn(d[0], __dmul_rn(dx, d[3])), __dmul_rn(dy, d[6])), __dmul_rn(dz, d[7]));
    const double a2 = __dadd_rn(__dadd_rn(__dadd_rn(d[1], __dmul_rn(dx, d[6])), __dmul_rn(dy, d[4])), __dmul_rn(dz, d[8]));
    const double a3 = __dadd_rn(__dadd_rn(__dadd_rn(d[2], __dmul_rn(dx, d[7])), __dmul_rn(dy, d[8])), __dmul_rn(dz, d[5]));
    ax[s] = a1;
    ay[s] = a2;
    az[s] = a3;
    const double u = __dadd_rn(vx[s], __dmul_rn(__dmul_rn(a1, cv), dt));
    const double v = __dadd_rn(vy[s], __dmul_rn(__dmul_rn(a2, cv), dt));
    const double w = __dadd_rn(vz[s], __dmul_rn(__dmul_rn(a3, cv), dt));
    vx[s] = u;
    vy[s] = v;
    vz[s] = w;
    const double sa = __dadd_rn(__dadd_rn(__dmul_rn(a1, a1), __dmul_rn(a2, a2)), __dmul_rn(a3, a3));
    mv = fmax(mv, __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(sa, cv), cv), dt), dt));
    x[s] = mwrap(__dadd_rn(px, __dmul_rn(__dmul_rn(u, cp), dt)), x0, x1, bc);
    y[s] = mwrap(__dadd_rn(py, __dmul_rn(__dmul_rn(v, cp), dt)), y0, y1, bc);
    z[s] = mwrap(__dadd_rn(pz, __dmul_rn(__dmul_rn(w, cp), dt)), z0, z1, bc);
    const double sv = __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w));
    mxx = fmax(mxx, __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(sv, cp), cp), dt), dt));
  }
  mv = block_max(mv);
  __syncthreads();  // block_max's shared scratch is reused below
  mxx = block_max(mxx);
  if (threadIdx.x == 0) {
    atomic_max_nonneg(maxbits_v, mv);
    atomic_max_nonneg(maxbits_x, mxx);
  }
}

// max over the cells of n_p / h / h / h, in the reference's operation order
// (controller.cpp:150-156); values are non-negative, so atomicMax on the bits is exact
__global__ void max_cell_density(int m, const int *__restrict__ count, const double *__restrict__ h,
                                 unsigned long long *maxbits) {
  double mx = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const double hi = h[i];
    mx = fmax(mx, __ddiv_rn(__ddiv_rn(__ddiv_rn((double)count[i], hi), hi), hi));
  }
  mx = block_max(mx);
  if (threadIdx.x == 0) atomic_max_nonneg(maxbits, mx);
}

}  // namespace

int apc_mover_max_density(apc_context *c, double *out) {
  const int m = c->nc + c->nv + c->nb;
  unsigned long long *mb = (unsigned long long *)(c->counters + 104);
  APC_CUDA_TRY(c, cudaMemsetAsync(mb, 0, sizeof(unsigned long long), c->s));
  const int G = std::max(1, std::min((m + 255) / 256, apc_sm_count(c) * 8));
  max_cell_density<<<G, 256, 0, c->s>>>(m, c->ccount, c->ch, mb);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaGetLastError());
  unsigned long long *hb = (unsigned long long *)(c->h_pinned + 12);  // pinned, 8-byte aligned
  APC_CUDA_TRY(c, cudaMemcpyAsync(hb, mb, sizeof(*hb), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, apc_stream_wait(c));
  memcpy(out, hb, sizeof(double));
  return APC_OK;
}

int apc_mover_velocity(apc_context *c, double dt, double c_vel, double *max_dv) {
  const int n = c->n, M = c->nc + c->nv;
  APC_TRY(apc_velocities_sorted(c));
  APC_TRY(apc_ensure(c, &c->cell_of, (size_t)n + 1, nullptr));
  APC_CUDA_TRY(c, cudaMemsetAsync(c->cell_of, 0xff, sizeof(int) * (size_t)n, c->s));
  APC_CUDA_TRY(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->s));
  const int sms = apc_sm_count(c);
  cell_of_particles<<<std::max(1, std::min((M + 7) / 8, sms * 16)), 256, 0, c->s>>>(M, c->cfirst, c->ccount,
                                                                                   c->cell_of);
  unsigned long long *mb = (unsigned long long *)(c->counters + 96);
  APC_CUDA_TRY(c, cudaMemsetAsync(mb, 0, sizeof(unsigned long long), c->s));
  const int G = std::max(1, std::min((n + 255) / 256, sms * 8));
  kick<<<G, 256, 0, c->s>>>(n, M, c->cell_of, c->deriv, c->cx, c->cy, c->cz, c->px, c->py, c->pz, c->pvx,
                            c->pvy, c->pvz, c->pax, c->pay, c->paz, c_vel, dt, mb, c->d_err);
  apc_count_launch(c, 2);
  APC_CUDA_TRY(c, cudaGetLastError());
  int derr = 0;
  APC_TRY(apc_read_errors(c, &derr));
  if (derr & DERR_NEIGH) {
    c->err = "a particle lies in no selected cell";
    return APC_ERR_CUDA;
  }
  if (max_dv) {
    unsigned long long *hb = (unsigned long long *)(c->h_pinned + 12);  // pinned, 8-byte aligned
    APC_CUDA_TRY(c, cudaMemcpyAsync(hb, mb, sizeof(*hb), cudaMemcpyDeviceToHost, c->s));
    APC_CUDA_TRY(c, apc_stream_wait(c));
    double v;
    memcpy(&v, hb, sizeof(v));
    *max_dv = std::sqrt(v);
  }
  return APC_OK;
}

int apc_mover_position(apc_context *c, double dt, double c_pos, double *max_dx) {
  const int n = c->n;
  APC_TRY(apc_velocities_sorted(c));
  unsigned long long *mb = (unsigned long long *)(c->counters + 100);
  APC_CUDA_TRY(c, cudaMemsetAsync(mb, 0, sizeof(unsigned long long), c->s));
  const int G = std::max(1, std::min((n + 255) / 256, apc_sm_count(c) * 8));
  const double *b = c->cfg.box;
  drift<<<G, 256, 0, c->s>>>(n, c->px, c->py, c->pz, c->pvx, c->pvy, c->pvz, c_pos, dt, b[0], b[1], b[2], b[3],
                             b[4], b[5], c->cfg.bc, mb);
  apc_count_launch(c);
  APC_CUDA_TRY(c, cudaGetLastError());
  if (max_dx) {
    unsigned long long *hb = (unsigned long long *)(c->h_pinned + 12);  // pinned, 8-byte aligned
    APC_CUDA_TRY(c, cudaMemcpyAsync(hb, mb, sizeof(*hb), cudaMemcpyDeviceToHost, c->s));
    APC_CUDA_TRY(c, apc_stream_wait(c));
    double v;
    memcpy(&v, hb, sizeof(v));
    *max_dx = std::sqrt(v);
  }
  return APC_OK;
}

// Interpolation + kick + drift in one pass (apc_step); one readback for both maxima and
// the error flag.
int apc_mover_kick_drift(apc_context *c, double dt, double c_vel, double c_pos, double *max_dv, double *max_dx) {
  const int n = c->n, M = c->nc + c->nv;
  APC_TRY(apc_velocities_sorted(c));
  APC_TRY(apc_ensure(c, &c->cell_of, (size_t)n + 1, nullptr));
  APC_CUDA_TRY(c, cudaMemsetAsync(c->cell_of, 0xff, sizeof(int) * (size_t)n, c->s));
  APC_CUDA_TRY(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->s));
  const int sms = apc_sm_count(c);
  cell_of_particles<<<std::max(1, std::min((M + 7) / 8, sms * 16)), 256, 0, c->s>>>(M, c->cfirst, c->ccount,
                                                                                   c->cell_of);
  // counters + 96 .. + 99: the two maxima (8 bytes each)
  unsigned long long *mb = (unsigned long long *)(c->counters + 96);
  APC_CUDA_TRY(c, cudaMemsetAsync(mb, 0, 2 * sizeof(unsigned long long), c->s));
  const int G = std::max(1, std::min((n + 255) / 256, sms * 8));
  const double *b = c->cfg.box;
  kick_drift<<<G, 256, 0, c->s>>>(n, M, c->cell_of, c->deriv, c->cx, c->cy, c->cz, c->px, c->py, c->pz, c->pvx,
                                  c->pvy, c->pvz, c->pax, c->pay, c->paz, c_vel, c_pos, dt, b[0], b[1], b[2], b[3],
                                  b[4], b[5], c->cfg.bc, mb, mb + 1, c->d_err);
  apc_count_launch(c, 2);
  APC_CUDA_TRY(c, cudaGetLastError());
  unsigned long long *hb = (unsigned long long *)(c->h_pinned + 12);  // pinned, 8-byte aligned: 2 maxima
  APC_CUDA_TRY(c, cudaMemcpyAsync(hb, mb, 2 * sizeof(*hb), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, cudaMemcpyAsync(c->h_pinned + 16, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->s));
  APC_CUDA_TRY(c, apc_stream_wait(c));
  if (c->h_pinned[16] & DERR_NEIGH) {
    c->err = "a particle lies in no selected cell";
    return APC_ERR_CUDA;
  }
  double v[2];
  memcpy(v, hb, sizeof(v));
  if (max_dv) *max_dv = std::sqrt(v[0]);
  if (max_dx) *max_dx = std::sqrt(v[1]);
  return APC_OK;
}
