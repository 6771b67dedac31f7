// Interpolation + kick for callers that cannot allocate device memory.
//
// Some embedders own every byte of device memory themselves: a host framework with its
// own pooled allocator that forbids outside cudaMalloc, or a real-time loop where the
// implicit device synchronisation of cudaMalloc/cudaFree is not acceptable.  For them
// this entry point runs the same interpolation + kick as apc_move_velocity, on buffers
// the caller passes in, and takes its scratch (the particle -> cell map and the
// max-change accumulator) from a fixed array compiled into the library instead of
// allocating it.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "apc_internal.cuh"

namespace {

// Scratch shared by every call on a device: APC_NOALLOC_MAX_PARTICLES cell indices plus
// one 8-byte accumulator.  Every GPU that loads the library holds it until the process exits.
constexpr size_t kNoallocScratchBytes = sizeof(int) * (size_t)APC_NOALLOC_MAX_PARTICLES + 256;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void *g_scratch_ptr[kMaxDevices] = {nullptr};

// acc[1] error bits: a range that runs outside [0, n), ranges that overlap, a particle no
// range covers
enum : unsigned long long { kBadRange = 1, kOverlap = 2, kUncovered = 4 };

__global__ void noalloc_cell_map(int m, const int *__restrict__ first, const int *__restrict__ count, int n,
                                 int *__restrict__ cell_of, unsigned long long *acc) {
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  for (int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < m; i += gridDim.x * wpb) {
    const long long f = first[i], c = count[i];
    if (c < 0 || (c > 0 && (f < 0 || f + c > n))) {
      if (lane == 0) atomicOr(acc + 1, kBadRange);
      continue;
    }
    for (long long k = lane; k < c; k += 32)
      if (atomicCAS(cell_of + f + k, -1, i) != -1) atomicOr(acc + 1, kOverlap);
  }
}

__global__ void noalloc_coverage(int n, const int *__restrict__ cell_of, unsigned long long *acc) {
  bool hole = false;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) hole |= cell_of[s] < 0;
  if (__any_sync(0xffffffffu, hole) && (threadIdx.x & 31) == 0) atomicOr(acc + 1, kUncovered);
}

// same arithmetic, operand order and rounding as the kick of apc_move_velocity
__global__ void __launch_bounds__(256) noalloc_kick(int n, int m, const int *__restrict__ cell_of,
                                                    const double *__restrict__ deriv, const double *__restrict__ cx,
                                                    const double *__restrict__ cy, const double *__restrict__ cz,
                                                    const double *__restrict__ x, const double *__restrict__ y,
                                                    const double *__restrict__ z, double *__restrict__ vx,
                                                    double *__restrict__ vy, double *__restrict__ vz,
                                                    double *__restrict__ ax, double *__restrict__ ay,
                                                    double *__restrict__ az, double cv, double dt,
                                                    unsigned long long *acc) {
  __shared__ double sm[8];
  // malformed cell ranges (found by the two kernels before this one on the stream) leave
  // every output untouched
  if (*(volatile unsigned long long *)(acc + 1) != 0ull) return;
  double mx = 0.0;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int i = cell_of[s];
    if (i < 0 || i >= m) continue;  // unreachable once the checks above passed
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
    mx = fmax(mx, __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(sq, cv), cv), dt), dt));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b = fmax(b, sm[w]);
    atomicMax(acc, (unsigned long long)__double_as_longlong(b));
  }
}

// Device address of the scratch array for `dev`, looked up once per device with that
// device current.  In host code the array's name is only a host-side stand-in, so the
// kernels are always given this address.
int scratch_for(int dev, void **out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_scratch_ptr[dev]) {
    *out = g_scratch_ptr[dev];
    return APC_OK;
  }
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    return APC_ERR_CUDA;
  }
  g_scratch_ptr[dev] = p;
  *out = p;
  return APC_OK;
}

}  // namespace

extern "C" int apc_move_velocity_noalloc(int n_particles, int n_cells, const int *first, const int *count,
                                         const double *cx, const double *cy, const double *cz,
                                         const double *deriv9, const double *x, const double *y,
                                         const double *z, double *vx, double *vy, double *vz, double *ax,
                                         double *ay, double *az, double dt, double c_vel, double *max_dv,
                                         void *stream) {
  if (n_particles < 1 || n_cells < 1) return APC_ERR_INVALID_ARG;
  if (n_particles > APC_NOALLOC_MAX_PARTICLES) return APC_ERR_INVALID_ARG;  // beyond the scratch array
  if (!first || !count || !cx || !cy || !cz || !deriv9 || !x || !y || !z || !vx || !vy || !vz || !ax || !ay ||
      !az)
    return APC_ERR_INVALID_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return APC_ERR_CUDA;
  }
  void *base = nullptr;
  int rc = scratch_for(dev, &base);
  if (rc != APC_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  int *cell_of = (int *)base;
  unsigned long long *acc = (unsigned long long *)((unsigned char *)base + kNoallocScratchBytes - 256);
  // the array keeps the previous call's contents: reset what must start known
  if (cudaMemsetAsync(cell_of, 0xff, sizeof(int) * (size_t)n_particles, s) != cudaSuccess ||
      cudaMemsetAsync(acc, 0, 2 * sizeof(unsigned long long), s) != cudaSuccess) {
    cudaGetLastError();
    return APC_ERR_CUDA;
  }
  int sms = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int gp = std::max(1, std::min((n_particles + 255) / 256, sms * 8));
  noalloc_cell_map<<<std::max(1, std::min((n_cells + 7) / 8, sms * 16)), 256, 0, s>>>(n_cells, first, count,
                                                                                      n_particles, cell_of, acc);
  noalloc_coverage<<<gp, 256, 0, s>>>(n_particles, cell_of, acc);
  noalloc_kick<<<gp, 256, 0, s>>>(
      n_particles, n_cells, cell_of, deriv9, cx, cy, cz, x, y, z, vx, vy, vz, ax, ay, az, c_vel, dt, acc);
  if (cudaGetLastError() != cudaSuccess) return APC_ERR_CUDA;
  unsigned long long host[2] = {0, 0};
  if (cudaMemcpyAsync(host, acc, sizeof(host), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return APC_ERR_CUDA;
  }
  // cell ranges outside [0, n), overlapping, or leaving a particle uncovered: caller input,
  // so an invalid argument (the context path builds its ranges itself); nothing was written
  if (host[1]) return APC_ERR_INVALID_ARG;
  if (max_dv) {
    double v;
    std::memcpy(&v, &host[0], sizeof(v));
    *max_dv = std::sqrt(v);
  }
  return APC_OK;
}
