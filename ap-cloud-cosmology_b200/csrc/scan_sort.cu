// Device-wide exclusive scan (int32) and stable LSD radix sort of (u64 key, u32 value)
// pairs for sm_100a.  Both are plain HBM-bound passes: the sort moves 12 bytes per
// element per 8-bit digit pass, the scan 8 bytes per element.
#include <cuda_runtime.h>

#include "apc_internal.cuh"

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int warp_incl_scan(int v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// exclusive scan of one tile held as kScanItems consecutive items per thread;
// returns the tile total through *total
__device__ __forceinline__ void block_scan_tile(int (&v)[kScanItems], int *total) {
  __shared__ int warp_sums[kScanThreads / 32 + 1];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int t = v[k];
    v[k] = s;
    s += t;
  }
  int incl = warp_incl_scan(s);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = lane < kScanThreads / 32 ? warp_sums[lane] : 0;
    int wi = warp_incl_scan(w);
    if (lane < kScanThreads / 32) warp_sums[lane] = wi - w;
    if (lane == kScanThreads / 32 - 1) warp_sums[kScanThreads / 32] = wi;  // total (slot 32 ok)
  }
  __syncthreads();
  int base = warp_sums[warp] + incl - s;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) v[k] += base;
  *total = warp_sums[kScanThreads / 32];
  __syncthreads();
}

__global__ void __launch_bounds__(kScanThreads) scan_tile_sums(const int *in, int n, int *sums) {
  const long long t0 = (long long)blockIdx.x * kScanTile;
  int s = 0;
  for (int k = 0; k < kScanItems; ++k) {
    long long i = t0 + (long long)threadIdx.x * kScanItems + k;
    if (i < n) s += in[i];
  }
  __shared__ int red[kScanThreads / 32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    int w = red[threadIdx.x];
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    if (threadIdx.x == 0) sums[blockIdx.x] = w;
  }
}

// single-block exclusive scan of the tile sums (loops over chunks)
__global__ void __launch_bounds__(kScanThreads) scan_sums(int *sums, int nsums, int *total) {
  int carry = 0;
  for (int c0 = 0; c0 < nsums; c0 += kScanTile) {
    int v[kScanItems];
    for (int k = 0; k < kScanItems; ++k) {
      int i = c0 + threadIdx.x * kScanItems + k;
      v[k] = i < nsums ? sums[i] : 0;
    }
    int t;
    block_scan_tile(v, &t);
    for (int k = 0; k < kScanItems; ++k) {
      int i = c0 + threadIdx.x * kScanItems + k;
      if (i < nsums) sums[i] = v[k] + carry;
    }
    carry += t;
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

// the whole scan in one block, for short arrays: chunks of a tile in order with a carry.
// Each chunk is read completely before it is written, so out may alias in.
constexpr int kScanSingleMax = 2 * kScanTile;
__global__ void __launch_bounds__(kScanThreads) scan_single(const int *in, int *out, int n, int *total) {
  int carry = 0;
  for (int c0 = 0; c0 < n; c0 += kScanTile) {
    int v[kScanItems];
    for (int k = 0; k < kScanItems; ++k) {
      const int i = c0 + threadIdx.x * kScanItems + k;
      v[k] = i < n ? in[i] : 0;
    }
    int t;
    block_scan_tile(v, &t);
    for (int k = 0; k < kScanItems; ++k) {
      const int i = c0 + threadIdx.x * kScanItems + k;
      if (i < n) out[i] = v[k] + carry;
    }
    carry += t;
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void __launch_bounds__(kScanThreads) scan_apply(const int *in, int *out, int n,
                                                          const int *sums) {
  const long long t0 = (long long)blockIdx.x * kScanTile;
  int v[kScanItems];
  for (int k = 0; k < kScanItems; ++k) {
    long long i = t0 + (long long)threadIdx.x * kScanItems + k;
    v[k] = i < n ? in[i] : 0;
  }
  int t;
  block_scan_tile(v, &t);
  const int base = sums[blockIdx.x];
  for (int k = 0; k < kScanItems; ++k) {
    long long i = t0 + (long long)threadIdx.x * kScanItems + k;
    if (i < n) out[i] = v[k] + base;
  }
}

// ---------------------------------------------------------------- radix sort

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortRows = 16;                       // rows of 32 items per warp
constexpr int kSortTile = kSortThreads * kSortRows; // 4096 items per block

__global__ void __launch_bounds__(kSortThreads) radix_hist(const uint64_t *keys, int n, int shift,
                                                           int nblocks, uint32_t *hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long long t0 = (long long)blockIdx.x * kSortTile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int r = 0; r < kSortRows; ++r) {
    long long i = t0 + (long long)warp * 32 * kSortRows + r * 32 + lane;
    bool ok = i < n;
    unsigned d = ok ? (unsigned)((keys[i] >> shift) & 0xffu) : 256u;
    unsigned peers = __match_any_sync(0xffffffffu, d);
    if (ok && lane == __ffs(peers) - 1) atomicAdd(&h[d], (uint32_t)__popc(peers));
  }
  __syncthreads();
  hist[(size_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter.  Within a tile, an item's rank among the tile's items of its digit is
// (earlier warps' counts) + (earlier rows of its warp) + (earlier lanes of its row).  The
// tile is first staged in shared memory in digit order, then written out by consecutive
// threads, so each digit's run goes to consecutive global addresses (coalesced).
struct ScatterSmem {
  uint64_t key[kSortTile];
  uint32_t val[kSortTile];
  uint32_t wcount[kSortWarps][256];
  uint32_t bstart[256];  // tile-local start of each digit
  uint32_t goff[256];    // global start of each digit's run of this tile
  uint32_t wsum[kSortWarps];
};

__global__ void __launch_bounds__(kSortThreads) radix_scatter(const uint64_t *keys_in,
                                                              const uint32_t *vals_in,
                                                              uint64_t *keys_out, uint32_t *vals_out,
                                                              int n, int shift, int nblocks,
                                                              const uint32_t *offsets) {
  extern __shared__ __align__(16) unsigned char scatter_smem[];
  ScatterSmem &S = *reinterpret_cast<ScatterSmem *>(scatter_smem);
  for (int k = threadIdx.x; k < kSortWarps * 256; k += kSortThreads) (&S.wcount[0][0])[k] = 0;
  __syncthreads();
  const long long t0 = (long long)blockIdx.x * kSortTile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  uint64_t kk[kSortRows];
  uint32_t vv[kSortRows];
  uint32_t rk[kSortRows];
#pragma unroll
  for (int r = 0; r < kSortRows; ++r) {
    long long i = t0 + (long long)warp * 32 * kSortRows + r * 32 + lane;
    bool ok = i < n;
    kk[r] = ok ? keys_in[i] : 0ull;
    vv[r] = ok ? vals_in[i] : 0u;
    unsigned d = ok ? (unsigned)((kk[r] >> shift) & 0xffu) : 256u;
    unsigned peers = __match_any_sync(0xffffffffu, d);
    unsigned prior = ok ? S.wcount[warp][d] : 0u;
    rk[r] = prior + __popc(peers & lt);
    __syncwarp();
    if (ok && lane == __ffs(peers) - 1) S.wcount[warp][d] = prior + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {
    // thread d: the tile's count of digit d and the earlier warps' counts; then the
    // tile-local digit starts by a block exclusive scan over d
    const int d = threadIdx.x;
    uint32_t run = 0;
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = S.wcount[w][d];
      S.wcount[w][d] = run;
      run += c;
    }
    uint32_t incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) S.wsum[warp] = incl;
    __syncthreads();
    uint32_t before = 0;
    for (int w = 0; w < warp; ++w) before += S.wsum[w];
    S.bstart[d] = before + incl - run;
    S.goff[d] = offsets[(size_t)d * nblocks + blockIdx.x];
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortRows; ++r) {
    long long i = t0 + (long long)warp * 32 * kSortRows + r * 32 + lane;
    if (i < n) {
      const unsigned d = (unsigned)((kk[r] >> shift) & 0xffu);
      const uint32_t lp = S.bstart[d] + S.wcount[warp][d] + rk[r];
      S.key[lp] = kk[r];
      S.val[lp] = vv[r];
    }
  }
  __syncthreads();
  const int cnt = (int)min((long long)kSortTile, (long long)n - t0);
  for (int p = threadIdx.x; p < cnt; p += kSortThreads) {
    const uint64_t k = S.key[p];
    const unsigned d = (unsigned)((k >> shift) & 0xffu);
    const uint32_t pos = S.goff[d] + ((uint32_t)p - S.bstart[d]);
    keys_out[pos] = k;
    vals_out[pos] = S.val[p];
  }
}

}  // namespace

int apc_exclusive_scan(apc_context *c, const int *in, int *out, int n, int *total_dev) {
  if (n <= 0) {
    if (total_dev) APC_CUDA_TRY(c, cudaMemsetAsync(total_dev, 0, sizeof(int), c->s));
    return APC_OK;
  }
  if (n <= kScanSingleMax) {
    scan_single<<<1, kScanThreads, 0, c->s>>>(in, out, n, total_dev);
    apc_count_launch(c);
    APC_CUDA_TRY(c, cudaGetLastError());
    return APC_OK;
  }
  int tiles = (n + kScanTile - 1) / kScanTile;
  APC_TRY(apc_ensure(c, &c->scan_tmp, (size_t)tiles + 1, nullptr));
  scan_tile_sums<<<tiles, kScanThreads, 0, c->s>>>(in, n, c->scan_tmp);
  scan_sums<<<1, kScanThreads, 0, c->s>>>(c->scan_tmp, tiles, total_dev);
  scan_apply<<<tiles, kScanThreads, 0, c->s>>>(in, out, n, c->scan_tmp);
  apc_count_launch(c, 3);
  APC_CUDA_TRY(c, cudaGetLastError());
  return APC_OK;
}

int apc_radix_sort_u64(apc_context *c, uint64_t *keys, uint32_t *vals, uint64_t *keys_alt,
                       uint32_t *vals_alt, int n, int lo_bit, int hi_bit, bool *in_alt) {
  *in_alt = false;
  if (n <= 1) return APC_OK;
  const int nblocks = (n + kSortTile - 1) / kSortTile;
  const size_t hn = (size_t)nblocks * 256;
  APC_TRY(apc_ensure(c, &c->sort_hist, hn, nullptr));
  uint64_t *ki = keys, *ko = keys_alt;
  uint32_t *vi = vals, *vo = vals_alt;
  APC_CUDA_TRY(c, cudaFuncSetAttribute(radix_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(ScatterSmem)));
  for (int shift = lo_bit; shift < hi_bit; shift += 8) {
    radix_hist<<<nblocks, kSortThreads, 0, c->s>>>(ki, n, shift, nblocks, c->sort_hist);
    APC_TRY(apc_exclusive_scan(c, (const int *)c->sort_hist, (int *)c->sort_hist, (int)hn, nullptr));
    radix_scatter<<<nblocks, kSortThreads, sizeof(ScatterSmem), c->s>>>(ki, vi, ko, vo, n, shift, nblocks,
                                                                        c->sort_hist);
    apc_count_launch(c, 2);
    APC_CUDA_TRY(c, cudaGetLastError());
    uint64_t *tk = ki; ki = ko; ko = tk;
    uint32_t *tv = vi; vi = vo; vo = tv;
    *in_alt = !*in_alt;
  }
  return APC_OK;
}
