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

constexpr int kSortMaxPasses = 8;                  // 64-bit keys, 8-bit digits
constexpr uint32_t kLookAggregate = 1u << 30;      // look-back word: the tile's own count
constexpr uint32_t kLookPrefix = 2u << 30;         // look-back word: count of every tile up to this one
constexpr uint32_t kLookValue = (1u << 30) - 1u;
constexpr long long kSortSpinLimit = 1ll << 22;

// Every pass's digit histogram over the whole array in one read of the keys: per block in
// shared memory (one atomic per distinct digit of a warp row), then added to ghist.
__global__ void __launch_bounds__(kSortThreads) radix_hist_all(const uint64_t *__restrict__ keys, int n,
                                                               int lo_bit, int npasses, uint32_t *ghist) {
  __shared__ uint32_t h[kSortMaxPasses][256];
  for (int k = threadIdx.x; k < kSortMaxPasses * 256; k += kSortThreads) (&h[0][0])[k] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long long stride = (long long)gridDim.x * kSortThreads;
  const long long rounds = (n + stride - 1) / stride;  // the same for every lane (match_any)
  for (long long rd = 0; rd < rounds; ++rd) {
    const long long i = rd * stride + (long long)blockIdx.x * kSortThreads + threadIdx.x;
    const bool ok = i < n;
    const uint64_t k = ok ? keys[i] : 0ull;
    for (int p = 0; p < npasses; ++p) {
      const unsigned d = ok ? (unsigned)((k >> (lo_bit + 8 * p)) & 0xffu) : 256u;
      const unsigned peers = __match_any_sync(0xffffffffu, d);
      if (ok && lane == __ffs(peers) - 1) atomicAdd(&h[p][d], (uint32_t)__popc(peers));
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < npasses * 256; k += kSortThreads) {
    const uint32_t v = (&h[0][0])[k];
    if (v) atomicAdd(ghist + k, v);
  }
}

// One pass, stable (one-sweep form).  Each block takes the next tile from a counter, so
// every tile before it is held by a block that is running or done.  Within the tile an
// item's rank among the tile's items of its digit is (earlier warps' counts) + (earlier
// rows of its warp) + (earlier lanes of its row).  The tile publishes its digit counts,
// then finds the counts of all earlier tiles by walking back over their published words
// (an earlier tile's inclusive prefix ends the walk), and publishes its own prefix.  Its
// items go to (items of smaller digits) + (earlier tiles' items of the digit) + rank,
// staged in shared memory in digit order so that each digit's run is written by
// consecutive threads.  A walk that waits more than kSortSpinLimit polls raises DERR_SORT.
struct ScatterSmem {
  uint64_t key[kSortTile];
  uint32_t val[kSortTile];
  uint32_t wcount[kSortWarps][256];
  uint32_t bstart[256];  // tile-local start of each digit
  uint32_t goff[256];    // global start of each digit's run of this tile
  uint32_t wsum[kSortWarps];
  int tile;
};

__global__ void __launch_bounds__(kSortThreads) radix_onesweep(const uint64_t *__restrict__ keys_in,
                                                               const uint32_t *__restrict__ vals_in,
                                                               uint64_t *__restrict__ keys_out,
                                                               uint32_t *__restrict__ vals_out, int n, int shift,
                                                               const uint32_t *__restrict__ hist, uint32_t *look,
                                                               unsigned *counter, int *err) {
  extern __shared__ __align__(16) unsigned char scatter_smem[];
  ScatterSmem &S = *reinterpret_cast<ScatterSmem *>(scatter_smem);
  for (int k = threadIdx.x; k < kSortWarps * 256; k += kSortThreads) (&S.wcount[0][0])[k] = 0;
  if (threadIdx.x == 0) S.tile = (int)atomicAdd(counter, 1u);
  __syncthreads();
  const int tile = S.tile;
  const long long t0 = (long long)tile * kSortTile;
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
    // thread d: the tile's count of digit d and the earlier warps' counts, the tile-local
    // digit starts (block scan over d), the digit's start in the output (scan of the
    // histogram over d) and the earlier tiles' count of d (look-back)
    const int d = threadIdx.x;
    uint32_t run = 0;
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = S.wcount[w][d];
      S.wcount[w][d] = run;
      run += c;
    }
    uint32_t *mine = look + (size_t)tile * 256 + d;
    atomicExch(mine, (tile == 0 ? kLookPrefix : kLookAggregate) | run);
    const uint32_t hd = hist[d];
    uint32_t incl = run, hincl = hd;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      const uint32_t th = __shfl_up_sync(0xffffffffu, hincl, o);
      if (lane >= o) {
        incl += t;
        hincl += th;
      }
    }
    if (lane == 31) S.wsum[warp] = incl;
    __shared__ uint32_t hsum[kSortWarps];
    if (lane == 31) hsum[warp] = hincl;
    uint32_t excl = 0;
    if (tile > 0) {
      int tp = tile - 1;
      long long spins = 0;
      while (true) {
        const uint32_t v = *reinterpret_cast<volatile uint32_t *>(look + (size_t)tp * 256 + d);
        if (v & (kLookAggregate | kLookPrefix)) {
          excl += v & kLookValue;
          if ((v & kLookPrefix) || tp == 0) break;
          --tp;
        } else if (++spins > kSortSpinLimit) {
          atomicOr(err, DERR_SORT);
          break;
        }
      }
      atomicExch(mine, kLookPrefix | (excl + run));
    }
    __syncthreads();
    uint32_t before = 0, hbefore = 0;
    for (int w = 0; w < warp; ++w) {
      before += S.wsum[w];
      hbefore += hsum[w];
    }
    S.bstart[d] = before + incl - run;
    S.goff[d] = hbefore + hincl - hd + excl;
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
  if (n <= 1 || hi_bit <= lo_bit) return APC_OK;
  const int npasses = std::min(kSortMaxPasses, (hi_bit - lo_bit + 7) / 8);
  const int ntiles = (n + kSortTile - 1) / kSortTile;
  // workspace: every pass's histogram (256 each), the passes' tile counters, and the
  // passes' look-back words (ntiles x 256 each), all zeroed for this sort
  const size_t nh = (size_t)kSortMaxPasses * 256, nc = 256, nl = (size_t)npasses * ntiles * 256;
  APC_TRY(apc_ensure(c, &c->sort_hist, nh + nc + nl, nullptr));
  uint32_t *ghist = c->sort_hist;
  unsigned *counters = c->sort_hist + nh;
  uint32_t *look = c->sort_hist + nh + nc;
  APC_CUDA_TRY(c, cudaMemsetAsync(c->sort_hist, 0, sizeof(uint32_t) * (nh + nc + nl), c->s));
  APC_CUDA_TRY(c, cudaFuncSetAttribute(radix_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(ScatterSmem)));
  const int hblocks = std::max(1, std::min(ntiles * 4, apc_sm_count(c) * 8));
  radix_hist_all<<<hblocks, kSortThreads, 0, c->s>>>(keys, n, lo_bit, npasses, ghist);
  apc_count_launch(c);
  uint64_t *ki = keys, *ko = keys_alt;
  uint32_t *vi = vals, *vo = vals_alt;
  for (int p = 0; p < npasses; ++p) {
    radix_onesweep<<<ntiles, kSortThreads, sizeof(ScatterSmem), c->s>>>(
        ki, vi, ko, vo, n, lo_bit + 8 * p, ghist + (size_t)p * 256, look + (size_t)p * ntiles * 256,
        counters + p, c->d_err);
    apc_count_launch(c);
    APC_CUDA_TRY(c, cudaGetLastError());
    uint64_t *tk = ki; ki = ko; ko = tk;
    uint32_t *tv = vi; vi = vo; vo = tv;
    *in_alt = !*in_alt;
  }
  return APC_OK;
}
