// K4: stable LSD radix sort of 64-bit keys with 32-bit payloads, and
// exclusive scans.  Each 8-bit pass is histogram -> scan -> scatter; the
// scatter ranks keys with warp match/ballot so the pass is stable (warp w of
// a block owns keys [w*256, w*256+256) of the block's 2048-key tile).
#include "common.cuh"

namespace phys {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
#ifndef SORT_ITEMS
#define SORT_ITEMS 8
#endif
constexpr int kItems = SORT_ITEMS;               // rounds of 32 keys per warp
constexpr int kTileKeys = kThreads * kItems;     // 2048 keys per block
constexpr int kWarpKeys = 32 * kItems;           // 256 keys per warp
constexpr int kBins = 256;

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned r;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
  return r;
}

__global__ void __launch_bounds__(kThreads)
radix_hist_kernel(const uint64_t* __restrict__ keys, int64_t n, int shift, int nblocks,
                  uint32_t* __restrict__ hist) {
  __shared__ uint32_t cnt[kWarps][kBins];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kWarps * kBins; i += kThreads) (&cnt[0][0])[i] = 0;
  __syncthreads();
  const int64_t base = blockIdx.x * (int64_t)kTileKeys + warp * kWarpKeys;
#pragma unroll 4
  for (int r = 0; r < kItems; ++r) {
    const int64_t idx = base + r * 32 + lane;
    const bool v = idx < n;
    const unsigned act = __ballot_sync(0xffffffffu, v);
    if (v) {
      const uint32_t d = (uint32_t)(keys[idx] >> shift) & 0xFFu;
      const unsigned peers = __match_any_sync(act, d);
      if (lane == __ffs(peers) - 1) cnt[warp][d] += __popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kBins; d += kThreads) {
    uint32_t s = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) s += cnt[w][d];
    hist[(size_t)d * nblocks + blockIdx.x] = s;
  }
}

// Exclusive scan of `count` u32 values in one block (in place allowed).
__global__ void __launch_bounds__(1024)
scan_single_kernel(const uint32_t* in, uint32_t* out, int64_t count, uint32_t* total) {
  __shared__ uint32_t wsum[32];
  __shared__ uint32_t carry_s;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) carry_s = 0;
  __syncthreads();
  for (int64_t base = 0; base < count; base += 4096) {
    uint32_t v[4];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      int64_t idx = base + tid * 4 + k;
      v[k] = idx < count ? in[idx] : 0u;
      s += v[k];
    }
    uint32_t inc = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = wsum[lane];
      uint32_t wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += t;
      }
      wsum[lane] = wi - w;  // exclusive warp offsets
    }
    __syncthreads();
    const uint32_t carry = carry_s;
    uint32_t run = carry + wsum[warp] + inc - s;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      int64_t idx = base + tid * 4 + k;
      if (idx < count) out[idx] = run;
      run += v[k];
    }
    __syncthreads();
    if (tid == 1023) carry_s = run;
    __syncthreads();
  }
  if (tid == 0 && total) *total = carry_s;
}

// Scatter of one 2048-key tile.  Keys are ranked per warp (match/ballot, so
// the pass is stable), then placed in shared memory in digit order and
// written out run by run: consecutive threads write consecutive addresses
// of one digit's run instead of 32 scattered places per warp.
constexpr int kScatterSmem =
    kWarps * kBins * 4 + kTileKeys * 8 + kTileKeys * 4 + 2 * kBins * 4 + 32 * 4;

template <bool kHasVals>
__global__ void __launch_bounds__(kThreads)
radix_scatter_kernel(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                     uint64_t* __restrict__ kout, uint32_t* __restrict__ vout, int64_t n,
                     int shift, int nblocks, const uint32_t* __restrict__ offs) {
  extern __shared__ __align__(16) unsigned char ssm[];
  uint64_t* skey = reinterpret_cast<uint64_t*>(ssm);                          // kTileKeys
  uint32_t* sval = reinterpret_cast<uint32_t*>(ssm + kTileKeys * 8);          // kTileKeys
  uint32_t(*cnt)[kBins] = reinterpret_cast<uint32_t(*)[kBins]>(ssm + kTileKeys * 12);
  uint32_t* local_off = reinterpret_cast<uint32_t*>(ssm + kTileKeys * 12 + kWarps * kBins * 4);
  uint32_t* gbase = local_off + kBins;
  uint32_t* wsum = gbase + kBins;  // 32 entries
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kWarps * kBins; i += kThreads) (&cnt[0][0])[i] = 0;
  __syncthreads();
  const int64_t tile0 = blockIdx.x * (int64_t)kTileKeys;
  const int64_t base = tile0 + warp * kWarpKeys;
  const unsigned lt = lanemask_lt();
  uint64_t key[kItems];
  uint32_t rank[kItems];
#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    const int64_t idx = base + r * 32 + lane;
    const bool v = idx < n;
    key[r] = v ? kin[idx] : 0ull;
    const uint32_t d = (uint32_t)(key[r] >> shift) & 0xFFu;
    const unsigned act = __ballot_sync(0xffffffffu, v);
    rank[r] = 0;
    if (v) {
      const unsigned peers = __match_any_sync(act, d);
      rank[r] = cnt[warp][d] + __popc(peers & lt);
      __syncwarp(act);
      if (lane == __ffs(peers) - 1) cnt[warp][d] += __popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  // digit d (one per thread): tile-local start of its run, and where the run
  // goes in the output
  static_assert(kThreads == kBins, "one thread per digit");
  {
    const int d = threadIdx.x;
    uint32_t tot = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) tot += cnt[w][d];
    uint32_t inc = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    uint32_t woff = 0;
    for (int w = 0; w < warp; ++w) woff += wsum[w];
    const uint32_t lo = woff + inc - tot;  // exclusive over digits
    local_off[d] = lo;
    gbase[d] = offs[(size_t)d * nblocks + blockIdx.x] - lo;
    uint32_t run = lo;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t t = cnt[w][d];
      cnt[w][d] = run;
      run += t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    const int64_t idx = base + r * 32 + lane;
    if (idx < n) {
      const uint32_t d = (uint32_t)(key[r] >> shift) & 0xFFu;
      const uint32_t lpos = cnt[warp][d] + rank[r];
      skey[lpos] = key[r];
      if (kHasVals) sval[lpos] = vin[idx];
    }
  }
  __syncthreads();
  const int tile_n = (int)min64(kTileKeys, n - tile0);
  for (int i = threadIdx.x; i < tile_n; i += kThreads) {
    const uint64_t k = skey[i];
    const uint32_t d = (uint32_t)(k >> shift) & 0xFFu;
    const uint32_t pos = gbase[d] + (uint32_t)i;
    kout[pos] = k;
    if (kHasVals) vout[pos] = sval[i];
  }
}

// Multi-block exclusive scan of int32 values: block sums, scan of the sums,
// then per-block scan with the offset.
constexpr int kScanItems = 4;
constexpr int kScanBlock = 1024;
constexpr int kScanTile = kScanItems * kScanBlock;

__device__ __forceinline__ uint32_t block_exclusive(uint32_t s, uint32_t* wsum, uint32_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) wsum[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = wsum[lane];
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    wsum[lane] = wi - w;
    if (lane == 31) wsum[32] = wi;
  }
  __syncthreads();
  total = wsum[32];
  return wsum[warp] + inc - s;
}

__global__ void __launch_bounds__(kScanBlock)
scan_block_sums_kernel(const int32_t* __restrict__ in, int64_t n, uint32_t* __restrict__ sums) {
  __shared__ uint32_t wsum[33];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t idx = blockIdx.x * (int64_t)kScanTile + threadIdx.x * kScanItems + k;
    if (idx < n) s += (uint32_t)in[idx];
  }
  uint32_t total;
  block_exclusive(s, wsum, total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanBlock)
scan_apply_kernel(const int32_t* __restrict__ in, int32_t* __restrict__ out, int64_t n,
                  const uint32_t* __restrict__ offs) {
  __shared__ uint32_t wsum[33];
  uint32_t v[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t idx = blockIdx.x * (int64_t)kScanTile + threadIdx.x * kScanItems + k;
    v[k] = idx < n ? (uint32_t)in[idx] : 0u;
    s += v[k];
  }
  uint32_t total;
  uint32_t run = offs[blockIdx.x] + block_exclusive(s, wsum, total);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t idx = blockIdx.x * (int64_t)kScanTile + threadIdx.x * kScanItems + k;
    if (idx < n) out[idx] = (int32_t)run;
    run += v[k];
  }
}

}  // namespace

int radix_sort_u64(phys_ctx* c, uint64_t* keys, uint32_t* vals, uint64_t* keys_alt,
                   uint32_t* vals_alt, int64_t n, int begin_bit, int end_bit, bool* in_alt) {
  *in_alt = false;
  if (n <= 1 || end_bit <= begin_bit) return PHYS_OK;
  static bool smem_set = false;  // per process: the kernels' attributes are fixed
  if (!smem_set) {
    PHYS_CUDA(c, cudaFuncSetAttribute(radix_scatter_kernel<true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, kScatterSmem));
    PHYS_CUDA(c, cudaFuncSetAttribute(radix_scatter_kernel<false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, kScatterSmem));
    smem_set = true;
  }
  const int nblocks = (int)ceil_div(n, kTileKeys);
  int st = PHYS_OK;
  uint32_t* hist = (uint32_t*)ws_get(c, WS_HIST, sizeof(uint32_t) * (size_t)kBins * nblocks, &st);
  if (st) return st;
  uint64_t *ki = keys, *ko = keys_alt;
  uint32_t *vi = vals, *vo = vals_alt;
  for (int shift = begin_bit; shift < end_bit; shift += 8) {
    PHYS_LAUNCH(c, radix_hist_kernel, nblocks, kThreads, 0, ki, n, shift, nblocks, hist);
    // digit-major offsets: one exclusive scan over all blocks' counts
    PHYS_TRY(scan_exclusive_i32(c, reinterpret_cast<const int32_t*>(hist),
                                reinterpret_cast<int32_t*>(hist), (int64_t)kBins * nblocks));
    if (vals) {
      PHYS_LAUNCH(c, radix_scatter_kernel<true>, nblocks, kThreads, kScatterSmem, ki, vi, ko, vo,
                  n, shift, nblocks, hist);
    } else {
      PHYS_LAUNCH(c, radix_scatter_kernel<false>, nblocks, kThreads, kScatterSmem, ki, vi, ko, vo,
                  n, shift, nblocks, hist);
    }
    uint64_t* tk = ki;
    ki = ko;
    ko = tk;
    uint32_t* tv = vi;
    vi = vo;
    vo = tv;
    *in_alt = !*in_alt;
  }
  return PHYS_OK;
}

// out[k] = sum_{j<k} in[j] for k in [0, n); out may alias in.
int scan_exclusive_i32(phys_ctx* c, const int32_t* in, int32_t* out, int64_t n) {
  if (n <= 0) return PHYS_OK;
  const int64_t nb = ceil_div(n, kScanTile);
  int st = PHYS_OK;
  uint32_t* sums = (uint32_t*)ws_get(c, WS_SCAN_TMP, sizeof(uint32_t) * (nb + 1), &st);
  if (st) return st;
  PHYS_LAUNCH(c, scan_block_sums_kernel, (int)nb, kScanBlock, 0, in, n, sums);
  PHYS_LAUNCH(c, scan_single_kernel, 1, 1024, 0, sums, sums, nb, (uint32_t*)nullptr);
  PHYS_LAUNCH(c, scan_apply_kernel, (int)nb, kScanBlock, 0, in, out, n, sums);
  return PHYS_OK;
}

}  // namespace phys
