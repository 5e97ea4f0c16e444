// K4: stable LSD radix sort of 64-bit keys with 32-bit payloads, and
// exclusive scans.  One read of the keys counts the digits of every 8-bit
// pass; then each pass is ONE kernel over 2048-key tiles (decoupled
// look-back, after Merrill & Garland's single-pass prefix scan and the
// Onesweep radix sort of Adinets & Merrill): a tile ranks its keys with warp
// ballots (stable: warp w owns keys [w*256, w*256+256) of the tile),
// publishes its digit counts, adds up its predecessors' published counts or
// inclusive prefixes per digit, publishes its own inclusive prefix, and
// writes its keys out run by run.  Tiles are numbered in the order blocks
// start (an atomic counter), so a tile only waits for tiles whose blocks are
// already running and publish their counts without waiting themselves.
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
constexpr int kMaxPasses = 8;
// tile status word: 2-bit flag | 30-bit count
constexpr uint32_t kFlagAggregate = 1u << 30;  // the tile's own digit count
constexpr uint32_t kFlagPrefix = 2u << 30;     // count of this and every earlier tile
constexpr uint32_t kValueMask = (1u << 30) - 1u;
constexpr int kLookback = 8;                   // tiles read per look-back step

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned r;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
  return r;
}

// Lanes of `act` whose 8-bit digit equals this lane's: one ballot per bit
// (warp-collective; every lane passes a digit).
__device__ __forceinline__ unsigned match_digit(unsigned act, uint32_t d) {
  unsigned peers = act;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const unsigned m = __ballot_sync(0xffffffffu, (d >> b) & 1u);
    peers &= ((d >> b) & 1u) ? m : ~m;
  }
  return peers;
}

// Digit counts of passes [0, npass) (digit p = bits begin_bit + 8p ..) in one
// read of the keys.  Each warp counts into its own rows of shared memory
// (shared-memory atomics), the block's rows are summed and added to ghist.
constexpr int kDigitsThreads = 128;
constexpr int kDigitsSmem = (kDigitsThreads / 32) * kMaxPasses * kBins * 4;

__global__ void __launch_bounds__(kDigitsThreads)
radix_digits_kernel(const uint64_t* __restrict__ keys, int64_t n, int begin_bit, int npass,
                    uint32_t* __restrict__ ghist) {
  extern __shared__ __align__(16) unsigned char dsm[];
  uint32_t* cnt = reinterpret_cast<uint32_t*>(dsm);  // [warp][pass][digit]
  const int warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < (kDigitsThreads / 32) * kMaxPasses * kBins; i += kDigitsThreads)
    cnt[i] = 0;
  __syncthreads();
  uint32_t* mine = cnt + warp * kMaxPasses * kBins;
  const int64_t stride = (int64_t)gridDim.x * kDigitsThreads;
  for (int64_t idx = blockIdx.x * (int64_t)kDigitsThreads + threadIdx.x; idx < n; idx += stride) {
    const uint64_t k = keys[idx];
    for (int p = 0; p < npass; ++p)
      atomicAdd(&mine[p * kBins + ((uint32_t)(k >> (begin_bit + 8 * p)) & 0xFFu)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < npass * kBins; i += kDigitsThreads) {
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < kDigitsThreads / 32; ++w) c += cnt[w * kMaxPasses * kBins + i];
    if (c) atomicAdd(&ghist[i], c);
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

// One pass over one 2048-key tile.  Keys are ranked per warp (ballots,
// so the pass is stable), the tile's offsets come from the look-back, then
// the keys are placed in shared memory in digit order and written out run by
// run: consecutive threads write consecutive addresses of one digit's run
// instead of 32 scattered places per warp.
constexpr int kScatterSmem =
    kWarps * kBins * 4 + kTileKeys * 8 + kTileKeys * 4 + 2 * kBins * 4 + 64 * 4 + 16;

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
  return *reinterpret_cast<const volatile uint32_t*>(p);
}
__device__ __forceinline__ void st_volatile(uint32_t* p, uint32_t v) {
  *reinterpret_cast<volatile uint32_t*>(p) = v;
}

template <bool kHasVals>
__global__ void __launch_bounds__(kThreads)
radix_pass_kernel(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                  uint64_t* __restrict__ kout, uint32_t* __restrict__ vout, int64_t n, int shift,
                  const uint32_t* __restrict__ counts, uint32_t* __restrict__ status,
                  int32_t* __restrict__ tile_ctr, int32_t* __restrict__ err, int64_t spin_limit) {
  extern __shared__ __align__(16) unsigned char ssm[];
  uint64_t* skey = reinterpret_cast<uint64_t*>(ssm);                          // kTileKeys
  uint32_t* sval = reinterpret_cast<uint32_t*>(ssm + kTileKeys * 8);          // kTileKeys
  uint32_t(*cnt)[kBins] = reinterpret_cast<uint32_t(*)[kBins]>(ssm + kTileKeys * 12);
  uint32_t* local_off = reinterpret_cast<uint32_t*>(ssm + kTileKeys * 12 + kWarps * kBins * 4);
  uint32_t* gbase = local_off + kBins;
  uint32_t* wsum = gbase + kBins;  // 2 x 32 entries
  int* s_tile = reinterpret_cast<int*>(wsum + 64);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) *s_tile = atomicAdd(tile_ctr, 1);
  for (int i = threadIdx.x; i < kWarps * kBins; i += kThreads) (&cnt[0][0])[i] = 0;
  __syncthreads();
  const int tile = *s_tile;
  const int64_t tile0 = tile * (int64_t)kTileKeys;
  const int64_t base = tile0 + warp * kWarpKeys;
  const unsigned lt = lanemask_lt();
  uint64_t key[kItems];
  uint32_t rank[kItems], val[kItems];
  // every load of the tile first, so that they are in flight together: the
  // ranking rounds below synchronise the warp, which loads may not cross
#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    const int64_t idx = base + r * 32 + lane;
    key[r] = idx < n ? kin[idx] : 0ull;
    if (kHasVals) val[r] = idx < n ? vin[idx] : 0u;
  }
#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    const int64_t idx = base + r * 32 + lane;
    const bool v = idx < n;
    const uint32_t d = (uint32_t)(key[r] >> shift) & 0xFFu;
    const unsigned act = __ballot_sync(0xffffffffu, v);
    const unsigned peers = match_digit(act, d);
    rank[r] = 0;
    if (v) {
      rank[r] = cnt[warp][d] + __popc(peers & lt);
      __syncwarp(act);
      if (lane == __ffs(peers) - 1) cnt[warp][d] += __popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  // digit d (one per thread): the tile's count, published at once; the
  // tile-local start of its run and the pass's global start of the digit
  // (exclusive scans over digits); then the earlier tiles' count of d
  static_assert(kThreads == kBins, "one thread per digit");
  {
    const int d = threadIdx.x;
    uint32_t tot = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) tot += cnt[w][d];
    uint32_t* mine = status + (size_t)tile * kBins + d;
    st_volatile(mine, (tile == 0 ? kFlagPrefix : kFlagAggregate) | tot);
    const uint32_t gcount = counts[d];
    uint32_t inc = tot, ginc = gcount;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
      const uint32_t g = __shfl_up_sync(0xffffffffu, ginc, o);
      if (lane >= o) {
        inc += t;
        ginc += g;
      }
    }
    if (lane == 31) {
      wsum[warp] = inc;
      wsum[32 + warp] = ginc;
    }
    __syncthreads();
    uint32_t woff = 0, gwoff = 0;
    for (int w = 0; w < warp; ++w) {
      woff += wsum[w];
      gwoff += wsum[32 + w];
    }
    const uint32_t lo = woff + inc - tot;         // exclusive over digits, in the tile
    const uint32_t gstart = gwoff + ginc - gcount;  // exclusive over digits, whole pass
    uint32_t before = 0;                            // digit d in tiles [0, tile)
    if (tile > 0) {
      // walk back kLookback tiles at a time (independent loads), adding
      // counts up to the nearest inclusive prefix; wait only on a tile that
      // has not published yet (below tile 0 reads as an empty prefix).  A
      // wait gives up after spin_limit re-reads: the tile raises
      // kStatTimeout and takes the silent tile as an empty prefix, so its
      // offsets are wrong but every write below stays inside [0, n) (the
      // output is then no permutation; the kernels that index with it check
      // the flag first: sort_failed in common.cuh)
      int pred = tile - 1;
      int64_t spins = 0;
      bool done = false;
      while (!done) {
        uint32_t w[kLookback];
#pragma unroll
        for (int j = 0; j < kLookback; ++j)
          w[j] = pred - j >= 0 ? ld_volatile(status + (size_t)(pred - j) * kBins + d) : kFlagPrefix;
#pragma unroll
        for (int j = 0; j < kLookback; ++j) {
          if (done) break;
          uint32_t x = w[j];
          while ((x & ~kValueMask) == 0) {  // not published yet
            if (++spins > spin_limit) {
              atomicOr(err, kStatTimeout);
              x = kFlagPrefix;
              break;
            }
            x = ld_volatile(status + (size_t)(pred - j) * kBins + d);
          }
          before += x & kValueMask;
          done = (x & ~kValueMask) == kFlagPrefix;
        }
        pred -= kLookback;
      }
      st_volatile(mine, kFlagPrefix | ((before + tot) & kValueMask));
    }
    local_off[d] = lo;
    gbase[d] = gstart + before - lo;
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
      if (kHasVals) sval[lpos] = val[r];
    }
  }
  __syncthreads();
  const int tile_n = (int)min64(kTileKeys, n - tile0);
  for (int i = threadIdx.x; i < tile_n; i += kThreads) {
    const uint64_t k = skey[i];
    const uint32_t d = (uint32_t)(k >> shift) & 0xFFu;
    const uint32_t pos = gbase[d] + (uint32_t)i;
    if (pos < (uint64_t)n) {  // always, unless a look-back timed out
      kout[pos] = k;
      if (kHasVals) vout[pos] = sval[i];
    }
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
  if (n > (int64_t)kValueMask)
    return fail(c, PHYS_ERR_ARG, "radix sort of %lld keys: at most 2^30 - 1", (long long)n);
  if (!c->sort_smem_set) {  // once per context, on its device
    PHYS_CUDA(c, cudaFuncSetAttribute(radix_pass_kernel<true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, kScatterSmem));
    PHYS_CUDA(c, cudaFuncSetAttribute(radix_pass_kernel<false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, kScatterSmem));
    PHYS_CUDA(c, cudaFuncSetAttribute(radix_digits_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, kDigitsSmem));
    c->sort_smem_set = true;
  }
  const int npass = (end_bit - begin_bit + 7) / 8;
  if (npass > kMaxPasses) return fail(c, PHYS_ERR_ARG, "radix sort over more than 64 bits");
  const int64_t ntiles = ceil_div(n, kTileKeys);
  // [digit counts: npass x 256][tile counters: 256][tile status: npass x ntiles x 256]
  const size_t words = (size_t)npass * kBins + kBins + (size_t)npass * ntiles * kBins;
  int st = PHYS_OK;
  uint32_t* hist = (uint32_t*)ws_get(c, WS_HIST, sizeof(uint32_t) * words, &st);
  if (st) return st;
  int32_t* tile_ctr = reinterpret_cast<int32_t*>(hist + (size_t)npass * kBins);
  uint32_t* status = hist + (size_t)npass * kBins + kBins;
  PHYS_CUDA(c, cudaMemsetAsync(hist, 0, sizeof(uint32_t) * words, c->stream));
  int sms = 0;
  PHYS_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  const int dgrid = (int)std::max<int64_t>(1, std::min<int64_t>(8 * (int64_t)sms,
                                                                ceil_div(n, 8 * kDigitsThreads)));
  PHYS_LAUNCH(c, radix_digits_kernel, dgrid, kDigitsThreads, kDigitsSmem, keys, n, begin_bit,
              npass, hist);
  uint64_t *ki = keys, *ko = keys_alt;
  uint32_t *vi = vals, *vo = vals_alt;
  for (int p = 0; p < npass; ++p) {
    const int shift = begin_bit + 8 * p;
    const uint32_t* counts = hist + (size_t)p * kBins;
    uint32_t* pst = status + (size_t)p * ntiles * kBins;
    if (vals) {
      PHYS_LAUNCH(c, radix_pass_kernel<true>, (int)ntiles, kThreads, kScatterSmem, ki, vi, ko, vo,
                  n, shift, counts, pst, tile_ctr + p, c->d_status, c->sort_spin_limit);
    } else {
      PHYS_LAUNCH(c, radix_pass_kernel<false>, (int)ntiles, kThreads, kScatterSmem, ki, vi, ko,
                  vo, n, shift, counts, pst, tile_ctr + p, c->d_status, c->sort_spin_limit);
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
