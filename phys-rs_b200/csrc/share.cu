// Target shares: one system's force evaluation split over GPUs that each
// hold the whole state.  Share r of w covers targets [r c, min(n, (r+1) c)),
// c = share_chunk(n, w): body indices for the direct sum, sorted (key-order)
// positions for Barnes-Hut, whose every GPU builds the same tree.  A share's
// accelerations are packed into a block of 3 c doubles (ax | ay | az, padded
// with zeros); after an all-gather of the blocks every GPU scatters all of
// them back into its acceleration arrays.  The exchange is the only data
// that crosses between GPUs (24 bytes per body per evaluation), and the
// values are the ones a single GPU computes: a target's sum does not depend
// on which share evaluated it.
#include "common.cuh"

namespace phys {
namespace {

constexpr int kBlock = 256;

int grid_for(int64_t n) {
  int64_t g = ceil_div(n, kBlock);
  if (g > 148 * 8) g = 148 * 8;
  if (g < 1) g = 1;
  return (int)g;
}

// out[k c + j] = a_k[body of target lo + j], zero past the share's end.
__global__ void share_pack_kernel(int64_t lo, int64_t hi, int64_t chunk,
                                  const uint32_t* __restrict__ perm, const double* __restrict__ ax,
                                  const double* __restrict__ ay, const double* __restrict__ az,
                                  double* __restrict__ out) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < chunk;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = lo + j;
    double a = 0.0, b = 0.0, d = 0.0;
    if (q < hi) {
      const int64_t i = perm ? (int64_t)perm[q] : q;
      a = ax[i];
      b = ay[i];
      d = az[i];
    }
    out[j] = a;
    out[chunk + j] = b;
    out[2 * chunk + j] = d;
  }
}

// a_k[body of target q] = gathered[(q / c) 3 c + k c + q % c] for all n.
__global__ void share_unpack_kernel(int64_t n, int64_t chunk, const uint32_t* __restrict__ perm,
                                    const double* __restrict__ g, double* __restrict__ ax,
                                    double* __restrict__ ay, double* __restrict__ az,
                                    int32_t* status) {
  bool bad = false;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = q / chunk, j = q - r * chunk;
    const double* blk = g + r * 3 * chunk;
    const int64_t i = perm ? (int64_t)perm[q] : q;
    const double a = blk[j], b = blk[chunk + j], d = blk[2 * chunk + j];
    ax[i] = a;
    ay[i] = b;
    az[i] = d;
    bad |= !isfinite(a) || !isfinite(b) || !isfinite(d);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status, kStatNonfinite);
}

}  // namespace

int share_pack(phys_ctx* c, int64_t lo, int64_t hi, int64_t chunk, const uint32_t* perm,
               double* out) {
  PHYS_LAUNCH(c, share_pack_kernel, grid_for(chunk), kBlock, 0, lo, hi, chunk, perm, c->ax, c->ay,
              c->az, out);
  return PHYS_OK;
}

int share_unpack(phys_ctx* c, int64_t chunk, const uint32_t* perm, const double* gathered) {
  PHYS_LAUNCH(c, share_unpack_kernel, grid_for(c->n), kBlock, 0, c->n, chunk, perm, gathered,
              c->ax, c->ay, c->az, c->d_status);
  return PHYS_OK;
}

}  // namespace phys
