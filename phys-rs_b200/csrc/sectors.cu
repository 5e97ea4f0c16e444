// The reference's (Sector, LocalPosition) state kept on the device across
// Velocity-Verlet ticks (the ECS components of src/core/coordinates.rs):
// flattened positions for each force pass (gravity.rs:38-47, with the
// Barnes-Hut system's per-body origin, gravity_tree.rs:280-291), integration
// of LocalPosition (integrators.rs:63-104), and sector_boundary_system
// (src/physics/origin.rs:16-24, normalize_position, coordinates.rs:82-103)
// after every velocity step.
#include "common.cuh"

namespace phys {
namespace {

constexpr int kBlock = 256;

int grid_for(int64_t n) {
  int64_t g = ceil_div(n, kBlock);
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (int)g;
}

// abs = (sector - origin) * sector_size + local (origin: body 0's sector, or
// each body's own with bh_quirk), written to x/y/z.
__global__ void __launch_bounds__(kBlock)
flatten_from_kernel(int64_t n, const int64_t* __restrict__ sx, const int64_t* __restrict__ sy,
                    const int64_t* __restrict__ sz, const double* __restrict__ lx,
                    const double* __restrict__ ly, const double* __restrict__ lz, double ss,
                    int bh_quirk, double* __restrict__ x, double* __restrict__ y,
                    double* __restrict__ z) {
  const int64_t ox = sx[0], oy = sy[0], oz = sz[0];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t dx = bh_quirk ? 0 : (int64_t)((uint64_t)sx[i] - (uint64_t)ox);
    const int64_t dy = bh_quirk ? 0 : (int64_t)((uint64_t)sy[i] - (uint64_t)oy);
    const int64_t dz = bh_quirk ? 0 : (int64_t)((uint64_t)sz[i] - (uint64_t)oz);
    x[i] = xadd(xmul(__ll2double_rn(dx), ss), lx[i]);
    y[i] = xadd(xmul(__ll2double_rn(dy), ss), ly[i]);
    z[i] = xadd(xmul(__ll2double_rn(dz), ss), lz[i]);
  }
}

// Rust's `f as i64`: saturating, NaN -> 0.
__device__ __forceinline__ int64_t sat_i64(double v) {
  if (v != v) return 0;
  if (v >= 9223372036854775807.0) return INT64_MAX;
  if (v <= -9223372036854775808.0) return INT64_MIN;
  return (int64_t)v;
}

// normalize_position (coordinates.rs:82-103) per axis:
//   shift = round(local / sector_size); if shift != 0 { sector += shift as
//   i64; local -= shift * sector_size }   (round: half away from zero)
__device__ __forceinline__ bool norm_axis(int64_t& s, double& l, double ss) {
  const double shift = round(xdiv(l, ss));
  if (shift != 0.0) {  // NaN != 0 as well: sector += 0, local becomes NaN
    s = (int64_t)((uint64_t)s + (uint64_t)sat_i64(shift));
    l = xsub(l, xmul(shift, ss));
    return true;
  }
  return false;
}

__global__ void __launch_bounds__(kBlock)
normalize_kernel(int64_t n, int64_t* __restrict__ sx, int64_t* __restrict__ sy,
                 int64_t* __restrict__ sz, double* __restrict__ lx, double* __restrict__ ly,
                 double* __restrict__ lz, double ss, int32_t* __restrict__ shifted) {
  bool any = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t s0 = sx[i], s1 = sy[i], s2 = sz[i];
    double l0 = lx[i], l1 = ly[i], l2 = lz[i];
    const bool a = norm_axis(s0, l0, ss);
    const bool b = norm_axis(s1, l1, ss);
    const bool c = norm_axis(s2, l2, ss);
    if (a || b || c) {
      sx[i] = s0;
      sy[i] = s1;
      sz[i] = s2;
      lx[i] = l0;
      ly[i] = l1;
      lz[i] = l2;
      any = true;
    }
  }
  if (__any_sync(0xffffffffu, any) && (threadIdx.x & 31) == 0) atomicOr(shifted, 1);
}

}  // namespace

int sector_state_alloc(phys_ctx* c, int64_t n) {
  if (n <= c->sec_cap) return PHYS_OK;
  if (c->sec) {
    cudaStreamSynchronize(c->stream);
    cudaFree(c->sec);
    c->sec = nullptr;
    c->sec_cap = 0;
  }
  const int64_t cap = n < 1024 ? 1024 : n;
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, 6 * 8 * size_t(cap));
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc(sector state)");
  c->sec = static_cast<int64_t*>(p);
  c->loc = reinterpret_cast<double*>(c->sec + 3 * cap);
  c->sec_cap = cap;
  return PHYS_OK;
}

int sector_flatten(phys_ctx* c, bool bh_quirk) {
  if (c->n == 0) return PHYS_OK;
  const int64_t cap = c->sec_cap;
  PHYS_LAUNCH(c, flatten_from_kernel, grid_for(c->n), kBlock, 0, c->n, c->sec, c->sec + cap,
              c->sec + 2 * cap, c->loc, c->loc + cap, c->loc + 2 * cap, c->sector_size,
              (int)bh_quirk, c->x, c->y, c->z);
  return PHYS_OK;
}

int sector_normalize(phys_ctx* c, int32_t* shifted) {
  if (c->n == 0) return PHYS_OK;
  const int64_t cap = c->sec_cap;
  PHYS_LAUNCH(c, normalize_kernel, grid_for(c->n), kBlock, 0, c->n, c->sec, c->sec + cap,
              c->sec + 2 * cap, c->loc, c->loc + cap, c->loc + 2 * cap, c->sector_size, shifted);
  return PHYS_OK;
}

}  // namespace phys
