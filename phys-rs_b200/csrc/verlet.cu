// Velocity-Verlet kick/drift kernels and the sector flattening kernel.
// All arithmetic uses non-contracting IEEE intrinsics so every update is
// bit-identical to the reference's Rust f64 code.
#include "common.cuh"

namespace phys {
namespace {

constexpr int kBlock = 256;

// velocity_verlet_position_system (integrators.rs:63-83):
//   prev = a;  x += v*dt + a*(0.5*dt*dt)
__global__ void drift_kernel(int64_t n, double dt, double* __restrict__ x, double* __restrict__ y,
                             double* __restrict__ z, const double* __restrict__ vx,
                             const double* __restrict__ vy, const double* __restrict__ vz,
                             const double* __restrict__ ax, const double* __restrict__ ay,
                             const double* __restrict__ az, double* __restrict__ pax,
                             double* __restrict__ pay, double* __restrict__ paz) {
  const double h2 = xmul(xmul(0.5, dt), dt);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double a0 = ax[i], a1 = ay[i], a2 = az[i];
    pax[i] = a0;
    pay[i] = a1;
    paz[i] = a2;
    x[i] = xadd(x[i], xadd(xmul(vx[i], dt), xmul(a0, h2)));
    y[i] = xadd(y[i], xadd(xmul(vy[i], dt), xmul(a1, h2)));
    z[i] = xadd(z[i], xadd(xmul(vz[i], dt), xmul(a2, h2)));
  }
}

// velocity_verlet_velocity_system (integrators.rs:92-104):
//   v += (prev + a) * (0.5*dt)
__global__ void kick_kernel(int64_t n, double dt, double* __restrict__ vx, double* __restrict__ vy,
                            double* __restrict__ vz, const double* __restrict__ ax,
                            const double* __restrict__ ay, const double* __restrict__ az,
                            const double* __restrict__ pax, const double* __restrict__ pay,
                            const double* __restrict__ paz, int32_t* status) {
  const double hdt = xmul(0.5, dt);
  bool bad = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double v0 = xadd(vx[i], xmul(xadd(pax[i], ax[i]), hdt));
    double v1 = xadd(vy[i], xmul(xadd(pay[i], ay[i]), hdt));
    double v2 = xadd(vz[i], xmul(xadd(paz[i], az[i]), hdt));
    vx[i] = v0;
    vy[i] = v1;
    vz[i] = v2;
    bad |= !isfinite(v0) || !isfinite(v1) || !isfinite(v2);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status, kStatNonfinite);
}

// Velocity step of tick s fused with the position step of tick s+1.  The
// reference's first force pass of tick s+1 recomputes a(x_{s+1}), which the
// second pass of tick s already produced bit-for-bit, so a is reused.
__global__ void kick_drift_kernel(int64_t n, double dt, double* __restrict__ x,
                                  double* __restrict__ y, double* __restrict__ z,
                                  double* __restrict__ vx, double* __restrict__ vy,
                                  double* __restrict__ vz, const double* __restrict__ ax,
                                  const double* __restrict__ ay, const double* __restrict__ az,
                                  double* __restrict__ pax, double* __restrict__ pay,
                                  double* __restrict__ paz, int32_t* status) {
  const double hdt = xmul(0.5, dt);
  const double h2 = xmul(xmul(0.5, dt), dt);
  bool bad = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double a0 = ax[i], a1 = ay[i], a2 = az[i];
    double v0 = xadd(vx[i], xmul(xadd(pax[i], a0), hdt));
    double v1 = xadd(vy[i], xmul(xadd(pay[i], a1), hdt));
    double v2 = xadd(vz[i], xmul(xadd(paz[i], a2), hdt));
    vx[i] = v0;
    vy[i] = v1;
    vz[i] = v2;
    pax[i] = a0;
    pay[i] = a1;
    paz[i] = a2;
    double p0 = xadd(x[i], xadd(xmul(v0, dt), xmul(a0, h2)));
    double p1 = xadd(y[i], xadd(xmul(v1, dt), xmul(a1, h2)));
    double p2 = xadd(z[i], xadd(xmul(v2, dt), xmul(a2, h2)));
    x[i] = p0;
    y[i] = p1;
    z[i] = p2;
    bad |= !isfinite(v0) || !isfinite(v1) || !isfinite(v2) || !isfinite(p0) || !isfinite(p1) ||
           !isfinite(p2);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status, kStatNonfinite);
}

// gravity.rs:38-47: abs = (sector - origin) * sector_size + local, origin =
// sector of body 0; with bh_quirk each body is its own origin
// (gravity_tree.rs:280-291).  In place over the local positions.
__global__ void flatten_kernel(int64_t n, const int64_t* __restrict__ sx,
                               const int64_t* __restrict__ sy, const int64_t* __restrict__ sz,
                               double* __restrict__ x, double* __restrict__ y,
                               double* __restrict__ z, double ss, int bh_quirk) {
  const int64_t ox = sx[0], oy = sy[0], oz = sz[0];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t dx = bh_quirk ? 0 : (int64_t)((uint64_t)sx[i] - (uint64_t)ox);
    int64_t dy = bh_quirk ? 0 : (int64_t)((uint64_t)sy[i] - (uint64_t)oy);
    int64_t dz = bh_quirk ? 0 : (int64_t)((uint64_t)sz[i] - (uint64_t)oz);
    x[i] = xadd(xmul(__ll2double_rn(dx), ss), x[i]);
    y[i] = xadd(xmul(__ll2double_rn(dy), ss), y[i]);
    z[i] = xadd(xmul(__ll2double_rn(dz), ss), z[i]);
  }
}

int grid_for(int64_t n) {
  int64_t g = ceil_div(n, kBlock);
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

int verlet_drift(phys_ctx* c, double dt) { return verlet_drift_pos(c, dt, c->x, c->y, c->z); }

// The position step on the given position arrays (LocalPosition in sector mode).
int verlet_drift_pos(phys_ctx* c, double dt, double* x, double* y, double* z) {
  PHYS_LAUNCH(c, drift_kernel, grid_for(c->n), kBlock, 0, c->n, dt, x, y, z, c->vx, c->vy, c->vz,
              c->ax, c->ay, c->az, c->pax, c->pay, c->paz);
  return PHYS_OK;
}

int verlet_kick(phys_ctx* c, double dt) {
  PHYS_LAUNCH(c, kick_kernel, grid_for(c->n), kBlock, 0, c->n, dt, c->vx, c->vy, c->vz, c->ax,
              c->ay, c->az, c->pax, c->pay, c->paz, c->d_status);
  return PHYS_OK;
}

int verlet_kick_drift(phys_ctx* c, double dt) {
  PHYS_LAUNCH(c, kick_drift_kernel, grid_for(c->n), kBlock, 0, c->n, dt, c->x, c->y, c->z, c->vx,
              c->vy, c->vz, c->ax, c->ay, c->az, c->pax, c->pay, c->paz, c->d_status);
  return PHYS_OK;
}

int flatten_sectors(phys_ctx* c, const int64_t* dsx, const int64_t* dsy, const int64_t* dsz,
                    const double* dlx, const double* dly, const double* dlz, double sector_size,
                    int bh_quirk) {
  (void)dlx;
  (void)dly;
  (void)dlz;
  PHYS_LAUNCH(c, flatten_kernel, grid_for(c->n), kBlock, 0, c->n, dsx, dsy, dsz, c->x, c->y,
              c->z, sector_size, bh_quirk);
  return PHYS_OK;
}

}  // namespace phys
