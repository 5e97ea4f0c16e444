// NFW phantom halo (src/physics/nfw.rs): the system's per-body force and its
// fusion into the acceleration epilogue.  Arithmetic follows nfw.rs in
// operation order with non-contracting IEEE intrinsics; ln(1 + x) is CUDA's
// double log (within 1 ulp; the reference calls the platform's libm).
#include "common.cuh"

namespace phys {
namespace {

constexpr int kBlock = 256;
constexpr double kGSi = 6.67430e-11;               // constants.rs:7
constexpr double kPi = 3.141592653589793;          // std::f64::consts::PI
constexpr double kCenterSkip = 1e-10;              // nfw.rs:123

struct Halo {
  double rho_0, rs, cx, cy, cz;
};

// nfw_enclosed_mass (nfw.rs:76-83)
__device__ __forceinline__ double enclosed_mass(double r, const Halo& h) {
  if (r <= 0.0 || h.rs <= 0.0) return 0.0;
  const double x = xdiv(r, h.rs);
  const double rs3 = xmul(xmul(h.rs, h.rs), h.rs);  // rs.powi(3)
  const double factor = xmul(xmul(xmul(4.0, kPi), h.rho_0), rs3);
  const double opx = xadd(1.0, x);
  return xmul(factor, xsub(log(opx), xdiv(x, opx)));
}

// nfw_gravity_system body (nfw.rs:120-138): the force on one body, or false
// at the centre.
__device__ __forceinline__ bool halo_force(double px, double py, double pz, double m,
                                           const Halo& h, double& f0, double& f1, double& f2) {
  const double rx = xsub(px, h.cx), ry = xsub(py, h.cy), rz = xsub(pz, h.cz);
  const double r = xsqrt(xlen2(rx, ry, rz));
  if (r < kCenterSkip) return false;
  const double menc = enclosed_mass(r, h);
  const double hx = xdiv(rx, r), hy = xdiv(ry, r), hz = xdiv(rz, r);
  const double fmag = xdiv(xmul(xmul(kGSi, menc), m), xmul(r, r));
  f0 = xmul(-hx, fmag);
  f1 = xmul(-hy, fmag);
  f2 = xmul(-hz, fmag);
  return true;
}

// Force += f_nfw
__global__ void __launch_bounds__(kBlock)
nfw_force_kernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                 const double* __restrict__ z, const double* __restrict__ m, Halo h,
                 double* __restrict__ fx, double* __restrict__ fy, double* __restrict__ fz) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double f0, f1, f2;
    if (halo_force(x[i], y[i], z[i], m[i], h, f0, f1, f2)) {
      fx[i] = xadd(fx[i], f0);
      fy[i] = xadd(fy[i], f1);
      fz[i] = xadd(fz[i], f2);
    }
  }
}

// a = (F_gravity + f_nfw) / m  (Force += in system order, then
// compute_acceleration_system, integrators.rs:110-118)
__global__ void __launch_bounds__(kBlock)
nfw_accel_kernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                 const double* __restrict__ z, const double* __restrict__ m, Halo h,
                 const double* __restrict__ fx, const double* __restrict__ fy,
                 const double* __restrict__ fz, double* __restrict__ ax, double* __restrict__ ay,
                 double* __restrict__ az, int32_t* status) {
  bool bad = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double mi = m[i];
    double F0 = fx[i], F1 = fy[i], F2 = fz[i];
    double f0, f1, f2;
    if (halo_force(x[i], y[i], z[i], mi, h, f0, f1, f2)) {
      F0 = xadd(F0, f0);
      F1 = xadd(F1, f1);
      F2 = xadd(F2, f2);
    }
    const double a0 = xdiv(F0, mi), a1 = xdiv(F1, mi), a2 = xdiv(F2, mi);
    ax[i] = a0;
    ay[i] = a1;
    az[i] = a2;
    bad |= !isfinite(a0) || !isfinite(a1) || !isfinite(a2);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status, kStatNonfinite);
}

Halo to_halo(const phys_nfw_halo& p) {
  return Halo{p.rho_0, p.scale_radius, p.center[0], p.center[1], p.center[2]};
}

int grid_for(int64_t n) { return (int)std::min<int64_t>(ceil_div(n, kBlock), 148 * 16); }

}  // namespace

int nfw_add_forces(phys_ctx* c, const phys_nfw_halo& halo, const double* px, const double* py,
                   const double* pz, double* fx, double* fy, double* fz) {
  if (c->n == 0) return PHYS_OK;
  PHYS_LAUNCH(c, nfw_force_kernel, grid_for(c->n), kBlock, 0, c->n, px, py, pz, c->m,
              to_halo(halo), fx, fy, fz);
  return PHYS_OK;
}

int nfw_accel(phys_ctx* c, const phys_nfw_halo& halo, const double* px, const double* py,
              const double* pz, const double* fx, const double* fy, const double* fz, double* ax,
              double* ay, double* az) {
  if (c->n == 0) return PHYS_OK;
  PHYS_LAUNCH(c, nfw_accel_kernel, grid_for(c->n), kBlock, 0, c->n, px, py, pz, c->m,
              to_halo(halo), fx, fy, fz, ax, ay, az, c->d_status);
  return PHYS_OK;
}

}  // namespace phys

// Host scalars (nfw.rs:61-92), the same formulas and operation order: one
// rounding per operation as written (the host compiler targets baseline
// x86-64, which has no FMA instruction to contract into, and no fast-math).
extern "C" {

double phys_nfw_density(double r, double rho_0, double rs) {
  if (r <= 0.0 || rs <= 0.0) return 0.0;
  const double x = r / rs;
  const double opx = 1.0 + x;
  return rho_0 / (x * (opx * opx));
}

double phys_nfw_enclosed_mass(double r, double rho_0, double rs) {
  if (r <= 0.0 || rs <= 0.0) return 0.0;
  const double x = r / rs;
  const double factor = 4.0 * 3.141592653589793 * rho_0 * (rs * rs * rs);
  return factor * (std::log(1.0 + x) - x / (1.0 + x));
}

double phys_nfw_circular_velocity(double r, double rho_0, double rs) {
  const double m_enc = phys_nfw_enclosed_mass(r, rho_0, rs);
  return std::sqrt(std::fmax(6.67430e-11 * m_enc / r, 0.0));
}

}  // extern "C"
