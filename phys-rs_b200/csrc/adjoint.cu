// K9: hand-written adjoint of the direct-sum acceleration and the
// Velocity-Verlet step (integrators.rs:63-104 with gravity.rs:53-69 and
// a = F/m), for the gradient of a trajectory loss
//     L = sum_i |x_i(T) - target_i|^2
// with respect to initial positions, velocities and masses.
//
// Forward program (f64, the sliced direct sum of direct.cu):
//     a_0 = A(x_0)
//     x_{k+1} = x_k + (v_k dt + a_k dt^2/2)
//     a_{k+1} = A(x_{k+1})
//     v_{k+1} = v_k + (a_k + a_{k+1}) dt/2
// Reverse sweep (bars are adjoints), k = T-1 .. 0:
//     abar_{k+1} += (dt/2) vbar_{k+1}
//     xbar_{k+1} += J(x_{k+1})^T abar_{k+1};  mbar += (dA/dm)^T abar_{k+1}
//     abar_k      = (dt/2) vbar_{k+1} + (dt^2/2) xbar_{k+1}
//     vbar_k      = vbar_{k+1} + dt xbar_{k+1};  xbar_k = xbar_{k+1}
// then xbar_0 += J(x_0)^T abar_0, mbar += (dA/dm)^T abar_0.
// With a_i = G sum_{j != i} m_j r_ij / s^3 (r_ij = x_j - x_i,
// s^2 = |r_ij|^2 + eps^2) and K_ij = I/s^3 - 3 r r^T / s^5 (symmetric):
//     (J^T w)_j = G sum_{i != j} K_ij (m_j w_i - m_i w_j)
//     (dA/dm)^T w)_j = G sum_{i != j} (r_ij . w_i) / s^3
// States are checkpointed every `checkpoint` steps and each segment is
// recomputed (deterministically, bit for bit) during the reverse sweep.
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace phys {
namespace {

constexpr int kTile = 128;
constexpr int kBlock = 256;

int grid_for(int64_t n) { return (int)std::min<int64_t>(std::max<int64_t>(ceil_div(n, kBlock), 1), 148 * 8); }

// x += v dt + a dt^2/2 ; per component arrays of n.
__global__ void adj_drift(int64_t n, double dt, double* __restrict__ x,
                          const double* __restrict__ v, const double* __restrict__ a) {
  const double h2 = xmul(xmul(0.5, dt), dt);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = xadd(x[i], xadd(xmul(v[i], dt), xmul(a[i], h2)));
}

// v += (a_old + a_new) dt/2
__global__ void adj_kick(int64_t n, double dt, double* __restrict__ v,
                         const double* __restrict__ a0, const double* __restrict__ a1) {
  const double hdt = xmul(0.5, dt);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * n;
       i += (int64_t)gridDim.x * blockDim.x)
    v[i] = xadd(v[i], xmul(xadd(a0[i], a1[i]), hdt));
}

// Per-block partial sums of (x - t)^2 and xbar = 2 (x - t).
__global__ void loss_kernel(int64_t n, const double* __restrict__ x,
                            const double* __restrict__ t, double* __restrict__ xbar,
                            double* __restrict__ part) {
  __shared__ double sh[kBlock];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double d = x[i] - t[i];
    s = fma(d, d, s);
    if (xbar) xbar[i] = 2.0 * d;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int k = kBlock / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void sum_kernel(int nparts, const double* __restrict__ part, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double s = 0.0;
  for (int b = 0; b < nparts; ++b) s += part[b];
  out[0] = s;
}

// abar += h * vbar
__global__ void adj_pre(int64_t n, double h, double* __restrict__ abar,
                        const double* __restrict__ vbar) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * n;
       i += (int64_t)gridDim.x * blockDim.x)
    abar[i] = fma(h, vbar[i], abar[i]);
}

// abar = h vbar + h2 xbar ; vbar += dt xbar
__global__ void adj_post(int64_t n, double dt, double* __restrict__ abar,
                         double* __restrict__ vbar, const double* __restrict__ xbar) {
  const double h = 0.5 * dt, h2 = 0.5 * dt * dt;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double vb = vbar[i], xb = xbar[i];
    abar[i] = fma(h, vb, h2 * xb);
    vbar[i] = fma(dt, xb, vb);
  }
}

// VJP of the acceleration at positions (x, y, z) with weights w (SoA, n
// each): per target j and source slice, partial (ux, uy, uz, gm).
__global__ void __launch_bounds__(kTile)
vjp_kernel(int64_t n, int64_t slice_len, const double* __restrict__ x,
           const double* __restrict__ y, const double* __restrict__ z,
           const double* __restrict__ m, const double* __restrict__ wx,
           const double* __restrict__ wy, const double* __restrict__ wz, double eps2,
           double* __restrict__ part) {
  __shared__ double4 ts[kTile];
  __shared__ double4 tw[kTile];
  const int64_t j = blockIdx.x * (int64_t)kTile + threadIdx.x;
  const bool valid = j < n;
  const double xj = valid ? x[j] : 0.0, yj = valid ? y[j] : 0.0, zj = valid ? z[j] : 0.0;
  const double mj = valid ? m[j] : 0.0;
  const double wjx = valid ? wx[j] : 0.0, wjy = valid ? wy[j] : 0.0, wjz = valid ? wz[j] : 0.0;
  const int64_t lo = blockIdx.y * slice_len;
  const int64_t hi = min64(n, lo + slice_len);
  double ux = 0.0, uy = 0.0, uz = 0.0, gm = 0.0;
  for (int64_t base = lo; base < hi; base += kTile) {
    const int64_t i = base + threadIdx.x;
    __syncthreads();
    if (i < hi) {
      ts[threadIdx.x] = make_double4(x[i], y[i], z[i], m[i]);
      tw[threadIdx.x] = make_double4(wx[i], wy[i], wz[i], 0.0);
    } else {
      ts[threadIdx.x] = make_double4(0, 0, 0, 0);
      tw[threadIdx.x] = make_double4(0, 0, 0, 0);
    }
    __syncthreads();
    const int cnt = (int)min64(kTile, hi - base);
    for (int k = 0; k < cnt; ++k) {
      const bool self = base + k == j;
      const double4 s = ts[k];
      const double4 w = tw[k];
      const double rx = xj - s.x, ry = yj - s.y, rz = zj - s.z;  // r_ij = x_j - x_i
      const double s2 = self ? 1.0 : fma(rx, rx, fma(ry, ry, fma(rz, rz, eps2)));
      const double inv = rsqrt(s2);
      const double inv2 = inv * inv;
      const double inv3 = self ? 0.0 : inv2 * inv;
      const double inv5 = inv3 * inv2;
      // q = m_j w_i - m_i w_j ; K q = q / s^3 - 3 r (r . q) / s^5
      const double qx = mj * w.x - s.w * wjx;
      const double qy = mj * w.y - s.w * wjy;
      const double qz = mj * w.z - s.w * wjz;
      const double rq3 = 3.0 * fma(rx, qx, fma(ry, qy, rz * qz)) * inv5;
      ux += qx * inv3 - rx * rq3;
      uy += qy * inv3 - ry * rq3;
      uz += qz * inv3 - rz * rq3;
      gm = fma(fma(rx, w.x, fma(ry, w.y, rz * w.z)), inv3, gm);
    }
  }
  if (!valid) return;
  double* p = part + (size_t)blockIdx.y * 4 * n;
  p[j] = ux;
  p[n + j] = uy;
  p[2 * n + j] = uz;
  p[3 * n + j] = gm;
}

// xbar += G sum_slices u ; mbar += G sum_slices gm (slice order fixed): one
// thread per (target, component), its slices' loads in flight together.
__global__ void vjp_reduce(int64_t n, int nsl, const double* __restrict__ part, double G,
                           double* __restrict__ xbar, double* __restrict__ mbar) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < 4 * n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(e / n);
    const int64_t j = e - k * n;
    const double u = slice_sum(part + k * n + j, 4 * (size_t)n, nsl);
    double* out = k < 3 ? xbar + k * n + j : mbar + j;
    *out += G * u;
  }
}

int64_t slices_for(int64_t n) {
  int64_t s = ceil_div(148LL * 2048, ceil_div(n, kTile) * kTile);
  s = std::min<int64_t>(s, ceil_div(n, kTile));
  return std::max<int64_t>(s, 1);
}

struct Adj {
  int64_t n, T, K, nck;
  double *X, *V, *A, *A2;   // 3n each
  double *ckpt;             // nck * 6n
  double *seg;              // (K+1) * 3n
  double *xbar, *vbar, *abar, *mbar, *tgt;
  double *fpart, *vpart, *lpart, *loss;
  int64_t fsl, vsl;
};

int force(phys_ctx* c, const phys_params* p, Adj& a, const double* x, double* out) {
  const int64_t n = a.n;
  int st = direct_accel_launch_scratch(c->stream, n, x, x + n, x + 2 * n, c->m, p->G, p->eps,
                                       PHYS_F64, a.fsl, a.fpart, nullptr, nullptr, c->d_status,
                                       out, out + n, out + 2 * n);
  c->launches += 2;
  if (st) return cuda_fail(c, cudaGetLastError(), "adjoint force launch");
  return PHYS_OK;
}

int step(phys_ctx* c, const phys_params* p, Adj& a, double dt) {
  PHYS_LAUNCH(c, adj_drift, grid_for(a.n), kBlock, 0, a.n, dt, a.X, a.V, a.A);
  PHYS_TRY(force(c, p, a, a.X, a.A2));
  PHYS_LAUNCH(c, adj_kick, grid_for(a.n), kBlock, 0, a.n, dt, a.V, a.A, a.A2);
  std::swap(a.A, a.A2);
  return PHYS_OK;
}

int vjp(phys_ctx* c, const phys_params* p, Adj& a, const double* x) {
  const int64_t n = a.n;
  const int64_t slice_len = ceil_div(ceil_div(n, a.vsl), kTile) * kTile;
  const int64_t nsl = ceil_div(n, slice_len);
  dim3 grid((unsigned)ceil_div(n, kTile), (unsigned)nsl);
  PHYS_LAUNCH(c, vjp_kernel, grid, kTile, 0, n, slice_len, x, x + n, x + 2 * n, c->m, a.abar,
              a.abar + n, a.abar + 2 * n, p->eps * p->eps, a.vpart);
  PHYS_LAUNCH(c, vjp_reduce, grid_for(4 * n), kBlock, 0, n, (int)nsl, a.vpart, p->G, a.xbar,
              a.mbar);
  return PHYS_OK;
}

int setup(phys_ctx* c, int64_t T, int64_t K, bool reverse, Adj& a) {
  const int64_t n = c->n;
  a.n = n;
  a.T = T;
  a.K = reverse ? K : 0;
  a.nck = reverse ? std::max<int64_t>(ceil_div(T, K), 1) : 0;
  a.fsl = slices_for(n);
  a.vsl = slices_for(n);
  const size_t doubles = 12 * n + a.nck * 6 * n + (a.K + 1) * 3 * n + 13 * n;
  int st = PHYS_OK;
  double* b = (double*)ws_get(c, WS_ADJ0, sizeof(double) * doubles, &st);
  if (st) return st;
  a.X = b; b += 3 * n;
  a.V = b; b += 3 * n;
  a.A = b; b += 3 * n;
  a.A2 = b; b += 3 * n;
  a.ckpt = b; b += a.nck * 6 * n;
  a.seg = b; b += (a.K + 1) * 3 * n;
  a.xbar = b; b += 3 * n;
  a.vbar = b; b += 3 * n;
  a.abar = b; b += 3 * n;
  a.mbar = b; b += n;
  a.tgt = b; b += 3 * n;
  a.fpart = (double*)ws_get(c, WS_ADJ1, sizeof(double) * 3 * n * a.fsl, &st);
  if (st) return st;
  a.vpart = (double*)ws_get(c, WS_ADJ2, sizeof(double) * 4 * n * a.vsl, &st);
  if (st) return st;
  a.lpart = (double*)ws_get(c, WS_ADJ3, sizeof(double) * (148 * 8 + 8), &st);
  if (st) return st;
  a.loss = a.lpart + 148 * 8;
  return PHYS_OK;
}

int copy_d2d(phys_ctx* c, double* dst, const double* src, int64_t count) {
  PHYS_CUDA(c, cudaMemcpyAsync(dst, src, sizeof(double) * count, cudaMemcpyDeviceToDevice,
                               c->stream));
  return PHYS_OK;
}

// A segment's launches are the same for every segment of the same length
// (same kernels, same buffers: the forward steps, their recomputation, the
// reverse steps), so each kind is captured in a CUDA graph once per length
// and replayed: one launch per segment instead of several per step, and the
// same kernels in the same order, so the results are the same bit for bit.
// Segments whose host-side state does not return to its start (an odd
// number of steps swaps a.A and a.A2) are launched directly.
struct Replay {
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  int64_t len[2] = {-1, -1};  // segment length captured in each slot
  uint64_t launches[2] = {0, 0};
  Replay() = default;
  Replay(const Replay&) = delete;
  Replay& operator=(const Replay&) = delete;
  ~Replay() {
    for (cudaGraphExec_t e : exec)
      if (e) cudaGraphExecDestroy(e);
  }
};

template <class F>
int run_segment(phys_ctx* c, Replay& R, int64_t len, bool replayable, F&& enqueue) {
  int slot = R.len[0] == len ? 0 : (R.len[1] == len ? 1 : -1);
  if (replayable && slot < 0) {
    slot = R.exec[0] ? 1 : 0;
    if (R.exec[slot]) {
      cudaGraphExecDestroy(R.exec[slot]);
      R.exec[slot] = nullptr;
      R.len[slot] = -1;
    }
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      const uint64_t l0 = c->launches;
      const int st = enqueue();
      cudaGraph_t g = nullptr;
      const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
      cudaGraphExec_t exec = nullptr;
      const bool ok = st == PHYS_OK && e == cudaSuccess && g &&
                      cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
      if (g) cudaGraphDestroy(g);
      R.launches[slot] = c->launches - l0;
      c->launches = l0;
      if (ok) {
        R.exec[slot] = exec;
        R.len[slot] = len;
      } else {
        // nothing ran: the segment is launched directly below (the
        // capture's host-side state changes were a whole even segment)
        if (exec) cudaGraphExecDestroy(exec);
        cudaGetLastError();
        c->err.clear();
        slot = -1;
      }
    } else {
      cudaGetLastError();
      slot = -1;
    }
  }
  if (!replayable || slot < 0) return enqueue();
  PHYS_CUDA(c, cudaGraphLaunch(R.exec[slot], c->stream));
  c->launches += R.launches[slot];
  return PHYS_OK;
}

// x0, v0 of the context state into a.X, a.V (SoA blocks of 3n).
int load_initial(phys_ctx* c, Adj& a) {
  const int64_t n = a.n;
  PHYS_TRY(copy_d2d(c, a.X, c->x, n));
  PHYS_TRY(copy_d2d(c, a.X + n, c->y, n));
  PHYS_TRY(copy_d2d(c, a.X + 2 * n, c->z, n));
  PHYS_TRY(copy_d2d(c, a.V, c->vx, n));
  PHYS_TRY(copy_d2d(c, a.V + n, c->vy, n));
  PHYS_TRY(copy_d2d(c, a.V + 2 * n, c->vz, n));
  return PHYS_OK;
}

int forward(phys_ctx* c, const phys_params* p, Adj& a, double dt, bool keep_ckpt,
            Replay* R = nullptr) {
  PHYS_TRY(load_initial(c, a));
  PHYS_TRY(force(c, p, a, a.X, a.A));
  if (!keep_ckpt) {
    for (int64_t k = 0; k < a.T; ++k) PHYS_TRY(step(c, p, a, dt));
    return PHYS_OK;
  }
  for (int64_t k0 = 0; k0 < a.T; k0 += a.K) {
    double* ck = a.ckpt + (k0 / a.K) * 6 * a.n;
    PHYS_TRY(copy_d2d(c, ck, a.X, 3 * a.n));
    PHYS_TRY(copy_d2d(c, ck + 3 * a.n, a.V, 3 * a.n));
    const int64_t len = std::min<int64_t>(a.K, a.T - k0);
    auto steps = [&]() -> int {
      for (int64_t j = 0; j < len; ++j) PHYS_TRY(step(c, p, a, dt));
      return PHYS_OK;
    };
    if (R)
      PHYS_TRY(run_segment(c, *R, len, len % 2 == 0, steps));
    else
      PHYS_TRY(steps());
  }
  return PHYS_OK;
}

int loss_of(phys_ctx* c, Adj& a, bool grad, double* out) {
  const int g = grid_for(3 * a.n);
  PHYS_LAUNCH(c, loss_kernel, g, kBlock, 0, a.n, a.X, a.tgt, grad ? a.xbar : nullptr, a.lpart);
  PHYS_LAUNCH(c, sum_kernel, 1, 32, 0, g, a.lpart, a.loss);
  PHYS_CUDA(c, cudaMemcpyAsync(out, a.loss, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  return PHYS_OK;
}

int check_args(phys_ctx* c, const phys_params* p, int64_t nsteps, int64_t K, const double* tx,
               const double* ty, const double* tz) {
  if (!p) return fail(c, PHYS_ERR_ARG, "params is NULL");
  if (p->precision != PHYS_F64) return fail(c, PHYS_ERR_ARG, "adjoint runs in PHYS_F64");
  if (nsteps < 0 || K <= 0) return fail(c, PHYS_ERR_ARG, "nsteps >= 0 and checkpoint > 0");
  if (!tx || !ty || !tz) return fail(c, PHYS_ERR_ARG, "targets are required");
  if (c->n < 2) return fail(c, PHYS_ERR_STATE, "need at least 2 bodies");
  return PHYS_OK;
}

int upload_targets(phys_ctx* c, Adj& a, const double* tx, const double* ty, const double* tz) {
  const int64_t n = a.n;
  PHYS_CUDA(c, cudaMemcpyAsync(a.tgt, tx, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  PHYS_CUDA(c, cudaMemcpyAsync(a.tgt + n, ty, sizeof(double) * n, cudaMemcpyHostToDevice,
                               c->stream));
  PHYS_CUDA(c, cudaMemcpyAsync(a.tgt + 2 * n, tz, sizeof(double) * n, cudaMemcpyHostToDevice,
                               c->stream));
  return PHYS_OK;
}

}  // namespace

int trajectory_loss(phys_ctx* c, const phys_params* p, double dt, int64_t nsteps,
                    const double* tx, const double* ty, const double* tz, double* loss,
                    double* xT, double* yT, double* zT) {
  PHYS_TRY(check_args(c, p, nsteps, 1, tx, ty, tz));
  Adj a{};
  PHYS_TRY(setup(c, nsteps, 1, false, a));
  PHYS_TRY(upload_targets(c, a, tx, ty, tz));
  PHYS_TRY(forward(c, p, a, dt, false));
  double l = 0.0;
  PHYS_TRY(loss_of(c, a, false, &l));
  double* outs[3] = {xT, yT, zT};
  for (int k = 0; k < 3; ++k)
    if (outs[k])
      PHYS_CUDA(c, cudaMemcpyAsync(outs[k], a.X + k * a.n, sizeof(double) * a.n,
                                   cudaMemcpyDeviceToHost, c->stream));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  *loss = l;
  return PHYS_OK;
}

int adjoint(phys_ctx* c, const phys_params* p, double dt, int64_t nsteps, int64_t K,
            const double* tx, const double* ty, const double* tz, double* loss, double* gxyz[3],
            double* gvxyz[3], double* gm) {
  PHYS_TRY(check_args(c, p, nsteps, K, tx, ty, tz));
  Adj a{};
  PHYS_TRY(setup(c, nsteps, K, true, a));
  const int64_t n = a.n;
  PHYS_TRY(upload_targets(c, a, tx, ty, tz));
  Replay fwd, rec, rev;  // captured segments: forward, recomputation, reverse
  PHYS_TRY(forward(c, p, a, dt, true, &fwd));
  double l = 0.0;
  PHYS_TRY(loss_of(c, a, true, &l));  // xbar = dL/dx_T
  PHYS_CUDA(c, cudaMemsetAsync(a.vbar, 0, sizeof(double) * 3 * n, c->stream));
  PHYS_CUDA(c, cudaMemsetAsync(a.abar, 0, sizeof(double) * 3 * n, c->stream));
  PHYS_CUDA(c, cudaMemsetAsync(a.mbar, 0, sizeof(double) * n, c->stream));
  const double h = 0.5 * dt;
  for (int64_t s = a.nck - 1; s >= 0 && a.T > 0; --s) {
    const int64_t k0 = s * a.K;
    const int64_t len = std::min<int64_t>(a.K, a.T - k0);
    // recompute the segment: seg[j] = x_{k0 + j}, j = 0..len
    const double* ck = a.ckpt + s * 6 * n;
    PHYS_TRY(copy_d2d(c, a.X, ck, 3 * n));
    PHYS_TRY(copy_d2d(c, a.V, ck + 3 * n, 3 * n));
    auto recompute = [&]() -> int {
      PHYS_TRY(force(c, p, a, a.X, a.A));
      PHYS_TRY(copy_d2d(c, a.seg, a.X, 3 * n));
      for (int64_t j = 0; j < len; ++j) {
        PHYS_TRY(step(c, p, a, dt));
        PHYS_TRY(copy_d2d(c, a.seg + (j + 1) * 3 * n, a.X, 3 * n));
      }
      return PHYS_OK;
    };
    PHYS_TRY(run_segment(c, rec, len, len % 2 == 0, recompute));
    auto reverse = [&]() -> int {
      for (int64_t j = len - 1; j >= 0; --j) {  // reverse of step k = k0 + j
        PHYS_LAUNCH(c, adj_pre, grid_for(3 * n), kBlock, 0, n, h, a.abar, a.vbar);
        PHYS_TRY(vjp(c, p, a, a.seg + (j + 1) * 3 * n));
        PHYS_LAUNCH(c, adj_post, grid_for(3 * n), kBlock, 0, n, dt, a.abar, a.vbar, a.xbar);
      }
      return PHYS_OK;
    };
    PHYS_TRY(run_segment(c, rev, len, true, reverse));
  }
  // a_0 = A(x_0)
  PHYS_TRY(load_initial(c, a));
  PHYS_TRY(vjp(c, p, a, a.X));
  for (int k = 0; k < 3; ++k) {
    if (gxyz[k])
      PHYS_CUDA(c, cudaMemcpyAsync(gxyz[k], a.xbar + k * n, sizeof(double) * n,
                                   cudaMemcpyDeviceToHost, c->stream));
    if (gvxyz[k])
      PHYS_CUDA(c, cudaMemcpyAsync(gvxyz[k], a.vbar + k * n, sizeof(double) * n,
                                   cudaMemcpyDeviceToHost, c->stream));
  }
  if (gm)
    PHYS_CUDA(c, cudaMemcpyAsync(gm, a.mbar, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                 c->stream));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  *loss = l;
  return PHYS_OK;
}

}  // namespace phys
