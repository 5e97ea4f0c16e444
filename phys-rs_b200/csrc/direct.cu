// K1: softened all-pairs direct sum (brute_force_gravity_system,
// src/physics/gravity.rs:53-69), in three precisions.
//
// Layout: sources are staged through shared memory in tiles; every lane of a
// warp reads the same source (shared-memory broadcast) while owning one
// target.  For small N the source range is split into `slices` so the grid
// covers all SMs; slice partials are reduced in slice order (deterministic).
#include "common.cuh"

namespace phys {
namespace {

// ---------------------------------------------------------------------------
// F64_EXACT: the reference's arithmetic, j in order 0..N-1, no FMA.
//   r = x_j - x_i; r2 = len2(r); s2 = r2 + eps2; s3 = s2 * sqrt(s2)
//   sc = ((G*m_i)*m_j)/s3; F += r*sc            (gravity.rs:58-65)
// Only the additions into F are ordered; the terms r*sc are independent.  A
// block takes kXT targets: in round k its compute warps evaluate the terms
// of sources [k kXJ, (k+1) kXJ) against every target into shared memory
// (each thread one source against two targets, the source of round k+1
// loaded ahead), while lane t of warp 0 adds round k-1's terms of target t
// in j order, skipping j == i as the reference does.  The divides and square
// roots, whose latency bounded the one-thread-per-target form, run in
// parallel; the sum is the reference's bit for bit.  The floor of any exact
// form is the ordered chain of N - 1 dependent f64 additions per component
// (an f64 add waits ≈ 8 cycles for the one before it: ≈ 4 us at N = 1024);
// the kernel takes ≈ 4 times that.
// ---------------------------------------------------------------------------
constexpr int kXT = 8;                    // targets per block
constexpr int kXJ = 64;                   // sources per round
constexpr int kXCompute = kXT * kXJ / 2;  // compute threads: two targets each
// Warp 0 adds; the compute warps are the first kXCompute / 32 warps whose
// index is not a multiple of 4, so none shares warp 0's scheduler (warps are
// spread over an SM's four schedulers by index): warps 1-3, 5-7, 9, 10 of
// 12; warps 4, 8 and 11 return at once.  The round barrier is a named
// barrier over the 9 working warps only.
constexpr int kXWarps = 12;
constexpr int kXBlock = 32 * kXWarps;
constexpr int kXWorking = 32 + kXCompute;
static_assert(kXT <= 32 && kXCompute % 32 == 0 && kXJ % 32 == 0, "exact block layout");
static_assert(kXCompute / 32 == 8 && kXWorking == 288, "bar.sync count below");

__global__ void __launch_bounds__(kXBlock)
direct_exact_kernel(int64_t n, int64_t t0, int64_t t1, const double* __restrict__ x,
                    const double* __restrict__ y, const double* __restrict__ z,
                    const double* __restrict__ m, double G, double eps2, int want_force,
                    double* __restrict__ ox, double* __restrict__ oy, double* __restrict__ oz,
                    int32_t* status) {
  __shared__ double term[2][3][kXT][kXJ + 1];  // [round parity][x, y, z][target][source]
  __shared__ double4 tgt[kXT];                 // x_i, y_i, z_i, G*m_i
  const int w = threadIdx.x >> 5;
  const int cw = (w % 4 == 0) ? -1 : w - 1 - w / 4;  // compute warp 0..7, or -1
  if (w != 0 && (cw < 0 || cw >= kXCompute / 32)) return;  // idle: no barrier
  // tid: warp 0 keeps its lanes; compute warp cw acts as threads 32 + 32 cw + lane
  const int tid = w == 0 ? (int)threadIdx.x : 32 + cw * 32 + (int)(threadIdx.x & 31);
  const int64_t i0 = t0 + blockIdx.x * (int64_t)kXT;
  if (tid < kXT) {
    const int64_t i = i0 + tid;
    tgt[tid] = i < t1 ? make_double4(x[i], y[i], z[i], xmul(G, m[i]))
                      : make_double4(0.0, 0.0, 0.0, 0.0);
  }
  asm volatile("bar.sync 1, 288;" ::: "memory");  // kXWorking
  const int64_t rounds = ceil_div(n, kXJ);
  // compute threads: source slot jj, targets ta and ta + kXT/2
  const int c = tid - 32, jj = c % kXJ, ta = c / kXJ;
  double4 src = make_double4(0.0, 0.0, 0.0, 0.0);
  if (tid >= 32 && jj < n) src = make_double4(x[jj], y[jj], z[jj], m[jj]);
  double fx = 0.0, fy = 0.0, fz = 0.0;  // warp 0, lane t < kXT: target t
  for (int64_t k = 0; k <= rounds; ++k) {
    const int b = (int)(k & 1);
    if (tid >= 32) {
      if (k < rounds) {
        const int64_t j = k * kXJ + jj;
        const int64_t jn = j + kXJ;
        double4 next = make_double4(0.0, 0.0, 0.0, 0.0);
        if (jn < n) next = make_double4(x[jn], y[jn], z[jn], m[jn]);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int t = ta + h * (kXT / 2);
          const double4 T = tgt[t];
          double ax = 0.0, ay = 0.0, az = 0.0;
          if (j < n && i0 + t < t1) {
            const double rx = xsub(src.x, T.x), ry = xsub(src.y, T.y), rz = xsub(src.z, T.z);
            const double s2 = xadd(xlen2(rx, ry, rz), eps2);
            const double sc = xdiv(xmul(T.w, src.w), xmul(s2, xsqrt(s2)));
            ax = xmul(rx, sc);
            ay = xmul(ry, sc);
            az = xmul(rz, sc);
          }
          term[b][0][t][jj] = ax;
          term[b][1][t][jj] = ay;
          term[b][2][t][jj] = az;
        }
        src = next;
      }
    } else if (k > 0 && tid < kXT) {
      const int pb = b ^ 1;
      const int64_t jb = (k - 1) * kXJ;
      const int cnt = (int)min64(kXJ, n - jb);
      // j == i sits at slot self, if in [0, cnt): the slots before and after
      // it as two straight runs, so that the loads run ahead of the adds
      const int64_t self = i0 + tid - jb;
      const int q1 = (int)(self < 0 ? 0 : self < cnt ? self : cnt);
      const int q2 = self >= 0 && self < cnt ? q1 + 1 : q1;
      const double* tx = term[pb][0][tid];
      const double* ty = term[pb][1][tid];
      const double* tz = term[pb][2][tid];
#pragma unroll 16
      for (int q = 0; q < q1; ++q) {
        fx = xadd(fx, tx[q]);
        fy = xadd(fy, ty[q]);
        fz = xadd(fz, tz[q]);
      }
#pragma unroll 16
      for (int q = q2; q < cnt; ++q) {
        fx = xadd(fx, tx[q]);
        fy = xadd(fy, ty[q]);
        fz = xadd(fz, tz[q]);
      }
    }
    asm volatile("bar.sync 1, 288;" ::: "memory");  // kXWorking
  }
  if (tid >= 32) return;
  const int64_t i = i0 + tid;
  const bool valid = tid < kXT && i < t1;
  if (valid) {
    if (!want_force) {  // compute_acceleration_system: a = F / m (integrators.rs:115)
      const double mi = m[i];
      fx = xdiv(fx, mi);
      fy = xdiv(fy, mi);
      fz = xdiv(fz, mi);
    }
    ox[i] = fx;
    oy[i] = fy;
    oz[i] = fz;
  }
  bool bad = valid && (!isfinite(fx) || !isfinite(fy) || !isfinite(fz));
  if (__any_sync(0xffffffffu, bad) && tid == 0) atomicOr(status, kStatNonfinite);
}

// ---------------------------------------------------------------------------
// F64: same law with FMA and rsqrt, accumulating sum m_j r / s^3 (G applied
// at the end).  Sources in [slice_lo, slice_hi); tile-aligned, so the tile
// holding the block's own targets (the only one that can contain j == i) is
// warp-uniform and takes the checked loop.
// ---------------------------------------------------------------------------
constexpr int kTile = 128;

template <bool kChecked>
__device__ __forceinline__ void f64_tile(const double4* __restrict__ t, int cnt, int self,
                                         double xi, double yi, double zi, double eps2,
                                         double& ax, double& ay, double& az) {
#pragma unroll 4
  for (int k = 0; k < cnt; ++k) {
    const double4 s = t[k];
    const double rx = s.x - xi, ry = s.y - yi, rz = s.z - zi;
    double r2 = fma(rx, rx, fma(ry, ry, fma(rz, rz, eps2)));
    double mj = s.w;
    if (kChecked && k == self) {
      mj = 0.0;
      r2 = 1.0;
    }
    const double inv = rsqrt(r2);
    const double w = mj * (inv * inv * inv);
    ax = fma(rx, w, ax);
    ay = fma(ry, w, ay);
    az = fma(rz, w, az);
  }
}

__global__ void __launch_bounds__(kTile)
direct_f64_kernel(int64_t n, int64_t t0, int64_t t1, int64_t slice_len,
                  const double* __restrict__ x, const double* __restrict__ y,
                  const double* __restrict__ z, const double* __restrict__ m, double G,
                  double eps2, int want_force, double* __restrict__ ox, double* __restrict__ oy,
                  double* __restrict__ oz, double* __restrict__ part, int32_t* status) {
  __shared__ double4 tile[kTile];
  const int64_t tbase = t0 + blockIdx.x * (int64_t)kTile;  // t0: a multiple of kTile
  const int64_t i = tbase + threadIdx.x;
  const bool valid = i < t1;
  const double xi = valid ? x[i] : 0.0, yi = valid ? y[i] : 0.0, zi = valid ? z[i] : 0.0;
  const int64_t lo = blockIdx.y * slice_len;
  const int64_t hi = min64(n, lo + slice_len);
  double ax = 0.0, ay = 0.0, az = 0.0;
  for (int64_t base = lo; base < hi; base += kTile) {
    int64_t j = base + threadIdx.x;
    __syncthreads();
    tile[threadIdx.x] = j < hi ? make_double4(x[j], y[j], z[j], m[j]) : make_double4(0, 0, 0, 0);
    __syncthreads();
    const int cnt = (int)min64(kTile, hi - base);
    if (base == tbase)
      f64_tile<true>(tile, cnt, threadIdx.x, xi, yi, zi, eps2, ax, ay, az);
    else
      f64_tile<false>(tile, cnt, -1, xi, yi, zi, eps2, ax, ay, az);
  }
  if (!valid) return;
  if (gridDim.y == 1) {
    double s = want_force ? G * m[i] : G;
    ox[i] = ax * s;
    oy[i] = ay * s;
    oz[i] = az * s;
    if (!isfinite(ax) || !isfinite(ay) || !isfinite(az)) atomicOr(status, kStatNonfinite);
  } else {
    double* p = part + (size_t)blockIdx.y * 3 * n;
    p[i] = ax;
    p[n + i] = ay;
    p[2 * n + i] = az;
  }
}

// ---------------------------------------------------------------------------
// F32C: f32 pair terms.  Positions are double-float pairs (hi, lo); the
// separation r = (hi_j - hi_i) + (lo_j - lo_i) keeps ~1e-7 relative accuracy
// however close the pair is compared with |x|.  Each group of 32 terms is
// summed in plain f32 and folded into a per-target (hi, lo) accumulator with
// Knuth's two-sum.
// ---------------------------------------------------------------------------
__global__ void split_bodies_kernel(int64_t n, const double* __restrict__ x,
                                    const double* __restrict__ y, const double* __restrict__ z,
                                    const double* __restrict__ m, float4* __restrict__ bh,
                                    float4* __restrict__ bl, int32_t* status) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float4 h, l;
    split_df(x[i], h.x, l.x);
    split_df(y[i], h.y, l.y);
    split_df(z[i], h.z, l.z);
    h.w = (float)m[i];
    l.w = 0.f;
    bh[i] = h;
    bl[i] = l;
    if (!isfinite(x[i]) || !isfinite(y[i]) || !isfinite(z[i]) || !isfinite(m[i]))
      atomicOr(status, kStatNonfinite);
  }
}

template <bool kChecked>
__device__ __forceinline__ void f32_group(const float4* __restrict__ th,
                                          const float4* __restrict__ tl, int k0, int k1, int self,
                                          float xh, float yh, float zh, float xl, float yl,
                                          float zl, float eps2, float& px, float& py,
                                          float& pz) {
#pragma unroll 8
  for (int k = k0; k < k1; ++k) {
    const float4 h = th[k];
    const float4 l = tl[k];
    const float rx = (h.x - xh) + (l.x - xl);
    const float ry = (h.y - yh) + (l.y - yl);
    const float rz = (h.z - zh) + (l.z - zl);
    float r2 = fmaf(rx, rx, fmaf(ry, ry, fmaf(rz, rz, eps2)));
    float mj = h.w;
    if (kChecked && k == self) {
      mj = 0.f;
      r2 = 1.f;
    }
    const float inv = rsqrt_sfu(r2);
    const float w = mj * (inv * inv * inv);
    px = fmaf(rx, w, px);
    py = fmaf(ry, w, py);
    pz = fmaf(rz, w, pz);
  }
}

__global__ void __launch_bounds__(kTile)
direct_f32c_kernel(int64_t n, int64_t t0, int64_t t1, int64_t slice_len,
                   const float4* __restrict__ bh, const float4* __restrict__ bl,
                   const double* __restrict__ m, double G, float eps2, int want_force,
                   double* __restrict__ ox, double* __restrict__ oy, double* __restrict__ oz,
                   double* __restrict__ part, int32_t* status) {
  __shared__ float4 th[kTile];
  __shared__ float4 tl[kTile];
  const int64_t tbase = t0 + blockIdx.x * (int64_t)kTile;  // t0: a multiple of kTile
  const int64_t i = tbase + threadIdx.x;
  const bool valid = i < t1;
  float4 hi4 = valid ? bh[i] : make_float4(0, 0, 0, 0);
  float4 lo4 = valid ? bl[i] : make_float4(0, 0, 0, 0);
  const int64_t lo = blockIdx.y * slice_len;
  const int64_t hi = min64(n, lo + slice_len);
  float ahx = 0.f, ahy = 0.f, ahz = 0.f, alx = 0.f, aly = 0.f, alz = 0.f;
  for (int64_t base = lo; base < hi; base += kTile) {
    int64_t j = base + threadIdx.x;
    __syncthreads();
    th[threadIdx.x] = j < hi ? bh[j] : make_float4(0, 0, 0, 0);
    tl[threadIdx.x] = j < hi ? bl[j] : make_float4(0, 0, 0, 0);
    __syncthreads();
    const int cnt = (int)min64(kTile, hi - base);
    const bool diag = base == tbase;
    for (int k0 = 0; k0 < cnt; k0 += 32) {
      const int k1 = min(cnt, k0 + 32);
      float px = 0.f, py = 0.f, pz = 0.f;
      if (diag)
        f32_group<true>(th, tl, k0, k1, threadIdx.x, hi4.x, hi4.y, hi4.z, lo4.x, lo4.y, lo4.z,
                        eps2, px, py, pz);
      else
        f32_group<false>(th, tl, k0, k1, -1, hi4.x, hi4.y, hi4.z, lo4.x, lo4.y, lo4.z, eps2, px,
                         py, pz);
      float s, e;
      two_sum(ahx, px, s, e);
      ahx = s;
      alx += e;
      two_sum(ahy, py, s, e);
      ahy = s;
      aly += e;
      two_sum(ahz, pz, s, e);
      ahz = s;
      alz += e;
    }
  }
  if (!valid) return;
  const double ax = (double)ahx + (double)alx;
  const double ay = (double)ahy + (double)aly;
  const double az = (double)ahz + (double)alz;
  if (gridDim.y == 1) {
    double s = want_force ? G * m[i] : G;
    ox[i] = ax * s;
    oy[i] = ay * s;
    oz[i] = az * s;
    if (!isfinite(ax) || !isfinite(ay) || !isfinite(az)) atomicOr(status, kStatNonfinite);
  } else {
    double* p = part + (size_t)blockIdx.y * 3 * n;
    p[i] = ax;
    p[n + i] = ay;
    p[2 * n + i] = az;
  }
}

// Sum slice partials in slice order and apply G (and m_i for forces), for
// targets [t0, t1) of partials laid out with stride n per component: one
// thread per (target, component), its slices' loads in flight together.
__global__ void slice_reduce_kernel(int64_t n, int64_t t0, int64_t t1, int nslices,
                                    const double* __restrict__ part,
                                    const double* __restrict__ m, double G, int want_force,
                                    double* __restrict__ ox, double* __restrict__ oy,
                                    double* __restrict__ oz, int32_t* status) {
  const int64_t nt = t1 - t0;
  bool bad = false;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < 3 * nt;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(e / nt);
    const int64_t i = t0 + (e - k * nt);
    const double a = slice_sum(part + k * n + i, 3 * (size_t)n, nslices);
    const double sc = want_force ? G * m[i] : G;
    (k == 0 ? ox : k == 1 ? oy : oz)[i] = a * sc;
    bad |= !isfinite(a);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status, kStatNonfinite);
}

// Subset of targets (index list), all sources; one thread per (target,
// slice).  The self pair is skipped by index.  F64_EXACT keeps the reference
// op order with one slice; F64 / F32C use FMA + rsqrt in f64 (the subset
// serves as the f64 reference, so F32C is not used here).
__global__ void __launch_bounds__(kTile)
direct_targets_kernel(int64_t n, int64_t nt, const int64_t* __restrict__ tidx, int64_t slice_len,
                      const double* __restrict__ x, const double* __restrict__ y,
                      const double* __restrict__ z, const double* __restrict__ m, double G,
                      double eps2, int exact, double* __restrict__ part, double* __restrict__ ox,
                      double* __restrict__ oy, double* __restrict__ oz, int32_t* status) {
  __shared__ double4 tile[kTile];
  const int64_t t = blockIdx.x * (int64_t)kTile + threadIdx.x;
  const bool valid = t < nt;
  const int64_t i = valid ? tidx[t] : -1;
  const bool ok = valid && i >= 0 && i < n;
  if (valid && !ok) atomicOr(status, kStatOverflow);
  const double xi = ok ? x[i] : 0.0, yi = ok ? y[i] : 0.0, zi = ok ? z[i] : 0.0;
  const double mi = ok ? m[i] : 0.0;
  const double gm = xmul(G, mi);
  const int64_t lo = blockIdx.y * slice_len;
  const int64_t hi = min64(n, lo + slice_len);
  double ax = 0.0, ay = 0.0, az = 0.0;
  for (int64_t base = lo; base < hi; base += kTile) {
    const int64_t j = base + threadIdx.x;
    __syncthreads();
    tile[threadIdx.x] = j < hi ? make_double4(x[j], y[j], z[j], m[j]) : make_double4(0, 0, 0, 0);
    __syncthreads();
    const int cnt = (int)min64(kTile, hi - base);
    if (exact) {
      for (int k = 0; k < cnt; ++k) {
        if (base + k == i) continue;
        const double4 s = tile[k];
        const double rx = xsub(s.x, xi), ry = xsub(s.y, yi), rz = xsub(s.z, zi);
        const double s2 = xadd(xlen2(rx, ry, rz), eps2);
        const double sc = xdiv(xmul(gm, s.w), xmul(s2, xsqrt(s2)));
        ax = xadd(ax, xmul(rx, sc));
        ay = xadd(ay, xmul(ry, sc));
        az = xadd(az, xmul(rz, sc));
      }
    } else {
#pragma unroll 4
      for (int k = 0; k < cnt; ++k) {
        const double4 s = tile[k];
        const double rx = s.x - xi, ry = s.y - yi, rz = s.z - zi;
        const bool self = base + k == i;
        const double r2 = self ? 1.0 : fma(rx, rx, fma(ry, ry, fma(rz, rz, eps2)));
        const double inv = rsqrt(r2);
        const double w = self ? 0.0 : s.w * (inv * inv * inv);
        ax = fma(rx, w, ax);
        ay = fma(ry, w, ay);
        az = fma(rz, w, az);
      }
    }
  }
  if (!valid) return;
  if (exact) {  // a = F / m
    ox[t] = xdiv(ax, mi);
    oy[t] = xdiv(ay, mi);
    oz[t] = xdiv(az, mi);
    return;
  }
  double* pp = part + (size_t)blockIdx.y * 3 * nt;
  pp[t] = ax;
  pp[nt + t] = ay;
  pp[2 * nt + t] = az;
}

// Slices so that about two waves of 148 SMs x 2048 threads are resident;
// every slice spans whole tiles.
int64_t choose_slices(int64_t n) {
  const int64_t want_threads = 148LL * 2048;
  int64_t s = ceil_div(want_threads, ceil_div(n, kTile) * kTile);
  int64_t max_s = ceil_div(n, kTile);
  if (s > max_s) s = max_s;
  if (s < 1) s = 1;
  return s;
}

}  // namespace

int direct_eval(phys_ctx* c, const phys_params* p, bool want_force, double* ox, double* oy,
                double* oz) {
  const int64_t n = c->n;
  const double eps2 = p->eps * p->eps;
  PHYS_CUDA(c, cudaMemsetAsync(c->d_counter, 0, sizeof(unsigned long long), c->stream));
  if (!c->capturing) PHYS_CUDA(c, cudaEventRecord(c->ev[6], c->stream));
  // targets [t0, t1): all, or the share (t0 a multiple of kTile); the slices
  // follow from n alone, so a target's sum does not depend on the share
  int64_t t0 = 0, t1 = n;
  target_range(c, n, t0, t1);
  if (t0 % kTile) return fail(c, PHYS_ERR_ARG, "direct-sum share must start on a tile");
  const int64_t nt = t1 - t0;
  if (nt <= 0) {
    if (!c->capturing) PHYS_CUDA(c, cudaEventRecord(c->ev[7], c->stream));
    c->tm.interactions = 0;
    return PHYS_OK;
  }
  if (p->precision == PHYS_F64_EXACT) {
    PHYS_LAUNCH(c, direct_exact_kernel, (int)ceil_div(nt, kXT), kXBlock, 0, n, t0, t1, c->x, c->y,
                c->z, c->m, p->G, eps2, (int)want_force, ox, oy, oz, c->d_status);
  } else {
    const int64_t slices = choose_slices(n);
    const int64_t slice_len = ceil_div(ceil_div(n, slices), kTile) * kTile;
    const int64_t nsl = ceil_div(n, slice_len);
    double* part = nullptr;
    int st = PHYS_OK;
    if (nsl > 1) {
      part = (double*)ws_get(c, WS_DIRECT_PART, sizeof(double) * 3 * n * nsl, &st);
      if (st) return st;
    }
    dim3 grid((unsigned)ceil_div(nt, kTile), (unsigned)nsl);
    if (p->precision == PHYS_F64) {
      PHYS_LAUNCH(c, direct_f64_kernel, grid, kTile, 0, n, t0, t1, slice_len, c->x, c->y, c->z,
                  c->m, p->G, eps2, (int)want_force, ox, oy, oz, part, c->d_status);
    } else {
      float4* bh = (float4*)ws_get(c, WS_BODY_HI, sizeof(float4) * n, &st);
      if (st) return st;
      float4* bl = (float4*)ws_get(c, WS_BODY_LO, sizeof(float4) * n, &st);
      if (st) return st;
      int g = (int)min64(ceil_div(n, 256), 148 * 8);
      PHYS_LAUNCH(c, split_bodies_kernel, g, 256, 0, n, c->x, c->y, c->z, c->m, bh, bl,
                  c->d_status);
      PHYS_LAUNCH(c, direct_f32c_kernel, grid, kTile, 0, n, t0, t1, slice_len, bh, bl, c->m,
                  p->G, (float)eps2, (int)want_force, ox, oy, oz, part, c->d_status);
    }
    if (nsl > 1) {
      int g = (int)min64(ceil_div(3 * nt, 256), 148 * 8);
      PHYS_LAUNCH(c, slice_reduce_kernel, g, 256, 0, n, t0, t1, (int)nsl, part, c->m, p->G,
                  (int)want_force, ox, oy, oz, c->d_status);
    }
  }
  if (!c->capturing) PHYS_CUDA(c, cudaEventRecord(c->ev[7], c->stream));
  c->tm.interactions = (uint64_t)nt * (uint64_t)(n - 1);
  c->tm.bbox_ms = c->tm.keys_ms = c->tm.sort_ms = c->tm.tree_ms = 0.0;
  c->tm.nodes = 0;
  c->tm.max_depth = 0;
  return PHYS_OK;
}

// Sliced F64 / F32C direct sum on caller-owned device buffers and stream,
// with caller-provided scratch: `part` (3 * n * nslices doubles), `bh`/`bl`
// (n float4 each, F32C only) and the status word.  Launches the same kernels
// as direct_eval; allocates nothing.
cudaError_t direct_accel_launch_scratch(cudaStream_t s, int64_t n, const double* x,
                                        const double* y,
                                const double* z, const double* m, double G, double eps,
                                int precision, int64_t nslices, double* part, float4* bh,
                                float4* bl, int32_t* status, double* ox, double* oy,
                                double* oz) {
  const double eps2 = eps * eps;
  const int64_t slice_len = ceil_div(ceil_div(n, nslices), kTile) * kTile;
  const int64_t nsl = ceil_div(n, slice_len);
  dim3 grid((unsigned)ceil_div(n, kTile), (unsigned)nsl);
  const int g = (int)min64(ceil_div(n, 256), 148 * 8);
  if (precision == PHYS_F64) {
    direct_f64_kernel<<<grid, kTile, 0, s>>>(n, 0, n, slice_len, x, y, z, m, G, eps2, 0, ox, oy,
                                             oz, part, status);
  } else {
    split_bodies_kernel<<<g, 256, 0, s>>>(n, x, y, z, m, bh, bl, status);
    direct_f32c_kernel<<<grid, kTile, 0, s>>>(n, 0, n, slice_len, bh, bl, m, G, (float)eps2, 0,
                                              ox, oy, oz, part, status);
  }
  if (nsl > 1)
    slice_reduce_kernel<<<(int)min64(ceil_div(3 * n, 256), 148 * 8), 256, 0, s>>>(
        n, 0, n, (int)nsl, part, m, G, 0, ox, oy, oz, status);
  return cudaGetLastError();  // the launch error, if any (and clears it)
}

int direct_targets(phys_ctx* c, const phys_params* p, int64_t nt, const int64_t* d_tidx,
                   double* ox, double* oy, double* oz) {
  const int64_t n = c->n;
  const double eps2 = p->eps * p->eps;
  const bool exact = p->precision == PHYS_F64_EXACT;
  int64_t nsl = 1;
  if (!exact) {
    nsl = ceil_div(148LL * 2048, ceil_div(nt, kTile) * kTile);
    if (nsl > ceil_div(n, kTile)) nsl = ceil_div(n, kTile);
    if (nsl < 1) nsl = 1;
  }
  const int64_t slice_len = ceil_div(ceil_div(n, nsl), kTile) * kTile;
  nsl = ceil_div(n, slice_len);
  int st = PHYS_OK;
  double* part = (double*)ws_get(c, WS_DIRECT_PART, sizeof(double) * 3 * nt * nsl, &st);
  if (st) return st;
  dim3 grid((unsigned)ceil_div(nt, kTile), (unsigned)nsl);
  PHYS_LAUNCH(c, direct_targets_kernel, grid, kTile, 0, n, nt, d_tidx, slice_len, c->x, c->y,
              c->z, c->m, p->G, eps2, (int)exact, part, ox, oy, oz, c->d_status);
  if (!exact) {
    int g = (int)min64(ceil_div(3 * nt, 256), 148 * 8);
    PHYS_LAUNCH(c, slice_reduce_kernel, g, 256, 0, nt, 0, nt, (int)nsl, part, c->m, p->G, 0, ox,
                oy, oz, c->d_status);
  }
  return PHYS_OK;
}

}  // namespace phys
