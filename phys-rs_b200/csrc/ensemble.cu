// K8: batched ensemble of independent small systems (N <= 64 each).
//
// Each system is the reference's direct-sum Velocity-Verlet tick
// (gravity.rs:53-69 + integrators.rs:63-118) applied to its own bodies only.
// One persistent kernel runs a chunk of steps for every system: a group of G
// lanes (G = 8, 16 or 32; several groups per warp when G < 32) takes the next
// system from a global queue (systems in descending N, longest first), keeps
// the system's f64 state in shared memory for the whole chunk and returns it
// to HBM at the end.  Pair terms are F32C (double-float relative coordinates,
// two-sum accumulation) or F64_EXACT (reference op order, bit-identical).
// The host captures the chunk launches of a run in a CUDA graph; an
// autotuner picks G by timing a few steps of each candidate.
#include <algorithm>
#include <numeric>
#include <vector>

#include "common.cuh"

namespace phys {
namespace {

constexpr int kMaxSys = 64;        // bodies per system
constexpr int kEnsBlock = 64;      // threads per block

struct GroupSmem {
  double x[kMaxSys], y[kMaxSys], z[kMaxSys];
  double vx[kMaxSys], vy[kMaxSys], vz[kMaxSys];
  double ax[kMaxSys], ay[kMaxSys], az[kMaxSys];
  double pax[kMaxSys], pay[kMaxSys], paz[kMaxSys];
  double m[kMaxSys];
  // F32C staging, structure of arrays so that a float2 load gives two
  // consecutive bodies (slot N of an odd-N system is a massless pad far away)
  float hx[kMaxSys], hy[kMaxSys], hz[kMaxSys], hm[kMaxSys];  // hi parts, m (f32)
  float lx[kMaxSys], ly[kMaxSys], lz[kMaxSys];               // lo parts
};

template <int G>
__device__ __forceinline__ unsigned group_mask() {
  if constexpr (G == 32) {
    return 0xffffffffu;
  } else {
    const unsigned lane = threadIdx.x & 31;
    return ((1u << G) - 1u) << (lane & ~(unsigned)(G - 1));
  }
}

__device__ __forceinline__ void split_into(GroupSmem* S, int i) {
  split_df(S->x[i], S->hx[i], S->lx[i]);
  split_df(S->y[i], S->hy[i], S->ly[i]);
  split_df(S->z[i], S->hz[i], S->lz[i]);
  S->hm[i] = (float)S->m[i];
}

__device__ __forceinline__ void set_pad(GroupSmem* S, int i) {
  S->hx[i] = S->hy[i] = S->hz[i] = 1e15f;
  S->hm[i] = S->lx[i] = S->ly[i] = S->lz[i] = 0.f;
}

__device__ __forceinline__ float2 ld2(const float* p) {
  return *reinterpret_cast<const float2*>(p);
}

// F32C accelerations of the group's own targets, TC targets per pass.  Two
// sources per packed f32x2 operation (bodies j, j+1; an odd N reads the pad
// at slot N); partial sums of 16 sources folded into a (hi, lo) accumulator
// by two-sum.
template <int G, int TC>
__device__ void group_forces_f32c(GroupSmem* S, int N, int gl, double Gc, float eps2f) {
  const float2 e2 = make_float2(eps2f, eps2f);
  for (int i0 = gl; i0 < N; i0 += G * TC) {
    float2 nhx[TC], nhy[TC], nhz[TC], nlx[TC], nly[TC], nlz[TC], px[TC], py[TC], pz[TC];
    float hx[TC], hy[TC], hz[TC], lx[TC], ly[TC], lz[TC];
    int idx[TC];
#pragma unroll
    for (int t = 0; t < TC; ++t) {
      idx[t] = i0 + t * G;
      const int ii = idx[t] < N ? idx[t] : i0;
      nhx[t] = make_float2(-S->hx[ii], -S->hx[ii]);
      nhy[t] = make_float2(-S->hy[ii], -S->hy[ii]);
      nhz[t] = make_float2(-S->hz[ii], -S->hz[ii]);
      nlx[t] = make_float2(-S->lx[ii], -S->lx[ii]);
      nly[t] = make_float2(-S->ly[ii], -S->ly[ii]);
      nlz[t] = make_float2(-S->lz[ii], -S->lz[ii]);
      hx[t] = hy[t] = hz[t] = lx[t] = ly[t] = lz[t] = 0.f;
      px[t] = py[t] = pz[t] = make_float2(0.f, 0.f);
    }
    for (int j0 = 0; j0 < N; j0 += 16) {
      const int j1 = min(N, j0 + 16);
      for (int j = j0; j < j1; j += 2) {
        const float2 sx = ld2(S->hx + j), sy = ld2(S->hy + j), sz = ld2(S->hz + j);
        const float2 sm = ld2(S->hm + j);
        const float2 tx = ld2(S->lx + j), ty = ld2(S->ly + j), tz = ld2(S->lz + j);
#pragma unroll
        for (int t = 0; t < TC; ++t) {
          const float2 rx = __fadd2_rn(__fadd2_rn(sx, nhx[t]), __fadd2_rn(tx, nlx[t]));
          const float2 ry = __fadd2_rn(__fadd2_rn(sy, nhy[t]), __fadd2_rn(ty, nly[t]));
          const float2 rz = __fadd2_rn(__fadd2_rn(sz, nhz[t]), __fadd2_rn(tz, nlz[t]));
          const float2 r2 = __ffma2_rn(rx, rx, __ffma2_rn(ry, ry, __ffma2_rn(rz, rz, e2)));
          const float2 inv = make_float2(rsqrt_sfu(r2.x), rsqrt_sfu(r2.y));
          float2 w = __fmul2_rn(sm, __fmul2_rn(__fmul2_rn(inv, inv), inv));
          if (j == idx[t]) w.x = 0.f;       // self (i == j skipped, gravity.rs:56)
          if (j + 1 == idx[t]) w.y = 0.f;
          px[t] = __ffma2_rn(rx, w, px[t]);
          py[t] = __ffma2_rn(ry, w, py[t]);
          pz[t] = __ffma2_rn(rz, w, pz[t]);
        }
      }
#pragma unroll
      for (int t = 0; t < TC; ++t) {
        float s, e;
        two_sum(hx[t], px[t].x + px[t].y, s, e); hx[t] = s; lx[t] += e;
        two_sum(hy[t], py[t].x + py[t].y, s, e); hy[t] = s; ly[t] += e;
        two_sum(hz[t], pz[t].x + pz[t].y, s, e); hz[t] = s; lz[t] += e;
        px[t] = py[t] = pz[t] = make_float2(0.f, 0.f);
      }
    }
#pragma unroll
    for (int t = 0; t < TC; ++t) {
      if (idx[t] < N) {
        S->ax[idx[t]] = Gc * ((double)hx[t] + (double)lx[t]);
        S->ay[idx[t]] = Gc * ((double)hy[t] + (double)ly[t]);
        S->az[idx[t]] = Gc * ((double)hz[t] + (double)lz[t]);
      }
    }
  }
}

// Accelerations of the group's own targets (i = gl, gl+G, ...) into S->a.
template <int G, bool kExact>
__device__ void group_forces(GroupSmem* S, int N, int gl, double Gc, double eps2) {
  if (kExact) {
    for (int i = gl; i < N; i += G) {
      const double xi = S->x[i], yi = S->y[i], zi = S->z[i], mi = S->m[i];
      const double gm = xmul(Gc, mi);
      double fx = 0.0, fy = 0.0, fz = 0.0;
      for (int j = 0; j < N; ++j) {
        if (j == i) continue;
        const double rx = xsub(S->x[j], xi), ry = xsub(S->y[j], yi), rz = xsub(S->z[j], zi);
        const double s2 = xadd(xlen2(rx, ry, rz), eps2);
        const double sc = xdiv(xmul(gm, S->m[j]), xmul(s2, xsqrt(s2)));
        fx = xadd(fx, xmul(rx, sc));
        fy = xadd(fy, xmul(ry, sc));
        fz = xadd(fz, xmul(rz, sc));
      }
      S->ax[i] = xdiv(fx, mi);  // a = F / m (integrators.rs:115)
      S->ay[i] = xdiv(fy, mi);
      S->az[i] = xdiv(fz, mi);
    }
    return;
  }
  // targets per lane for this system: 1, 2 or (up to 8 in passes of) 4
  const float eps2f = (float)eps2;
  const int tpl = (N + G - 1) / G;
  if (tpl <= 1)
    group_forces_f32c<G, 1>(S, N, gl, Gc, eps2f);
  else if (tpl == 2 || G == 32)
    group_forces_f32c<G, 2>(S, N, gl, Gc, eps2f);
  else
    group_forces_f32c<G, 4>(S, N, gl, Gc, eps2f);
}

template <int G, bool kExact>
__global__ void __launch_bounds__(kEnsBlock)
ensemble_kernel(int nsys, const int32_t* __restrict__ order, const int64_t* __restrict__ off,
                double* __restrict__ x, double* __restrict__ y, double* __restrict__ z,
                double* __restrict__ vx, double* __restrict__ vy, double* __restrict__ vz,
                double* __restrict__ ax, double* __restrict__ ay, double* __restrict__ az,
                const double* __restrict__ m, double Gc, double eps2, double dt, int nsteps,
                int need_accel, int* queue, int32_t* status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int gid = threadIdx.x / G, gl = threadIdx.x % G;
  GroupSmem* S = reinterpret_cast<GroupSmem*>(smem_raw) + gid;
  const unsigned gm = group_mask<G>();
  const double h2 = xmul(xmul(0.5, dt), dt), hdt = xmul(0.5, dt);
  for (;;) {
    int s = 0;
    if (gl == 0) s = atomicAdd(queue, 1);
    s = __shfl_sync(gm, s, 0, G);
    if (s >= nsys) break;
    const int sys = order[s];
    const int64_t b = off[sys];
    const int N = (int)(off[sys + 1] - b);
    if (N > kMaxSys || N < 0) {
      if (gl == 0) atomicOr(status, kStatOverflow);
      continue;
    }
    for (int i = gl; i < N; i += G) {
      S->x[i] = x[b + i];
      S->y[i] = y[b + i];
      S->z[i] = z[b + i];
      S->vx[i] = vx[b + i];
      S->vy[i] = vy[b + i];
      S->vz[i] = vz[b + i];
      S->ax[i] = ax[b + i];
      S->ay[i] = ay[b + i];
      S->az[i] = az[b + i];
      S->m[i] = m[b + i];
      split_into(S, i);
    }
    if ((N & 1) && gl == 0) set_pad(S, N);  // N <= kMaxSys - 1 here
    __syncwarp(gm);
    if (need_accel && N >= 2) group_forces<G, kExact>(S, N, gl, Gc, eps2);
    if (need_accel && N < 2)
      for (int i = gl; i < N; i += G) S->ax[i] = S->ay[i] = S->az[i] = 0.0;
    __syncwarp(gm);
    for (int st = 0; st < nsteps; ++st) {
      // velocity_verlet_position_system: prev = a; x += v dt + a dt^2/2
      for (int i = gl; i < N; i += G) {
        const double a0 = S->ax[i], a1 = S->ay[i], a2 = S->az[i];
        S->pax[i] = a0;
        S->pay[i] = a1;
        S->paz[i] = a2;
        S->x[i] = xadd(S->x[i], xadd(xmul(S->vx[i], dt), xmul(a0, h2)));
        S->y[i] = xadd(S->y[i], xadd(xmul(S->vy[i], dt), xmul(a1, h2)));
        S->z[i] = xadd(S->z[i], xadd(xmul(S->vz[i], dt), xmul(a2, h2)));
        split_into(S, i);
      }
      __syncwarp(gm);
      if (N >= 2) group_forces<G, kExact>(S, N, gl, Gc, eps2);
      __syncwarp(gm);
      // velocity_verlet_velocity_system: v += (prev + a) dt/2
      for (int i = gl; i < N; i += G) {
        S->vx[i] = xadd(S->vx[i], xmul(xadd(S->pax[i], S->ax[i]), hdt));
        S->vy[i] = xadd(S->vy[i], xmul(xadd(S->pay[i], S->ay[i]), hdt));
        S->vz[i] = xadd(S->vz[i], xmul(xadd(S->paz[i], S->az[i]), hdt));
      }
      __syncwarp(gm);
    }
    bool bad = false;
    for (int i = gl; i < N; i += G) {
      x[b + i] = S->x[i];
      y[b + i] = S->y[i];
      z[b + i] = S->z[i];
      vx[b + i] = S->vx[i];
      vy[b + i] = S->vy[i];
      vz[b + i] = S->vz[i];
      ax[b + i] = S->ax[i];
      ay[b + i] = S->ay[i];
      az[b + i] = S->az[i];
      bad |= !isfinite(S->x[i]) || !isfinite(S->vx[i]) || !isfinite(S->ax[i]);
    }
    if (bad) atomicOr(status, kStatNonfinite);
    __syncwarp(gm);
  }
}

using EnsKernel = void (*)(int, const int32_t*, const int64_t*, double*, double*, double*,
                           double*, double*, double*, double*, double*, double*, const double*,
                           double, double, double, int, int, int*, int32_t*);

EnsKernel pick(int G, bool exact) {
  if (exact) {
    switch (G) {
      case 8: return ensemble_kernel<8, true>;
      case 16: return ensemble_kernel<16, true>;
      default: return ensemble_kernel<32, true>;
    }
  }
  switch (G) {
    case 8: return ensemble_kernel<8, false>;
    case 16: return ensemble_kernel<16, false>;
    default: return ensemble_kernel<32, false>;
  }
}

struct EnsView {
  double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az, *m;
};

EnsView view(phys_ctx* c) {
  double* b = reinterpret_cast<double*>(c->ws[WS_ENS0].p);
  const int64_t n = c->ens_nbody;
  return EnsView{b, b + n, b + 2 * n, b + 3 * n, b + 4 * n, b + 5 * n, b + 6 * n, b + 7 * n,
                 b + 8 * n, b + 9 * n};
}

struct LaunchCfg {
  EnsKernel k;
  size_t smem;
  int64_t grid;
};

// Kernel attributes and the persistent grid size (queried outside capture).
int prepare(phys_ctx* c, const phys_params* p, int G, LaunchCfg* cfg) {
  const bool exact = p->precision == PHYS_F64_EXACT;
  cfg->k = pick(G, exact);
  cfg->smem = sizeof(GroupSmem) * (kEnsBlock / G);
  PHYS_CUDA(c, cudaFuncSetAttribute(cfg->k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)cfg->smem));
  int per_sm = 0;
  PHYS_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cfg->k, kEnsBlock,
                                                             cfg->smem));
  int sms = 148;
  PHYS_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  const int groups_per_block = kEnsBlock / G;
  cfg->grid = std::min<int64_t>((int64_t)std::max(per_sm, 1) * sms,
                                ceil_div(c->ens_nsys, groups_per_block));
  return PHYS_OK;
}

// Enqueue one run of `nsteps` steps in chunks of `chunk` steps (one launch each).
int enqueue_run(phys_ctx* c, const phys_params* p, const LaunchCfg& cfg, double dt,
                int64_t nsteps, int64_t chunk, bool need_accel_first) {
  EnsView v = view(c);
  int* queue = reinterpret_cast<int*>(c->ws[WS_ENS3].p);
  const double eps2 = p->eps * p->eps;
  int64_t done = 0;
  int ci = 0;
  bool need = need_accel_first;
  do {
    const int64_t k_steps = std::min<int64_t>(chunk, nsteps - done);
    PHYS_CUDA(c, cudaMemsetAsync(queue + ci, 0, sizeof(int), c->stream));
    cfg.k<<<(unsigned)cfg.grid, kEnsBlock, cfg.smem, c->stream>>>(
        (int)c->ens_nsys, reinterpret_cast<const int32_t*>(c->ws[WS_ENS2].p),
        reinterpret_cast<const int64_t*>(c->ws[WS_ENS1].p), v.x, v.y, v.z, v.vx, v.vy, v.vz, v.ax,
        v.ay, v.az, v.m, p->G, eps2, dt, (int)k_steps, need ? 1 : 0, queue + ci, c->d_status);
    c->launches++;
    PHYS_TRY(check_launch(c, "ensemble_kernel"));
    need = false;
    done += k_steps;
    ci = (ci + 1) & 1023;
  } while (done < nsteps);
  return PHYS_OK;
}

}  // namespace

int ensemble_load(phys_ctx* c, int64_t nsys, const int64_t* off, const double* x, const double* y,
                  const double* z, const double* vx, const double* vy, const double* vz,
                  const double* m) {
  const int64_t n = off[nsys];
  if (off[0] != 0) return fail(c, PHYS_ERR_ARG, "offsets[0] must be 0");
  std::vector<int32_t> order(nsys);
  for (int64_t s = 0; s < nsys; ++s) {
    const int64_t k = off[s + 1] - off[s];
    if (k < 0 || k > kMaxSys)
      return fail(c, PHYS_ERR_ARG, "system %lld has %lld bodies (1..%d supported)", (long long)s,
                  (long long)k, kMaxSys);
    order[s] = (int32_t)s;
  }
  // longest first: the tail of the persistent queue holds the cheapest systems
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
    return (off[a + 1] - off[a]) > (off[b + 1] - off[b]);
  });
  int st = PHYS_OK;
  double* base = (double*)ws_get(c, WS_ENS0, sizeof(double) * 10 * (n > 0 ? n : 1), &st);
  if (st) return st;
  ws_get(c, WS_ENS1, sizeof(int64_t) * (nsys + 1), &st);
  if (st) return st;
  ws_get(c, WS_ENS2, sizeof(int32_t) * (nsys > 0 ? nsys : 1), &st);
  if (st) return st;
  ws_get(c, WS_ENS3, sizeof(int) * 1024, &st);
  if (st) return st;
  c->ens_nsys = nsys;
  c->ens_nbody = n;
  c->ens_accel_valid = false;
  EnsView v = view(c);
  const double* src[7] = {x, y, z, vx, vy, vz, m};
  double* dst[7] = {v.x, v.y, v.z, v.vx, v.vy, v.vz, v.m};
  for (int k = 0; k < 7; ++k) {
    if (src[k])
      PHYS_CUDA(c, cudaMemcpyAsync(dst[k], src[k], sizeof(double) * n, cudaMemcpyHostToDevice,
                                   c->stream));
    else
      PHYS_CUDA(c, cudaMemsetAsync(dst[k], 0, sizeof(double) * n, c->stream));
  }
  PHYS_CUDA(c, cudaMemsetAsync(v.ax, 0, sizeof(double) * 3 * n, c->stream));
  PHYS_CUDA(c, cudaMemcpyAsync(c->ws[WS_ENS1].p, off, sizeof(int64_t) * (nsys + 1),
                               cudaMemcpyHostToDevice, c->stream));
  PHYS_CUDA(c, cudaMemcpyAsync(c->ws[WS_ENS2].p, order.data(), sizeof(int32_t) * nsys,
                               cudaMemcpyHostToDevice, c->stream));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  (void)base;
  return PHYS_OK;
}

int ensemble_run(phys_ctx* c, const phys_params* p, double dt, int64_t nsteps, int G,
                 int64_t chunk) {
  if (c->ens_nsys <= 0) return fail(c, PHYS_ERR_STATE, "no ensemble loaded");
  if (G != 8 && G != 16 && G != 32) return fail(c, PHYS_ERR_ARG, "group size must be 8, 16 or 32");
  if (chunk <= 0) chunk = nsteps > 0 ? nsteps : 1;
  LaunchCfg cfg;
  PHYS_TRY(prepare(c, p, G, &cfg));
  // Capture the chunk launches of this run in a CUDA graph, then replay it.
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  PHYS_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int st = enqueue_run(c, p, cfg, dt, nsteps, chunk, !c->ens_accel_valid);
  cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
  if (st) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
  PHYS_CUDA(c, cudaEventRecord(c->ev[6], c->stream));
  e = cudaGraphLaunch(exec, c->stream);
  if (e == cudaSuccess) e = cudaEventRecord(c->ev[7], c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaGraphExecDestroy(exec);
  if (e != cudaSuccess) return cuda_fail(c, e, "ensemble graph launch");
  c->ens_accel_valid = true;
  return PHYS_OK;
}

int ensemble_download(phys_ctx* c, double* x, double* y, double* z, double* vx, double* vy,
                      double* vz, double* ax, double* ay, double* az) {
  EnsView v = view(c);
  const int64_t n = c->ens_nbody;
  double* dst[9] = {x, y, z, vx, vy, vz, ax, ay, az};
  double* src[9] = {v.x, v.y, v.z, v.vx, v.vy, v.vz, v.ax, v.ay, v.az};
  for (int k = 0; k < 9; ++k)
    if (dst[k])
      PHYS_CUDA(c, cudaMemcpyAsync(dst[k], src[k], sizeof(double) * n, cudaMemcpyDeviceToHost,
                                   c->stream));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  return PHYS_OK;
}

// Times `probe_steps` steps for each group size from the same starting state
// (saved and restored around the probes) and keeps the fastest.
int ensemble_autotune(phys_ctx* c, const phys_params* p, double dt, int64_t probe_steps,
                      int32_t* best, double* ms3) {
  if (c->ens_nsys <= 0) return fail(c, PHYS_ERR_STATE, "no ensemble loaded");
  const int64_t n = c->ens_nbody;
  int st = PHYS_OK;
  double* save = (double*)ws_get(c, WS_ENS4, sizeof(double) * 9 * (n > 0 ? n : 1), &st);
  if (st) return st;
  EnsView v = view(c);
  const bool valid0 = c->ens_accel_valid;
  PHYS_CUDA(c, cudaMemcpyAsync(save, v.x, sizeof(double) * 9 * n, cudaMemcpyDeviceToDevice,
                               c->stream));
  const int cand[3] = {8, 16, 32};
  double best_ms = 1e300;
  int best_g = 32;
  for (int k = 0; k < 3; ++k) {
    c->ens_accel_valid = true;  // time steps only; the force of the start state is reused
    PHYS_TRY(ensemble_run(c, p, dt, probe_steps, cand[k], probe_steps));
    float ms = 0.f;
    PHYS_CUDA(c, cudaEventElapsedTime(&ms, c->ev[6], c->ev[7]));
    if (ms3) ms3[k] = ms;
    if (ms < best_ms) {
      best_ms = ms;
      best_g = cand[k];
    }
    PHYS_CUDA(c, cudaMemcpyAsync(v.x, save, sizeof(double) * 9 * n, cudaMemcpyDeviceToDevice,
                                 c->stream));
  }
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  c->ens_accel_valid = valid0;
  c->ens_group = best_g;
  if (best) *best = best_g;
  return PHYS_OK;
}

}  // namespace phys
