// K10: f64 energy / momentum diagnostics (src/physics/energy.rs:21-56,
// integrators.rs:123-129) and the FP32 / FP64 pipe-peak probe used as
// roofline denominators.
#include "common.cuh"

namespace phys {
namespace {

constexpr int kBlock = 256;
constexpr int kTile = 128;

// Neumaier-compensated f64 accumulator.
struct CSum {
  double s = 0.0, c = 0.0;
  __device__ void add(double v) {
    const double t = s + v;
    if (fabs(s) >= fabs(v))
      c += (s - t) + v;
    else
      c += (v - t) + s;
    s = t;
  }
  __device__ double get() const { return s + c; }
};

// Per-block compensated partials of KE = sum 0.5*m*|v|^2 and p = sum m*v.
__global__ void __launch_bounds__(kBlock)
ke_mom_kernel(int64_t n, const double* __restrict__ vx, const double* __restrict__ vy,
              const double* __restrict__ vz, const double* __restrict__ m,
              double* __restrict__ part) {
  __shared__ double sh[4][kBlock];
  CSum ke, px, py, pz;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double a = vx[i], b = vy[i], c = vz[i], mm = m[i];
    ke.add(xmul(xmul(0.5, mm), xlen2(a, b, c)));  // 0.5 * m * |v|^2 (energy.rs:27)
    px.add(xmul(a, mm));                          // p = v * m (integrators.rs:127)
    py.add(xmul(b, mm));
    pz.add(xmul(c, mm));
  }
  sh[0][threadIdx.x] = ke.get();
  sh[1][threadIdx.x] = px.get();
  sh[2][threadIdx.x] = py.get();
  sh[3][threadIdx.x] = pz.get();
  __syncthreads();
  for (int s = kBlock / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; ++k) part[blockIdx.x * 4 + k] = sh[k][0];
}

// Unsoftened potential -sum_{i<j} G m_i m_j / r, r^2 == 0 skipped
// (energy.rs:43-54): each target i sums its pairs j > i over shared tiles.
__global__ void __launch_bounds__(kTile)
pe_kernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
          const double* __restrict__ z, const double* __restrict__ m, double G,
          double* __restrict__ part) {
  __shared__ double4 tile[kTile];
  __shared__ double red[kTile];
  const int64_t i = blockIdx.x * (int64_t)kTile + threadIdx.x;
  const bool valid = i < n;
  const double xi = valid ? x[i] : 0, yi = valid ? y[i] : 0, zi = valid ? z[i] : 0;
  const double gmi = valid ? xmul(G, m[i]) : 0.0;
  CSum acc;
  const int64_t start = blockIdx.x * (int64_t)kTile;
  for (int64_t base = start; base < n; base += kTile) {
    const int64_t j = base + threadIdx.x;
    __syncthreads();
    tile[threadIdx.x] = j < n ? make_double4(x[j], y[j], z[j], m[j]) : make_double4(0, 0, 0, 0);
    __syncthreads();
    const int cnt = (int)min64(kTile, n - base);
    for (int k = 0; k < cnt; ++k) {
      if (base + k <= i) continue;
      const double4 s = tile[k];
      const double dx = xsub(s.x, xi), dy = xsub(s.y, yi), dz = xsub(s.z, zi);
      const double r2 = xlen2(dx, dy, dz);
      if (r2 > 0.0) acc.add(-xdiv(xmul(gmi, s.w), xsqrt(r2)));
    }
  }
  red[threadIdx.x] = valid ? acc.get() : 0.0;
  __syncthreads();
  for (int s = kTile / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void final_kernel(int nke, int npe, const double* __restrict__ ke_part,
                             const double* __restrict__ pe_part, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  CSum ke, px, py, pz, pe;
  for (int b = 0; b < nke; ++b) {
    ke.add(ke_part[b * 4]);
    px.add(ke_part[b * 4 + 1]);
    py.add(ke_part[b * 4 + 2]);
    pz.add(ke_part[b * 4 + 3]);
  }
  for (int b = 0; b < npe; ++b) pe.add(pe_part[b]);
  out[0] = ke.get();
  out[1] = pe.get();
  out[2] = px.get();
  out[3] = py.get();
  out[4] = pz.get();
}

// FMA-rate probes: 8 independent chains per thread.
__global__ void ffma_probe(int iters, float seed, float* out) {
  float a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed + k * 1e-3f + threadIdx.x * 1e-7f;
  const float b = 0.999999f, c = 1e-7f;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = fmaf(a[k], b, c);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  if (s == 12345.678f) out[0] = s;  // keeps the chains live
}

__global__ void ffma2_probe(int iters, float seed, float* out) {
  float2 a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = make_float2(seed + k * 1e-3f, seed - k * 1e-3f + threadIdx.x * 1e-7f);
  const float2 b = make_float2(0.999999f, 0.999998f), c = make_float2(1e-7f, 2e-7f);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = __ffma2_rn(a[k], b, c);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k].x + a[k].y;
  if (s == 12345.678f) out[0] = s;
}

__global__ void dfma_probe(int iters, double seed, double* out) {
  double a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed + k * 1e-3 + threadIdx.x * 1e-9;
  const double b = 0.999999999, c = 1e-12;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  if (s == 12345.678) out[0] = s;
}

}  // namespace

int diagnostics(phys_ctx* c, double G, double* out5) {
  const int64_t n = c->n;
  const int nke = 148 * 2;
  const int npe = (int)ceil_div(n, kTile);
  int st = PHYS_OK;
  double* buf = (double*)ws_get(c, WS_DIRECT_PART, sizeof(double) * (4 * nke + npe + 8), &st);
  if (st) return st;
  double* ke_part = buf;
  double* pe_part = buf + 4 * nke;
  double* out = pe_part + npe;
  PHYS_LAUNCH(c, ke_mom_kernel, nke, kBlock, 0, n, c->vx, c->vy, c->vz, c->m, ke_part);
  PHYS_LAUNCH(c, pe_kernel, npe, kTile, 0, n, c->x, c->y, c->z, c->m, G, pe_part);
  PHYS_LAUNCH(c, final_kernel, 1, 32, 0, nke, npe, ke_part, pe_part, out);
  PHYS_CUDA(c, cudaMemcpyAsync(out5, out, sizeof(double) * 5, cudaMemcpyDeviceToHost, c->stream));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  return PHYS_OK;
}

int probe_peaks(phys_ctx* c, double* fp32, double* fp32x2, double* fp64) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  const int blocks = sms * 8, threads = 256;
  int st = PHYS_OK;
  void* scratch = ws_get(c, WS_ADJ4, 64, &st);
  if (st) return st;
  cudaEvent_t e0 = c->ev[8], e1 = c->ev[9];
  float ms = 0.f;
  // warm-up then timed
  const int it32 = 1 << 14, it64 = 1 << 12;
  PHYS_LAUNCH(c, ffma_probe, blocks, threads, 0, 256, 1.0f, (float*)scratch);
  PHYS_CUDA(c, cudaEventRecord(e0, c->stream));
  PHYS_LAUNCH(c, ffma_probe, blocks, threads, 0, it32, 1.0f, (float*)scratch);
  PHYS_CUDA(c, cudaEventRecord(e1, c->stream));
  PHYS_CUDA(c, cudaEventSynchronize(e1));
  PHYS_CUDA(c, cudaEventElapsedTime(&ms, e0, e1));
  *fp32 = 2.0 * 8.0 * it32 * (double)blocks * threads / (ms * 1e-3) / 1e12;
  PHYS_LAUNCH(c, ffma2_probe, blocks, threads, 0, 256, 1.0f, (float*)scratch);
  PHYS_CUDA(c, cudaEventRecord(e0, c->stream));
  PHYS_LAUNCH(c, ffma2_probe, blocks, threads, 0, it32, 1.0f, (float*)scratch);
  PHYS_CUDA(c, cudaEventRecord(e1, c->stream));
  PHYS_CUDA(c, cudaEventSynchronize(e1));
  PHYS_CUDA(c, cudaEventElapsedTime(&ms, e0, e1));
  *fp32x2 = 4.0 * 8.0 * it32 * (double)blocks * threads / (ms * 1e-3) / 1e12;
  PHYS_LAUNCH(c, dfma_probe, blocks, threads, 0, 64, 1.0, (double*)scratch);
  PHYS_CUDA(c, cudaEventRecord(e0, c->stream));
  PHYS_LAUNCH(c, dfma_probe, blocks, threads, 0, it64, 1.0, (double*)scratch);
  PHYS_CUDA(c, cudaEventRecord(e1, c->stream));
  PHYS_CUDA(c, cudaEventSynchronize(e1));
  PHYS_CUDA(c, cudaEventElapsedTime(&ms, e0, e1));
  *fp64 = 2.0 * 8.0 * it64 * (double)blocks * threads / (ms * 1e-3) / 1e12;
  return PHYS_OK;
}

}  // namespace phys
