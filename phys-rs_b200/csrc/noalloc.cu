// Direct-sum accelerations that allocate no memory: for callers that must
// not allocate device memory once they are running.  An engine's fixed-step
// loop, for instance, may set up all of its buffers at start-up and forbid
// cudaMalloc / cudaFree afterwards, because those calls can synchronise the
// whole device and stall a tick; a host application may also hand this
// library only memory from its own pool.  Such a caller passes its own device
// buffers for inputs and outputs, and the scratch this computation needs (the
// F32C double-float body split, the per-slice partial sums and a status word)
// lives in one fixed array in device memory, below.
//
// The array is file-scope `static __device__`: every GPU that loads the
// library holds it (about 7.3 MiB) until the process exits.  Its size fixes
// the maximum problem size, kMaxBodies.  All calls share it and it keeps the
// previous call's contents, so calls whose work overlaps on the GPU (two
// streams, or two host threads) race on it; callers must order them.
// The array's device address is looked up once per device and kept for the
// life of the process; cudaDeviceReset destroys the device's context, and
// with it the array at that address, so a process that resets a device must
// not call this entry point on that device again.
#include <mutex>

#include "common.cuh"

namespace {

constexpr int64_t kMaxBodies = 32768;
constexpr int64_t kMaxSlices = 8;
constexpr size_t kStatusBytes = 256;
constexpr size_t kSplitBytes = 2 * sizeof(float4) * kMaxBodies;        // F32C body split
constexpr size_t kPartBytes = 3 * sizeof(double) * kMaxBodies * kMaxSlices;  // slice partials
constexpr size_t kScratchBytes = kStatusBytes + kSplitBytes + kPartBytes;

// In host code this name is only a stand-in for the device symbol: its
// device address comes from cudaGetSymbolAddress (per device, below).
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_dev[kMaxDevices] = {};

void set_err(char* buf, size_t len, const char* fmt, ...) {
  if (!buf || len == 0) return;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, len, fmt, ap);
  va_end(ap);
}

}  // namespace

extern "C" int phys_direct_accel_noalloc(int64_t n, const double* x, const double* y,
                                         const double* z, const double* m, double G, double eps,
                                         int32_t precision, double* ax, double* ay, double* az,
                                         void* stream, char* errbuf, size_t errlen) {
  if (n < 0 || n > kMaxBodies) {
    set_err(errbuf, errlen,
            "phys_direct_accel_noalloc: n = %lld is outside 0..%lld, the bodies its fixed "
            "scratch area holds",
            (long long)n, (long long)kMaxBodies);
    return PHYS_ERR_ARG;
  }
  if (precision != PHYS_F64 && precision != PHYS_F32C) {
    set_err(errbuf, errlen, "phys_direct_accel_noalloc: precision must be PHYS_F64 or PHYS_F32C");
    return PHYS_ERR_ARG;
  }
  if (n > 0 && (!x || !y || !z || !m || !ax || !ay || !az)) {
    set_err(errbuf, errlen, "phys_direct_accel_noalloc: device pointers must not be NULL");
    return PHYS_ERR_ARG;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n < 2) {  // no pairs (gravity.rs:49-51): zero accelerations
    cudaError_t e = cudaSuccess;
    for (double* o : {ax, ay, az})
      if (n > 0 && e == cudaSuccess) e = cudaMemsetAsync(o, 0, sizeof(double) * n, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_err(errbuf, errlen, "phys_direct_accel_noalloc: %s", cudaGetErrorString(e));
      return PHYS_ERR_CUDA;
    }
    return PHYS_OK;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_err(errbuf, errlen, "phys_direct_accel_noalloc: no usable current device");
    return PHYS_ERR_CUDA;
  }
  // Set-up, once per device, with that device current: the device address
  // of the scratch array.  The first call on each device does this.
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_dev[dev]) {
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_scratch);
      if (e != cudaSuccess || !ptr) {
        cudaGetLastError();
        set_err(errbuf, errlen, "phys_direct_accel_noalloc: cudaGetSymbolAddress failed: %s",
                cudaGetErrorString(e));
        return PHYS_ERR_CUDA;
      }
      g_scratch_dev[dev] = ptr;
    }
    base = static_cast<unsigned char*>(g_scratch_dev[dev]);
  }
  int32_t* status = reinterpret_cast<int32_t*>(base);
  float4* bh = reinterpret_cast<float4*>(base + kStatusBytes);
  float4* bl = bh + kMaxBodies;
  double* part = reinterpret_cast<double*>(base + kStatusBytes + kSplitBytes);
  // Slices: enough (target, slice) threads to cover the SMs, at most kMaxSlices.
  int64_t nslices = phys::ceil_div(148LL * 2048, phys::ceil_div(n, 128) * 128);
  if (nslices > kMaxSlices) nslices = kMaxSlices;
  if (nslices > phys::ceil_div(n, 128)) nslices = phys::ceil_div(n, 128);
  if (nslices < 1) nslices = 1;
  // The status word must start at zero; the split and partial areas are
  // fully overwritten before they are read.
  e = cudaMemsetAsync(status, 0, sizeof(int32_t), s);
  if (e != cudaSuccess) {
    set_err(errbuf, errlen, "phys_direct_accel_noalloc: %s", cudaGetErrorString(e));
    return PHYS_ERR_CUDA;
  }
  e = phys::direct_accel_launch_scratch(s, n, x, y, z, m, G, eps, precision, nslices, part, bh,
                                         bl, status, ax, ay, az);
  if (e != cudaSuccess) {
    set_err(errbuf, errlen, "phys_direct_accel_noalloc: launch failed: %s (%s)",
            cudaGetErrorName(e), cudaGetErrorString(e));
    return PHYS_ERR_CUDA;
  }
  int32_t hs = 0;
  e = cudaMemcpyAsync(&hs, status, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_err(errbuf, errlen, "phys_direct_accel_noalloc: %s", cudaGetErrorString(e));
    return PHYS_ERR_CUDA;
  }
  if (hs & phys::kStatNonfinite) {
    set_err(errbuf, errlen, "phys_direct_accel_noalloc: non-finite input or result");
    return PHYS_ERR_NONFINITE;
  }
  return PHYS_OK;
}
