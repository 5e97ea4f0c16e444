// Internal declarations shared by the libphysgpu translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/physgpu.h"

namespace phys {

constexpr int kMaxDepth = 40;            // gravity_tree.rs:30
constexpr double kMinNodeSize = 1e-8;    // gravity_tree.rs:34
constexpr int kMaxLevels = kMaxDepth + 1;
constexpr int kMaxLeafCap = 16;

// Device status word bits (reduced into ctx->d_status by kernels).
constexpr int kStatNonfinite = 1;
constexpr int kStatTimeout = 2;
constexpr int kStatOverflow = 4;

// Growable device buffer (bytes).  Memory is released by the context.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// Per-tree constants written on the device by the bbox kernel and read by
// every later kernel of the force evaluation (no host round trip).
struct TreeHeader {
  double center[3];
  double half;                   // root half size (gravity_tree.rs:316)
  double theta2;                 // theta * theta
  double s2[kMaxLevels];         // (2 h_d)^2 per depth, h_d = half * 0.5^d by repeated halving
  int32_t dstar;                 // guard depth: first d with d >= 40 or h_d < 1e-8
  int32_t nonfinite;             // any non-finite input coordinate
  int64_t nnodes;                // nodes of the current tree
  double min_mass;               // smallest body mass
};

}  // namespace phys

struct phys_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  // second stream for work that runs beside the main stream's kernels; it
  // forks from and joins back into `stream` within one library call
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  // copy stream of phys_verlet_tick_host: the positions go back to the host
  // while the force pass runs (copy_x: page-locked host arrays, or null)
  cudaStream_t copy = nullptr;
  cudaEvent_t copy_fork = nullptr, copy_done = nullptr;
  double* copy_x[3] = {nullptr, nullptr, nullptr};
  std::string err;
  uint64_t launches = 0;
  phys_timings tm{};

  // ---- body state (SoA, caller order) ----
  int64_t n = 0, cap = 0;
  double *x = nullptr, *y = nullptr, *z = nullptr;
  double *vx = nullptr, *vy = nullptr, *vz = nullptr;
  double *m = nullptr;
  double *ax = nullptr, *ay = nullptr, *az = nullptr;     // Acceleration
  double *pax = nullptr, *pay = nullptr, *paz = nullptr;  // PreviousAcceleration
  double *fx = nullptr, *fy = nullptr, *fz = nullptr;     // gravity force scratch
  bool accel_valid = false;
  phys_nfw_halo halo{};   // NFW phantom halo added to accelerations when halo_on
  bool halo_on = false;
  // (Sector, LocalPosition) state kept on the device (sector_mode): sec =
  // sx | sy | sz (int64), loc = lx | ly | lz, each sec_cap long; x/y/z then
  // hold the flattened positions of the last force pass.
  int32_t* d_shift = nullptr;  // device flag: a body changed sector in the last normalisation
  bool sector_mode = false;
  double sector_size = 0.0;
  int64_t* sec = nullptr;
  double* loc = nullptr;
  int64_t sec_cap = 0;
  phys_params accel_params{};
  bool last_eval_bh = false;   // the interaction count lives in d_counter
  bool last_eval_group = false;  // ev[10], ev[11] bracket the group walk's list evaluation

  // ---- target shares (one system split over GPUs) ----
  // While share_hi >= 0 an evaluation computes only the targets [share_lo,
  // share_hi): body indices for the direct sum, sorted (key-order) positions
  // for Barnes-Hut.  share_world > 0 after phys_gravity_accel_share until the
  // matching phys_gravity_accel_unshare (any other evaluation or a new
  // upload clears it); share_perm is the sorted-to-index map of that
  // evaluation's tree (the last tree's while evaluating; then a copy in a
  // workspace slot that only the share entry points use).
  int64_t share_lo = 0, share_hi = -1;
  int32_t share_world = 0;
  const uint32_t* share_perm = nullptr;
  phys_params share_params{};

  // ---- batched ensemble (independent small systems) ----
  int64_t ens_nsys = 0, ens_nbody = 0;
  bool ens_accel_valid = false;
  int ens_group = 0;           // autotuned configuration code (0: not tuned)
  int64_t ens_n32 = 0, ens_n16 = 0;  // systems (sorted by size) with > 16 and > 8 bodies

  // ---- per-device launch data, kept per context ----
  // A kernel's dynamic shared-memory limit (cudaFuncSetAttribute) is set on
  // the device that is current when it is raised, so it is raised once per
  // context, after the context has made its own device current; nothing is
  // shared between contexts or threads.  occ_gwalk: resident blocks per SM of
  // the group-walk kernels (list, evaluation F64 / F32C, re-queued walk F64 /
  // F32C), 0 until queried.
  int occ_gwalk[5] = {};
  bool sort_smem_set = false;
  // Bound on one look-back wait of the radix sort, in re-reads of a tile's
  // status word (see sort.cu); phys_debug_set_wait_limit lowers it in tests.
  int64_t sort_spin_limit = int64_t(1) << 20;

  // ---- CUDA graph of one direct-sum tick (force pass + fused velocity and
  // position steps), replayed for the middle ticks of phys_verlet_steps; kept
  // while what it was captured with is unchanged (ws_gen counts every move
  // of a device buffer: a workspace slot or the state arrays) ----
  cudaGraphExec_t tick_exec = nullptr;
  uint64_t tick_launches = 0;  // kernel launches in one replay
  phys_params tick_params{};
  double tick_dt = 0.0;
  int64_t tick_n = -1;
  bool tick_halo_on = false;
  phys_nfw_halo tick_halo{};
  uint64_t tick_gen = ~uint64_t(0);
  uint64_t ws_gen = 0;
  bool capturing = false;  // enqueueing into a capture: no timing events

  // ---- small device scalars ----
  int32_t* d_status = nullptr;               // kStat* bits
  unsigned long long* d_counter = nullptr;   // interaction counter
  phys::TreeHeader* d_hdr = nullptr;
  double* d_partials = nullptr;              // reduction partials (diagnostics, bbox)
  size_t partials_cap = 0;

  // ---- host staging (pinned) ----
  void* h_stage = nullptr;
  size_t h_stage_bytes = 0;
  int32_t* h_small = nullptr;                // pinned scalars for status / counts

  // ---- workspace buffers (grown on demand, named) ----
  phys::DevBuf ws[48];

  // ---- events for per-phase timings ----
  cudaEvent_t ev[12] = {};
};

// ---- helpers (ctx.cu) ----
namespace phys {
int fail(phys_ctx* c, int code, const char* fmt, ...);
int cuda_fail(phys_ctx* c, cudaError_t e, const char* what);
// Ensure workspace slot `slot` holds at least `bytes`; returns device pointer.
void* ws_get(phys_ctx* c, int slot, size_t bytes, int* status);
// Typed form: *out = workspace slot with room for `count` T; returns a status.
template <class T>
int ws_alloc(phys_ctx* c, int slot, int64_t count, T** out) {
  int st = 0;
  *out = static_cast<T*>(ws_get(c, slot, sizeof(T) * (size_t)(count > 0 ? count : 1), &st));
  return st;
}
int ensure_pinned(phys_ctx* c, size_t bytes);
int check_launch(phys_ctx* c, const char* what);
int read_status(phys_ctx* c, int32_t* out);

// Workspace slot ids.
enum WsSlot {
  WS_KEYS_HI = 0, WS_KEYS_LO, WS_IDX, WS_KEYS_HI_ALT, WS_IDX_ALT, WS_HIST,
  WS_LCP, WS_NCOUNT, WS_NFIRST, WS_SCAN_TMP,
  WS_LINK, WS_NODE_PM, WS_NODE_HI, WS_NODE_LO, WS_PARENT, WS_ARRIVE, WS_NODE_S,
  WS_BODY_PM, WS_BODY_HI, WS_BODY_LO,
  WS_KEEP, WS_NEWID,
  WS_ENTRIES, WS_ENTRIES_ALT, WS_EOFF, WS_ENTRY_BODY,
  WS_DIRECT_PART, WS_ADJ0, WS_ADJ1, WS_ADJ2, WS_ADJ3, WS_ADJ4,
  WS_ENS0, WS_ENS1, WS_ENS2, WS_ENS3, WS_ENS4, WS_ENS5, WS_ENS6, WS_ENS7,
  WS_GROUPS, WS_GROUP_OFF, WS_GROUP_CTR, WS_GROUP_POOL, WS_GROUP_ITEMS, WS_SHARE_PERM, WS_BODY_IN,
  WS_COUNT_
};
static_assert(WS_COUNT_ <= sizeof(phys_ctx::ws) / sizeof(DevBuf), "workspace slots");

// ---- kernels' host launchers (per .cu file) ----
// nfw.cu (px/py/pz: the positions the halo acts on)
int nfw_add_forces(phys_ctx* c, const phys_nfw_halo& halo, const double* px, const double* py,
                   const double* pz, double* fx, double* fy, double* fz);
int nfw_accel(phys_ctx* c, const phys_nfw_halo& halo, const double* px, const double* py,
              const double* pz, const double* fx, const double* fy, const double* fz, double* ax,
              double* ay, double* az);
// sectors.cu
int sector_state_alloc(phys_ctx* c, int64_t n);
int sector_flatten(phys_ctx* c, bool bh_quirk);
int sector_normalize(phys_ctx* c, int32_t* shifted);
// direct.cu
int direct_eval(phys_ctx* c, const phys_params* p, bool want_force, double* ox, double* oy,
                double* oz);
int direct_targets(phys_ctx* c, const phys_params* p, int64_t nt, const int64_t* d_tidx,
                   double* ox, double* oy, double* oz);
// Launches on stream s with caller-provided scratch; returns the launch error.
cudaError_t direct_accel_launch_scratch(cudaStream_t s, int64_t n, const double* x,
                                        const double* y, const double* z, const double* m,
                                        double G, double eps, int precision, int64_t nslices,
                                        double* part, float4* bh, float4* bl, int32_t* status,
                                        double* ox, double* oy, double* oz);
// tree.cu
int bh_eval(phys_ctx* c, const phys_params* p, bool want_force, double* ox, double* oy,
            double* oz);
int bh_export(phys_ctx* c, const phys_params* p, int64_t cap, int64_t* nnodes, int32_t* depth,
              int64_t* count, double* mass, double* com, int64_t* leaf_body, int64_t* body_leaf,
              uint64_t* keys_hi, uint64_t* keys_lo, int64_t* perm, double* root4);
// sort.cu
int radix_sort_u64(phys_ctx* c, uint64_t* keys, uint32_t* vals, uint64_t* keys_alt,
                   uint32_t* vals_alt, int64_t n, int begin_bit, int end_bit, bool* result_in_alt);
int scan_exclusive_i32(phys_ctx* c, const int32_t* in, int32_t* out, int64_t n);
// share.cu (targets of one share into a block of 3 * chunk; all blocks back)
int share_pack(phys_ctx* c, int64_t lo, int64_t hi, int64_t chunk, const uint32_t* perm,
               double* out);
int share_unpack(phys_ctx* c, int64_t chunk, const uint32_t* perm, const double* gathered);
// verlet.cu
int verlet_drift(phys_ctx* c, double dt);
int verlet_kick(phys_ctx* c, double dt);
int verlet_drift_pos(phys_ctx* c, double dt, double* x, double* y, double* z);
int verlet_kick_drift(phys_ctx* c, double dt);
int flatten_sectors(phys_ctx* c, const int64_t* dsx, const int64_t* dsy, const int64_t* dsz,
                    const double* dlx, const double* dly, const double* dlz, double sector_size,
                    int bh_quirk);
// ensemble.cu
int ensemble_load(phys_ctx* c, int64_t nsys, const int64_t* off, const double* x, const double* y,
                  const double* z, const double* vx, const double* vy, const double* vz,
                  const double* m);
int ensemble_run(phys_ctx* c, const phys_params* p, double dt, int64_t nsteps, int G,
                 int64_t chunk);
int ensemble_download(phys_ctx* c, double* x, double* y, double* z, double* vx, double* vy,
                      double* vz, double* ax, double* ay, double* az);
int ensemble_autotune(phys_ctx* c, const phys_params* p, double dt, int64_t probe_steps,
                      int32_t* best, double* ms3);
// adjoint.cu
int trajectory_loss(phys_ctx* c, const phys_params* p, double dt, int64_t nsteps,
                    const double* tx, const double* ty, const double* tz, double* loss,
                    double* xT, double* yT, double* zT);
int adjoint(phys_ctx* c, const phys_params* p, double dt, int64_t nsteps, int64_t K,
            const double* tx, const double* ty, const double* tz, double* loss, double* gxyz[3],
            double* gvxyz[3], double* gm);
// diag.cu
int diagnostics(phys_ctx* c, double G, double* out5);
int probe_peaks(phys_ctx* c, double* fp32, double* fp32x2, double* fp64);
int debug_divide(phys_ctx* c, int64_t n, const double* a, const double* b, double* q);
}  // namespace phys

#define PHYS_LAUNCH_ON(c, strm, kernel, grid, block, smem, ...)            \
  do {                                                                     \
    kernel<<<(grid), (block), (smem), (strm)>>>(__VA_ARGS__);              \
    (c)->launches++;                                                       \
    int _st = phys::check_launch((c), #kernel);                            \
    if (_st) return _st;                                                   \
  } while (0)

#define PHYS_LAUNCH(c, kernel, grid, block, smem, ...) \
  PHYS_LAUNCH_ON(c, (c)->stream, kernel, grid, block, smem, __VA_ARGS__)

#define PHYS_CUDA(c, call)                                                 \
  do {                                                                     \
    cudaError_t _e = (call);                                               \
    if (_e != cudaSuccess) return phys::cuda_fail((c), _e, #call);         \
  } while (0)

#define PHYS_TRY(expr)            \
  do {                            \
    int _s = (expr);              \
    if (_s) return _s;            \
  } while (0)

// ---- device helpers ----
namespace phys {

// IEEE double ops that the compiler may not contract into FMAs: the
// reference's Rust arithmetic rounds every + and * separately.
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double xsqrt(double a) { return __dsqrt_rn(a); }
// glam DVec3::length_squared: (x*x + y*y) + z*z
__device__ __forceinline__ double xlen2(double x, double y, double z) {
  return xadd(xadd(xmul(x, x), xmul(y, y)), xmul(z, z));
}

// a / b rounded to nearest from y = RN(1/b), computed ahead of a (Markstein's
// correction: P. Markstein, "Computation of elementary functions on the IBM
// RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990).  q0 = RN(a y)
// lies within 1.5 ulp of a/b; q1 = RN(q0 + y RN(a - b q0)) within one ulp;
// the remainder r1 = a - b q1 is then exact in an FMA, and RN(q1 + r1 y)
// is RN(a/b): with b's significand B < 2^53 the term r1 (b y - 1) stays
// below b |a/b - m| for every midpoint m (B^2 + B < 2^106), and a/b is never
// a midpoint.  Valid while no step underflows or overflows, which
// div_recip_num_ok(a) and div_recip_den_ok(b) guarantee (|a| and b in
// [2^-500, 2^501); a = +0 also gives +0; only positive b is accepted; both
// tests read the exponent bits on the integer pipe).  A chain of these
// divisions has five dependent operations per step, where a full division
// recomputes the reciprocal on the critical path.
__device__ __forceinline__ double div_recip(double a, double b, double y) {
  const double q0 = __dmul_rn(a, y);
  const double r0 = __fma_rn(-b, q0, a);
  const double q1 = __fma_rn(r0, y, q0);
  const double r1 = __fma_rn(-b, q1, a);
  return __fma_rn(r1, y, q1);
}
__device__ __forceinline__ bool div_recip_den_ok(double b) {
  // sign clear and biased exponent in [523, 1523] (a negative b shifts to a
  // negative value, far out of range as unsigned)
  return (unsigned long long)(__double_as_longlong(b) >> 52) - 523ull <= 1000ull;
}
__device__ __forceinline__ bool div_recip_num_ok(double a) {
  const long long bits = __double_as_longlong(a);
  return (unsigned long long)((bits >> 52) & 0x7ff) - 523ull <= 1000ull || bits == 0;
}

// Knuth two-sum: s + e == a + b exactly.
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
  s = __fadd_rn(a, b);
  float bb = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

// 1/sqrt(x) straight from the SFU: PTX rsqrt.approx.ftz.f32, relative error
// at most 2^-22.9 (the bound the PTX ISA states).  Every caller passes
// r^2 + eps^2 or a squared distance, so subnormal inputs do not arise in
// practice; flushing them lets the call compile to the one SFU instruction,
// without the input range handling a non-FTZ build adds around it.
__device__ __forceinline__ float rsqrt_sfu(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// sum_{s < nsl} p[s stride], added in slice order from 0.0 (the order the
// results depend on); the loads go out eight slices at a time.
__device__ __forceinline__ double slice_sum(const double* __restrict__ p, size_t stride,
                                            int nsl) {
  double a = 0.0;
  int s = 0;
  for (; s + 8 <= nsl; s += 8) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = p[(size_t)(s + u) * stride];
#pragma unroll
    for (int u = 0; u < 8; ++u) a += v[u];
  }
  for (; s < nsl; ++s) a += p[(size_t)s * stride];
  return a;
}

// True when a radix sort earlier in this call gave up a bounded wait
// (kStatTimeout in the status word): its output need not be a permutation.
// Kernels that index with a sort's output, or read records built from one,
// return at once, and the call fails with PHYS_ERR_TIMEOUT.  The flag is
// written by kernels earlier on the same stream (or on a stream that waited
// for them), so a later launch reads it settled.
__device__ __forceinline__ bool sort_failed(const int32_t* status) {
  return (*reinterpret_cast<const volatile int32_t*>(status) & kStatTimeout) != 0;
}

// Split a double into a float pair with hi + lo ~= v to ~2^-48 relative.
__device__ __forceinline__ void split_df(double v, float& hi, float& lo) {
  hi = __double2float_rn(v);
  lo = __double2float_rn(v - (double)hi);
}

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
__host__ __device__ inline int64_t min64(int64_t a, int64_t b) { return a < b ? a : b; }

// Targets [lo, hi) of the current evaluation of n bodies: all of them unless
// a target share is set (phys_gravity_accel_share).
inline void target_range(const phys_ctx* c, int64_t n, int64_t& lo, int64_t& hi) {
  lo = 0;
  hi = n;
  if (c->share_hi >= 0) {
    lo = min64(c->share_lo, n);
    hi = min64(c->share_hi, n);
  }
}
// Targets per share when n bodies are split into `world` shares: a multiple
// of 128 (the direct sum's tile), so that every share starts on a tile.
inline int64_t share_chunk(int64_t n, int64_t world) {
  return world > 0 ? ceil_div(ceil_div(n, world), 128) * 128 : 0;
}

}  // namespace phys
