// Context, device state, error handling and the public entry points that
// orchestrate the kernels of the other translation units.
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"

namespace phys {

int fail(phys_ctx* c, int code, const char* fmt, ...) {
  if (c) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    c->err = buf;
  }
  return code;
}

int cuda_fail(phys_ctx* c, cudaError_t e, const char* what) {
  int code = (e == cudaErrorMemoryAllocation) ? PHYS_ERR_OOM : PHYS_ERR_CUDA;
  cudaGetLastError();  // clear non-sticky errors
  return fail(c, code, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

int check_launch(phys_ctx* c, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(c, e, what);
  return PHYS_OK;
}

void* ws_get(phys_ctx* c, int slot, size_t bytes, int* status) {
  DevBuf& b = c->ws[slot];
  if (bytes == 0) bytes = 16;
  if (b.bytes >= bytes) return b.p;
  if (b.p) {
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
      *status = cuda_fail(c, e, "cudaStreamSynchronize(ws grow)");
      return nullptr;
    }
    cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
  }
  size_t want = bytes + bytes / 8;  // headroom for slowly growing sizes
  want = (want + 255) & ~size_t(255);
  ++c->ws_gen;
  cudaError_t e = cudaMalloc(&b.p, want);
  if (e != cudaSuccess) {
    b.p = nullptr;
    *status = cuda_fail(c, e, "cudaMalloc(workspace)");
    return nullptr;
  }
  b.bytes = want;
  return b.p;
}

int ensure_pinned(phys_ctx* c, size_t bytes) {
  if (c->h_stage_bytes >= bytes) return PHYS_OK;
  if (c->h_stage) {
    cudaStreamSynchronize(c->stream);
    cudaFreeHost(c->h_stage);
    c->h_stage = nullptr;
    c->h_stage_bytes = 0;
  }
  cudaError_t e = cudaMallocHost(&c->h_stage, bytes);
  if (e != cudaSuccess) {
    c->h_stage = nullptr;
    return cuda_fail(c, e, "cudaMallocHost(staging)");
  }
  c->h_stage_bytes = bytes;
  return PHYS_OK;
}

int read_status(phys_ctx* c, int32_t* out) {
  PHYS_CUDA(c, cudaMemcpyAsync(c->h_small, c->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost,
                               c->stream));
  PHYS_CUDA(c, cudaMemcpyAsync(c->h_small + 2, c->d_counter, 2 * sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, c->stream));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  *out = c->h_small[0];
  if (c->last_eval_bh) {
    unsigned long long v[2];
    memcpy(v, c->h_small + 2, sizeof v);
    c->tm.interactions = v[0];
    c->tm.walk_eval_interactions = c->last_eval_group ? v[1] : 0;
  }
  return PHYS_OK;
}

}  // namespace phys

using namespace phys;

// Every entry point that touches the device makes the context's device
// current first, so contexts on different devices can be used from one
// thread in any order.
#define PHYS_ENTER(c)                                    \
  do {                                                   \
    if (!(c)) return PHYS_ERR_ARG;                       \
    PHYS_CUDA((c), cudaSetDevice((c)->device));          \
  } while (0)

namespace {

int ensure_state(phys_ctx* c, int64_t n) {
  if (n <= c->cap) return PHYS_OK;
  if (c->x) {
    cudaStreamSynchronize(c->stream);
    cudaFree(c->x);
    c->x = nullptr;
    c->cap = 0;
  }
  int64_t cap = n < 1024 ? 1024 : n;
  double* base = nullptr;
  ++c->ws_gen;
  cudaError_t e = cudaMalloc(&base, sizeof(double) * 16 * size_t(cap));
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc(state)");
  double** slots[16] = {&c->x,  &c->y,  &c->z,  &c->vx,  &c->vy,  &c->vz,  &c->m,  &c->ax,
                        &c->ay, &c->az, &c->pax, &c->pay, &c->paz, &c->fx, &c->fy, &c->fz};
  for (int k = 0; k < 16; ++k) *slots[k] = base + size_t(k) * cap;
  c->cap = cap;
  return PHYS_OK;
}

int h2d(phys_ctx* c, double* dst, const double* src, int64_t n) {
  if (src) {
    PHYS_CUDA(c, cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  } else {
    PHYS_CUDA(c, cudaMemsetAsync(dst, 0, sizeof(double) * n, c->stream));
  }
  return PHYS_OK;
}

int d2h(phys_ctx* c, double* dst, const double* src, int64_t n) {
  if (dst)
    PHYS_CUDA(c, cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  return PHYS_OK;
}

int check_params(phys_ctx* c, const phys_params* p) {
  if (!p) return fail(c, PHYS_ERR_ARG, "params is NULL");
  if (p->method != PHYS_DIRECT && p->method != PHYS_BARNES_HUT)
    return fail(c, PHYS_ERR_ARG, "unknown method %d", p->method);
  if (p->precision < PHYS_F64_EXACT || p->precision > PHYS_F32C)
    return fail(c, PHYS_ERR_ARG, "unknown precision %d", p->precision);
  if (p->leaf_cap < 1 || p->leaf_cap > kMaxLeafCap)
    return fail(c, PHYS_ERR_ARG, "leaf_cap %d outside 1..%d", p->leaf_cap, kMaxLeafCap);
  if (p->method == PHYS_BARNES_HUT && p->precision == PHYS_F64_EXACT && p->leaf_cap != 1)
    return fail(c, PHYS_ERR_ARG, "F64_EXACT Barnes-Hut follows the reference octree: leaf_cap 1");
  if (p->flags & ~PHYS_FLAG_GROUP_WALK) return fail(c, PHYS_ERR_ARG, "unknown flags 0x%x", p->flags);
  if ((p->flags & PHYS_FLAG_GROUP_WALK) &&
      (p->method != PHYS_BARNES_HUT || p->precision == PHYS_F64_EXACT))
    return fail(c, PHYS_ERR_ARG, "the group walk is Barnes-Hut with PHYS_F64 or PHYS_F32C");
  if (!(p->theta >= 0.0)) return fail(c, PHYS_ERR_ARG, "theta must be >= 0");
  return PHYS_OK;
}

bool same_params(const phys_params& a, const phys_params& b) {
  return a.G == b.G && a.eps == b.eps && a.theta == b.theta && a.method == b.method &&
         a.precision == b.precision && a.leaf_cap == b.leaf_cap && a.flags == b.flags;
}

// One gravity evaluation on the device: accelerations into c->ax..
// (want_force false) or forces into c->fx.. (want_force true).
int eval_gravity(phys_ctx* c, const phys_params* p, bool want_force) {
  double* ox = want_force ? c->fx : c->ax;
  double* oy = want_force ? c->fy : c->ay;
  double* oz = want_force ? c->fz : c->az;
  if (c->n < 2) {  // gravity.rs:49-51: no pairs, forces stay zero
    PHYS_CUDA(c, cudaMemsetAsync(ox, 0, sizeof(double) * c->n, c->stream));
    PHYS_CUDA(c, cudaMemsetAsync(oy, 0, sizeof(double) * c->n, c->stream));
    PHYS_CUDA(c, cudaMemsetAsync(oz, 0, sizeof(double) * c->n, c->stream));
    c->tm.interactions = 0;
    return PHYS_OK;
  }
  c->last_eval_bh = p->method == PHYS_BARNES_HUT;
  c->last_eval_group = c->last_eval_bh && (p->flags & PHYS_FLAG_GROUP_WALK);
  if (p->method == PHYS_DIRECT) return direct_eval(c, p, want_force, ox, oy, oz);
  return bh_eval(c, p, want_force, ox, oy, oz);
}

// Forces or accelerations as the reference schedule forms them: with an NFW
// halo set, a = (F_gravity + F_nfw) / m (src/main.rs:109-110, nfw.rs:103-139,
// integrators.rs:110-118).
int eval(phys_ctx* c, const phys_params* p, bool want_force) {
  c->share_world = 0;  // a pending share is void once anything else is evaluated
  // sector mode: positions flattened for this pass (the Barnes-Hut system's
  // per-body origin for Barnes-Hut, gravity_tree.rs:280-291)
  if (c->sector_mode) PHYS_TRY(sector_flatten(c, p->method == PHYS_BARNES_HUT));
  if (want_force || !c->halo_on) return eval_gravity(c, p, want_force);
  PHYS_TRY(eval_gravity(c, p, true));
  // the halo reads LocalPosition (nfw.rs:118)
  const int64_t cap = c->sec_cap;
  const double* px = c->sector_mode ? c->loc : c->x;
  const double* py = c->sector_mode ? c->loc + cap : c->y;
  const double* pz = c->sector_mode ? c->loc + 2 * cap : c->z;
  return nfw_accel(c, c->halo, px, py, pz, c->fx, c->fy, c->fz, c->ax, c->ay, c->az);
}

// Positions for a call that reads c->x directly: in sector mode, flattened
// with the direct-sum origin (gravity.rs:38-47) or the Barnes-Hut quirk.
int positions_ready(phys_ctx* c, bool bh_quirk) {
  return c->sector_mode ? sector_flatten(c, bh_quirk) : PHYS_OK;
}


float ev_ms(cudaEvent_t a, cudaEvent_t b);

int finish_status(phys_ctx* c) {
  int32_t st = 0;
  PHYS_TRY(read_status(c, &st));
  if (c->last_eval_bh) {
    c->tm.bbox_ms = ev_ms(c->ev[2], c->ev[3]);
    c->tm.keys_ms = ev_ms(c->ev[3], c->ev[4]);
    c->tm.sort_ms = ev_ms(c->ev[4], c->ev[5]);
    c->tm.tree_ms = ev_ms(c->ev[5], c->ev[6]);
  }
  c->tm.walk_ms = ev_ms(c->ev[6], c->ev[7]);
  c->tm.walk_eval_ms = c->last_eval_group ? ev_ms(c->ev[10], c->ev[11]) : 0.0;
  if (st & kStatTimeout) return fail(c, PHYS_ERR_TIMEOUT, "a bounded device wait timed out");
  if (st & kStatOverflow) return fail(c, PHYS_ERR_CUDA, "device workspace overflow");
  if (st & kStatNonfinite)
    return fail(c, PHYS_ERR_NONFINITE, "non-finite value in positions, masses or results");
  return PHYS_OK;
}

int reset_status(phys_ctx* c) {
  PHYS_CUDA(c, cudaMemsetAsync(c->d_status, 0, sizeof(int32_t), c->stream));
  return PHYS_OK;
}

float ev_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
    cudaGetLastError();
    return 0.f;
  }
  return ms;
}

// The reference tick loop on the (Sector, LocalPosition) state: position
// step on LocalPosition, force pass, velocity step, sector_boundary_system
// (src/main.rs:103-140,149).  a(x) of the velocity step's force pass is reused
// by the next tick's first pass unless a body changed sector: then the
// flattened positions (and with the Barnes-Hut quirk the positions
// themselves) changed, and the pass is run again as the reference does.
int verlet_steps_sectors(phys_ctx* c, const phys_params* p, double dt, int64_t nsteps,
                         bool sync) {
  const int64_t cap = c->sec_cap;
  double *lx = c->loc, *ly = c->loc + cap, *lz = c->loc + 2 * cap;
  int32_t* h_shift = c->h_small + 16;
  for (int64_t s = 0; s < nsteps; ++s) {
    if (!c->accel_valid || (c->accel_params.method != -1 && !same_params(c->accel_params, *p))) {
      PHYS_TRY(eval(c, p, false));  // chain 1 force pass
      c->accel_valid = true;
      c->accel_params = *p;
    }
    PHYS_TRY(verlet_drift_pos(c, dt, lx, ly, lz));
    c->accel_valid = false;
    PHYS_TRY(eval(c, p, false));  // chain 2 force pass
    PHYS_TRY(verlet_kick(c, dt));
    PHYS_CUDA(c, cudaMemsetAsync(c->d_shift, 0, sizeof(int32_t), c->stream));
    PHYS_TRY(sector_normalize(c, c->d_shift));
    PHYS_CUDA(c, cudaMemcpyAsync(h_shift, c->d_shift, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                 c->stream));
    PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
    c->accel_valid = *h_shift == 0;
    c->accel_params = *p;
  }
  PHYS_CUDA(c, cudaEventRecord(c->ev[1], c->stream));
  if (sync) {
    PHYS_TRY(finish_status(c));
    c->tm.total_ms = ev_ms(c->ev[0], c->ev[1]);
  }
  return PHYS_OK;
}

static bool same_halo(const phys_nfw_halo& a, const phys_nfw_halo& b) {
  return a.rho_0 == b.rho_0 && a.scale_radius == b.scale_radius && a.center[0] == b.center[0] &&
         a.center[1] == b.center[1] && a.center[2] == b.center[2] && a.enabled == b.enabled;
}

// The graph of one direct-sum tick body (force pass at x, then the velocity
// step fused with the next position step), captured once and kept while n,
// the parameters, dt, the halo and every device buffer are the same.  Its
// kernels are the ones the loop would launch, so a replay is bit-identical
// to them.  Returns false (nothing captured, nothing left pending) when the
// capture fails; the caller then launches the tick itself.
static bool tick_graph(phys_ctx* c, const phys_params* p, double dt) {
  if (c->tick_exec && c->tick_n == c->n && same_params(c->tick_params, *p) && c->tick_dt == dt &&
      c->tick_halo_on == c->halo_on && (!c->halo_on || same_halo(c->tick_halo, c->halo)) &&
      c->tick_gen == c->ws_gen)
    return true;
  if (c->tick_exec) {
    cudaGraphExecDestroy(c->tick_exec);
    c->tick_exec = nullptr;
  }
  if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  const uint64_t gen0 = c->ws_gen, l0 = c->launches;
  c->capturing = true;
  int st = eval(c, p, false);
  if (st == PHYS_OK) st = verlet_kick_drift(c, dt);
  c->capturing = false;
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  cudaGraphExec_t exec = nullptr;
  const bool ok = st == PHYS_OK && e == cudaSuccess && g && c->ws_gen == gen0 &&
                  cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();
  const uint64_t nl = c->launches - l0;  // counted as they are replayed
  c->launches = l0;
  if (!ok) {
    if (exec) cudaGraphExecDestroy(exec);
    c->err.clear();
    return false;
  }
  c->tick_exec = exec;
  c->tick_launches = nl;
  c->tick_n = c->n;
  c->tick_params = *p;
  c->tick_dt = dt;
  c->tick_halo_on = c->halo_on;
  c->tick_halo = c->halo;
  c->tick_gen = c->ws_gen;
  return true;
}

int verlet_steps(phys_ctx* c, const phys_params* p, double dt, int64_t nsteps, bool sync) {
  PHYS_TRY(check_params(c, p));
  if (nsteps < 0) return fail(c, PHYS_ERR_ARG, "nsteps < 0");
  if (c->n == 0) return fail(c, PHYS_ERR_STATE, "no body state uploaded");
  if (!(dt == dt)) return fail(c, PHYS_ERR_ARG, "dt is NaN");
  PHYS_TRY(reset_status(c));
  PHYS_CUDA(c, cudaEventRecord(c->ev[0], c->stream));
  if (c->sector_mode) return verlet_steps_sectors(c, p, dt, nsteps, sync);
  // accel_params.method == -1: the caller supplied a(x) (Acceleration
  // component), valid whatever the params.
  if (!c->accel_valid || (c->accel_params.method != -1 && !same_params(c->accel_params, *p))) {
    PHYS_TRY(eval(c, p, false));  // chain 1 force pass of the first tick
    c->accel_valid = true;
  }
  c->accel_params = *p;
  // the direct sum's ticks have no host synchronisation: the middle ones
  // replay a captured graph of one tick (one launch instead of a handful)
  const bool by_graph = p->method == PHYS_DIRECT && nsteps >= 4 && !c->copy_x[0];
  for (int64_t s = 0; s < nsteps; ++s) {
    if (by_graph && s == 1 && tick_graph(c, p, dt)) {
      // ticks 1 .. nsteps-2: force pass, velocity step, next position step
      for (; s + 1 < nsteps; ++s) {
        PHYS_CUDA(c, cudaGraphLaunch(c->tick_exec, c->stream));
        c->launches += c->tick_launches;
      }
    }
    if (s == 0) {
      PHYS_TRY(verlet_drift(c, dt));
      if (nsteps == 1 && c->copy_x[0]) {
        // the tick's positions are final: copy them back beside the force pass
        PHYS_CUDA(c, cudaEventRecord(c->copy_fork, c->stream));
        PHYS_CUDA(c, cudaStreamWaitEvent(c->copy, c->copy_fork, 0));
        const double* src[3] = {c->x, c->y, c->z};
        for (int k = 0; k < 3; ++k)
          PHYS_CUDA(c, cudaMemcpyAsync(c->copy_x[k], src[k], sizeof(double) * c->n,
                                       cudaMemcpyDeviceToHost, c->copy));
        PHYS_CUDA(c, cudaEventRecord(c->copy_done, c->copy));
      }
    }
    c->accel_valid = false;
    PHYS_TRY(eval(c, p, false));  // chain 2 force pass at x_{n+1}
    c->accel_valid = true;
    if (s + 1 < nsteps)
      PHYS_TRY(verlet_kick_drift(c, dt));  // velocity step of tick s, position step of s+1
    else
      PHYS_TRY(verlet_kick(c, dt));
  }
  PHYS_CUDA(c, cudaEventRecord(c->ev[1], c->stream));
  if (sync) {
    PHYS_TRY(finish_status(c));
    c->tm.total_ms = ev_ms(c->ev[0], c->ev[1]);
  }
  return PHYS_OK;
}

}  // namespace

extern "C" {

const char* phys_status_string(int s) {
  switch (s) {
    case PHYS_OK: return "ok";
    case PHYS_ERR_ARG: return "invalid argument";
    case PHYS_ERR_CUDA: return "CUDA error";
    case PHYS_ERR_OOM: return "out of memory";
    case PHYS_ERR_NONFINITE: return "non-finite value";
    case PHYS_ERR_TIMEOUT: return "device wait timed out";
    case PHYS_ERR_STATE: return "invalid call order";
    default: return "unknown status";
  }
}

const char* phys_last_error(const phys_ctx* c) { return c ? c->err.c_str() : "null context"; }

int phys_ctx_create(int device, phys_ctx** out) {
  if (!out) return PHYS_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return PHYS_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) return PHYS_ERR_ARG;
  phys_ctx* c = new (std::nothrow) phys_ctx();
  if (!c) return PHYS_ERR_OOM;
  c->device = device;
  int st = PHYS_OK;
  do {
    if ((e = cudaSetDevice(device)) != cudaSuccess) { st = cuda_fail(c, e, "cudaSetDevice"); break; }
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) {
      st = cuda_fail(c, e, "cudaStreamCreate");
      break;
    }
    for (auto& ev : c->ev)
      if ((e = cudaEventCreate(&ev)) != cudaSuccess) { st = cuda_fail(c, e, "cudaEventCreate"); break; }
    if (st) break;
    if ((e = cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking)) != cudaSuccess) {
      st = cuda_fail(c, e, "cudaStreamCreate(side)");
      break;
    }
    if ((e = cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming)) != cudaSuccess) {
      st = cuda_fail(c, e, "cudaEventCreate(fork/join)");
      break;
    }
    if ((e = cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->copy_fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->copy_done, cudaEventDisableTiming)) != cudaSuccess) {
      st = cuda_fail(c, e, "cudaStreamCreate(copy)");
      break;
    }
    char* small = nullptr;
    if ((e = cudaMalloc(&small, 4096)) != cudaSuccess) { st = cuda_fail(c, e, "cudaMalloc(small)"); break; }
    c->d_status = reinterpret_cast<int32_t*>(small);
    // [0] interactions of the last evaluation, [1] of the group walk's list evaluation
    c->d_counter = reinterpret_cast<unsigned long long*>(small + 256);
    c->d_hdr = reinterpret_cast<TreeHeader*>(small + 512);
    c->d_shift = reinterpret_cast<int32_t*>(small + 3840);
    static_assert(512 + sizeof(TreeHeader) <= 3840, "small device block layout");
    if ((e = cudaMemset(small, 0, 4096)) != cudaSuccess) { st = cuda_fail(c, e, "cudaMemset"); break; }
    if ((e = cudaMallocHost(&c->h_small, 4096)) != cudaSuccess) {
      st = cuda_fail(c, e, "cudaMallocHost(small)");
      break;
    }
  } while (0);
  if (st) {
    phys_ctx_destroy(c);
    return st;
  }
  *out = c;
  return PHYS_OK;
}

int phys_ctx_destroy(phys_ctx* c) {
  if (!c) return PHYS_OK;
  cudaSetDevice(c->device);
  if (c->side) cudaStreamSynchronize(c->side);
  if (c->copy) cudaStreamSynchronize(c->copy);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto& b : c->ws)
    if (b.p) cudaFree(b.p);
  if (c->x) cudaFree(c->x);
  if (c->sec) cudaFree(c->sec);
  if (c->d_status) cudaFree(c->d_status);
  if (c->d_partials) cudaFree(c->d_partials);
  if (c->h_stage) cudaFreeHost(c->h_stage);
  if (c->h_small) cudaFreeHost(c->h_small);
  for (auto& ev : c->ev)
    if (ev) cudaEventDestroy(ev);
  if (c->fork) cudaEventDestroy(c->fork);
  if (c->join) cudaEventDestroy(c->join);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->copy_fork) cudaEventDestroy(c->copy_fork);
  if (c->copy_done) cudaEventDestroy(c->copy_done);
  if (c->copy) cudaStreamDestroy(c->copy);
  if (c->tick_exec) cudaGraphExecDestroy(c->tick_exec);
  if (c->stream) cudaStreamDestroy(c->stream);
  cudaGetLastError();
  delete c;
  return PHYS_OK;
}

void* phys_ctx_stream(phys_ctx* c) { return c ? (void*)c->stream : nullptr; }

int phys_last_timings(const phys_ctx* c, phys_timings* out) {
  if (!c || !out) return PHYS_ERR_ARG;
  *out = c->tm;
  out->launches = c->launches;
  return PHYS_OK;
}

int64_t phys_state_size(const phys_ctx* c) { return c ? c->n : -1; }

int phys_state_upload(phys_ctx* c, int64_t n, const double* x, const double* y, const double* z,
                      const double* vx, const double* vy, const double* vz, const double* m) {
  PHYS_ENTER(c);
  if (n < 0 || n > (int64_t(1) << 31) - 1) return fail(c, PHYS_ERR_ARG, "n=%lld out of range", (long long)n);
  if (n > 0 && (!x || !y || !z || !m)) return fail(c, PHYS_ERR_ARG, "positions and masses are required");
  PHYS_TRY(ensure_state(c, n));
  c->n = n;
  c->share_world = 0;  // a pending share's tree order belongs to the old state
  c->sector_mode = false;
  c->accel_valid = false;
  if (n == 0) return PHYS_OK;
  PHYS_TRY(h2d(c, c->x, x, n));
  PHYS_TRY(h2d(c, c->y, y, n));
  PHYS_TRY(h2d(c, c->z, z, n));
  PHYS_TRY(h2d(c, c->vx, vx, n));
  PHYS_TRY(h2d(c, c->vy, vy, n));
  PHYS_TRY(h2d(c, c->vz, vz, n));
  PHYS_TRY(h2d(c, c->m, m, n));
  PHYS_TRY(h2d(c, c->ax, nullptr, n));
  PHYS_TRY(h2d(c, c->ay, nullptr, n));
  PHYS_TRY(h2d(c, c->az, nullptr, n));
  PHYS_TRY(h2d(c, c->pax, nullptr, n));
  PHYS_TRY(h2d(c, c->pay, nullptr, n));
  PHYS_TRY(h2d(c, c->paz, nullptr, n));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  return PHYS_OK;
}

int phys_state_upload_sectors(phys_ctx* c, int64_t n, const int64_t* sx, const int64_t* sy,
                              const int64_t* sz, const double* lx, const double* ly,
                              const double* lz, double sector_size, int32_t bh_quirk,
                              const double* vx, const double* vy, const double* vz,
                              const double* m) {
  PHYS_ENTER(c);
  if (n < 0 || n > (int64_t(1) << 31) - 1) return fail(c, PHYS_ERR_ARG, "n out of range");
  if (n > 0 && (!sx || !sy || !sz || !lx || !ly || !lz || !m))
    return fail(c, PHYS_ERR_ARG, "sectors, local positions and masses are required");
  PHYS_TRY(ensure_state(c, n));
  c->n = n;
  c->share_world = 0;  // a pending share's tree order belongs to the old state
  c->sector_mode = false;
  c->accel_valid = false;
  if (n == 0) return PHYS_OK;
  // Stage sectors in the force scratch arrays (same size as int64) and the
  // local positions in x/y/z, then flatten in place on the device.
  int64_t* dsx = reinterpret_cast<int64_t*>(c->fx);
  int64_t* dsy = reinterpret_cast<int64_t*>(c->fy);
  int64_t* dsz = reinterpret_cast<int64_t*>(c->fz);
  PHYS_CUDA(c, cudaMemcpyAsync(dsx, sx, 8 * n, cudaMemcpyHostToDevice, c->stream));
  PHYS_CUDA(c, cudaMemcpyAsync(dsy, sy, 8 * n, cudaMemcpyHostToDevice, c->stream));
  PHYS_CUDA(c, cudaMemcpyAsync(dsz, sz, 8 * n, cudaMemcpyHostToDevice, c->stream));
  PHYS_TRY(h2d(c, c->x, lx, n));
  PHYS_TRY(h2d(c, c->y, ly, n));
  PHYS_TRY(h2d(c, c->z, lz, n));
  PHYS_TRY(flatten_sectors(c, dsx, dsy, dsz, c->x, c->y, c->z, sector_size, bh_quirk));
  PHYS_TRY(h2d(c, c->vx, vx, n));
  PHYS_TRY(h2d(c, c->vy, vy, n));
  PHYS_TRY(h2d(c, c->vz, vz, n));
  PHYS_TRY(h2d(c, c->m, m, n));
  PHYS_TRY(h2d(c, c->ax, nullptr, n));
  PHYS_TRY(h2d(c, c->ay, nullptr, n));
  PHYS_TRY(h2d(c, c->az, nullptr, n));
  PHYS_TRY(h2d(c, c->pax, nullptr, n));
  PHYS_TRY(h2d(c, c->pay, nullptr, n));
  PHYS_TRY(h2d(c, c->paz, nullptr, n));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  return PHYS_OK;
}

int phys_state_upload_sector_state(phys_ctx* c, int64_t n, const int64_t* sx, const int64_t* sy,
                                   const int64_t* sz, const double* lx, const double* ly,
                                   const double* lz, double sector_size, const double* vx,
                                   const double* vy, const double* vz, const double* m) {
  PHYS_ENTER(c);
  if (n < 0 || n > (int64_t(1) << 31) - 1) return fail(c, PHYS_ERR_ARG, "n out of range");
  if (n > 0 && (!sx || !sy || !sz || !lx || !ly || !lz || !m))
    return fail(c, PHYS_ERR_ARG, "sectors, local positions and masses are required");
  if (!(sector_size > 0.0)) return fail(c, PHYS_ERR_ARG, "sector_size must be > 0");
  PHYS_TRY(ensure_state(c, n));
  PHYS_TRY(sector_state_alloc(c, n));
  c->n = n;
  c->share_world = 0;  // a pending share's tree order belongs to the old state
  c->sector_mode = true;
  c->sector_size = sector_size;
  c->accel_valid = false;
  if (n == 0) return PHYS_OK;
  const int64_t cap = c->sec_cap;
  const int64_t* hs[3] = {sx, sy, sz};
  const double* hl[3] = {lx, ly, lz};
  for (int k = 0; k < 3; ++k) {
    PHYS_CUDA(c, cudaMemcpyAsync(c->sec + k * cap, hs[k], 8 * n, cudaMemcpyHostToDevice,
                                 c->stream));
    PHYS_TRY(h2d(c, c->loc + k * cap, hl[k], n));
  }
  PHYS_TRY(h2d(c, c->vx, vx, n));
  PHYS_TRY(h2d(c, c->vy, vy, n));
  PHYS_TRY(h2d(c, c->vz, vz, n));
  PHYS_TRY(h2d(c, c->m, m, n));
  double* zero[6] = {c->ax, c->ay, c->az, c->pax, c->pay, c->paz};
  for (double* d : zero) PHYS_TRY(h2d(c, d, nullptr, n));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  return PHYS_OK;
}

int phys_state_download_sector_state(phys_ctx* c, int64_t* sx, int64_t* sy, int64_t* sz,
                                     double* lx, double* ly, double* lz) {
  PHYS_ENTER(c);
  if (!c->sector_mode) return fail(c, PHYS_ERR_STATE, "no sector state uploaded");
  const int64_t n = c->n, cap = c->sec_cap;
  if (n == 0) return PHYS_OK;
  int64_t* hs[3] = {sx, sy, sz};
  double* hl[3] = {lx, ly, lz};
  for (int k = 0; k < 3; ++k) {
    if (hs[k])
      PHYS_CUDA(c, cudaMemcpyAsync(hs[k], c->sec + k * cap, 8 * n, cudaMemcpyDeviceToHost,
                                   c->stream));
    PHYS_TRY(d2h(c, hl[k], c->loc + k * cap, n));
  }
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  return PHYS_OK;
}

int phys_state_set_accel(phys_ctx* c, const double* ax, const double* ay, const double* az) {
  PHYS_ENTER(c);
  if (!ax || !ay || !az) return fail(c, PHYS_ERR_ARG, "accelerations are required");
  PHYS_TRY(h2d(c, c->ax, ax, c->n));
  PHYS_TRY(h2d(c, c->ay, ay, c->n));
  PHYS_TRY(h2d(c, c->az, az, c->n));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  c->accel_valid = true;
  c->accel_params.method = -1;  // valid for any params: the caller vouches for it
  return PHYS_OK;
}

int phys_state_download(phys_ctx* c, double* x, double* y, double* z, double* vx, double* vy,
                        double* vz, double* ax, double* ay, double* az) {
  PHYS_ENTER(c);
  int64_t n = c->n;
  if (n == 0) return PHYS_OK;
  const int64_t cap = c->sec_cap;
  PHYS_TRY(d2h(c, x, c->sector_mode ? c->loc : c->x, n));  // LocalPosition in sector mode
  PHYS_TRY(d2h(c, y, c->sector_mode ? c->loc + cap : c->y, n));
  PHYS_TRY(d2h(c, z, c->sector_mode ? c->loc + 2 * cap : c->z, n));
  PHYS_TRY(d2h(c, vx, c->vx, n));
  PHYS_TRY(d2h(c, vy, c->vy, n));
  PHYS_TRY(d2h(c, vz, c->vz, n));
  PHYS_TRY(d2h(c, ax, c->ax, n));
  PHYS_TRY(d2h(c, ay, c->ay, n));
  PHYS_TRY(d2h(c, az, c->az, n));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  return PHYS_OK;
}

static int comp_ptrs(phys_ctx* c, int32_t comp, double** a, double** b, double** d) {
  switch (comp) {
    case PHYS_COMP_POSITION:  // LocalPosition in sector mode
      if (c->sector_mode) {
        *a = c->loc;
        *b = c->loc + c->sec_cap;
        *d = c->loc + 2 * c->sec_cap;
      } else {
        *a = c->x;
        *b = c->y;
        *d = c->z;
      }
      return PHYS_OK;
    case PHYS_COMP_VELOCITY: *a = c->vx; *b = c->vy; *d = c->vz; return PHYS_OK;
    case PHYS_COMP_ACCELERATION: *a = c->ax; *b = c->ay; *d = c->az; return PHYS_OK;
    case PHYS_COMP_PREV_ACCELERATION: *a = c->pax; *b = c->pay; *d = c->paz; return PHYS_OK;
    case PHYS_COMP_MASS: *a = c->m; *b = nullptr; *d = nullptr; return PHYS_OK;
    default: return fail(c, PHYS_ERR_ARG, "unknown component %d", comp);
  }
}

int phys_component_write(phys_ctx* c, int32_t comp, const double* a, const double* b,
                         const double* d) {
  PHYS_ENTER(c);
  if (c->n == 0) return fail(c, PHYS_ERR_STATE, "no body state uploaded");
  double *da = nullptr, *db = nullptr, *dd = nullptr;
  PHYS_TRY(comp_ptrs(c, comp, &da, &db, &dd));
  if (!a || (db && (!b || !d))) return fail(c, PHYS_ERR_ARG, "component arrays are required");
  PHYS_TRY(h2d(c, da, a, c->n));
  if (db) {
    PHYS_TRY(h2d(c, db, b, c->n));
    PHYS_TRY(h2d(c, dd, d, c->n));
  }
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  if (comp == PHYS_COMP_POSITION || comp == PHYS_COMP_MASS) c->accel_valid = false;
  if (comp == PHYS_COMP_ACCELERATION) {
    c->accel_valid = true;
    c->accel_params.method = -1;
  }
  return PHYS_OK;
}

int phys_component_read(phys_ctx* c, int32_t comp, double* a, double* b, double* d) {
  PHYS_ENTER(c);
  double *da = nullptr, *db = nullptr, *dd = nullptr;
  PHYS_TRY(comp_ptrs(c, comp, &da, &db, &dd));
  if (c->n == 0) return PHYS_OK;
  PHYS_TRY(d2h(c, a, da, c->n));
  if (db) {
    PHYS_TRY(d2h(c, b, db, c->n));
    PHYS_TRY(d2h(c, d, dd, c->n));
  }
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  return PHYS_OK;
}

int phys_vv_position_step(phys_ctx* c, double dt) {
  PHYS_ENTER(c);
  if (c->n == 0) return fail(c, PHYS_ERR_STATE, "no body state uploaded");
  PHYS_TRY(reset_status(c));
  PHYS_TRY(verlet_drift(c, dt));
  c->accel_valid = false;
  return finish_status(c);
}

int phys_vv_velocity_step(phys_ctx* c, double dt) {
  PHYS_ENTER(c);
  if (c->n == 0) return fail(c, PHYS_ERR_STATE, "no body state uploaded");
  PHYS_TRY(reset_status(c));
  PHYS_TRY(verlet_kick(c, dt));
  return finish_status(c);
}

int phys_gravity_forces(phys_ctx* c, const phys_params* p, double* fx, double* fy, double* fz) {
  PHYS_ENTER(c);
  PHYS_TRY(check_params(c, p));
  if (!fx || !fy || !fz) return fail(c, PHYS_ERR_ARG, "force arrays are required");
  int64_t n = c->n;
  if (n < 2) return PHYS_OK;  // gravity.rs:49-51
  PHYS_TRY(reset_status(c));
  PHYS_CUDA(c, cudaEventRecord(c->ev[0], c->stream));
  PHYS_TRY(eval(c, p, true));
  PHYS_CUDA(c, cudaEventRecord(c->ev[1], c->stream));
  PHYS_TRY(ensure_pinned(c, sizeof(double) * 3 * n));
  double* h = static_cast<double*>(c->h_stage);
  PHYS_TRY(d2h(c, h, c->fx, n));
  PHYS_TRY(d2h(c, h + n, c->fy, n));
  PHYS_TRY(d2h(c, h + 2 * n, c->fz, n));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  int st = finish_status(c);
  c->tm.total_ms = ev_ms(c->ev[0], c->ev[1]);
  if (st) return st;
  for (int64_t i = 0; i < n; ++i) {  // Force += computed (gravity.rs:71-73)
    fx[i] += h[i];
    fy[i] += h[n + i];
    fz[i] += h[2 * n + i];
  }
  return PHYS_OK;
}

int phys_nfw_forces(phys_ctx* c, const phys_nfw_halo* halo, double* fx, double* fy, double* fz) {
  PHYS_ENTER(c);
  if (!halo) return fail(c, PHYS_ERR_ARG, "halo is NULL");
  if (halo->reserved != 0) return fail(c, PHYS_ERR_ARG, "phys_nfw_halo.reserved must be 0");
  if (!halo->enabled) return PHYS_OK;  // nfw.rs:108-110
  if (!fx || !fy || !fz) return fail(c, PHYS_ERR_ARG, "force arrays are required");
  const int64_t n = c->n;
  if (n == 0) return PHYS_OK;
  PHYS_TRY(reset_status(c));
  PHYS_CUDA(c, cudaMemsetAsync(c->fx, 0, sizeof(double) * n, c->stream));
  PHYS_CUDA(c, cudaMemsetAsync(c->fy, 0, sizeof(double) * n, c->stream));
  PHYS_CUDA(c, cudaMemsetAsync(c->fz, 0, sizeof(double) * n, c->stream));
  const int64_t cap = c->sec_cap;  // the halo reads LocalPosition (nfw.rs:118)
  PHYS_TRY(nfw_add_forces(c, *halo, c->sector_mode ? c->loc : c->x,
                          c->sector_mode ? c->loc + cap : c->y,
                          c->sector_mode ? c->loc + 2 * cap : c->z, c->fx, c->fy, c->fz));
  PHYS_TRY(ensure_pinned(c, sizeof(double) * 3 * n));
  double* h = static_cast<double*>(c->h_stage);
  PHYS_TRY(d2h(c, h, c->fx, n));
  PHYS_TRY(d2h(c, h + n, c->fy, n));
  PHYS_TRY(d2h(c, h + 2 * n, c->fz, n));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  c->last_eval_bh = false;
  c->last_eval_group = false;
  PHYS_TRY(finish_status(c));
  for (int64_t i = 0; i < n; ++i) {  // force.0 += f_vec (nfw.rs:138)
    fx[i] += h[i];
    fy[i] += h[n + i];
    fz[i] += h[2 * n + i];
  }
  return PHYS_OK;
}

int phys_set_nfw_halo(phys_ctx* c, const phys_nfw_halo* halo) {
  PHYS_ENTER(c);
  if (halo && halo->reserved != 0) return fail(c, PHYS_ERR_ARG, "phys_nfw_halo.reserved must be 0");
  c->halo_on = halo && halo->enabled;
  if (halo) c->halo = *halo;
  c->accel_valid = false;  // a(x) changes with the halo
  return PHYS_OK;
}

int phys_gravity_accel(phys_ctx* c, const phys_params* p, double* ax, double* ay, double* az) {
  PHYS_ENTER(c);
  PHYS_TRY(check_params(c, p));
  if (c->n == 0) return fail(c, PHYS_ERR_STATE, "no body state uploaded");
  PHYS_TRY(reset_status(c));
  PHYS_CUDA(c, cudaEventRecord(c->ev[0], c->stream));
  PHYS_TRY(eval(c, p, false));
  PHYS_CUDA(c, cudaEventRecord(c->ev[1], c->stream));
  c->accel_valid = true;
  c->accel_params = *p;
  PHYS_TRY(d2h(c, ax, c->ax, c->n));
  PHYS_TRY(d2h(c, ay, c->ay, c->n));
  PHYS_TRY(d2h(c, az, c->az, c->n));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  int st = finish_status(c);
  c->tm.total_ms = ev_ms(c->ev[0], c->ev[1]);
  return st;
}

int64_t phys_share_chunk(int64_t n, int32_t world) {
  return (n < 0 || world < 1) ? -1 : share_chunk(n, world);
}

int phys_gravity_accel_share(phys_ctx* c, const phys_params* p, int32_t rank, int32_t world,
                             double* share_out) {
  PHYS_ENTER(c);
  PHYS_TRY(check_params(c, p));
  if (c->n == 0) return fail(c, PHYS_ERR_STATE, "no body state uploaded");
  if (world < 1 || rank < 0 || rank >= world)
    return fail(c, PHYS_ERR_ARG, "share %d of %d", (int)rank, (int)world);
  if (!share_out) return fail(c, PHYS_ERR_ARG, "share_out is required");
  const int64_t n = c->n, chunk = share_chunk(n, world);
  const int64_t lo = min64(n, (int64_t)rank * chunk), hi = min64(n, lo + chunk);
  PHYS_TRY(reset_status(c));
  // the evaluation writes the share's targets (and the rest of their
  // groups); zero first, so that no target outside holds a stale or
  // non-finite value
  double* o[3] = {c->ax, c->ay, c->az};
  if (c->halo_on) o[0] = c->fx, o[1] = c->fy, o[2] = c->fz;
  for (double* a : o) PHYS_CUDA(c, cudaMemsetAsync(a, 0, sizeof(double) * n, c->stream));
  PHYS_CUDA(c, cudaEventRecord(c->ev[0], c->stream));
  c->share_lo = lo;
  c->share_hi = hi;
  const int st_eval = eval(c, p, false);
  c->share_lo = 0;
  c->share_hi = -1;
  PHYS_TRY(st_eval);
  uint32_t* perm = nullptr;
  if (p->method == PHYS_BARNES_HUT && n >= 2) {
    // keep the tree's order for the scatter in a slot of its own
    PHYS_TRY(ws_alloc(c, WS_SHARE_PERM, n, &perm));
    PHYS_CUDA(c, cudaMemcpyAsync(perm, c->share_perm, sizeof(uint32_t) * n,
                                 cudaMemcpyDeviceToDevice, c->stream));
  }
  PHYS_TRY(share_pack(c, lo, hi, chunk, perm, share_out));
  PHYS_CUDA(c, cudaEventRecord(c->ev[1], c->stream));
  c->accel_valid = false;  // the acceleration arrays hold this share only
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  int st = finish_status(c);
  c->tm.total_ms = ev_ms(c->ev[0], c->ev[1]);
  if (st == PHYS_OK) {
    c->share_world = world;
    c->share_perm = perm;
    c->share_params = *p;
  }
  return st;
}

int phys_gravity_accel_unshare(phys_ctx* c, int32_t world, const double* gathered) {
  PHYS_ENTER(c);
  if (c->share_world == 0)
    return fail(c, PHYS_ERR_STATE, "no share evaluation to complete on this context");
  if (world != c->share_world)
    return fail(c, PHYS_ERR_ARG, "world %d differs from the share evaluation's %d", (int)world,
                (int)c->share_world);
  if (!gathered) return fail(c, PHYS_ERR_ARG, "gathered is required");
  PHYS_TRY(reset_status(c));
  PHYS_TRY(share_unpack(c, share_chunk(c->n, world), c->share_perm, gathered));
  c->share_world = 0;
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  int32_t st = 0;
  PHYS_TRY(read_status(c, &st));
  if (st & kStatNonfinite)
    return fail(c, PHYS_ERR_NONFINITE, "non-finite value in the gathered accelerations");
  c->accel_valid = true;
  c->accel_params = c->share_params;
  return PHYS_OK;
}

int phys_direct_accel_targets(phys_ctx* c, const phys_params* p, int64_t nt,
                              const int64_t* targets, double* ax, double* ay, double* az) {
  PHYS_ENTER(c);
  PHYS_TRY(check_params(c, p));
  PHYS_TRY(positions_ready(c, false));
  if (nt < 0 || (nt > 0 && (!targets || !ax || !ay || !az)))
    return fail(c, PHYS_ERR_ARG, "targets and outputs are required");
  if (c->n < 2 || nt == 0) {
    for (int64_t k = 0; k < nt; ++k) ax[k] = ay[k] = az[k] = 0.0;
    return PHYS_OK;
  }
  int st = PHYS_OK;
  int64_t* dt = (int64_t*)ws_get(c, WS_ADJ3, sizeof(int64_t) * nt, &st);
  if (st) return st;
  double* out = (double*)ws_get(c, WS_ADJ2, sizeof(double) * 3 * nt, &st);
  if (st) return st;
  PHYS_TRY(reset_status(c));
  PHYS_CUDA(c, cudaMemcpyAsync(dt, targets, sizeof(int64_t) * nt, cudaMemcpyHostToDevice, c->stream));
  PHYS_TRY(direct_targets(c, p, nt, dt, out, out + nt, out + 2 * nt));
  PHYS_TRY(d2h(c, ax, out, nt));
  PHYS_TRY(d2h(c, ay, out + nt, nt));
  PHYS_TRY(d2h(c, az, out + 2 * nt, nt));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  int32_t sw = 0;
  PHYS_TRY(read_status(c, &sw));
  if (sw & kStatOverflow) return fail(c, PHYS_ERR_ARG, "target index out of range");
  if (sw & kStatNonfinite) return fail(c, PHYS_ERR_NONFINITE, "non-finite result");
  return PHYS_OK;
}

int phys_verlet_steps(phys_ctx* c, const phys_params* p, double dt, int64_t nsteps) {
  PHYS_ENTER(c);
  return verlet_steps(c, p, dt, nsteps, true);
}

// Whether every pointer is page-locked host memory (an asynchronous copy
// from it does not wait for the host).
static bool all_pinned(const double* const* a, int k) {
  for (int i = 0; i < k; ++i) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, a[i]) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    if (at.type != cudaMemoryTypeHost) return false;
  }
  return true;
}

int phys_verlet_tick_host(phys_ctx* c, const phys_params* p, double dt, int64_t n, double* x,
                          double* y, double* z, double* vx, double* vy, double* vz,
                          const double* m, double* ax, double* ay, double* az) {
  PHYS_ENTER(c);
  if (!x || !y || !z || !vx || !vy || !vz || !m || !ax || !ay || !az)
    return fail(c, PHYS_ERR_ARG, "every state array is required");
  PHYS_TRY(phys_state_upload(c, n, x, y, z, vx, vy, vz, m));
  if (n == 0) return PHYS_OK;
  PHYS_TRY(h2d(c, c->ax, ax, n));
  PHYS_TRY(h2d(c, c->ay, ay, n));
  PHYS_TRY(h2d(c, c->az, az, n));
  c->accel_valid = true;
  c->accel_params.method = -1;  // the caller's Acceleration component
  const double* xs[3] = {x, y, z};
  const bool early = all_pinned(xs, 3);
  if (early) {
    c->copy_x[0] = x;
    c->copy_x[1] = y;
    c->copy_x[2] = z;
  }
  const int st_run = verlet_steps(c, p, dt, 1, false);
  c->copy_x[0] = c->copy_x[1] = c->copy_x[2] = nullptr;
  if (early) PHYS_CUDA(c, cudaStreamWaitEvent(c->stream, c->copy_done, 0));
  PHYS_TRY(st_run);
  if (!early) {
    PHYS_TRY(d2h(c, x, c->x, n));
    PHYS_TRY(d2h(c, y, c->y, n));
    PHYS_TRY(d2h(c, z, c->z, n));
  }
  PHYS_TRY(d2h(c, vx, c->vx, n));
  PHYS_TRY(d2h(c, vy, c->vy, n));
  PHYS_TRY(d2h(c, vz, c->vz, n));
  PHYS_TRY(d2h(c, ax, c->ax, n));
  PHYS_TRY(d2h(c, ay, c->ay, n));
  PHYS_TRY(d2h(c, az, c->az, n));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  const int st = finish_status(c);
  c->tm.total_ms = ev_ms(c->ev[0], c->ev[1]);
  return st;
}

int phys_verlet_steps_async(phys_ctx* c, const phys_params* p, double dt, int64_t nsteps) {
  PHYS_ENTER(c);
  return verlet_steps(c, p, dt, nsteps, false);
}

int phys_diagnostics(phys_ctx* c, double G, double* out5) {
  if (!c || !out5) return PHYS_ERR_ARG;
  PHYS_ENTER(c);
  if (c->n == 0) return fail(c, PHYS_ERR_STATE, "no body state uploaded");
  PHYS_TRY(positions_ready(c, false));
  return diagnostics(c, G, out5);
}

int phys_bh_export(phys_ctx* c, const phys_params* p, int64_t cap, int64_t* nnodes,
                   int32_t* depth, int64_t* count, double* mass, double* com,
                   int64_t* leaf_body, int64_t* body_leaf, uint64_t* keys_hi, uint64_t* keys_lo,
                   int64_t* perm, double* root4) {
  PHYS_ENTER(c);
  PHYS_TRY(check_params(c, p));
  PHYS_TRY(positions_ready(c, true));
  if (c->n < 2) return fail(c, PHYS_ERR_STATE, "need at least 2 bodies");
  if (cap < 0) return fail(c, PHYS_ERR_ARG, "cap < 0");
  PHYS_TRY(reset_status(c));
  PHYS_TRY(bh_export(c, p, cap, nnodes, depth, count, mass, com, leaf_body, body_leaf, keys_hi,
                     keys_lo, perm, root4));
  return finish_status(c);
}

int phys_ensemble_load(phys_ctx* c, int64_t nsys, const int64_t* off, const double* x,
                       const double* y, const double* z, const double* vx, const double* vy,
                       const double* vz, const double* m) {
  PHYS_ENTER(c);
  if (nsys <= 0 || !off || !x || !y || !z || !m)
    return fail(c, PHYS_ERR_ARG, "nsys > 0, offsets, positions and masses are required");
  return ensemble_load(c, nsys, off, x, y, z, vx, vy, vz, m);
}

int phys_ensemble_run(phys_ctx* c, const phys_params* p, double dt, int64_t nsteps,
                      int32_t group, int64_t chunk) {
  if (!c || !p) return PHYS_ERR_ARG;
  PHYS_ENTER(c);
  if (p->precision != PHYS_F64_EXACT && p->precision != PHYS_F32C)
    return fail(c, PHYS_ERR_ARG, "ensemble precision must be F64_EXACT or F32C");
  if (nsteps < 0 || chunk < 0) return fail(c, PHYS_ERR_ARG, "nsteps and chunk must be >= 0");
  PHYS_TRY(reset_status(c));
  if (group == 0) {
    if (c->ens_group == 0) PHYS_TRY(ensemble_autotune(c, p, dt, 8, nullptr, nullptr));
    group = c->ens_group;
  }
  PHYS_TRY(ensemble_run(c, p, dt, nsteps, group, chunk));
  c->tm.walk_ms = ev_ms(c->ev[6], c->ev[7]);
  c->last_eval_bh = false;
  c->last_eval_group = false;
  int32_t sw = 0;
  PHYS_TRY(read_status(c, &sw));
  if (sw & kStatOverflow) return fail(c, PHYS_ERR_ARG, "system larger than 64 bodies");
  if (sw & kStatNonfinite) return fail(c, PHYS_ERR_NONFINITE, "non-finite ensemble state");
  return PHYS_OK;
}

int phys_ensemble_download(phys_ctx* c, double* x, double* y, double* z, double* vx, double* vy,
                           double* vz, double* ax, double* ay, double* az) {
  PHYS_ENTER(c);
  if (c->ens_nsys <= 0) return fail(c, PHYS_ERR_STATE, "no ensemble loaded");
  return ensemble_download(c, x, y, z, vx, vy, vz, ax, ay, az);
}

int phys_ensemble_autotune(phys_ctx* c, const phys_params* p, double dt, int64_t probe_steps,
                           int32_t* best, double* ms3) {
  if (!c || !p) return PHYS_ERR_ARG;
  PHYS_ENTER(c);
  if (probe_steps <= 0) return fail(c, PHYS_ERR_ARG, "probe_steps must be > 0");
  PHYS_TRY(reset_status(c));
  return ensemble_autotune(c, p, dt, probe_steps, best, ms3);
}

int phys_adjoint_direct(phys_ctx* c, const phys_params* p, double dt, int64_t nsteps,
                        int64_t checkpoint, const double* tx, const double* ty, const double* tz,
                        double* loss, double* gx, double* gy, double* gz, double* gvx,
                        double* gvy, double* gvz, double* gm) {
  if (!c || !loss) return PHYS_ERR_ARG;
  PHYS_ENTER(c);
  PHYS_TRY(reset_status(c));
  PHYS_TRY(positions_ready(c, false));
  PHYS_CUDA(c, cudaEventRecord(c->ev[0], c->stream));
  double* gxyz[3] = {gx, gy, gz};
  double* gvxyz[3] = {gvx, gvy, gvz};
  PHYS_TRY(adjoint(c, p, dt, nsteps, checkpoint, tx, ty, tz, loss, gxyz, gvxyz, gm));
  PHYS_CUDA(c, cudaEventRecord(c->ev[1], c->stream));
  c->last_eval_bh = false;
  c->last_eval_group = false;
  int st = finish_status(c);
  c->tm.total_ms = ev_ms(c->ev[0], c->ev[1]);
  return st;
}

int phys_trajectory_loss(phys_ctx* c, const phys_params* p, double dt, int64_t nsteps,
                         const double* tx, const double* ty, const double* tz, double* loss,
                         double* xT, double* yT, double* zT) {
  if (!c || !loss) return PHYS_ERR_ARG;
  PHYS_ENTER(c);
  PHYS_TRY(reset_status(c));
  PHYS_TRY(positions_ready(c, false));
  PHYS_TRY(trajectory_loss(c, p, dt, nsteps, tx, ty, tz, loss, xT, yT, zT));
  c->last_eval_bh = false;
  c->last_eval_group = false;
  return finish_status(c);
}

int phys_debug_set_wait_limit(phys_ctx* c, int64_t spins) {
  if (!c) return PHYS_ERR_ARG;
  c->sort_spin_limit = spins < 0 ? (int64_t(1) << 20) : spins;
  return PHYS_OK;
}

int phys_debug_divide(phys_ctx* c, int64_t n, const double* a, const double* b, double* q) {
  if (!c || n < 0 || (n > 0 && (!a || !b || !q))) return PHYS_ERR_ARG;
  PHYS_ENTER(c);
  return debug_divide(c, n, a, b, q);
}

int phys_probe_peaks(phys_ctx* c, double* fp32, double* fp32x2, double* fp64) {
  if (!c || !fp32 || !fp32x2 || !fp64) return PHYS_ERR_ARG;
  PHYS_ENTER(c);
  return probe_peaks(c, fp32, fp32x2, fp64);
}

}  // extern "C"
