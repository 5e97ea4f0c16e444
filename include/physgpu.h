/*
 * physgpu.h -- C ABI of the B200 gravity library (libphysgpu.so).
 *
 * This is the drop-in boundary for the gravity path of Doritozzzz/phys-rs.
 * The reference has no FFI for this path: its "plugin API" is a set of
 * bevy_ecs system functions registered in a Schedule (src/main.rs:103-140).
 * Each entry point below names the reference system or code whose work it
 * replaces, so a Rust `extern "C"` block can wrap them in systems of the
 * same signatures.
 *
 * Conventions
 *  - Plain pointers and sizes; arrays are structure-of-arrays, f64, length n,
 *    in the caller's (ECS query) order.  Host pointers, except the DEVICE
 *    buffers of phys_direct_accel_noalloc and of the target-share calls
 *    (phys_gravity_accel_share / _unshare), as their comments say.
 *  - Every call returns a status (PHYS_OK == 0).  No call aborts, throws or
 *    traps; on error phys_last_error() describes it.
 *  - A context owns its CUDA streams (a main stream, and a second one that
 *    forks from and joins back into it within a call) and all device memory
 *    it uses.  It is not thread-safe (use one context per thread); contexts
 *    share no state, and every call makes its context's device current, so
 *    contexts on several devices may be used from one thread.  Calls
 *    are synchronous at return, like the reference's blocking readback
 *    (src/gpu/buffers.rs:163-213), except phys_verlet_steps_async.
 *  - Body state stays resident on the device between calls, so multi-step
 *    runs do not cross PCIe.
 */
#ifndef PHYSGPU_H
#define PHYSGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PHYS_OK 0
#define PHYS_ERR_ARG 1        /* bad argument (null pointer, size, enum)      */
#define PHYS_ERR_CUDA 2       /* CUDA runtime error                           */
#define PHYS_ERR_OOM 3        /* device or pinned allocation failed           */
#define PHYS_ERR_NONFINITE 4  /* NaN/Inf in inputs or results                 */
#define PHYS_ERR_TIMEOUT 5    /* a bounded device-side wait gave up           */
#define PHYS_ERR_STATE 6      /* call order (e.g. no state uploaded)          */

/* ---- force method / precision ----------------------------------------- */
#define PHYS_DIRECT 0         /* brute_force_gravity_system (gravity.rs:27-74)         */
#define PHYS_BARNES_HUT 1     /* barnes_hut_gravity_system (gravity_tree.rs:260-338)   */

#define PHYS_F64_EXACT 0      /* reference op order, IEEE sqrt/div, no FMA, reference
                                 summation order (direct: j order; BH: nested child
                                 sums, insertion-order centre of mass): bit-identical
                                 to the reference's f64 arithmetic                    */
#define PHYS_F64 1            /* f64 with FMA and rsqrt, flat sums, parallel COM     */
#define PHYS_F32C 2           /* f32 pair terms on double-float relative coordinates,
                                 two-sum compensated f32 accumulation, f64 state     */

/* Barnes-Hut walk per group of 64 key-adjacent bodies (PHYS_F64 and
 * PHYS_F32C only): a cell is taken as a monopole only when the reference's
 * criterion (2h)^2 < theta^2 d^2 holds for the nearest point of the group's
 * bounding box (so for every body of the group); the accepted cells and the
 * bodies of opened leaves form one interaction list that the whole group
 * evaluates, and pairs inside the group are exact.  No cell is taken as a
 * monopole that the per-body criterion would open, and every pair the
 * per-body walk takes exactly stays exact; the walk order and the sums are
 * not the reference's.  No counterpart in the reference
 * (gravity_tree.rs:171-209 walks per body). */
#define PHYS_FLAG_GROUP_WALK 1

typedef struct phys_ctx phys_ctx;

/* UniverseConfig (src/core/config.rs:26-59) fields the gravity path reads,
 * plus the method switches. */
typedef struct phys_params {
  double G;           /* gravitational_constant                               */
  double eps;         /* softening_epsilon (eps^2 is added to r^2)            */
  double theta;       /* barnes_hut_theta                                     */
  int32_t method;     /* PHYS_DIRECT or PHYS_BARNES_HUT                       */
  int32_t precision;  /* PHYS_F64_EXACT, PHYS_F64 or PHYS_F32C                */
  int32_t leaf_cap;   /* BH leaf capacity: 1 = the reference octree; 2..16 =
                         bucket leaves (criterion on the cell, exact pairs when
                         opened).  F64_EXACT requires 1.                      */
  int32_t flags;      /* 0, or PHYS_FLAG_GROUP_WALK                          */
} phys_params;

/* Per-call device timings of the last force evaluation / step (CUDA events
 * on the context's stream) and counters. */
typedef struct phys_timings {
  double total_ms;      /* whole last call                                    */
  double bbox_ms;       /* bounding cube (gravity_tree.rs:305-317)            */
  double keys_ms;       /* descent keys                                       */
  double sort_ms;       /* radix sort + equal-prefix fixup                    */
  double tree_ms;       /* topology, mass and centre of mass                  */
  double walk_ms;       /* theta walk or direct-sum kernel                    */
  double verlet_ms;     /* kick/drift kernels                                 */
  uint64_t interactions;/* pair + monopole interactions of the last evaluation */
  uint64_t launches;    /* kernels launched by this context since creation    */
  int64_t nodes;        /* octree nodes of the last BH evaluation             */
  int32_t max_depth;    /* guard depth D* of the last BH tree                 */
  int32_t reserved;
  double walk_eval_ms;  /* group walk: the list-evaluation kernel alone (part
                           of walk_ms); 0 for the other walks              */
  uint64_t walk_eval_interactions; /* group walk: interactions evaluated by
                           that kernel (the rest: re-queued subgroups)      */
} phys_timings;

/* ---- context ------------------------------------------------------------ */
const char* phys_status_string(int status);
const char* phys_last_error(const phys_ctx* ctx);
int phys_ctx_create(int device, phys_ctx** out);
int phys_ctx_destroy(phys_ctx* ctx);
/* The cudaStream_t the context launches on (for callers that time or order
 * work around it).  Work the context puts on its second stream is joined
 * back into this one before the call returns or queues anything after it. */
void* phys_ctx_stream(phys_ctx* ctx);
int phys_last_timings(const phys_ctx* ctx, phys_timings* out);

/* ---- body state --------------------------------------------------------- */
/* Upload absolute positions, velocities (may be NULL: zero) and masses
 * (the Mass / LocalPosition / Velocity components of the query).  Invalidates
 * the cached acceleration. */
int phys_state_upload(phys_ctx* ctx, int64_t n, const double* x, const double* y,
                      const double* z, const double* vx, const double* vy, const double* vz,
                      const double* m);
/* Same, from (Sector, LocalPosition) pairs: positions are flattened on the
 * device as (sector - origin) * sector_size + local with origin = the first
 * body's sector (gravity.rs:38-47).  With bh_quirk != 0 every body is
 * measured from its own sector, as barnes_hut_gravity_system does
 * (gravity_tree.rs:280-291: `first` is never cleared). */
int phys_state_upload_sectors(phys_ctx* ctx, int64_t n, const int64_t* sx, const int64_t* sy,
                              const int64_t* sz, const double* lx, const double* ly,
                              const double* lz, double sector_size, int32_t bh_quirk,
                              const double* vx, const double* vy, const double* vz,
                              const double* m);
/* Keep the (Sector, LocalPosition) components themselves on the device
 * (src/core/coordinates.rs).  Afterwards every force pass flattens them
 * (origin: the first body's sector for the direct sum, each body's own for
 * Barnes-Hut, gravity_tree.rs:280-291), phys_verlet_steps integrates
 * LocalPosition and runs sector_boundary_system (src/physics/origin.rs:16-24,
 * normalize_position in coordinates.rs:82-103) after every velocity step, as
 * the reference schedule does (src/main.rs:149), and the POSITION component
 * and phys_state_download's positions are LocalPosition.  A tick in which a
 * body changed sector costs a second force pass (the reference always runs
 * two).  phys_state_upload / phys_state_upload_sectors leave this mode. */
int phys_state_upload_sector_state(phys_ctx* ctx, int64_t n, const int64_t* sx,
                                   const int64_t* sy, const int64_t* sz, const double* lx,
                                   const double* ly, const double* lz, double sector_size,
                                   const double* vx, const double* vy, const double* vz,
                                   const double* m);
/* The Sector (any of sx/sy/sz may be NULL) and LocalPosition components of a
 * context in that mode. */
int phys_state_download_sector_state(phys_ctx* ctx, int64_t* sx, int64_t* sy, int64_t* sz,
                                     double* lx, double* ly, double* lz);
/* Set the Acceleration component (the a(x_n) a Velocity-Verlet tick starts
 * from) and mark it valid for phys_verlet_steps. */
int phys_state_set_accel(phys_ctx* ctx, const double* ax, const double* ay, const double* az);
/* Download any of positions, velocities, accelerations (NULL skips). */
int phys_state_download(phys_ctx* ctx, double* x, double* y, double* z, double* vx, double* vy,
                        double* vz, double* ax, double* ay, double* az);
int64_t phys_state_size(const phys_ctx* ctx);

/* Per-component access to the device-resident state, one ECS component at a
 * time (src/components/dynamics.rs:13-37, src/core/coordinates.rs:26).
 * MASS uses only the first pointer.  Writing POSITION or MASS invalidates the
 * cached acceleration; writing ACCELERATION marks it valid. */
#define PHYS_COMP_POSITION 0
#define PHYS_COMP_VELOCITY 1
#define PHYS_COMP_ACCELERATION 2
#define PHYS_COMP_PREV_ACCELERATION 3
#define PHYS_COMP_MASS 4
int phys_component_write(phys_ctx* ctx, int32_t component, const double* a, const double* b,
                         const double* c);
int phys_component_read(phys_ctx* ctx, int32_t component, double* a, double* b, double* c);

/* ---- gravity (one force evaluation at the uploaded positions) ---------- */
/* brute_force_gravity_system / barnes_hut_gravity_system: ADDS the
 * gravitational force to fx/fy/fz (Force += F, gravity.rs:71-73,
 * gravity_tree.rs:333-337).  Returns without touching them for n < 2
 * (gravity.rs:49-51). */
int phys_gravity_forces(phys_ctx* ctx, const phys_params* p, double* fx, double* fy, double* fz);
/* The same evaluation followed by compute_acceleration_system (a = F/m,
 * integrators.rs:110-118) with Force reset to zero first (forces.rs:15-19).
 * Writes ax/ay/az (each may be NULL to keep the result on the device only)
 * and caches a(x) for phys_verlet_steps. */
int phys_gravity_accel(phys_ctx* ctx, const phys_params* p, double* ax, double* ay, double* az);

/* Direct-sum accelerations (a = F/m, all n sources) for a subset of targets:
 * targets[k] in [0, n), results in ax[k] (host arrays of length nt).  Used as
 * the f64 direct-sum reference for Barnes-Hut runs at sizes where the full
 * O(N^2) sum is too costly.  p->method is ignored (direct sum). */
int phys_direct_accel_targets(phys_ctx* ctx, const phys_params* p, int64_t nt,
                              const int64_t* targets, double* ax, double* ay, double* az);

/* ---- target shares: one system split over GPUs ------------------------- */
/* No counterpart in the reference (it runs on one CPU).  Every GPU holds the
 * whole state (same upload, same integration), and each evaluates a share
 * of the targets of the phys_gravity_accel evaluation: share `rank` of
 * `world` covers targets [rank*c, min(n, (rank+1)*c)), c =
 * phys_share_chunk(n, world) (a multiple of 128), by body index for the
 * direct sum and by sorted (key-order) position for Barnes-Hut, whose every
 * GPU builds the same tree.  The values equal a one-GPU evaluation's bit for
 * bit: a target's sum does not depend on the share that computes it.
 *
 * phys_share_chunk: targets per share (-1 for n < 0 or world < 1). */
int64_t phys_share_chunk(int64_t n, int32_t world);
/* Evaluates share `rank` of `world` (accelerations a = F/m, with the NFW
 * halo when one is set) and packs them into share_out, a DEVICE buffer of
 * 3*c doubles on this context's device: ax | ay | az of the share's targets
 * in target order, zero-padded to c.  Synchronous at return.  The caller
 * then all-gathers the world blocks (rank r's block at offset r*3*c, e.g.
 * ncclAllGather over NVLink, 24 bytes per body) and completes the
 * evaluation with phys_gravity_accel_unshare before any other evaluation on
 * this context. */
int phys_gravity_accel_share(phys_ctx* ctx, const phys_params* p, int32_t rank, int32_t world,
                             double* share_out);
/* Scatters the gathered blocks (DEVICE buffer, world*3*c doubles) into the
 * context's acceleration arrays for all n bodies and caches them as the
 * evaluation's result (as phys_gravity_accel does), so that
 * phys_vv_position_step / phys_vv_velocity_step continue from it.
 * PHYS_ERR_STATE without a preceding share evaluation; PHYS_ERR_NONFINITE
 * if a gathered value is not finite. */
int phys_gravity_accel_unshare(phys_ctx* ctx, int32_t world, const double* gathered);

/* ---- NFW phantom halo (src/physics/nfw.rs) ------------------------------ */
/* NfwHaloConfig (nfw.rs:24-47): rho(r) = rho_0 / ((r/Rs)(1 + r/Rs)^2),
 * centred at `center` (local coordinates). */
typedef struct phys_nfw_halo {
  double rho_0;         /* central characteristic density [kg m^-3]          */
  double scale_radius;  /* Rs [m]                                            */
  double center[3];     /* halo centre, local coordinates [m]                */
  int32_t enabled;      /* 0: the system and the fused term do nothing       */
  int32_t reserved;     /* must be 0                                         */
} phys_nfw_halo;

/* nfw_density, nfw_enclosed_mass, nfw_circular_velocity (nfw.rs:61-92):
 * host-side scalars, the reference's formulas and operation order (0 for
 * r <= 0 or Rs <= 0; G is constants.rs:7). */
double phys_nfw_density(double r, double rho_0, double rs);
double phys_nfw_enclosed_mass(double r, double rho_0, double rs);
double phys_nfw_circular_velocity(double r, double rho_0, double rs);

/* nfw_gravity_system (nfw.rs:103-139) on the device: adds
 * -G M(r) m / r^2 * r_hat to fx/fy/fz (Force +=) for every body of the
 * context, r measured from the halo centre to the body's position as
 * uploaded, bodies closer than 1e-10 m skipped.  G = 6.67430e-11
 * (constants.rs:7), not phys_params.G, as in the reference.  Nothing happens
 * when the halo is disabled. */
int phys_nfw_forces(phys_ctx* ctx, const phys_nfw_halo* halo, double* fx, double* fy,
                    double* fz);
/* Makes every later acceleration of this context (phys_gravity_accel,
 * phys_verlet_steps) include the halo the way the reference schedule does
 * (src/main.rs:109-110,128-129: gravity, then nfw_gravity_system, then
 * a = F/m): a = (F_gravity + F_nfw) / m.  NULL or enabled == 0 removes it.
 * Invalidates the cached acceleration. */
int phys_set_nfw_halo(phys_ctx* ctx, const phys_nfw_halo* halo);

/* ---- integration -------------------------------------------------------- */
/* nsteps Velocity-Verlet ticks on the device-resident state: each tick is
 * velocity_verlet_position_system (integrators.rs:63-83), a force evaluation
 * + a = F/m, velocity_verlet_velocity_system (integrators.rs:92-104).
 * The reference evaluates gravity twice per tick (src/main.rs:109,128); the
 * first evaluation repeats the previous tick's second one at the same
 * positions, so it is taken from the cache: the trajectory is the same. */
int phys_verlet_steps(phys_ctx* ctx, const phys_params* p, double dt, int64_t nsteps);
/* The two halves of the tick as separate systems, on the device state:
 * velocity_verlet_position_system (PreviousAcceleration = Acceleration;
 * x += v dt + a dt^2/2) and velocity_verlet_velocity_system
 * (v += (PreviousAcceleration + Acceleration) dt/2). */
int phys_vv_position_step(phys_ctx* ctx, double dt);
int phys_vv_velocity_step(phys_ctx* ctx, double dt);
/* As phys_verlet_steps but returns once the work is enqueued on the
 * context's stream (host sync only for the BH node count). */
int phys_verlet_steps_async(phys_ctx* ctx, const phys_params* p, double dt, int64_t nsteps);
/* One tick on host state in one call, the work of phys_state_upload +
 * phys_state_set_accel (a: the Acceleration component, PreviousAcceleration
 * of the position step) + phys_verlet_steps(1) + phys_state_download,
 * results in place (x, v, a; m is read only).  When x, y, z are page-locked
 * (cudaHostAlloc / cudaHostRegister) their copy back runs while the force
 * pass computes.  Synchronous at return. */
int phys_verlet_tick_host(phys_ctx* ctx, const phys_params* p, double dt, int64_t n, double* x,
                          double* y, double* z, double* vx, double* vy, double* vz,
                          const double* m, double* ax, double* ay, double* az);

/* ---- batched ensemble of independent small systems ------------------- */
/* Thousands of independent systems (1..64 bodies each) in CSR layout:
 * system s owns bodies [offsets[s], offsets[s+1]), offsets[0] == 0.  Each
 * system evolves under the reference's direct-sum Velocity-Verlet tick
 * (gravity.rs:53-69, integrators.rs:63-118) with no coupling between
 * systems.  Loading invalidates the cached accelerations. */
int phys_ensemble_load(phys_ctx* ctx, int64_t nsys, const int64_t* offsets, const double* x,
                       const double* y, const double* z, const double* vx, const double* vy,
                       const double* vz, const double* m);
/* nsteps ticks of every system in persistent kernels (one launch per
 * `chunk` steps, 0 = all steps in one launch), the launches captured in a
 * CUDA graph.  `config` chooses the launch shape: lanes per system (8, 16
 * or 32: 32 / lanes systems per warp at a time; or PHYS_ENS_BY_SIZE: 32
 * lanes for systems of more than 16 bodies, 16 for 9..16, 8 for at most 8,
 * a warp moving on to the smaller systems once the larger ones are taken),
 * plus optionally PHYS_ENS_WARPS(2 or 4) warps per block (default 2); 0 =
 * the autotuned configuration (autotuning on first use).  With 32 lanes, a
 * system of 33..64 bodies gives every lane one target and shares the
 * remaining targets among lane streams that each take a part of the sources.
 * p->precision: F64_EXACT or F32C; method and theta are ignored. */
#define PHYS_ENS_BY_SIZE 1
#define PHYS_ENS_WARPS(w) ((w) << 8)
#define PHYS_ENS_CANDIDATES 6
int phys_ensemble_run(phys_ctx* ctx, const phys_params* p, double dt, int64_t nsteps,
                      int32_t config, int64_t chunk);
int phys_ensemble_download(phys_ctx* ctx, double* x, double* y, double* z, double* vx,
                           double* vy, double* vz, double* ax, double* ay, double* az);
/* Times probe_steps steps of each of the PHYS_ENS_CANDIDATES configurations
 * from the current state (restored afterwards) and keeps the fastest for
 * later runs: lanes per system 8, 16, 32 and PHYS_ENS_BY_SIZE with 2 warps
 * per block, then 32 and PHYS_ENS_BY_SIZE with 4 warps per block, in that
 * order.  best_config receives the chosen code; ms (optional, room for
 * PHYS_ENS_CANDIDATES) the timings in the same order. */
int phys_ensemble_autotune(phys_ctx* ctx, const phys_params* p, double dt, int64_t probe_steps,
                           int32_t* best_config, double* ms);

/* ---- trajectory gradients (hand-written adjoint) ------------------------ */
/* No counterpart in the reference (it has no differentiation).  Loss
 *   L = sum_i |x_i(T) - target_i|^2
 * after nsteps Velocity-Verlet ticks (integrators.rs:63-104) of the direct
 * sum (gravity.rs:53-69), p->precision must be PHYS_F64, started from the
 * uploaded state (which is left unchanged).  phys_adjoint_direct returns L
 * and dL/dx0, dL/dv0, dL/dm (each output may be NULL) by a reverse sweep
 * through the acceleration's Jacobian and the Verlet step, checkpointing
 * (x, v) every `checkpoint` steps and recomputing each segment.
 * phys_trajectory_loss is the same forward pass only (finite differences). */
int phys_adjoint_direct(phys_ctx* ctx, const phys_params* p, double dt, int64_t nsteps,
                        int64_t checkpoint, const double* tx, const double* ty, const double* tz,
                        double* loss, double* gx, double* gy, double* gz, double* gvx,
                        double* gvy, double* gvz, double* gm);
int phys_trajectory_loss(phys_ctx* ctx, const phys_params* p, double dt, int64_t nsteps,
                         const double* tx, const double* ty, const double* tz, double* loss,
                         double* xT, double* yT, double* zT);

/* ---- diagnostics (src/physics/energy.rs:21-56, integrators.rs:123-129) -- */
/* out[0] = kinetic energy sum 1/2 m v^2, out[1] = unsoftened potential energy
 * -sum_{i<j} G m_i m_j / r (r^2 == 0 pairs skipped), out[2..4] = total linear
 * momentum sum m v.  f64 on the device with compensated sums. */
int phys_diagnostics(phys_ctx* ctx, double G, double* out5);

/* ---- Barnes-Hut tree export (parity checks) ----------------------------- */
/* Builds the octree for the uploaded positions with params p (method is
 * ignored) and exports, in pre-order over non-empty cells (children in
 * octant order 0..7, the order compute_force visits them):
 *   depth, count (bodies in the cell), mass, com (3*cap, xyz interleaved),
 *   leaf_body (stored body of a leaf, -1 for internal cells),
 *   body_leaf (per body: id of the leaf whose cell holds it),
 * plus per body the 120-bit descent key (keys_hi: octants 0..20, keys_lo:
 * octants 21..39), the sorted permutation, and root4 = (cx, cy, cz, half).
 * Any output pointer may be NULL.  *nnodes receives the node count; arrays
 * are filled up to cap entries. */
int phys_bh_export(phys_ctx* ctx, const phys_params* p, int64_t cap, int64_t* nnodes,
                   int32_t* depth, int64_t* count, double* mass, double* com,
                   int64_t* leaf_body, int64_t* body_leaf, uint64_t* keys_hi,
                   uint64_t* keys_lo, int64_t* perm, double* root4);

/* ---- direct sum without allocation --------------------------------------- */
/* No counterpart in the reference.  For callers that must not allocate
 * device memory once running: an engine tick that fixed all its buffers at
 * start-up (cudaMalloc / cudaFree can synchronise the whole device and stall
 * the tick), or a host application that lends this library only memory from
 * its own pool.  Computes direct-sum accelerations
 *   a_i = G sum_{j != i} m_j r_ij / (|r_ij|^2 + eps^2)^{3/2}
 * for n <= 32768 bodies whose positions, masses and outputs are in the
 * caller's DEVICE memory, on the caller's stream (NULL: default stream),
 * precision PHYS_F64 or PHYS_F32C.  It allocates nothing: its scratch is one
 * fixed device array of about 7.3 MiB that every GPU loading the library
 * keeps until the process exits.  The first call on each device looks up the
 * array's device address (cudaGetSymbolAddress) and should come before any
 * stream capture; the address is kept for the life of the process, so a
 * process that calls cudaDeviceReset on a device must not call this entry
 * point on that device again.  All calls share the array, so calls that
 * overlap on the GPU race: order them.  n outside 0..32768 returns PHYS_ERR_ARG with a
 * message in errbuf (optional, errlen bytes).  Synchronous at return (it
 * reads its status word back), so no call can be captured in a CUDA graph. */
int phys_direct_accel_noalloc(int64_t n, const double* x, const double* y, const double* z,
                              const double* m, double G, double eps, int32_t precision,
                              double* ax, double* ay, double* az, void* stream, char* errbuf,
                              size_t errlen);

/* ---- failure injection for tests ---------------------------------------- */
/* No counterpart in the reference.  Sets the bound on each bounded device
 * wait of this context's radix sorts (re-reads of a predecessor tile's status
 * word; default 2^20, restored by spins < 0).  With a bound of 0 the first
 * wait gives up at once, as a stalled predecessor would after the default
 * bound: the evaluation then stops before building on the unfinished order
 * and returns PHYS_ERR_TIMEOUT, and the context stays usable.  Whether a wait
 * occurs at all depends on how the sort's tiles are scheduled, so a caller
 * that wants to see the timeout needs a sort of many tiles (e.g. 2^20
 * bodies). */
int phys_debug_set_wait_limit(phys_ctx* ctx, int64_t spins);

/* No counterpart in the reference.  q[i] = a[i] / b[i] (host arrays of n)
 * through the division of the tree's centre-of-mass recurrence
 * (gravity_tree.rs:113-118 divides by the new total mass): a correction
 * from the correctly rounded reciprocal of b where |a| and b lie in
 * [2^-500, 2^501) (and b > 0), the IEEE division elsewhere.  Both are
 * meant to give the correctly rounded quotient; tests compare q bit for
 * bit with IEEE division. */
int phys_debug_divide(phys_ctx* ctx, int64_t n, const double* a, const double* b, double* q);

/* ---- measured pipe peaks (roofline denominators) ----------------------- */
/* Times FFMA, packed FFMA2 (f32x2) and DFMA loops on every SM; returns
 * TFLOP/s counting an FMA as 2 flops (FFMA2 as 4). */
int phys_probe_peaks(phys_ctx* ctx, double* fp32_tflops, double* fp32x2_tflops,
                     double* fp64_tflops);

#ifdef __cplusplus
}
#endif
#endif /* PHYSGPU_H */
