//! Raw bindings of include/physgpu.h, one `extern "C"` declaration per entry
//! point, in the header's order.  Types follow the header exactly: `int` and
//! `int32_t` are `i32`, `int64_t` is `i64`, `uint64_t` is `u64`, `double` is
//! `f64`, `size_t` is `usize`; host arrays are structure-of-arrays `f64`.
#![allow(non_camel_case_types, non_snake_case, dead_code)]

use std::os::raw::{c_char, c_int, c_void};

pub const PHYS_OK: c_int = 0;
pub const PHYS_ERR_ARG: c_int = 1;
pub const PHYS_ERR_CUDA: c_int = 2;
pub const PHYS_ERR_OOM: c_int = 3;
pub const PHYS_ERR_NONFINITE: c_int = 4;
pub const PHYS_ERR_TIMEOUT: c_int = 5;
pub const PHYS_ERR_STATE: c_int = 6;

pub const PHYS_DIRECT: i32 = 0;
pub const PHYS_BARNES_HUT: i32 = 1;

pub const PHYS_F64_EXACT: i32 = 0;
pub const PHYS_F64: i32 = 1;
pub const PHYS_F32C: i32 = 2;

pub const PHYS_FLAG_GROUP_WALK: i32 = 1;

pub const PHYS_COMP_POSITION: i32 = 0;
pub const PHYS_COMP_VELOCITY: i32 = 1;
pub const PHYS_COMP_ACCELERATION: i32 = 2;
pub const PHYS_COMP_PREV_ACCELERATION: i32 = 3;
pub const PHYS_COMP_MASS: i32 = 4;

pub const PHYS_ENS_BY_SIZE: i32 = 1;
pub const PHYS_ENS_CANDIDATES: i32 = 6;
/// Warps per block in an ensemble configuration code.
pub const fn phys_ens_warps(w: i32) -> i32 {
    w << 8
}

/// Opaque device context.
#[repr(C)]
pub struct phys_ctx {
    _private: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct phys_params {
    pub G: f64,
    pub eps: f64,
    pub theta: f64,
    pub method: i32,
    pub precision: i32,
    pub leaf_cap: i32,
    pub flags: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct phys_timings {
    pub total_ms: f64,
    pub bbox_ms: f64,
    pub keys_ms: f64,
    pub sort_ms: f64,
    pub tree_ms: f64,
    pub walk_ms: f64,
    pub verlet_ms: f64,
    pub interactions: u64,
    pub launches: u64,
    pub nodes: i64,
    pub max_depth: i32,
    pub reserved: i32,
    pub walk_eval_ms: f64,
    pub walk_eval_interactions: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct phys_nfw_halo {
    pub rho_0: f64,
    pub scale_radius: f64,
    pub center: [f64; 3],
    pub enabled: i32,
    pub reserved: i32,
}

extern "C" {
    // ---- context ----
    pub fn phys_status_string(status: c_int) -> *const c_char;
    pub fn phys_last_error(ctx: *const phys_ctx) -> *const c_char;
    pub fn phys_ctx_create(device: c_int, out: *mut *mut phys_ctx) -> c_int;
    pub fn phys_ctx_destroy(ctx: *mut phys_ctx) -> c_int;
    pub fn phys_ctx_stream(ctx: *mut phys_ctx) -> *mut c_void;
    pub fn phys_last_timings(ctx: *const phys_ctx, out: *mut phys_timings) -> c_int;

    // ---- body state ----
    pub fn phys_state_upload(ctx: *mut phys_ctx, n: i64, x: *const f64, y: *const f64,
                             z: *const f64, vx: *const f64, vy: *const f64, vz: *const f64,
                             m: *const f64) -> c_int;
    pub fn phys_state_upload_sectors(ctx: *mut phys_ctx, n: i64, sx: *const i64, sy: *const i64,
                                     sz: *const i64, lx: *const f64, ly: *const f64,
                                     lz: *const f64, sector_size: f64, bh_quirk: i32,
                                     vx: *const f64, vy: *const f64, vz: *const f64,
                                     m: *const f64) -> c_int;
    pub fn phys_state_upload_sector_state(ctx: *mut phys_ctx, n: i64, sx: *const i64,
                                          sy: *const i64, sz: *const i64, lx: *const f64,
                                          ly: *const f64, lz: *const f64, sector_size: f64,
                                          vx: *const f64, vy: *const f64, vz: *const f64,
                                          m: *const f64) -> c_int;
    pub fn phys_state_download_sector_state(ctx: *mut phys_ctx, sx: *mut i64, sy: *mut i64,
                                            sz: *mut i64, lx: *mut f64, ly: *mut f64,
                                            lz: *mut f64) -> c_int;
    pub fn phys_state_set_accel(ctx: *mut phys_ctx, ax: *const f64, ay: *const f64,
                                az: *const f64) -> c_int;
    pub fn phys_state_download(ctx: *mut phys_ctx, x: *mut f64, y: *mut f64, z: *mut f64,
                               vx: *mut f64, vy: *mut f64, vz: *mut f64, ax: *mut f64,
                               ay: *mut f64, az: *mut f64) -> c_int;
    pub fn phys_state_size(ctx: *const phys_ctx) -> i64;
    pub fn phys_component_write(ctx: *mut phys_ctx, component: i32, a: *const f64,
                                b: *const f64, c: *const f64) -> c_int;
    pub fn phys_component_read(ctx: *mut phys_ctx, component: i32, a: *mut f64, b: *mut f64,
                               c: *mut f64) -> c_int;

    // ---- gravity ----
    pub fn phys_gravity_forces(ctx: *mut phys_ctx, p: *const phys_params, fx: *mut f64,
                               fy: *mut f64, fz: *mut f64) -> c_int;
    pub fn phys_gravity_accel(ctx: *mut phys_ctx, p: *const phys_params, ax: *mut f64,
                              ay: *mut f64, az: *mut f64) -> c_int;
    pub fn phys_direct_accel_targets(ctx: *mut phys_ctx, p: *const phys_params, nt: i64,
                                     targets: *const i64, ax: *mut f64, ay: *mut f64,
                                     az: *mut f64) -> c_int;

    // ---- target shares: one system split over GPUs (device buffers) ----
    pub fn phys_share_chunk(n: i64, world: i32) -> i64;
    pub fn phys_gravity_accel_share(ctx: *mut phys_ctx, p: *const phys_params, rank: i32,
                                    world: i32, share_out: *mut f64) -> c_int;
    pub fn phys_gravity_accel_unshare(ctx: *mut phys_ctx, world: i32,
                                      gathered: *const f64) -> c_int;

    // ---- NFW phantom halo ----
    pub fn phys_nfw_density(r: f64, rho_0: f64, rs: f64) -> f64;
    pub fn phys_nfw_enclosed_mass(r: f64, rho_0: f64, rs: f64) -> f64;
    pub fn phys_nfw_circular_velocity(r: f64, rho_0: f64, rs: f64) -> f64;
    pub fn phys_nfw_forces(ctx: *mut phys_ctx, halo: *const phys_nfw_halo, fx: *mut f64,
                           fy: *mut f64, fz: *mut f64) -> c_int;
    pub fn phys_set_nfw_halo(ctx: *mut phys_ctx, halo: *const phys_nfw_halo) -> c_int;

    // ---- integration ----
    pub fn phys_verlet_steps(ctx: *mut phys_ctx, p: *const phys_params, dt: f64,
                             nsteps: i64) -> c_int;
    pub fn phys_verlet_tick_host(ctx: *mut phys_ctx, p: *const phys_params, dt: f64, n: i64,
                                 x: *mut f64, y: *mut f64, z: *mut f64, vx: *mut f64,
                                 vy: *mut f64, vz: *mut f64, m: *const f64, ax: *mut f64,
                                 ay: *mut f64, az: *mut f64) -> c_int;
    pub fn phys_vv_position_step(ctx: *mut phys_ctx, dt: f64) -> c_int;
    pub fn phys_vv_velocity_step(ctx: *mut phys_ctx, dt: f64) -> c_int;
    pub fn phys_verlet_steps_async(ctx: *mut phys_ctx, p: *const phys_params, dt: f64,
                                   nsteps: i64) -> c_int;

    // ---- batched ensemble ----
    pub fn phys_ensemble_load(ctx: *mut phys_ctx, nsys: i64, offsets: *const i64,
                              x: *const f64, y: *const f64, z: *const f64, vx: *const f64,
                              vy: *const f64, vz: *const f64, m: *const f64) -> c_int;
    pub fn phys_ensemble_run(ctx: *mut phys_ctx, p: *const phys_params, dt: f64, nsteps: i64,
                             config: i32, chunk: i64) -> c_int;
    pub fn phys_ensemble_download(ctx: *mut phys_ctx, x: *mut f64, y: *mut f64, z: *mut f64,
                                  vx: *mut f64, vy: *mut f64, vz: *mut f64, ax: *mut f64,
                                  ay: *mut f64, az: *mut f64) -> c_int;
    pub fn phys_ensemble_autotune(ctx: *mut phys_ctx, p: *const phys_params, dt: f64,
                                  probe_steps: i64, best_config: *mut i32,
                                  ms: *mut f64) -> c_int;

    // ---- trajectory gradients ----
    pub fn phys_adjoint_direct(ctx: *mut phys_ctx, p: *const phys_params, dt: f64, nsteps: i64,
                               checkpoint: i64, tx: *const f64, ty: *const f64, tz: *const f64,
                               loss: *mut f64, gx: *mut f64, gy: *mut f64, gz: *mut f64,
                               gvx: *mut f64, gvy: *mut f64, gvz: *mut f64,
                               gm: *mut f64) -> c_int;
    pub fn phys_trajectory_loss(ctx: *mut phys_ctx, p: *const phys_params, dt: f64, nsteps: i64,
                                tx: *const f64, ty: *const f64, tz: *const f64, loss: *mut f64,
                                xT: *mut f64, yT: *mut f64, zT: *mut f64) -> c_int;

    // ---- diagnostics ----
    pub fn phys_diagnostics(ctx: *mut phys_ctx, G: f64, out5: *mut f64) -> c_int;

    // ---- Barnes-Hut tree export ----
    pub fn phys_bh_export(ctx: *mut phys_ctx, p: *const phys_params, cap: i64, nnodes: *mut i64,
                          depth: *mut i32, count: *mut i64, mass: *mut f64, com: *mut f64,
                          leaf_body: *mut i64, body_leaf: *mut i64, keys_hi: *mut u64,
                          keys_lo: *mut u64, perm: *mut i64, root4: *mut f64) -> c_int;

    // ---- direct sum without allocation ----
    pub fn phys_direct_accel_noalloc(n: i64, x: *const f64, y: *const f64, z: *const f64,
                                     m: *const f64, G: f64, eps: f64, precision: i32,
                                     ax: *mut f64, ay: *mut f64, az: *mut f64,
                                     stream: *mut c_void, errbuf: *mut c_char,
                                     errlen: usize) -> c_int;

    // ---- failure injection for tests ----
    pub fn phys_debug_set_wait_limit(ctx: *mut phys_ctx, spins: i64) -> c_int;
    pub fn phys_debug_divide(ctx: *mut phys_ctx, n: i64, a: *const f64, b: *const f64,
                             q: *mut f64) -> c_int;

    // ---- measured pipe peaks ----
    pub fn phys_probe_peaks(ctx: *mut phys_ctx, fp32_tflops: *mut f64, fp32x2_tflops: *mut f64,
                            fp64_tflops: *mut f64) -> c_int;
}
