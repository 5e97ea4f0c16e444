//! Safe Rust API over libphysgpu (include/physgpu.h): the B200 gravity path
//! for phys-rs.
//!
//! * [`PhysGpu`] owns one device context (CUDA streams and device-resident
//!   bodies).  It is `Send` but not `Sync`: one thread uses it at a time, as
//!   bevy runs a system on one worker thread.
//! * [`PhysGpu::trajectory_gradient`] is the reverse-mode API: the gradient
//!   of L = sum_i |x_i(T) - target_i|^2 after T Velocity-Verlet ticks of the
//!   direct sum, with respect to the initial positions, velocities and
//!   masses, from the library's hand-written adjoint (checkpoint every K
//!   ticks, each segment recomputed).
//! * [`with_thread_context`] and [`gravity_settings`] let ECS systems keep
//!   the reference's signatures (drop_in/gpu_gravity.rs): the context lives
//!   in a thread-local slot, the method switches in a process-wide setting.
//!
//! Every call returns `Result<_, PhysError>`; nothing panics across the FFI.
pub mod ffi;

use std::cell::RefCell;
use std::ffi::CStr;
use std::ptr::{null, null_mut, NonNull};
use std::sync::RwLock;

/// A failed library call: the status code (`ffi::PHYS_ERR_*`) and the
/// library's message.
#[derive(Debug, Clone, PartialEq)]
pub struct PhysError {
    pub status: i32,
    pub message: String,
}

impl std::fmt::Display for PhysError {
    fn fmt(&self, f: &mut std::fmt::Formatter<'_>) -> std::fmt::Result {
        write!(f, "{} (status {})", self.message, self.status)
    }
}

impl std::error::Error for PhysError {}

pub type Result<T> = std::result::Result<T, PhysError>;

/// Force method, precision and Barnes-Hut switches (phys_params without the
/// UniverseConfig scalars).
#[derive(Clone, Copy, Debug, PartialEq)]
pub struct GravitySettings {
    pub method: i32,
    pub precision: i32,
    pub leaf_cap: i32,
    pub flags: i32,
    /// CUDA device of the thread-local contexts.
    pub device: i32,
}

impl Default for GravitySettings {
    /// The reference's arithmetic: direct sum, bit-identical f64.
    fn default() -> Self {
        Self {
            method: ffi::PHYS_DIRECT,
            precision: ffi::PHYS_F64_EXACT,
            leaf_cap: 1,
            flags: 0,
            device: 0,
        }
    }
}

impl GravitySettings {
    /// phys_params from these switches and UniverseConfig's G, eps, theta.
    pub fn params(&self, g: f64, eps: f64, theta: f64) -> ffi::phys_params {
        ffi::phys_params {
            G: g,
            eps,
            theta,
            method: self.method,
            precision: self.precision,
            leaf_cap: self.leaf_cap,
            flags: self.flags,
        }
    }
}

static SETTINGS: RwLock<Option<GravitySettings>> = RwLock::new(None);

/// Sets the switches the drop-in systems use (call once at start-up).
pub fn set_gravity_settings(s: GravitySettings) {
    if let Ok(mut w) = SETTINGS.write() {
        *w = Some(s);
    }
}

/// The switches set by [`set_gravity_settings`], or the default.
pub fn gravity_settings() -> GravitySettings {
    SETTINGS.read().ok().and_then(|r| *r).unwrap_or_default()
}

thread_local! {
    static THREAD_CTX: RefCell<Option<PhysGpu>> = const { RefCell::new(None) };
}

/// Runs `f` with this thread's context, created on first use on
/// `gravity_settings().device`.
pub fn with_thread_context<T>(f: impl FnOnce(&mut PhysGpu) -> Result<T>) -> Result<T> {
    THREAD_CTX.with(|slot| {
        let mut slot = slot.borrow_mut();
        if slot.is_none() {
            *slot = Some(PhysGpu::new(gravity_settings().device)?);
        }
        f(slot.as_mut().expect("context just created"))
    })
}

/// Structure-of-arrays 3-vectors, one Vec per component.
#[derive(Clone, Debug, Default, PartialEq)]
pub struct Soa3 {
    pub x: Vec<f64>,
    pub y: Vec<f64>,
    pub z: Vec<f64>,
}

impl Soa3 {
    pub fn zeros(n: usize) -> Self {
        Self { x: vec![0.0; n], y: vec![0.0; n], z: vec![0.0; n] }
    }
    pub fn len(&self) -> usize {
        self.x.len()
    }
    pub fn is_empty(&self) -> bool {
        self.x.is_empty()
    }
    fn check_len(&self, n: usize, what: &str) -> Result<()> {
        if self.x.len() != n || self.y.len() != n || self.z.len() != n {
            return Err(PhysError {
                status: ffi::PHYS_ERR_ARG,
                message: format!("{what}: {} / {} / {} components for {n} bodies",
                                 self.x.len(), self.y.len(), self.z.len()),
            });
        }
        Ok(())
    }
}

/// Gradient of a trajectory loss (see [`PhysGpu::trajectory_gradient`]).
#[derive(Clone, Debug, Default)]
pub struct Grad {
    pub loss: f64,
    /// dL/dx0
    pub dx: Soa3,
    /// dL/dv0
    pub dv: Soa3,
    /// dL/dm
    pub dm: Vec<f64>,
}

/// Energy and momentum (energy.rs:21-56, integrators.rs:123-129).
#[derive(Clone, Copy, Debug, Default, PartialEq)]
pub struct Diagnostics {
    pub kinetic: f64,
    pub potential: f64,
    pub momentum: [f64; 3],
}

/// One device context.
pub struct PhysGpu {
    ctx: NonNull<ffi::phys_ctx>,
    n: usize,
}

// The context is used by one thread at a time (C ABI: one context per
// thread); moving it between threads is fine.
unsafe impl Send for PhysGpu {}

impl PhysGpu {
    pub fn new(device: i32) -> Result<Self> {
        let mut raw = null_mut();
        let st = unsafe { ffi::phys_ctx_create(device, &mut raw) };
        match NonNull::new(raw) {
            Some(ctx) if st == ffi::PHYS_OK => Ok(Self { ctx, n: 0 }),
            _ => Err(PhysError { status: st, message: status_string(st) }),
        }
    }

    fn raw(&self) -> *mut ffi::phys_ctx {
        self.ctx.as_ptr()
    }

    fn check(&self, st: i32) -> Result<()> {
        if st == ffi::PHYS_OK {
            return Ok(());
        }
        let message = unsafe { CStr::from_ptr(ffi::phys_last_error(self.raw())) }
            .to_string_lossy()
            .into_owned();
        Err(PhysError { status: st, message })
    }

    /// Bodies currently on the device.
    pub fn len(&self) -> usize {
        self.n
    }
    pub fn is_empty(&self) -> bool {
        self.n == 0
    }

    /// Absolute positions, velocities (None: zero) and masses.
    pub fn upload(&mut self, pos: &Soa3, vel: Option<&Soa3>, m: &[f64]) -> Result<()> {
        let n = m.len();
        pos.check_len(n, "positions")?;
        if let Some(v) = vel {
            v.check_len(n, "velocities")?;
        }
        let (vx, vy, vz) = match vel {
            Some(v) => (v.x.as_ptr(), v.y.as_ptr(), v.z.as_ptr()),
            None => (null(), null(), null()),
        };
        self.check(unsafe {
            ffi::phys_state_upload(self.raw(), n as i64, pos.x.as_ptr(), pos.y.as_ptr(),
                                   pos.z.as_ptr(), vx, vy, vz, m.as_ptr())
        })?;
        self.n = n;
        Ok(())
    }

    /// Bodies as (Sector, LocalPosition, Mass): flattened on the device
    /// (gravity.rs:38-47; `bh_quirk` measures every body from its own
    /// sector, as barnes_hut_gravity_system does, gravity_tree.rs:280-291).
    pub fn upload_sectors(&mut self, sector: [&[i64]; 3], local: &Soa3, sector_size: f64,
                          bh_quirk: bool, vel: Option<&Soa3>, m: &[f64]) -> Result<()> {
        let n = m.len();
        local.check_len(n, "local positions")?;
        if sector.iter().any(|s| s.len() != n) {
            return Err(arg_error("sectors: wrong length"));
        }
        let (vx, vy, vz) = match vel {
            Some(v) => {
                v.check_len(n, "velocities")?;
                (v.x.as_ptr(), v.y.as_ptr(), v.z.as_ptr())
            }
            None => (null(), null(), null()),
        };
        self.check(unsafe {
            ffi::phys_state_upload_sectors(self.raw(), n as i64, sector[0].as_ptr(),
                                           sector[1].as_ptr(), sector[2].as_ptr(),
                                           local.x.as_ptr(), local.y.as_ptr(), local.z.as_ptr(),
                                           sector_size, bh_quirk as i32, vx, vy, vz, m.as_ptr())
        })?;
        self.n = n;
        Ok(())
    }

    /// Keeps (Sector, LocalPosition) on the device: later ticks flatten per
    /// force pass and run sector_boundary_system on the device.
    pub fn upload_sector_state(&mut self, sector: [&[i64]; 3], local: &Soa3, sector_size: f64,
                               vel: &Soa3, m: &[f64]) -> Result<()> {
        let n = m.len();
        local.check_len(n, "local positions")?;
        vel.check_len(n, "velocities")?;
        if sector.iter().any(|s| s.len() != n) {
            return Err(arg_error("sectors: wrong length"));
        }
        self.check(unsafe {
            ffi::phys_state_upload_sector_state(self.raw(), n as i64, sector[0].as_ptr(),
                                                sector[1].as_ptr(), sector[2].as_ptr(),
                                                local.x.as_ptr(), local.y.as_ptr(),
                                                local.z.as_ptr(), sector_size, vel.x.as_ptr(),
                                                vel.y.as_ptr(), vel.z.as_ptr(), m.as_ptr())
        })?;
        self.n = n;
        Ok(())
    }

    /// (Sector, LocalPosition) of a context in sector mode.
    pub fn download_sector_state(&mut self) -> Result<([Vec<i64>; 3], Soa3)> {
        let n = self.n;
        let mut s = [vec![0i64; n], vec![0i64; n], vec![0i64; n]];
        let mut l = Soa3::zeros(n);
        let [sx, sy, sz] = &mut s;
        self.check(unsafe {
            ffi::phys_state_download_sector_state(self.raw(), sx.as_mut_ptr(), sy.as_mut_ptr(),
                                                  sz.as_mut_ptr(), l.x.as_mut_ptr(),
                                                  l.y.as_mut_ptr(), l.z.as_mut_ptr())
        })?;
        Ok((s, l))
    }

    /// Sets the Acceleration component a Verlet tick starts from.
    pub fn set_accel(&mut self, a: &Soa3) -> Result<()> {
        a.check_len(self.n, "accelerations")?;
        self.check(unsafe {
            ffi::phys_state_set_accel(self.raw(), a.x.as_ptr(), a.y.as_ptr(), a.z.as_ptr())
        })
    }

    /// (positions, velocities, accelerations) from the device.
    pub fn download(&mut self) -> Result<(Soa3, Soa3, Soa3)> {
        let n = self.n;
        let (mut x, mut v, mut a) = (Soa3::zeros(n), Soa3::zeros(n), Soa3::zeros(n));
        self.check(unsafe {
            ffi::phys_state_download(self.raw(), x.x.as_mut_ptr(), x.y.as_mut_ptr(),
                                     x.z.as_mut_ptr(), v.x.as_mut_ptr(), v.y.as_mut_ptr(),
                                     v.z.as_mut_ptr(), a.x.as_mut_ptr(), a.y.as_mut_ptr(),
                                     a.z.as_mut_ptr())
        })?;
        Ok((x, v, a))
    }

    /// Force += gravity (brute_force_gravity_system / barnes_hut_gravity_system).
    pub fn add_gravity_forces(&mut self, p: &ffi::phys_params, force: &mut Soa3) -> Result<()> {
        force.check_len(self.n, "forces")?;
        self.check(unsafe {
            ffi::phys_gravity_forces(self.raw(), p, force.x.as_mut_ptr(), force.y.as_mut_ptr(),
                                     force.z.as_mut_ptr())
        })
    }

    /// a = F/m of gravity (and the NFW halo when set); also cached on the
    /// device for the next Verlet tick.
    pub fn gravity_accel(&mut self, p: &ffi::phys_params) -> Result<Soa3> {
        let mut a = Soa3::zeros(self.n);
        self.check(unsafe {
            ffi::phys_gravity_accel(self.raw(), p, a.x.as_mut_ptr(), a.y.as_mut_ptr(),
                                    a.z.as_mut_ptr())
        })?;
        Ok(a)
    }

    /// velocity_verlet_position_system on the device state
    /// (PreviousAcceleration = Acceleration; x += v dt + a dt^2/2).
    pub fn vv_position_step(&mut self, dt: f64) -> Result<()> {
        self.check(unsafe { ffi::phys_vv_position_step(self.raw(), dt) })
    }

    /// velocity_verlet_velocity_system on the device state
    /// (v += (PreviousAcceleration + Acceleration) dt/2).
    pub fn vv_velocity_step(&mut self, dt: f64) -> Result<()> {
        self.check(unsafe { ffi::phys_vv_velocity_step(self.raw(), dt) })
    }

    /// Share `rank` of `world` of the acceleration evaluation
    /// (phys_gravity_accel_share) for one system held whole by every GPU,
    /// packed into `share_out`; the caller all-gathers the shares (NCCL)
    /// and completes the evaluation with `accel_unshare`.
    ///
    /// # Safety
    /// `share_out` must point to 3 * share_chunk(n, world) f64 of device
    /// memory on this context's GPU.
    pub unsafe fn accel_share(&mut self, p: &ffi::phys_params, rank: i32, world: i32,
                              share_out: *mut f64) -> Result<()> {
        self.check(ffi::phys_gravity_accel_share(self.raw(), p, rank, world, share_out))
    }

    /// Scatters the gathered shares into the acceleration state
    /// (phys_gravity_accel_unshare).
    ///
    /// # Safety
    /// `gathered` must point to world * 3 * share_chunk(n, world) f64 of
    /// device memory on this context's GPU.
    pub unsafe fn accel_unshare(&mut self, world: i32, gathered: *const f64) -> Result<()> {
        self.check(ffi::phys_gravity_accel_unshare(self.raw(), world, gathered))
    }

    /// nsteps Velocity-Verlet ticks on the device-resident state.
    pub fn verlet_steps(&mut self, p: &ffi::phys_params, dt: f64, nsteps: i64) -> Result<()> {
        self.check(unsafe { ffi::phys_verlet_steps(self.raw(), p, dt, nsteps) })
    }

    /// One tick on host state in one call (phys_verlet_tick_host): position
    /// step, force pass, velocity step; x, v and a updated in place.
    pub fn verlet_tick_host(&mut self, p: &ffi::phys_params, dt: f64, x: &mut Soa3,
                            v: &mut Soa3, m: &[f64], a: &mut Soa3) -> Result<()> {
        let n = m.len();
        x.check_len(n, "positions")?;
        v.check_len(n, "velocities")?;
        a.check_len(n, "accelerations")?;
        self.check(unsafe {
            ffi::phys_verlet_tick_host(self.raw(), p, dt, n as i64, x.x.as_mut_ptr(),
                                       x.y.as_mut_ptr(), x.z.as_mut_ptr(), v.x.as_mut_ptr(),
                                       v.y.as_mut_ptr(), v.z.as_mut_ptr(), m.as_ptr(),
                                       a.x.as_mut_ptr(), a.y.as_mut_ptr(), a.z.as_mut_ptr())
        })?;
        self.n = n;
        Ok(())
    }

    /// nfw_gravity_system's halo in every later acceleration (None removes it).
    pub fn set_nfw_halo(&mut self, halo: Option<&ffi::phys_nfw_halo>) -> Result<()> {
        let h = halo.map_or(null(), |h| h as *const _);
        self.check(unsafe { ffi::phys_set_nfw_halo(self.raw(), h) })
    }

    pub fn diagnostics(&mut self, g: f64) -> Result<Diagnostics> {
        let mut out = [0.0f64; 5];
        self.check(unsafe { ffi::phys_diagnostics(self.raw(), g, out.as_mut_ptr()) })?;
        Ok(Diagnostics { kinetic: out[0], potential: out[1], momentum: [out[2], out[3], out[4]] })
    }

    /// Independent small systems in CSR layout (offsets[0] == 0).
    pub fn ensemble_load(&mut self, offsets: &[i64], pos: &Soa3, vel: &Soa3, m: &[f64])
                         -> Result<()> {
        let n = m.len();
        pos.check_len(n, "positions")?;
        vel.check_len(n, "velocities")?;
        if offsets.len() < 2 || offsets[offsets.len() - 1] != n as i64 {
            return Err(arg_error("offsets must end at the body count"));
        }
        self.check(unsafe {
            ffi::phys_ensemble_load(self.raw(), (offsets.len() - 1) as i64, offsets.as_ptr(),
                                    pos.x.as_ptr(), pos.y.as_ptr(), pos.z.as_ptr(),
                                    vel.x.as_ptr(), vel.y.as_ptr(), vel.z.as_ptr(), m.as_ptr())
        })
    }

    /// nsteps ticks of every system; config 0 uses the autotuned launch shape
    /// (lanes per system | ffi::phys_ens_warps(warps per block) otherwise).
    pub fn ensemble_run(&mut self, p: &ffi::phys_params, dt: f64, nsteps: i64, config: i32,
                        chunk: i64) -> Result<()> {
        self.check(unsafe { ffi::phys_ensemble_run(self.raw(), p, dt, nsteps, config, chunk) })
    }

    /// Times every candidate launch shape and keeps the fastest: (best
    /// configuration code, the candidates' timings in ms).
    pub fn ensemble_autotune(&mut self, p: &ffi::phys_params, dt: f64, probe_steps: i64)
                             -> Result<(i32, Vec<f64>)> {
        let mut best = 0i32;
        let mut ms = vec![0.0f64; ffi::PHYS_ENS_CANDIDATES as usize];
        self.check(unsafe {
            ffi::phys_ensemble_autotune(self.raw(), p, dt, probe_steps, &mut best, ms.as_mut_ptr())
        })?;
        Ok((best, ms))
    }

    /// Reverse mode: loss and gradient of L = sum_i |x_i(T) - target_i|^2
    /// after `nsteps` Velocity-Verlet ticks of the direct sum (p.precision
    /// must be PHYS_F64) from the uploaded state, which is left unchanged;
    /// (x, v) checkpointed every `checkpoint` ticks.
    pub fn trajectory_gradient(&mut self, p: &ffi::phys_params, dt: f64, nsteps: i64,
                               checkpoint: i64, targets: &Soa3) -> Result<Grad> {
        let n = self.n;
        targets.check_len(n, "targets")?;
        let mut g = Grad { loss: 0.0, dx: Soa3::zeros(n), dv: Soa3::zeros(n), dm: vec![0.0; n] };
        self.check(unsafe {
            ffi::phys_adjoint_direct(self.raw(), p, dt, nsteps, checkpoint, targets.x.as_ptr(),
                                     targets.y.as_ptr(), targets.z.as_ptr(), &mut g.loss,
                                     g.dx.x.as_mut_ptr(), g.dx.y.as_mut_ptr(),
                                     g.dx.z.as_mut_ptr(), g.dv.x.as_mut_ptr(),
                                     g.dv.y.as_mut_ptr(), g.dv.z.as_mut_ptr(),
                                     g.dm.as_mut_ptr())
        })?;
        Ok(g)
    }

    /// The same forward pass only: (loss, final positions).
    pub fn trajectory_loss(&mut self, p: &ffi::phys_params, dt: f64, nsteps: i64,
                           targets: &Soa3) -> Result<(f64, Soa3)> {
        let n = self.n;
        targets.check_len(n, "targets")?;
        let mut loss = 0.0;
        let mut xt = Soa3::zeros(n);
        self.check(unsafe {
            ffi::phys_trajectory_loss(self.raw(), p, dt, nsteps, targets.x.as_ptr(),
                                      targets.y.as_ptr(), targets.z.as_ptr(), &mut loss,
                                      xt.x.as_mut_ptr(), xt.y.as_mut_ptr(), xt.z.as_mut_ptr())
        })?;
        Ok((loss, xt))
    }

    /// Device timings and counters of the last call.
    pub fn timings(&self) -> ffi::phys_timings {
        let mut t = ffi::phys_timings::default();
        unsafe { ffi::phys_last_timings(self.raw(), &mut t) };
        t
    }
}

impl Drop for PhysGpu {
    fn drop(&mut self) {
        unsafe {
            ffi::phys_ctx_destroy(self.raw());
        }
    }
}

fn arg_error(msg: &str) -> PhysError {
    PhysError { status: ffi::PHYS_ERR_ARG, message: msg.to_string() }
}

/// The library's name for a status code.
/// Targets per share when `n` bodies are split over `world` GPUs
/// (phys_share_chunk).
pub fn share_chunk(n: usize, world: i32) -> usize {
    let c = unsafe { ffi::phys_share_chunk(n as i64, world) };
    if c < 0 { 0 } else { c as usize }
}

pub fn status_string(st: i32) -> String {
    unsafe { CStr::from_ptr(ffi::phys_status_string(st)) }.to_string_lossy().into_owned()
}
