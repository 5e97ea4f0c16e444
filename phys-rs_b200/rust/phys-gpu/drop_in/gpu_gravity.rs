//! GPU gravity systems for phys-rs (add as src/physics/gpu_gravity.rs, with
//! `phys-gpu = { path = ".../phys-rs_b200/rust/phys-gpu" }` in Cargo.toml).
//!
//! `gpu_gravity_system` has the signature of barnes_hut_gravity_system
//! (src/physics/gravity_tree.rs:260-263) and replaces it, or
//! brute_force_gravity_system (src/physics/gravity.rs:27-30), in both chains
//! of the Velocity-Verlet schedule (src/main.rs:109,128).  Its switches
//! (method, precision, leaf capacity, walk, device) come from
//! `phys_gpu::set_gravity_settings`, called once at start-up; G, softening
//! and theta come from UniverseConfig as in the reference.  The GPU context
//! is the calling thread's (phys_gpu::with_thread_context), so the system
//! needs no extra parameter.
//!
//! `gpu_verlet_tick` runs a whole tick on the device instead (position step,
//! force pass, a = F/m, velocity step, sector_boundary_system), one force
//! evaluation per tick: the first of the reference's two passes per tick is
//! at the positions of the previous tick's second pass, so the trajectory is
//! the same.
//!
//! `gpu_energy_system` replaces compute_kinetic_energy_system and
//! compute_potential_energy_system (src/physics/energy.rs:21-56): the
//! O(N^2) unsoftened potential runs on the device in f64.
use bevy_ecs::prelude::*;

use crate::components::dynamics::{Acceleration, Force, Mass, PreviousAcceleration, Velocity};
use crate::core::config::UniverseConfig;
use crate::physics::energy::EnergyMonitor;
use crate::core::coordinates::{LocalPosition, Sector};
use crate::core::time::SimulationTime;
use phys_gpu::{ffi, gravity_settings, with_thread_context, Soa3};

/// Force += gravity, computed on the GPU.  Same query, resource, ordering
/// and semantics as the reference systems: Force is added to, fewer than two
/// bodies return early (gravity.rs:49-51), positions are flattened from
/// (Sector, LocalPosition) relative to the first body's sector, or per body
/// for Barnes-Hut (gravity_tree.rs:280-291).  On a library error the forces
/// are left as they were and the error is reported on stderr.
pub fn gpu_gravity_system(
    mut query: Query<(Entity, &mut Force, &Mass, &Sector, &LocalPosition)>,
    config: Res<UniverseConfig>,
) {
    let n = query.iter().len();
    if n < 2 {
        return;
    }
    let settings = gravity_settings();
    let mut sector = [Vec::with_capacity(n), Vec::with_capacity(n), Vec::with_capacity(n)];
    let mut local = Soa3 {
        x: Vec::with_capacity(n),
        y: Vec::with_capacity(n),
        z: Vec::with_capacity(n),
    };
    let mut mass = Vec::with_capacity(n);
    for (_, _, m, s, l) in query.iter() {
        sector[0].push(s.0.x);
        sector[1].push(s.0.y);
        sector[2].push(s.0.z);
        local.x.push(l.0.x);
        local.y.push(l.0.y);
        local.z.push(l.0.z);
        mass.push(m.0);
    }
    let p = settings.params(config.gravitational_constant, config.softening_epsilon,
                            config.barnes_hut_theta);
    let bh_quirk = settings.method == ffi::PHYS_BARNES_HUT;
    let mut f = Soa3::zeros(n);
    let res = with_thread_context(|gpu| {
        gpu.upload_sectors([&sector[0], &sector[1], &sector[2]], &local, config.sector_size,
                           bh_quirk, None, &mass)?;
        gpu.add_gravity_forces(&p, &mut f)
    });
    if let Err(e) = res {
        eprintln!("gpu_gravity_system: {e}; Force left unchanged");
        return;
    }
    // query order is the upload order (gravity.rs:71-73 writes back by zip)
    for (i, (_, mut force, _, _, _)) in query.iter_mut().enumerate() {
        force.0.x += f.x[i];
        force.0.y += f.y[i];
        force.0.z += f.z[i];
    }
}

/// One Velocity-Verlet tick on the device for every body with the
/// integrator's components (integrators.rs:63-118, src/main.rs:103-140),
/// gravity as configured by `set_gravity_settings` (plus the NFW halo if the
/// thread's context has one set), sector normalisation included.
pub fn gpu_verlet_tick(
    time: Res<SimulationTime>,
    config: Res<UniverseConfig>,
    mut query: Query<(
        &mut Sector,
        &mut LocalPosition,
        &mut Velocity,
        &Mass,
        &mut Acceleration,
        &mut PreviousAcceleration,
    )>,
) {
    let n = query.iter().len();
    if n == 0 {
        return;
    }
    let settings = gravity_settings();
    let mut sector = [Vec::with_capacity(n), Vec::with_capacity(n), Vec::with_capacity(n)];
    let (mut local, mut vel, mut acc) = (Soa3::zeros(0), Soa3::zeros(0), Soa3::zeros(0));
    let mut mass = Vec::with_capacity(n);
    for (s, l, v, m, a, _) in query.iter() {
        sector[0].push(s.0.x);
        sector[1].push(s.0.y);
        sector[2].push(s.0.z);
        local.x.push(l.0.x);
        local.y.push(l.0.y);
        local.z.push(l.0.z);
        vel.x.push(v.0.x);
        vel.y.push(v.0.y);
        vel.z.push(v.0.z);
        acc.x.push(a.0.x);
        acc.y.push(a.0.y);
        acc.z.push(a.0.z);
        mass.push(m.0);
    }
    let p = settings.params(config.gravitational_constant, config.softening_epsilon,
                            config.barnes_hut_theta);
    let res = with_thread_context(|gpu| {
        gpu.upload_sector_state([&sector[0], &sector[1], &sector[2]], &local,
                                config.sector_size, &vel, &mass)?;
        gpu.set_accel(&acc)?;
        gpu.verlet_steps(&p, time.dt, 1)?;
        let (s, l) = gpu.download_sector_state()?;
        let (_, v, a) = gpu.download()?;
        Ok((s, l, v, a))
    });
    let (s, l, v, a) = match res {
        Ok(out) => out,
        Err(e) => {
            eprintln!("gpu_verlet_tick: {e}; state left unchanged");
            return;
        }
    };
    for (i, (mut sec, mut loc, mut vel, _, mut acc, mut prev)) in query.iter_mut().enumerate() {
        prev.0 = acc.0; // velocity_verlet_position_system keeps a(x_n)
        sec.0.x = s[0][i];
        sec.0.y = s[1][i];
        sec.0.z = s[2][i];
        loc.0.x = l.x[i];
        loc.0.y = l.y[i];
        loc.0.z = l.z[i];
        vel.0.x = v.x[i];
        vel.0.y = v.y[i];
        vel.0.z = v.z[i];
        acc.0.x = a.x[i];
        acc.0.y = a.y[i];
        acc.0.z = a.z[i];
    }
}

/// Kinetic and unsoftened potential energy into the EnergyMonitor, as
/// compute_kinetic_energy_system + compute_potential_energy_system
/// (energy.rs:21-56: pairs with r^2 == 0 skipped), computed on the device
/// with compensated f64 sums.
pub fn gpu_energy_system(
    query: Query<(&Mass, &Velocity, &Sector, &LocalPosition)>,
    config: Res<UniverseConfig>,
    mut monitor: ResMut<EnergyMonitor>,
) {
    let n = query.iter().len();
    if n == 0 {
        return;
    }
    let mut sector = [Vec::with_capacity(n), Vec::with_capacity(n), Vec::with_capacity(n)];
    let (mut local, mut vel) = (Soa3::zeros(0), Soa3::zeros(0));
    let mut mass = Vec::with_capacity(n);
    for (m, v, s, l) in query.iter() {
        sector[0].push(s.0.x);
        sector[1].push(s.0.y);
        sector[2].push(s.0.z);
        local.x.push(l.0.x);
        local.y.push(l.0.y);
        local.z.push(l.0.z);
        vel.x.push(v.0.x);
        vel.y.push(v.0.y);
        vel.z.push(v.0.z);
        mass.push(m.0);
    }
    let res = with_thread_context(|gpu| {
        gpu.upload_sectors([&sector[0], &sector[1], &sector[2]], &local, config.sector_size,
                           false, Some(&vel), &mass)?;
        gpu.diagnostics(config.gravitational_constant)
    });
    match res {
        Ok(d) => {
            monitor.kinetic_energy = d.kinetic;
            monitor.potential_energy = d.potential;
        }
        Err(e) => eprintln!("gpu_energy_system: {e}; EnergyMonitor left unchanged"),
    }
}
