// physgpu.hpp -- C++ host layer over the C ABI (include/physgpu.h).
//
// Mirrors the reference's gravity plugin API: bevy_ecs systems over
// components (src/physics/gravity.rs, gravity_tree.rs, integrators.rs,
// forces.rs, energy.rs) become free functions over a structure-of-arrays
// World, with UniverseConfig / SimulationTime carrying the same fields and
// defaults as src/core/config.rs:26-79 and src/core/time.rs:16-77.  All
// gravity and integration work runs on the GPU through libphysgpu; there is
// no CPU fallback (a missing device or library surfaces as an error Status).
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "../../include/physgpu.h"

namespace physgpu {

// src/core/config.rs:26-79 (gravity-path fields, same defaults)
struct UniverseConfig {
  double gravitational_constant = 6.67430e-11;  // src/core/constants.rs:7
  double softening_epsilon = 1e-4;
  double barnes_hut_theta = 0.5;
  double sector_size = 1e12;
};

// src/physics/nfw.rs:24-47 (same defaults: a Milky-Way-like halo, off)
struct NfwHaloConfig {
  double rho_0 = 1.4e-21;
  double scale_radius = 6.17e20;
  std::array<double, 3> center{0.0, 0.0, 0.0};
  bool enabled = false;
  phys_nfw_halo raw() const {
    phys_nfw_halo h{};
    h.rho_0 = rho_0;
    h.scale_radius = scale_radius;
    for (int k = 0; k < 3; ++k) h.center[k] = center[k];
    h.enabled = enabled ? 1 : 0;
    return h;
  }
};

// src/core/time.rs:16-77
struct SimulationTime {
  double dt = 1.0 / 60.0;
  uint64_t tick = 0;
  double elapsed = 0.0;
  static SimulationTime with_dt(double dt) {
    SimulationTime t;
    t.dt = dt;
    return t;
  }
  void advance_tick() {
    tick += 1;
    elapsed += dt;
  }
};

using Vec3 = std::array<double, 3>;
using IVec3 = std::array<int64_t, 3>;

// Components on the gravity path (src/components/dynamics.rs:13-37,
// src/core/coordinates.rs:19-26), one row per entity in query order.
struct World {
  std::vector<double> mass;
  std::vector<IVec3> sector;
  std::vector<Vec3> local, velocity, force, acceleration, prev_acceleration;

  size_t spawn(double m, Vec3 pos, IVec3 sec = {0, 0, 0}, Vec3 vel = {0, 0, 0},
               Vec3 acc = {0, 0, 0}, Vec3 prev = {0, 0, 0}) {
    mass.push_back(m);
    local.push_back(pos);
    sector.push_back(sec);
    velocity.push_back(vel);
    force.push_back({0, 0, 0});
    acceleration.push_back(acc);
    prev_acceleration.push_back(prev);
    return mass.size() - 1;
  }
  size_t size() const { return mass.size(); }
};

struct Status {
  int code = PHYS_OK;
  std::string message;
  bool ok() const { return code == PHYS_OK; }
};

enum class Precision : int32_t { F64Exact = PHYS_F64_EXACT, F64 = PHYS_F64, F32C = PHYS_F32C };

// RAII owner of one device context (CUDA stream + device-resident bodies).
class Context {
 public:
  explicit Context(int device = 0) { status_.code = phys_ctx_create(device, &ctx_); }
  ~Context() {
    if (ctx_) phys_ctx_destroy(ctx_);
  }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  Context(Context&& o) noexcept : ctx_(std::exchange(o.ctx_, nullptr)), status_(o.status_) {}

  bool ok() const { return ctx_ != nullptr; }
  const Status& create_status() const { return status_; }
  phys_ctx* raw() { return ctx_; }
  Status check(int code) const {
    Status s;
    s.code = code;
    if (code != PHYS_OK) s.message = ctx_ ? phys_last_error(ctx_) : phys_status_string(code);
    return s;
  }

 private:
  phys_ctx* ctx_ = nullptr;
  Status status_;
};

namespace detail {

struct Soa {
  std::vector<int64_t> sx, sy, sz;
  std::vector<double> lx, ly, lz, vx, vy, vz;
};

inline Soa gather(const World& w) {
  Soa s;
  const size_t n = w.size();
  for (auto* v : {&s.sx, &s.sy, &s.sz}) v->resize(n);
  for (auto* v : {&s.lx, &s.ly, &s.lz, &s.vx, &s.vy, &s.vz}) v->resize(n);
  for (size_t i = 0; i < n; ++i) {
    s.sx[i] = w.sector[i][0];
    s.sy[i] = w.sector[i][1];
    s.sz[i] = w.sector[i][2];
    s.lx[i] = w.local[i][0];
    s.ly[i] = w.local[i][1];
    s.lz[i] = w.local[i][2];
    s.vx[i] = w.velocity[i][0];
    s.vy[i] = w.velocity[i][1];
    s.vz[i] = w.velocity[i][2];
  }
  return s;
}

inline Status upload(Context& ctx, const World& w, const UniverseConfig& cfg, bool bh_quirk) {
  Soa s = gather(w);
  return ctx.check(phys_state_upload_sectors(
      ctx.raw(), (int64_t)w.size(), s.sx.data(), s.sy.data(), s.sz.data(), s.lx.data(),
      s.ly.data(), s.lz.data(), cfg.sector_size, bh_quirk ? 1 : 0, s.vx.data(), s.vy.data(),
      s.vz.data(), w.mass.data()));
}

inline Status gravity(World& w, const UniverseConfig& cfg, Context& ctx, int32_t method,
                      Precision prec, int32_t leaf_cap, int32_t flags = 0) {
  if (w.size() < 2) return {};  // gravity.rs:49-51
  const bool bh = method == PHYS_BARNES_HUT;
  Status st = upload(ctx, w, cfg, bh);
  if (!st.ok()) return st;
  phys_params p{cfg.gravitational_constant, cfg.softening_epsilon, cfg.barnes_hut_theta,
                method, (int32_t)prec, leaf_cap, flags};
  const size_t n = w.size();
  std::vector<double> fx(n), fy(n), fz(n);
  for (size_t i = 0; i < n; ++i) {
    fx[i] = w.force[i][0];
    fy[i] = w.force[i][1];
    fz[i] = w.force[i][2];
  }
  st = ctx.check(phys_gravity_forces(ctx.raw(), &p, fx.data(), fy.data(), fz.data()));
  if (!st.ok()) return st;  // Force left unchanged on error
  for (size_t i = 0; i < n; ++i) w.force[i] = {fx[i], fy[i], fz[i]};
  return st;
}

inline Status write3(Context& ctx, int32_t comp, const std::vector<Vec3>& v) {
  const size_t n = v.size();
  std::vector<double> a(n), b(n), c(n);
  for (size_t i = 0; i < n; ++i) {
    a[i] = v[i][0];
    b[i] = v[i][1];
    c[i] = v[i][2];
  }
  return ctx.check(phys_component_write(ctx.raw(), comp, a.data(), b.data(), c.data()));
}

inline Status read3(Context& ctx, int32_t comp, std::vector<Vec3>& v) {
  const size_t n = v.size();
  std::vector<double> a(n), b(n), c(n);
  Status st = ctx.check(phys_component_read(ctx.raw(), comp, a.data(), b.data(), c.data()));
  if (!st.ok()) return st;
  for (size_t i = 0; i < n; ++i) v[i] = {a[i], b[i], c[i]};
  return st;
}

// The integrators update LocalPosition itself (integrators.rs:80), so the
// local coordinates go to the device unflattened.
inline Status state_to_device(World& w, Context& ctx) {
  Soa s = gather(w);
  Status st = ctx.check(phys_state_upload(ctx.raw(), (int64_t)w.size(), s.lx.data(), s.ly.data(),
                                          s.lz.data(), s.vx.data(), s.vy.data(), s.vz.data(),
                                          w.mass.data()));
  if (st.ok()) st = write3(ctx, PHYS_COMP_ACCELERATION, w.acceleration);
  if (st.ok()) st = write3(ctx, PHYS_COMP_PREV_ACCELERATION, w.prev_acceleration);
  return st;
}

}  // namespace detail

// src/physics/forces.rs:15-19
inline void reset_forces(World& w) {
  for (auto& f : w.force) f = {0.0, 0.0, 0.0};
}

// src/physics/gravity.rs:27-74: Force += softened direct sum.
inline Status brute_force_gravity_system(World& w, const UniverseConfig& cfg, Context& ctx,
                                         Precision prec = Precision::F64Exact) {
  return detail::gravity(w, cfg, ctx, PHYS_DIRECT, prec, 1);
}

// src/physics/gravity_tree.rs:260-338: Force += Barnes-Hut.  group_walk walks
// the tree once per cell group of at most 64 bodies (F64 / F32C only; a
// stricter opening test, not the reference's traversal).
inline Status barnes_hut_gravity_system(World& w, const UniverseConfig& cfg, Context& ctx,
                                        Precision prec = Precision::F64Exact,
                                        int32_t leaf_cap = 1, bool group_walk = false) {
  return detail::gravity(w, cfg, ctx, PHYS_BARNES_HUT, prec, leaf_cap,
                         group_walk ? PHYS_FLAG_GROUP_WALK : 0);
}

// src/physics/nfw.rs:103-139: Force += the NFW halo's pull, from LocalPosition
// (the reference ignores Sector here); nothing when the halo is disabled.
inline Status nfw_gravity_system(World& w, const NfwHaloConfig& halo, Context& ctx) {
  if (!halo.enabled || w.size() == 0) return {};
  detail::Soa s = detail::gather(w);
  Status st = ctx.check(phys_state_upload(ctx.raw(), (int64_t)w.size(), s.lx.data(), s.ly.data(),
                                          s.lz.data(), nullptr, nullptr, nullptr, w.mass.data()));
  if (!st.ok()) return st;
  const size_t n = w.size();
  std::vector<double> fx(n), fy(n), fz(n);
  for (size_t i = 0; i < n; ++i) {
    fx[i] = w.force[i][0];
    fy[i] = w.force[i][1];
    fz[i] = w.force[i][2];
  }
  const phys_nfw_halo h = halo.raw();
  st = ctx.check(phys_nfw_forces(ctx.raw(), &h, fx.data(), fy.data(), fz.data()));
  if (!st.ok()) return st;
  for (size_t i = 0; i < n; ++i) w.force[i] = {fx[i], fy[i], fz[i]};
  return st;
}

// src/physics/integrators.rs:110-118: a = F / m (host loop, like the
// reference system; the device path fuses it into phys_gravity_accel).
inline void compute_acceleration_system(World& w) {
  for (size_t i = 0; i < w.size(); ++i)
    for (int k = 0; k < 3; ++k) w.acceleration[i][k] = w.force[i][k] / w.mass[i];
}

// src/physics/integrators.rs:63-83 on the device.
inline Status velocity_verlet_position_system(World& w, const SimulationTime& t, Context& ctx) {
  Status st = detail::state_to_device(w, ctx);
  if (st.ok()) st = ctx.check(phys_vv_position_step(ctx.raw(), t.dt));
  if (st.ok()) st = detail::read3(ctx, PHYS_COMP_POSITION, w.local);
  if (st.ok()) st = detail::read3(ctx, PHYS_COMP_PREV_ACCELERATION, w.prev_acceleration);
  return st;
}

// src/physics/integrators.rs:92-104 on the device.
inline Status velocity_verlet_velocity_system(World& w, const SimulationTime& t, Context& ctx) {
  Status st = detail::state_to_device(w, ctx);
  if (st.ok()) st = ctx.check(phys_vv_velocity_step(ctx.raw(), t.dt));
  if (st.ok()) st = detail::read3(ctx, PHYS_COMP_VELOCITY, w.velocity);
  return st;
}

// A whole Velocity-Verlet schedule (src/main.rs:103-150) of `ticks` ticks,
// device-resident: one upload of the (Sector, LocalPosition) state, ticks on
// the GPU (flatten per force pass, LocalPosition integrated,
// sector_boundary_system after every velocity step), one download of Sector,
// LocalPosition, Velocity, Acceleration and PreviousAcceleration.  The first
// tick recomputes a(x), as the schedule's first force pass does.
inline Status run_velocity_verlet(World& w, const UniverseConfig& cfg, SimulationTime& t,
                                  Context& ctx, int32_t method, Precision prec,
                                  int32_t leaf_cap, int64_t ticks, int32_t flags = 0) {
  const size_t n = w.size();
  detail::Soa s = detail::gather(w);
  Status st = ctx.check(phys_state_upload_sector_state(
      ctx.raw(), (int64_t)n, s.sx.data(), s.sy.data(), s.sz.data(), s.lx.data(), s.ly.data(),
      s.lz.data(), cfg.sector_size, s.vx.data(), s.vy.data(), s.vz.data(), w.mass.data()));
  if (!st.ok()) return st;
  phys_params p{cfg.gravitational_constant, cfg.softening_epsilon, cfg.barnes_hut_theta,
                method, (int32_t)prec, leaf_cap, flags};
  st = ctx.check(phys_verlet_steps(ctx.raw(), &p, t.dt, ticks));
  if (!st.ok()) return st;
  for (int64_t k = 0; k < ticks; ++k) t.advance_tick();
  st = ctx.check(phys_state_download_sector_state(ctx.raw(), s.sx.data(), s.sy.data(),
                                                  s.sz.data(), s.lx.data(), s.ly.data(),
                                                  s.lz.data()));
  if (!st.ok()) return st;
  for (size_t i = 0; i < n; ++i) {
    w.sector[i] = {s.sx[i], s.sy[i], s.sz[i]};
    w.local[i] = {s.lx[i], s.ly[i], s.lz[i]};
  }
  st = detail::read3(ctx, PHYS_COMP_VELOCITY, w.velocity);
  if (st.ok()) st = detail::read3(ctx, PHYS_COMP_ACCELERATION, w.acceleration);
  if (st.ok()) st = detail::read3(ctx, PHYS_COMP_PREV_ACCELERATION, w.prev_acceleration);
  return st;
}

// src/physics/energy.rs:21-56 and the momentum sum of integrators.rs:123-129.
struct Energy {
  double kinetic = 0.0, potential = 0.0;
  Vec3 momentum{0, 0, 0};
};
inline Status energy_diagnostics(World& w, const UniverseConfig& cfg, Context& ctx, Energy* out) {
  Status st = detail::upload(ctx, w, cfg, false);
  if (!st.ok()) return st;
  double o[5];
  st = ctx.check(phys_diagnostics(ctx.raw(), cfg.gravitational_constant, o));
  if (st.ok()) *out = Energy{o[0], o[1], {o[2], o[3], o[4]}};
  return st;
}

}  // namespace physgpu
