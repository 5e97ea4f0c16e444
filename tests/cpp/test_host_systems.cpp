// C++ port of the reference's known-answer tests for the gravity path, run
// through the C++ host layer (phys-rs_b200/host/physgpu.hpp) on the GPU, plus
// bit-exact comparisons with the CPU oracle (oracle/liboracle.so).
// Exit code 0 when every check passes.
#include <cmath>
#include <cstdio>
#include <random>

#include "../../phys-rs_b200/host/physgpu.hpp"

extern "C" {
void oracle_direct_forces(int64_t n, const double* x, const double* y, const double* z,
                          const double* m, double g, double eps, int nthreads, double* fx,
                          double* fy, double* fz);
void oracle_bh_forces(int64_t n, const double* x, const double* y, const double* z,
                      const double* m, double g, double eps, double theta, int nthreads,
                      double* fx, double* fy, double* fz, double* timings);
}

using namespace physgpu;

static int failures = 0;
#define CHECK(cond, ...)                              \
  do {                                                \
    if (!(cond)) {                                    \
      std::printf("FAIL %s:%d: ", __FILE__, __LINE__); \
      std::printf(__VA_ARGS__);                        \
      std::printf("\n");                               \
      ++failures;                                     \
    }                                                 \
  } while (0)

static double norm(const Vec3& a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

// gravity.rs:81-103
static void figure_8(Context& ctx) {
  World w;
  w.spawn(1.0, {-0.97000436, 0.24308753, 0.0});
  w.spawn(1.0, {0.97000436, -0.24308753, 0.0});
  w.spawn(1.0, {0.0, 0.0, 0.0});
  UniverseConfig cfg;
  cfg.softening_epsilon = 0.0;
  Status st = brute_force_gravity_system(w, cfg, ctx);
  CHECK(st.ok(), "%s", st.message.c_str());
  double sx = 0, sy = 0;
  for (auto& f : w.force) {
    CHECK(std::isfinite(f[0]) && std::isfinite(f[1]) && std::isfinite(f[2]), "finite");
    sx += f[0];
    sy += f[1];
  }
  CHECK(std::fabs(sx) < 1e-10 && std::fabs(sy) < 1e-10, "momentum %g %g", sx, sy);
}

// gravity.rs:106-130
static void kepler(Context& ctx) {
  World w;
  UniverseConfig cfg;
  cfg.softening_epsilon = 0.0;
  w.spawn(1e12, {0, 0, 0});
  size_t small = w.spawn(1.0, {100.0, 0, 0});
  Status st = brute_force_gravity_system(w, cfg, ctx);
  CHECK(st.ok(), "%s", st.message.c_str());
  const double expected = -(cfg.gravitational_constant * 1e12 * 1.0) / (100.0 * 100.0);
  CHECK(std::fabs(w.force[small][0] - expected) < 1e-10, "fx %g vs %g", w.force[small][0],
        expected);
  CHECK(w.force[small][1] == 0.0 && w.force[small][2] == 0.0, "fy fz zero");
}

// gravity_tree.rs:350-416
static void bh_two_bodies(Context& ctx) {
  World w;
  UniverseConfig cfg;
  size_t e1 = w.spawn(1e10, {0, 0, 0});
  size_t e2 = w.spawn(2e10, {100.0, 0, 0});
  Status st = barnes_hut_gravity_system(w, cfg, ctx);
  CHECK(st.ok(), "%s", st.message.c_str());
  const double eps2 = cfg.softening_epsilon * cfg.softening_epsilon, r2 = 1e4;
  const double expected =
      cfg.gravitational_constant * 1e10 * 2e10 * 100.0 / (std::sqrt(r2 + eps2) * (r2 + eps2));
  CHECK(w.force[e1][0] > 0 && w.force[e2][0] < 0, "directions");
  CHECK(std::fabs(w.force[e1][0] - expected) / expected < 1e-10, "magnitude");
  Vec3 s{w.force[e1][0] + w.force[e2][0], w.force[e1][1] + w.force[e2][1],
         w.force[e1][2] + w.force[e2][2]};
  CHECK(norm(s) < 1e-20, "third law %g", norm(s));
}

// gravity_tree.rs:420-487
static void bh_theta_zero(Context& ctx) {
  World wb, wd;
  UniverseConfig cfg;
  cfg.barnes_hut_theta = 0.0;
  const double ms[4] = {1e10, 2e10, 3e10, 5e10};
  const Vec3 ps[4] = {{0, 0, 0}, {100, 0, 0}, {0, 200, 0}, {150, 150, 0}};
  for (int i = 0; i < 4; ++i) {
    wb.spawn(ms[i], ps[i]);
    wd.spawn(ms[i], ps[i]);
  }
  CHECK(barnes_hut_gravity_system(wb, cfg, ctx).ok(), "bh");
  CHECK(brute_force_gravity_system(wd, cfg, ctx).ok(), "bf");
  for (int i = 0; i < 4; ++i) {
    Vec3 d{wb.force[i][0] - wd.force[i][0], wb.force[i][1] - wd.force[i][1],
           wb.force[i][2] - wd.force[i][2]};
    CHECK(norm(d) / std::fmax(norm(wd.force[i]), 1e-30) < 1e-8, "body %d", i);
  }
}

// gravity_tree.rs:491-556
static void bh_bounded_error(Context& ctx) {
  World w5, w0;
  UniverseConfig c5, c0;
  c0.barnes_hut_theta = 0.0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      w5.spawn(1e8, {i * 10.0, j * 10.0, 0});
      w0.spawn(1e8, {i * 10.0, j * 10.0, 0});
    }
  w5.spawn(5e10, {1000, 0, 0});
  w0.spawn(5e10, {1000, 0, 0});
  CHECK(barnes_hut_gravity_system(w5, c5, ctx).ok(), "bh 0.5");
  CHECK(barnes_hut_gravity_system(w0, c0, ctx).ok(), "bh 0");
  const Vec3& a = w5.force.back();
  const Vec3& b = w0.force.back();
  Vec3 d{a[0] - b[0], a[1] - b[1], a[2] - b[2]};
  CHECK(norm(d) / norm(b) < 0.05, "distant body error %g", norm(d) / norm(b));
  // the same bound through the group walk (F64, bucket leaves of 8)
  World g5 = w5;
  for (auto& f : g5.force) f = {0, 0, 0};
  CHECK(barnes_hut_gravity_system(g5, c5, ctx, Precision::F64, 8, true).ok(), "group 0.5");
  const Vec3& g = g5.force.back();
  Vec3 dg{g[0] - b[0], g[1] - b[1], g[2] - b[2]};
  CHECK(norm(dg) / norm(b) < 0.05, "group walk distant body error %g", norm(dg) / norm(b));
}

// integrators.rs:288-348 (300 ticks of the 6283-tick orbit, same per-tick bound)
static void circular_orbit(Context& ctx) {
  World w;
  w.spawn(1.0, {1, 0, 0}, {0, 0, 0}, {0, 1, 0}, {-1, 0, 0}, {-1, 0, 0});
  SimulationTime t = SimulationTime::with_dt(0.001);
  for (int s = 0; s < 300; ++s) {
    CHECK(velocity_verlet_position_system(w, t, ctx).ok(), "position system");
    const Vec3 r = w.local[0];
    const double rm = norm(r);
    w.acceleration[0] = {-r[0] / (rm * rm * rm), -r[1] / (rm * rm * rm), -r[2] / (rm * rm * rm)};
    CHECK(velocity_verlet_velocity_system(w, t, ctx).ok(), "velocity system");
    t.advance_tick();
  }
  const Vec3 v = w.velocity[0];
  const double e = 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) - 1.0 / norm(w.local[0]);
  CHECK(std::fabs(e + 0.5) < 1e-4, "energy drift %g", std::fabs(e + 0.5));
}

// F64_EXACT direct sum and Barnes-Hut vs the oracle, bit for bit.
static void exact_vs_oracle(Context& ctx) {
  std::mt19937_64 rng(42);
  std::normal_distribution<double> nd(0.0, 1.0);
  std::uniform_real_distribution<double> ud(0.5, 1.5);
  const int n = 3000;
  World w;
  std::vector<double> x(n), y(n), z(n), m(n);
  for (int i = 0; i < n; ++i) {
    x[i] = nd(rng);
    y[i] = nd(rng);
    z[i] = nd(rng);
    m[i] = ud(rng);
    w.spawn(m[i], {x[i], y[i], z[i]});
  }
  UniverseConfig cfg;
  cfg.gravitational_constant = 1.0;
  cfg.softening_epsilon = 0.01;
  for (int method = 0; method < 2; ++method) {
    reset_forces(w);
    Status st = method == 0 ? brute_force_gravity_system(w, cfg, ctx)
                            : barnes_hut_gravity_system(w, cfg, ctx);
    CHECK(st.ok(), "%s", st.message.c_str());
    std::vector<double> fx(n), fy(n), fz(n);
    if (method == 0)
      oracle_direct_forces(n, x.data(), y.data(), z.data(), m.data(), 1.0, 0.01, 4, fx.data(),
                           fy.data(), fz.data());
    else
      oracle_bh_forces(n, x.data(), y.data(), z.data(), m.data(), 1.0, 0.01, 0.5, 4, fx.data(),
                       fy.data(), fz.data(), nullptr);
    int bad = 0;
    for (int i = 0; i < n; ++i)
      bad += (w.force[i][0] != 0.0 + fx[i]) || (w.force[i][1] != 0.0 + fy[i]) ||
             (w.force[i][2] != 0.0 + fz[i]);
    CHECK(bad == 0, "method %d: %d bodies differ from the oracle", method, bad);
  }
}

// nfw.rs:103-139: |F| = G M(r) m / r^2 toward the centre; disabled = no-op.
static void nfw_halo(Context& ctx) {
  World w;
  w.spawn(2e30, {3e20, 4e20, 0});
  w.spawn(1e30, {0, 0, 0});  // at the centre: skipped
  NfwHaloConfig h;
  CHECK(nfw_gravity_system(w, h, ctx).ok(), "disabled halo");
  CHECK(w.force[0][0] == 0.0 && w.force[0][1] == 0.0, "disabled halo changed Force");
  h.enabled = true;
  CHECK(nfw_gravity_system(w, h, ctx).ok(), "nfw system");
  const double r = 5e20;
  const double mag = 6.67430e-11 * phys_nfw_enclosed_mass(r, h.rho_0, h.scale_radius) * 2e30 /
                     (r * r);
  CHECK(std::fabs(w.force[0][0] + 0.6 * mag) < 1e-12 * mag &&
            std::fabs(w.force[0][1] + 0.8 * mag) < 1e-12 * mag,
        "halo force %g %g vs %g", w.force[0][0], w.force[0][1], mag);
  CHECK(w.force[1][0] == 0.0 && w.force[1][1] == 0.0 && w.force[1][2] == 0.0, "centre body");
}

// run_velocity_verlet on the resident sector state: a free body crossing a
// sector boundary ends in the next sector (coordinates.rs:82-103).
static void sector_crossing(Context& ctx) {
  World w;
  w.spawn(1.0, {0.49e12, 0, 0}, {0, 0, 0}, {1e10, 0, 0});
  UniverseConfig cfg;  // sector_size 1e12
  SimulationTime t = SimulationTime::with_dt(1.0);
  CHECK(run_velocity_verlet(w, cfg, t, ctx, PHYS_DIRECT, Precision::F64Exact, 1, 2).ok(),
        "run");
  CHECK(w.sector[0][0] == 1 && w.sector[0][1] == 0, "sector %lld", (long long)w.sector[0][0]);
  CHECK(w.local[0][0] == (0.49e12 + 1e10 + 1e10) - 1e12, "local %.17g", w.local[0][0]);
  CHECK(t.tick == 2, "ticks");
}

int main() {
  Context ctx(0);
  if (!ctx.ok()) {
    std::printf("FAIL: no device context (status %d)\n", ctx.create_status().code);
    return 2;
  }
  figure_8(ctx);
  kepler(ctx);
  bh_two_bodies(ctx);
  bh_theta_zero(ctx);
  bh_bounded_error(ctx);
  circular_orbit(ctx);
  exact_vs_oracle(ctx);
  nfw_halo(ctx);
  sector_crossing(ctx);
  std::printf("%s (%d failures)\n", failures ? "FAILED" : "ok", failures);
  return failures ? 1 : 0;
}
