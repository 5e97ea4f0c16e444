// CPU oracle for the phys-rs gravity path.  TEST INFRASTRUCTURE ONLY.
//
// This file restates, in C++, the f64 arithmetic of the reference's gravity
// systems so that the CUDA library can be checked against it.  It is used by
// tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline and
// reference legs, and by nothing else; the product never links or calls it.
//
// The reference (Doritozzzz/phys-rs) is Rust and cannot be built here (no
// cargo, no crate sources).  Parity is pinned by re-running the reference's
// own known-answer tests against this oracle (tests/test_oracle_kats.py):
//   src/physics/gravity.rs:81-130        figure-8 momentum, Kepler force
//   src/physics/gravity_tree.rs:350-556   BH two-body, theta=0, bounded error
//   src/physics/integrators.rs:288-348    Verlet circular-orbit energy drift
// Those tests carry tolerances (1e-10 .. 5%), not golden bits.  Bit-level
// agreement with glam 0.32.1's DVec3 (a dependency absent from the reference
// tree) rests on its scalar definitions: length_squared = x*x + y*y + z*z
// evaluated left to right, and per-component + - * / with no FMA.  Rust never
// contracts a*b+c into an FMA, so this file is compiled with
// -ffp-contract=off -fno-fast-math on x86-64 SSE2.
//
// Threading mirrors rayon's `par_iter().with_min_len(1024)`: targets are split
// into contiguous chunks of at least 1024, one std::thread per chunk.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <utility>
#include <vector>

namespace {

struct V3 {
  double x, y, z;
};
inline V3 v3(double x, double y, double z) { return V3{x, y, z}; }
inline V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 mul(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 divs(V3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }
// glam DVec3::length_squared == dot(self, self) == (x*x + y*y) + z*z
inline double len2(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }

// Split [0, n) into chunks of at least `min_len` (rayon with_min_len) and run
// fn(lo, hi) on up to `nthreads` threads.
template <class F>
void par_chunks(int64_t n, int nthreads, int64_t min_len, F fn) {
  if (nthreads < 1) nthreads = 1;
  int64_t max_chunks = n / min_len;
  if (max_chunks < 1) max_chunks = 1;
  int64_t nchunks = std::min<int64_t>(nthreads, max_chunks);
  if (nchunks <= 1) {
    fn(int64_t(0), n);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(nchunks);
  for (int64_t c = 0; c < nchunks; ++c) {
    int64_t lo = n * c / nchunks, hi = n * (c + 1) / nchunks;
    th.emplace_back([=] { fn(lo, hi); });
  }
  for (auto& t : th) t.join();
}

// ---------------------------------------------------------------------------
// Direct sum: src/physics/gravity.rs:53-69 (pair law at 58-65).
// ---------------------------------------------------------------------------
inline V3 direct_one(int64_t i, int64_t n, const double* x, const double* y,
                     const double* z, const double* m, double g, double eps2) {
  V3 fs = v3(0.0, 0.0, 0.0);
  const V3 ti = v3(x[i], y[i], z[i]);
  const double mi = m[i];
  for (int64_t j = 0; j < n; ++j) {
    if (i == j) continue;
    V3 r = sub(v3(x[j], y[j], z[j]), ti);
    double r2 = len2(r);
    double s2 = r2 + eps2;
    double s = std::sqrt(s2);
    double s3 = s2 * s;
    double sc = ((g * mi) * m[j]) / s3;
    fs = add(fs, mul(r, sc));
  }
  return fs;
}

// ---------------------------------------------------------------------------
// Barnes-Hut: src/physics/gravity_tree.rs.  A pointer octree with boxed
// children, built by serial insertion in body-index order, exactly as the
// reference does (constants 30/34, octant and child centre 90-107, insert
// 110-154, compute_force 171-209, pair law 218-234, bbox 305-317).
// ---------------------------------------------------------------------------
constexpr uint32_t kMaxDepth = 40;       // gravity_tree.rs:30
constexpr double kMinNodeSize = 1e-8;    // gravity_tree.rs:34

struct Body {
  V3 pos;
  double mass;
  int64_t index;
};

enum Kind : uint8_t { kEmpty = 0, kLeaf = 1, kInternal = 2 };

struct Node {
  V3 center;
  double half;
  double total_mass;
  V3 com;
  Kind kind;
  Body body;          // valid when kind == kLeaf
  Node* children;     // 8 nodes when kind == kInternal
  int64_t count;      // bodies inserted (bookkeeping for export only)
  uint32_t depth;     // bookkeeping for export only

  void init(V3 c, double h, uint32_t d) {
    center = c;
    half = h;
    total_mass = 0.0;
    com = v3(0.0, 0.0, 0.0);
    kind = kEmpty;
    children = nullptr;
    count = 0;
    depth = d;
  }
  int octant(V3 p) const {  // gravity_tree.rs:90-96
    int idx = 0;
    if (p.x >= center.x) idx |= 1;
    if (p.y >= center.y) idx |= 2;
    if (p.z >= center.z) idx |= 4;
    return idx;
  }
  V3 child_center(int o) const {  // gravity_tree.rs:100-107
    double q = half * 0.5;
    return v3(center.x + ((o & 1) ? q : -q), center.y + ((o & 2) ? q : -q),
              center.z + ((o & 4) ? q : -q));
  }
  void insert(const Body& b, uint32_t d) {  // gravity_tree.rs:110-154
    double new_total = total_mass + b.mass;
    if (new_total > 0.0) com = divs(add(mul(com, total_mass), mul(b.pos, b.mass)), new_total);
    total_mass = new_total;
    count += 1;
    if (d >= kMaxDepth || half < kMinNodeSize) {
      // Guard leaf: overwrites the stored body (gravity_tree.rs:121-126).
      if (kind == kInternal) free_children();
      kind = kLeaf;
      body = b;
      return;
    }
    if (kind == kEmpty) {
      kind = kLeaf;
      body = b;
    } else if (kind == kLeaf) {
      Body existing = body;
      double hs = half * 0.5;
      children = new Node[8];
      for (int i = 0; i < 8; ++i) children[i].init(child_center(i), hs, depth + 1);
      kind = kInternal;
      children[octant(existing.pos)].insert(existing, d + 1);
      children[octant(b.pos)].insert(b, d + 1);
    } else {
      children[octant(b.pos)].insert(b, d + 1);
    }
  }
  void free_children() {
    if (children) {
      for (int i = 0; i < 8; ++i) children[i].free_children();
      delete[] children;
      children = nullptr;
    }
  }
  V3 compute_force(const Body& t, double theta, double g, double eps2) const;
};

inline V3 gravity_pair(const Body& t, V3 sp, double sm, double g, double eps2) {
  V3 r = sub(sp, t.pos);  // gravity_tree.rs:225-233
  double r2 = len2(r);
  double s2 = r2 + eps2;
  double s = std::sqrt(s2);
  double s3 = s2 * s;
  double sc = ((g * t.mass) * sm) / s3;
  return mul(r, sc);
}

V3 Node::compute_force(const Body& t, double theta, double g, double eps2) const {
  switch (kind) {  // gravity_tree.rs:178-208
    case kEmpty:
      return v3(0.0, 0.0, 0.0);
    case kLeaf:
      if (body.index == t.index) return v3(0.0, 0.0, 0.0);
      return gravity_pair(t, body.pos, body.mass, g, eps2);
    default: {
      V3 r = sub(com, t.pos);
      double d2 = len2(r);
      double s = half * 2.0;
      if (s * s < theta * theta * d2) return gravity_pair(t, com, total_mass, g, eps2);
      V3 f = v3(0.0, 0.0, 0.0);
      for (int c = 0; c < 8; ++c)
        if (children[c].total_mass > 0.0) f = add(f, children[c].compute_force(t, theta, g, eps2));
      return f;
    }
  }
}

struct Tree {
  Node root;
  std::vector<Body> bodies;
  ~Tree() { root.free_children(); }
};

// gravity_tree.rs:305-323: bounding cube then serial insertion.
void build_tree(Tree& T, int64_t n, const double* x, const double* y, const double* z,
                const double* m) {
  T.bodies.resize(n);
  for (int64_t i = 0; i < n; ++i) T.bodies[i] = Body{v3(x[i], y[i], z[i]), m[i], i};
  V3 mn = T.bodies[0].pos, mx = T.bodies[0].pos;
  for (int64_t i = 0; i < n; ++i) {  // glam DVec3::min/max == f64::min/max per lane
    const V3 p = T.bodies[i].pos;
    mn = v3(std::fmin(mn.x, p.x), std::fmin(mn.y, p.y), std::fmin(mn.z, p.z));
    mx = v3(std::fmax(mx.x, p.x), std::fmax(mx.y, p.y), std::fmax(mx.z, p.z));
  }
  V3 ext = sub(mx, mn);
  double max_extent = std::fmax(std::fmax(ext.x, ext.y), ext.z);
  double half = max_extent * 0.55 + 1.0;
  V3 center = mul(add(mn, mx), 0.5);
  T.root.init(center, half, 0);
  for (int64_t i = 0; i < n; ++i) T.root.insert(T.bodies[i], 0);
}

// Pre-order export of the non-empty nodes (children visited 0..7).
struct Exporter {
  int64_t cap, cnt = 0;
  int32_t* depth;
  int64_t* count;
  double *mass, *cx, *cy, *cz;
  int64_t* leaf_body;  // -1 for internal nodes
  int64_t* body_leaf;  // per body: pre-order id of the leaf whose cell holds it
  std::vector<std::pair<const Node*, int64_t>> ids;
  void visit(const Node& nd) {
    if (nd.kind == kEmpty) return;
    int64_t id = cnt++;
    if (id < cap) {
      depth[id] = int32_t(nd.depth);
      count[id] = nd.count;
      mass[id] = nd.total_mass;
      cx[id] = nd.com.x;
      cy[id] = nd.com.y;
      cz[id] = nd.com.z;
      leaf_body[id] = nd.kind == kLeaf ? nd.body.index : -1;
    }
    ids.emplace_back(&nd, id);
    if (nd.kind == kInternal)
      for (int c = 0; c < 8; ++c) visit(nd.children[c]);
  }
};

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

extern "C" {

// gravity.rs:38-47 (direct sum: origin = first body's sector).  With
// `bh_quirk` set, gravity_tree.rs:280-291 is followed instead: `first` is
// never cleared there, so every body is measured from its own sector and the
// absolute position is 0*sector_size + local.
void oracle_flatten(int64_t n, const int64_t* sx, const int64_t* sy, const int64_t* sz,
                    const double* lx, const double* ly, const double* lz, double sector_size,
                    int bh_quirk, double* x, double* y, double* z) {
  if (n <= 0) return;
  int64_t ox = sx[0], oy = sy[0], oz = sz[0];
  for (int64_t i = 0; i < n; ++i) {
    if (bh_quirk) {
      ox = sx[i];
      oy = sy[i];
      oz = sz[i];
    }
    x[i] = double(int64_t(uint64_t(sx[i]) - uint64_t(ox))) * sector_size + lx[i];
    y[i] = double(int64_t(uint64_t(sy[i]) - uint64_t(oy))) * sector_size + ly[i];
    z[i] = double(int64_t(uint64_t(sz[i]) - uint64_t(oz))) * sector_size + lz[i];
  }
}

// brute_force_gravity_system's computed forces (gravity.rs:53-69).  Writes the
// force sums (the caller adds them to its Force components, gravity.rs:71-73).
// Returns early, writing nothing, for n < 2 (gravity.rs:49-51).
void oracle_direct_forces(int64_t n, const double* x, const double* y, const double* z,
                          const double* m, double g, double eps, int nthreads, double* fx,
                          double* fy, double* fz) {
  if (n < 2) return;
  const double eps2 = eps * eps;
  par_chunks(n, nthreads, 1024, [&](int64_t lo, int64_t hi) {
    for (int64_t i = lo; i < hi; ++i) {
      V3 f = direct_one(i, n, x, y, z, m, g, eps2);
      fx[i] = f.x;
      fy[i] = f.y;
      fz[i] = f.z;
    }
  });
}

// Direct-sum forces for a subset of targets (CPU baseline samples and large
// spot checks).  Same arithmetic as oracle_direct_forces.
void oracle_direct_forces_targets(int64_t n, const double* x, const double* y, const double* z,
                                  const double* m, double g, double eps, int64_t nt,
                                  const int64_t* targets, int nthreads, double* fx, double* fy,
                                  double* fz) {
  const double eps2 = eps * eps;
  par_chunks(nt, nthreads, 64, [&](int64_t lo, int64_t hi) {
    for (int64_t k = lo; k < hi; ++k) {
      V3 f = direct_one(targets[k], n, x, y, z, m, g, eps2);
      fx[k] = f.x;
      fy[k] = f.y;
      fz[k] = f.z;
    }
  });
}

// barnes_hut_gravity_system's computed forces (gravity_tree.rs:305-330).
// `timings` (optional, 2 doubles) receives build and walk seconds.
void oracle_bh_forces(int64_t n, const double* x, const double* y, const double* z,
                      const double* m, double g, double eps, double theta, int nthreads,
                      double* fx, double* fy, double* fz, double* timings) {
  if (n < 2) return;
  const double eps2 = eps * eps;
  double t0 = now_s();
  Tree T;
  build_tree(T, n, x, y, z, m);
  double t1 = now_s();
  par_chunks(n, nthreads, 1024, [&](int64_t lo, int64_t hi) {
    for (int64_t i = lo; i < hi; ++i) {
      V3 f = T.root.compute_force(T.bodies[i], theta, g, eps2);
      fx[i] = f.x;
      fy[i] = f.y;
      fz[i] = f.z;
    }
  });
  double t2 = now_s();
  if (timings) {
    timings[0] = t1 - t0;
    timings[1] = t2 - t1;
  }
}

// Barnes-Hut forces for a subset of targets on the full tree (CPU baseline
// sample).  timings[0] = serial build seconds, timings[1] = walk seconds.
void oracle_bh_forces_targets(int64_t n, const double* x, const double* y, const double* z,
                              const double* m, double g, double eps, double theta, int64_t nt,
                              const int64_t* targets, int nthreads, double* fx, double* fy,
                              double* fz, double* timings) {
  const double eps2 = eps * eps;
  double t0 = now_s();
  Tree T;
  build_tree(T, n, x, y, z, m);
  double t1 = now_s();
  par_chunks(nt, nthreads, 64, [&](int64_t lo, int64_t hi) {
    for (int64_t k = lo; k < hi; ++k) {
      V3 f = T.root.compute_force(T.bodies[targets[k]], theta, g, eps2);
      fx[k] = f.x;
      fy[k] = f.y;
      fz[k] = f.z;
    }
  });
  double t2 = now_s();
  if (timings) {
    timings[0] = t1 - t0;
    timings[1] = t2 - t1;
  }
}

// Builds the reference octree and exports its non-empty nodes in pre-order.
// Returns the node count (arrays are filled up to `cap`).  Also writes the
// root cube (center xyz, half) to root4 when given.
int64_t oracle_bh_export(int64_t n, const double* x, const double* y, const double* z,
                         const double* m, int64_t cap, int32_t* depth, int64_t* count,
                         double* mass, double* cx, double* cy, double* cz, int64_t* leaf_body,
                         int64_t* body_leaf, double* root4) {
  if (n < 1) return 0;
  Tree T;
  build_tree(T, n, x, y, z, m);
  if (root4) {
    root4[0] = T.root.center.x;
    root4[1] = T.root.center.y;
    root4[2] = T.root.center.z;
    root4[3] = T.root.half;
  }
  if (body_leaf)
    for (int64_t i = 0; i < n; ++i) body_leaf[i] = -1;
  Exporter E{cap, 0, depth, count, mass, cx, cy, cz, leaf_body, body_leaf, {}};
  E.visit(T.root);
  if (body_leaf) {
    // Cell membership: follow the insertion rule (octant per level) down to
    // the leaf whose cell holds each body; guard leaves hold every body that
    // reached them, including the ones whose slot was overwritten.
    std::sort(E.ids.begin(), E.ids.end());
    for (int64_t i = 0; i < n; ++i) {
      const Node* nd = &T.root;
      while (nd->kind == kInternal) nd = &nd->children[nd->octant(T.bodies[i].pos)];
      auto it = std::lower_bound(E.ids.begin(), E.ids.end(), std::make_pair(nd, int64_t(-1)));
      body_leaf[i] = (it != E.ids.end() && it->first == nd) ? it->second : -1;
    }
  }
  return E.cnt;
}

// The reference's per-level descent for one position (the octants insert
// follows), emitted as a 120-bit key: hi = octants 0..20 (bits 62..0, octant 0
// in bits 62..60), lo = octants 21..39 (bits 56..0).  `levels` octants are
// produced; deeper octants are zero.
void oracle_descent_keys(int64_t n, const double* x, const double* y, const double* z,
                         const double* root4, int levels, uint64_t* hi, uint64_t* lo) {
  for (int64_t i = 0; i < n; ++i) {
    double cx = root4[0], cy = root4[1], cz = root4[2], h = root4[3];
    uint64_t kh = 0, kl = 0;
    for (int d = 0; d < 40; ++d) {
      uint64_t o = 0;
      if (d < levels) {
        if (x[i] >= cx) o |= 1;
        if (y[i] >= cy) o |= 2;
        if (z[i] >= cz) o |= 4;
        double q = h * 0.5;
        cx = cx + ((o & 1) ? q : -q);
        cy = cy + ((o & 2) ? q : -q);
        cz = cz + ((o & 4) ? q : -q);
        h = q;
      }
      if (d < 21)
        kh |= o << (60 - 3 * d);
      else
        kl |= o << (54 - 3 * (d - 21));
    }
    hi[i] = kh;
    lo[i] = kl;
  }
}

// compute_acceleration_system: a = F / m (integrators.rs:110-118).
void oracle_accel(int64_t n, const double* fx, const double* fy, const double* fz,
                  const double* m, double* ax, double* ay, double* az) {
  for (int64_t i = 0; i < n; ++i) {
    ax[i] = fx[i] / m[i];
    ay[i] = fy[i] / m[i];
    az[i] = fz[i] / m[i];
  }
}

// velocity_verlet_position_system (integrators.rs:63-83).
void oracle_vv_position(int64_t n, double dt, double* x, double* y, double* z, const double* vx,
                        const double* vy, const double* vz, const double* ax, const double* ay,
                        const double* az, double* pax, double* pay, double* paz) {
  const double half_dt_sq = 0.5 * dt * dt;
  for (int64_t i = 0; i < n; ++i) {
    pax[i] = ax[i];
    pay[i] = ay[i];
    paz[i] = az[i];
    x[i] = x[i] + (vx[i] * dt + ax[i] * half_dt_sq);
    y[i] = y[i] + (vy[i] * dt + ay[i] * half_dt_sq);
    z[i] = z[i] + (vz[i] * dt + az[i] * half_dt_sq);
  }
}

// velocity_verlet_velocity_system (integrators.rs:92-104).
void oracle_vv_velocity(int64_t n, double dt, double* vx, double* vy, double* vz,
                        const double* ax, const double* ay, const double* az, const double* pax,
                        const double* pay, const double* paz) {
  const double half_dt = 0.5 * dt;
  for (int64_t i = 0; i < n; ++i) {
    vx[i] = vx[i] + (pax[i] + ax[i]) * half_dt;
    vy[i] = vy[i] + (pay[i] + ay[i]) * half_dt;
    vz[i] = vz[i] + (paz[i] + az[i]) * half_dt;
  }
}

// nfw_density (nfw.rs:61-67)
double oracle_nfw_density(double r, double rho_0, double rs) {
  if (r <= 0.0 || rs <= 0.0) return 0.0;
  const double x = r / rs;
  const double opx = 1.0 + x;
  return rho_0 / (x * (opx * opx));  // powi(2)
}

// nfw_enclosed_mass (nfw.rs:76-83)
double oracle_nfw_enclosed_mass(double r, double rho_0, double rs) {
  if (r <= 0.0 || rs <= 0.0) return 0.0;
  const double x = r / rs;
  const double factor = 4.0 * 3.141592653589793 * rho_0 * (rs * rs * rs);  // powi(3)
  return factor * (std::log(1.0 + x) - x / (1.0 + x));
}

// nfw_circular_velocity (nfw.rs:88-91), G = constants.rs:7
double oracle_nfw_circular_velocity(double r, double rho_0, double rs) {
  const double m_enc = oracle_nfw_enclosed_mass(r, rho_0, rs);
  return std::sqrt(std::fmax(6.67430e-11 * m_enc / r, 0.0));
}

// nfw_gravity_system (nfw.rs:103-139): Force += -r_hat * (G M(r) m / r^2)
// for every body at r >= 1e-10 from the centre.  halo = {rho_0, Rs, cx, cy, cz}.
void oracle_nfw_forces(int64_t n, const double* x, const double* y, const double* z,
                       const double* m, const double* halo, double* fx, double* fy,
                       double* fz) {
  const double rho_0 = halo[0], rs = halo[1];
  const V3 c = v3(halo[2], halo[3], halo[4]);
  for (int64_t i = 0; i < n; ++i) {
    const V3 rv = sub(v3(x[i], y[i], z[i]), c);
    const double r = std::sqrt(len2(rv));
    if (r < 1e-10) continue;
    const double m_enc = oracle_nfw_enclosed_mass(r, rho_0, rs);
    const V3 rh = divs(rv, r);
    const double f_mag = 6.67430e-11 * m_enc * m[i] / (r * r);
    const V3 f = mul(v3(-rh.x, -rh.y, -rh.z), f_mag);
    fx[i] = fx[i] + f.x;
    fy[i] = fy[i] + f.y;
    fz[i] = fz[i] + f.z;
  }
}

}  // extern "C"

// One reference force pass: reset_forces (forces.rs:15-19), the gravity system
// (method 0 direct, 1 Barnes-Hut), nfw_gravity_system when `halo` is given
// (src/main.rs:109-110), compute_acceleration_system.
static void force_pass(int64_t n, const double* x, const double* y, const double* z,
                       const double* m, double g, double eps, double theta, int method,
                       int nthreads, double* fx, double* fy, double* fz, double* ax, double* ay,
                       double* az, const double* halo, const double* hx = nullptr,
                       const double* hy = nullptr, const double* hz = nullptr) {
  for (int64_t i = 0; i < n; ++i) fx[i] = fy[i] = fz[i] = 0.0;
  std::vector<double> gx(n, 0.0), gy(n, 0.0), gz(n, 0.0);
  if (method == 0)
    oracle_direct_forces(n, x, y, z, m, g, eps, nthreads, gx.data(), gy.data(), gz.data());
  else
    oracle_bh_forces(n, x, y, z, m, g, eps, theta, nthreads, gx.data(), gy.data(), gz.data(),
                     nullptr);
  for (int64_t i = 0; i < n; ++i) {  // Force += computed (gravity.rs:71-73)
    fx[i] = fx[i] + gx[i];
    fy[i] = fy[i] + gy[i];
    fz[i] = fz[i] + gz[i];
  }
  // the halo reads LocalPosition (nfw.rs:118): hx/hy/hz when given
  if (halo) oracle_nfw_forces(n, hx ? hx : x, hy ? hy : y, hz ? hz : z, m, halo, fx, fy, fz);
  oracle_accel(n, fx, fy, fz, m, ax, ay, az);
}

extern "C" {

// The reference's Velocity-Verlet tick (src/main.rs:103-140), `nsteps` times:
// chain 1 = force pass, position step; chain 2 = force pass, velocity step.
// a/pa arrays hold Acceleration / PreviousAcceleration in and out.
// `halo` (NULL or {rho_0, Rs, cx, cy, cz}) adds nfw_gravity_system to both
// force passes.
void oracle_vv_run_halo(int64_t n, double* x, double* y, double* z, double* vx, double* vy,
                        double* vz, const double* m, double g, double eps, double theta,
                        int method, double dt, int64_t nsteps, int nthreads, double* ax,
                        double* ay, double* az, double* pax, double* pay, double* paz,
                        const double* halo) {
  std::vector<double> fx(n), fy(n), fz(n);
  for (int64_t s = 0; s < nsteps; ++s) {
    force_pass(n, x, y, z, m, g, eps, theta, method, nthreads, fx.data(), fy.data(), fz.data(),
               ax, ay, az, halo);
    oracle_vv_position(n, dt, x, y, z, vx, vy, vz, ax, ay, az, pax, pay, paz);
    force_pass(n, x, y, z, m, g, eps, theta, method, nthreads, fx.data(), fy.data(), fz.data(),
               ax, ay, az, halo);
    oracle_vv_velocity(n, dt, vx, vy, vz, ax, ay, az, pax, pay, paz);
  }
}

// Rust `f as i64`: saturating, NaN -> 0.
static int64_t sat_i64(double v) {
  if (v != v) return 0;
  if (v >= 9223372036854775807.0) return INT64_MAX;
  if (v <= -9223372036854775808.0) return INT64_MIN;
  return (int64_t)v;
}

// sector_boundary_system (origin.rs:16-24) = normalize_position per body
// (coordinates.rs:82-103).  Returns 1 if any body changed sector.
int oracle_normalize(int64_t n, int64_t* sx, int64_t* sy, int64_t* sz, double* lx, double* ly,
                     double* lz, double sector_size) {
  int any = 0;
  int64_t* S[3] = {sx, sy, sz};
  double* L[3] = {lx, ly, lz};
  for (int64_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      const double shift = std::round(L[k][i] / sector_size);
      if (shift != 0.0) {
        S[k][i] = (int64_t)((uint64_t)S[k][i] + (uint64_t)sat_i64(shift));
        L[k][i] -= shift * sector_size;
        any = 1;
      }
    }
  return any;
}

// The reference's Velocity-Verlet tick on (Sector, LocalPosition)
// (src/main.rs:103-150): each force pass flattens the positions
// (gravity.rs:38-47; Barnes-Hut: each body its own origin,
// gravity_tree.rs:280-291), the integrators update LocalPosition, and
// sector_boundary_system runs after the velocity step.
void oracle_vv_run_sectors(int64_t n, int64_t* sx, int64_t* sy, int64_t* sz, double* lx,
                           double* ly, double* lz, double* vx, double* vy, double* vz,
                           const double* m, double sector_size, double g, double eps,
                           double theta, int method, double dt, int64_t nsteps, int nthreads,
                           double* ax, double* ay, double* az, double* pax, double* pay,
                           double* paz, const double* halo) {
  std::vector<double> fx(n), fy(n), fz(n), x(n), y(n), z(n);
  const int quirk = method == 1 ? 1 : 0;
  for (int64_t s = 0; s < nsteps; ++s) {
    oracle_flatten(n, sx, sy, sz, lx, ly, lz, sector_size, quirk, x.data(), y.data(), z.data());
    force_pass(n, x.data(), y.data(), z.data(), m, g, eps, theta, method, nthreads, fx.data(),
               fy.data(), fz.data(), ax, ay, az, halo, lx, ly, lz);
    oracle_vv_position(n, dt, lx, ly, lz, vx, vy, vz, ax, ay, az, pax, pay, paz);
    oracle_flatten(n, sx, sy, sz, lx, ly, lz, sector_size, quirk, x.data(), y.data(), z.data());
    force_pass(n, x.data(), y.data(), z.data(), m, g, eps, theta, method, nthreads, fx.data(),
               fy.data(), fz.data(), ax, ay, az, halo, lx, ly, lz);
    oracle_vv_velocity(n, dt, vx, vy, vz, ax, ay, az, pax, pay, paz);
    oracle_normalize(n, sx, sy, sz, lx, ly, lz, sector_size);
  }
}

void oracle_vv_run(int64_t n, double* x, double* y, double* z, double* vx, double* vy,
                   double* vz, const double* m, double g, double eps, double theta, int method,
                   double dt, int64_t nsteps, int nthreads, double* ax, double* ay, double* az,
                   double* pax, double* pay, double* paz) {
  oracle_vv_run_halo(n, x, y, z, vx, vy, vz, m, g, eps, theta, method, dt, nsteps, nthreads, ax,
                     ay, az, pax, pay, paz, nullptr);
}

// compute_kinetic_energy_system (energy.rs:21-30), compute_potential_energy_system
// (energy.rs:34-56, unsoftened, pairs in iter_combinations order, r2 == 0
// skipped) and the total linear momentum sum of update_momentum_system
// (integrators.rs:123-129).  Positions are in one sector, so displacement is
// 0*sector_size + (b - a) (coordinates.rs:51-65).
void oracle_energy(int64_t n, const double* x, const double* y, const double* z,
                   const double* vx, const double* vy, const double* vz, const double* m,
                   double g, double* out5) {
  double ke = 0.0;
  for (int64_t i = 0; i < n; ++i) ke += 0.5 * m[i] * len2(v3(vx[i], vy[i], vz[i]));
  double pe = 0.0;
  for (int64_t a = 0; a < n; ++a)
    for (int64_t b = a + 1; b < n; ++b) {
      V3 d = add(v3(0.0, 0.0, 0.0), sub(v3(x[b], y[b], z[b]), v3(x[a], y[a], z[a])));
      double r2 = len2(d);
      if (r2 > 0.0) {
        double r = std::sqrt(r2);
        pe -= (g * m[a] * m[b]) / r;
      }
    }
  V3 p = v3(0.0, 0.0, 0.0);
  for (int64_t i = 0; i < n; ++i) p = add(p, mul(v3(vx[i], vy[i], vz[i]), m[i]));
  out5[0] = ke;
  out5[1] = pe;
  out5[2] = p.x;
  out5[3] = p.y;
  out5[4] = p.z;
}

// Independent systems (CSR `off`, nsys+1 entries): each one stepped with the
// reference's direct-sum Velocity-Verlet tick, single-threaded per system,
// systems spread over threads.
void oracle_ensemble_run(int64_t nsys, const int64_t* off, double* x, double* y, double* z,
                         double* vx, double* vy, double* vz, const double* m, double g, double eps,
                         double dt, int64_t nsteps, int nthreads, double* ax, double* ay,
                         double* az) {
  par_chunks(nsys, nthreads, 1, [&](int64_t lo, int64_t hi) {
    for (int64_t s = lo; s < hi; ++s) {
      int64_t b = off[s], k = off[s + 1] - off[s];
      std::vector<double> pax(k), pay(k), paz(k);
      oracle_vv_run(k, x + b, y + b, z + b, vx + b, vy + b, vz + b, m + b, g, eps, 0.0, 0, dt,
                    nsteps, 1, ax + b, ay + b, az + b, pax.data(), pay.data(), paz.data());
    }
  });
}

}  // extern "C"
