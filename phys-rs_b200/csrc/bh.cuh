// Barnes-Hut tree layout shared by the build (tree.cu) and the walk (walk.cu).
//
// Nodes are the non-empty cells of the octree in pre-order (children in
// octant order 0..7, the order OctreeNode::compute_force visits them,
// gravity_tree.rs:200-204).  Per node:
//   link  int4  {next, start, end, meta}
//         next  = pre-order index after the node's subtree (skip pointer)
//         start, end = the cell's bodies in key-sorted order [start, end)
//         meta  = depth | kLeaf | kGuard | kGate
//   rec   walk record: for a one-body leaf (and a guard leaf with leaf_cap 1)
//         the stored body's own position and mass; otherwise the cell's
//         centre of mass and total mass.  double4 for f64 walks; for f32
//         walks two float4: (x_hi, y_hi, z_hi, m) and (x_lo, y_lo, z_lo, 0).
//   mc    double4 aggregate (com x, y, z, total mass) of all bodies in the
//         cell (the reference's center_of_mass / total_mass fields).
#pragma once

#include "common.cuh"

namespace phys {

constexpr int kMetaDepth = 0xff;
constexpr int kMetaLeaf = 1 << 8;    // leaf cell (no children in this tree)
constexpr int kMetaGuard = 1 << 9;   // leaf at the guard depth D* (gravity_tree.rs:121-126)
constexpr int kMetaGate = 1 << 10;   // total_mass > 0 (children are visited only then,
                                     // gravity_tree.rs:201)

// Walk records (array of structures, 48 B, one per node, read with three
// independent 16-B loads):
//   l = {next, self, start, meta}: self = sorted position of the body a
//   one-body leaf stores (-1 otherwise, also the self-exclusion test);
//   start = first body of a bucket leaf; meta = depth | kWLeaf | count << 8.
//   A cell whose total mass is not > 0 (other than the root) gets depth
//   kWSkip, which no lane can be active at, so the warp jumps over it.
constexpr int kWDepth = 63;
constexpr int kWSkip = 63;
constexpr int kWLeaf = 1 << 6;
struct __align__(16) Rec32 {
  float4 a;  // x_hi, y_hi, z_hi, mass
  float4 b;  // x_lo, y_lo, z_lo, ropen2 = s_d^2 / theta^2 (-1: one-body leaf, always taken)
  int4 l;
};
// Paired F32C record for the two-targets-per-lane walk: every value stored
// twice so packed f32x2 instructions take it straight from the load.
struct __align__(16) Rec32x2 {
  float4 q0;  // x_hi, x_hi, y_hi, y_hi
  float4 q1;  // z_hi, z_hi, mass, mass
  float4 q2;  // x_lo, x_lo, y_lo, y_lo
  float4 q3;  // z_lo, z_lo, ropen2, ropen2
  int4 l;
};
struct __align__(16) Body32x2 {
  float4 q0, q1, q2, q3;  // same layout, ropen2 slot unused
};
// Group-walk record, breadth-first order (children of a cell contiguous).
// l = {a, (b << 2) | type, first body, end body} (sorted positions; the
// cell holds bodies [first, end)).  internal: a = first child, b = child
// count; one-body leaf: a = the body it stands for (the last inserted one for
// a guard leaf of capacity 1); bucket leaf: a = first body, b = body count;
// skip: a cell whose total mass is not > 0 (never the root).
constexpr int kGroupMax = 64;  // bodies per target group (one warp, two per lane)
constexpr int kGInternal = 0;
constexpr int kGSingle = 1;
constexpr int kGBucket = 2;
constexpr int kGSkip = 3;
struct __align__(16) GNode {
  float4 hi;    // x_hi, y_hi, z_hi, mass (f32)
  float4 lo;    // x_lo, y_lo, z_lo, cell side squared (2h)^2 (f32)
  int4 l;
  double4 c64;  // x, y, z, mass (f64)
};
static_assert(sizeof(GNode) == 80, "GNode layout");
struct __align__(16) Rec64 {
  double4 a;  // x, y, z, mass
  int4 l;
};

struct BhTree {
  int64_t n = 0;
  int64_t nnodes = 0;
  int leaf_cap = 1;
  const int4* link = nullptr;
  const double4* rec64 = nullptr;     // exact walk: record per node (with `link`)
  const Rec32* w32 = nullptr;         // F32C walk records
  const Rec32x2* w32x2 = nullptr;     // F32C paired walk records
  const Body32x2* body2 = nullptr;    // sorted bodies, paired layout
  const Rec64* w64 = nullptr;         // F64 walk records
  const double4* mc = nullptr;
  const uint32_t* perm = nullptr;     // sorted position -> caller index
  const double4* body64 = nullptr;    // sorted bodies (x, y, z, m)
  const float4* body_hi = nullptr;    // sorted bodies, double-float hi + f32 mass
  const float4* body_lo = nullptr;
  const TreeHeader* hdr = nullptr;
  const GNode* gnode = nullptr;       // group-walk records (breadth-first)
  const int2* groups = nullptr;       // group-walk target groups: body ranges [x, y),
                                      // room for n more (re-queued subgroups) after n
  const int32_t* ngroups = nullptr;   // device: number of groups
  int32_t* group_ctr = nullptr;       // device: walk counters (reset per walk)
  const uint64_t* keys_hi_sorted = nullptr;  // descent keys, octants 0..20, sorted
  const uint64_t* keys_lo = nullptr;         // octants 21..39, caller order
};

// tree.cu
// full_com: the reference-form centre of mass of every cell (export); else
// cells no target can take as a monopole get only their mass.
int bh_build(phys_ctx* c, const phys_params* p, bool need_f32, BhTree* t, bool need_group = false,
             bool full_com = true);
// walk.cu
int bh_group_walk(phys_ctx* c, const phys_params* p, const BhTree& t, bool want_force,
                  double* ox, double* oy, double* oz);
int bh_walk(phys_ctx* c, const phys_params* p, const BhTree& t, bool want_force, double* ox,
            double* oy, double* oz);

}  // namespace phys
