// Group walk (PHYS_FLAG_GROUP_WALK): Barnes-Hut forces for a group of up to
// 64 key-adjacent bodies per warp from one shared interaction list.
//
// The reference walks the octree once per body (gravity_tree.rs:171-209,
// criterion (2h)^2 < theta^2 d^2 at :194).  Here the bodies are split into
// groups that each lie inside one cell (the children of a cell with more
// than 64 bodies, consecutive small siblings packed together; built with the
// tree), and the tree is walked once per group:
//   - a warp pops up to 32 cells from a stack in shared memory, one per
//     lane, and tests each against the group's bounding box: a cell is a
//     monopole only when (2h)^2 < theta^2 d_min^2, d_min the distance from
//     its centre of mass to the nearest point of the box (d_min <= d for
//     every target, so the per-body criterion holds for each of them);
//   - an opened cell pushes its children (contiguous in the breadth-first
//     record array); a one-body leaf, an accepted cell and every body of an
//     opened bucket leaf become entries of the group's interaction list;
//   - the group's own bodies never enter the list: a cell whose bodies all
//     belong to the group is skipped, one that holds some of them is always
//     opened, and pairs inside the group are summed exactly in a separate
//     pass that skips i == j.
// Three launches:
//   1. glist_kernel walks every group and writes its list as 4-byte codes
//      (cell or body index) to a per-warp region of a global pool; a group
//      whose list passes kGListLimit entries (a sparse group whose box
//      reaches a much denser region) is abandoned and re-queued as
//      subgroups of kGSplit consecutive bodies, whose lists are far shorter;
//   2. geval_kernel evaluates the lists: batches of kEB entries stream
//      through shared memory (cp.async, two batches in flight), then every
//      lane accumulates its one or two targets over the batch (broadcast
//      loads; the target layouts are described at Evaluator);
//   3. gwalk_kernel walks and evaluates the re-queued subgroups in one pass
//      (list in shared memory, evaluated whenever it fills), on a second
//      stream beside geval_kernel: these are a few hundred serial walks at
//      most, bound by the latency of their tree reads, not by throughput.
// The list arithmetic is the per-body walk's: F64 = f64 FMA + rsqrt on
// absolute coordinates; F32C = f32 pair terms on double-float coordinates
// relative to the group's first body, r = (hi_j - hi_i) + (lo_j - lo_i), two
// list entries per packed f32x2 operation, partial sums folded into a
// (hi, lo) accumulator by two-sum every kGFlushPairs entry pairs (counted
// across the near and far lists and across staging batches).  The
// opening decisions are made in f32 for both precisions (with a 1e-5
// relative margin toward opening), so both evaluate the same lists.
//
// Stack bound: a round pops k cells and pushes at most 8 children per cell.
// While the stack holds at most kGThrottle - 7 ids, k is limited so that it
// cannot grow past kGThrottle; above that the warp pops one cell per round,
// which is a depth-first walk: it adds at most 7 ids per level below the
// popped cell, so the stack never holds more than kGThrottle + 7 * kMaxLevels
// + 1 <= kGStack ids.  Every round pops at least one cell and a well-formed
// tree has each cell pushed once, so a walk ends after at most nnodes pops;
// a malformed tree (child index not after its parent, more pops than cells)
// sets kStatOverflow and the warp stops.
#include <algorithm>
#include <climits>

#include "bh.cuh"

#ifndef GWALK_FLUSH_PAIRS
#define GWALK_FLUSH_PAIRS 64
#endif
#ifndef GWALK_LIST_LIMIT
#define GWALK_LIST_LIMIT 8192
#endif
#ifndef GWALK_SPLIT
#define GWALK_SPLIT 1
#endif
#ifndef GWALK_FAR
#define GWALK_FAR 0.0625
#endif
#ifndef GEVAL_UNROLL
#define GEVAL_UNROLL 2
#endif
#ifndef GLIST_MIN_BLOCKS
#define GLIST_MIN_BLOCKS 1
#endif
#ifndef GEVAL_MIN_BLOCKS
#define GEVAL_MIN_BLOCKS 4
#endif
#ifndef GWALK_PREFETCH
#define GWALK_PREFETCH 0
#endif
#ifndef GWALK_POOL_PER_BODY
#define GWALK_POOL_PER_BODY 128
#endif

namespace phys {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kGWarps = 4;  // evaluating kernels
constexpr int kGBlock = 32 * kGWarps;
constexpr int kLWarps = 8;  // list kernel
constexpr int kLBlock = 32 * kLWarps;
constexpr int kGStack = 1024;  // node ids per warp
constexpr int kGList = 256;    // shared-memory list entries per warp, 32 bytes each
constexpr int kGThrottle = kGStack - 8 - 7 * kMaxLevels;
constexpr int kGFlushPairs = GWALK_FLUSH_PAIRS;
constexpr int kEvalUnroll = GEVAL_UNROLL;  // 4-entry chunks in flight per lane
constexpr int kGListLimit = GWALK_LIST_LIMIT;  // first-pass budget (typical lists: 3-4k)
constexpr int kGSplit = GWALK_SPLIT;            // bodies per re-queued subgroup
// list codes a region must have free before a walk starts: the first-pass
// budget plus one round's entries (32 cells, bucket leaves of at most
// kMaxLeafCap bodies) and slack
constexpr int kGRegionNeed = kGListLimit + 32 * kMaxLeafCap + 64;
// fused kernel, per warp: stack | list | emission records (end, kind, a, olo,
// ohi and the source double4 per lane)
constexpr int kGListOff = kGStack * 4;
constexpr int kGRecOff = kGListOff + kGList * 32;
constexpr int kGSmemWarp = kGRecOff + 5 * 32 * 4 + 32 * 32;
constexpr int kGSmem = kGWarps * kGSmemWarp;
constexpr int kLSmem = kLWarps * kGStack * 4;  // list kernel: stacks
// evaluation kernel, per warp: near list (7 arrays) | far list (4 arrays) of
// kEB entries, then two staging buffers of kEB source records
#ifndef GEVAL_BATCH
#define GEVAL_BATCH 128
#endif
constexpr int kEB = GEVAL_BATCH;  // list entries per staging batch
constexpr int kEListBytes = kEB * 7 * 4 + kEB * 4 * 4;
constexpr int kESmemWarp = kEListBytes + 2 * kEB * 32;
constexpr int kESmem = kGWarps * kESmemWarp;
static_assert(kEListBytes % 32 == 0 && kEB >= kGroupMax && kEB % 32 == 0,
              "evaluation kernel layout");
static_assert(kGroupMax == 64, "two targets per lane");
static_assert(kGThrottle >= 7 * 32 + 7, "stack too small for batched pops");
static_assert(kGThrottle + 7 * kMaxLevels + 1 <= kGStack, "stack bound");
// kGFlushPairs % 4: the split layouts (33-48-body groups) step through the
// chunks two at a time and need an even chunk count between flushes.
static_assert(kGList % 4 == 0 && kGFlushPairs % 4 == 0, "list chunks of 4 entries");
static_assert((kGRecOff + 5 * 32 * 4) % 16 == 0, "record alignment");

__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }
// Two consecutive floats from an 8-byte-aligned shared-memory address.
__device__ __forceinline__ float2 ld2(const float* p) {
  return *reinterpret_cast<const float2*>(p);
}

__device__ __forceinline__ double4 ldg_d4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  const double2 a = __ldg(q), b = __ldg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

// 16-byte asynchronous copy global -> shared (L2 only), its commit and wait.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

// Packed two-sum: s + e == a + b exactly, per component.
__device__ __forceinline__ void two_sum2(float2 a, float2 b, float2& s, float2& e) {
  s = __fadd2_rn(a, b);
  const float2 bb = __fadd2_rn(s, make_float2(-a.x, -a.y));
  const float2 ab = __fadd2_rn(s, make_float2(-bb.x, -bb.y));
  e = __fadd2_rn(__fadd2_rn(a, make_float2(-ab.x, -ab.y)), __fadd2_rn(b, make_float2(-bb.x, -bb.y)));
}

// ---------------------------------------------------------------------------
// Group box and node classification
// ---------------------------------------------------------------------------
struct Box {
  float cx, cy, cz, bx, by, bz;  // centre and half extent, relative to X0
  float hx, lx, hy, ly, hz, lz;  // X0 as double-float
};

// Warp-collective: box of the targets ta, tb of every lane (idle lanes pass
// X0, a group body).
__device__ __forceinline__ Box group_box(double4 X0, double4 ta, double4 tb) {
  Box B;
  const float ax = (float)(ta.x - X0.x), ay = (float)(ta.y - X0.y), az = (float)(ta.z - X0.z);
  const float bx = (float)(tb.x - X0.x), by = (float)(tb.y - X0.y), bz = (float)(tb.z - X0.z);
  const float mnx = warp_min(fminf(ax, bx)), mxx = warp_max(fmaxf(ax, bx));
  const float mny = warp_min(fminf(ay, by)), mxy = warp_max(fmaxf(ay, by));
  const float mnz = warp_min(fminf(az, bz)), mxz = warp_max(fmaxf(az, bz));
  B.cx = 0.5f * (mnx + mxx);
  B.cy = 0.5f * (mny + mxy);
  B.cz = 0.5f * (mnz + mxz);
  // widened by the rounding of the f32 coordinates (a few ulp of |c| + b)
  B.bx = 0.5f * (mxx - mnx);
  B.by = 0.5f * (mxy - mny);
  B.bz = 0.5f * (mxz - mnz);
  B.bx = B.bx * (1.0f + 1e-6f) + 1e-6f * (fabsf(B.cx) + B.bx);
  B.by = B.by * (1.0f + 1e-6f) + 1e-6f * (fabsf(B.cy) + B.by);
  B.bz = B.bz * (1.0f + 1e-6f) + 1e-6f * (fabsf(B.cz) + B.bz);
  split_df(X0.x, B.hx, B.lx);
  split_df(X0.y, B.hy, B.ly);
  split_df(X0.z, B.hz, B.lz);
  return B;
}

// What one popped cell contributes: children to push, and list entries
// (kind 1: the cell itself / the body of a one-body leaf, source c64 of
// record a; kind 2: the bodies [a, a + nent) of a bucket leaf, skipping the
// group's range [olo, ohi)).
struct NodeOut {
  int npush, cfirst, nent, kind, a, olo, ohi;
  bool malformed;
  double4 c64;
};

template <bool kNeedC64>
__device__ __forceinline__ void classify(int nd, int base, int gend, int nnodes, const Box& B,
                                         float theta2f, const GNode* __restrict__ gn,
                                         NodeOut& o) {
  o.npush = o.cfirst = o.nent = o.kind = o.a = o.olo = o.ohi = 0;
  o.malformed = false;
  o.c64 = make_double4(0.0, 0.0, 0.0, 0.0);
  if (nd < 0) return;
  // the whole record in one round trip
  const GNode* g = gn + nd;
  const int4 l = __ldg(&g->l);
  const float4 h = __ldg(&g->hi), lo = __ldg(&g->lo);
  if (kNeedC64) o.c64 = ldg_d4(&g->c64);
  const int type = l.y & 3, cnt = l.y >> 2;
  const bool inside = l.z >= base && l.w <= gend;  // only group bodies
  if (type == kGSkip || inside) return;
  if (type == kGSingle) {
    if (l.x < base || l.x >= gend) {
      o.nent = 1;
      o.kind = 1;
      o.a = nd;
    }
    return;
  }
  const bool overlap = l.z < gend && l.w > base;
  bool acc = false;
  if (!overlap) {
    const float rx = (h.x - B.hx) + (lo.x - B.lx);
    const float ry = (h.y - B.hy) + (lo.y - B.ly);
    const float rz = (h.z - B.hz) + (lo.z - B.lz);
    const float dx = fmaxf(fabsf(rx - B.cx) - B.bx, 0.f);
    const float dy = fmaxf(fabsf(ry - B.cy) - B.by, 0.f);
    const float dz = fmaxf(fabsf(rz - B.cz) - B.bz, 0.f);
    const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    acc = lo.w < theta2f * d2 * (1.0f - 1e-5f);
  }
  if (acc) {
    o.nent = 1;
    o.kind = 1;
    o.a = nd;
  } else if (type == kGInternal) {
    if (l.x <= nd || cnt < 1 || cnt > 8 || l.x + cnt > nnodes) {
      o.malformed = true;
    } else {
      o.npush = cnt;
      o.cfirst = l.x;
    }
  } else {  // bucket leaf opened: its bodies outside the group
    o.a = l.z;
    o.olo = max(l.z, base);
    o.ohi = min(l.w, gend);
    o.nent = (l.w - l.z) - max(o.ohi - o.olo, 0);
    o.kind = 2;
  }
}

// Sorted position of entry j of a bucket leaf's bodies outside the group.
__device__ __forceinline__ int bucket_body(int a, int olo, int ohi, int j) {
  int q = a + j;
  if (olo < ohi && q >= olo) q += ohi - olo;
  return q;
}

// Walks the tree for the group [base, gend); sink(etot, eoff, o) receives
// each round's entries (etot in all, this lane's at eoff) and returns false
// to stop.  Returns 1 when the walk completed, 0 when the list passed
// `limit` entries or the sink stopped it, -1 on a malformed tree or a full
// stack.
template <bool kNeedC64, class Sink>
__device__ __forceinline__ int traverse(int lane, int base, int gend, int nnodes, int limit,
                                        int* stk, const Box& B, float theta2f,
                                        const GNode* __restrict__ gn, Sink& sink) {
  int ssize = 1, listed = 0;
  long long pops = 0;
  if (lane == 0) stk[0] = 0;
  __syncwarp();
  while (ssize > 0) {
    if (listed > limit) return 0;
    const int k = ssize <= kGThrottle - 7 ? min(min(32, ssize), (kGThrottle - ssize) / 7) : 1;
    const int nd = lane < k ? stk[ssize - 1 - lane] : -1;
    ssize -= k;
    pops += k;
    __syncwarp();
    NodeOut o;
    classify<kNeedC64>(nd, base, gend, nnodes, B, theta2f, gn, o);
    if (pops > nnodes) o.malformed = true;
    // both scans first (independent chains), then pushes, then entries
    const int pin = warp_incl_scan(o.npush, lane);
    const int ein = warp_incl_scan(o.nent, lane);
    const int ptot = __shfl_sync(kFull, pin, 31);
    const int etot = __shfl_sync(kFull, ein, 31);
    if (__any_sync(kFull, o.malformed) || ssize + ptot > kGStack) return -1;
    for (int c = 0; c < o.npush; ++c) stk[ssize + pin - o.npush + c] = o.cfirst + c;
    if (GWALK_PREFETCH && o.npush > 0) {
      // the children are popped in the next rounds: bring their records
      // (contiguous, breadth-first) into L1 now, so those rounds' loads do
      // not wait for L2
      const uintptr_t a0 = reinterpret_cast<uintptr_t>(gn + o.cfirst) & ~uintptr_t(127);
      const uintptr_t a1 = reinterpret_cast<uintptr_t>(gn + o.cfirst + o.npush);
      for (uintptr_t a = a0; a < a1; a += 128)
        asm volatile("prefetch.global.L1 [%0];" ::"l"(a));
    }
    ssize += ptot;
    listed += etot;
    if (etot > 0 && !sink(etot, ein - o.nent, o)) return 0;
    __syncwarp();  // pushes and entries visible to every lane
  }
  return 1;
}

// ---------------------------------------------------------------------------
// Evaluation of a list against the group's targets
// ---------------------------------------------------------------------------
// The F32C list in shared memory is a structure of arrays (slot-consecutive
// writes hit distinct banks; the evaluation reads four entries per 16-byte
// load).
// Target layouts: one per lane (at most 32 bodies); two per lane, 2l and
// 2l + 1 (33..64 bodies; F32C 49..64); F32C 33..48 bodies: target a = l and
// target b = 32 + l mod (32 / rb), the lanes of b split into rb = 2 (41..48
// bodies) or 4 (33..40) streams that each take a 1/rb share of the list's
// entries for b, so that the second slot carries no idle lanes; the
// streams' sums for b are added at the end.
template <bool kF32, int kL>
struct Evaluator {
  int lane, nvalid, ia, ib;
  bool va, vb;
  bool two;  // a second target per lane (more than 32 bodies), else one
  int rb;    // streams sharing each b target (2 or 4), 0: one lane per target
  double4 X0, ta, tb;
  double eps2;
  float* f;        // F32C list: hx, hy, hz, m, lx, ly, lz arrays of kL
  float* ff;       // F32C far list: hx, hy, hz, m arrays of kL (or null)
  double4* lst64;  // F64 list
  float2 nhxa, nhya, nhza, nlxa, nlya, nlza, nhxb, nhyb, nhzb, nlxb, nlyb, nlzb;
  float2 e2;
  float2 pxa, pya, pza, pxb, pyb, pzb;  // partials (entry halves)
  int pend;                             // 4-entry chunks in the partials
  float2 Hx, Hy, Hz, Lx, Ly, Lz;        // (target a, target b)
  double ax, ay, az, bx, by, bz;        // F64 sums

  __device__ __forceinline__ void init(int lane_, int base, int gend,
                                       const double4* __restrict__ body64, unsigned char* lbase,
                                       double eps2_) {
    lane = lane_;
    nvalid = gend - base;
    two = nvalid > 32;
    rb = (kF32 && two && nvalid <= 48) ? (nvalid <= 40 ? 4 : 2) : 0;
    if (rb) {
      ia = base + lane;
      ib = base + 32 + lane % (32 / rb);
    } else {
      ia = two ? base + 2 * lane : base + lane;
      ib = two ? ia + 1 : gend;
    }
    va = ia < gend;
    vb = ib < gend;
    X0 = body64[base];
    ta = va ? body64[ia] : X0;
    tb = vb ? body64[ib] : X0;
    eps2 = eps2_;
    f = reinterpret_cast<float*>(lbase);
    ff = f + 7 * kL;
    lst64 = reinterpret_cast<double4*>(lbase);
    float h, l;
    split_df(ta.x - X0.x, h, l); nhxa = make_float2(-h, -h); nlxa = make_float2(-l, -l);
    split_df(ta.y - X0.y, h, l); nhya = make_float2(-h, -h); nlya = make_float2(-l, -l);
    split_df(ta.z - X0.z, h, l); nhza = make_float2(-h, -h); nlza = make_float2(-l, -l);
    split_df(tb.x - X0.x, h, l); nhxb = make_float2(-h, -h); nlxb = make_float2(-l, -l);
    split_df(tb.y - X0.y, h, l); nhyb = make_float2(-h, -h); nlyb = make_float2(-l, -l);
    split_df(tb.z - X0.z, h, l); nhzb = make_float2(-h, -h); nlzb = make_float2(-l, -l);
    const float e = (float)eps2;
    e2 = make_float2(e, e);
    const float2 z = make_float2(0.f, 0.f);
    pxa = pya = pza = pxb = pyb = pzb = z;
    Hx = Hy = Hz = Lx = Ly = Lz = z;
    ax = ay = az = bx = by = bz = 0.0;
    pend = 0;
  }

  // The partials are folded into (H, L) every kFlushChunks chunks, across
  // the near and far lists and across batches.
  static constexpr int kFlushChunks = kGFlushPairs / 2;
  __device__ __forceinline__ void chunks_done(int k) {
    pend += k;
    if (pend >= kFlushChunks) {
      flush();
      pend = 0;
    }
  }

  // List slot from an absolute position + mass.
  __device__ __forceinline__ void put(int slot, double4 src) {
    if (kF32) {
      float h, l;
      split_df(src.x - X0.x, h, l);
      f[slot] = h;
      f[4 * kL + slot] = l;
      split_df(src.y - X0.y, h, l);
      f[kL + slot] = h;
      f[5 * kL + slot] = l;
      split_df(src.z - X0.z, h, l);
      f[2 * kL + slot] = h;
      f[6 * kL + slot] = l;
      f[3 * kL + slot] = (float)src.w;
    } else {
      lst64[slot] = src;
    }
  }

  __device__ __forceinline__ void flush() {
    float2 s, e;
    two_sum2(Hx, make_float2(pxa.x + pxa.y, pxb.x + pxb.y), s, e);
    Hx = s;
    Lx = __fadd2_rn(Lx, e);
    two_sum2(Hy, make_float2(pya.x + pya.y, pyb.x + pyb.y), s, e);
    Hy = s;
    Ly = __fadd2_rn(Ly, e);
    two_sum2(Hz, make_float2(pza.x + pza.y, pzb.x + pzb.y), s, e);
    Hz = s;
    Lz = __fadd2_rn(Lz, e);
    const float2 z = make_float2(0.f, 0.f);
    pxa = pya = pza = pxb = pyb = pzb = z;
  }

  // One F32C entry pair against one target; skip_e / skip_f zero the halves
  // that are the target itself (in-group pass).
  __device__ __forceinline__ void term32(float2 hx, float2 hy, float2 hz, float2 mm, float2 lx,
                                         float2 ly, float2 lz, float2 nhx, float2 nhy, float2 nhz,
                                         float2 nlx, float2 nly, float2 nlz, bool skip_e,
                                         bool skip_f, float2& px, float2& py, float2& pz) {
    const float2 rx = __fadd2_rn(__fadd2_rn(hx, nhx), __fadd2_rn(lx, nlx));
    const float2 ry = __fadd2_rn(__fadd2_rn(hy, nhy), __fadd2_rn(ly, nly));
    const float2 rz = __fadd2_rn(__fadd2_rn(hz, nhz), __fadd2_rn(lz, nlz));
    const float2 r2 = __ffma2_rn(rx, rx, __ffma2_rn(ry, ry, __ffma2_rn(rz, rz, e2)));
    const float2 inv = make_float2(rsqrt_sfu(r2.x), rsqrt_sfu(r2.y));
    float2 w = __fmul2_rn(mm, __fmul2_rn(__fmul2_rn(inv, inv), inv));
    if (skip_e) w.x = 0.f;
    if (skip_f) w.y = 0.f;
    px = __ffma2_rn(rx, w, px);
    py = __ffma2_rn(ry, w, py);
    pz = __ffma2_rn(rz, w, pz);
  }

  __device__ __forceinline__ void term64(double4 s, double4 t, double& sx, double& sy,
                                         double& sz) {
    const double rx = s.x - t.x, ry = s.y - t.y, rz = s.z - t.z;
    const double inv = rsqrt(fma(rx, rx, fma(ry, ry, fma(rz, rz, eps2))));
    const double w = s.w * (inv * inv * inv);
    sx = fma(rx, w, sx);
    sy = fma(ry, w, sy);
    sz = fma(rz, w, sz);
  }

  // Near chunks [q0, q1) of the list (double-float offsets) against the
  // lane's target a, and target b when kTwo.  One instantiation per target
  // count keeps all of a chunk's terms in one basic block, free to
  // interleave.
  template <bool kSelf, bool kTwo>
  __device__ __forceinline__ void near_chunks(int q0, int q1) {
    const float4* HX = reinterpret_cast<const float4*>(f);
    const float4* HY = reinterpret_cast<const float4*>(f + kL);
    const float4* HZ = reinterpret_cast<const float4*>(f + 2 * kL);
    const float4* MM = reinterpret_cast<const float4*>(f + 3 * kL);
    const float4* LX = reinterpret_cast<const float4*>(f + 4 * kL);
    const float4* LY = reinterpret_cast<const float4*>(f + 5 * kL);
    const float4* LZ = reinterpret_cast<const float4*>(f + 6 * kL);
#pragma unroll kEvalUnroll
    for (int q = q0; q < q1; ++q) {
      const float4 hx = HX[q], hy = HY[q], hz = HZ[q], mm = MM[q];
      const float4 lx = LX[q], ly = LY[q], lz = LZ[q];
      // in-group pass, the target's own slot: two per lane: target a is
      // slot 2*lane, target b 2*lane + 1 (chunk lane/2, pair lane & 1);
      // one per lane: slot lane (chunk lane/4, pair (lane/2) & 1, half
      // lane & 1)
      bool a0e = false, a0f = false, a1e = false, a1f = false, b0 = false, b1 = false;
      if (kSelf) {
        if (kTwo) {
          const bool in = q == (lane >> 1);
          a0e = b0 = in && !(lane & 1);
          a1e = b1 = in && (lane & 1);
        } else {
          const bool in = q == (lane >> 2);
          const bool p1 = (lane >> 1) & 1, h1 = lane & 1;
          a0e = in && !p1 && !h1;
          a0f = in && !p1 && h1;
          a1e = in && p1 && !h1;
          a1f = in && p1 && h1;
        }
      }
      term32(lo2(hx), lo2(hy), lo2(hz), lo2(mm), lo2(lx), lo2(ly), lo2(lz), nhxa, nhya, nhza,
             nlxa, nlya, nlza, a0e, a0f, pxa, pya, pza);
      term32(hi2(hx), hi2(hy), hi2(hz), hi2(mm), hi2(lx), hi2(ly), hi2(lz), nhxa, nhya, nhza,
             nlxa, nlya, nlza, a1e, a1f, pxa, pya, pza);
      if (kTwo) {
        term32(lo2(hx), lo2(hy), lo2(hz), lo2(mm), lo2(lx), lo2(ly), lo2(lz), nhxb, nhyb, nhzb,
               nlxb, nlyb, nlzb, false, b0, pxb, pyb, pzb);
        term32(hi2(hx), hi2(hy), hi2(hz), hi2(mm), hi2(lx), hi2(ly), hi2(lz), nhxb, nhyb, nhzb,
               nlxb, nlyb, nlzb, false, b1, pxb, pyb, pzb);
      }
    }
  }

  // Near chunks [q0, q1) (q1 - q0 even) in the split layout: target a takes
  // both chunks of a pair, target b the share of this lane's stream (kR = 2:
  // one chunk, kR = 4: one entry pair), read with its own loads.
  template <bool kSelf, int kR>
  __device__ __forceinline__ void near_split(int q0, int q1) {
    const float4* HX = reinterpret_cast<const float4*>(f);
    const float4* HY = reinterpret_cast<const float4*>(f + kL);
    const float4* HZ = reinterpret_cast<const float4*>(f + 2 * kL);
    const float4* MM = reinterpret_cast<const float4*>(f + 3 * kL);
    const float4* LX = reinterpret_cast<const float4*>(f + 4 * kL);
    const float4* LY = reinterpret_cast<const float4*>(f + 5 * kL);
    const float4* LZ = reinterpret_cast<const float4*>(f + 6 * kL);
    constexpr int kLps = 32 / kR;                      // lanes per stream
    const int st = lane / kLps, tb = 32 + lane % kLps;  // stream, b's slot
    const int pa = lane & 3;                            // a's slot: chunk lane/4
    for (int q = q0; q < q1; q += 2) {
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int qa = q + k;
        const float4 hx = HX[qa], hy = HY[qa], hz = HZ[qa], mm = MM[qa];
        const float4 lx = LX[qa], ly = LY[qa], lz = LZ[qa];
        const bool in = kSelf && qa == (lane >> 2);
        term32(lo2(hx), lo2(hy), lo2(hz), lo2(mm), lo2(lx), lo2(ly), lo2(lz), nhxa, nhya, nhza,
               nlxa, nlya, nlza, in && pa == 0, in && pa == 1, pxa, pya, pza);
        term32(hi2(hx), hi2(hy), hi2(hz), hi2(mm), hi2(lx), hi2(ly), hi2(lz), nhxa, nhya, nhza,
               nlxa, nlya, nlza, in && pa == 2, in && pa == 3, pxa, pya, pza);
      }
      if (kR == 2) {
        const int qb = q + st;
        const float4 hx = HX[qb], hy = HY[qb], hz = HZ[qb], mm = MM[qb];
        const float4 lx = LX[qb], ly = LY[qb], lz = LZ[qb];
        const bool in = kSelf && qb == (tb >> 2);
        const int pb = tb & 3;
        term32(lo2(hx), lo2(hy), lo2(hz), lo2(mm), lo2(lx), lo2(ly), lo2(lz), nhxb, nhyb, nhzb,
               nlxb, nlyb, nlzb, in && pb == 0, in && pb == 1, pxb, pyb, pzb);
        term32(hi2(hx), hi2(hy), hi2(hz), hi2(mm), hi2(lx), hi2(ly), hi2(lz), nhxb, nhyb, nhzb,
               nlxb, nlyb, nlzb, in && pb == 2, in && pb == 3, pxb, pyb, pzb);
      } else {
        const int e = 4 * q + 2 * st;  // the stream's entry pair (e, e + 1)
        const float2 hx = ld2(f + e), hy = ld2(f + kL + e), hz = ld2(f + 2 * kL + e);
        const float2 mm = ld2(f + 3 * kL + e);
        const float2 lx = ld2(f + 4 * kL + e), ly = ld2(f + 5 * kL + e),
                     lz = ld2(f + 6 * kL + e);
        term32(hx, hy, hz, mm, lx, ly, lz, nhxb, nhyb, nhzb, nlxb, nlyb, nlzb,
               kSelf && e == tb, kSelf && e + 1 == tb, pxb, pyb, pzb);
      }
    }
  }

  // Evaluates list slots [0, nl) for both targets (warp-collective).
  template <bool kSelf>
  __device__ __forceinline__ void eval(int nl) {
    if (kF32) {
      // pad to a multiple of 4 (split layout: 8) with massless entries far
      // away
      const int np = rb ? (nl + 7) & ~7 : (nl + 3) & ~3;
      if (lane < np - nl) {
        const int s = nl + lane;
        f[s] = f[kL + s] = f[2 * kL + s] = 1e15f;
        f[3 * kL + s] = f[4 * kL + s] = f[5 * kL + s] = f[6 * kL + s] = 0.f;
      }
      __syncwarp();
      const int nq = np >> 2;
      for (int q0 = 0; q0 < nq;) {
        const int q1 = min(q0 + (kFlushChunks - pend), nq);
        if (rb == 4)
          near_split<kSelf, 4>(q0, q1);
        else if (rb == 2)
          near_split<kSelf, 2>(q0, q1);
        else if (two)
          near_chunks<kSelf, true>(q0, q1);
        else
          near_chunks<kSelf, false>(q0, q1);
        chunks_done(q1 - q0);
        q0 = q1;
      }
    } else {
      __syncwarp();
#pragma unroll 2
      for (int e = 0; e < nl; ++e) {
        const double4 s = lst64[e];
        if (!(kSelf && e == (two ? 2 * lane : lane))) term64(s, ta, ax, ay, az);
        if (two && !(kSelf && e == 2 * lane + 1)) term64(s, tb, bx, by, bz);
      }
    }
    __syncwarp();
  }

  // One far F32C entry pair against one target: plain f32 offsets from X0.
  __device__ __forceinline__ void term32f(float2 hx, float2 hy, float2 hz, float2 mm,
                                          float2 nhx, float2 nhy, float2 nhz, float2& px,
                                          float2& py, float2& pz) {
    const float2 rx = __fadd2_rn(hx, nhx);
    const float2 ry = __fadd2_rn(hy, nhy);
    const float2 rz = __fadd2_rn(hz, nhz);
    const float2 r2 = __ffma2_rn(rx, rx, __ffma2_rn(ry, ry, __ffma2_rn(rz, rz, e2)));
    const float2 inv = make_float2(rsqrt_sfu(r2.x), rsqrt_sfu(r2.y));
    const float2 w = __fmul2_rn(mm, __fmul2_rn(__fmul2_rn(inv, inv), inv));
    px = __ffma2_rn(rx, w, px);
    py = __ffma2_rn(ry, w, py);
    pz = __ffma2_rn(rz, w, pz);
  }

  // Far chunks [q0, q1) against target a, and target b when kTwo.
  template <bool kTwo>
  __device__ __forceinline__ void far_chunks(int q0, int q1) {
    const float4* HX = reinterpret_cast<const float4*>(ff);
    const float4* HY = reinterpret_cast<const float4*>(ff + kL);
    const float4* HZ = reinterpret_cast<const float4*>(ff + 2 * kL);
    const float4* MM = reinterpret_cast<const float4*>(ff + 3 * kL);
#pragma unroll kEvalUnroll
    for (int q = q0; q < q1; ++q) {
      const float4 hx = HX[q], hy = HY[q], hz = HZ[q], mm = MM[q];
      term32f(lo2(hx), lo2(hy), lo2(hz), lo2(mm), nhxa, nhya, nhza, pxa, pya, pza);
      term32f(hi2(hx), hi2(hy), hi2(hz), hi2(mm), nhxa, nhya, nhza, pxa, pya, pza);
      if (kTwo) {
        term32f(lo2(hx), lo2(hy), lo2(hz), lo2(mm), nhxb, nhyb, nhzb, pxb, pyb, pzb);
        term32f(hi2(hx), hi2(hy), hi2(hz), hi2(mm), nhxb, nhyb, nhzb, pxb, pyb, pzb);
      }
    }
  }

  // Far chunks [q0, q1) (q1 - q0 even) in the split layout (as near_split).
  template <int kR>
  __device__ __forceinline__ void far_split(int q0, int q1) {
    const float4* HX = reinterpret_cast<const float4*>(ff);
    const float4* HY = reinterpret_cast<const float4*>(ff + kL);
    const float4* HZ = reinterpret_cast<const float4*>(ff + 2 * kL);
    const float4* MM = reinterpret_cast<const float4*>(ff + 3 * kL);
    constexpr int kLps = 32 / kR;
    const int st = lane / kLps;
    for (int q = q0; q < q1; q += 2) {
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const float4 hx = HX[q + k], hy = HY[q + k], hz = HZ[q + k], mm = MM[q + k];
        term32f(lo2(hx), lo2(hy), lo2(hz), lo2(mm), nhxa, nhya, nhza, pxa, pya, pza);
        term32f(hi2(hx), hi2(hy), hi2(hz), hi2(mm), nhxa, nhya, nhza, pxa, pya, pza);
      }
      if (kR == 2) {
        const int qb = q + st;
        const float4 hx = HX[qb], hy = HY[qb], hz = HZ[qb], mm = MM[qb];
        term32f(lo2(hx), lo2(hy), lo2(hz), lo2(mm), nhxb, nhyb, nhzb, pxb, pyb, pzb);
        term32f(hi2(hx), hi2(hy), hi2(hz), hi2(mm), nhxb, nhyb, nhzb, pxb, pyb, pzb);
      } else {
        const int e = 4 * q + 2 * st;
        term32f(ld2(ff + e), ld2(ff + kL + e), ld2(ff + 2 * kL + e), ld2(ff + 3 * kL + e), nhxb,
                nhyb, nhzb, pxb, pyb, pzb);
      }
    }
  }

  // Evaluates far-list slots [0, nl) for both targets (warp-collective).
  __device__ __forceinline__ void eval_far(int nl) {
    const int np = rb ? (nl + 7) & ~7 : (nl + 3) & ~3;
    if (lane < np - nl) {
      const int s = nl + lane;
      ff[s] = ff[kL + s] = ff[2 * kL + s] = 1e15f;
      ff[3 * kL + s] = 0.f;
    }
    __syncwarp();
    const int nq = np >> 2;
    for (int q0 = 0; q0 < nq;) {
      const int q1 = min(q0 + (kFlushChunks - pend), nq);
      if (rb == 4)
        far_split<4>(q0, q1);
      else if (rb == 2)
        far_split<2>(q0, q1);
      else if (two)
        far_chunks<true>(q0, q1);
      else
        far_chunks<false>(q0, q1);
      chunks_done(q1 - q0);
      q0 = q1;
    }
    __syncwarp();
  }

  // Streams list entries codes[0, len) through two staging buffers of kL
  // source records (stage: 2 * kL double4) and evaluates each batch
  // (warp-collective).  Lane l copies entries l, l + 32, ... of a batch with
  // cp.async and converts the same entries, so its own copies are all it
  // waits for; batch b + 2 is in flight while batch b is evaluated, and the
  // entry codes are read one batch further ahead.  F32C: an entry whose
  // distance from the group's box is at least GWALK_FAR box half-diagonals b
  // goes to the far list, whose plain f32 offsets from X0 need no low parts
  // (targets lie within 2b of X0, so the separation's error is below
  // 2^-24 (2|r| + 4b) <= 66 * 2^-24 |r| at a sixteenth of a half-diagonal,
  // about 4e-6 for the nearest far entries and far less for most: the
  // F32C-vs-F64 median stays at 5e-8); the rest go to the near list
  // (double-float).  F64: the staged records are the list.
  __device__ __forceinline__ void stream_eval(const uint32_t* __restrict__ codes, int len,
                                              const GNode* __restrict__ gn,
                                              const double4* __restrict__ body64, const Box& B,
                                              float far2, double4* stage) {
    constexpr int kPer = kL / 32;
    const int nb = (len + kL - 1) / kL;
    if (nb == 0) return;
    uint32_t pc[kPer];  // codes of the next batch to issue (~0u: none)
    auto load_codes = [&](int b) {
#pragma unroll
      for (int j = 0; j < kPer; ++j) {
        const int e = b * kL + lane + 32 * j;
        pc[j] = e < len ? __ldcg(codes + e) : ~0u;  // read once: L2 only
      }
    };
    auto issue = [&](int b) {
      double4* dst = stage + (b & 1) * kL;
#pragma unroll
      for (int j = 0; j < kPer; ++j) {
        if (pc[j] != ~0u) {
          const int id = (int)(pc[j] >> 1);
          const double4* src = (pc[j] & 1u) ? body64 + id : &gn[id].c64;
          double4* d = dst + lane + 32 * j;
          cp_async16(d, src);
          cp_async16(reinterpret_cast<char*>(d) + 16, reinterpret_cast<const char*>(src) + 16);
        }
      }
      cp_async_commit();
    };
    load_codes(0);
    issue(0);
    if (nb > 1) {
      load_codes(1);
      issue(1);
    }
    if (nb > 2) load_codes(2);
    const unsigned lt = (1u << lane) - 1u;
    for (int b = 0; b < nb; ++b) {
      if (b + 1 < nb)
        cp_async_wait<1>();
      else
        cp_async_wait<0>();
      double4* buf = stage + (b & 1) * kL;
      const int n_b = min(kL, len - b * kL);
      if (kF32) {
        int nnear = 0, nfar = 0;
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
          const int e = lane + 32 * j;
          const bool valid = e < n_b;
          const double4 src = valid ? buf[e] : X0;
          // offsets from X0; their low parts (as split_df) only for near entries
          const double ox = src.x - X0.x, oy = src.y - X0.y, oz = src.z - X0.z;
          const float hx = __double2float_rn(ox), hy = __double2float_rn(oy),
                      hz = __double2float_rn(oz);
          const float dx = fmaxf(fabsf(hx - B.cx) - B.bx, 0.f);
          const float dy = fmaxf(fabsf(hy - B.cy) - B.by, 0.f);
          const float dz = fmaxf(fabsf(hz - B.cz) - B.bz, 0.f);
          const bool far = valid && fmaf(dx, dx, fmaf(dy, dy, dz * dz)) >= far2;
          const unsigned fm = __ballot_sync(kFull, far);
          const unsigned nm = __ballot_sync(kFull, valid && !far);
          const float m = (float)src.w;
          if (far) {
            const int q = nfar + __popc(fm & lt);
            ff[q] = hx;
            ff[kL + q] = hy;
            ff[2 * kL + q] = hz;
            ff[3 * kL + q] = m;
          } else if (valid) {
            const int q = nnear + __popc(nm & lt);
            f[q] = hx;
            f[kL + q] = hy;
            f[2 * kL + q] = hz;
            f[3 * kL + q] = m;
            f[4 * kL + q] = __double2float_rn(ox - (double)hx);
            f[5 * kL + q] = __double2float_rn(oy - (double)hy);
            f[6 * kL + q] = __double2float_rn(oz - (double)hz);
          }
          nfar += __popc(fm);
          nnear += __popc(nm);
        }
        __syncwarp();  // this buffer is free: refill it with batch b + 2
        if (b + 2 < nb) {
          issue(b + 2);
          if (b + 3 < nb) load_codes(b + 3);
        }
        if (nnear) eval<false>(nnear);
        if (nfar) eval_far(nfar);
      } else {
        __syncwarp();  // every lane's copies visible
        double4* keep = lst64;
        lst64 = buf;
        eval<false>(n_b);
        lst64 = keep;
        if (b + 2 < nb) {
          issue(b + 2);
          if (b + 3 < nb) load_codes(b + 3);
        }
      }
    }
  }

  // Pairs inside the group, exact, i != j.
  __device__ __forceinline__ void self_pass() {
    if (rb) {
      if (va) put(lane, ta);
      if (vb && lane < 32 / rb) put(32 + lane, tb);
    } else {
      if (va) put(two ? 2 * lane : lane, ta);
      if (vb) put(2 * lane + 1, tb);
    }
    eval<true>(nvalid);
  }

  __device__ __forceinline__ void finish(const double4* __restrict__ body64,
                                         const uint32_t* __restrict__ perm, double G,
                                         int want_force, double* __restrict__ ox,
                                         double* __restrict__ oy, double* __restrict__ oz,
                                         int32_t* status) {
    auto out = [&](int pp, double fx, double fy, double fz) {
      const double sc = want_force ? G * body64[pp].w : G;
      fx *= sc;
      fy *= sc;
      fz *= sc;
      const uint32_t i = perm[pp];
      ox[i] = fx;
      oy[i] = fy;
      oz[i] = fz;
      if (!isfinite(fx) || !isfinite(fy) || !isfinite(fz)) atomicOr(status, kStatNonfinite);
    };
    if (kF32) {
      flush();  // the partials of the last chunks
      if (va) out(ia, (double)Hx.x + (double)Lx.x, (double)Hy.x + (double)Ly.x,
                  (double)Hz.x + (double)Lz.x);
      double bx_ = (double)Hx.y + (double)Lx.y, by_ = (double)Hy.y + (double)Ly.y,
             bz_ = (double)Hz.y + (double)Lz.y;
      if (rb) {  // add the streams' sums of the same b target
        for (int o = 32 / rb; o < 32; o <<= 1) {
          bx_ += __shfl_xor_sync(kFull, bx_, o);
          by_ += __shfl_xor_sync(kFull, by_, o);
          bz_ += __shfl_xor_sync(kFull, bz_, o);
        }
      }
      if (vb && (!rb || lane < 32 / rb)) out(ib, bx_, by_, bz_);
    } else {
      if (va) out(ia, ax, ay, az);
      if (vb) out(ib, bx, by, bz);
    }
  }
};

// Takes the next work index for the warp.
__device__ __forceinline__ int next_item(int lane, int32_t* ctr) {
  int gi = 0;
  if (lane == 0) gi = atomicAdd(ctr, 1);
  return __shfl_sync(kFull, gi, 0);
}

__device__ __forceinline__ bool bad_range(int2 gr, int n) {
  return gr.x < 0 || gr.y > n || gr.y - gr.x < 1 || gr.y - gr.x > kGroupMax;
}

// Re-queues [gr.x, gr.y) as subgroups of kGSplit bodies (lane 0).  The
// subgroups are disjoint and non-empty: at most n of them in all.
__device__ __forceinline__ bool requeue(int2 gr, int n, int2* retry, int32_t* nretry) {
  const int nsub = (gr.y - gr.x + kGSplit - 1) / kGSplit;
  const int at = atomicAdd(nretry, nsub);
  bool ok = true;
  for (int k = 0; k < nsub; ++k) {
    if (at + k < n) {
      retry[at + k] = make_int2(gr.x + k * kGSplit, min(gr.x + (k + 1) * kGSplit, gr.y));
    } else {
      ok = false;
    }
  }
  return ok;
}

// ---------------------------------------------------------------------------
// 1. lists.  Entry codes: cell record nd -> nd << 1; body q -> q << 1 | 1.
// Items: n int4 {first body, end body, 0, list length}, then n int64 pool
// offsets.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kLBlock, GLIST_MIN_BLOCKS)
glist_kernel(int n, int q0, int q1, int nnodes, const GNode* __restrict__ gn,
             const int2* __restrict__ groups,
             const int32_t* __restrict__ ngroups_p, int32_t* __restrict__ ctr,
             const double4* __restrict__ body64, float theta2f, uint32_t* __restrict__ pool,
             int64_t pool_per_warp, int64_t nspill, int32_t* __restrict__ spill_ctr,
             int4* __restrict__ items, int32_t* __restrict__ nitems, int2* __restrict__ retry,
             int32_t* __restrict__ nretry, int32_t* status) {
  if (sort_failed(status)) return;  // records built on an unfinished sort
  extern __shared__ __align__(16) unsigned char gsm[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int* stk = reinterpret_cast<int*>(gsm) + wid * kGStack;
  const int64_t warps = (int64_t)gridDim.x * kLWarps;
  int64_t region0 = (blockIdx.x * (int64_t)kLWarps + wid) * pool_per_warp;
  uint32_t* region = pool + region0;
  int cap = (int)min64(pool_per_warp, (int64_t)INT_MAX);
  int64_t* offs = reinterpret_cast<int64_t*>(items + n);
  const int ngroups = min(*ngroups_p, n);
  int roff = 0;  // used part of the region
  bool bad = false;
  for (;;) {
    const int gi = next_item(lane, ctr);
    if (gi >= ngroups) break;
    const int2 gr = groups[gi];
    if (bad_range(gr, n)) {
      bad = true;
      break;
    }
    const int base = gr.x, gend = gr.y;
    if (gend <= q0 || base >= q1) continue;  // no target of the share [q0, q1)
    if (cap - roff < kGRegionNeed) {
      // too little room left for a list of the largest length: continue in
      // a fresh spill region, so that whether a group is re-queued depends
      // on its list alone, not on which groups this warp took before
      int sreg = 0;
      if (lane == 0) sreg = atomicAdd(spill_ctr, 1);
      sreg = __shfl_sync(kFull, sreg, 0);
      if (sreg < nspill) {
        region0 = warps * pool_per_warp + sreg * (int64_t)kGRegionNeed;
        region = pool + region0;
        cap = kGRegionNeed;
        roff = 0;
      }
    }
    const double4 X0 = body64[base];
    const int ia = base + 2 * lane, ib = ia + 1;
    const double4 ta = ia < gend ? body64[ia] : X0;
    const double4 tb = ib < gend ? body64[ib] : X0;
    const Box B = group_box(X0, ta, tb);
    int used = 0;
    auto sink = [&](int etot, int eoff, const NodeOut& o) -> bool {
      // full (spill regions exhausted, or a guard leaf of very many bodies):
      // re-queue
      if (roff + used + etot > cap) return false;
      uint32_t* dst = region + roff + used + eoff;
      if (o.kind == 1) {
        dst[0] = (uint32_t)o.a << 1;
      } else {
        for (int j = 0; j < o.nent; ++j)
          dst[j] = ((uint32_t)bucket_body(o.a, o.olo, o.ohi, j) << 1) | 1u;
      }
      used += etot;
      return true;
    };
    const int r = traverse<false>(lane, base, gend, nnodes, kGListLimit, stk, B, theta2f, gn,
                                  sink);
    if (r < 0) {
      bad = true;
      break;
    }
    if (lane == 0) {
      if (r == 1) {
        const int it = atomicAdd(nitems, 1);
        if (it < n) {
          items[it] = make_int4(base, gend, 0, used);
          offs[it] = region0 + roff;
        } else {
          bad = true;
        }
      } else if (!requeue(gr, n, retry, nretry)) {
        bad = true;
      }
    }
    if (r == 1) roff += used;
    __syncwarp();
  }
  if (bad && lane == 0) atomicOr(status, kStatOverflow);
}

// ---------------------------------------------------------------------------
// 2. evaluation of the lists
// ---------------------------------------------------------------------------
template <bool kF32>
__global__ void __launch_bounds__(kGBlock, GEVAL_MIN_BLOCKS)
geval_kernel(int n, const GNode* __restrict__ gn, const int4* __restrict__ items,
             const int32_t* __restrict__ nitems_p, int32_t* __restrict__ ctr,
             const uint32_t* __restrict__ pool, const double4* __restrict__ body64,
             const uint32_t* __restrict__ perm, double G, double eps2, int want_force,
             double* __restrict__ ox, double* __restrict__ oy, double* __restrict__ oz,
             unsigned long long* counter, int32_t* status) {
  if (sort_failed(status)) return;  // records built on an unfinished sort
  extern __shared__ __align__(16) unsigned char gsm[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned char* lbase = gsm + wid * kESmemWarp;
  const int nitems = min(*nitems_p, n);
  const int64_t* offs = reinterpret_cast<const int64_t*>(items + n);
  unsigned long long ninter = 0;
  for (;;) {
    const int it = next_item(lane, ctr);
    if (it >= nitems) break;
    const int4 item = items[it];
    const uint32_t* codes = pool + offs[it];
    const int len = item.w;
    Evaluator<kF32, kEB> E;
    E.init(lane, item.x, item.y, body64, lbase, eps2);
    const Box B = group_box(E.X0, E.ta, E.tb);
    const float far2 = (float)(GWALK_FAR * GWALK_FAR) * fmaf(B.bx, B.bx, fmaf(B.by, B.by, B.bz * B.bz));
    E.self_pass();
    ninter += (unsigned long long)E.nvalid * (unsigned long long)(E.nvalid - 1 + len);
    E.stream_eval(codes, len, gn, body64, B, far2,
                  reinterpret_cast<double4*>(lbase + kEListBytes));
    E.finish(body64, perm, G, want_force, ox, oy, oz, status);
  }
  if (lane == 0 && ninter) {  // the same on every lane
    atomicAdd(counter, ninter);
    atomicAdd(counter + 1, ninter);
  }
}

// ---------------------------------------------------------------------------
// 3. walk + evaluation in one pass (re-queued subgroups)
// ---------------------------------------------------------------------------
template <bool kF32>
__global__ void __launch_bounds__(kGBlock, 4)
gwalk_kernel(int n, int nnodes, const GNode* __restrict__ gn, const int2* __restrict__ groups,
             const int32_t* __restrict__ ngroups_p, int32_t* __restrict__ ctr,
             const double4* __restrict__ body64, const uint32_t* __restrict__ perm, double G,
             double eps2, float theta2f, int want_force, double* __restrict__ ox,
             double* __restrict__ oy, double* __restrict__ oz, unsigned long long* counter,
             int32_t* status) {
  if (sort_failed(status)) return;  // records built on an unfinished sort
  extern __shared__ __align__(16) unsigned char gsm[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned char* ws = gsm + wid * kGSmemWarp;
  int* stk = reinterpret_cast<int*>(ws);
  int* rec = reinterpret_cast<int*>(ws + kGRecOff);
  int* r_end = rec;
  int* r_kind = rec + 32;
  int* r_a = rec + 64;
  int* r_olo = rec + 96;
  int* r_ohi = rec + 128;
  double4* r_src = reinterpret_cast<double4*>(rec + 160);
  const int ngroups = min(*ngroups_p, n);
  unsigned long long ninter = 0;
  bool bad = false;
  for (;;) {
    const int gi = next_item(lane, ctr);
    if (gi >= ngroups) break;
    const int2 gr = groups[gi];
    if (bad_range(gr, n)) {
      bad = true;
      break;
    }
    Evaluator<kF32, kGList> E;
    E.init(lane, gr.x, gr.y, body64, ws + kGListOff, eps2);
    const Box B = group_box(E.X0, E.ta, E.tb);
    E.self_pass();
    const unsigned long long nv = (unsigned long long)E.nvalid;
    unsigned long long ni = nv * (nv - 1);
    int lsize = 0;
    auto sink = [&](int etot, int eoff, const NodeOut& o) -> bool {
      if (lsize + etot > kGList && lsize > 0) {
        E.template eval<false>(lsize);
        ni += (unsigned long long)lsize * nv;
        lsize = 0;
      }
      if (etot <= kGList) {
        // every lane writes its own entries at its scan offset
        const int s0 = lsize + eoff;
        if (o.kind == 1) {
          E.put(s0, o.c64);
        } else {
          for (int j = 0; j < o.nent; ++j)
            E.put(s0 + j, ldg_d4(&body64[bucket_body(o.a, o.olo, o.ohi, j)]));
        }
        lsize += etot;
        return true;
      }
      // more entries than the list holds (a leaf of many bodies at the guard
      // depth): windows of kGList entries spread over the lanes
      r_end[lane] = eoff + o.nent;
      r_kind[lane] = o.kind;
      r_src[lane] = o.c64;
      r_a[lane] = o.a;
      r_olo[lane] = o.olo;
      r_ohi[lane] = o.ohi;
      __syncwarp();
      for (int done = 0; done < etot;) {
        if (lsize == kGList) {
          E.template eval<false>(lsize);
          ni += (unsigned long long)lsize * nv;
          lsize = 0;
        }
        const int take = min(etot - done, kGList - lsize);
        for (int e = done + lane; e < done + take; e += 32) {
          // owner: the first lane whose inclusive end exceeds e
          int lo = 0, hi = 31;
          while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (r_end[mid] > e) hi = mid;
            else lo = mid + 1;
          }
          const int j = e - (lo ? r_end[lo - 1] : 0);
          const double4 src = r_kind[lo] == 1
                                  ? r_src[lo]
                                  : ldg_d4(&body64[bucket_body(r_a[lo], r_olo[lo], r_ohi[lo], j)]);
          E.put(lsize + (e - done), src);
        }
        lsize += take;
        done += take;
      }
      __syncwarp();
      return true;
    };
    const int r = traverse<true>(lane, gr.x, gr.y, nnodes, INT_MAX, stk, B, theta2f, gn, sink);
    if (r != 1) {
      bad = true;
      break;
    }
    if (lsize > 0) {
      E.template eval<false>(lsize);
      ni += (unsigned long long)lsize * nv;
    }
    ninter += ni;
    E.finish(body64, perm, G, want_force, ox, oy, oz, status);
  }
  if (lane == 0) {
    if (bad) atomicOr(status, kStatOverflow);
    if (ninter) atomicAdd(counter, ninter);  // the same on every lane
  }
}

// Resident blocks per SM of a kernel with its dynamic shared memory, and its
// shared-memory limit raised on the context's device (cached in the context:
// the kernel's resources are fixed).
template <class K>
int occupancy(phys_ctx* c, K kernel, int block, int smem, int* cache) {
  if (!*cache) {
    PHYS_CUDA(c, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int b = 0;
    PHYS_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, block, smem));
    *cache = b > 0 ? b : 1;
  }
  return PHYS_OK;
}

template <bool kF32>
int launch(phys_ctx* c, const phys_params* p, const BhTree& t, bool want_force, double* ox,
           double* oy, double* oz) {
  int& occ_list = c->occ_gwalk[0];
  int& occ_eval = c->occ_gwalk[kF32 ? 2 : 1];
  int& occ_fused = c->occ_gwalk[kF32 ? 4 : 3];
  PHYS_TRY(occupancy(c, glist_kernel, kLBlock, kLSmem, &occ_list));
  PHYS_TRY(occupancy(c, geval_kernel<kF32>, kGBlock, kESmem, &occ_eval));
  PHYS_TRY(occupancy(c, gwalk_kernel<kF32>, kGBlock, kGSmem, &occ_fused));
  int sms = 0;
  PHYS_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  const int64_t n = t.n;
  const int grid_list = (int)min64((int64_t)sms * occ_list, ceil_div(n, (int64_t)kLWarps));
  const int grid_eval = (int)min64((int64_t)sms * occ_eval, ceil_div(n, (int64_t)kGWarps));
  const int grid_fused = (int)min64((int64_t)sms * occ_fused, ceil_div(n, (int64_t)kGWarps));
  // list pool: one region per list warp, each at least one full list
  const int64_t warps = (int64_t)grid_list * kLWarps;
  const int64_t pool_per_warp = std::max((int64_t)kGRegionNeed,
                                         ceil_div(n * (int64_t)GWALK_POOL_PER_BODY, warps));
  const int64_t nspill = warps;  // spill regions of kGRegionNeed codes, one per warp
  uint32_t* pool = nullptr;
  int4* items = nullptr;  // n int4 items, then n int64 pool offsets
  PHYS_TRY(ws_alloc(c, WS_GROUP_POOL, warps * pool_per_warp + nspill * kGRegionNeed, &pool));
  PHYS_TRY(ws_alloc(c, WS_GROUP_ITEMS, 2 * n, &items));
  // group_ctr: [0] list counter, [1] re-queued count, [2] items, [3]
  // evaluation counter, [4] second-walk counter, [5] spill regions taken
  int32_t* ctr = t.group_ctr;
  PHYS_CUDA(c, cudaMemsetAsync(ctr, 0, 6 * sizeof(int32_t), c->stream));
  const double eps2 = p->eps * p->eps;
  const float theta2f = (float)(p->theta * p->theta);
  int2* retry = const_cast<int2*>(t.groups) + n;
  // a share evaluates the groups that hold any of its targets (sorted
  // positions [q0, q1)); their other bodies get the same values as on the
  // rank that owns them
  int64_t q0 = 0, q1 = n;
  target_range(c, n, q0, q1);
  PHYS_LAUNCH(c, glist_kernel, grid_list, kLBlock, kLSmem, (int)n, (int)q0, (int)q1,
              (int)t.nnodes, t.gnode,
              t.groups, t.ngroups, ctr, t.body64, theta2f, pool, pool_per_warp, nspill, ctr + 5,
              items, ctr + 2,
              retry, ctr + 1, c->d_status);
  // The re-queued subgroups (a few hundred serial, latency-bound walks at
  // most) run on the side stream beside the list evaluation; it is launched
  // first so that its warps holding work are resident from the start.  Both
  // kernels write disjoint bodies and add to the counters atomically; the
  // main stream joins the side stream before anything reads the results.
  PHYS_CUDA(c, cudaEventRecord(c->fork, c->stream));
  PHYS_CUDA(c, cudaStreamWaitEvent(c->side, c->fork, 0));
  PHYS_LAUNCH_ON(c, c->side, gwalk_kernel<kF32>, grid_fused, kGBlock, kGSmem, (int)n,
                 (int)t.nnodes, t.gnode, retry, ctr + 1, ctr + 4, t.body64, t.perm, p->G, eps2,
                 theta2f, (int)want_force, ox, oy, oz, c->d_counter, c->d_status);
  PHYS_CUDA(c, cudaEventRecord(c->join, c->side));
  PHYS_CUDA(c, cudaEventRecord(c->ev[10], c->stream));
  PHYS_LAUNCH(c, geval_kernel<kF32>, grid_eval, kGBlock, kESmem, (int)n, t.gnode, items, ctr + 2,
              ctr + 3, pool, t.body64, t.perm, p->G, eps2, (int)want_force, ox, oy, oz,
              c->d_counter, c->d_status);  // adds to counter[0] and counter[1]
  PHYS_CUDA(c, cudaEventRecord(c->ev[11], c->stream));
  PHYS_CUDA(c, cudaStreamWaitEvent(c->stream, c->join, 0));
  return PHYS_OK;
}

}  // namespace

int bh_group_walk(phys_ctx* c, const phys_params* p, const BhTree& t, bool want_force,
                  double* ox, double* oy, double* oz) {
  if (!t.gnode || !t.groups) return fail(c, PHYS_ERR_STATE, "group walk without group records");
  if (t.n > INT32_MAX / 2 - kGroupMax || t.nnodes > INT32_MAX / 2)
    return fail(c, PHYS_ERR_ARG, "group walk: %lld bodies is too many", (long long)t.n);
  return p->precision == PHYS_F32C ? launch<true>(c, p, t, want_force, ox, oy, oz)
                                   : launch<false>(c, p, t, want_force, ox, oy, oz);
}

}  // namespace phys
