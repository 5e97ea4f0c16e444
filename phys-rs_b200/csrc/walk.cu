// K6: theta-criterion walk (OctreeNode::compute_force, gravity_tree.rs:171-209).
//
// Warp-coherent, stackless union traversal over the pre-order node array.
// A warp owns 32 consecutive key-sorted targets (spatially close) and visits
// nodes in pre-order; each lane applies the reference's own criterion
// (s*s < theta*theta*d2 -> monopole at the centre of mass) and the warp
// descends into a node's children when any lane opened it (__any_sync),
// otherwise it jumps over the subtree with the skip pointer.  A lane is
// active at a node only if it opened every ancestor (tracked by `open_to`,
// the number of consecutive opened levels on the current path), so no lane
// ever double-counts a cell.  All lanes read the same node: every node load
// is one broadcast transaction.
//
// Variants:
//   F64_EXACT  reference arithmetic (no FMA, IEEE sqrt/div) and the
//              reference's nested summation: the force of an opened cell is
//              0 + sum of its children in octant order, added into the parent
//              as one term.  Per-lane accumulators per depth live in local
//              memory; closing a level adds it into the level above.
//   F64        flat f64 sum of m_j r / s^3, FMA + rsqrt.
//   F32C       f32 pair terms on double-float relative coordinates
//              r = (hi_j - hi_i) + (lo_j - lo_i); f32 partial sums folded
//              into a (hi, lo) accumulator with two-sum every 16 nodes.
#include "bh.cuh"

#ifndef WALK_BRANCHY
#define WALK_BRANCHY 0
#endif
#ifndef WALK_PAIRED
#define WALK_PAIRED 1
#endif
#ifndef WALK_UNROLL
#define WALK_UNROLL 0
#endif

namespace phys {
namespace {

constexpr int kWalkBlock = 128;

__device__ __forceinline__ void warp_count(unsigned ninter, unsigned long long* counter) {
  unsigned long long v = ninter;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(counter, v);
}

template <bool kF32>
__global__ void __launch_bounds__(kWalkBlock)
walk_kernel(int q0, int n, int nnodes, const Rec32* __restrict__ w32, const Rec64* __restrict__ w64,
            const double4* __restrict__ body64, const float4* __restrict__ body_hi,
            const float4* __restrict__ body_lo, const uint32_t* __restrict__ perm,
            const TreeHeader* __restrict__ hdr, double G, double eps2, int want_force,
            double* __restrict__ ox, double* __restrict__ oy, double* __restrict__ oz,
            unsigned long long* counter, int32_t* status) {
  __shared__ double s2d[kWDepth + 1];
  if (!kF32) {
    for (int d = threadIdx.x; d <= kWDepth; d += blockDim.x)
      s2d[d] = d < kMaxLevels ? hdr->s2[d] : 0.0;
    __syncthreads();
  }
  const double theta2 = hdr->theta2;
  const float eps2f = (float)eps2;
  const int p = q0 + blockIdx.x * kWalkBlock + threadIdx.x;  // targets [q0, n)
  const bool valid = p < n;

  double tx = 0, ty = 0, tz = 0;
  float thx = 0, thy = 0, thz = 0, tlx = 0, tly = 0, tlz = 0;
  if (valid) {
    if (kF32) {
      const float4 h = body_hi[p], l = body_lo[p];
      thx = h.x; thy = h.y; thz = h.z;
      tlx = l.x; tly = l.y; tlz = l.z;
    } else {
      const double4 b = body64[p];
      tx = b.x; ty = b.y; tz = b.z;
    }
  }
  double ax = 0, ay = 0, az = 0;            // F64 sums
  float hx = 0, hy = 0, hz = 0;             // F32C compensated sums (hi)
  float lx = 0, ly = 0, lz = 0;             //                      (lo)
  float px = 0, py = 0, pz = 0;             // F32C partial since last flush
  unsigned ninter = 0;
  // open_to = number of consecutive opened levels on the current path; a
  // lane is active at a node of depth d iff open_to == d.  Lanes past the end
  // start at -1 and are never active.
  int open_to = valid ? 0 : -1;
  int node = 0;

  auto flush = [&]() {
    float s, e;
    two_sum(hx, px, s, e);
    hx = s;
    lx += e;
    two_sum(hy, py, s, e);
    hy = s;
    ly += e;
    two_sum(hz, pz, s, e);
    hz = s;
    lz += e;
    px = py = pz = 0.f;
  };

  // Visit body.  Returns the next node; always > node, so the loop ends
  // even on a malformed tree.
  auto visit = [&](int nd) -> int {
    int4 L;
    float4 A, B;
    double4 A64;
    if (kF32) {
      const Rec32* rp = w32 + nd;
      A = rp->a;
      B = rp->b;
      L = rp->l;
    } else {
      const Rec64* rp = w64 + nd;
      A64 = rp->a;
      L = rp->l;
    }
    const int d = L.w & kWDepth;
    open_to = min(open_to, d);
    const bool act = open_to == d;
    bool acc;
    if (kF32) {
      const float rx = (A.x - thx) + (B.x - tlx);
      const float ry = (A.y - thy) + (B.y - tly);
      const float rz = (A.z - thz) + (B.z - tlz);
      const float d2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
      acc = d2 > B.w;  // one-body leaves carry -1: always an exact pair
      const bool use = act && acc && L.y != p;
#if WALK_BRANCHY
      if (use) {
        const float inv = rsqrt_sfu(d2 + eps2f);
        const float w = A.w * (inv * inv * inv);
        px = fmaf(rx, w, px);
        py = fmaf(ry, w, py);
        pz = fmaf(rz, w, pz);
      }
#else
      const float inv = rsqrt_sfu(d2 + eps2f);
      const float w = use ? A.w * (inv * inv * inv) : 0.f;
      px = fmaf(rx, w, px);
      py = fmaf(ry, w, py);
      pz = fmaf(rz, w, pz);
#endif
      ninter += use;
    } else {
      const double rx = A64.x - tx, ry = A64.y - ty, rz = A64.z - tz;
      const double d2 = fma(rx, rx, fma(ry, ry, rz * rz));
      acc = L.y >= 0 || s2d[d] < theta2 * d2;  // gravity_tree.rs:194
      const bool use = act && acc && L.y != p;
      if (use) {
        const double inv = rsqrt(d2 + eps2);
        const double w = A64.w * (inv * inv * inv);
        ax = fma(rx, w, ax);
        ay = fma(ry, w, ay);
        az = fma(rz, w, az);
      }
      ninter += use;
    }
    const bool open = act && !acc;
    int nxt = L.x;
    if (__any_sync(0xffffffffu, open)) {
      if (L.w & kWLeaf) {
        // Bucket leaf opened: exact pairs with its bodies (skipping self).
        const int q1 = L.z + (L.w >> 8);
        for (int q = L.z; q < q1; ++q) {
          const bool use = open && q != p;
          if (kF32) {
            const float4 h = body_hi[q], l = body_lo[q];
            const float rx = (h.x - thx) + (l.x - tlx);
            const float ry = (h.y - thy) + (l.y - tly);
            const float rz = (h.z - thz) + (l.z - tlz);
            const float inv = rsqrt_sfu(fmaf(rx, rx, fmaf(ry, ry, fmaf(rz, rz, eps2f))));
            const float w = use ? h.w * (inv * inv * inv) : 0.f;
            px = fmaf(rx, w, px);
            py = fmaf(ry, w, py);
            pz = fmaf(rz, w, pz);
          } else {
            const double4 b = body64[q];
            if (use) {
              const double rx = b.x - tx, ry = b.y - ty, rz = b.z - tz;
              const double inv = rsqrt(fma(rx, rx, fma(ry, ry, fma(rz, rz, eps2))));
              const double w = b.w * (inv * inv * inv);
              ax = fma(rx, w, ax);
              ay = fma(ry, w, ay);
              az = fma(rz, w, az);
            }
          }
          ninter += use;
        }
      } else {
        if (open) open_to = d + 1;
        nxt = nd + 1;
      }
    }
    return max(nxt, nd + 1);
  };

  // Sixteen visits per flush of the f32 partial sums into the compensated
  // accumulator.
#if WALK_UNROLL
  while (node < nnodes) {
#pragma unroll
    for (int k = 0; k < WALK_UNROLL; ++k) {
      if (node >= nnodes) break;
      node = visit(node);
    }
    if (kF32) flush();
  }
#else
  unsigned iter = 0;
  while (node < nnodes) {
    node = visit(node);
    if (kF32 && ((++iter & 15u) == 0u)) flush();
  }
#endif
  warp_count(ninter, counter);
  if (!valid) return;
  double fx, fy, fz;
  if (kF32) {
    flush();
    fx = (double)hx + (double)lx;
    fy = (double)hy + (double)ly;
    fz = (double)hz + (double)lz;
  } else {
    fx = ax;
    fy = ay;
    fz = az;
  }
  const double sc = want_force ? G * body64[p].w : G;
  fx *= sc;
  fy *= sc;
  fz *= sc;
  const uint32_t i = perm[p];
  ox[i] = fx;
  oy[i] = fy;
  oz[i] = fz;
  if (!isfinite(fx) || !isfinite(fy) || !isfinite(fz)) atomicOr(status, kStatNonfinite);
}

// ---------------------------------------------------------------------------
// F32C walk, two key-adjacent targets per lane (64 per warp).  The per-target
// arithmetic runs on packed f32x2 instructions (one instruction for both
// targets), which halves the issue slots of the floating-point work; node
// and body records are stored pre-duplicated (x, x, y, y, ...) so the packed
// operands come straight from the 16-byte loads.  Decisions stay per target.
// ---------------------------------------------------------------------------
constexpr int kWalk2Block = 128;

__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

__global__ void __launch_bounds__(kWalk2Block)
walk2_kernel(int q64, int n, int nnodes, const Rec32x2* __restrict__ w, const Body32x2* __restrict__ body2,
             const double4* __restrict__ body64, const uint32_t* __restrict__ perm, double G,
             double eps2, int want_force, double* __restrict__ ox, double* __restrict__ oy,
             double* __restrict__ oz, unsigned long long* counter, int32_t* status) {
  const int lane = threadIdx.x & 31;
  // targets [64 q64, n), 64 per warp (a multiple of 64: pa even)
  const int base = (q64 + blockIdx.x * (kWalk2Block / 32) + (threadIdx.x >> 5)) * 64;
  const int pa = base + 2 * lane, pb = pa + 1;
  const bool va = pa < n, vb = pb < n;
  float2 nhx, nhy, nhz, nlx, nly, nlz;  // negated target coordinates (a, b)
  {
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 a0 = va ? body2[pa].q0 : z4, a1 = va ? body2[pa].q1 : z4;
    const float4 a2 = va ? body2[pa].q2 : z4, a3 = va ? body2[pa].q3 : z4;
    const float4 b0 = vb ? body2[pb].q0 : z4, b1 = vb ? body2[pb].q1 : z4;
    const float4 b2 = vb ? body2[pb].q2 : z4, b3 = vb ? body2[pb].q3 : z4;
    nhx = make_float2(-a0.x, -b0.x);
    nhy = make_float2(-a0.z, -b0.z);
    nhz = make_float2(-a1.x, -b1.x);
    nlx = make_float2(-a2.x, -b2.x);
    nly = make_float2(-a2.z, -b2.z);
    nlz = make_float2(-a3.x, -b3.x);
  }
  const float eps2f = (float)eps2;
  const float2 e2 = make_float2(eps2f, eps2f);
  float2 px = make_float2(0.f, 0.f), py = px, pz = px;  // partial sums since last flush
  float hxa = 0, hya = 0, hza = 0, lxa = 0, lya = 0, lza = 0;  // compensated, target a
  float hxb = 0, hyb = 0, hzb = 0, lxb = 0, lyb = 0, lzb = 0;  // compensated, target b
  int oa = va ? 0 : -1, ob = vb ? 0 : -1;  // opened levels on the current path
  unsigned ninter = 0;

  auto flush = [&]() {
    float s, e;
    two_sum(hxa, px.x, s, e); hxa = s; lxa += e;
    two_sum(hya, py.x, s, e); hya = s; lya += e;
    two_sum(hza, pz.x, s, e); hza = s; lza += e;
    two_sum(hxb, px.y, s, e); hxb = s; lxb += e;
    two_sum(hyb, py.y, s, e); hyb = s; lyb += e;
    two_sum(hzb, pz.y, s, e); hzb = s; lzb += e;
    px = py = pz = make_float2(0.f, 0.f);
  };
  // Packed separation from a paired record (q0..q3) to both targets.
  auto sep = [&](float4 q0, float4 q1, float4 q2, float4 q3, float2& rx, float2& ry,
                 float2& rz) {
    rx = __fadd2_rn(__fadd2_rn(lo2(q0), nhx), __fadd2_rn(lo2(q2), nlx));
    ry = __fadd2_rn(__fadd2_rn(hi2(q0), nhy), __fadd2_rn(hi2(q2), nly));
    rz = __fadd2_rn(__fadd2_rn(lo2(q1), nhz), __fadd2_rn(lo2(q3), nlz));
  };
  auto accum = [&](float2 rx, float2 ry, float2 rz, float2 r2, float2 m2, bool ua, bool ub) {
    const float2 inv = make_float2(rsqrt_sfu(r2.x), rsqrt_sfu(r2.y));
    float2 wg = __fmul2_rn(m2, __fmul2_rn(__fmul2_rn(inv, inv), inv));
    wg.x = ua ? wg.x : 0.f;
    wg.y = ub ? wg.y : 0.f;
    px = __ffma2_rn(rx, wg, px);
    py = __ffma2_rn(ry, wg, py);
    pz = __ffma2_rn(rz, wg, pz);
    ninter += (unsigned)ua + (unsigned)ub;
  };

  auto visit = [&](int nd) -> int {
    const Rec32x2* rp = w + nd;
    const float4 q0 = rp->q0, q1 = rp->q1, q2 = rp->q2, q3 = rp->q3;
    const int4 L = rp->l;
    const int d = L.w & kWDepth;
    oa = min(oa, d);
    ob = min(ob, d);
    const bool acta = oa == d, actb = ob == d;
    float2 rx, ry, rz;
    sep(q0, q1, q2, q3, rx, ry, rz);
    const float2 d2 = __ffma2_rn(rx, rx, __ffma2_rn(ry, ry, __fmul2_rn(rz, rz)));
    const bool acca = d2.x > q3.z, accb = d2.y > q3.w;  // -1 for one-body leaves
    accum(rx, ry, rz, __fadd2_rn(d2, e2), hi2(q1), acta && acca && L.y != pa,
          actb && accb && L.y != pb);
    const bool opa = acta && !acca, opb = actb && !accb;
    int nxt = L.x;
    if (__any_sync(0xffffffffu, opa || opb)) {
      if (L.w & kWLeaf) {
        const int qe = L.z + (L.w >> 8);
        for (int q = L.z; q < qe; ++q) {
          const Body32x2* bp = body2 + q;
          const float4 b0 = bp->q0, b1 = bp->q1, b2 = bp->q2, b3 = bp->q3;
          float2 bx, by, bz;
          sep(b0, b1, b2, b3, bx, by, bz);
          const float2 r2 = __ffma2_rn(bx, bx, __ffma2_rn(by, by, __ffma2_rn(bz, bz, e2)));
          accum(bx, by, bz, r2, hi2(b1), opa && q != pa, opb && q != pb);
        }
      } else {
        if (opa) oa = d + 1;
        if (opb) ob = d + 1;
        nxt = nd + 1;
      }
    }
    return max(nxt, nd + 1);
  };

  int node = 0;
  unsigned iter = 0;
  while (node < nnodes) {
    node = visit(node);
    if ((++iter & 15u) == 0u) flush();
  }
  flush();
  warp_count(ninter, counter);
  auto out = [&](int pp, float hx, float hy, float hz, float lx, float ly, float lz) {
    double fx = (double)hx + (double)lx, fy = (double)hy + (double)ly,
           fz = (double)hz + (double)lz;
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
  if (va) out(pa, hxa, hya, hza, lxa, lya, lza);
  if (vb) out(pb, hxb, hyb, hzb, lxb, lyb, lzb);
}

// ---------------------------------------------------------------------------
// F64_EXACT walk (leaf capacity 1).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kWalkBlock)
walk_exact_kernel(int64_t q0, int64_t n, int64_t nnodes, const int4* __restrict__ link,
                  const double4* __restrict__ rec64, const double4* __restrict__ body64,
                  const uint32_t* __restrict__ perm, const TreeHeader* __restrict__ hdr, double G,
                  double eps2, int want_force, double* __restrict__ ox, double* __restrict__ oy,
                  double* __restrict__ oz, unsigned long long* counter, int32_t* status) {
  __shared__ double s2d[kMaxLevels];
  for (int d = threadIdx.x; d < kMaxLevels; d += blockDim.x) s2d[d] = hdr->s2[d];
  __syncthreads();
  const double theta2 = hdr->theta2;
  const int64_t p = q0 + blockIdx.x * (int64_t)kWalkBlock + threadIdx.x;  // targets [q0, n)
  const bool valid = p < n;
  double tx = 0, ty = 0, tz = 0, mi = 0;
  if (valid) {
    const double4 b = body64[p];
    tx = b.x;
    ty = b.y;
    tz = b.z;
    mi = b.w;
  }
  const double gm = xmul(G, mi);
  // acc[d] collects the terms of the nodes at depth d (children of the lane's
  // opened node at depth d-1); acc[0] is the root's own term.
  double acc[kMaxLevels + 1][3];
  acc[0][0] = acc[0][1] = acc[0][2] = 0.0;
  unsigned ninter = 0;
  int open_to = 0;
  int32_t node = 0;

  // compute_gravity_pair (gravity_tree.rs:218-234)
  auto pair = [&](double4 s, int slot) {
    const double rx = xsub(s.x, tx), ry = xsub(s.y, ty), rz = xsub(s.z, tz);
    const double r2 = xlen2(rx, ry, rz);
    const double s2 = xadd(r2, eps2);
    const double s3 = xmul(s2, xsqrt(s2));
    const double sc = xdiv(xmul(gm, s.w), s3);
    acc[slot][0] = xadd(acc[slot][0], xmul(rx, sc));
    acc[slot][1] = xadd(acc[slot][1], xmul(ry, sc));
    acc[slot][2] = xadd(acc[slot][2], xmul(rz, sc));
  };
  auto close_to = [&](int d) {  // finish the lane's opened cells at depths >= d
    for (int k = open_to; k > d; --k) {
      acc[k - 1][0] = xadd(acc[k - 1][0], acc[k][0]);
      acc[k - 1][1] = xadd(acc[k - 1][1], acc[k][1]);
      acc[k - 1][2] = xadd(acc[k - 1][2], acc[k][2]);
    }
    if (open_to > d) open_to = d;
  };

  while (node < nnodes) {
    const int4 lk = link[node];
    if (lk.x <= node || lk.x > nnodes) {  // malformed tree: report, never spin
      if ((threadIdx.x & 31) == 0) atomicOr(status, kStatOverflow);
      break;
    }
    const int d = lk.w & kMetaDepth;
    close_to(d);
    const bool act = valid && open_to == d && ((lk.w & kMetaGate) || node == 0);
    if (lk.w & kMetaLeaf) {
      const int sp = (lk.z - lk.y) == 1 ? lk.y : lk.z - 1;
      if (act && sp != p) {
        pair(rec64[node], d);
        ++ninter;
      }
      node = lk.x;
    } else {
      const double4 s = rec64[node];
      const double rx = xsub(s.x, tx), ry = xsub(s.y, ty), rz = xsub(s.z, tz);
      const double d2 = xlen2(rx, ry, rz);
      const bool open = act && !(s2d[d] < xmul(theta2, d2));
      if (act && !open) {
        pair(s, d);
        ++ninter;
      }
      if (open) {
        acc[d + 1][0] = acc[d + 1][1] = acc[d + 1][2] = 0.0;
        open_to = d + 1;
      }
      node = __any_sync(0xffffffffu, open) ? node + 1 : lk.x;
    }
  }
  close_to(0);
  warp_count(ninter, counter);
  if (!valid) return;
  double fx = acc[0][0], fy = acc[0][1], fz = acc[0][2];
  if (!want_force) {  // a = F / m (integrators.rs:115)
    fx = xdiv(fx, mi);
    fy = xdiv(fy, mi);
    fz = xdiv(fz, mi);
  }
  const uint32_t i = perm[p];
  ox[i] = fx;
  oy[i] = fy;
  oz[i] = fz;
  if (!isfinite(fx) || !isfinite(fy) || !isfinite(fz)) atomicOr(status, kStatNonfinite);
}

}  // namespace

int bh_walk(phys_ctx* c, const phys_params* p, const BhTree& t, bool want_force, double* ox,
            double* oy, double* oz) {
  const int64_t n = t.n;
  const double eps2 = p->eps * p->eps;
  // targets: sorted positions [q0, q1), all or the share
  int64_t q0 = 0, q1 = n;
  target_range(c, n, q0, q1);
  const int64_t nt = q1 > q0 ? q1 - q0 : 0;
  const int grid = (int)ceil_div(nt > 0 ? nt : 1, kWalkBlock);
  PHYS_CUDA(c, cudaMemsetAsync(c->d_counter, 0, 2 * sizeof(unsigned long long), c->stream));
  PHYS_CUDA(c, cudaEventRecord(c->ev[6], c->stream));
  if (p->flags & PHYS_FLAG_GROUP_WALK) {
    PHYS_TRY(bh_group_walk(c, p, t, want_force, ox, oy, oz));
  } else if (p->precision == PHYS_F64_EXACT) {
    PHYS_LAUNCH(c, walk_exact_kernel, grid, kWalkBlock, 0, q0, q1, t.nnodes, t.link, t.rec64, t.body64,
                t.perm, t.hdr, p->G, eps2, (int)want_force, ox, oy, oz, c->d_counter, c->d_status);
  } else if (p->precision == PHYS_F64) {
    PHYS_LAUNCH(c, walk_kernel<false>, grid, kWalkBlock, 0, (int)q0, (int)q1, (int)t.nnodes, t.w32, t.w64,
                t.body64, t.body_hi, t.body_lo, t.perm, t.hdr, p->G, eps2, (int)want_force, ox, oy,
                oz, c->d_counter, c->d_status);
  } else if (WALK_PAIRED && t.w32x2) {
    if (q0 % 64) return fail(c, PHYS_ERR_ARG, "per-body walk share must start at a multiple of 64");
    const int grid2 = (int)ceil_div(nt > 0 ? nt : 1, 64 * (kWalk2Block / 32));
    PHYS_LAUNCH(c, walk2_kernel, grid2, kWalk2Block, 0, (int)(q0 / 64), (int)q1, (int)t.nnodes, t.w32x2, t.body2,
                t.body64, t.perm, p->G, eps2, (int)want_force, ox, oy, oz, c->d_counter,
                c->d_status);
  } else {
    PHYS_LAUNCH(c, walk_kernel<true>, grid, kWalkBlock, 0, (int)q0, (int)q1, (int)t.nnodes, t.w32, t.w64,
                t.body64, t.body_hi, t.body_lo, t.perm, t.hdr, p->G, eps2, (int)want_force, ox, oy,
                oz, c->d_counter, c->d_status);
  }
  PHYS_CUDA(c, cudaEventRecord(c->ev[7], c->stream));
  return PHYS_OK;
}

}  // namespace phys
