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
walk_kernel(int n, int nnodes, const Rec32* __restrict__ w32, const Rec64* __restrict__ w64,
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
  const int p = blockIdx.x * kWalkBlock + threadIdx.x;
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
      const float inv = rsqrtf(d2 + eps2f);
      const float w = use ? A.w * (inv * inv * inv) : 0.f;
      px = fmaf(rx, w, px);
      py = fmaf(ry, w, py);
      pz = fmaf(rz, w, pz);
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
            const float inv = rsqrtf(fmaf(rx, rx, fmaf(ry, ry, fmaf(rz, rz, eps2f))));
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
  while (node < nnodes) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      if (node >= nnodes) break;
      node = visit(node);
    }
    if (kF32) flush();
  }
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
// F64_EXACT walk (leaf capacity 1).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kWalkBlock)
walk_exact_kernel(int64_t n, int64_t nnodes, const int4* __restrict__ link,
                  const double4* __restrict__ rec64, const double4* __restrict__ body64,
                  const uint32_t* __restrict__ perm, const TreeHeader* __restrict__ hdr, double G,
                  double eps2, int want_force, double* __restrict__ ox, double* __restrict__ oy,
                  double* __restrict__ oz, unsigned long long* counter, int32_t* status) {
  __shared__ double s2d[kMaxLevels];
  for (int d = threadIdx.x; d < kMaxLevels; d += blockDim.x) s2d[d] = hdr->s2[d];
  __syncthreads();
  const double theta2 = hdr->theta2;
  const int64_t p = blockIdx.x * (int64_t)kWalkBlock + threadIdx.x;
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
  const int grid = (int)ceil_div(n, kWalkBlock);
  PHYS_CUDA(c, cudaMemsetAsync(c->d_counter, 0, sizeof(unsigned long long), c->stream));
  PHYS_CUDA(c, cudaEventRecord(c->ev[6], c->stream));
  if (p->precision == PHYS_F64_EXACT) {
    PHYS_LAUNCH(c, walk_exact_kernel, grid, kWalkBlock, 0, n, t.nnodes, t.link, t.rec64, t.body64,
                t.perm, t.hdr, p->G, eps2, (int)want_force, ox, oy, oz, c->d_counter, c->d_status);
  } else if (p->precision == PHYS_F64) {
    PHYS_LAUNCH(c, walk_kernel<false>, grid, kWalkBlock, 0, (int)n, (int)t.nnodes, t.w32, t.w64,
                t.body64, t.body_hi, t.body_lo, t.perm, t.hdr, p->G, eps2, (int)want_force, ox, oy,
                oz, c->d_counter, c->d_status);
  } else {
    PHYS_LAUNCH(c, walk_kernel<true>, grid, kWalkBlock, 0, (int)n, (int)t.nnodes, t.w32, t.w64,
                t.body64, t.body_hi, t.body_lo, t.perm, t.hdr, p->G, eps2, (int)want_force, ox, oy,
                oz, c->d_counter, c->d_status);
  }
  PHYS_CUDA(c, cudaEventRecord(c->ev[7], c->stream));
  return PHYS_OK;
}

}  // namespace phys
