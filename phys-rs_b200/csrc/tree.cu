// Barnes-Hut octree build on the device: bounding cube (K2), descent keys
// (K3), radix sort + equal-prefix fixup (K4), linear pre-order octree with
// per-cell mass and centre of mass (K5).
//
// The tree equals the reference's (gravity_tree.rs:110-154 run over the
// bodies in index order): a cell is split iff it holds >= 2 bodies and lies
// above the guard depth D* (depth >= 40 or half size < 1e-8); a cell at D*
// is a leaf that keeps the LAST inserted body while its mass and centre of
// mass count all of them.  Cell boundaries are the reference's f64 centres
// c +/- h/2 applied level by level, which the descent key reproduces bit for
// bit: octant = (x >= cx) | (y >= cy) << 1 | (z >= cz) << 2 per level.
//
// Ownership rule used to emit nodes in pre-order without recursion: with
// L[p] = common prefix length (octants, capped at D*) of sorted keys p, p+1
// (L[-1] = L[n-1] = -1), sorted position p owns the cells that start at p:
//   L[p-1] >= D*           -> none (inside a guard group)
//   L[p]   >= D*           -> internal cells at depths L[p-1]+1 .. D*-1, guard leaf at D*
//   otherwise              -> internal cells at depths L[p-1]+1 .. L[p],
//                             leaf at max(L[p-1], L[p]) + 1
// Pre-order = order of (start, depth), so node ids are a prefix sum.
#include <climits>
#include <vector>

#include "bh.cuh"

namespace phys {
namespace {

constexpr int kBlock = 256;

int grid_for(int64_t n, int block = kBlock, int cap = 148 * 16) {
  int64_t g = ceil_div(n, block);
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// ---------------------------------------------------------------------------
// K2: bounding cube, gravity_tree.rs:305-317.
// ---------------------------------------------------------------------------
constexpr int kBboxGrid = 296;

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__global__ void __launch_bounds__(kBlock)
bbox_partial_kernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                    const double* __restrict__ z, const double* __restrict__ m,
                    double* __restrict__ part, int32_t* status) {
  __shared__ double sh[7][kBlock / 32];
  double v[7] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY, INFINITY};
  bool bad = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double a = x[i], b = y[i], cc = z[i], mm = m[i];
    v[6] = fmin(v[6], mm);
    v[0] = fmin(v[0], a);
    v[1] = fmin(v[1], b);
    v[2] = fmin(v[2], cc);
    v[3] = fmax(v[3], a);
    v[4] = fmax(v[4], b);
    v[5] = fmax(v[5], cc);
    bad |= !isfinite(a) || !isfinite(b) || !isfinite(cc) || !isfinite(mm);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 3; ++k) v[k] = warp_min(v[k]);
#pragma unroll
  for (int k = 3; k < 6; ++k) v[k] = warp_max(v[k]);
  v[6] = warp_min(v[6]);
  if (lane == 0)
    for (int k = 0; k < 7; ++k) sh[k][warp] = v[k];
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(status, kStatNonfinite);
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      const bool mn = k < 3 || k == 6;
      double t = lane < kBlock / 32 ? sh[k][lane] : (mn ? INFINITY : -INFINITY);
      t = mn ? warp_min(t) : warp_max(t);
      if (lane == 0) part[blockIdx.x * 7 + k] = t;
    }
  }
}

// One warp: min/max of the partials (exact and order-free), then lane 0
// derives the cube and the per-depth constants.
__global__ void bbox_final_kernel(int nparts, const double* __restrict__ part, double theta,
                                  TreeHeader* hdr, const int32_t* status) {
  const int lane = threadIdx.x & 31;
  if (threadIdx.x >= 32) return;
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  double mmin = INFINITY;
  for (int b = lane; b < nparts; b += 32) {
    for (int k = 0; k < 3; ++k) {
      mn[k] = fmin(mn[k], part[b * 7 + k]);
      mx[k] = fmax(mx[k], part[b * 7 + 3 + k]);
    }
    mmin = fmin(mmin, part[b * 7 + 6]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    for (int k = 0; k < 3; ++k) {
      mn[k] = fmin(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
      mx[k] = fmax(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
    }
    mmin = fmin(mmin, __shfl_xor_sync(0xffffffffu, mmin, o));
  }
  if (lane != 0) return;
  hdr->min_mass = mmin;
  // extent = max - min; max_extent = x.max(y).max(z); half = max_extent*0.55 + 1
  const double ex = xsub(mx[0], mn[0]), ey = xsub(mx[1], mn[1]), ez = xsub(mx[2], mn[2]);
  const double max_extent = fmax(fmax(ex, ey), ez);
  const double half = xadd(xmul(max_extent, 0.55), 1.0);
  for (int k = 0; k < 3; ++k) hdr->center[k] = xmul(xadd(mn[k], mx[k]), 0.5);
  hdr->half = half;
  hdr->theta2 = xmul(theta, theta);
  double h = half;
  int dstar = -1;
  for (int d = 0; d < kMaxLevels; ++d) {
    const double s = xmul(h, 2.0);  // full side length (gravity_tree.rs:192)
    hdr->s2[d] = xmul(s, s);
    if (dstar < 0 && (d >= kMaxDepth || h < kMinNodeSize)) dstar = d;
    h = xmul(h, 0.5);  // child half size (gravity_tree.rs:137)
  }
  hdr->dstar = dstar;
  hdr->nonfinite = (*status & kStatNonfinite) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// K3: descent keys.  hi = octants 0..20 (octant d in bits 62-3d..60-3d), lo =
// octants 21..39 (bits 56..0); octants below D* are zero for every body.
// Each body's (x, y, z, m) also goes into one 32-byte record, so that the
// gather into key order after the sort reads one sector per body instead of
// one per component.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock)
keys_kernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
            const double* __restrict__ z, const double* __restrict__ m,
            const TreeHeader* __restrict__ hdr, uint64_t* __restrict__ khi,
            uint64_t* __restrict__ klo, uint32_t* __restrict__ idx, double4* __restrict__ rec) {
  const double c0 = hdr->center[0], c1 = hdr->center[1], c2 = hdr->center[2];
  const double h0 = hdr->half;
  const int D = hdr->dstar;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double px = x[i], py = y[i], pz = z[i];
    double cx = c0, cy = c1, cz = c2, h = h0;
    uint64_t kh = 0, kl = 0;
    for (int d = 0; d < D; ++d) {
      const uint32_t o = (px >= cx ? 1u : 0u) | (py >= cy ? 2u : 0u) | (pz >= cz ? 4u : 0u);
      const double q = xmul(h, 0.5);  // child_center, gravity_tree.rs:100-107
      cx = xadd(cx, (o & 1u) ? q : -q);
      cy = xadd(cy, (o & 2u) ? q : -q);
      cz = xadd(cz, (o & 4u) ? q : -q);
      h = q;
      if (d < 21)
        kh |= (uint64_t)o << (60 - 3 * d);
      else
        kl |= (uint64_t)o << (54 - 3 * (d - 21));
    }
    khi[i] = kh;
    klo[i] = kl;
    idx[i] = (uint32_t)i;
    rec[i] = make_double4(px, py, pz, m[i]);
  }
}

// Bodies whose first 21 octants agree are ordered by (lo, index) in place.
// The radix pass over hi is stable on index-ordered input, so each run is
// already in index order; runs are rare (cells of side 2h/2^21).
__device__ __forceinline__ bool key_less(const uint64_t* klo, uint32_t a, uint32_t b) {
  const uint64_t la = klo[a], lb = klo[b];
  return la < lb || (la == lb && a < b);
}

__global__ void run_fixup_kernel(int64_t n, const uint64_t* __restrict__ hs,
                                 uint32_t* __restrict__ perm, const uint64_t* __restrict__ klo,
                                 uint32_t* __restrict__ tmp, const int32_t* status) {
  if (sort_failed(status)) return;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p + 1 < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t h = hs[p];
    if (hs[p + 1] != h) continue;
    if (p > 0 && hs[p - 1] == h) continue;
    int64_t e = p + 2;
    while (e < n && hs[e] == h) ++e;
    const int64_t len = e - p;
    uint32_t* a = perm + p;
    if (len <= 32) {
      for (int64_t i = 1; i < len; ++i) {
        const uint32_t v = a[i];
        int64_t j = i - 1;
        while (j >= 0 && key_less(klo, v, a[j])) {
          a[j + 1] = a[j];
          --j;
        }
        a[j + 1] = v;
      }
    } else {  // bottom-up merge sort through tmp[p..e)
      uint32_t* src = a;
      uint32_t* dst = tmp + p;
      for (int64_t w = 1; w < len; w *= 2) {
        for (int64_t lo = 0; lo < len; lo += 2 * w) {
          int64_t mid = min(lo + w, len), hi = min(lo + 2 * w, len);
          int64_t i = lo, j = mid, k = lo;
          while (i < mid && j < hi) dst[k++] = key_less(klo, src[j], src[i]) ? src[j++] : src[i++];
          while (i < mid) dst[k++] = src[i++];
          while (j < hi) dst[k++] = src[j++];
        }
        uint32_t* t = src;
        src = dst;
        dst = t;
      }
      if (src != a)
        for (int64_t i = 0; i < len; ++i) a[i] = src[i];
    }
  }
}

__global__ void __launch_bounds__(kBlock)
gather_sorted_kernel(int64_t n, const uint32_t* __restrict__ perm, const uint64_t* __restrict__ klo,
                     const double4* __restrict__ rec, uint64_t* __restrict__ lo_s,
                     double4* __restrict__ body64,
                     float4* __restrict__ body_hi, float4* __restrict__ body_lo,
                     Body32x2* __restrict__ body2, const int32_t* status) {
  if (sort_failed(status)) return;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t i = perm[p];
    lo_s[p] = klo[i];
    const double4 b = rec[i];
    body64[p] = b;
    if (body_hi) {
      float4 h, l;
      split_df(b.x, h.x, l.x);
      split_df(b.y, h.y, l.y);
      split_df(b.z, h.z, l.z);
      h.w = (float)b.w;
      l.w = 0.f;
      body_hi[p] = h;
      body_lo[p] = l;
      if (body2) {
        Body32x2 q;
        q.q0 = make_float4(h.x, h.x, h.y, h.y);
        q.q1 = make_float4(h.z, h.z, h.w, h.w);
        q.q2 = make_float4(l.x, l.x, l.y, l.y);
        q.q3 = make_float4(l.z, l.z, 0.f, 0.f);
        body2[p] = q;
      }
    }
  }
}

__device__ __forceinline__ int lcp_octants(uint64_t ha, uint64_t la, uint64_t hb, uint64_t lb) {
  if (ha != hb) return (__clzll((long long)(ha ^ hb)) - 1) / 3;
  if (la != lb) return 21 + (__clzll((long long)(la ^ lb)) - 7) / 3;
  return kMaxDepth;
}

__global__ void __launch_bounds__(kBlock)
lcp_count_kernel(int64_t n, const uint64_t* __restrict__ hs, const uint64_t* __restrict__ ls,
                 const TreeHeader* __restrict__ hdr, int32_t* __restrict__ L,
                 int32_t* __restrict__ cnt) {
  const int D = hdr->dstar;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p <= n;
       p += (int64_t)gridDim.x * blockDim.x) {
    if (p == n) {
      cnt[n] = 0;
      continue;
    }
    const int Ln = p + 1 < n ? min(lcp_octants(hs[p], ls[p], hs[p + 1], ls[p + 1]), D) : -1;
    const int Lp = p > 0 ? min(lcp_octants(hs[p - 1], ls[p - 1], hs[p], ls[p]), D) : -1;
    L[p] = Ln;
    int c;
    if (Lp >= D)
      c = 0;
    else if (Ln >= D)
      c = D - Lp;
    else
      c = max(0, Ln - Lp) + 1;
    cnt[p] = c;
  }
}

// Keys truncated to the first d octants.
__device__ __forceinline__ void trunc_key(uint64_t h, uint64_t l, int d, uint64_t& th,
                                          uint64_t& tl) {
  if (d <= 21) {
    const uint64_t keep = (1ull << 63) - 1;
    const uint64_t drop = d == 21 ? 0ull : ((1ull << (63 - 3 * d)) - 1);
    th = h & (keep ^ drop);
    tl = 0;
  } else {
    th = h;
    const uint64_t keep = (1ull << 57) - 1;
    const int dd = d - 21;
    const uint64_t drop = dd >= 19 ? 0ull : ((1ull << (57 - 3 * dd)) - 1);
    tl = l & (keep ^ drop);
  }
}

// First q > p whose key differs from key p in the first d octants (n if none).
__device__ int64_t cell_end(int64_t n, const uint64_t* __restrict__ hs,
                            const uint64_t* __restrict__ ls, int64_t p, int d) {
  uint64_t ph, pl;
  trunc_key(hs[p], ls[p], d, ph, pl);
  auto same = [&](int64_t q) {
    uint64_t qh, ql;
    trunc_key(hs[q], ls[q], d, qh, ql);
    return qh == ph && ql == pl;
  };
  // gallop: find hi with !same(hi) or hi == n
  int64_t lo = p + 1, step = 1, hi = p + 1;
  while (hi < n && same(hi)) {
    lo = hi + 1;
    hi = p + 1 + step;
    step <<= 1;
    if (hi > n) hi = n;
  }
  // answer in [lo, hi]
  while (lo < hi) {
    const int64_t mid = lo + (hi - lo) / 2;
    if (same(mid))
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(kBlock)
emit_nodes_kernel(int64_t n, const uint64_t* __restrict__ hs, const uint64_t* __restrict__ ls,
                  const int32_t* __restrict__ L, const int32_t* __restrict__ cnt,
                  const int32_t* __restrict__ first, const TreeHeader* __restrict__ hdr,
                  int4* __restrict__ link) {
  const int D = hdr->dstar;
  const int32_t total = first[n];
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int c = cnt[p];
    if (c == 0) continue;
    const int32_t f = first[p];
    const int Lp = p > 0 ? L[p - 1] : -1;
    const int Ln = L[p];
    const bool guard = Ln >= D;
    for (int k = 0; k < c; ++k) {
      const int d = Lp + 1 + k;
      const bool leaf = k == c - 1;
      int64_t end;
      if (leaf && !guard)
        end = p + 1;
      else
        end = cell_end(n, hs, ls, p, d);
      const int32_t next = end < n ? first[end] : total;
      int meta = d;
      if (leaf) meta |= kMetaLeaf;
      if (leaf && guard) meta |= kMetaGuard;
      link[f + k] = make_int4(next, (int)p, (int)end, meta);
    }
  }
}

// Bucket leaves of capacity C > 1, emitted directly: a cell survives iff its
// parent holds more than C bodies (the root always).  For sorted position p,
// e*(p) = the deepest depth at which the cell holding p has more than C
// bodies: C + 1 consecutive keys containing p share e octants iff the
// minimum of their C adjacent common prefixes is >= e, so
//   e*(p) = max over q in [p - C, p] of min(L[q], ..., L[q + C - 1])
// (-1 when fewer than C + 1 keys exist).  Position p owns the cells at depths
// Lp+1 .. dl (dl its leaf's depth in the full tree); of those it keeps the
// ones no deeper than e*(p) + 1, and the deepest one kept is a leaf.
__global__ void __launch_bounds__(kBlock)
prune_count_kernel(int64_t n, const int32_t* __restrict__ L, const TreeHeader* __restrict__ hdr,
                   int C, int32_t* __restrict__ cnt, int32_t* __restrict__ emax) {
  const int D = hdr->dstar;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p <= n;
       p += (int64_t)gridDim.x * blockDim.x) {
    if (p == n) {
      cnt[n] = 0;
      continue;
    }
    int best = -1;
    const int64_t q0 = p - C > 0 ? p - C : 0;
    for (int64_t q = q0; q <= p && q + C <= n - 1; ++q) {
      int m = INT_MAX;
      for (int i = 0; i < C; ++i) m = min(m, L[q + i]);
      best = max(best, m);
    }
    emax[p] = best;
    const int Lp = p > 0 ? L[p - 1] : -1;
    const int Ln = L[p];  // -1 for the last position
    int c = 0;
    if (Lp < D) {
      const int dl = Ln >= D ? D : max(Lp, Ln) + 1;
      c = max(0, min(dl, best + 1) - Lp);
    }
    cnt[p] = c;
  }
}

// One thread per kept cell (the cells of one position can be many, each
// with a search for its end: a thread per position would leave the long
// chains near the root to a few threads).  Cell k belongs to the last
// position p with first[p] <= k.
__global__ void __launch_bounds__(kBlock)
emit_pruned_kernel(int64_t n, const uint64_t* __restrict__ hs, const uint64_t* __restrict__ ls,
                   const int32_t* __restrict__ L, const int32_t* __restrict__ cnt,
                   const int32_t* __restrict__ first, const TreeHeader* __restrict__ hdr,
                   int4* __restrict__ link) {
  const int D = hdr->dstar;
  const int32_t total = first[n];
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = 0, hi = n - 1;  // largest p with first[p] <= k (first[n] = total > k)
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (first[mid] <= k)
        lo = mid;
      else
        hi = mid - 1;
    }
    const int64_t p = lo;
    const int c = cnt[p];
    const int kk = (int)(k - first[p]);
    const int Lp = p > 0 ? L[p - 1] : -1;
    const int Ln = L[p];
    const bool guard = Ln >= D;
    const int dl = guard ? D : max(Lp, Ln) + 1;
    const int d = Lp + 1 + kk;
    const bool full_leaf = d == dl;
    const bool leaf = kk == c - 1;
    const int64_t end = (full_leaf && !guard) ? p + 1 : cell_end(n, hs, ls, p, d);
    const int32_t next = end < n ? first[end] : total;
    int meta = d;
    if (leaf) meta |= kMetaLeaf;
    if (full_leaf && guard) meta |= kMetaGuard;
    link[k] = make_int4(next, (int)p, (int)end, meta);
  }
}

// parent / number of children, by walking each internal node's child chain.
__global__ void __launch_bounds__(kBlock)
children_kernel(int64_t nnodes, const int4* __restrict__ link, int32_t* __restrict__ parent,
                int32_t* __restrict__ nchild, int32_t* status) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnodes;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int4 lk = link[k];
    if (k == 0) parent[0] = -1;
    int cc = 0;
    if (!(lk.w & kMetaLeaf)) {
      int32_t ch = (int32_t)k + 1;
      while (ch < lk.x && cc < 8) {  // an octree cell has at most 8 children
        parent[ch] = (int32_t)k;
        const int32_t nx = link[ch].x;
        if (nx <= ch) break;
        ch = nx;
        ++cc;
      }
      if (ch < lk.x) atomicOr(status, kStatOverflow);
    }
    nchild[k] = cc;
  }
}

// ---------------------------------------------------------------------------
// Mass / centre of mass, parallel form: sums of m and m*x, leaves over their
// bodies in key order, internal cells over their children in octant order
// (fixed order: deterministic), propagated bottom-up by the last-arriving
// child.  Differs from the reference's insertion-order running mean by ulps.
// ---------------------------------------------------------------------------
// arrive[] += 1 with acquire-release order at GPU scope; returns the old
// count.  Orders the caller's earlier stores before it and later loads after
// it, in place of a fence on each side of a relaxed atomic.
__device__ __forceinline__ int32_t arrive_acq_rel(int32_t* p) {
  int32_t old;
  asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(old) : "l"(p) : "memory");
  return old;
}

__global__ void __launch_bounds__(kBlock)
com_upward_kernel(int64_t nnodes, const int4* __restrict__ link,
                  const int32_t* __restrict__ parent, const int32_t* __restrict__ nchild,
                  int32_t* __restrict__ arrive, const double4* __restrict__ body64,
                  double4* __restrict__ sums, int32_t* status) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnodes;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int4 lk = link[k];
    if (!(lk.w & kMetaLeaf)) continue;
    double sx = 0.0, sy = 0.0, sz = 0.0, sm = 0.0;
    for (int q = lk.y; q < lk.z; ++q) {
      const double4 b = body64[q];
      sx = fma(b.w, b.x, sx);
      sy = fma(b.w, b.y, sy);
      sz = fma(b.w, b.z, sz);
      sm += b.w;
    }
    sums[k] = make_double4(sx, sy, sz, sm);
    int32_t cur = (int32_t)k;
    while (cur != 0) {
      const int32_t par = parent[cur];
      if (par < 0 || par >= cur) {  // parents precede children in pre-order
        atomicOr(status, kStatOverflow);
        break;
      }
      // release: this child's sums are visible to whoever arrives last;
      // acquire: the last arrival sees every sibling's sums
      if (arrive_acq_rel(&arrive[par]) != nchild[par] - 1) break;
      const int32_t stop = link[par].x;
      double ax = 0.0, ay = 0.0, az = 0.0, am = 0.0;
      int guard = 0;
      for (int32_t ch = par + 1; ch < stop && guard < 8; ch = link[ch].x, ++guard) {
        const double2* sp = reinterpret_cast<const double2*>(&sums[ch]);
        const double2 v0 = __ldcg(sp), v1 = __ldcg(sp + 1);  // L2: written by other threads
        ax += v0.x;
        ay += v0.y;
        az += v1.x;
        am += v1.y;
      }
      sums[par] = make_double4(ax, ay, az, am);
      cur = par;
    }
  }
}

// ---------------------------------------------------------------------------
// Mass / centre of mass, reference form (gravity_tree.rs:113-118): for every
// cell the running mean com = (com*M + p*m) / (M + m) over its bodies in
// index (insertion) order.  Segments (node, body) pairs sorted by node then
// index, then one thread per node runs the recurrence.
// ---------------------------------------------------------------------------
__global__ void node_count_kernel(int64_t nnodes, const int4* __restrict__ link,
                                  int32_t* __restrict__ cnt) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k <= nnodes;
       k += (int64_t)gridDim.x * blockDim.x)
    cnt[k] = k < nnodes ? link[k].z - link[k].y : 0;
}

__global__ void __launch_bounds__(kBlock)
expand_kernel(int64_t total, int64_t nnodes, const int32_t* __restrict__ eoff,
              const int4* __restrict__ link, const uint32_t* __restrict__ perm,
              uint64_t* __restrict__ entries) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = 0, hi = nnodes;  // last k with eoff[k] <= e
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) / 2;
      if (eoff[mid] <= e)
        lo = mid;
      else
        hi = mid;
    }
    const int q = link[lo].y + (int)(e - eoff[lo]);
    entries[e] = ((uint64_t)lo << 32) | perm[q];
  }
}

//
// With skip_unused, a cell that no target can take as a monopole is not
// summed at all: a cell of side s is taken only if s^2 < theta^2 |com - x|^2,
// and com and x both lie in the root cube of half size H (com as a convex
// combination of bodies: every mass positive, else nothing is skipped), so
// |com - x|^2 <= 12 H^2; when s^2 >= theta^2 12 H^2 (with a 1e-6 margin for
// rounding) the walk opens the cell whatever its centre of mass (a NaN
// distance opens it too).  Such a cell gets a NaN centre of mass and mass
// +inf: nothing reads either, and a positive mass sets the same gate
// (mass > 0) as the exact sum of positive masses.  This is the root for
// theta <= 0.577 and every internal cell for theta = 0; it removes the
// longest chains, the root's one step per body.
__device__ __forceinline__ bool com_unused(bool can_skip, double bound, int4 lk,
                                           const TreeHeader* __restrict__ hdr) {
  return can_skip && !(lk.w & kMetaLeaf) && hdr->s2[lk.w & kMetaDepth] >= bound;
}

// Bodies of the (cell, body) pairs in pair order, so that each cell's
// recurrence streams them from consecutive addresses (cells skipped by
// com_unused are left out).
__global__ void __launch_bounds__(kBlock)
gather_entries_kernel(int64_t total, const uint64_t* __restrict__ entries,
                      const double* __restrict__ x, const double* __restrict__ y,
                      const double* __restrict__ z, const double* __restrict__ m,
                      const int4* __restrict__ link, const TreeHeader* __restrict__ hdr,
                      int skip_unused, double4* __restrict__ eb, const int32_t* status) {
  if (sort_failed(status)) return;
  const bool can_skip = skip_unused && hdr->min_mass > 0.0;
  const double bound = hdr->theta2 * 12.0 * hdr->half * hdr->half * (1.0 + 1e-6);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t v = entries[e];
    if (com_unused(can_skip, bound, link[v >> 32], hdr)) continue;
    const uint32_t b = (uint32_t)(v & 0xffffffffu);
    eb[e] = make_double4(x[b], y[b], z[b], m[b]);
  }
}

// Cells with at least kLongChain bodies run on a warp each
// (com_recurrence_long_kernel), the rest on a thread each.
constexpr int kLongChain = 2048;

// The reference recurrence over a cell's gathered bodies eb[e0, e1)
// (gravity_tree.rs:113-118): M' = M + m, and when M' > 0,
// c = (c M + x m) / M' per coordinate.  kFast divides through div_recip by
// RN(1/M'), which depends only on the mass chain and so is computed off the
// critical path (a multiply, an add and the five operations of div_recip per
// body instead of a multiply, an add and a division); it returns false when
// a step left div_recip's range (or M' <= 0), and the caller then reruns the
// cell with kFast = false, the reference's division.  Both give the IEEE
// result of every step.  The next batch's loads are issued before the
// current batch's chain, so the chain does not wait for memory.
template <bool kFast>
__device__ __forceinline__ bool com_chain(const double4* __restrict__ eb, int64_t e0, int64_t e1,
                                          double4& out) {
  double M = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
  bool ok = true;
  auto step = [&](const double4 b) {
    const double nt = xadd(M, b.w);
    if (kFast) {
      const double y = __drcp_rn(nt);
      const double ax = xadd(xmul(cx, M), xmul(b.x, b.w));
      const double ay = xadd(xmul(cy, M), xmul(b.y, b.w));
      const double az = xadd(xmul(cz, M), xmul(b.z, b.w));
      ok &= div_recip_den_ok(nt) & div_recip_num_ok(ax) & div_recip_num_ok(ay) &
            div_recip_num_ok(az);
      cx = div_recip(ax, nt, y);
      cy = div_recip(ay, nt, y);
      cz = div_recip(az, nt, y);
    } else if (nt > 0.0) {
      cx = xdiv(xadd(xmul(cx, M), xmul(b.x, b.w)), nt);
      cy = xdiv(xadd(xmul(cy, M), xmul(b.y, b.w)), nt);
      cz = xdiv(xadd(xmul(cz, M), xmul(b.z, b.w)), nt);
    }
    M = nt;
  };
  constexpr int kB = 8;
  double4 cur[kB], nxt[kB];
#pragma unroll
  for (int u = 0; u < kB; ++u)
    cur[u] = e0 + u < e1 ? eb[e0 + u] : make_double4(0.0, 0.0, 0.0, 0.0);
  for (int64_t e = e0; e < e1; e += kB) {
#pragma unroll
    for (int u = 0; u < kB; ++u)
      nxt[u] = e + kB + u < e1 ? eb[e + kB + u] : make_double4(0.0, 0.0, 0.0, 0.0);
    if (e + kB <= e1) {
#pragma unroll
      for (int u = 0; u < kB; ++u) step(cur[u]);
    } else {
      for (int u = 0; u < kB; ++u)
        if (e + u < e1) step(cur[u]);
    }
#pragma unroll
    for (int u = 0; u < kB; ++u) cur[u] = nxt[u];
  }
  out = make_double4(cx, cy, cz, M);
  return ok;
}

// One thread per cell runs com_chain over the cell's gathered bodies.
// Cells of kLongChain bodies or more are appended to `longs` (count in
// longs[nnodes]) instead.
__global__ void __launch_bounds__(kBlock)
com_recurrence_kernel(int64_t nnodes, const int32_t* __restrict__ eoff,
                      const double4* __restrict__ eb, double4* __restrict__ mc,
                      const int4* __restrict__ link, const TreeHeader* __restrict__ hdr,
                      int skip_unused, int32_t* __restrict__ longs, const int32_t* status) {
  if (sort_failed(status)) return;
  // the bound holds when every centre of mass is a convex combination of
  // bodies (all masses positive)
  const bool can_skip = skip_unused && hdr->min_mass > 0.0;
  const double bound = hdr->theta2 * 12.0 * hdr->half * hdr->half * (1.0 + 1e-6);
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnodes;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e0 = eoff[k], e1 = eoff[k + 1];
    if (com_unused(can_skip, bound, link[k], hdr)) {
      const double nan = __longlong_as_double(0x7ff8000000000000ll);
      mc[k] = make_double4(nan, nan, nan, __longlong_as_double(0x7ff0000000000000ll));
      continue;
    }
    if (e1 - e0 >= kLongChain) {
      longs[atomicAdd(&longs[nnodes], 1)] = (int32_t)k;
      continue;
    }
    double4 r;
    if (!com_chain<true>(eb, e0, e1, r)) com_chain<false>(eb, e0, e1, r);
    mc[k] = r;
  }
}

// The same recurrence for the cells listed by com_recurrence_kernel, a warp
// per cell: the warp stages 32 bodies at a time in shared memory (one
// coalesced 1 KiB read, the next batch's in flight) while lanes 0, 1 and 2
// run the x, y and z chains.
constexpr int kLongWarps = 4;
struct LongStage {
  double4 rec[2][32];           // two batches of body records (x, y, z, m)
  double nt[2][32], y[2][32];   // per body: running mass M + m, RN(1/(M + m))
};

// The reference's form (com_chain<false> per coordinate lane): the fallback.
__device__ void com_chain_warp_ieee(const double4* __restrict__ eb, int64_t e0, int64_t e1,
                                   LongStage& S, int lane, double4& out) {
  const double4 zero = make_double4(0.0, 0.0, 0.0, 0.0);
  double M = 0.0, cc = 0.0;  // lane j < 3: coordinate j
  double4 v = e0 + lane < e1 ? eb[e0 + lane] : zero;
  for (int64_t e = e0; e < e1; e += 32) {
    S.rec[0][lane] = v;
    __syncwarp();
    v = e + 32 + lane < e1 ? eb[e + 32 + lane] : zero;
    const int cnt = (int)min((int64_t)32, e1 - e);
    if (lane < 3) {
      const double* q = reinterpret_cast<const double*>(&S.rec[0][0]);
      for (int u = 0; u < cnt; ++u) {
        const double p = q[4 * u + lane], mm = q[4 * u + 3];
        const double nt = xadd(M, mm);
        if (nt > 0.0) cc = xdiv(xadd(xmul(cc, M), xmul(p, mm)), nt);
        M = nt;
      }
    }
    __syncwarp();
  }
  const double cy = __shfl_sync(0xffffffffu, cc, 1), cz = __shfl_sync(0xffffffffu, cc, 2);
  out = make_double4(cc, cy, cz, M);
}

// The fast form: per body a multiply, an add and div_recip's five
// operations, with nothing else on the chain.  The running masses of a
// batch (the reference's additions, in order) are summed by lane 0 while the
// batch before it runs, and the whole warp then forms the batch's 32
// reciprocals at once (__drcp_rn, correctly rounded, as div_recip requires),
// so the chain's loop over a full batch has no branch and its shared-memory
// loads can be issued ahead.  Returns false (warp-uniform) when a step left
// div_recip's range or the running mass was not positive; the caller then
// reruns the cell in the reference's form.
__device__ bool com_chain_warp_fast(const double4* __restrict__ eb, int64_t e0, int64_t e1,
                                    LongStage& S, int lane, double4& out) {
  const double4 zero = make_double4(0.0, 0.0, 0.0, 0.0);
  const int64_t len = e1 - e0;
  S.rec[0][lane] = lane < len ? eb[e0 + lane] : zero;
  double4 v = 32 + lane < len ? eb[e0 + 32 + lane] : zero;
  __syncwarp();
  if (lane == 0) {  // running masses of batch 0
    double M = 0.0;
    const int c0 = (int)min((int64_t)32, len);
    for (int u = 0; u < c0; ++u) {
      M = xadd(M, S.rec[0][u].w);
      S.nt[0][u] = M;
    }
  }
  __syncwarp();
  S.y[0][lane] = __drcp_rn(S.nt[0][lane]);  // lanes past the batch: unused
  __syncwarp();
  bool ok = true;
  double cc = 0.0, M = 0.0;  // lane j < 3: coordinate j; M = mass before the body
  for (int64_t base = e0; base < e1; base += 32) {
    const int cur = (int)(((base - e0) >> 5) & 1), nxt = cur ^ 1;
    const int cnt = (int)min((int64_t)32, e1 - base);
    const int cntn = (int)max((int64_t)0, min((int64_t)32, e1 - base - 32));
    if (cntn > 0) S.rec[nxt][lane] = v;
    __syncwarp();
    v = base + 64 + lane < e1 ? eb[base + 64 + lane] : zero;
    if (lane < 3) {
      const double* __restrict__ rc = reinterpret_cast<const double*>(&S.rec[cur][0]);
      const double* __restrict__ rn = reinterpret_cast<const double*>(&S.rec[nxt][0]);
      const double* __restrict__ ntc = S.nt[cur];
      const double* __restrict__ yc = S.y[cur];
      auto step = [&](int u) {
        const double nt = ntc[u];
        const double a = xadd(xmul(cc, M), xmul(rc[4 * u + lane], rc[4 * u + 3]));
        ok &= div_recip_den_ok(nt) & div_recip_num_ok(a);
        cc = div_recip(a, nt, yc[u]);
        M = nt;
      };
      if (cnt == 32) {
        // the next batch's running masses, in registers until the batch is
        // done (a store into the arrays the loop reads would keep the
        // loads behind it)
        double Mn[32];
        double acc = ntc[31];  // running mass before the next batch
#pragma unroll
        for (int u = 0; u < 32; ++u) {
          step(u);
          acc = xadd(acc, rn[4 * u + 3]);  // bodies past cntn: never stored
          Mn[u] = acc;
        }
        if (lane == 0) {
#pragma unroll
          for (int u = 0; u < 32; ++u)
            if (u < cntn) S.nt[nxt][u] = Mn[u];
        }
      } else {  // the last batch of the cell
        for (int u = 0; u < cnt; ++u) step(u);
      }
    }
    __syncwarp();
    if (cntn > 0) S.y[nxt][lane] = __drcp_rn(S.nt[nxt][lane]);
    __syncwarp();
  }
  const double cy = __shfl_sync(0xffffffffu, cc, 1), cz = __shfl_sync(0xffffffffu, cc, 2);
  out = make_double4(cc, cy, cz, M);
  return !__any_sync(0xffffffffu, !ok);
}

__global__ void __launch_bounds__(32 * kLongWarps)
com_recurrence_long_kernel(int64_t nnodes, const int32_t* __restrict__ eoff,
                           const double4* __restrict__ eb, double4* __restrict__ mc,
                           const int32_t* __restrict__ longs, const int32_t* status) {
  if (sort_failed(status)) return;
  __shared__ LongStage stage[kLongWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nlong = min(longs[nnodes], (int32_t)nnodes);
  for (int i = blockIdx.x * kLongWarps + w; i < nlong; i += gridDim.x * kLongWarps) {
    const int k = longs[i];
    const int64_t e0 = eoff[k], e1 = eoff[k + 1];
    double4 r;
    if (!com_chain_warp_fast(eb, e0, e1, stage[w], lane, r))
      com_chain_warp_ieee(eb, e0, e1, stage[w], lane, r);
    if (lane == 0) mc[k] = r;
    __syncwarp();
  }
}

// q[i] = a[i] / b[i] through the centre-of-mass chains' division: div_recip
// where its range holds, the IEEE division elsewhere (a test-only check
// that both give the correctly rounded quotient).
__global__ void __launch_bounds__(kBlock)
debug_divide_kernel(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                    double* __restrict__ q) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double x = a[i], d = b[i];
    q[i] = div_recip_den_ok(d) && div_recip_num_ok(x) ? div_recip(x, d, __drcp_rn(d))
                                                      : xdiv(x, d);
  }
}

// Walk records + gate bit.  `mc` holds either raw sums (parallel form, turned
// into com = S/M here) or finished (com, M) (reference form).
__global__ void __launch_bounds__(kBlock)
finalize_kernel(int64_t nnodes, int4* __restrict__ link, double4* __restrict__ mc, int sums,
                int leaf_cap, const double4* __restrict__ body64, const TreeHeader* __restrict__ hdr,
                double4* __restrict__ rec64, Rec32* __restrict__ w32, Rec64* __restrict__ w64,
                Rec32x2* __restrict__ w32x2) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnodes;
       k += (int64_t)gridDim.x * blockDim.x) {
    int4 lk = link[k];
    double4 a = mc[k];
    if (sums) {
      const double M = a.w;
      if (M > 0.0)
        a = make_double4(a.x / M, a.y / M, a.z / M, M);
      else
        a = make_double4(0.0, 0.0, 0.0, M);
      mc[k] = a;
    }
    const bool gate = a.w > 0.0;
    if (gate) lk.w |= kMetaGate;
    link[k].w = lk.w;
    const int d = lk.w & kMetaDepth;
    const int cntb = lk.z - lk.y;
    const bool leaf = lk.w & kMetaLeaf;
    int self = -1;
    double4 r = a;
    if (leaf && cntb == 1) {
      self = lk.y;
    } else if (leaf && (lk.w & kMetaGuard) && leaf_cap == 1) {
      self = lk.z - 1;  // the last inserted (highest index) body
    }
    if (self >= 0) r = body64[self];
    if (rec64) rec64[k] = r;
    int wmeta = (gate || k == 0) ? d : kWSkip;
    if (leaf && self < 0) wmeta |= kWLeaf | (cntb << 8);
    const int4 wl = make_int4(lk.x, self, lk.y, wmeta);
    if (w64) {
      Rec64 o;
      o.a = r;
      o.l = wl;
      w64[k] = o;
    }
    if (w32 || w32x2) {
      Rec32 o;
      split_df(r.x, o.a.x, o.b.x);
      split_df(r.y, o.a.y, o.b.y);
      split_df(r.z, o.a.z, o.b.z);
      o.a.w = (float)r.w;
      // accept iff s^2 < theta^2 d^2  <=>  d^2 > s^2 / theta^2 (inf for theta = 0)
      o.b.w = self >= 0 ? -1.0f : (float)(hdr->s2[d] / hdr->theta2);
      o.l = wl;
      if (w32) w32[k] = o;
      if (w32x2) {
        Rec32x2 q;
        q.q0 = make_float4(o.a.x, o.a.x, o.a.y, o.a.y);
        q.q1 = make_float4(o.a.z, o.a.z, o.a.w, o.a.w);
        q.q2 = make_float4(o.b.x, o.b.x, o.b.y, o.b.y);
        q.q3 = make_float4(o.b.z, o.b.z, o.b.w, o.b.w);
        q.l = wl;
        w32x2[k] = q;
      }
    }
  }
}

// Breadth-first order: node ids stably sorted by depth (one radix pass on
// pre-order input); inverse map.
__global__ void depth_key_kernel(int64_t nnodes, const int4* __restrict__ link,
                                 uint64_t* __restrict__ key, uint32_t* __restrict__ val) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnodes;
       k += (int64_t)gridDim.x * blockDim.x) {
    key[k] = (uint64_t)(link[k].w & kMetaDepth);
    val[k] = (uint32_t)k;
  }
}

__global__ void invert_kernel(int64_t nnodes, const uint32_t* __restrict__ bfs2pre,
                              int32_t* __restrict__ pre2bfs, const int32_t* status) {
  if (sort_failed(status)) return;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nnodes;
       j += (int64_t)gridDim.x * blockDim.x)
    pre2bfs[bfs2pre[j]] = (int32_t)j;
}

__global__ void __launch_bounds__(kBlock)
gnode_kernel(int64_t nnodes, const uint32_t* __restrict__ bfs2pre,
             const int32_t* __restrict__ pre2bfs, const int4* __restrict__ link,
             const double4* __restrict__ mc, const int32_t* __restrict__ nchild, int leaf_cap,
             const double4* __restrict__ body64, const TreeHeader* __restrict__ hdr,
             GNode* __restrict__ g, const int32_t* status) {
  if (sort_failed(status)) return;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nnodes;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)bfs2pre[j];
    const int4 lk = link[k];
    const int d = lk.w & kMetaDepth;
    const int cntb = lk.z - lk.y;
    const bool leaf = lk.w & kMetaLeaf;
    double4 r = mc[k];
    int4 l;
    if (!(lk.w & kMetaGate) && k != 0) {
      l = make_int4(0, kGSkip, lk.y, lk.z);
    } else if (leaf && (cntb == 1 || ((lk.w & kMetaGuard) && leaf_cap == 1))) {
      const int self = cntb == 1 ? lk.y : lk.z - 1;  // guard leaf: last inserted body
      r = body64[self];
      l = make_int4(self, (1 << 2) | kGSingle, lk.y, lk.z);
    } else if (leaf) {
      l = make_int4(lk.y, (cntb << 2) | kGBucket, lk.y, lk.z);
    } else {
      // children of a pre-order cell start at k + 1
      l = make_int4(pre2bfs[k + 1], (nchild[k] << 2) | kGInternal, lk.y, lk.z);
    }
    GNode o;
    split_df(r.x, o.hi.x, o.lo.x);
    split_df(r.y, o.hi.y, o.lo.y);
    split_df(r.z, o.hi.z, o.lo.z);
    o.hi.w = (float)r.w;
    o.lo.w = (float)hdr->s2[d];
    o.l = l;
    o.c64 = r;
    g[j] = o;
  }
}

// Bodies per target group that the build aims at (at most kGroupMax, the
// walk's capacity).
#ifndef GWALK_GROUP_BODIES
#define GWALK_GROUP_BODIES 64
#endif
constexpr int kGroupBuild = GWALK_GROUP_BODIES;
static_assert(kGroupBuild >= 1 && kGroupBuild <= kGroupMax, "group size");

// Target groups of the group walk: every cell with more than kGroupBuild
// bodies splits its children into runs of consecutive children with at most
// kGroupBuild bodies between them, each run inside one half of the cell
// along z (octants 0-3 or 4-7: a run across the middle, e.g. octants 3 and
// 4, would join diagonal neighbours into a box as large as the cell); a
// child with more starts its own groups;
// a leaf with more (guard depth) is cut into chunks; a root with at most
// kGroupBuild bodies is one group.  The groups partition the bodies into
// key-contiguous ranges that each lie inside one cell.  Cells are taken in
// breadth-first order, so the groups of large shallow cells (the sparse
// outskirts, whose walks are the longest) come first and the walk's dynamic
// scheduling starts them early.  Pass 1 counts per cell (cnt, indexed by
// breadth-first position j, cnt[nnodes] = 0 for the scan), pass 2 writes the
// ranges from the scanned offsets.
template <bool kEmit>
__global__ void group_kernel(int64_t nnodes, const uint32_t* __restrict__ bfs2pre,
                             const int4* __restrict__ link, const int32_t* __restrict__ nchild,
                             const uint64_t* __restrict__ hs, const uint64_t* __restrict__ klo,
                             const uint32_t* __restrict__ perm,
                             int32_t* __restrict__ cnt, const int32_t* __restrict__ off,
                             int2* __restrict__ out, int64_t cap, const int32_t* status) {
  if (sort_failed(status)) return;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j <= nnodes;
       j += (int64_t)gridDim.x * blockDim.x) {
    if (j == nnodes) {
      if (!kEmit) cnt[j] = 0;
      continue;
    }
    const int64_t k = bfs2pre[j];
    const int4 lk = link[k];
    const int ck = lk.z - lk.y;
    int r = 0;
    auto put = [&](int b0, int b1) {
      if (kEmit && off[j] + r < cap) out[off[j] + r] = make_int2(b0, b1);
      ++r;
    };
    if (ck <= kGroupBuild) {
      if (k == 0) put(lk.y, lk.z);
    } else if (lk.w & kMetaLeaf) {
      for (int b = lk.y; b < lk.z; b += kGroupBuild) put(b, min(b + kGroupBuild, lk.z));
    } else {
      int c = (int)k + 1, rb = -1, re = -1, ob = 0;
      const int nc = nchild[k];
      const int d = lk.w & kMetaDepth;
      for (int i = 0; i < nc && c < nnodes; ++i) {
        const int4 lc = link[c];
        const int cc = lc.z - lc.y;
        // the child's octant: digit d of its first body's descent key
        const int oc = d < 21 ? (int)((hs[lc.y] >> (60 - 3 * d)) & 7)
                              : (int)((klo[perm[lc.y]] >> (54 - 3 * (d - 21))) & 7);
        if (cc > kGroupBuild) {
          if (rb >= 0) put(rb, re);
          rb = -1;
        } else if (rb >= 0 && (ob >> 2) == (oc >> 2) && re - rb + cc <= kGroupBuild) {
          re = lc.z;
        } else {
          if (rb >= 0) put(rb, re);
          rb = lc.y;
          re = lc.z;
          ob = oc;
        }
        c = lc.x;
      }
      if (rb >= 0) put(rb, re);
    }
    if (!kEmit) cnt[j] = r;
  }
}

}  // namespace

// Builds the tree for the current positions.  One host synchronisation reads
// the node count (and the status word).
int bh_build(phys_ctx* c, const phys_params* p, bool need_f32, BhTree* t, bool need_group,
             bool full_com) {
  const int64_t n = c->n;
  const bool exact = p->precision == PHYS_F64_EXACT;
  uint64_t* khi = nullptr;
  PHYS_TRY(ws_alloc(c, WS_KEYS_HI, n, &khi));
  uint64_t* klo = nullptr;
  PHYS_TRY(ws_alloc(c, WS_KEYS_LO, n, &klo));
  uint32_t* idx = nullptr;
  PHYS_TRY(ws_alloc(c, WS_IDX, n, &idx));
  uint64_t* khi_alt = nullptr;
  PHYS_TRY(ws_alloc(c, WS_KEYS_HI_ALT, n, &khi_alt));
  uint32_t* idx_alt = nullptr;
  PHYS_TRY(ws_alloc(c, WS_IDX_ALT, n, &idx_alt));
  uint64_t* lo_s = nullptr;
  PHYS_TRY(ws_alloc(c, WS_ENS7, n, &lo_s));
  double4* body64 = nullptr;
  PHYS_TRY(ws_alloc(c, WS_BODY_PM, n, &body64));
  float4* body_hi = nullptr;
  float4* body_lo = nullptr;
  Body32x2* body2 = nullptr;
  if (need_f32) {
    PHYS_TRY(ws_alloc(c, WS_BODY_HI, n, &body_hi));
    PHYS_TRY(ws_alloc(c, WS_BODY_LO, n, &body_lo));
    PHYS_TRY(ws_alloc(c, WS_ENS6, n, &body2));
  }
  int32_t* L = nullptr;
  PHYS_TRY(ws_alloc(c, WS_LCP, n + 1, &L));
  int32_t* cnt = nullptr;
  PHYS_TRY(ws_alloc(c, WS_NCOUNT, n + 1, &cnt));
  int32_t* first = nullptr;
  PHYS_TRY(ws_alloc(c, WS_NFIRST, n + 1, &first));
  if (!c->d_partials || c->partials_cap < 7 * kBboxGrid) {
    if (c->d_partials) cudaFree(c->d_partials);
    c->d_partials = nullptr;
    PHYS_CUDA(c, cudaMalloc(&c->d_partials, sizeof(double) * 8 * kBboxGrid));
    c->partials_cap = 8 * kBboxGrid;
  }

  PHYS_CUDA(c, cudaEventRecord(c->ev[2], c->stream));
  PHYS_LAUNCH(c, bbox_partial_kernel, kBboxGrid, kBlock, 0, n, c->x, c->y, c->z, c->m,
              c->d_partials, c->d_status);
  PHYS_LAUNCH(c, bbox_final_kernel, 1, 32, 0, kBboxGrid, c->d_partials, p->theta, c->d_hdr,
              c->d_status);
  PHYS_CUDA(c, cudaEventRecord(c->ev[3], c->stream));
  double4* rec = nullptr;
  PHYS_TRY(ws_alloc(c, WS_BODY_IN, n, &rec));
  PHYS_LAUNCH(c, keys_kernel, grid_for(n), kBlock, 0, n, c->x, c->y, c->z, c->m, c->d_hdr, khi,
              klo, idx, rec);
  PHYS_CUDA(c, cudaEventRecord(c->ev[4], c->stream));
  bool in_alt = false;
  PHYS_TRY(radix_sort_u64(c, khi, idx, khi_alt, idx_alt, n, 0, 64, &in_alt));
  uint64_t* hs = in_alt ? khi_alt : khi;
  uint32_t* perm = in_alt ? idx_alt : idx;
  uint32_t* spare = in_alt ? idx : idx_alt;
  PHYS_LAUNCH(c, run_fixup_kernel, grid_for(n), kBlock, 0, n, hs, perm, klo, spare, c->d_status);
  PHYS_LAUNCH(c, gather_sorted_kernel, grid_for(n), kBlock, 0, n, perm, klo, rec, lo_s, body64,
              body_hi, body_lo, body2, c->d_status);
  PHYS_CUDA(c, cudaEventRecord(c->ev[5], c->stream));
  PHYS_LAUNCH(c, lcp_count_kernel, grid_for(n + 1), kBlock, 0, n, hs, lo_s, c->d_hdr, L, cnt);
  // bucket leaves: count only the cells that survive (no full tree)
  const bool pruned = p->leaf_cap > 1;
  int32_t* emax = nullptr;
  if (pruned) {
    PHYS_TRY(ws_alloc(c, WS_NEWID, n + 1, &emax));
    PHYS_LAUNCH(c, prune_count_kernel, grid_for(n + 1), kBlock, 0, n, L, c->d_hdr, p->leaf_cap,
                cnt, emax);
  }
  PHYS_TRY(scan_exclusive_i32(c, cnt, first, n + 1));
  // node count, header and status word back to the host: a key sort that
  // gave up a bounded wait ends the evaluation here, before any kernel
  // builds on its order (the kernels between the sort and this point
  // checked the flag themselves)
  int32_t* hsm = c->h_small;
  PHYS_CUDA(c, cudaMemcpyAsync(hsm, first + n, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  PHYS_CUDA(c, cudaMemcpyAsync(hsm + 1, &c->d_hdr->dstar, sizeof(int32_t), cudaMemcpyDeviceToHost,
                               c->stream));
  PHYS_CUDA(c, cudaMemcpyAsync(hsm + 2, c->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost,
                               c->stream));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  if (hsm[2] & kStatTimeout)
    return fail(c, PHYS_ERR_TIMEOUT, "radix sort of the descent keys: a bounded wait timed out");
  const int64_t nnodes = hsm[0];
  const int dstar = hsm[1];
  if (nnodes < 1 || nnodes > (int64_t)n * (kMaxLevels + 1))
    return fail(c, PHYS_ERR_CUDA, "tree build produced %lld nodes for %lld bodies",
                (long long)nnodes, (long long)n);
  int4* link = nullptr;
  PHYS_TRY(ws_alloc(c, WS_LINK, nnodes, &link));
  int32_t* parent = nullptr;
  PHYS_TRY(ws_alloc(c, WS_PARENT, nnodes + 1, &parent));
  int32_t* nchild = nullptr;
  PHYS_TRY(ws_alloc(c, WS_ARRIVE, 2 * (nnodes + 1), &nchild));
  int32_t* arrive = nchild + (nnodes + 1);
  if (pruned) {
    PHYS_LAUNCH(c, emit_pruned_kernel, grid_for(nnodes), kBlock, 0, n, hs, lo_s, L, cnt, first,
                c->d_hdr, link);
  } else {
    PHYS_LAUNCH(c, emit_nodes_kernel, grid_for(n), kBlock, 0, n, hs, lo_s, L, cnt, first,
                c->d_hdr, link);
  }
  PHYS_LAUNCH(c, children_kernel, grid_for(nnodes), kBlock, 0, nnodes, link, parent, nchild,
              c->d_status);
  double4* mc = nullptr;
  PHYS_TRY(ws_alloc(c, WS_NODE_S, nnodes, &mc));
  if (exact) {
    int32_t* ncnt = nullptr;
    PHYS_TRY(ws_alloc(c, WS_KEEP, nnodes + 1, &ncnt));
    int32_t* eoff = nullptr;
    PHYS_TRY(ws_alloc(c, WS_EOFF, nnodes + 1, &eoff));
    PHYS_LAUNCH(c, node_count_kernel, grid_for(nnodes + 1), kBlock, 0, nnodes, link, ncnt);
    PHYS_TRY(scan_exclusive_i32(c, ncnt, eoff, nnodes + 1));
    PHYS_CUDA(c, cudaMemcpyAsync(hsm, eoff + nnodes, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                 c->stream));
    PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
    const int64_t total = (uint32_t)hsm[0];
    if (total <= 0 || total >= (int64_t(1) << 31))
      return fail(c, PHYS_ERR_ARG, "exact centre of mass needs < 2^31 (cell, body) pairs");
    uint64_t* ent = nullptr;
    PHYS_TRY(ws_alloc(c, WS_ENTRIES, total, &ent));
    uint64_t* ent_alt = nullptr;
    PHYS_TRY(ws_alloc(c, WS_ENTRIES_ALT, total, &ent_alt));
    PHYS_LAUNCH(c, expand_kernel, grid_for(total), kBlock, 0, total, nnodes, eoff, link, perm, ent);
    int bits_b = 1, bits_n = 1;
    while ((int64_t(1) << bits_b) < n) ++bits_b;
    while ((int64_t(1) << bits_n) < nnodes) ++bits_n;
    bool alt1 = false, alt2 = false;
    PHYS_TRY(radix_sort_u64(c, ent, nullptr, ent_alt, nullptr, total, 0, bits_b, &alt1));
    uint64_t* e1 = alt1 ? ent_alt : ent;
    uint64_t* e1_alt = alt1 ? ent : ent_alt;
    PHYS_TRY(radix_sort_u64(c, e1, nullptr, e1_alt, nullptr, total, 32, 32 + bits_n, &alt2));
    uint64_t* es = alt2 ? e1_alt : e1;
    double4* eb = nullptr;
    PHYS_TRY(ws_alloc(c, WS_ENTRY_BODY, total, &eb));
    PHYS_LAUNCH(c, gather_entries_kernel, grid_for(total), kBlock, 0, total, es, c->x, c->y,
                c->z, c->m, link, c->d_hdr, full_com ? 0 : 1, eb, c->d_status);
    // the node counts are consumed by the scan: their array takes the list
    // of long cells, its count in the last slot
    int32_t* longs = ncnt;
    PHYS_CUDA(c, cudaMemsetAsync(longs + nnodes, 0, sizeof(int32_t), c->stream));
    PHYS_LAUNCH(c, com_recurrence_kernel, grid_for(nnodes, 128, 1 << 30), 128, 0, nnodes, eoff, eb,
                mc, link, c->d_hdr, full_com ? 0 : 1, longs, c->d_status);
    PHYS_LAUNCH(c, com_recurrence_long_kernel, 148 * 4, 32 * kLongWarps, 0, nnodes, eoff, eb, mc,
                longs, c->d_status);
  } else {
    PHYS_CUDA(c, cudaMemsetAsync(arrive, 0, sizeof(int32_t) * (nnodes + 1), c->stream));
    PHYS_LAUNCH(c, com_upward_kernel, grid_for(nnodes), kBlock, 0, nnodes, link, parent, nchild,
                arrive, body64, mc, c->d_status);
  }
  double4* rec64 = nullptr;
  Rec32* w32 = nullptr;
  Rec64* w64 = nullptr;
  Rec32x2* w32x2 = nullptr;
  if (exact) PHYS_TRY(ws_alloc(c, WS_NODE_PM, nnodes, &rec64));
#ifndef WALK_PAIRED
#define WALK_PAIRED 1
#endif
  if (need_f32 && WALK_PAIRED)
    PHYS_TRY(ws_alloc(c, WS_NODE_HI, nnodes, &w32x2));
  else if (need_f32)
    PHYS_TRY(ws_alloc(c, WS_NODE_HI, nnodes, &w32));
  else if (!exact && !need_group)
    PHYS_TRY(ws_alloc(c, WS_NODE_LO, nnodes, &w64));
  PHYS_LAUNCH(c, finalize_kernel, grid_for(nnodes), kBlock, 0, nnodes, link, mc, exact ? 0 : 1,
              p->leaf_cap, body64, c->d_hdr, rec64, w32, w64, w32x2);
  if (need_group) {
    // breadth-first records for the group walk
    uint64_t *dk = nullptr, *dk_alt = nullptr;
    uint32_t *dv = nullptr, *dv_alt = nullptr;
    int32_t* pre2bfs = nullptr;
    GNode* g = nullptr;
    PHYS_TRY(ws_alloc(c, WS_ENTRIES, nnodes, &dk));
    PHYS_TRY(ws_alloc(c, WS_ENTRIES_ALT, nnodes, &dk_alt));
    PHYS_TRY(ws_alloc(c, WS_KEEP, nnodes, &dv));
    PHYS_TRY(ws_alloc(c, WS_NEWID, nnodes, &dv_alt));
    PHYS_TRY(ws_alloc(c, WS_EOFF, nnodes + 1, &pre2bfs));
    PHYS_TRY(ws_alloc(c, WS_ENS5, nnodes, &g));
    PHYS_LAUNCH(c, depth_key_kernel, grid_for(nnodes), kBlock, 0, nnodes, link, dk, dv);
    bool alt = false;
    PHYS_TRY(radix_sort_u64(c, dk, dv, dk_alt, dv_alt, nnodes, 0, 8, &alt));
    const uint32_t* bfs2pre = alt ? dv_alt : dv;
    PHYS_LAUNCH(c, invert_kernel, grid_for(nnodes), kBlock, 0, nnodes, bfs2pre, pre2bfs,
                c->d_status);
    PHYS_LAUNCH(c, gnode_kernel, grid_for(nnodes), kBlock, 0, nnodes, bfs2pre, pre2bfs, link, mc,
                nchild, p->leaf_cap, body64, c->d_hdr, g, c->d_status);
    t->gnode = g;
    int32_t *gcnt = nullptr, *goff = nullptr, *gctr = nullptr;
    int2* groups = nullptr;
    PHYS_TRY(ws_alloc(c, WS_NCOUNT, nnodes + 1, &gcnt));
    PHYS_TRY(ws_alloc(c, WS_GROUP_OFF, nnodes + 1, &goff));
    PHYS_TRY(ws_alloc(c, WS_GROUPS, 2 * n, &groups));  // groups, then re-queued subgroups
    PHYS_TRY(ws_alloc(c, WS_GROUP_CTR, 8, &gctr));
    PHYS_LAUNCH(c, group_kernel<false>, grid_for(nnodes + 1), kBlock, 0, nnodes, bfs2pre, link,
                nchild, hs, klo, perm, gcnt, goff, groups, n, c->d_status);
    PHYS_TRY(scan_exclusive_i32(c, gcnt, goff, nnodes + 1));
    PHYS_LAUNCH(c, group_kernel<true>, grid_for(nnodes + 1), kBlock, 0, nnodes, bfs2pre, link,
                nchild, hs, klo, perm, gcnt, goff, groups, n, c->d_status);
    t->groups = groups;
    t->ngroups = goff + nnodes;
    t->group_ctr = gctr;
  }
  t->n = n;
  t->nnodes = nnodes;
  t->leaf_cap = p->leaf_cap;
  t->link = link;
  t->rec64 = rec64;
  t->w32 = w32;
  t->w64 = w64;
  t->w32x2 = w32x2;
  t->body2 = body2;
  t->mc = mc;
  t->perm = perm;
  t->body64 = body64;
  t->body_hi = body_hi;
  t->body_lo = body_lo;
  t->hdr = c->d_hdr;
  t->keys_hi_sorted = hs;
  t->keys_lo = klo;
  c->tm.nodes = nnodes;
  c->tm.max_depth = dstar;
  return PHYS_OK;
}

int bh_eval(phys_ctx* c, const phys_params* p, bool want_force, double* ox, double* oy,
            double* oz) {
  BhTree t;
  const bool group = (p->flags & PHYS_FLAG_GROUP_WALK) != 0;
  // the exact form's forces need no centre of mass of cells no target can
  // take as a monopole
  PHYS_TRY(bh_build(c, p, p->precision == PHYS_F32C && !group, &t, group, false));
  c->share_perm = t.perm;  // sorted position -> body, for a target share
  return bh_walk(c, p, t, want_force, ox, oy, oz);
}

int bh_export(phys_ctx* c, const phys_params* p, int64_t cap, int64_t* nnodes, int32_t* depth,
              int64_t* count, double* mass, double* com, int64_t* leaf_body, int64_t* body_leaf,
              uint64_t* keys_hi, uint64_t* keys_lo, int64_t* perm_out, double* root4) {
  BhTree t;
  PHYS_TRY(bh_build(c, p, false, &t));
  const int64_t n = c->n, nn = t.nnodes;
  std::vector<int4> link(nn);
  std::vector<double4> mc(nn);
  std::vector<uint32_t> perm(n);
  TreeHeader hdr;
  PHYS_CUDA(c, cudaMemcpyAsync(link.data(), t.link, sizeof(int4) * nn, cudaMemcpyDeviceToHost,
                               c->stream));
  PHYS_CUDA(c, cudaMemcpyAsync(mc.data(), t.mc, sizeof(double4) * nn, cudaMemcpyDeviceToHost,
                               c->stream));
  PHYS_CUDA(c, cudaMemcpyAsync(perm.data(), t.perm, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost,
                               c->stream));
  PHYS_CUDA(c, cudaMemcpyAsync(&hdr, t.hdr, sizeof(TreeHeader), cudaMemcpyDeviceToHost, c->stream));
  std::vector<uint64_t> hs(keys_hi ? n : 0);
  if (keys_hi)
    PHYS_CUDA(c, cudaMemcpyAsync(hs.data(), t.keys_hi_sorted, sizeof(uint64_t) * n,
                                 cudaMemcpyDeviceToHost, c->stream));
  if (keys_lo)
    PHYS_CUDA(c, cudaMemcpyAsync(keys_lo, t.keys_lo, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost,
                                 c->stream));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  if (keys_hi)  // the sort reordered hi; undo it through the permutation
    for (int64_t q = 0; q < n; ++q) keys_hi[perm[q]] = hs[q];
  if (nnodes) *nnodes = nn;
  if (root4) {
    root4[0] = hdr.center[0];
    root4[1] = hdr.center[1];
    root4[2] = hdr.center[2];
    root4[3] = hdr.half;
  }
  if (perm_out)
    for (int64_t q = 0; q < n; ++q) perm_out[q] = perm[q];
  if (body_leaf)
    for (int64_t i = 0; i < n; ++i) body_leaf[i] = -1;
  for (int64_t k = 0; k < nn; ++k) {
    const int4 lk = link[k];
    const bool leaf = lk.w & kMetaLeaf;
    if (k < cap) {
      if (depth) depth[k] = lk.w & kMetaDepth;
      if (count) count[k] = lk.z - lk.y;
      if (mass) mass[k] = mc[k].w;
      if (com) {
        com[3 * k] = mc[k].x;
        com[3 * k + 1] = mc[k].y;
        com[3 * k + 2] = mc[k].z;
      }
      if (leaf_body) {
        int64_t lb = -1;
        if (leaf) {
          if (lk.z - lk.y == 1)
            lb = perm[lk.y];
          else if ((lk.w & kMetaGuard) && t.leaf_cap == 1)
            lb = perm[lk.z - 1];
          else
            lb = -2;  // bucket leaf holding several bodies
        }
        leaf_body[k] = lb;
      }
    }
    if (leaf && body_leaf)
      for (int q = lk.y; q < lk.z; ++q) body_leaf[perm[q]] = k;
  }
  return PHYS_OK;
}

int debug_divide(phys_ctx* c, int64_t n, const double* a, const double* b, double* q) {
  if (n <= 0) return PHYS_OK;
  int st = PHYS_OK;
  double* d = (double*)ws_get(c, WS_ADJ2, sizeof(double) * 3 * n, &st);
  if (st) return st;
  const size_t bytes = sizeof(double) * (size_t)n;
  PHYS_CUDA(c, cudaMemcpyAsync(d, a, bytes, cudaMemcpyHostToDevice, c->stream));
  PHYS_CUDA(c, cudaMemcpyAsync(d + n, b, bytes, cudaMemcpyHostToDevice, c->stream));
  PHYS_LAUNCH(c, debug_divide_kernel, grid_for(n), kBlock, 0, n, d, d + n, d + 2 * n);
  PHYS_CUDA(c, cudaMemcpyAsync(q, d + 2 * n, bytes, cudaMemcpyDeviceToHost, c->stream));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  return PHYS_OK;
}

}  // namespace phys
