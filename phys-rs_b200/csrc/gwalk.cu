// Group walk (PHYS_FLAG_GROUP_WALK): Barnes-Hut forces for a group of up to
// 64 key-adjacent bodies per warp from one shared interaction list.
//
// The reference walks the octree once per body (gravity_tree.rs:171-209,
// criterion (2h)^2 < theta^2 d^2 at :194).  Here the bodies are split into
// groups that each lie inside one cell (the children of a cell with more
// than 64 bodies, consecutive small siblings packed together; built with the
// tree), a warp takes groups from a global counter, bounds each with a box,
// and walks the tree once for all its bodies:
//   - the warp pops up to 32 cells from a stack in shared memory, one per
//     lane, and tests each against the box: a cell is a monopole only when
//     (2h)^2 < theta^2 d_min^2, d_min the distance from its centre of mass to
//     the nearest point of the box (d_min <= d for every target, so the
//     per-body criterion holds for each of them);
//   - an opened cell pushes its children (contiguous in the breadth-first
//     record array); a one-body leaf, an accepted cell and every body of an
//     opened bucket leaf become entries of the interaction list, spread over
//     the lanes (each lane writes consecutive slots);
//   - the group's own bodies never enter the list: a cell whose bodies all
//     belong to the group is skipped, one that holds some of them is always
//     opened, and pairs inside the group are summed exactly in a separate
//     pass that skips i == j;
//   - a full list is evaluated by all targets at once: lane l reads the
//     entries as broadcast shared-memory loads and accumulates its two
//     targets.
// The list arithmetic is the per-body walk's: F64 = f64 FMA + rsqrt on
// absolute coordinates; F32C = f32 pair terms on double-float coordinates
// relative to the group's first body, r = (hi_j - hi_i) + (lo_j - lo_i), two
// list entries per packed f32x2 operation, partial sums folded into a
// (hi, lo) accumulator by two-sum every kGFlushPairs entry pairs.  The
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
#include <climits>

#include "bh.cuh"

#ifndef GWALK_FLUSH_PAIRS
#define GWALK_FLUSH_PAIRS 8
#endif

namespace phys {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kGWarps = 4;
constexpr int kGBlock = 32 * kGWarps;
constexpr int kGStack = 1024;   // node ids per warp
constexpr int kGList = 256;     // list entries per warp, 32 bytes each
constexpr int kGThrottle = kGStack - 8 - 7 * kMaxLevels;
constexpr int kGFlushPairs = GWALK_FLUSH_PAIRS;
constexpr int kGListLimit = 8192;  // first-pass list budget (a typical group lists ~3-4k)
constexpr int kGSplit = 4;         // bodies per re-queued subgroup
// per warp: stack | list | emission records (end, kind, a, olo, ohi per lane)
constexpr int kGListOff = kGStack * 4;
constexpr int kGRecOff = kGListOff + kGList * 32;
constexpr int kGSmemWarp = kGRecOff + 5 * 32 * 4;
constexpr int kGSmem = kGWarps * kGSmemWarp;
static_assert(kGroupMax == 64, "two targets per lane");
static_assert(kGThrottle >= 7 * 32 + 7, "stack too small for batched pops");
static_assert(kGThrottle + 7 * kMaxLevels + 1 <= kGStack, "stack bound");
static_assert(kGList % 4 == 0 && kGFlushPairs % 2 == 0, "list chunks of 4 entries");

__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

__device__ __forceinline__ double4 ldg_d4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  const double2 a = __ldg(q), b = __ldg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
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

// F32C list, structure of arrays (slot-consecutive writes hit distinct banks;
// the evaluation reads four entries per 16-byte load).
struct List32 {
  float *hx, *hy, *hz, *m, *lx, *ly, *lz;
};

// Forces on the bodies [base, gend).  Returns false, with nothing written,
// when the interaction list grows past `limit` entries.
template <bool kF32>
__device__ __forceinline__ bool group_forces(
    int lane, int base, int gend, int nnodes, int limit, int* stk, unsigned char* lbase, int* rec,
    const GNode* __restrict__ gn, const double4* __restrict__ body64,
    const uint32_t* __restrict__ perm, double G, double eps2, float theta2f, int want_force,
    double* __restrict__ ox, double* __restrict__ oy, double* __restrict__ oz,
    unsigned long long& ninter_out, bool& bad, int32_t* status) {
  const int nvalid = gend - base;
  const int ia = base + 2 * lane, ib = ia + 1;
  const bool va = ia < gend, vb = ib < gend;
  const double4 X0 = body64[base];
  const double4 ta = va ? body64[ia] : X0;
  const double4 tb = vb ? body64[ib] : X0;
  List32 L;
  {
    float* f = reinterpret_cast<float*>(lbase);
    L.hx = f;
    L.hy = f + kGList;
    L.hz = f + 2 * kGList;
    L.m = f + 3 * kGList;
    L.lx = f + 4 * kGList;
    L.ly = f + 5 * kGList;
    L.lz = f + 6 * kGList;
  }
  double4* lst64 = reinterpret_cast<double4*>(lbase);
  int* r_end = rec;
  int* r_kind = rec + 32;
  int* r_a = rec + 64;
  int* r_olo = rec + 96;
  int* r_ohi = rec + 128;

  // group box in f32, relative to X0 (idle lanes sit at X0, a group body)
  float cx, cy, cz, bx, by, bz;
  {
    const float ax_ = (float)(ta.x - X0.x), ay_ = (float)(ta.y - X0.y), az_ = (float)(ta.z - X0.z);
    const float bx_ = (float)(tb.x - X0.x), by_ = (float)(tb.y - X0.y), bz_ = (float)(tb.z - X0.z);
    const float mnx = warp_min(fminf(ax_, bx_)), mxx = warp_max(fmaxf(ax_, bx_));
    const float mny = warp_min(fminf(ay_, by_)), mxy = warp_max(fmaxf(ay_, by_));
    const float mnz = warp_min(fminf(az_, bz_)), mxz = warp_max(fmaxf(az_, bz_));
    cx = 0.5f * (mnx + mxx);
    cy = 0.5f * (mny + mxy);
    cz = 0.5f * (mnz + mxz);
    // widen by the rounding of the f32 coordinates (a few ulp of |c| + b)
    bx = 0.5f * (mxx - mnx);
    by = 0.5f * (mxy - mny);
    bz = 0.5f * (mxz - mnz);
    bx = bx * (1.0f + 1e-6f) + 1e-6f * (fabsf(cx) + bx);
    by = by * (1.0f + 1e-6f) + 1e-6f * (fabsf(cy) + by);
    bz = bz * (1.0f + 1e-6f) + 1e-6f * (fabsf(cz) + bz);
  }
  float x0hx, x0lx, x0hy, x0ly, x0hz, x0lz;
  split_df(X0.x, x0hx, x0lx);
  split_df(X0.y, x0hy, x0ly);
  split_df(X0.z, x0hz, x0lz);

  // F32C target state: negated double-float offsets from X0, duplicated for
  // packed operands (both halves = the same target)
  float2 nhxa, nhya, nhza, nlxa, nlya, nlza, nhxb, nhyb, nhzb, nlxb, nlyb, nlzb;
  {
    float h, l;
    split_df(ta.x - X0.x, h, l); nhxa = make_float2(-h, -h); nlxa = make_float2(-l, -l);
    split_df(ta.y - X0.y, h, l); nhya = make_float2(-h, -h); nlya = make_float2(-l, -l);
    split_df(ta.z - X0.z, h, l); nhza = make_float2(-h, -h); nlza = make_float2(-l, -l);
    split_df(tb.x - X0.x, h, l); nhxb = make_float2(-h, -h); nlxb = make_float2(-l, -l);
    split_df(tb.y - X0.y, h, l); nhyb = make_float2(-h, -h); nlyb = make_float2(-l, -l);
    split_df(tb.z - X0.z, h, l); nhzb = make_float2(-h, -h); nlzb = make_float2(-l, -l);
  }
  const float eps2f = (float)eps2;
  const float2 e2 = make_float2(eps2f, eps2f);
  const float2 z2 = make_float2(0.f, 0.f);
  float2 pxa = z2, pya = z2, pza = z2, pxb = z2, pyb = z2, pzb = z2;  // partials (entry halves)
  float2 Hx = z2, Hy = z2, Hz = z2, Lx = z2, Ly = z2, Lz = z2;        // (target a, target b)
  double ax = 0, ay = 0, az = 0, bxs = 0, bys = 0, bzs = 0;          // F64 sums
  unsigned long long ninter = (unsigned long long)nvalid * (unsigned long long)(nvalid - 1);
  int listed = 0;  // entries emitted so far

  auto flush = [&]() {
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
    pxa = pya = pza = pxb = pyb = pzb = z2;
  };

  // One F32C entry pair against one target; skip_e / skip_f zero the halves
  // that are the target itself (in-group pass).
  auto term32 = [&](float2 hx, float2 hy, float2 hz, float2 mm, float2 lx, float2 ly, float2 lz,
                    float2 nhx, float2 nhy, float2 nhz, float2 nlx, float2 nly, float2 nlz,
                    bool skip_e, bool skip_f, float2& px, float2& py, float2& pz) {
    const float2 rx = __fadd2_rn(__fadd2_rn(hx, nhx), __fadd2_rn(lx, nlx));
    const float2 ry = __fadd2_rn(__fadd2_rn(hy, nhy), __fadd2_rn(ly, nly));
    const float2 rz = __fadd2_rn(__fadd2_rn(hz, nhz), __fadd2_rn(lz, nlz));
    const float2 r2 = __ffma2_rn(rx, rx, __ffma2_rn(ry, ry, __ffma2_rn(rz, rz, e2)));
    const float2 inv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
    float2 w = __fmul2_rn(mm, __fmul2_rn(__fmul2_rn(inv, inv), inv));
    if (skip_e) w.x = 0.f;
    if (skip_f) w.y = 0.f;
    px = __ffma2_rn(rx, w, px);
    py = __ffma2_rn(ry, w, py);
    pz = __ffma2_rn(rz, w, pz);
  };

  // F64 entry against one target
  auto term64 = [&](double4 s, double4 t, double& sx, double& sy, double& sz) {
    const double rx = s.x - t.x, ry = s.y - t.y, rz = s.z - t.z;
    const double inv = rsqrt(fma(rx, rx, fma(ry, ry, fma(rz, rz, eps2))));
    const double w = s.w * (inv * inv * inv);
    sx = fma(rx, w, sx);
    sy = fma(ry, w, sy);
    sz = fma(rz, w, sz);
  };

  // Writes list slot `slot` from an absolute position + mass.
  auto put = [&](int slot, double4 src) {
    if (kF32) {
      float h, l;
      split_df(src.x - X0.x, h, l);
      L.hx[slot] = h;
      L.lx[slot] = l;
      split_df(src.y - X0.y, h, l);
      L.hy[slot] = h;
      L.ly[slot] = l;
      split_df(src.z - X0.z, h, l);
      L.hz[slot] = h;
      L.lz[slot] = l;
      L.m[slot] = (float)src.w;
    } else {
      lst64[slot] = src;
    }
  };

  // Evaluates list slots [0, nl) for both targets.
  auto eval = [&](int nl, bool self) {
    if (kF32) {
      // pad to a multiple of 4 with massless entries far away
      const int np = (nl + 3) & ~3;
      if (lane < np - nl) {
        const int s = nl + lane;
        L.hx[s] = L.hy[s] = L.hz[s] = 1e15f;
        L.m[s] = L.lx[s] = L.ly[s] = L.lz[s] = 0.f;
      }
      __syncwarp();
      const int nq = np >> 2;
      const float4* HX = reinterpret_cast<const float4*>(L.hx);
      const float4* HY = reinterpret_cast<const float4*>(L.hy);
      const float4* HZ = reinterpret_cast<const float4*>(L.hz);
      const float4* MM = reinterpret_cast<const float4*>(L.m);
      const float4* LX = reinterpret_cast<const float4*>(L.lx);
      const float4* LY = reinterpret_cast<const float4*>(L.ly);
      const float4* LZ = reinterpret_cast<const float4*>(L.lz);
      constexpr int kQ = kGFlushPairs / 2;  // 4-entry chunks per flush
      const int myq = self ? (lane >> 1) : -1;
      for (int q0 = 0; q0 < nq; q0 += kQ) {
        const int q1 = min(q0 + kQ, nq);
#pragma unroll 2
        for (int q = q0; q < q1; ++q) {
          const float4 hx = HX[q], hy = HY[q], hz = HZ[q], mm = MM[q];
          const float4 lx = LX[q], ly = LY[q], lz = LZ[q];
          // target a is slot 2*lane, target b slot 2*lane + 1: chunk lane/2,
          // pair (lane & 1)
          const bool m0 = q == myq && !(lane & 1);
          const bool m1 = q == myq && (lane & 1);
          term32(lo2(hx), lo2(hy), lo2(hz), lo2(mm), lo2(lx), lo2(ly), lo2(lz), nhxa, nhya, nhza,
                 nlxa, nlya, nlza, m0, false, pxa, pya, pza);
          term32(lo2(hx), lo2(hy), lo2(hz), lo2(mm), lo2(lx), lo2(ly), lo2(lz), nhxb, nhyb, nhzb,
                 nlxb, nlyb, nlzb, false, m0, pxb, pyb, pzb);
          term32(hi2(hx), hi2(hy), hi2(hz), hi2(mm), hi2(lx), hi2(ly), hi2(lz), nhxa, nhya, nhza,
                 nlxa, nlya, nlza, m1, false, pxa, pya, pza);
          term32(hi2(hx), hi2(hy), hi2(hz), hi2(mm), hi2(lx), hi2(ly), hi2(lz), nhxb, nhyb, nhzb,
                 nlxb, nlyb, nlzb, false, m1, pxb, pyb, pzb);
        }
        flush();
      }
    } else {
      __syncwarp();
#pragma unroll 2
      for (int e = 0; e < nl; ++e) {
        const double4 s = lst64[e];
        if (!(self && e == 2 * lane)) term64(s, ta, ax, ay, az);
        if (!(self && e == 2 * lane + 1)) term64(s, tb, bxs, bys, bzs);
      }
    }
    __syncwarp();
  };

  // ---- pairs inside the group (exact, i != j) ----
  if (va) put(2 * lane, ta);
  if (vb) put(2 * lane + 1, tb);
  eval(nvalid, true);

  // ---- tree walk ----
  int ssize = 1, lsize = 0;
  long long pops = 0;
  if (lane == 0) stk[0] = 0;
  __syncwarp();
  while (ssize > 0) {
    if (listed > limit) return false;
    const int k = ssize <= kGThrottle - 7 ? min(min(32, ssize), (kGThrottle - ssize) / 7) : 1;
    const int nd = lane < k ? stk[ssize - 1 - lane] : -1;
    ssize -= k;
    pops += k;
    __syncwarp();
    int npush = 0, cfirst = 0, nent = 0, kind = 0, a = 0, olo = 0, ohi = 0;
    bool malformed = pops > nnodes;
    if (nd >= 0) {
      const GNode* g = gn + nd;
      const int4 l = __ldg(&g->l);
      const int type = l.y & 3, cnt = l.y >> 2;
      const bool inside = l.z >= base && l.w <= gend;  // only group bodies
      if (type == kGSkip || inside) {
      } else if (type == kGSingle) {
        if (l.x < base || l.x >= gend) {
          nent = 1;
          kind = 1;
          a = nd;
        }
      } else {
        const bool overlap = l.z < gend && l.w > base;
        bool acc = false;
        if (!overlap) {
          const float4 h = __ldg(&g->hi), lo = __ldg(&g->lo);
          const float rx = (h.x - x0hx) + (lo.x - x0lx);
          const float ry = (h.y - x0hy) + (lo.y - x0ly);
          const float rz = (h.z - x0hz) + (lo.z - x0lz);
          const float dx = fmaxf(fabsf(rx - cx) - bx, 0.f);
          const float dy = fmaxf(fabsf(ry - cy) - by, 0.f);
          const float dz = fmaxf(fabsf(rz - cz) - bz, 0.f);
          const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
          acc = lo.w < theta2f * d2 * (1.0f - 1e-5f);
        }
        if (acc) {
          nent = 1;
          kind = 1;
          a = nd;
        } else if (type == kGInternal) {
          if (l.x <= nd || cnt < 1 || cnt > 8 || l.x + cnt > nnodes) {
            malformed = true;
          } else {
            npush = cnt;
            cfirst = l.x;
          }
        } else {  // bucket leaf opened: its bodies outside the group
          a = l.z;
          olo = max(l.z, base);
          ohi = min(l.w, gend);
          nent = (l.w - l.z) - max(ohi - olo, 0);
          kind = 2;
        }
      }
    }
    const int pin = warp_incl_scan(npush, lane);
    const int ptot = __shfl_sync(kFull, pin, 31);
    if (__any_sync(kFull, malformed) || ssize + ptot > kGStack) {
      bad = true;
      break;
    }
    for (int c = 0; c < npush; ++c) stk[ssize + pin - npush + c] = cfirst + c;
    ssize += ptot;
    __syncwarp();  // pushes visible to the next round's pops
    const int ein = warp_incl_scan(nent, lane);
    const int etot = __shfl_sync(kFull, ein, 31);
    listed += etot;
    if (etot > 0) {
      r_end[lane] = ein;
      r_kind[lane] = kind;
      r_a[lane] = a;
      r_olo[lane] = olo;
      r_ohi[lane] = ohi;
      __syncwarp();
      for (int done = 0; done < etot;) {
        if (lsize == kGList) {
          eval(lsize, false);
          ninter += (unsigned long long)lsize * (unsigned long long)nvalid;
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
          double4 src;
          if (r_kind[lo] == 1) {
            src = ldg_d4(&gn[r_a[lo]].c64);
          } else {
            int q = r_a[lo] + j;
            const int ol = r_olo[lo], oh = r_ohi[lo];
            if (ol < oh && q >= ol) q += oh - ol;
            src = ldg_d4(&body64[q]);
          }
          put(lsize + (e - done), src);
        }
        lsize += take;
        done += take;
      }
      __syncwarp();
    }
  }
  if (bad) return true;
  if (lsize > 0) {
    eval(lsize, false);
    ninter += (unsigned long long)lsize * (unsigned long long)nvalid;
  }
  ninter_out += ninter;

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
    if (va) out(ia, (double)Hx.x + (double)Lx.x, (double)Hy.x + (double)Ly.x,
                (double)Hz.x + (double)Lz.x);
    if (vb) out(ib, (double)Hx.y + (double)Lx.y, (double)Hy.y + (double)Ly.y,
                (double)Hz.y + (double)Lz.y);
  } else {
    if (va) out(ia, ax, ay, az);
    if (vb) out(ib, bxs, bys, bzs);
  }
  return true;
}

// Persistent warps: each takes the next group from the counter until none
// is left.  First pass (retry != nullptr): a group whose list passes
// kGListLimit entries is abandoned and re-queued as subgroups of kGSplit
// consecutive bodies (a group whose box reaches a much denser region; its
// small subgroups have far shorter lists).  Second pass: the re-queued
// subgroups, without a limit.
template <bool kF32>
__global__ void __launch_bounds__(kGBlock)
gwalk_kernel(int n, int nnodes, const GNode* __restrict__ gn, const int2* __restrict__ groups,
             const int32_t* __restrict__ ngroups_p, int32_t* __restrict__ ctr,
             int2* __restrict__ retry, int32_t* __restrict__ nretry,
             const double4* __restrict__ body64, const uint32_t* __restrict__ perm, double G,
             double eps2, float theta2f, int want_force, double* __restrict__ ox,
             double* __restrict__ oy, double* __restrict__ oz, unsigned long long* counter,
             int32_t* status) {
  extern __shared__ __align__(16) unsigned char gsm[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned char* ws = gsm + wid * kGSmemWarp;
  int* stk = reinterpret_cast<int*>(ws);
  int* rec = reinterpret_cast<int*>(ws + kGRecOff);
  const int ngroups = min(*ngroups_p, n);
  const int limit = retry ? kGListLimit : INT_MAX;
  unsigned long long ninter = 0;
  bool bad = false;
  for (;;) {
    int gi = 0;
    if (lane == 0) gi = atomicAdd(ctr, 1);
    gi = __shfl_sync(kFull, gi, 0);
    if (gi >= ngroups) break;
    const int2 gr = groups[gi];
    if (gr.x < 0 || gr.y > n || gr.y - gr.x < 1 || gr.y - gr.x > kGroupMax) {
      bad = true;
      break;
    }
    const bool done =
        group_forces<kF32>(lane, gr.x, gr.y, nnodes, limit, stk, ws + kGListOff, rec, gn, body64,
                           perm, G, eps2, theta2f, want_force, ox, oy, oz, ninter, bad, status);
    if (bad) break;
    if (!done && lane == 0) {
      // subgroups are disjoint and non-empty: at most n of them in all
      const int nsub = (gr.y - gr.x + kGSplit - 1) / kGSplit;
      const int at = atomicAdd(nretry, nsub);
      for (int k = 0; k < nsub; ++k) {
        if (at + k < n) {
          retry[at + k] = make_int2(gr.x + k * kGSplit, min(gr.x + (k + 1) * kGSplit, gr.y));
        } else {
          bad = true;
        }
      }
    }
    __syncwarp();
  }
  if (lane == 0) {
    if (bad) atomicOr(status, kStatOverflow);
    if (ninter) atomicAdd(counter, ninter);  // the same on every lane
  }
}

template <bool kF32>
int launch(phys_ctx* c, const phys_params* p, const BhTree& t, bool want_force, double* ox,
           double* oy, double* oz) {
  static int blocks_per_sm = 0;  // per process; the kernel and its resources are fixed
  if (!blocks_per_sm) {
    PHYS_CUDA(c, cudaFuncSetAttribute(gwalk_kernel<kF32>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem));
    int b = 0;
    PHYS_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, gwalk_kernel<kF32>, kGBlock,
                                                               kGSmem));
    blocks_per_sm = b > 0 ? b : 1;
  }
  int sms = 0;
  PHYS_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  const int64_t max_blocks = ceil_div(t.n, (int64_t)kGWarps);
  const int grid = (int)min64((int64_t)sms * blocks_per_sm, max_blocks);
  // group_ctr: [0] first-pass counter, [1] second-pass counter, [2] re-queued count
  PHYS_CUDA(c, cudaMemsetAsync(t.group_ctr, 0, 3 * sizeof(int32_t), c->stream));
  const double eps2 = p->eps * p->eps;
  const float theta2f = (float)(p->theta * p->theta);
  int2* retry = const_cast<int2*>(t.groups) + t.n;
  PHYS_LAUNCH(c, gwalk_kernel<kF32>, grid, kGBlock, kGSmem, (int)t.n, (int)t.nnodes, t.gnode,
              t.groups, t.ngroups, t.group_ctr, retry, t.group_ctr + 2, t.body64, t.perm, p->G,
              eps2, theta2f, (int)want_force, ox, oy, oz, c->d_counter, c->d_status);
  PHYS_LAUNCH(c, gwalk_kernel<kF32>, grid, kGBlock, kGSmem, (int)t.n, (int)t.nnodes, t.gnode,
              retry, t.group_ctr + 2, t.group_ctr + 1, (int2*)nullptr, (int32_t*)nullptr,
              t.body64, t.perm, p->G, eps2, theta2f, (int)want_force, ox, oy, oz, c->d_counter,
              c->d_status);
  return PHYS_OK;
}

}  // namespace

int bh_group_walk(phys_ctx* c, const phys_params* p, const BhTree& t, bool want_force,
                  double* ox, double* oy, double* oz) {
  if (!t.gnode || !t.groups) return fail(c, PHYS_ERR_STATE, "group walk without group records");
  if (t.n > INT32_MAX - kGroupMax || t.nnodes > INT32_MAX)
    return fail(c, PHYS_ERR_ARG, "group walk: %lld bodies is too many", (long long)t.n);
  return p->precision == PHYS_F32C ? launch<true>(c, p, t, want_force, ox, oy, oz)
                                   : launch<false>(c, p, t, want_force, ox, oy, oz);
}

}  // namespace phys
