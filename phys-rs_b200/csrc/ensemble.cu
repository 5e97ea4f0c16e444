// K8: batched ensemble of independent small systems (N <= 64 each).
//
// Each system is the reference's direct-sum Velocity-Verlet tick
// (gravity.rs:53-69 + integrators.rs:63-118) applied to its own bodies only.
// One persistent kernel runs a chunk of steps for every system: a group of G
// lanes (G = 8, 16 or 32; several groups per warp when G < 32) takes the next
// system from a global queue (systems in descending N, longest first), keeps
// the system's f64 state in shared memory for the whole chunk and returns it
// to HBM at the end.  Pair terms are F32C (double-float relative coordinates,
// two-sum accumulation) or F64_EXACT (reference op order, bit-identical).
// The host captures the chunk launches of a run in a CUDA graph; an
// autotuner picks G by timing a few steps of each candidate.
#include <algorithm>
#include <cstddef>
#include <numeric>
#include <vector>

#include "common.cuh"

namespace phys {
namespace {

constexpr int kMaxSys = 64;        // bodies per system
constexpr int kEnsCandidates = PHYS_ENS_CANDIDATES;
// F32C: sources per partial sum before it is folded into the compensated
// (hi, lo) accumulator (a system has at most 64)
constexpr int kFold = 32;

// Per-group state in shared memory for systems of at most MAXN bodies.
template <int MAXN>
struct GroupSmemT {
  double x[MAXN], y[MAXN], z[MAXN];
  double vx[MAXN], vy[MAXN], vz[MAXN];
  double ax[MAXN], ay[MAXN], az[MAXN];
  double pax[MAXN], pay[MAXN], paz[MAXN];
  double m[MAXN];
  // F32C staging, structure of arrays so that a float2 load gives two
  // consecutive bodies (slot N of an odd-N system is a massless pad far away)
  float hx[MAXN], hy[MAXN], hz[MAXN], hm[MAXN];  // hi parts, m (f32)
  float lx[MAXN], ly[MAXN], lz[MAXN];            // lo parts
};
using GroupSmem = GroupSmemT<kMaxSys>;
// With lanes per system chosen by size, a warp's shared memory holds one
// 64-body group, two 16-body groups or four 8-body groups in turn.
// quads of sources are read with 16-byte loads
static_assert(sizeof(GroupSmemT<8>) % 16 == 0 && sizeof(GroupSmemT<16>) % 16 == 0 &&
                  sizeof(GroupSmem) % 16 == 0 && offsetof(GroupSmemT<8>, hx) % 16 == 0 &&
                  offsetof(GroupSmemT<8>, hy) % 16 == 0,
              "16-byte aligned source arrays");
static_assert(2 * sizeof(GroupSmemT<16>) <= sizeof(GroupSmem) &&
                  4 * sizeof(GroupSmemT<8>) <= sizeof(GroupSmem),
              "sub-warp groups fit in a warp's share");

template <int G>
__device__ __forceinline__ unsigned group_mask() {
  if constexpr (G == 32) {
    return 0xffffffffu;
  } else {
    const unsigned lane = threadIdx.x & 31;
    return ((1u << G) - 1u) << (lane & ~(unsigned)(G - 1));
  }
}

template <class S_t>
__device__ __forceinline__ void split_into(S_t* S, int i) {
  split_df(S->x[i], S->hx[i], S->lx[i]);
  split_df(S->y[i], S->hy[i], S->ly[i]);
  split_df(S->z[i], S->hz[i], S->lz[i]);
  S->hm[i] = (float)S->m[i];
}

template <class S_t>
__device__ __forceinline__ void set_pad(S_t* S, int i) {
  S->hx[i] = S->hy[i] = S->hz[i] = 1e15f;
  S->hm[i] = S->lx[i] = S->ly[i] = S->lz[i] = 0.f;
}

__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

// Four consecutive sources (bodies j..j+3, j a multiple of 4) in seven
// 16-byte shared-memory loads; slots past N are massless pads far away.
struct QuadSrc {
  float4 sx, sy, sz, sm, tx, ty, tz;
};
template <class S_t>
__device__ __forceinline__ QuadSrc load_quad(const S_t* S, int j) {
  auto q = [&](const float* a) { return *reinterpret_cast<const float4*>(a + j); };
  return QuadSrc{q(S->hx), q(S->hy), q(S->hz), q(S->hm), q(S->lx), q(S->ly), q(S->lz)};
}

// One source pair against one target.  kSkip zeroes the halves that are
// the target itself (i == j is skipped, gravity.rs:56); with eps^2 > 0 it is
// not needed: the self separation is exactly 0 (hi - hi + lo - lo) and
// r^2 = eps^2, so the term adds exactly 0.
template <bool kSkip>
__device__ __forceinline__ void pair_term(float2 sx, float2 sy, float2 sz, float2 sm, float2 tx,
                                          float2 ty, float2 tz, float2 nhx, float2 nhy,
                                          float2 nhz, float2 nlx, float2 nly, float2 nlz,
                                          float2 e2, bool skip0, bool skip1, float2& px,
                                          float2& py, float2& pz) {
  const float2 rx = __fadd2_rn(__fadd2_rn(sx, nhx), __fadd2_rn(tx, nlx));
  const float2 ry = __fadd2_rn(__fadd2_rn(sy, nhy), __fadd2_rn(ty, nly));
  const float2 rz = __fadd2_rn(__fadd2_rn(sz, nhz), __fadd2_rn(tz, nlz));
  const float2 r2 = __ffma2_rn(rx, rx, __ffma2_rn(ry, ry, __ffma2_rn(rz, rz, e2)));
  const float2 inv = make_float2(rsqrt_sfu(r2.x), rsqrt_sfu(r2.y));
  float2 w = __fmul2_rn(sm, __fmul2_rn(__fmul2_rn(inv, inv), inv));
  if (kSkip) {
    if (skip0) w.x = 0.f;
    if (skip1) w.y = 0.f;
  }
  px = __ffma2_rn(rx, w, px);
  py = __ffma2_rn(ry, w, py);
  pz = __ffma2_rn(rz, w, pz);
}

// Folds packed partial sums into a (hi, lo) accumulator by two-sum.
__device__ __forceinline__ void fold(float2& p, float& h, float& l) {
  float s, e;
  two_sum(h, p.x + p.y, s, e);
  h = s;
  l += e;
  p = make_float2(0.f, 0.f);
}

// The negated double-float position of target i, packed for f32x2 terms.
struct TargetNeg {
  float2 hx, hy, hz, lx, ly, lz;
};
template <class S_t>
__device__ __forceinline__ TargetNeg target_neg(const S_t* S, int i) {
  auto n = [](float v) { return make_float2(-v, -v); };
  return TargetNeg{n(S->hx[i]), n(S->hy[i]), n(S->hz[i]), n(S->lx[i]), n(S->ly[i]), n(S->lz[i])};
}

// F32C accelerations of the group's own targets, TC targets per pass.  The
// sources come four at a time (two packed f32x2 pairs: sources j, j+1 and
// j+2, j+3); with one target per lane the two pairs go to separate partial
// sums, so two dependency chains interleave.  Partial sums of kFold sources are
// folded into a (hi, lo) accumulator by two-sum.
template <int G, int TC, bool kSkip, class S_t>
__device__ void group_forces_f32c(S_t* S, int N, int gl, double Gc, float eps2f) {
  const float2 e2 = make_float2(eps2f, eps2f);
  constexpr int kSets = TC == 1 ? 2 : 1;
  const int n4 = (N + 3) & ~3;
  for (int i0 = gl; i0 < N; i0 += G * TC) {
    TargetNeg tn[TC];
    float2 px[kSets][TC], py[kSets][TC], pz[kSets][TC];
    float hx[TC], hy[TC], hz[TC], lx[TC], ly[TC], lz[TC];
    int idx[TC];
#pragma unroll
    for (int t = 0; t < TC; ++t) {
      idx[t] = i0 + t * G;
      tn[t] = target_neg(S, idx[t] < N ? idx[t] : i0);
      hx[t] = hy[t] = hz[t] = lx[t] = ly[t] = lz[t] = 0.f;
#pragma unroll
      for (int k = 0; k < kSets; ++k) px[k][t] = py[k][t] = pz[k][t] = make_float2(0.f, 0.f);
    }
    for (int j0 = 0; j0 < n4; j0 += kFold) {
      const int j1 = min(n4, j0 + kFold);
      for (int j = j0; j < j1; j += 4) {
        const QuadSrc q = load_quad(S, j);
#pragma unroll
        for (int t = 0; t < TC; ++t) {
          const TargetNeg& a = tn[t];
          pair_term<kSkip>(lo2(q.sx), lo2(q.sy), lo2(q.sz), lo2(q.sm), lo2(q.tx), lo2(q.ty),
                           lo2(q.tz), a.hx, a.hy, a.hz, a.lx, a.ly, a.lz, e2, j == idx[t],
                           j + 1 == idx[t], px[0][t], py[0][t], pz[0][t]);
          pair_term<kSkip>(hi2(q.sx), hi2(q.sy), hi2(q.sz), hi2(q.sm), hi2(q.tx), hi2(q.ty),
                           hi2(q.tz), a.hx, a.hy, a.hz, a.lx, a.ly, a.lz, e2, j + 2 == idx[t],
                           j + 3 == idx[t], px[kSets - 1][t], py[kSets - 1][t],
                           pz[kSets - 1][t]);
        }
      }
#pragma unroll
      for (int t = 0; t < TC; ++t) {
#pragma unroll
        for (int k = 0; k < kSets; ++k) {
          fold(px[k][t], hx[t], lx[t]);
          fold(py[k][t], hy[t], ly[t]);
          fold(pz[k][t], hz[t], lz[t]);
        }
      }
    }
#pragma unroll
    for (int t = 0; t < TC; ++t) {
      if (idx[t] < N) {
        S->ax[idx[t]] = Gc * ((double)hx[t] + (double)lx[t]);
        S->ay[idx[t]] = Gc * ((double)hy[t] + (double)ly[t]);
        S->az[idx[t]] = Gc * ((double)hz[t] + (double)lz[t]);
      }
    }
  }
}

__device__ __forceinline__ int next_pow2(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

// F32C forces of a 33..64-body system on one warp without idle second
// slots: lane l takes target a = l over every source, and one of the
// nb = N - 32 second targets, b = 32 + l mod lps (lps = nb rounded up to a
// power of two), over its stream's share of the sources: the warp's
// r = 32 / lps streams take alternate groups of four sources, and their sums
// for the same b are added by shuffles at the end.  Each round covers r
// source quads: all r against a (two interleaved chains), one (the
// stream's own) against b.
// kR = 1 (49..64 bodies: one stream, b = 32 + l) fixes the layout at
// compile time, so b's quad is a's and is loaded once; kR = 0 derives the
// streams from N.
template <bool kSkip, int kR, class S_t>
__device__ void group_forces_f32c_split(S_t* S, int N, int gl, double Gc, float eps2f) {
  const float2 e2 = make_float2(eps2f, eps2f);
  const int nb = N - 32;
  const int lps = kR ? 32 / kR : next_pow2(nb), r = kR ? kR : 32 / lps;
  const int st = gl / lps, tb = 32 + gl % lps;
  const int ta = gl;
  const int tbv = tb < N ? tb : ta;  // lanes without a valid b compute a dummy (discarded)
  const TargetNeg A = target_neg(S, ta), B = target_neg(S, tbv);
  const float2 z2 = make_float2(0.f, 0.f);
  float2 pax0 = z2, pay0 = z2, paz0 = z2, pax1 = z2, pay1 = z2, paz1 = z2;
  float2 pbx = z2, pby = z2, pbz = z2;
  float hax = 0.f, hay = 0.f, haz = 0.f, lax = 0.f, lay = 0.f, laz = 0.f;
  float hbx = 0.f, hby = 0.f, hbz = 0.f, lbx = 0.f, lby = 0.f, lbz = 0.f;
  const int nq = (N + 3) >> 2;  // source quads
  int fa = 0, fb = 0;           // quads in the partial sums
  for (int q0 = 0; q0 < nq; q0 += r) {
    for (int k = 0; k < r && q0 + k < nq; ++k) {
      const int j = 4 * (q0 + k);
      const QuadSrc q = load_quad(S, j);
      pair_term<kSkip>(lo2(q.sx), lo2(q.sy), lo2(q.sz), lo2(q.sm), lo2(q.tx), lo2(q.ty),
                       lo2(q.tz), A.hx, A.hy, A.hz, A.lx, A.ly, A.lz, e2, j == ta, j + 1 == ta,
                       pax0, pay0, paz0);
      pair_term<kSkip>(hi2(q.sx), hi2(q.sy), hi2(q.sz), hi2(q.sm), hi2(q.tx), hi2(q.ty),
                       hi2(q.tz), A.hx, A.hy, A.hz, A.lx, A.ly, A.lz, e2, j + 2 == ta,
                       j + 3 == ta, pax1, pay1, paz1);
      if (++fa == kFold / 4) {
        fold(pax0, hax, lax);
        fold(pay0, hay, lay);
        fold(paz0, haz, laz);
        fold(pax1, hax, lax);
        fold(pay1, hay, lay);
        fold(paz1, haz, laz);
        fa = 0;
      }
    }
    const int qb = q0 + st;
    if (qb < nq) {
      const int j = 4 * qb;
      const QuadSrc q = load_quad(S, j);
      pair_term<kSkip>(lo2(q.sx), lo2(q.sy), lo2(q.sz), lo2(q.sm), lo2(q.tx), lo2(q.ty),
                       lo2(q.tz), B.hx, B.hy, B.hz, B.lx, B.ly, B.lz, e2, j == tbv,
                       j + 1 == tbv, pbx, pby, pbz);
      pair_term<kSkip>(hi2(q.sx), hi2(q.sy), hi2(q.sz), hi2(q.sm), hi2(q.tx), hi2(q.ty),
                       hi2(q.tz), B.hx, B.hy, B.hz, B.lx, B.ly, B.lz, e2, j + 2 == tbv,
                       j + 3 == tbv, pbx, pby, pbz);
      if (++fb == kFold / 4) {
        fold(pbx, hbx, lbx);
        fold(pby, hby, lby);
        fold(pbz, hbz, lbz);
        fb = 0;
      }
    }
  }
  fold(pax0, hax, lax);
  fold(pay0, hay, lay);
  fold(paz0, haz, laz);
  fold(pax1, hax, lax);
  fold(pay1, hay, lay);
  fold(paz1, haz, laz);
  fold(pbx, hbx, lbx);
  fold(pby, hby, lby);
  fold(pbz, hbz, lbz);
  S->ax[ta] = Gc * ((double)hax + (double)lax);
  S->ay[ta] = Gc * ((double)hay + (double)lay);
  S->az[ta] = Gc * ((double)haz + (double)laz);
  double bx = (double)hbx + (double)lbx, by = (double)hby + (double)lby,
         bz = (double)hbz + (double)lbz;
  for (int o = lps; o < 32; o <<= 1) {  // the streams' sums of the same b
    bx += __shfl_xor_sync(0xffffffffu, bx, o);
    by += __shfl_xor_sync(0xffffffffu, by, o);
    bz += __shfl_xor_sync(0xffffffffu, bz, o);
  }
  if (st == 0 && tb < N) {
    S->ax[tb] = Gc * bx;
    S->ay[tb] = Gc * by;
    S->az[tb] = Gc * bz;
  }
}

// Targets per lane for this system: one, or passes of kMaxTC (two) when
// the system has more bodies than the group has lanes (8 or 16 lanes only:
// 32 lanes take 33..64 bodies in the split layout).
template <int G, int kMaxTC, bool kSkip, class S_t>
__device__ __forceinline__ void group_forces_f32c_any(S_t* S, int N, int gl, double Gc,
                                                      float eps2f) {
  if (G == 32 && N > 32) {
    if (N > 48)
      group_forces_f32c_split<kSkip, 1>(S, N, gl, Gc, eps2f);
    else
      group_forces_f32c_split<kSkip, 0>(S, N, gl, Gc, eps2f);
    return;
  }
  if (kMaxTC == 1 || N <= G)
    group_forces_f32c<G, 1, kSkip>(S, N, gl, Gc, eps2f);
  else
    group_forces_f32c<G, (kMaxTC > 1 ? 2 : 1), kSkip>(S, N, gl, Gc, eps2f);
}

// Accelerations of the group's own targets (i = gl, gl+G, ...) into S->a.
template <int G, bool kExact, int kMaxTC, class S_t>
__device__ void group_forces(S_t* S, int N, int gl, double Gc, double eps2) {
  if (kExact) {
    for (int i = gl; i < N; i += G) {
      const double xi = S->x[i], yi = S->y[i], zi = S->z[i], mi = S->m[i];
      const double gm = xmul(Gc, mi);
      double fx = 0.0, fy = 0.0, fz = 0.0;
      for (int j = 0; j < N; ++j) {
        if (j == i) continue;
        const double rx = xsub(S->x[j], xi), ry = xsub(S->y[j], yi), rz = xsub(S->z[j], zi);
        const double s2 = xadd(xlen2(rx, ry, rz), eps2);
        const double sc = xdiv(xmul(gm, S->m[j]), xmul(s2, xsqrt(s2)));
        fx = xadd(fx, xmul(rx, sc));
        fy = xadd(fy, xmul(ry, sc));
        fz = xadd(fz, xmul(rz, sc));
      }
      S->ax[i] = xdiv(fx, mi);  // a = F / m (integrators.rs:115)
      S->ay[i] = xdiv(fy, mi);
      S->az[i] = xdiv(fz, mi);
    }
    return;
  }
  const float eps2f = (float)eps2;
  if (eps2f > 0.f)
    group_forces_f32c_any<G, kMaxTC, false>(S, N, gl, Gc, eps2f);
  else  // eps = 0: the self pair must be skipped by index
    group_forces_f32c_any<G, kMaxTC, true>(S, N, gl, Gc, eps2f);
}

struct EnsArgs {
  int nsys;
  const int32_t* order;
  const int64_t* off;
  double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az;
  const double* m;
  double Gc, eps2, dt;
  int nsteps, need_accel;
  int* queue;      // three work counters of this launch
  int32_t* status;
  int n32, n16;    // by-size mode: systems [0, n32) have > 16 bodies, [n32, n16) 9..16
};

// A group of G lanes takes systems s in [lo, hi) from the counter and runs
// `nsteps` reference ticks on each with its state in shared memory.
template <int G, bool kExact, int kMaxTC, class S_t>
__device__ void drain(S_t* S, const EnsArgs& a, int lo, int hi, int* ctr, int maxn) {
  const int gl = (threadIdx.x & 31) % G;
  const unsigned gm = group_mask<G>();
  const double dt = a.dt;
  const double h2 = xmul(xmul(0.5, dt), dt), hdt = xmul(0.5, dt);
  for (;;) {
    int s = 0;
    if (gl == 0) s = lo + atomicAdd(ctr, 1);
    s = __shfl_sync(gm, s, 0, G);
    if (s >= hi) break;
    const int sys = a.order[s];
    const int64_t b = a.off[sys];
    const int N = (int)(a.off[sys + 1] - b);
    // slots up to N rounded up to 4 are used (maxn is a multiple of 4)
    if (N < 0 || N > maxn) {
      if (gl == 0) atomicOr(a.status, kStatOverflow);
      continue;
    }
    for (int i = gl; i < N; i += G) {
      S->x[i] = a.x[b + i];
      S->y[i] = a.y[b + i];
      S->z[i] = a.z[b + i];
      S->vx[i] = a.vx[b + i];
      S->vy[i] = a.vy[b + i];
      S->vz[i] = a.vz[b + i];
      S->ax[i] = a.ax[b + i];
      S->ay[i] = a.ay[b + i];
      S->az[i] = a.az[b + i];
      S->m[i] = a.m[b + i];
      split_into(S, i);
    }
    // slots N .. N rounded up to 4 are massless pads (the quads of sources)
    for (int i = N + gl; i < ((N + 3) & ~3); i += G) set_pad(S, i);
    __syncwarp(gm);
    if (a.need_accel && N >= 2) group_forces<G, kExact, kMaxTC>(S, N, gl, a.Gc, a.eps2);
    if (a.need_accel && N < 2)
      for (int i = gl; i < N; i += G) S->ax[i] = S->ay[i] = S->az[i] = 0.0;
    __syncwarp(gm);
    for (int st = 0; st < a.nsteps; ++st) {
      // velocity_verlet_position_system: prev = a; x += v dt + a dt^2/2
      for (int i = gl; i < N; i += G) {
        const double a0 = S->ax[i], a1 = S->ay[i], a2 = S->az[i];
        S->pax[i] = a0;
        S->pay[i] = a1;
        S->paz[i] = a2;
        S->x[i] = xadd(S->x[i], xadd(xmul(S->vx[i], dt), xmul(a0, h2)));
        S->y[i] = xadd(S->y[i], xadd(xmul(S->vy[i], dt), xmul(a1, h2)));
        S->z[i] = xadd(S->z[i], xadd(xmul(S->vz[i], dt), xmul(a2, h2)));
        split_into(S, i);
      }
      __syncwarp(gm);
      if (N >= 2) group_forces<G, kExact, kMaxTC>(S, N, gl, a.Gc, a.eps2);
      __syncwarp(gm);
      // velocity_verlet_velocity_system: v += (prev + a) dt/2
      for (int i = gl; i < N; i += G) {
        S->vx[i] = xadd(S->vx[i], xmul(xadd(S->pax[i], S->ax[i]), hdt));
        S->vy[i] = xadd(S->vy[i], xmul(xadd(S->pay[i], S->ay[i]), hdt));
        S->vz[i] = xadd(S->vz[i], xmul(xadd(S->paz[i], S->az[i]), hdt));
      }
      __syncwarp(gm);
    }
    bool bad = false;
    for (int i = gl; i < N; i += G) {
      a.x[b + i] = S->x[i];
      a.y[b + i] = S->y[i];
      a.z[b + i] = S->z[i];
      a.vx[b + i] = S->vx[i];
      a.vy[b + i] = S->vy[i];
      a.vz[b + i] = S->vz[i];
      a.ax[b + i] = S->ax[i];
      a.ay[b + i] = S->ay[i];
      a.az[b + i] = S->az[i];
      bad |= !isfinite(S->x[i]) || !isfinite(S->vx[i]) || !isfinite(S->ax[i]);
    }
    if (bad) atomicOr(a.status, kStatNonfinite);
    __syncwarp(gm);
  }
}

// One persistent launch of BW warps per block.  G = 8, 16, 32: every system
// gets G lanes (32 / G systems per warp at a time).  G = 0: lanes by size —
// a warp takes the systems of more than 16 bodies one at a time, then two of
// 9..16 bodies at a time (16 lanes each), then four of at most 8.
template <int G, int BW, bool kExact>
__global__ void __launch_bounds__(32 * BW)
ensemble_kernel(EnsArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if constexpr (G != 0) {
    GroupSmem* S = reinterpret_cast<GroupSmem*>(smem_raw) + warp * (32 / G) + lane / G;
    drain<G, kExact, (G == 32 ? 1 : 2)>(S, a, 0, a.nsys, a.queue, kMaxSys);
  } else {
    unsigned char* base = smem_raw + warp * sizeof(GroupSmem);
    drain<32, kExact, 1>(reinterpret_cast<GroupSmem*>(base), a, 0, a.n32, a.queue, kMaxSys);
    drain<16, kExact, 1>(reinterpret_cast<GroupSmemT<16>*>(base) + (lane >> 4), a, a.n32, a.n16,
                      a.queue + 1, 16);
    drain<8, kExact, 1>(reinterpret_cast<GroupSmemT<8>*>(base) + (lane >> 3), a, a.n16, a.nsys,
                     a.queue + 2, 8);
  }
}

using EnsKernel = void (*)(EnsArgs);

template <int BW>
EnsKernel pick_bw(int G, bool exact) {
  switch (G) {
    case 8: return exact ? ensemble_kernel<8, BW, true> : ensemble_kernel<8, BW, false>;
    case 16: return exact ? ensemble_kernel<16, BW, true> : ensemble_kernel<16, BW, false>;
    case 32: return exact ? ensemble_kernel<32, BW, true> : ensemble_kernel<32, BW, false>;
    default: return exact ? ensemble_kernel<0, BW, true> : ensemble_kernel<0, BW, false>;
  }
}

EnsKernel pick(int G, int bw, bool exact) {
  return bw == 4 ? pick_bw<4>(G, exact) : pick_bw<2>(G, exact);
}

struct EnsView {
  double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az, *m;
};

EnsView view(phys_ctx* c) {
  double* b = reinterpret_cast<double*>(c->ws[WS_ENS0].p);
  const int64_t n = c->ens_nbody;
  return EnsView{b, b + n, b + 2 * n, b + 3 * n, b + 4 * n, b + 5 * n, b + 6 * n, b + 7 * n,
                 b + 8 * n, b + 9 * n};
}

struct LaunchCfg {
  EnsKernel k;
  size_t smem;
  int64_t grid;
  int block;
};

// Launch configuration code: lanes per system (8, 16, 32 or
// PHYS_ENS_BY_SIZE) | warps per block << 8 (2 or 4; 0 means 2).
bool decode(int code, int* G, int* bw) {
  const int g = code & 0xff, w = (code >> 8) & 0xff;
  if (code & ~0xffff) return false;
  if (g != 8 && g != 16 && g != 32 && g != PHYS_ENS_BY_SIZE) return false;
  if (w != 0 && w != 2 && w != 4) return false;
  *G = g == PHYS_ENS_BY_SIZE ? 0 : g;
  *bw = w == 0 ? 2 : w;
  return true;
}

// Kernel attributes and the persistent grid size (queried outside capture).
int prepare(phys_ctx* c, const phys_params* p, int code, LaunchCfg* cfg) {
  int G = 0, bw = 2;
  if (!decode(code, &G, &bw)) return fail(c, PHYS_ERR_ARG, "ensemble configuration 0x%x", code);
  const bool exact = p->precision == PHYS_F64_EXACT;
  cfg->k = pick(G, bw, exact);
  cfg->block = 32 * bw;
  const int groups_per_warp = G == 0 ? 1 : 32 / G;
  cfg->smem = sizeof(GroupSmem) * groups_per_warp * bw;
  PHYS_CUDA(c, cudaFuncSetAttribute(cfg->k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)cfg->smem));
  int per_sm = 0;
  PHYS_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cfg->k, cfg->block,
                                                             cfg->smem));
  int sms = 148;
  PHYS_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  const int64_t groups_per_block = (int64_t)groups_per_warp * bw;
  cfg->grid = std::min<int64_t>((int64_t)std::max(per_sm, 1) * sms,
                                ceil_div(c->ens_nsys, groups_per_block));
  if (cfg->grid < 1) cfg->grid = 1;
  return PHYS_OK;
}

// Enqueue one run of `nsteps` steps in chunks of `chunk` steps (one launch each).
int enqueue_run(phys_ctx* c, const phys_params* p, const LaunchCfg& cfg, double dt,
                int64_t nsteps, int64_t chunk, bool need_accel_first) {
  EnsView v = view(c);
  int* queue = reinterpret_cast<int*>(c->ws[WS_ENS3].p);
  EnsArgs a;
  a.nsys = (int)c->ens_nsys;
  a.order = reinterpret_cast<const int32_t*>(c->ws[WS_ENS2].p);
  a.off = reinterpret_cast<const int64_t*>(c->ws[WS_ENS1].p);
  a.x = v.x; a.y = v.y; a.z = v.z;
  a.vx = v.vx; a.vy = v.vy; a.vz = v.vz;
  a.ax = v.ax; a.ay = v.ay; a.az = v.az;
  a.m = v.m;
  a.Gc = p->G;
  a.eps2 = p->eps * p->eps;
  a.dt = dt;
  a.status = c->d_status;
  a.n32 = (int)c->ens_n32;
  a.n16 = (int)c->ens_n16;
  int64_t done = 0;
  int ci = 0;
  bool need = need_accel_first;
  do {
    const int64_t k_steps = std::min<int64_t>(chunk, nsteps - done);
    a.queue = queue + 4 * ci;  // three counters per launch
    a.nsteps = (int)k_steps;
    a.need_accel = need ? 1 : 0;
    PHYS_CUDA(c, cudaMemsetAsync(a.queue, 0, 4 * sizeof(int), c->stream));
    cfg.k<<<(unsigned)cfg.grid, cfg.block, cfg.smem, c->stream>>>(a);
    c->launches++;
    PHYS_TRY(check_launch(c, "ensemble_kernel"));
    need = false;
    done += k_steps;
    ci = (ci + 1) & 255;
  } while (done < nsteps);
  return PHYS_OK;
}

}  // namespace

int ensemble_load(phys_ctx* c, int64_t nsys, const int64_t* off, const double* x, const double* y,
                  const double* z, const double* vx, const double* vy, const double* vz,
                  const double* m) {
  const int64_t n = off[nsys];
  if (off[0] != 0) return fail(c, PHYS_ERR_ARG, "offsets[0] must be 0");
  std::vector<int32_t> order(nsys);
  for (int64_t s = 0; s < nsys; ++s) {
    const int64_t k = off[s + 1] - off[s];
    if (k < 0 || k > kMaxSys)
      return fail(c, PHYS_ERR_ARG, "system %lld has %lld bodies (1..%d supported)", (long long)s,
                  (long long)k, kMaxSys);
    order[s] = (int32_t)s;
  }
  // longest first: the tail of the persistent queue holds the cheapest systems
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
    return (off[a + 1] - off[a]) > (off[b + 1] - off[b]);
  });
  int st = PHYS_OK;
  double* base = (double*)ws_get(c, WS_ENS0, sizeof(double) * 10 * (n > 0 ? n : 1), &st);
  if (st) return st;
  ws_get(c, WS_ENS1, sizeof(int64_t) * (nsys + 1), &st);
  if (st) return st;
  ws_get(c, WS_ENS2, sizeof(int32_t) * (nsys > 0 ? nsys : 1), &st);
  if (st) return st;
  ws_get(c, WS_ENS3, sizeof(int) * 1024, &st);
  if (st) return st;
  c->ens_nsys = nsys;
  c->ens_nbody = n;
  // by-size launches: the sorted systems with more than 16, then 9..16 bodies
  int64_t n32 = 0, n16 = 0;
  for (int64_t s = 0; s < nsys; ++s) {
    const int64_t k = off[order[s] + 1] - off[order[s]];
    n32 += k > 16;
    n16 += k > 8;
  }
  c->ens_n32 = n32;
  c->ens_n16 = n16;
  c->ens_accel_valid = false;
  EnsView v = view(c);
  const double* src[7] = {x, y, z, vx, vy, vz, m};
  double* dst[7] = {v.x, v.y, v.z, v.vx, v.vy, v.vz, v.m};
  for (int k = 0; k < 7; ++k) {
    if (src[k])
      PHYS_CUDA(c, cudaMemcpyAsync(dst[k], src[k], sizeof(double) * n, cudaMemcpyHostToDevice,
                                   c->stream));
    else
      PHYS_CUDA(c, cudaMemsetAsync(dst[k], 0, sizeof(double) * n, c->stream));
  }
  PHYS_CUDA(c, cudaMemsetAsync(v.ax, 0, sizeof(double) * 3 * n, c->stream));
  PHYS_CUDA(c, cudaMemcpyAsync(c->ws[WS_ENS1].p, off, sizeof(int64_t) * (nsys + 1),
                               cudaMemcpyHostToDevice, c->stream));
  PHYS_CUDA(c, cudaMemcpyAsync(c->ws[WS_ENS2].p, order.data(), sizeof(int32_t) * nsys,
                               cudaMemcpyHostToDevice, c->stream));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  (void)base;
  return PHYS_OK;
}

int ensemble_run(phys_ctx* c, const phys_params* p, double dt, int64_t nsteps, int G,
                 int64_t chunk) {  // G: configuration code
  if (c->ens_nsys <= 0) return fail(c, PHYS_ERR_STATE, "no ensemble loaded");
  if (chunk <= 0) chunk = nsteps > 0 ? nsteps : 1;
  LaunchCfg cfg;
  PHYS_TRY(prepare(c, p, G, &cfg));
  // Capture the chunk launches of this run in a CUDA graph, then replay it.
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  PHYS_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int st = enqueue_run(c, p, cfg, dt, nsteps, chunk, !c->ens_accel_valid);
  cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
  if (st) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
  PHYS_CUDA(c, cudaEventRecord(c->ev[6], c->stream));
  e = cudaGraphLaunch(exec, c->stream);
  if (e == cudaSuccess) e = cudaEventRecord(c->ev[7], c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaGraphExecDestroy(exec);
  if (e != cudaSuccess) return cuda_fail(c, e, "ensemble graph launch");
  c->ens_accel_valid = true;
  return PHYS_OK;
}

int ensemble_download(phys_ctx* c, double* x, double* y, double* z, double* vx, double* vy,
                      double* vz, double* ax, double* ay, double* az) {
  EnsView v = view(c);
  const int64_t n = c->ens_nbody;
  double* dst[9] = {x, y, z, vx, vy, vz, ax, ay, az};
  double* src[9] = {v.x, v.y, v.z, v.vx, v.vy, v.vz, v.ax, v.ay, v.az};
  for (int k = 0; k < 9; ++k)
    if (dst[k])
      PHYS_CUDA(c, cudaMemcpyAsync(dst[k], src[k], sizeof(double) * n, cudaMemcpyDeviceToHost,
                                   c->stream));
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  return PHYS_OK;
}

// Times `probe_steps` steps for each candidate configuration from the same
// starting state (saved and restored around the probes) and keeps the
// fastest.  The candidates: lanes per system 8, 16, 32 and by size, two
// warps per block; 32 and by size, four warps per block.
const int kTuneCand[kEnsCandidates] = {8 | 2 << 8, 16 | 2 << 8, 32 | 2 << 8,
                                       PHYS_ENS_BY_SIZE | 2 << 8, 32 | 4 << 8,
                                       PHYS_ENS_BY_SIZE | 4 << 8};

int ensemble_autotune(phys_ctx* c, const phys_params* p, double dt, int64_t probe_steps,
                      int32_t* best, double* ms_out) {
  if (c->ens_nsys <= 0) return fail(c, PHYS_ERR_STATE, "no ensemble loaded");
  const int64_t n = c->ens_nbody;
  int st = PHYS_OK;
  double* save = (double*)ws_get(c, WS_ENS4, sizeof(double) * 9 * (n > 0 ? n : 1), &st);
  if (st) return st;
  EnsView v = view(c);
  const bool valid0 = c->ens_accel_valid;
  PHYS_CUDA(c, cudaMemcpyAsync(save, v.x, sizeof(double) * 9 * n, cudaMemcpyDeviceToDevice,
                               c->stream));
  double best_ms = 1e300;
  int best_cfg = kTuneCand[2];
  for (int k = 0; k < kEnsCandidates; ++k) {
    c->ens_accel_valid = true;  // time steps only; the force of the start state is reused
    PHYS_TRY(ensemble_run(c, p, dt, probe_steps, kTuneCand[k], probe_steps));
    float ms = 0.f;
    PHYS_CUDA(c, cudaEventElapsedTime(&ms, c->ev[6], c->ev[7]));
    if (ms_out) ms_out[k] = ms;
    if (ms < best_ms) {
      best_ms = ms;
      best_cfg = kTuneCand[k];
    }
    PHYS_CUDA(c, cudaMemcpyAsync(v.x, save, sizeof(double) * 9 * n, cudaMemcpyDeviceToDevice,
                                 c->stream));
  }
  PHYS_CUDA(c, cudaStreamSynchronize(c->stream));
  c->ens_accel_valid = valid0;
  c->ens_group = best_cfg;
  if (best) *best = best_cfg;
  return PHYS_OK;
}

}  // namespace phys
