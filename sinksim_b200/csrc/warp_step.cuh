// One time step of one simulation, computed by a team of W warps (W = 1, 2, 4 or 8). The physics is the reference's
// kernel::step in the "portable" (double precision) and "portable32" (single-precision column partials) numerics
// (engine/include/sinksim/kernel/step.hpp:41-54), reproduced bit for bit:
//
//   * the buoyancy integral keeps the reference's 256 partial sums (partial p sums columns p, p+256, ... in
//     order), reduces each group of 32 partials with the halving tree (offsets 16..1) and adds the eight group
//     results in order (kernel/reduce.hpp:12-79, hydro.hpp:241-258). The team's warps share the eight groups: lane l
//     holds partial w*32+l of group w, and a shuffle butterfly performs the tree, each pair combined as (lower, upper);
//   * a node pass keeps the reference's 32 lane partials over strided segments and the same tree
//     (hydro.hpp:305-316, reduce.hpp:52-71); a group of kLevelLanes lanes forms them, each lane combining several
//     tree lanes' partials in the tree's order before the shuffles, so a warp solves 32 / kLevelLanes groups at once;
//   * every other reduction (group sums, incidence gathers, sea inflow, excess, loads, monitors, water) runs in
//     the reference's serial order, and every expression keeps its operation order (no contraction: -fmad=false).
//     The one count that is not a floating-point sum, a node's degree, is formed with shared-memory atomics.
//
// Every thread of the team holds identical copies of the scalars it uses, so control flow stays uniform; the team's
// threads wait on one another only at the team barrier (Team::sync: __syncwarp for one warp, a named barrier for
// more) between phases that exchange per-node or per-connection arrays through shared memory.
#pragma once

#include <cstdint>

#include "device_model.h"
#include "portable_math.cuh"
#include "scheme.h"

namespace ssb {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kLanes = 32;

__device__ __forceinline__ Pose make_pose(const DevModel& M, double zO, double th, double ph) {
  const double cth = pm::cos(th), sth = pm::sin(th), cph = pm::cos(ph), sph = pm::sin(ph);
  Pose F;
  F.R00 = cth; F.R01 = sth * sph; F.R02 = sth * cph;
  F.R10 = 0;   F.R11 = cph;       F.R12 = -sph;
  F.R20 = -sth; F.R21 = cth * sph; F.R22 = cth * cph;
  F.tx = M.XO - (F.R00 * M.g0x + F.R01 * M.g0y + F.R02 * M.g0z);
  F.ty = M.YO - (F.R10 * M.g0x + F.R11 * M.g0y + F.R12 * M.g0z);
  F.tz = zO - (F.R20 * M.g0x + F.R21 * M.g0y + F.R22 * M.g0z);
  F.cth = cth;
  F.iR = 1 / F.R22;
  F.fR20 = static_cast<float>(F.R20);
  F.fR21 = static_cast<float>(F.R21);
  F.fR22 = static_cast<float>(F.R22);
  F.ftz = static_cast<float>(F.tz);
  F.fiR = 1.0f / F.fR22;
  return F;
}

__device__ __forceinline__ double world_z(const Pose& F, double x, double y, double z) {
  return F.R20 * x + F.R21 * y + F.R22 * z + F.tz;
}

// ----------------------------------------------------------------------------- butterfly steps of the canonical tree
// At offset `off` the tree combines partial l (l < off) with partial l + off. With xor shuffles every lane pairs
// with lane ^ off; sums are exact to swap (IEEE addition is commutative) and the min / max keep the reference's
// operand order (lower partner first), so every lane ends with the bits of the tree's lane 0.

template <class T>
__device__ __forceinline__ T bsum(T v, int off, unsigned mask = kFull) { return v + __shfl_xor_sync(mask, v, off); }

template <class T>
__device__ __forceinline__ T bmin(T v, int off, int lane, unsigned mask = kFull) {
  const T o = __shfl_xor_sync(mask, v, off);
  const bool lower = (lane & off) == 0;
  const T a = lower ? v : o, b = lower ? o : v;
  return (b < a) ? b : a;
}

template <class T>
__device__ __forceinline__ T bmax(T v, int off, int lane, unsigned mask = kFull) {
  const T o = __shfl_xor_sync(mask, v, off);
  const bool lower = (lane & off) == 0;
  const T a = lower ? v : o, b = lower ? o : v;
  return (b > a) ? b : a;
}

// ----------------------------------------------------------------------------- a team of W warps stepping one simulation

// Thread `rank` of the team (0 .. 32 W - 1), its warp and lane. Teams of more than one warp synchronise on their own
// named barrier (ids 1..15; 0 is __syncthreads), so teams in one block never wait on each other.
template <int W>
struct Team {
  int rank, warp, lane, bar;
  __device__ __forceinline__ void sync() const {
    if constexpr (W == 1) __syncwarp();
    else asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(W * 32) : "memory");
  }
  __device__ __forceinline__ bool leader() const { return rank == 0; }
};

// ----------------------------------------------------------------------------- buoyancy (hydro pass, tree order)

// One column into a buoyancy partial (kernel/reduce.hpp:39-49 in double, :131-142 in float): the same expressions in
// the same order for T = double (portable) and T = float (portable32).
template <class T>
struct ColPartial {
  T V, Mx, My, Mz, top;
};

template <class T>
__device__ __forceinline__ void clip_column(T x, T y, T lo, T hi, T A, T R20, T R21, T R22, T tz, T iR, ColPartial<T>& p) {
  const T base = R20 * x + R21 * y + tz;
  const T wt = base + R22 * hi;
  if (wt > p.top) p.top = wt;
  const T zp = -base * iR;
  if (zp <= lo) return;
  const T s = zp >= hi ? hi - lo : zp - lo;
  const T v = A * s;
  p.V += v; p.Mx += v * x; p.My += v * y; p.Mz += v * (lo + T(0.5) * s);
}

// One segment into a node-pass partial (kernel/reduce.hpp:52-71 in double, :144-164 in float).
template <class T>
struct SegPartial {
  T vol, dv, mx, my, mz, zmin, zmax;
};

template <class T>
__device__ __forceinline__ void clip_segment(T x, T y, T a, T b, T A, T R20, T R21, T R22, T tz, T iR, T h, SegPartial<T>& p) {
  const T base = R20 * x + R21 * y + tz;
  const T wa = base + R22 * a, wb = base + R22 * b;
  if (wa < p.zmin) p.zmin = wa;
  if (wb > p.zmax) p.zmax = wb;
  const T zp = (h - base) * iR;
  if (zp <= a) return;
  T L;
  if (zp >= b) {
    L = b - a;
  } else {
    L = zp - a;
    p.dv += A;
  }
  const T v = A * L;
  p.vol += v; p.mx += v * x; p.my += v * y; p.mz += v * (a + T(0.5) * L);
}

template <class T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// A load of the column table: through the read-only data cache from global memory, or from shared memory (SMEM: the
// table staged there).
template <bool SMEM, class P>
__device__ __forceinline__ P load_col(const P* p) {
  if constexpr (SMEM) return *p;
  else return __ldg(p);
}

// Lane `lane`'s partial of tree w: columns w*32 + lane + 256 k in increasing k, two at a time (loads of the second
// column issue before the first is clipped; the clips stay in order).
template <class T, bool SMEM = false>
__device__ __forceinline__ ColPartial<T> column_partial(const typename Vec2<T>::type* xy, const typename Vec2<T>::type* lh, const T* area,
                                                        int ncol, int first, T R20, T R21, T R22, T tz, T iR) {
  ColPartial<T> p{T(0), T(0), T(0), T(0), T(-1e9)};
  int i = first;
  for (; i + 256 < ncol; i += 512) {
    const auto a0 = load_col<SMEM>(xy + i), b0 = load_col<SMEM>(lh + i), a1 = load_col<SMEM>(xy + i + 256), b1 = load_col<SMEM>(lh + i + 256);
    const T A0 = load_col<SMEM>(area + i), A1 = load_col<SMEM>(area + i + 256);
    clip_column<T>(a0.x, a0.y, b0.x, b0.y, A0, R20, R21, R22, tz, iR, p);
    clip_column<T>(a1.x, a1.y, b1.x, b1.y, A1, R20, R21, R22, tz, iR, p);
  }
  if (i < ncol) {
    const auto a0 = load_col<SMEM>(xy + i), b0 = load_col<SMEM>(lh + i);
    clip_column<T>(a0.x, a0.y, b0.x, b0.y, load_col<SMEM>(area + i), R20, R21, R22, tz, iR, p);
  }
  return p;
}

// The column table staged in shared memory (stage_columns): (x, y) pairs, (zlo, zhi) pairs and footprints of every
// column, in the arithmetic's type, each array at a 16-byte boundary.
template <class T>
struct StagedColumns {
  std::size_t xy, lh, area, bytes;
};

template <class T>
__host__ __device__ __forceinline__ StagedColumns<T> staged_columns(int ncol) {
  using V2 = typename Vec2<T>::type;
  StagedColumns<T> c;
  const std::size_t n = static_cast<std::size_t>(ncol);
  auto up16 = [](std::size_t b) { return (b + 15) & ~static_cast<std::size_t>(15); };
  c.xy = 0;
  c.lh = up16(n * sizeof(V2));
  c.area = c.lh + up16(n * sizeof(V2));
  c.bytes = c.area + up16(n * sizeof(T));
  return c;
}

// The eight trees are spread over the team's warps (warp v computes trees v, v + W, ...); the tree results meet in
// shared memory and every thread adds them in the reference's order (trees 0..7).
template <bool MIXED, int W>
__device__ __forceinline__ void buoyancy_trees(const DevModel& M, const Pose& F, const Team<W>& T, double* trees, const unsigned char* cols) {
  const int lane = T.lane;
  for (int w = T.warp; w < 8; w += W) {
    double g[5];
    if constexpr (!MIXED) {
      ColPartial<double> p;
      if (cols) {
        const StagedColumns<double> c = staged_columns<double>(M.ncol);
        p = column_partial<double, true>(reinterpret_cast<const double2*>(cols + c.xy), reinterpret_cast<const double2*>(cols + c.lh),
                                         reinterpret_cast<const double*>(cols + c.area), M.ncol, w * kLanes + lane, F.R20, F.R21, F.R22, F.tz, F.iR);
      } else {
        p = column_partial<double>(M.colXY, M.colLH, M.colA, M.ncol, w * kLanes + lane, F.R20, F.R21, F.R22, F.tz, F.iR);
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        p.V = bsum(p.V, off); p.Mx = bsum(p.Mx, off); p.My = bsum(p.My, off); p.Mz = bsum(p.Mz, off);
        p.top = bmax(p.top, off, lane);
      }
      g[0] = p.V; g[1] = p.Mx; g[2] = p.My; g[3] = p.Mz; g[4] = p.top;
    } else {
      ColPartial<float> p;
      if (cols) {
        const StagedColumns<float> c = staged_columns<float>(M.ncol);
        p = column_partial<float, true>(reinterpret_cast<const float2*>(cols + c.xy), reinterpret_cast<const float2*>(cols + c.lh),
                                        reinterpret_cast<const float*>(cols + c.area), M.ncol, w * kLanes + lane, F.fR20, F.fR21, F.fR22, F.ftz, F.fiR);
      } else {
        p = column_partial<float>(M.colXYf, M.colLHf, M.colAf, M.ncol, w * kLanes + lane, F.fR20, F.fR21, F.fR22, F.ftz, F.fiR);
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        p.V = bsum(p.V, off); p.Mx = bsum(p.Mx, off); p.My = bsum(p.My, off); p.Mz = bsum(p.Mz, off);
        p.top = bmax(p.top, off, lane);
      }
      g[0] = p.V; g[1] = p.Mx; g[2] = p.My; g[3] = p.Mz; g[4] = p.top;
    }
    if (lane == 0) {
      double* t = trees + 5 * w;
      for (int k = 0; k < 5; ++k) t[k] = g[k];
    }
  }
}

// The buoyancy result from the eight trees (after a team barrier that follows buoyancy_trees): every thread adds
// them in the reference's order and holds the same values.
__device__ __forceinline__ Buoy buoyancy_finish(const double* trees) {
  double V = trees[0], Mx = trees[1], My = trees[2], Mz = trees[3], top = trees[4];
  for (int w = 1; w < 8; ++w) {
    const double* t = trees + 5 * w;
    V += t[0]; Mx += t[1]; My += t[2]; Mz += t[3];
    if (t[4] > top) top = t[4];
  }
  Buoy b;
  b.V = V;
  b.x = V > 0 ? Mx / V : 0;
  b.y = V > 0 ? My / V : 0;
  b.z = V > 0 ? Mz / V : 0;
  b.top = top;
  return b;
}

template <bool MIXED, int W>
__device__ __forceinline__ Buoy buoyancy(const DevModel& M, const Pose& F, const Team<W>& T, double* trees, const unsigned char* cols) {
  buoyancy_trees<MIXED, W>(M, F, T, trees, cols);
  T.sync();
  return buoyancy_finish(trees);
}

// ----------------------------------------------------------------------------- node pass (tree order)

struct PassR {
  double vol, dv, mx, my, mz, zmin, zmax;
};

// The kLevelLanes<MIXED> consecutive lanes of a warp that solve one group of nodes: `lane` is the lane in the warp, `sub` the
// lane in the group, `mask` the group's lanes.
struct LevelLanes {
  int lane, sub;
  unsigned mask;
};

// The partial of one lane of the 32-lane tree (the lane whose first segment is `first`): segments first + 32 k in
// increasing k, two at a time.
template <class T>
__device__ __forceinline__ SegPartial<T> segment_partial(const typename Vec2<T>::type* xy, const typename Vec2<T>::type* ab, const T* area,
                                                         int first, int end, T R20, T R21, T R22, T tz, T iR, T h) {
  SegPartial<T> p{T(0), T(0), T(0), T(0), T(0), T(1e9), T(-1e9)};
  int j = first;
  for (; j + kLanes < end; j += 2 * kLanes) {
    const auto a0 = __ldg(xy + j), b0 = __ldg(ab + j), a1 = __ldg(xy + j + kLanes), b1 = __ldg(ab + j + kLanes);
    const T A0 = __ldg(area + j), A1 = __ldg(area + j + kLanes);
    clip_segment<T>(a0.x, a0.y, b0.x, b0.y, A0, R20, R21, R22, tz, iR, h, p);
    clip_segment<T>(a1.x, a1.y, b1.x, b1.y, A1, R20, R21, R22, tz, iR, h, p);
  }
  if (j < end) {
    const auto a0 = __ldg(xy + j), b0 = __ldg(ab + j);
    clip_segment<T>(a0.x, a0.y, b0.x, b0.y, __ldg(area + j), R20, R21, R22, tz, iR, h, p);
  }
  return p;
}

// The partials of two tree lanes 16 apart (first segments fa and fa + 16), in one loop: each iteration takes the next
// segment of each, so the two accumulation chains run side by side; each keeps its own segments' order. fa's lane has
// at most one segment more than the other's.
template <class T>
__device__ __forceinline__ void segment_pair(const typename Vec2<T>::type* xy, const typename Vec2<T>::type* ab, const T* area, int fa,
                                             int end, T R20, T R21, T R22, T tz, T iR, T h, SegPartial<T>& pa, SegPartial<T>& pb) {
  pa = SegPartial<T>{T(0), T(0), T(0), T(0), T(0), T(1e9), T(-1e9)};
  pb = pa;
  int ja = fa;
  for (; ja + 16 < end; ja += kLanes) {
    const int jb = ja + 16;
    const auto a0 = __ldg(xy + ja), b0 = __ldg(ab + ja), a1 = __ldg(xy + jb), b1 = __ldg(ab + jb);
    const T A0 = __ldg(area + ja), A1 = __ldg(area + jb);
    clip_segment<T>(a0.x, a0.y, b0.x, b0.y, A0, R20, R21, R22, tz, iR, h, pa);
    clip_segment<T>(a1.x, a1.y, b1.x, b1.y, A1, R20, R21, R22, tz, iR, h, pb);
  }
  if (ja < end) {
    const auto a0 = __ldg(xy + ja), b0 = __ldg(ab + ja);
    clip_segment<T>(a0.x, a0.y, b0.x, b0.y, __ldg(area + ja), R20, R21, R22, tz, iR, h, pa);
  }
}

// One level of the tree inside a lane: the lower tree lane's partial `lo` takes in the upper one's, with the operand
// order of the butterfly steps.
template <class T>
__device__ __forceinline__ void tree_pair(SegPartial<T>& lo, const SegPartial<T>& up) {
  lo.vol = lo.vol + up.vol; lo.dv = lo.dv + up.dv; lo.mx = lo.mx + up.mx; lo.my = lo.my + up.my; lo.mz = lo.mz + up.mz;
  lo.zmin = (up.zmin < lo.zmin) ? up.zmin : lo.zmin;
  lo.zmax = (up.zmax > lo.zmax) ? up.zmax : lo.zmax;
}

// The node pass of node n at world level h: the 32 lane partials, the halving tree and the permeability scaling
// (hydro.hpp:295-316 / 338-349). Lane `sub` of a group of LANES lanes forms the partials of tree lanes sub + LANES j
// and combines them over the tree's upper levels (offsets 16 down to LANES) in registers; the lower levels are
// shuffles inside the group. Every lane of the group ends with the bits of tree lane 0.
template <class T, int LANES>
__device__ __forceinline__ PassR node_pass_body(const int* segStart, const int* segCount, const double* muArr, const typename Vec2<T>::type* xy,
                                                const typename Vec2<T>::type* ab, const T* area, T R20, T R21, T R22, T tz, T iR, double iRd,
                                                int n, double h, const LevelLanes& L) {
  const int s0 = __ldg(segStart + n), s1 = s0 + __ldg(segCount + n);
  const T hT = static_cast<T>(h);
  const int f = s0 + L.sub;
  SegPartial<T> p;
  if constexpr (LANES == 32) {
    p = segment_partial<T>(xy, ab, area, f, s1, R20, R21, R22, tz, iR, hT);
  } else if constexpr (LANES == 16) {
    SegPartial<T> b;
    segment_pair<T>(xy, ab, area, f, s1, R20, R21, R22, tz, iR, hT, p, b);   // tree lanes sub and sub + 16
    tree_pair(p, b);
  } else if constexpr (LANES == 8) {
    SegPartial<T> b, q, d;
    segment_pair<T>(xy, ab, area, f, s1, R20, R21, R22, tz, iR, hT, p, b);      // sub and sub + 16
    tree_pair(p, b);
    segment_pair<T>(xy, ab, area, f + 8, s1, R20, R21, R22, tz, iR, hT, q, d);  // sub + 8 and sub + 24
    tree_pair(q, d);
    tree_pair(p, q);
  }
#pragma unroll
  for (int off = LANES / 2; off > 0; off >>= 1) {
    p.vol = bsum(p.vol, off, L.mask); p.dv = bsum(p.dv, off, L.mask); p.mx = bsum(p.mx, off, L.mask);
    p.my = bsum(p.my, off, L.mask); p.mz = bsum(p.mz, off, L.mask);
    p.zmin = bmin(p.zmin, off, L.lane, L.mask); p.zmax = bmax(p.zmax, off, L.lane, L.mask);
  }
  const double mu = __ldg(muArr + n);
  PassR r;
  r.vol = static_cast<double>(p.vol) * mu;
  r.dv = static_cast<double>(p.dv) * mu * iRd;
  r.mx = static_cast<double>(p.mx) * mu; r.my = static_cast<double>(p.my) * mu; r.mz = static_cast<double>(p.mz) * mu;
  r.zmin = static_cast<double>(p.zmin); r.zmax = static_cast<double>(p.zmax);
  return r;
}

template <bool MIXED>
__device__ __forceinline__ PassR node_pass(const DevModel& M, const Pose& F, int n, double h, const LevelLanes& L) {
  if constexpr (!MIXED)
    return node_pass_body<double, kLevelLanes<false>>(M.segStart, M.segCount, M.mu, M.segXY, M.segLH, M.segAr, F.R20, F.R21, F.R22, F.tz, F.iR, F.iR, n, h, L);
  else
    return node_pass_body<float, kLevelLanes<true>>(M.segStart, M.segCount, M.mu, M.segXYf, M.segLHf, M.segArf, F.fR20, F.fR21, F.fR22, F.ftz, F.fiR, F.iR, n, h,
                                 L);
}

// ----------------------------------------------------------------------------- per-warp view of the slot in shared memory

struct Slot {
  double *vol, *level, *cx, *cy, *cz, *area, *zmax, *hEff, *aEff, *acc, *dV, *q, *tmp, *hydro;
  int* deg;
  int* misc;
  PassR* passes;
  std::uint8_t* merged;
  Pose* pose;
  Buoy* buoy;
  Parked* parked;
  const unsigned char* cols;  // the column table staged in the block's shared memory, or null (read from global)
};

__device__ __forceinline__ Slot carve_slot(unsigned char* base, const SlotLayout& L) {
  Slot s;
  s.vol = reinterpret_cast<double*>(base + L.vol);
  s.level = reinterpret_cast<double*>(base + L.level);
  s.cx = reinterpret_cast<double*>(base + L.cx);
  s.cy = reinterpret_cast<double*>(base + L.cy);
  s.cz = reinterpret_cast<double*>(base + L.cz);
  s.area = reinterpret_cast<double*>(base + L.area);
  s.zmax = reinterpret_cast<double*>(base + L.zmax);
  s.hEff = reinterpret_cast<double*>(base + L.hEff);
  s.aEff = reinterpret_cast<double*>(base + L.aEff);
  s.acc = reinterpret_cast<double*>(base + L.acc);
  s.dV = reinterpret_cast<double*>(base + L.dV);
  s.q = reinterpret_cast<double*>(base + L.q);
  s.tmp = L.tmp == kSlotAliasDV ? s.dV : reinterpret_cast<double*>(base + L.tmp);
  s.deg = reinterpret_cast<int*>(base + L.deg);
  s.hydro = reinterpret_cast<double*>(base + L.hydro);
  s.misc = reinterpret_cast<int*>(base + L.misc);
  s.passes = reinterpret_cast<PassR*>(base + L.passes);
  s.merged = base + L.merged;
  s.pose = reinterpret_cast<Pose*>(base + L.pose);
  s.buoy = reinterpret_cast<Buoy*>(base + L.buoy);
  s.parked = reinterpret_cast<Parked*>(base + L.parked);
  s.cols = nullptr;
  return s;
}

// ----------------------------------------------------------------------------- free-surface levels (kernel/levels.hpp)
// Group-uniform: the lanes of a level lane group run the solver on identical pass results and store identical values.
// Each solver is a loop around its one node-pass call site, in stages: the passes at the starting level, then either
// the passes at the top of a full node or group (for the centroids) or the passes of the bracketed Newton iteration.

__device__ __forceinline__ void set_centroid(Slot& S, int n, const PassR& p) {
  if (p.vol > kCentroidMinVolume) { S.cx[n] = p.mx / p.vol; S.cy[n] = p.my / p.vol; S.cz[n] = p.mz / p.vol; }
}

enum SolveStage { kStageFirst, kStageFull, kStageNewton };

// Where a step's forward computation records what its reverse (the adjoint, adjoint_kernel.cu) needs: every node pass of
// the level solve (node, pass number within the node's solve, level, result) and the solved levels. The batch kernels
// pass NoTape, whose hooks are empty and compile away.
struct NoTape {
  __device__ __forceinline__ void pass(int, int, double, const PassR&, const LevelLanes&) const {}
  template <int W>
  __device__ __forceinline__ void solved(const DevModel&, const Slot&, const Team<W>&) const {}
};

// One node (levels.hpp:13-49).
template <bool MIXED, class Tape>
__device__ __forceinline__ void solve_single(const DevModel& M, const Pose& F, Slot& S, int n, const LevelLanes& L, const Tape& tape) {
  const double V = S.vol[n], Vmax = __ldg(M.vmax + n);
  const double tol = jmax(1e-3 * Vmax, 0.5);
  double h = S.level[n];
  double hi = 0, a = 0, b = 0;
  int stage = kStageFirst, it = 0, slot = 0;
  PassR p;
  for (;;) {
    p = node_pass<MIXED>(M, F, n, h, L);
    tape.pass(n, slot++, h, p, L);
    if (stage == kStageFirst) {
      const double lo = p.zmin;
      hi = p.zmax;
      S.zmax[n] = hi;
      if (V <= kEmptyVolume) { S.level[n] = lo; S.area[n] = 0; return; }
      if (V >= Vmax * kFullFraction) { stage = kStageFull; h = hi; continue; }
      stage = kStageNewton;
      a = lo; b = hi;
      if (h < lo || h > hi) { h = jmin(hi, jmax(lo, h)); continue; }
    } else if (stage == kStageFull) {
      const double aov = __ldg(M.aov + n);
      S.level[n] = hi + jmax(0.0, V - Vmax) / aov;
      S.area[n] = aov;
      set_centroid(S, n, p);
      return;
    }
    // Newton: p is the pass at h, the it-th of at most kNewtonFast after the starting one
    if (it == kNewtonFast) break;
    const double err = p.vol - V;
    if (fabs(err) < tol) break;
    if (err > 0) b = h; else a = h;
    double hn = p.dv > kSlopeMin ? h - err / p.dv : 0.5 * (a + b);
    if (!(hn > a && hn < b)) hn = 0.5 * (a + b);
    h = hn;
    ++it;
  }
  S.level[n] = h; S.area[n] = p.dv;
  set_centroid(S, n, p);
}

// A merged group of N nodes at one common level (levels.hpp:54-162); P holds the members' passes.
template <bool MIXED, class Tape>
__device__ __forceinline__ void solve_group(const DevModel& M, const Pose& F, Slot& S, PassR* P, const int* m, int N, const LevelLanes& L,
                                            const Tape& tape) {
  double V = 0, Vmax = 0;
  for (int k = 0; k < N; ++k) { V += S.vol[__ldg(m + k)]; Vmax += __ldg(M.vmax + __ldg(m + k)); }
  bool allWet = true;
  int firstWet = -1;
  for (int k = 0; k < N; ++k) {
    if (S.vol[__ldg(m + k)] > 0) { if (firstWet < 0) firstWet = k; }
    else allWet = false;
  }
  double h;
  if (allWet) {
    double s = 0;
    for (int k = 0; k < N; ++k) s += S.level[__ldg(m + k)];
    h = s / static_cast<double>(N);
  } else {
    h = S.level[__ldg(m + (firstWet >= 0 ? firstWet : N - 1))];
  }
  const double tol = jmax(1e-3 * Vmax, 0.5);
  double hi = 0, a = 0, b = 0, dh = 0;
  int stage = kStageFirst, it = 0, slot = 0;
  for (;;) {
    for (int k = 0; k < N; ++k) {
      P[k] = node_pass<MIXED>(M, F, __ldg(m + k), h, L);
      tape.pass(__ldg(m + k), slot, h, P[k], L);
    }
    ++slot;
    if (stage == kStageFirst) {
      for (int k = 0; k < N; ++k) S.zmax[__ldg(m + k)] = P[k].zmax;
      double lo = P[0].zmin;
      hi = P[0].zmax;
      for (int k = 1; k < N; ++k) { if (P[k].zmin < lo) lo = P[k].zmin; if (P[k].zmax > hi) hi = P[k].zmax; }
      if (V <= kEmptyVolume) {
        for (int k = 0; k < N; ++k) { const int n = __ldg(m + k); S.vol[n] = 0; S.level[n] = P[k].zmin; S.area[n] = 0; }
        return;
      }
      if (V >= Vmax * kFullFraction) {
        const double over = jmax(0.0, V - Vmax);
        double aSum = 0;
        for (int k = 0; k < N; ++k) aSum += __ldg(M.aov + __ldg(m + k));
        dh = over / aSum;
        double assigned = 0;
        for (int k = 0; k < N - 1; ++k) {
          const int n = __ldg(m + k);
          const double v = __ldg(M.vmax + n) + dh * __ldg(M.aov + n);
          S.vol[n] = v;
          assigned += v;
        }
        S.vol[__ldg(m + N - 1)] = V - assigned;
        stage = kStageFull;
        h = hi;
        continue;
      }
      stage = kStageNewton;
      a = lo; b = hi;
      if (!(h >= lo && h <= hi)) { h = jmin(hi, jmax(lo, h)); continue; }
    } else if (stage == kStageFull) {
      for (int k = 0; k < N; ++k) {
        const int n = __ldg(m + k);
        S.level[n] = hi + dh; S.area[n] = __ldg(M.aov + n);
        set_centroid(S, n, P[k]);
      }
      return;
    }
    // Newton on the members' summed volume: P holds the passes at h
    if (it == kNewtonFast) break;
    double sum = 0;
    for (int k = 0; k < N; ++k) sum += P[k].vol;
    const double err = sum - V;
    if (fabs(err) < tol) break;
    if (err > 0) b = h; else a = h;
    double dvs = 0;
    for (int k = 0; k < N; ++k) dvs += P[k].dv;
    double hn = dvs > kSlopeMin ? h - err / dvs : 0.5 * (a + b);
    if (!(hn > a && hn < b)) hn = 0.5 * (a + b);
    h = hn;
    ++it;
  }
  double tot = 0;
  for (int k = 0; k < N; ++k) tot += P[k].vol;
  double assigned = 0;
  for (int k = 0; k < N - 1; ++k) {
    const int n = __ldg(m + k);
    double v = tot > 0 ? V * P[k].vol / tot : V / static_cast<double>(N);
    const double vm = __ldg(M.vmax + n);
    if (v > vm) v = vm;
    S.vol[n] = v;
    assigned += v;
  }
  const double vmaxLast = __ldg(M.vmax + __ldg(m + N - 1));
  if (V - assigned > vmaxLast) {
    // the last member would overflow: the ones before it hold V - vmaxLast, filled from the end (levels.hpp:136-155)
    const double need = V - vmaxLast;
    double capped = 0;
    for (int k = N - 2; k >= 0; --k) {
      double prior = 0;
      for (int j = 0; j < k; ++j) prior += S.vol[__ldg(m + j)];
      const int n = __ldg(m + k);
      const double v = (need - capped) - prior;
      const double vm = __ldg(M.vmax + n);
      if (v > vm && k > 0) {
        S.vol[n] = vm;
        capped += vm;
        continue;
      }
      S.vol[n] = v;
      break;
    }
    assigned = 0;
    for (int k = 0; k < N - 1; ++k) assigned += S.vol[__ldg(m + k)];
  }
  S.vol[__ldg(m + N - 1)] = V - assigned;
  for (int k = 0; k < N; ++k) {
    const int n = __ldg(m + k);
    S.level[n] = h; S.area[n] = P[k].dv;
    set_centroid(S, n, P[k]);
  }
}

// Groups are independent (a group's solve reads and writes only its members), so the team's level lane groups take
// them in turn: lane group u of the team (32 / kLevelLanes<MIXED> per warp) solves groups u, u + 32 W / kLevelLanes, ...
// (the reference's block gave them to its eight warps, device_step.cuh:270-281).
template <bool MIXED, int W, class Tape>
__device__ __forceinline__ void solve_levels(const DevModel& M, const Pose& F, Slot& S, const Team<W>& T, const Tape& tape) {
  constexpr int LANES = kLevelLanes<MIXED>, PER_WARP = 32 / LANES;
  LevelLanes L;
  L.lane = T.lane;
  L.sub = T.lane % LANES;
  const int grp = T.lane / LANES;
  if constexpr (LANES == 32) L.mask = kFull;
  else L.mask = ((1u << LANES) - 1u) << (grp * LANES);
  const int unit = T.warp * PER_WARP + grp;
  PassR* P = S.passes + static_cast<std::size_t>(unit) * M.maxGroup;
  // each lane group starts with the group of its own index, then takes the next one from the team's counter
  // (S.misc[2], set to the number of lane groups at the start of the step): the groups take different numbers of
  // passes, and a node's results do not depend on which lane group computes them
  for (int g = unit; g < M.ng;) {
    const int N = __ldg(M.gCount + g);
    const int* m = M.gNodes + __ldg(M.gStart + g);
    const int mode = __ldg(M.gMode + g);
    bool merged = false;
    if (N >= 2) {
      if (mode == 1) {
        merged = true;
      } else if (mode == 2) {
        const double zMw = world_z(F, __ldg(M.gpx + g), __ldg(M.gpy + g), __ldg(M.gpz + g));
        merged = true;
        for (int k = 0; k < N; ++k) {
          const int n = __ldg(m + k);
          if (!(S.vol[n] > kEmptyVolume && S.level[n] > zMw + M.gMargin)) { merged = false; break; }
        }
      }
    }
    S.merged[g] = merged ? 1 : 0;
    if (merged) solve_group<MIXED>(M, F, S, P, m, N, L, tape);
    else for (int k = 0; k < N; ++k) solve_single<MIXED>(M, F, S, __ldg(m + k), L, tape);
    int next = 0;
    if (L.sub == 0) next = atomicAdd(&S.misc[2], 1);
    g = __shfl_sync(L.mask, next, grp * LANES);
  }
  __syncwarp();  // the lane groups leave the loop after different numbers of groups
}

// ----------------------------------------------------------------------------- flows (kernel/flows.hpp:38-78)

__device__ __forceinline__ double connection_flow(const DevModel& M, const Pose& F, double t, const Slot& S, const std::uint8_t* en,
                                                  const double* area, const double* tOn, int c, double& qOut) {
  if (!__ldg(en + c) || __ldg(tOn + c) > t) { qOut = 0; return 0; }
  const int sk = __ldg(M.skip + c);
  if (sk >= 0 && S.merged[sk]) { qOut = 0; return 0; }
  const int a = __ldg(M.ca + c), b = __ldg(M.cb + c);
  const double zo = F.R20 * __ldg(M.kx + c) + F.R21 * __ldg(M.ky + c) + F.R22 * __ldg(M.kz + c) + F.tz;
  const double ha = a < 0 ? 0.0 : S.hEff[a], hbv = S.hEff[b];
  const double Ha = ha > zo ? ha - zo : 0.0, Hb = hbv > zo ? hbv - zo : 0.0;
  double q = 0;
  if (__ldg(M.law + c) == 0) {
    const double d = Ha - Hb;
    if (d != 0) q = __ldg(M.coef + c) * __ldg(area + c) * M.sq2g * d / pm::sqrt_rn(jmax(fabs(d), kOrificeHeadFloor));
  } else {
    const double H1 = Ha > Hb ? Ha : Hb;
    if (H1 > 0) {
      const double H2 = Ha > Hb ? Hb : Ha;
      double f = 1;
      if (H2 > 0) {
        const double r = H2 / H1;
        f = pm::pow(jmax(0.0, 1 - pm::pow(r, kWeirExponent)), kVillemonteExponent);
      }
      q = __ldg(M.coef + c) * __ldg(area + c) * kWeirCoefficient * M.sq2g * H1 * pm::sqrt_rn(H1) * f * (Ha >= Hb ? 1.0 : -1.0);
    }
  }
  if (q == 0) { qOut = 0; return 0; }
  double dV = q * M.dt;
  const int src = dV > 0 ? a : b, dst = dV > 0 ? b : a;
  const double hs = src < 0 ? 0.0 : S.hEff[src];
  const double hd = dst < 0 ? 0.0 : S.hEff[dst];
  const double inv = (src < 0 ? 0.0 : 1 / S.aEff[src]) + (dst < 0 ? 0.0 : 1 / S.aEff[dst]);
  const int degRef = src < 0 ? S.deg[dst] : (dst < 0 ? S.deg[src] : (S.deg[src] > S.deg[dst] ? S.deg[src] : S.deg[dst]));
  const double share = kLimiterShare / static_cast<double>(degRef > 1 ? degRef : 1);
  double lim = inv > 0 ? share * (hs - jmax(hd, zo)) / inv : fabs(dV);
  if (lim < 0) lim = 0;
  if (fabs(dV) > lim) dV = dV > 0 ? lim : -lim;
  qOut = dV / M.dt;
  return dV;
}

// Scalars of one simulation: identical in every lane of its warp.
struct SimRegs {
  double t, zO, pitch, roll, vz, wth, wph, calm;
  double inflow, Vb, hullTop, mw, bx, by, bz;
  int foundered;
  double founderT;
  int evCount;  // warp 0's count is the log's; the other warps' lag
};

// Every thread stores the same values (evCount, which differs between warps, stays in registers).
__device__ __forceinline__ void park(Parked* P, const SimRegs& R) {
  P->t = R.t; P->zO = R.zO; P->pitch = R.pitch; P->roll = R.roll; P->vz = R.vz; P->wth = R.wth; P->wph = R.wph;
  P->calm = R.calm; P->inflow = R.inflow; P->Vb = R.Vb; P->hullTop = R.hullTop; P->mw = R.mw; P->bx = R.bx;
  P->by = R.by; P->bz = R.bz; P->founderT = R.founderT; P->foundered = R.foundered;
}

__device__ __forceinline__ void unpark(const Parked* P, SimRegs& R) {
  R.t = P->t; R.zO = P->zO; R.pitch = P->pitch; R.roll = P->roll; R.vz = P->vz; R.wth = P->wth; R.wph = P->wph;
  R.calm = P->calm; R.inflow = P->inflow; R.Vb = P->Vb; R.hullTop = P->hullTop; R.mw = P->mw; R.bx = P->bx;
  R.by = P->by; R.bz = P->bz; R.founderT = P->founderT; R.foundered = P->foundered;
}

// Instance `inst`'s per-instance arrays. In a batch of one model each pointer is formed where it is used from the
// batch's base pointers (kernel parameters) and inst x the model's sizes, so a thread holds one index rather than
// eight pointers through the step; in a fleet (FLEET) the instance's offsets are loaded once when it is claimed.
template <bool FLEET>
struct InstPtrs;

template <>
struct InstPtrs<false> {
  const DevModel& M;
  const DevBatch& B;
  int inst;
  __device__ __forceinline__ std::size_t perConn() const { return static_cast<std::size_t>(inst) * M.nc; }
  __device__ __forceinline__ std::size_t perEvent() const { return static_cast<std::size_t>(inst) * M.evCap; }
  __device__ __forceinline__ std::size_t perNode() const { return static_cast<std::size_t>(inst) * M.nn; }
  __device__ __forceinline__ std::size_t perMonitor() const { return static_cast<std::size_t>(inst) * M.nmon; }
  __device__ __forceinline__ std::size_t perMark() const { return static_cast<std::size_t>(inst) * M.nmark; }
  __device__ __forceinline__ const std::uint8_t* en() const { return B.en + perConn(); }
  __device__ __forceinline__ const double* area() const { return B.area + perConn(); }
  __device__ __forceinline__ const double* tOn() const { return B.tOn + perConn(); }
  __device__ __forceinline__ double* evT() const { return B.evT + perEvent(); }
  __device__ __forceinline__ std::int32_t* evId() const { return B.evId + perEvent(); }
  __device__ __forceinline__ std::int32_t* evKind() const { return B.evKind + perEvent(); }
  __device__ __forceinline__ double* overT() const { return B.overT + perMonitor(); }
  __device__ __forceinline__ double* markT() const { return B.markT + perMark(); }
};

template <>
struct InstPtrs<true> {
  const DevModel& M;
  const DevBatch& B;
  int inst;
  const std::uint8_t* en_;
  const double *area_, *tOn_;
  double *evT_, *overT_, *markT_;
  std::int32_t *evId_, *evKind_;
  std::size_t node_;
  __device__ __forceinline__ InstPtrs(const DevModel& m, const DevBatch& b, int i) : M(m), B(b), inst(i) {
    const std::size_t c = static_cast<std::size_t>(B.connOff[i]), e = static_cast<std::size_t>(B.evOff[i]);
    en_ = B.en + c; area_ = B.area + c; tOn_ = B.tOn + c;
    evT_ = B.evT + e; evId_ = B.evId + e; evKind_ = B.evKind + e;
    overT_ = B.overT + B.monOff[i]; markT_ = B.markT + B.markOff[i];
    node_ = static_cast<std::size_t>(B.nodeOff[i]);
  }
  __device__ __forceinline__ std::size_t perNode() const { return node_; }
  __device__ __forceinline__ const std::uint8_t* en() const { return en_; }
  __device__ __forceinline__ const double* area() const { return area_; }
  __device__ __forceinline__ const double* tOn() const { return tOn_; }
  __device__ __forceinline__ double* evT() const { return evT_; }
  __device__ __forceinline__ std::int32_t* evId() const { return evId_; }
  __device__ __forceinline__ std::int32_t* evKind() const { return evKind_; }
  __device__ __forceinline__ double* overT() const { return overT_; }
  __device__ __forceinline__ double* markT() const { return markT_; }
};

// The event log belongs to warp 0 of the team: only its lane 0 writes, only its count is stored.
template <class IP>
__device__ __forceinline__ void push_event(const DevModel& M, SimRegs& R, const IP& I, int id, int kind, int lane) {
  if (R.evCount < M.evCap) {
    if (lane == 0) { I.evT()[R.evCount] = R.t; I.evId()[R.evCount] = id; I.evKind()[R.evCount] = kind; }
    R.evCount++;
  }
}

// ----------------------------------------------------------------------------- the step (kernel/step.hpp:41-54)
// Phases that exchange per-node or per-connection arrays are separated by team barriers; per-node and
// per-connection work is spread over all 32 W threads of the team; scalars are computed redundantly and identically
// by every thread, so every decision is uniform across the team.

template <bool MIXED, int W, class IP, class Tape = NoTape>
__device__ __forceinline__ void team_step(const DevModel& M, const Pose& F, SimRegs& R, Slot& S, const IP& I, const Team<W>& T,
                                          const Tape& tape = Tape{}) {
  constexpr int kStride = 32 * W;
  const int lane = T.lane, rank = T.rank;
  const double tNow = R.t;
  park(S.parked, R);  // until the volume update; no thread reads it before the barrier that ends that phase
  if constexpr (W > 8) {
    // The buoyancy's eight trees and the level solve need nothing from each other: the warps without a tree go on to
    // take node groups, and one barrier ends both (16-warp teams: the tail phase 517 against 534 ms on the bench
    // batch, the adjoint's forward 125 against 132 team-s per call; in teams of at most 8 warps, where every warp has
    // trees, the same order made the main phase slower, 2.75 against 2.60 s)
    buoyancy_trees<MIXED, W>(M, F, T, S.hydro, S.cols);
    solve_levels<MIXED, W>(M, F, S, T, tape);
    T.sync();
    *S.buoy = buoyancy_finish(S.hydro);  // every thread stores the same values
  } else {
    *S.buoy = buoyancy<MIXED, W>(M, F, T, S.hydro, S.cols);  // every thread stores the same values
    solve_levels<MIXED, W>(M, F, S, T, tape);
    T.sync();
  }
  // the group counter for the next step's level solve (read after this step's later barriers)
  if (T.leader()) S.misc[2] = W * (32 / kLevelLanes<MIXED>);
  tape.solved(M, S, T);

  // effective heads and areas, then degrees (flows.hpp:15-35)
  for (int n = rank; n < M.nn; n += kStride) {
    const double v = S.vol[n];
    S.hEff[n] = v > kEmptyVolume ? S.level[n] : kNoHead;
    S.aEff[n] = v >= __ldg(M.vmax + n) ? __ldg(M.aov + n) : jmax(S.area[n], __ldg(M.amin + n));
    S.deg[n] = 0;
  }
  T.sync();
  // A node's degree is the number of its incident connections that are enabled and not between two empty spaces. Each
  // such connection counts once at each of its nodes (the incidence lists hold it once at a when a >= 0 and once at b),
  // counted per connection with shared-memory atomics: an integer count, the same in any order, and one round of
  // independent loads instead of a walk down every node's incidence list.
  for (int c = rank; c < M.nc; c += kStride) {
    if (!__ldg(I.en() + c)) continue;
    const int a = __ldg(M.ca + c), b = __ldg(M.cb + c);
    if (a >= 0 && S.hEff[a] < kNoHeadTest && S.hEff[b] < kNoHeadTest) continue;
    if (a >= 0) atomicAdd(&S.deg[a], 1);
    atomicAdd(&S.deg[b], 1);
  }
  T.sync();
  for (int c = rank; c < M.nc; c += kStride) {
    double q;
    S.dV[c] = connection_flow(M, F, tNow, S, I.en(), I.area(), I.tOn(), c, q);
    S.q[c] = q;
  }
  T.sync();
  // per-node gathers in increasing connection order, then the volume update (flows.hpp:81-111)
  for (int n = rank; n < M.nn; n += kStride) {
    const int k0 = __ldg(M.incStart + n), k1 = k0 + __ldg(M.incCount + n);
    double acc = 0;
    for (int k = k0; k < k1; ++k) {
      const double d = S.dV[__ldg(M.incConn + k)];
      acc = __ldg(M.incSide + k) ? acc + d : acc - d;
    }
    double v = S.vol[n] + acc;
    if (v < 0) v = 0;
    const double vm = __ldg(M.vmax + n);
    double excess = 0;
    if (v > vm) {
      const double head = jmax(0.0, -S.zmax[n]);
      const double cap = vm + __ldg(M.aov + n) * head;
      if (v > cap) { excess = v - cap; v = cap; }
    }
    S.acc[n] = excess;
    S.vol[n] = v;
  }
  double seaIn = 0;
  for (int k = 0; k < M.nsea; ++k) seaIn += S.dV[__ldg(M.sea + k)];
  T.sync();
  unpark(S.parked, R);
  // the excess returns to the sea in node order (flows.hpp:114-118)
  for (int n0 = 0; n0 < M.nn; n0 += kLanes) {
    const int n = n0 + lane;
    unsigned mask = __ballot_sync(kFull, n < M.nn && S.acc[n] > 0);
    while (mask) {
      const int b = __ffs(mask) - 1;
      mask &= mask - 1;
      seaIn -= S.acc[n0 + b];
    }
  }
  R.inflow = seaIn / M.dt;
  // the loads' per-node terms overwrite area, zmax, hEff, aEff, acc and dV, all read for the last time above
  T.sync();

  // loads (body.hpp:11-40): per-node terms in parallel, sums in node order
  double* const t0 = S.area;
  double* const t1 = S.zmax;
  double* const t2 = S.hEff;
  double* const t3 = S.aEff;
  double* const t4 = S.acc;
  double* const t5 = S.tmp;
  const Buoy hb = *S.buoy;
  const double Wg = M.rho * M.g;
  const double Fb = Wg * hb.V;
  const double bxw = F.R00 * hb.x + F.R01 * hb.y + F.R02 * hb.z + F.tx;
  const double byw = F.R10 * hb.x + F.R11 * hb.y + F.R12 * hb.z + F.ty;
  double tauX = (byw - M.YO) * Fb, tauY = -(bxw - M.XO) * Fb;
  double Fz = Fb - M.g * M.ms;
  double mw = 0, Iw_p = 0, Iw_r = 0;
  const int NN = M.nn;
  for (int n = rank; n < NN; n += kStride) {
    const double V = S.vol[n];
    if (V <= 0) continue;
    const double x = S.cx[n], y = S.cy[n], z = S.cz[n];
    const double wx = F.R00 * x + F.R01 * y + F.R02 * z + F.tx - M.XO;
    const double wy = F.R10 * x + F.R11 * y + F.R12 * z + F.ty - M.YO;
    const double wz = F.R20 * x + F.R21 * y + F.R22 * z + F.tz - R.zO;
    const double f = -Wg * V;
    const double m = M.rho * V;
    t0[n] = wy * f;
    t1[n] = wx * f;
    t2[n] = f;
    t3[n] = m;
    t4[n] = m * (wx * wx + wz * wz);
    t5[n] = m * (wy * wy + wz * wz);
  }
  T.sync();
  for (int n = 0; n < NN; ++n) {
    if (S.vol[n] <= 0) continue;
    tauX += t0[n]; tauY -= t1[n]; Fz += t2[n];
    mw += t3[n];
    Iw_p += t4[n];
    Iw_r += t5[n];
  }
  const double Mth = tauY, Mph = tauX * F.cth;
  // integrate (body.hpp:42-57)
  const double dt = M.dt;
  const double mh = M.mh0 + mw;
  const double Ith = M.Ith0 + Iw_p, Iph = M.Iph0 + Iw_r;
  const double az = (Fz - M.cDz * R.vz - M.qz * fabs(R.vz) * R.vz) / mh;
  const double ath = (Mth - M.cDth * R.wth - M.qth * fabs(R.wth) * R.wth) / Ith;
  const double aph = (Mph - M.cDph * R.wph - M.qph * fabs(R.wph) * R.wph) / Iph;
  R.vz += az * dt; R.wth += ath * dt; R.wph += aph * dt;
  R.zO += R.vz * dt; R.pitch += R.wth * dt; R.roll += R.wph * dt;
  if (R.pitch > kPitchClamp) { R.pitch = kPitchClamp; R.wth = 0; }
  if (R.pitch < -kPitchClamp) { R.pitch = -kPitchClamp; R.wth = 0; }
  if (R.roll > kRollClamp) { R.roll = kRollClamp; R.wph = 0; }
  if (R.roll < -kRollClamp) { R.roll = -kRollClamp; R.wph = 0; }
  R.t += dt;
  R.Vb = hb.V; R.hullTop = hb.top; R.mw = mw;
  R.bx = hb.x; R.by = hb.y; R.bz = hb.z;

  // events (events.hpp:11-38): monitors in order, marks in order, then the founder rule; warp 0 keeps the log
  if (T.warp == 0) {
  for (int m0 = 0; m0 < M.nmon; m0 += kLanes) {
    const int m = m0 + lane;
    bool fire = false;
    if (m < M.nmon && I.overT()[m] < 0) {
      const int k0 = __ldg(M.monStart + m), k1 = k0 + __ldg(M.monCount + m);
      double over = 0;
      for (int k = k0; k < k1; ++k) {
        const double qc = S.q[__ldg(M.monConn + k)];
        if (qc > 0) over += qc;
      }
      fire = over > M.monThreshold;
      if (fire) I.overT()[m] = R.t;
    }
    unsigned mask = __ballot_sync(kFull, fire);
    while (mask) {
      const int b = __ffs(mask) - 1;
      mask &= mask - 1;
      push_event(M, R, I, m0 + b, 0, lane);
    }
  }
  for (int i0 = 0; i0 < M.nmark; i0 += kLanes) {
    const int i = i0 + lane;
    bool fire = false;
    if (i < M.nmark && I.markT()[i] < 0) {
      const double wz = world_z(F, __ldg(M.mkx + i), __ldg(M.mky + i), __ldg(M.mkz + i));
      const bool under = __ldg(M.mkWhen + i) == 0;
      fire = (under && wz < 0) || (!under && wz > 0);
      if (fire) I.markT()[i] = R.t;
    }
    unsigned mask = __ballot_sync(kFull, fire);
    while (mask) {
      const int b = __ffs(mask) - 1;
      mask &= mask - 1;
      push_event(M, R, I, i0 + b, 1, lane);
    }
  }
  }
  if (!R.foundered && (R.hullTop < M.hullTopBelow || fabs(R.pitch) > M.pitchAbsAbove || (R.Vb < M.buoyancyBelow && R.t > M.minT))) {
    R.foundered = 1;
    R.founderT = R.t;
    if (T.warp == 0) push_event(M, R, I, -1, 2, lane);
  }
  T.sync();
}

// Readouts at the current state (kernel/readouts.hpp:20-36): t, trim, list, water (t), inflow (t/min), draftF, draftA.
__device__ __forceinline__ void readouts(const DevModel& M, const SimRegs& R, const Slot& S, double* r7) {
  const Pose F = make_pose(M, R.zO, R.pitch, R.roll);
  double water = 0;
  for (int n = 0; n < M.nn; ++n) water += S.vol[n];
  r7[0] = R.t;
  r7[1] = R.pitch * 180 / kPi;
  r7[2] = R.roll * 180 / kPi;
  r7[3] = water * M.rho / 1000;
  r7[4] = R.inflow * M.rho / 1000 * 60;
  r7[5] = -world_z(F, M.xFP, 0, 0);
  r7[6] = -world_z(F, M.xAP, 0, 0);
}

}  // namespace ssb
