// The reverse (adjoint) of one time step in the portable numerics, FP64 throughout: given the adjoint of the state
// after a step (how much the objective changes per unit change of each state value) and the step's tape (what its
// forward computation recorded), it returns the adjoint of the state before the step and adds the step's share of
// the gradient with respect to every connection area.
//
// It differentiates the branch path the forward step takes (kernel::step, engine/include/sinksim/kernel/step.hpp:41-54):
//   * pose (frame.hpp:9-21): sin / cos by their derivatives at the recorded values;
//   * buoyancy (hydro.hpp:241-258, reduce.hpp:39-49): a column cut by the waterplane contributes through its wet
//     height, a dry or fully submerged one does not (the clip is piecewise linear; its kinks have measure zero);
//   * the level solve (levels.hpp:13-188): the recorded node passes are replayed through the solver's own decisions
//     (start, clamp, Newton or bisection update, break, full/empty cases, the merged group's proportional sharing), and
//     each update is differentiated as executed, Newton iterate by Newton iterate: a level that the solver left
//     unchanged because the volume error was inside its tolerance passes the previous level's adjoint through, one
//     that took a Newton step takes the volume's. A node pass contributes through the segments the level cuts
//     (d vol / d h = the free-surface area, which the pass itself returns) and through its pose; the lowest segment
//     bottom and highest top (a node's world extent) through the segment the reduction tree selects;
//   * flows (flows.hpp:38-118): orifice and weir laws with the Villemonte factor, the limiter when it binds (the flow
//     then follows the levels and areas, not the connection area), clamps at zero, the volume update and its cap;
//   * loads and the semi-implicit integration (body.hpp:11-57), with the pitch and roll clamps.
// Events and the founder rule never feed back into the physics and have no adjoint. The gradient with respect to a
// connection area comes only from that connection's flow law: area enters nowhere else.
//
// The functions here are host-and-device code: the GPU adjoint kernel (adjoint_kernel.cu) runs them with a team of
// warps, and the test harness runs the same code on the CPU with a one-thread team, against the FP64 tangent-linear
// restatement. A team type T provides rank / size (threads), warp / nwarps, lane / width (lanes per warp), sync(),
// warp_sum(x) (the sum over the warp's lanes, held by every lane) and reduce(values, K) (team-wide sums).
#pragma once

#include <cstddef>
#include <cstdint>

#include "device_model.h"
#include "portable_math.cuh"
#include "scheme.h"

namespace ssb {
namespace adj {

// Node passes of one node in one step's level solve, at most: the start, a clamped start or the pass at the top of a
// full node, and the solver's six Newton iterations.
constexpr int kMaxPasses = 8;
// Doubles per recorded node pass: level, vol, dv, mx, my, mz, zmin, zmax.
constexpr int kPassFields = 8;
// Members of a merged group that the adjoint handles (the reference's compiled hulls merge pairs).
constexpr int kMaxMembers = 4;

// Error bits an adjoint run reports (AdjointBatch::error): the step took a branch without an adjoint here, or the
// replay of the level solve did not meet the recorded passes.
enum AdjointError : std::int32_t { kErrCascade = 1, kErrReplay = 2, kErrGroupSize = 4 };

// Offsets (in doubles, then in int32 after the doubles) of one step's tape.
struct TapeLayout {
  std::size_t scal, pose, buoy, volIn, levelIn, cxIn, cyIn, czIn, volS, levelS, areaS, cxS, cyS, czS, zmaxS, passes, doubles;
  std::size_t npass, merged, ints, bytes;
};

SSB_HD TapeLayout tape_layout(int nn, int ng) {
  TapeLayout L{};
  const auto N = static_cast<std::size_t>(nn);
  std::size_t o = 0;
  L.scal = o; o += 7;    // t, zO, pitch, roll, vz, wth, wph before the step
  L.pose = o; o += 14;   // R00 .. R22, tx, ty, tz, cth, iR of the step
  L.buoy = o; o += 4;    // V, x, y, z of the step's buoyancy
  L.volIn = o; o += N; L.levelIn = o; o += N; L.cxIn = o; o += N; L.cyIn = o; o += N; L.czIn = o; o += N;
  L.volS = o; o += N; L.levelS = o; o += N; L.areaS = o; o += N; L.cxS = o; o += N; L.cyS = o; o += N; L.czS = o; o += N;
  L.zmaxS = o; o += N;
  L.passes = o; o += N * kMaxPasses * kPassFields;
  L.doubles = o;
  std::size_t i = 0;
  L.npass = i; i += N;
  L.merged = i; i += static_cast<std::size_t>(ng);
  L.ints = i;
  L.bytes = (L.doubles * sizeof(double) + L.ints * sizeof(std::int32_t) + 15) & ~static_cast<std::size_t>(15);
  return L;
}

// A step's tape in memory: doubles, then int32.
struct Tape {
  double* d;
  std::int32_t* i;
  TapeLayout L;
  SSB_HD double* pass(int n, int k) const { return d + L.passes + (static_cast<std::size_t>(n) * kMaxPasses + k) * kPassFields; }
};

SSB_HD Tape tape_at(unsigned char* base, const TapeLayout& L) {
  Tape t;
  t.d = reinterpret_cast<double*>(base);
  t.i = reinterpret_cast<std::int32_t*>(base + L.doubles * sizeof(double));
  t.L = L;
  return t;
}

// Forward pose values of a step, as recorded.
struct PoseD {
  double R00, R01, R02, R10, R11, R12, R20, R21, R22, tx, ty, tz, cth, iR;
};

// Adjoint of a pose (and of 1 / R22, which the passes use).
struct AdjPose {
  double R00, R01, R02, R10, R11, R12, R20, R21, R22, tx, ty, tz, cth, iR;
};
constexpr int kAdjPoseFields = 14;

SSB_HD void zero(AdjPose& a) {
  a.R00 = a.R01 = a.R02 = a.R10 = a.R11 = a.R12 = a.R20 = a.R21 = a.R22 = a.tx = a.ty = a.tz = a.cth = a.iR = 0;
}
SSB_HD double* fields(AdjPose& a) { return &a.R00; }

SSB_HD PoseD load_pose(const double* p) {
  PoseD F;
  F.R00 = p[0]; F.R01 = p[1]; F.R02 = p[2]; F.R10 = p[3]; F.R11 = p[4]; F.R12 = p[5]; F.R20 = p[6]; F.R21 = p[7]; F.R22 = p[8];
  F.tx = p[9]; F.ty = p[10]; F.tz = p[11]; F.cth = p[12]; F.iR = p[13];
  return F;
}

// The forward pose (frame.hpp:9-21) with portable sin / cos: the same operations as the step's.
SSB_HD PoseD pose_of(const DevModel& M, double zO, double th, double ph) {
  const double cth = pm::cos(th), sth = pm::sin(th), cph = pm::cos(ph), sph = pm::sin(ph);
  PoseD F;
  F.R00 = cth; F.R01 = sth * sph; F.R02 = sth * cph;
  F.R10 = 0;   F.R11 = cph;       F.R12 = -sph;
  F.R20 = -sth; F.R21 = cth * sph; F.R22 = cth * cph;
  F.tx = M.XO - (F.R00 * M.g0x + F.R01 * M.g0y + F.R02 * M.g0z);
  F.ty = M.YO - (F.R10 * M.g0x + F.R11 * M.g0y + F.R12 * M.g0z);
  F.tz = zO - (F.R20 * M.g0x + F.R21 * M.g0y + F.R22 * M.g0z);
  F.cth = cth;
  F.iR = 1 / F.R22;
  return F;
}

// Adjoint of the pose with respect to (zO, pitch, roll), added to a_zO, a_th, a_ph.
SSB_HD void pose_reverse(const DevModel& M, const PoseD& F, AdjPose a, double& a_zO, double& a_th, double& a_ph) {
  const double cth = F.R00, sth = -F.R20, cph = F.R11, sph = -F.R12;
  a.R22 -= a.iR * F.iR * F.iR;
  a_zO += a.tz;
  a.R20 -= a.tz * M.g0x; a.R21 -= a.tz * M.g0y; a.R22 -= a.tz * M.g0z;
  a.R10 -= a.ty * M.g0x; a.R11 -= a.ty * M.g0y; a.R12 -= a.ty * M.g0z;
  a.R00 -= a.tx * M.g0x; a.R01 -= a.tx * M.g0y; a.R02 -= a.tx * M.g0z;
  double a_cth = a.cth + a.R00 + a.R21 * sph + a.R22 * cph;
  double a_sth = a.R01 * sph + a.R02 * cph - a.R20;
  double a_cph = a.R02 * sth + a.R11 + a.R22 * cth;
  double a_sph = a.R01 * sth - a.R12 + a.R21 * cth;
  a_th += -sth * a_cth + cth * a_sth;
  a_ph += -sph * a_cph + cph * a_sph;
}

// The objective's readouts of a state: trim (degrees) and heave, the mean of the forward and aft drafts
// (kernel/readouts.hpp:20-36: draft = -world height of (x, 0, 0)).
SSB_HD void trim_heave(const DevModel& M, const PoseD& F, double pitch, double& trim, double& heave) {
  trim = pitch * 180 / kPi;
  const double dF = -(F.R20 * M.xFP + F.R21 * 0 + F.R22 * 0 + F.tz);
  const double dA = -(F.R20 * M.xAP + F.R21 * 0 + F.R22 * 0 + F.tz);
  heave = 0.5 * (dF + dA);
}

SSB_HD void trim_heave_reverse(const DevModel& M, double a_trim, double a_heave, AdjPose& aP, double& a_pitch) {
  a_pitch += a_trim * 180 / kPi;
  const double a_d = 0.5 * a_heave;  // both drafts
  aP.R20 -= a_d * (M.xFP + M.xAP);
  aP.tz -= 2 * a_d;
}

// ----------------------------------------------------------------------------- reductions over lanes

// Inclusive prefix sum of v over the lanes 0 .. lane of the warp (width 1: v itself).
SSB_HD int lane_prefix(int v, int lane, int width) {
#if defined(__CUDA_ARCH__)
  if (width == 32)
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
#endif
  (void)lane;
  (void)width;
  return v;
}

// The value of lane `src` (width 1: v itself).
SSB_HD int lane_value(int v, int src, int width) {
#if defined(__CUDA_ARCH__)
  if (width == 32) return __shfl_sync(0xffffffffu, v, src);
#endif
  (void)src;
  (void)width;
  return v;
}

SSB_HD double lane_sum(double v, int width) {
#if defined(__CUDA_ARCH__)
  if (width == 32)
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
#endif
  return v;
}

// The segment of node n that the node pass's 32-lane tree selects as the lowest segment bottom (want_min) or the highest
// top: each tree lane l scans segments s0 + l + 32 k keeping the first strict improvement, and the tree combines lane l
// with lane l + off (off = 16 .. 1), the lower lane winning ties (kernel/reduce.hpp:52-71 and :12-37). On the device
// the warp's lanes are the tree's lanes; on the host the lanes are emulated.
SSB_HD int pass_extreme(const DevModel& M, const PoseD& F, int n, bool want_min, int lane, int width) {
  const int s0 = M.segStart[n], s1 = s0 + M.segCount[n];
#if defined(__CUDA_ARCH__)
  if (width == 32) {
    double best = want_min ? 1e9 : -1e9;
    int idx = -1;
    auto seg = [&](const double2 xy, const double2 ab, int j) {
      const double base = F.R20 * xy.x + F.R21 * xy.y + F.tz;
      const double w = want_min ? base + F.R22 * ab.x : base + F.R22 * ab.y;
      if (want_min ? (w < best) : (w > best)) { best = w; idx = j; }
    };
    // two segments per round, both loaded before either is compared; each lane keeps its segments' order
    int j = s0 + lane;
    for (; j + 32 < s1; j += 64) {
      const double2 xy0 = M.segXY[j], ab0 = M.segLH[j], xy1 = M.segXY[j + 32], ab1 = M.segLH[j + 32];
      seg(xy0, ab0, j);
      seg(xy1, ab1, j + 32);
    }
    if (j < s1) seg(M.segXY[j], M.segLH[j], j);
    for (int off = 16; off > 0; off >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, off);
      const int oi = __shfl_xor_sync(0xffffffffu, idx, off);
      const bool lower = (lane & off) == 0;
      const double va = lower ? best : ob, vb = lower ? ob : best;
      const int ia = lower ? idx : oi, ib = lower ? oi : idx;
      const bool takeB = want_min ? (vb < va) : (vb > va);
      best = takeB ? vb : va;
      idx = takeB ? ib : ia;
    }
    return idx;
  }
#endif
  double best[32];
  int idx[32];
  for (int l = 0; l < 32; ++l) {
    best[l] = want_min ? 1e9 : -1e9;
    idx[l] = -1;
    for (int j = s0 + l; j < s1; j += 32) {
      const double2 xy = M.segXY[j], ab = M.segLH[j];
      const double base = F.R20 * xy.x + F.R21 * xy.y + F.tz;
      const double w = want_min ? base + F.R22 * ab.x : base + F.R22 * ab.y;
      if (want_min ? (w < best[l]) : (w > best[l])) { best[l] = w; idx[l] = j; }
    }
  }
  for (int off = 16; off > 0; off >>= 1)
    for (int l = 0; l < off; ++l)
      if (want_min ? (best[l + off] < best[l]) : (best[l + off] > best[l])) { best[l] = best[l + off]; idx[l] = idx[l + off]; }
  (void)lane;
  return idx[0];
}

// Adjoint of the world height of segment j's bottom (want_min) or top with respect to the pose.
SSB_HD void extreme_reverse(const DevModel& M, int j, bool bottom, double a_w, AdjPose& aP) {
  if (j < 0 || a_w == 0) return;
  const double2 xy = M.segXY[j], ab = M.segLH[j];
  aP.R20 += a_w * xy.x; aP.R21 += a_w * xy.y; aP.tz += a_w;
  aP.R22 += a_w * (bottom ? ab.x : ab.y);
}

// ----------------------------------------------------------------------------- node-pass reverse over segments

// Reverse of a node pass of node n at level h with adjoints av/amx/amy/amz of its (permeability-scaled) vol and
// moments: adds the pose adjoint to aP and returns this lane's share of d(outputs)/d h (sum over the warp's lanes for
// the total). Only segments the level cuts contribute (kernel/reduce.hpp:52-71: a full segment's height is b - a, a dry
// one adds nothing).
SSB_HD double pass_sweep1(const DevModel& M, const PoseD& F, int n, double h, double av, double amx, double amy, double amz, int lane, int width,
                          AdjPose& aP) {
  const int s0 = M.segStart[n], s1 = s0 + M.segCount[n];
  const double mu = M.mu[n];
  double aR20 = 0, aR21 = 0, atz = 0, aiR = 0, ah = 0;
  auto seg = [&](const double2 xy, const double2 ab, const double A) {
    const double base = F.R20 * xy.x + F.R21 * xy.y + F.tz;
    const double zp = (h - base) * F.iR;
    if (!(zp > ab.x && zp < ab.y)) return;
    const double L = zp - ab.x;
    const double aL = A * mu * (av + amx * xy.x + amy * xy.y + amz * (ab.x + L));
    ah += aL * F.iR;
    aiR += aL * (h - base);
    const double abase = -aL * F.iR;
    aR20 += abase * xy.x; aR21 += abase * xy.y; atz += abase;
  };
  // two segments per round, both loaded before either is used; each lane still visits its segments in order
  int j = s0 + lane;
  for (; j + width < s1; j += 2 * width) {
    const double2 xy0 = M.segXY[j], ab0 = M.segLH[j], xy1 = M.segXY[j + width], ab1 = M.segLH[j + width];
    const double A0 = M.segAr[j], A1 = M.segAr[j + width];
    seg(xy0, ab0, A0);
    seg(xy1, ab1, A1);
  }
  if (j < s1) seg(M.segXY[j], M.segLH[j], M.segAr[j]);
  aP.R20 += aR20; aP.R21 += aR21; aP.tz += atz; aP.iR += aiR;
  return ah;
}

// The pose adjoint of np passes of node n at levels h[i] whose vol has the adjoint av[i] and whose moments have none
// (their level adjoints are not needed).
SSB_HD void pass_sweep_levels(const DevModel& M, const PoseD& F, int n, int np, const double* h, const double* av, int lane, int width,
                              AdjPose& aP) {
  const int s0 = M.segStart[n], s1 = s0 + M.segCount[n];
  const double mu = M.mu[n];
  double aR20 = 0, aR21 = 0, atz = 0, aiR = 0;
  auto seg = [&](const double2 xy, const double2 ab, const double A) {
    const double base = F.R20 * xy.x + F.R21 * xy.y + F.tz;
    for (int i = 0; i < np; ++i) {
      const double zp = (h[i] - base) * F.iR;
      if (!(zp > ab.x && zp < ab.y)) continue;
      const double aL = A * mu * av[i];
      aiR += aL * (h[i] - base);
      const double abase = -aL * F.iR;
      aR20 += abase * xy.x; aR21 += abase * xy.y; atz += abase;
    }
  };
  int j = s0 + lane;
  for (; j + width < s1; j += 2 * width) {
    const double2 xy0 = M.segXY[j], ab0 = M.segLH[j], xy1 = M.segXY[j + width], ab1 = M.segLH[j + width];
    const double A0 = M.segAr[j], A1 = M.segAr[j + width];
    seg(xy0, ab0, A0);
    seg(xy1, ab1, A1);
  }
  if (j < s1) seg(M.segXY[j], M.segLH[j], M.segAr[j]);
  aP.R20 += aR20; aP.R21 += aR21; aP.tz += atz; aP.iR += aiR;
}

// Reverse of the buoyancy integral (kernel/reduce.hpp:39-49) over this thread's columns first, first + stride, ...: the
// adjoints of V, Mx, My, Mz into the pose adjoint. A column cut by the waterplane contributes through its wet height.
SSB_HD void buoyancy_sweep(const DevModel& M, const PoseD& F, double aV, double aMx, double aMy, double aMz, int first, int stride,
                           AdjPose& aP) {
  double aR20 = 0, aR21 = 0, atz = 0, aiR = 0;
  auto col = [&](const double2 xy, const double2 lh, const double A) {
    const double base = F.R20 * xy.x + F.R21 * xy.y + F.tz;
    const double zp = -base * F.iR;
    if (!(zp > lh.x && zp < lh.y)) return;
    const double s = zp - lh.x;
    const double as = A * (aV + aMx * xy.x + aMy * xy.y + aMz * (lh.x + s));
    aiR -= as * base;
    const double abase = -as * F.iR;
    aR20 += abase * xy.x; aR21 += abase * xy.y; atz += abase;
  };
  // two columns per round, both loaded before either is used; each thread keeps its columns' order
  int i = first;
  for (; i + stride < M.ncol; i += 2 * stride) {
    const double2 xy0 = M.colXY[i], lh0 = M.colLH[i], xy1 = M.colXY[i + stride], lh1 = M.colLH[i + stride];
    const double A0 = M.colA[i], A1 = M.colA[i + stride];
    col(xy0, lh0, A0);
    col(xy1, lh1, A1);
  }
  if (i < M.ncol) col(M.colXY[i], M.colLH[i], M.colA[i]);
  aP.R20 += aR20; aP.R21 += aR21; aP.tz += atz; aP.iR += aiR;
}

// ----------------------------------------------------------------------------- the level solve, replayed and reversed

// One unit of the level solve (a merged group, or a node solved alone) replayed from its recorded passes: which case
// the solver took and, per Newton update, whether it was a Newton or a bisection step and where the bracket ends came
// from (a pass index, or kSrcLo / kSrcHi for the node's world extent).
constexpr int kSrcLo = -1, kSrcHi = -2;

struct Replay {
  int N;
  int members[kMaxMembers];
  bool single;
  int cs;          // 0 empty, 1 full, 2 Newton
  int base, K;     // the first Newton pass (1 when the start was clamped into the extent), the final pass
  int startSrc;    // where the first Newton level came from when clamped (kSrcLo / kSrcHi); the start otherwise
  int loSrc, hiSrc;
  double V, Vmax, h0;
  bool allWet;
  int firstWet;
  bool newton[kMaxPasses];
  int aSrc[kMaxPasses], bSrc[kMaxPasses];
  bool ok;
};

static_assert(sizeof(Replay) % sizeof(std::int32_t) == 0, "a replay is copied in 32-bit words");

SSB_HD const double* rec(const Tape& t, int n, int k) { return t.pass(n, k); }

// Replays the solver's decisions (levels.hpp:13-49 for a node alone, :54-162 for a merged group) on the recorded passes,
// into r.
SSB_HD void replay_unit(const DevModel& M, const Tape& t, const int* members, int N, bool single, Replay& r) {
  r.N = N;
  r.single = single;
  r.ok = N <= kMaxMembers;
  r.cs = 0; r.base = 0; r.K = 0; r.startSrc = 0; r.loSrc = 0; r.hiSrc = 0;
  if (!r.ok) return;
  for (int k = 0; k < N; ++k) r.members[k] = members[k];
  const double* volIn = t.d + t.L.volIn;
  const double* levelIn = t.d + t.L.levelIn;
  double V = 0, Vmax = 0;
  for (int k = 0; k < N; ++k) { V += volIn[members[k]]; Vmax += M.vmax[members[k]]; }
  r.V = V; r.Vmax = Vmax;
  bool allWet = true;
  int firstWet = -1;
  for (int k = 0; k < N; ++k) {
    if (volIn[members[k]] > 0) { if (firstWet < 0) firstWet = k; }
    else allWet = false;
  }
  r.allWet = allWet; r.firstWet = firstWet;
  double h;
  if (single) {
    h = levelIn[members[0]];
  } else if (allWet) {
    double s = 0;
    for (int k = 0; k < N; ++k) s += levelIn[members[k]];
    h = s / static_cast<double>(N);
  } else {
    h = levelIn[members[firstWet >= 0 ? firstWet : N - 1]];
  }
  r.h0 = h;
  // the extent: the members' start passes
  double lo = rec(t, members[0], 0)[6], hi = rec(t, members[0], 0)[7];
  int loSrc = 0, hiSrc = 0;
  for (int k = 1; k < N; ++k) {
    const double* p = rec(t, members[k], 0);
    if (p[6] < lo) { lo = p[6]; loSrc = k; }
    if (p[7] > hi) { hi = p[7]; hiSrc = k; }
  }
  if (single) {
    // a node alone: the same extent as a group of one
    loSrc = 0; hiSrc = 0;
  }
  r.loSrc = loSrc; r.hiSrc = hiSrc;
  bool ok = true;
  for (int k = 0; k < N; ++k) ok = ok && rec(t, members[k], 0)[0] == h;
  if (V <= kEmptyVolume) { r.cs = 0; r.K = 0; r.ok = ok; return; }
  if (V >= Vmax * kFullFraction) { r.cs = 1; r.K = 1; r.ok = ok; return; }
  r.cs = 2;
  int base = 0;
  const bool clamp = single ? (h < lo || h > hi) : !(h >= lo && h <= hi);
  if (clamp) {
    const double hc = jmin(hi, jmax(lo, h));
    r.startSrc = h < lo ? kSrcLo : kSrcHi;
    h = hc;
    base = 1;
    for (int k = 0; k < N; ++k) ok = ok && rec(t, members[k], 1)[0] == h;
  }
  r.base = base;
  const double tol = jmax(1e-3 * Vmax, 0.5);
  double a = lo, b = hi;
  int aS = kSrcLo, bS = kSrcHi;
  int k = base;
  for (int it = 0; it < kNewtonFast; ++it) {
    double sum = 0, dvs = 0;
    for (int q = 0; q < N; ++q) sum += rec(t, members[q], k)[1];
    const double err = single ? rec(t, members[0], k)[1] - V : sum - V;
    if (fabs(err) < tol) break;
    if (err > 0) { b = h; bS = k; } else { a = h; aS = k; }
    for (int q = 0; q < N; ++q) dvs += rec(t, members[q], k)[2];
    if (single) dvs = rec(t, members[0], k)[2];
    double hn = dvs > kSlopeMin ? h - err / dvs : 0.5 * (a + b);
    bool nw = dvs > kSlopeMin;
    if (!(hn > a && hn < b)) { hn = 0.5 * (a + b); nw = false; }
    r.newton[k] = nw;
    r.aSrc[k] = aS; r.bSrc[k] = bS;
    h = hn;
    ++k;
    for (int q = 0; q < N; ++q) ok = ok && rec(t, members[q], k)[0] == h;
  }
  r.K = k;
  r.ok = ok;
}

// Adjoint inputs and outputs of one unit, per member: the solved values' adjoints in, the start values' adjoints out.
struct UnitAdj {
  // in (per member k): adjoints of the solved level, area, centroid, volume and extent top (zmax)
  double aLevel[kMaxMembers], aArea[kMaxMembers], aCx[kMaxMembers], aCy[kMaxMembers], aCz[kMaxMembers], aVol[kMaxMembers], aZmax[kMaxMembers];
  // out: adjoints of the step's starting volume, level and centroid
  double oVol[kMaxMembers], oLevel[kMaxMembers], oCx[kMaxMembers], oCy[kMaxMembers], oCz[kMaxMembers];
};

// Working memory of one unit's reverse, one per warp (shared memory on the device; the host harness keeps one on its
// stack). Its scalars are the same for every lane of the warp: lane 0 alone writes them, and the lanes read them after
// a warp sync, so no lane reads a value another is still updating.
struct UnitWork {
  Replay r;
  UnitAdj u;
  double av[kMaxMembers][kMaxPasses], adv[kMaxMembers][kMaxPasses];  // adjoints of each pass's vol and dv
  double amx[kMaxMembers], amy[kMaxMembers], amz[kMaxMembers];        // of the final pass's moments
  double hFinal[kMaxMembers];                                         // the final pass's level
  double ah[kMaxPasses];                                              // adjoints of the levels h_j
  double aZmin0[kMaxMembers], aZmax0[kMaxMembers];                    // of the members' extent bottom and top
  double hs[kMaxMembers][kMaxPasses], pv[kMaxMembers][kMaxPasses];    // the earlier passes the pose sweep visits
  int np[kMaxMembers];
  double aV, aLo, aHi, aH0;
  int err;
};

SSB_HD void warp_sync() {
#if defined(__CUDA_ARCH__)
  __syncwarp();
#endif
}

// Centroid of a pass (set_centroid, levels.hpp:46): adjoint of cx = mx / vol etc. into the pass's vol and moments, or the
// previous centroid's adjoint when the pass held too little water to move it.
SSB_HD void centroid_reverse(const double* p, double aCx, double aCy, double aCz, double& av, double& amx, double& amy, double& amz,
                             double& oCx, double& oCy, double& oCz) {
  if (p[1] > kCentroidMinVolume) {
    const double v = p[1];
    amx += aCx / v; amy += aCy / v; amz += aCz / v;
    av -= (aCx * (p[3] / v) + aCy * (p[4] / v) + aCz * (p[5] / v)) / v;
  } else {
    oCx += aCx; oCy += aCy; oCz += aCz;
  }
}

// Reverse of one unit, run by the lanes of one warp: lane 0 does the unit's scalar work in w, the lanes split the
// segment sweeps. Adds pose adjoints to aP (this lane's share) and returns false when the unit took a branch without an
// adjoint here (the cascade of levels.hpp:136-155), its error bit in *err. On entry w.r holds the replay and w.u's
// inputs are set (written by lane 0, then a warp sync); on return w.u's outputs are set (lane 0's, before the caller's
// warp sync).
SSB_HD bool unit_reverse(const DevModel& M, const PoseD& F, const Tape& t, UnitWork& w, int lane, int width, AdjPose& aP, int* err) {
  const Replay& r = w.r;
  UnitAdj& u = w.u;
  const int N = r.N;
  const int K = r.K;
  if (lane == 0) {
    for (int k = 0; k < N; ++k) {
      for (int i = 0; i <= K; ++i) w.av[k][i] = w.adv[k][i] = 0;
      w.amx[k] = w.amy[k] = w.amz[k] = 0;
      w.aZmin0[k] = 0;
      w.aZmax0[k] = u.aZmax[k];  // each member's own extent top is recorded from its start pass
      w.np[k] = 0;
      u.oVol[k] = u.oLevel[k] = u.oCx[k] = u.oCy[k] = u.oCz[k] = 0;
    }
    for (int i = 0; i <= K; ++i) w.ah[i] = 0;
    w.aV = w.aLo = w.aHi = w.aH0 = 0;
    w.err = 0;
    if (r.cs == 0) {
      // empty: the level is the member's own extent bottom; a group empties its members, a node alone keeps its volume
      for (int k = 0; k < N; ++k) {
        w.aZmin0[k] += u.aLevel[k];
        if (r.single) w.aV += u.aVol[k];
        u.oCx[k] += u.aCx[k]; u.oCy[k] += u.aCy[k]; u.oCz[k] += u.aCz[k];
      }
    } else if (r.cs == 1) {
      // full: volumes vmax + dh aov (the last takes the rest), level hi + dh, centroids at the top (levels.hpp:29-35, :91-111)
      double aSum = 0;
      for (int k = 0; k < N; ++k) aSum += M.aov[r.members[k]];
      double aDh = 0;
      double aV = u.aVol[N - 1];
      for (int k = 0; k < N - 1; ++k) aDh += (u.aVol[k] - u.aVol[N - 1]) * M.aov[r.members[k]];
      double aHi = 0;
      for (int k = 0; k < N; ++k) { aDh += u.aLevel[k]; aHi += u.aLevel[k]; }
      if (r.V - r.Vmax > 0) aV += aDh / aSum;
      w.aV = aV;
      w.aHi = aHi;
      for (int k = 0; k < N; ++k) {
        const double* p = rec(t, r.members[k], 1);
        centroid_reverse(p, u.aCx[k], u.aCy[k], u.aCz[k], w.av[k][1], w.amx[k], w.amy[k], w.amz[k], u.oCx[k], u.oCy[k], u.oCz[k]);
        w.hFinal[k] = p[0];
      }
    } else {
      // Newton: level h_K, area and centroid of the final passes, the group's water shared in proportion to them
      for (int k = 0; k < N; ++k) {
        w.ah[K] += u.aLevel[k];
        w.adv[k][K] += u.aArea[k];
        const double* p = rec(t, r.members[k], K);
        centroid_reverse(p, u.aCx[k], u.aCy[k], u.aCz[k], w.av[k][K], w.amx[k], w.amy[k], w.amz[k], u.oCx[k], u.oCy[k], u.oCz[k]);
        w.hFinal[k] = p[0];
      }
      if (r.single) {
        w.aV += u.aVol[0];
      } else {
        double tot = 0;
        for (int k = 0; k < N; ++k) tot += rec(t, r.members[k], K)[1];
        double assigned = 0, aTot = 0;
        double aV = u.aVol[N - 1];
        for (int k = 0; k < N - 1; ++k) {
          const double pk = rec(t, r.members[k], K)[1];
          double v = tot > 0 ? r.V * pk / tot : r.V / static_cast<double>(N);
          const bool capped = v > M.vmax[r.members[k]];
          if (capped) v = M.vmax[r.members[k]];
          assigned += v;
          const double a = u.aVol[k] - u.aVol[N - 1];
          if (capped) continue;
          if (tot > 0) {
            aV += a * pk / tot;
            w.av[k][K] += a * r.V / tot;
            aTot -= a * v / tot;
          } else {
            aV += a / static_cast<double>(N);
          }
        }
        w.aV = aV;
        if (r.V - assigned > M.vmax[r.members[N - 1]]) w.err = kErrCascade;
        else if (aTot != 0)
          for (int k = 0; k < N; ++k) w.av[k][K] += aTot;
      }
    }
  }
  warp_sync();
  if (w.err) { *err |= w.err; return false; }
  // the final passes: their level derivative (volume and moments), before the chain of updates
  if (r.cs != 0)
    for (int k = 0; k < N; ++k) {
      const double a1 = lane_sum(pass_sweep1(M, F, r.members[k], w.hFinal[k], w.av[k][K], w.amx[k], w.amy[k], w.amz[k], lane, width, aP), width);
      if (lane == 0) {
        if (r.cs == 1) w.aHi += a1;
        else w.ah[K] += a1;
      }
    }
  if (lane == 0) {
    if (r.cs == 2) {
      // the updates, last first: h_{j+1} = h_j - err_j / dv_j (Newton) or the bracket's midpoint (bisection)
      for (int j = K - 1; j >= r.base; --j) {
        if (r.newton[j]) {
          double e = 0, dvs = 0;
          for (int k = 0; k < N; ++k) { e += rec(t, r.members[k], j)[1]; dvs += rec(t, r.members[k], j)[2]; }
          e = e - r.V;
          w.ah[j] += w.ah[j + 1];
          const double aErr = -w.ah[j + 1] / dvs;
          const double aDvs = w.ah[j + 1] * e / (dvs * dvs);
          w.aV -= aErr;
          for (int k = 0; k < N; ++k) { w.av[k][j] += aErr; w.adv[k][j] += aDvs; }
        } else {
          const double half = 0.5 * w.ah[j + 1];
          const int srcs[2] = {r.aSrc[j], r.bSrc[j]};
          for (int s = 0; s < 2; ++s) {
            if (srcs[s] >= 0) w.ah[srcs[s]] += half;
            else if (srcs[s] == kSrcLo) w.aLo += half;
            else w.aHi += half;
          }
        }
        // pass j's own level dependence: d vol / d h is its free-surface area, its area does not depend on h
        for (int k = 0; k < N; ++k) w.ah[j] += w.av[k][j] * rec(t, r.members[k], j)[2];
      }
      // the first Newton level: the clamped start (the extent's bottom or top) or the start itself
      if (r.base == 1) {
        if (r.startSrc == kSrcLo) w.aLo += w.ah[1]; else w.aHi += w.ah[1];
      } else {
        w.aH0 += w.ah[0];
      }
      // the passes before the final one whose volume the chain reached: their pose adjoints come from a sweep
      for (int k = 0; k < N; ++k) {
        int np = 0;
        for (int j = r.base; j < K; ++j) {
          if (w.av[k][j] == 0) continue;
          w.hs[k][np] = rec(t, r.members[k], j)[0];
          w.pv[k][np] = w.av[k][j];
          ++np;
        }
        w.np[k] = np;
      }
    }
    // the extent: bottom and top of the unit's start passes
    if (N > 0) {
      w.aZmin0[r.loSrc] += w.aLo;
      w.aZmax0[r.hiSrc] += w.aHi;
    }
  }
  warp_sync();
  for (int k = 0; k < N; ++k)
    if (w.np[k]) pass_sweep_levels(M, F, r.members[k], w.np[k], w.hs[k], w.pv[k], lane, width, aP);
  // (every lane finds the same segment; lane 0 alone adds its terms)
  for (int k = 0; k < N; ++k) {
    if (w.aZmin0[k] != 0) {
      const int j = pass_extreme(M, F, r.members[k], true, lane, width);
      if (lane == 0) extreme_reverse(M, j, true, w.aZmin0[k], aP);
    }
    if (w.aZmax0[k] != 0) {
      const int j = pass_extreme(M, F, r.members[k], false, lane, width);
      if (lane == 0) extreme_reverse(M, j, false, w.aZmax0[k], aP);
    }
  }
  if (lane == 0) {
    // the free-surface area of every pass: dv = (sum of the cut segments' footprints) mu / R22; lane 0 alone adds it
    // to the pose adjoint, which is summed over the lanes afterwards
    for (int k = 0; k < N; ++k)
      for (int j = 0; j <= K && j < kMaxPasses; ++j)
        if (w.adv[k][j] != 0) aP.iR += w.adv[k][j] * rec(t, r.members[k], j)[2] / F.iR;
    // the start level and the unit's volume
    if (r.single) {
      u.oLevel[0] += w.aH0;
    } else if (r.allWet) {
      for (int k = 0; k < N; ++k) u.oLevel[k] += w.aH0 / static_cast<double>(N);
    } else {
      u.oLevel[r.firstWet >= 0 ? r.firstWet : N - 1] += w.aH0;
    }
    for (int k = 0; k < N; ++k) u.oVol[k] += w.aV;
  }
  return true;
}

// ----------------------------------------------------------------------------- flows

// Forward flow of connection c (kernel/flows.hpp:38-78) with the values its reverse needs.
struct FlowRec {
  bool active, limited, limZero, weir;
  int src, dst;
  double zo, ha, hb, Ha, Hb, d, u, H1, H2, r, p1, g, f, q, dV, dVpre, lim, inv, diff, hs, hd, share;
};

// The two powers of a submerged weir (r^1.5 and g^0.385) are kept per connection in pw (2 doubles each): the reverse
// recomputes a step's flows twice, and with `reuse` the second time takes them from there instead of calling pow.
SSB_HD FlowRec flow_forward(const DevModel& M, const PoseD& F, double t, const std::uint8_t* en, const double* area, const double* tOn,
                            const double* hEff, const double* aEff, const int* deg, const std::int32_t* merged, int c, double* pw, bool reuse) {
  FlowRec f{};
  f.active = false;
  if (!en[c] || tOn[c] > t) return f;
  const int sk = M.skip[c];
  if (sk >= 0 && merged[sk]) return f;
  const int a = M.ca[c], b = M.cb[c];
  f.zo = F.R20 * M.kx[c] + F.R21 * M.ky[c] + F.R22 * M.kz[c] + F.tz;
  f.ha = a < 0 ? 0.0 : hEff[a];
  f.hb = hEff[b];
  f.Ha = f.ha > f.zo ? f.ha - f.zo : 0.0;
  f.Hb = f.hb > f.zo ? f.hb - f.zo : 0.0;
  double q = 0;
  f.weir = M.law[c] != 0;
  if (!f.weir) {
    f.d = f.Ha - f.Hb;
    if (f.d != 0) {
      f.u = jmax(fabs(f.d), kOrificeHeadFloor);
      q = M.coef[c] * area[c] * M.sq2g * f.d / pm::sqrt_rn(f.u);
    }
  } else {
    f.H1 = f.Ha > f.Hb ? f.Ha : f.Hb;
    if (f.H1 > 0) {
      f.H2 = f.Ha > f.Hb ? f.Hb : f.Ha;
      f.f = 1;
      if (f.H2 > 0) {
        f.r = f.H2 / f.H1;
        f.p1 = reuse ? pw[2 * c] : pm::pow(f.r, kWeirExponent);
        f.g = 1 - f.p1;
        f.f = reuse ? pw[2 * c + 1] : pm::pow(jmax(0.0, f.g), kVillemonteExponent);
        if (!reuse) { pw[2 * c] = f.p1; pw[2 * c + 1] = f.f; }
      }
      q = M.coef[c] * area[c] * kWeirCoefficient * M.sq2g * f.H1 * pm::sqrt_rn(f.H1) * f.f * (f.Ha >= f.Hb ? 1.0 : -1.0);
    }
  }
  f.q = q;
  if (q == 0) return f;
  f.active = true;
  double dV = q * M.dt;
  f.dVpre = dV;
  f.src = dV > 0 ? a : b;
  f.dst = dV > 0 ? b : a;
  f.hs = f.src < 0 ? 0.0 : hEff[f.src];
  f.hd = f.dst < 0 ? 0.0 : hEff[f.dst];
  f.inv = (f.src < 0 ? 0.0 : 1 / aEff[f.src]) + (f.dst < 0 ? 0.0 : 1 / aEff[f.dst]);
  const int degRef = f.src < 0 ? deg[f.dst] : (f.dst < 0 ? deg[f.src] : (deg[f.src] > deg[f.dst] ? deg[f.src] : deg[f.dst]));
  f.share = kLimiterShare / static_cast<double>(degRef > 1 ? degRef : 1);
  f.diff = f.hs - jmax(f.hd, f.zo);
  double lim = f.inv > 0 ? f.share * f.diff / f.inv : fabs(dV);
  f.limZero = lim < 0;
  if (lim < 0) lim = 0;
  f.lim = lim;
  f.limited = fabs(dV) > lim;
  if (f.limited) dV = dV > 0 ? lim : -lim;
  f.dV = dV;
  return f;
}

// Node adjoints of one connection's flow: the levels (hEff) and limiter areas (aEff) at its a and b ends.
struct FlowAdj {
  double hA, hB, aA, aB;
};

// Reverse of flow_forward: the adjoint of its dV into the ends' level and area adjoints, the pose adjoint (through the
// opening's world height) and the connection area's gradient (returned).
SSB_HD double flow_reverse(const DevModel& M, const PoseD& F, const FlowRec& f, const double* aEff, const double* area, int c, double aDV,
                           FlowAdj& out, AdjPose& aP) {
  out.hA = out.hB = out.aA = out.aB = 0;
  if (!f.active || aDV == 0) return 0;
  const int a = M.ca[c];
  double aZo = 0, aHa = 0, aHb = 0, aArea = 0;
  double aHs = 0, aHd = 0;
  if (f.limited) {
    if (f.limZero || !(f.inv > 0)) return 0;
    const double aLim = f.dVpre > 0 ? aDV : -aDV;
    const double aDiff = aLim * f.share / f.inv;
    const double aInv = -aLim * f.lim / f.inv;
    aHs += aDiff;
    if (f.zo > f.hd) aZo -= aDiff; else aHd -= aDiff;
    if (f.src >= 0) { const double w = aEff[f.src]; const double g = -aInv / (w * w); if (f.src == a) out.aA += g; else out.aB += g; }
    if (f.dst >= 0) { const double w = aEff[f.dst]; const double g = -aInv / (w * w); if (f.dst == a) out.aA += g; else out.aB += g; }
    if (f.src >= 0) { if (f.src == a) out.hA += aHs; else out.hB += aHs; }
    if (f.dst >= 0) { if (f.dst == a) out.hA += aHd; else out.hB += aHd; }
  } else {
    const double aQ = aDV * M.dt;
    aArea = aQ * f.q / area[c];
    if (!f.weir) {
      // q = C area d / sqrt(u), u = max(|d|, floor)
      const double C = M.coef[c] * area[c] * M.sq2g;
      const double su = pm::sqrt_rn(f.u);
      double dqdd = C / su;
      if (!(kOrificeHeadFloor > fabs(f.d))) dqdd -= C * f.d * (f.d < 0 ? -1.0 : 1.0) / (2 * f.u * su);
      const double aD = aQ * dqdd;
      aHa += aD; aHb -= aD;
    } else {
      // q = K area H1^1.5 f(H2 / H1) sgn
      const double sgn = f.Ha >= f.Hb ? 1.0 : -1.0;
      const double K = M.coef[c] * area[c] * kWeirCoefficient * M.sq2g;
      const double sH1 = pm::sqrt_rn(f.H1);
      double aH1 = aQ * K * 1.5 * sH1 * f.f * sgn;
      double aH2 = 0;
      if (f.H2 > 0 && f.g > 0) {
        const double aF = aQ * K * f.H1 * sH1 * sgn;
        const double dfdr = kVillemonteExponent * (f.f / f.g) * (-kWeirExponent * f.p1 / f.r);
        const double aR = aF * dfdr;
        aH2 += aR / f.H1;
        aH1 -= aR * f.r / f.H1;
      }
      if (f.Ha > f.Hb) { aHa += aH1; aHb += aH2; } else { aHb += aH1; aHa += aH2; }
    }
    if (f.ha > f.zo) { aZo -= aHa; if (a >= 0) out.hA += aHa; }
    if (f.hb > f.zo) { aZo -= aHb; out.hB += aHb; }
  }
  aP.R20 += aZo * M.kx[c]; aP.R21 += aZo * M.ky[c]; aP.R22 += aZo * M.kz[c]; aP.tz += aZo;
  return aArea;
}

// ----------------------------------------------------------------------------- loads and integration

struct LoadSums {
  double Fz, tauX, tauY, mw, Iwp, Iwr;
};

// Reverse of the semi-implicit integration (body.hpp:42-57). s = (zO, pitch, roll, vz, wth, wph) before the step; aS
// holds their adjoints after the step on entry and the direct part of the adjoints before it on return. aL receives
// the adjoints of the loads: Fz, Mth, Mph, mw, Iw_p, Iw_r. A pitch or roll clamped at its limit, and its rate set to 0,
// are constants.
SSB_HD void integrate_reverse(const DevModel& M, const LoadSums& Ls, double cth, const double* s, double* aS, double* aL) {
  const double dt = M.dt;
  const double vz = s[3], wth = s[4], wph = s[5];
  const double mh = M.mh0 + Ls.mw;
  const double Ith = M.Ith0 + Ls.Iwp, Iph = M.Iph0 + Ls.Iwr;
  const double Mth = Ls.tauY, Mph = Ls.tauX * cth;
  const double az = (Ls.Fz - M.cDz * vz - M.qz * fabs(vz) * vz) / mh;
  const double ath = (Mth - M.cDth * wth - M.qth * fabs(wth) * wth) / Ith;
  const double aph = (Mph - M.cDph * wph - M.qph * fabs(wph) * wph) / Iph;
  const double th1 = s[1] + (wth + ath * dt) * dt, ph1 = s[2] + (wph + aph * dt) * dt;
  double aZ1 = aS[0], aTh1 = aS[1], aPh1 = aS[2], aVz1 = aS[3], aWth1 = aS[4], aWph1 = aS[5];
  if (th1 > kPitchClamp || th1 < -kPitchClamp) { aTh1 = 0; aWth1 = 0; }
  if (ph1 > kRollClamp || ph1 < -kRollClamp) { aPh1 = 0; aWph1 = 0; }
  aVz1 += aZ1 * dt;
  aWth1 += aTh1 * dt;
  aWph1 += aPh1 * dt;
  const double aAz = aVz1 * dt, aAth = aWth1 * dt, aAph = aWph1 * dt;
  aS[0] = aZ1; aS[1] = aTh1; aS[2] = aPh1;
  aS[3] = aVz1 + aAz * (-M.cDz - 2 * M.qz * fabs(vz)) / mh;
  aS[4] = aWth1 + aAth * (-M.cDth - 2 * M.qth * fabs(wth)) / Ith;
  aS[5] = aWph1 + aAph * (-M.cDph - 2 * M.qph * fabs(wph)) / Iph;
  aL[0] = aAz / mh;
  aL[1] = aAth / Ith;
  aL[2] = aAph / Iph;
  aL[3] = -aAz * az / mh;
  aL[4] = -aAth * ath / Ith;
  aL[5] = -aAph * aph / Iph;
}

// The buoyancy terms of the loads (body.hpp:11-19), the part every node's terms are added to.
SSB_HD LoadSums loads_buoyancy(const DevModel& M, const PoseD& F, const double* hb) {
  const double Wg = M.rho * M.g;
  const double Fb = Wg * hb[0];
  const double bxw = F.R00 * hb[1] + F.R01 * hb[2] + F.R02 * hb[3] + F.tx;
  const double byw = F.R10 * hb[1] + F.R11 * hb[2] + F.R12 * hb[3] + F.ty;
  LoadSums L;
  L.tauX = (byw - M.YO) * Fb;
  L.tauY = -(bxw - M.XO) * Fb;
  L.Fz = Fb - M.g * M.ms;
  L.mw = 0; L.Iwp = 0; L.Iwr = 0;
  return L;
}

// One node's terms of the loads (body.hpp:20-33): its flood water's weight at its centroid and its inertia.
SSB_HD void loads_node(const DevModel& M, const PoseD& F, double zO, double V, double x, double y, double z, LoadSums& L) {
  if (V <= 0) return;
  const double Wg = M.rho * M.g;
  const double wx = F.R00 * x + F.R01 * y + F.R02 * z + F.tx - M.XO;
  const double wy = F.R10 * x + F.R11 * y + F.R12 * z + F.ty - M.YO;
  const double wz = F.R20 * x + F.R21 * y + F.R22 * z + F.tz - zO;
  const double f = -Wg * V;
  const double m = M.rho * V;
  L.tauX += wy * f; L.tauY -= wx * f; L.Fz += f;
  L.mw += m; L.Iwp += m * (wx * wx + wz * wz); L.Iwr += m * (wy * wy + wz * wz);
}

// Reverse of the buoyancy terms: adjoints of the buoyancy result (V, x, y, z) into aHb and the pose adjoint.
SSB_HD void loads_buoyancy_reverse(const DevModel& M, const PoseD& F, const double* hb, const double* aL, double cthTauX, double* aHb,
                                   AdjPose& aP) {
  // aL: Fz, Mth, Mph, mw, Iwp, Iwr; Mph = tauX cth, so a_tauX = a_Mph cth (cthTauX: the cth the step used)
  const double aTauX = aL[2] * cthTauX, aTauY = aL[1], aFz = aL[0];
  const double Wg = M.rho * M.g;
  const double Fb = Wg * hb[0];
  const double bxw = F.R00 * hb[1] + F.R01 * hb[2] + F.R02 * hb[3] + F.tx;
  const double byw = F.R10 * hb[1] + F.R11 * hb[2] + F.R12 * hb[3] + F.ty;
  const double aByw = aTauX * Fb, aBxw = -aTauY * Fb;
  const double aFb = aTauX * (byw - M.YO) - aTauY * (bxw - M.XO) + aFz;
  aHb[0] = aFb * Wg;
  aHb[1] = aBxw * F.R00 + aByw * F.R10;
  aHb[2] = aBxw * F.R01 + aByw * F.R11;
  aHb[3] = aBxw * F.R02 + aByw * F.R12;
  aP.R00 += aBxw * hb[1]; aP.R01 += aBxw * hb[2]; aP.R02 += aBxw * hb[3]; aP.tx += aBxw;
  aP.R10 += aByw * hb[1]; aP.R11 += aByw * hb[2]; aP.R12 += aByw * hb[3]; aP.ty += aByw;
}

// Reverse of one node's load terms: the adjoints of its volume (after the update) and centroid, the pose adjoint and
// the adjoint of the zO the step started from (through the water's height above it).
SSB_HD void loads_node_reverse(const DevModel& M, const PoseD& F, double zO, double V, double x, double y, double z, const double* aL,
                               double cth, double& aV, double& ax, double& ay, double& az, double& aZo, AdjPose& aP) {
  aV = ax = ay = az = 0;
  if (V <= 0) return;
  const double aTauX = aL[2] * cth, aTauY = aL[1], aFz = aL[0], aMw = aL[3], aIwp = aL[4], aIwr = aL[5];
  const double Wg = M.rho * M.g;
  const double wx = F.R00 * x + F.R01 * y + F.R02 * z + F.tx - M.XO;
  const double wy = F.R10 * x + F.R11 * y + F.R12 * z + F.ty - M.YO;
  const double wz = F.R20 * x + F.R21 * y + F.R22 * z + F.tz - zO;
  const double f = -Wg * V;
  const double m = M.rho * V;
  const double aWy = aTauX * f + aIwr * m * 2 * wy;
  const double aWx = -aTauY * f + aIwp * m * 2 * wx;
  const double aWz = (aIwp + aIwr) * m * 2 * wz;
  const double aF = aTauX * wy - aTauY * wx + aFz;
  const double aM = aMw + aIwp * (wx * wx + wz * wz) + aIwr * (wy * wy + wz * wz);
  aV = -Wg * aF + M.rho * aM;
  ax = aWx * F.R00 + aWy * F.R10 + aWz * F.R20;
  ay = aWx * F.R01 + aWy * F.R11 + aWz * F.R21;
  az = aWx * F.R02 + aWy * F.R12 + aWz * F.R22;
  aP.R00 += aWx * x; aP.R01 += aWx * y; aP.R02 += aWx * z; aP.tx += aWx;
  aP.R10 += aWy * x; aP.R11 += aWy * y; aP.R12 += aWy * z; aP.ty += aWy;
  aP.R20 += aWz * x; aP.R21 += aWz * y; aP.R22 += aWz * z; aP.tz += aWz;
  aZo -= aWz;
}

// ----------------------------------------------------------------------------- the reverse of one step

#if defined(__CUDACC__)
#define SSB_HDT __host__ __device__
#else
#define SSB_HDT
#endif

// Per-team working arrays of the reverse (shared memory on the device): the forward values it recomputes and the
// adjoints it passes between phases.
struct RevSlot {
  double *hEff, *aEff, *dV, *volPost;   // per node / per connection: the step's flows, recomputed
  int* deg;
  std::int32_t* clip;                    // per node: 0, or 1 the update clipped the volume at 0, 2 at the cap
  double *aVolPost, *aCxs, *aCys, *aCzs, *aVs, *aAcc, *aZmx, *aLs, *aAs;
  double *faHA, *faHB, *faAA, *faAB;     // per connection: its flow's adjoints at its a and b ends
  double* red;                           // team reduction scratch: nwarps x 16
  UnitWork* work;                        // one per warp: the level solve's reverse, unit by unit
  std::uint8_t* plain;                   // per node: 1 when its unit's reverse was the empty node's pass-through
  std::int32_t* units;                   // the other units in group order: group << 16 | member (0xffff: the merged group)
  std::int32_t* nunits;                  // their number
  double* pw;                            // per connection: its weir's two powers (flow_forward)
  Replay* replays;                       // per listed unit: its replay
};

// The adjoint of the state between steps: per node in memory, the scalars (zO, pitch, roll, vz, wth, wph) in every
// thread's registers.
struct AdjState {
  double *aVol, *aLevel, *aCx, *aCy, *aCz;
};

// Reverse of one step (kernel::step, step.hpp:41-54). `a` holds the adjoint of the state after the step on entry and
// before it on return (aSc likewise for the scalars); grad[c] accumulates d objective / d area[c]. Returns false (with
// err bits) if the step took a branch without an adjoint here.
template <class T>
SSB_HDT bool reverse_step(const T& team, const DevModel& M, const Tape& tp, const std::uint8_t* en, const double* area, const double* tOn,
                          RevSlot& S, AdjState& a, double* aSc, double* grad, int* err) {
  const TapeLayout& L = tp.L;
  const PoseD F = load_pose(tp.d + L.pose);
  const double* st = tp.d + L.scal;
  const double t = st[0], zO = st[1];
  const double* hb = tp.d + L.buoy;
  const double* volS = tp.d + L.volS;
  const double* levelS = tp.d + L.levelS;
  const double* areaS = tp.d + L.areaS;
  const double* cxS = tp.d + L.cxS;
  const double* cyS = tp.d + L.cyS;
  const double* czS = tp.d + L.czS;
  const double* zmaxS = tp.d + L.zmaxS;
  const std::int32_t* merged = tp.i + L.merged;
  const int NN = M.nn, NC = M.nc;

  // ---- the step's flows, volume update and loads, recomputed (flows.hpp:15-118, body.hpp:11-40)
  for (int n = team.rank; n < NN; n += team.size) {
    const double v = volS[n];
    S.hEff[n] = v > kEmptyVolume ? levelS[n] : kNoHead;
    S.aEff[n] = v >= M.vmax[n] ? M.aov[n] : jmax(areaS[n], M.amin[n]);
    S.deg[n] = 0;
  }
  team.sync();
  for (int c = team.rank; c < NC; c += team.size) {
    if (!en[c]) continue;
    const int ca = M.ca[c], cb = M.cb[c];
    if (ca >= 0 && S.hEff[ca] < kNoHeadTest && S.hEff[cb] < kNoHeadTest) continue;
    if (ca >= 0) team.add_int(&S.deg[ca], 1);
    team.add_int(&S.deg[cb], 1);
  }
  team.sync();
  for (int c = team.rank; c < NC; c += team.size)
    S.dV[c] = flow_forward(M, F, t, en, area, tOn, S.hEff, S.aEff, S.deg, merged, c, S.pw, false).dV;
  team.sync();
  LoadSums Ls = loads_buoyancy(M, F, hb);
  double part[6] = {0, 0, 0, 0, 0, 0};
  for (int n = team.rank; n < NN; n += team.size) {
    const int k0 = M.incStart[n], k1 = k0 + M.incCount[n];
    double acc = 0;
    for (int k = k0; k < k1; ++k) {
      const double d = S.dV[M.incConn[k]];
      acc = M.incSide[k] ? acc + d : acc - d;
    }
    double v = volS[n] + acc;
    int clip = 0;
    if (v < 0) { v = 0; clip = 1; }
    const double vm = M.vmax[n];
    if (v > vm) {
      const double head = jmax(0.0, -zmaxS[n]);
      const double cap = vm + M.aov[n] * head;
      if (v > cap) { v = cap; clip = 2; }
    }
    S.volPost[n] = v;
    S.clip[n] = clip;
    LoadSums one{0, 0, 0, 0, 0, 0};
    loads_node(M, F, zO, v, cxS[n], cyS[n], czS[n], one);
    part[0] += one.Fz; part[1] += one.tauX; part[2] += one.tauY; part[3] += one.mw; part[4] += one.Iwp; part[5] += one.Iwr;
  }
  team.reduce(part, 6, S.red);
  Ls.Fz += part[0]; Ls.tauX += part[1]; Ls.tauY += part[2]; Ls.mw += part[3]; Ls.Iwp += part[4]; Ls.Iwr += part[5];

  // ---- integration and loads
  double aL[6];
  integrate_reverse(M, Ls, F.cth, st + 1, aSc, aL);
  AdjPose aP;
  zero(aP);
  double aZo = 0;
  double aHb[4];
  {
    AdjPose once;
    zero(once);
    loads_buoyancy_reverse(M, F, hb, aL, F.cth, aHb, once);
    once.cth += aL[2] * Ls.tauX;  // Mph = tauX cth
    if (team.rank == 0)
      for (int k = 0; k < kAdjPoseFields; ++k) fields(aP)[k] += fields(once)[k];
  }
  for (int n = team.rank; n < NN; n += team.size) {
    double aV, ax, ay, az;
    loads_node_reverse(M, F, zO, S.volPost[n], cxS[n], cyS[n], czS[n], aL, F.cth, aV, ax, ay, az, aZo, aP);
    S.aVolPost[n] = a.aVol[n] + aV;
    S.aCxs[n] = a.aCx[n] + ax;
    S.aCys[n] = a.aCy[n] + ay;
    S.aCzs[n] = a.aCz[n] + az;
    // the volume update (flows.hpp:99-111): clipped at 0 or at the cap, the volume no longer follows its inputs
    const double av = S.aVolPost[n];
    S.aVs[n] = 0; S.aAcc[n] = 0; S.aZmx[n] = 0;
    if (S.clip[n] == 0) {
      S.aVs[n] = av;
      S.aAcc[n] = av;
    } else if (S.clip[n] == 2) {
      if (-zmaxS[n] > 0) S.aZmx[n] = -M.aov[n] * av;
    }
  }
  team.sync();

  // ---- flows
  for (int c = team.rank; c < NC; c += team.size) {
    const int ca = M.ca[c], cb = M.cb[c];
    const double aDV = S.aAcc[cb] - (ca >= 0 ? S.aAcc[ca] : 0.0);
    FlowAdj fa;
    const FlowRec fr = flow_forward(M, F, t, en, area, tOn, S.hEff, S.aEff, S.deg, merged, c, S.pw, true);
    grad[c] += flow_reverse(M, F, fr, S.aEff, area, c, aDV, fa, aP);
    S.faHA[c] = fa.hA; S.faHB[c] = fa.hB; S.faAA[c] = fa.aA; S.faAB[c] = fa.aB;
  }
  team.sync();
  // heads and limiter areas (flows.hpp:15-19): per node, its connections' adjoints in incidence order
  for (int n = team.rank; n < NN; n += team.size) {
    const int k0 = M.incStart[n], k1 = k0 + M.incCount[n];
    double aH = 0, aA = 0;
    for (int k = k0; k < k1; ++k) {
      const int c = M.incConn[k];
      if (M.incSide[k]) { aH += S.faHB[c]; aA += S.faAB[c]; }
      else { aH += S.faHA[c]; aA += S.faAA[c]; }
    }
    const double v = volS[n];
    S.aLs[n] = a.aLevel[n] + (v > kEmptyVolume ? aH : 0.0);
    S.aAs[n] = (!(v >= M.vmax[n]) && !(M.amin[n] > areaS[n])) ? aA : 0.0;
  }
  team.sync();

  // ---- the level solve. Warp 0 lists the units in group order (a prefix sum over the groups, a warp's width of them
  // at a time), except the units that are a node alone and empty (most of them in a flooding run) when neither its
  // level nor its extent top has an adjoint and its one pass is the recorded start: the solver set the level to the
  // node's extent bottom and left volume and centroid as they were, so their adjoints pass through (what unit_reverse
  // does for such a unit, without its replay), written by the listing lane. The listed units are then dealt to the
  // warps in turn: a warp per merged group or node alone, lane 0 doing its scalar chain in the warp's work area.
  if (team.warp == 0) {
    int base = 0;
    for (int g0 = 0; g0 < M.ng; g0 += team.width) {
      const int g = g0 + team.lane;
      int c = 0;
      if (g < M.ng) {
        if (merged[g]) {
          c = 1;
        } else {
          const int* mem = M.gNodes + M.gStart[g];
          for (int k = 0; k < M.gCount[g]; ++k) {
            const int n = mem[k];
            S.plain[n] = tp.d[L.volIn + n] <= kEmptyVolume && tp.i[L.npass + n] == 1 && tp.pass(n, 0)[0] == tp.d[L.levelIn + n] &&
                         S.aLs[n] == 0 && S.aZmx[n] == 0;
            if (!S.plain[n]) {
              ++c;
              continue;
            }
            a.aVol[n] = 0.0 + (0.0 + S.aVs[n]);
            a.aLevel[n] = 0.0 + 0.0;
            a.aCx[n] = 0.0 + S.aCxs[n]; a.aCy[n] = 0.0 + S.aCys[n]; a.aCz[n] = 0.0 + S.aCzs[n];
          }
        }
      }
      const int incl = lane_prefix(c, team.lane, team.width);
      int at = base + incl - c;
      if (g < M.ng) {
        if (merged[g]) {
          S.units[at] = (g << 16) | 0xffff;
        } else {
          const int* mem = M.gNodes + M.gStart[g];
          for (int k = 0; k < M.gCount[g]; ++k)
            if (!S.plain[mem[k]]) S.units[at++] = (g << 16) | k;
        }
      }
      base += lane_value(incl, team.width - 1, team.width);
    }
    if (team.lane == 0) *S.nunits = base;
  }
  team.sync();
  const int nu = *S.nunits;
  // every unit's replay at once, a thread per unit (the replay is a chain of scalar decisions over the recorded passes)
  for (int i = team.rank; i < nu; i += team.size) {
    const int e = S.units[i];
    const int g = e >> 16, u = e & 0xffff;
    const bool isMerged = u == 0xffff;
    const int* um = M.gNodes + M.gStart[g] + (isMerged ? 0 : u);
    const int un = isMerged ? M.gCount[g] : 1;
    Replay& r = S.replays[i];
    replay_unit(M, tp, um, un, !isMerged, r);
    for (int k = 0; k < un && k < kMaxMembers; ++k) {
      const int want = r.cs == 0 ? 1 : (r.cs == 1 ? 2 : r.K + 1);
      r.ok = r.ok && tp.i[L.npass + um[k]] == want;
    }
  }
  team.sync();
  bool ok = true;
  UnitWork& w = S.work[team.warp];
  for (int i = team.warp; i < nu; i += team.nwarps) {
    {
      const int e = S.units[i];
      const int g = e >> 16, u = e & 0xffff;
      const int N = M.gCount[g];
      const int* mem = M.gNodes + M.gStart[g];
      const bool isMerged = u == 0xffff;
      const int* um = isMerged ? mem : mem + u;
      const int un = isMerged ? N : 1;
      if (un > kMaxMembers) { ok = false; *err |= kErrGroupSize; continue; }
      // the unit's replay into the warp's work area, a word per lane
      {
        const auto* src = reinterpret_cast<const std::int32_t*>(&S.replays[i]);
        auto* dst = reinterpret_cast<std::int32_t*>(&w.r);
        for (int k = team.lane; k < static_cast<int>(sizeof(Replay) / sizeof(std::int32_t)); k += team.width) dst[k] = src[k];
      }
      if (team.lane == 0) {
        for (int k = 0; k < un; ++k) {
          const int n = um[k];
          w.u.aLevel[k] = S.aLs[n]; w.u.aArea[k] = S.aAs[n]; w.u.aCx[k] = S.aCxs[n]; w.u.aCy[k] = S.aCys[n]; w.u.aCz[k] = S.aCzs[n];
          w.u.aVol[k] = S.aVs[n]; w.u.aZmax[k] = S.aZmx[n];
        }
      }
      warp_sync();
      bool done = w.r.ok;
      if (!done) {
        ok = false;
        *err |= kErrReplay;
      } else {
        int e = 0;
        if (!unit_reverse(M, F, tp, w, team.lane, team.width, aP, &e)) {
          ok = false;
          *err |= e;
          done = false;
        }
      }
      if (done && team.lane == 0)
        for (int k = 0; k < un; ++k) {
          const int n = um[k];
          a.aVol[n] = w.u.oVol[k]; a.aLevel[n] = w.u.oLevel[k];
          a.aCx[n] = w.u.oCx[k]; a.aCy[n] = w.u.oCy[k]; a.aCz[n] = w.u.oCz[k];
        }
      warp_sync();  // every lane is done with the work area before lane 0 fills it for the next unit
    }
  }

  // ---- buoyancy (reduce.hpp:39-49): the adjoint of V, x, y, z into V, Mx, My, Mz, then the columns. It needs only the
  // loads' adjoint, so each warp sweeps its columns as soon as its level-solve units are done, before the barrier
  {
    double aV = aHb[0], aMx = 0, aMy = 0, aMz = 0;
    if (hb[0] > 0) {
      aMx = aHb[1] / hb[0]; aMy = aHb[2] / hb[0]; aMz = aHb[3] / hb[0];
      aV -= (aHb[1] * hb[1] + aHb[2] * hb[2] + aHb[3] * hb[3]) / hb[0];
    }
    buoyancy_sweep(M, F, aV, aMx, aMy, aMz, team.rank, team.size, aP);
  }
  team.sync();

  // ---- the pose: every thread's share summed over the team, then (zO, pitch, roll)
  double red[kAdjPoseFields + 1];
  for (int k = 0; k < kAdjPoseFields; ++k) red[k] = fields(aP)[k];
  red[kAdjPoseFields] = aZo;
  team.reduce(red, kAdjPoseFields + 1, S.red);
  AdjPose tot;
  for (int k = 0; k < kAdjPoseFields; ++k) fields(tot)[k] = red[k];
  aSc[0] += red[kAdjPoseFields];
  pose_reverse(M, F, tot, aSc[0], aSc[1], aSc[2]);
  // (no barrier here: the caller synchronises the team before the tape or these work arrays are written again)
  return ok;
}

}  // namespace adj
}  // namespace ssb
