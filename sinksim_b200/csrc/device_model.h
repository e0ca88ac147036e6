// Device-side layout of one compiled model (ship + sim) and of a batch of its instances.
//
// Layout in HBM. Everything a step reads from the model is structure-of-arrays so that a warp reading entries
// j..j+31 moves whole 128-byte lines:
//   columns   x, y, dxdy, zlo, zhi                     [ncol] f64       the buoyancy clip (hydro pass)
//   segments  x, y, A (= dxdy of the column), a, e     [nseg] f64       the node pass, with the column gather of the
//                                                                       reference (segCol -> x, y, dxdy) resolved once
//                                                                       on the host, so a segment visit has no
//                                                                       dependent load
//   nodes, groups, connections, incidence (CSR), monitor lists (CSR), marks: small tables read through L1.
// Per instance (count instances): the connection fields a sweep may change (en, area, tOn), the state (t, pose,
// rates, per-node volume, level and centroid), the outputs, the event log, the readout curve and, for the first
// `traced` instances, the trace records. The state of an instance being stepped lives in shared memory and
// registers of its warp; global memory holds it between launches and after the run.
#pragma once

#include <cstdint>

#include <vector_types.h>

namespace ssb {

struct DevModel {
  // columns: (x, y) and (zlo, zhi) pairs, so one 16-byte load fetches two fields, and the footprint dxdy; the float
  // copies are the same values rounded to single precision once on the host (the portable32 column arithmetic
  // rounds every geometry value to float before using it, kernel/reduce.hpp:131-164)
  std::int32_t ncol;
  const double2 *colXY, *colLH;
  const double* colA;
  const float2 *colXYf, *colLHf;
  const float* colAf;
  // segments with the column gather resolved: (x, y) of the column, (a, e) of the segment, the column's dxdy
  std::int32_t nseg;
  const double2 *segXY, *segLH;
  const double* segAr;
  const float2 *segXYf, *segLHf;
  const float* segArf;
  // nodes
  std::int32_t nn;
  const double *mu, *vmax, *amin, *aov;
  const std::int32_t *segStart, *segCount;
  // groups
  std::int32_t ng;
  const std::int32_t *gStart, *gCount, *gNodes;
  const std::uint8_t* gMode;
  const double *gpx, *gpy, *gpz;
  double gMargin;
  std::int32_t maxGroup;
  // connections (the immutable fields)
  std::int32_t nc;
  const std::int32_t *ca, *cb, *skip;
  const std::uint8_t* law;
  const double *kx, *ky, *kz, *coef;
  // incidence: per node its connections in increasing order (side 1 at the b end), and the sea connections
  const std::int32_t *incStart, *incCount, *incConn;
  const std::uint8_t* incSide;
  std::int32_t nsea;
  const std::int32_t* sea;
  // monitors: per monitor its connections in increasing order
  std::int32_t nmon;
  double monThreshold;
  const std::int32_t *monStart, *monCount, *monConn;
  // marks
  std::int32_t nmark;
  const double *mkx, *mky, *mkz;
  const std::uint8_t* mkWhen;
  // founder rule
  double hullTopBelow, pitchAbsAbove, buoyancyBelow, minT;
  // physics and body
  double rho, g, sq2g, dt;
  double ms, g0x, g0y, g0z, XO, YO, mh0, Ith0, Iph0, cDz, cDth, cDph, qz, qth, qph;
  // readout geometry
  double xFP, xAP;
  std::int32_t evCap;
};

// An extra retire predicate evaluated after every step (the batching workloads' "sink" and "settle" rules); it
// never changes the physics. Disabled when enabled == 0.
struct RetireRule {
  std::int32_t enabled;
  double pitchLimit;           // rad: sink when |pitch| exceeds this ...
  double xDeck, yDeck, zDeck;  // ... and the deck edge at (xDeck, +-yDeck, zDeck) is below the sea
  double wthLimit;             // rad/s: settle when |pitch rate| stays below this ...
  double settleTime;           // s: ... for this long
};

// Why an instance stopped. kStable: the reference's "stop when stable" calm rule of Simulation::run
// (engine/src/simulation.cpp:179-182), which its GPU runner refused (apps/sinksim_cuda_run.cpp:28).
enum StopReason : std::int32_t { kRunning = 0, kFoundered = 1, kTimeLimit = 2, kSinkRule = 3, kSettleRule = 4, kStable = 5 };

// Bits of DevBatch::error, which a batch run reports to the host: kHealthNonFinite, an instance's rigid-body state
// (heave, pitch, roll or their rates) was not finite when the kernel stored it (a NaN or infinity in an input, or a
// model that diverged). The physics is not changed by it: the instance's results are what the step computed.
// kHealthStageTimeout: a block's copy of the column table into shared memory (stageColumns) did not complete within
// its wait limit; that block read the table from global memory instead, with the same results.
enum HealthBit : std::int32_t { kHealthNonFinite = 1, kHealthStageTimeout = 2 };

struct DevBatch {
  std::int32_t count;
  // connection fields per instance [count * nc]
  const std::uint8_t* en;
  const double* area;
  const double* tOn;
  // state per instance
  double* st;       // [count * 8]: t, zO, pitch, roll, vz, wth, wph, calm (seconds the settle rule has held)
  double* out;      // [count * 7]: inflow, Vb, hullTop, mw, bx, by, bz
  double *vol, *level, *cx, *cy, *cz;   // [count * nn]
  // events
  double* evT;             // [count * evCap]
  std::int32_t* evId;      // [count * evCap]
  std::int32_t* evKind;    // [count * evCap]
  std::int32_t* evCount;   // [count]
  double* overT;           // [count * nmon]
  double* markT;           // [count * nmark]
  std::int32_t* foundered; // [count]
  double* founderT;        // [count]
  long long* steps;        // [count]
  std::int32_t* stop;      // [count] StopReason
  // readout curve of every instance: 7 values per record when t >= nextCurve
  double curveEvery;       // <= 0 disables
  std::int32_t curveMax;
  double* curveRec;        // [count * curveMax * 7]
  std::int32_t* curveCount;
  double* nextCurve;
  // final readouts of every instance, computed on the device when the instance stops: 7 values
  double* finalRec;        // [count * 7]
  // traces of the first `traced` instances
  std::int32_t traced, denseSteps, maxSamples, recSize;
  double sampleEvery;
  double *denseRec, *sampleRec;
  std::int32_t *denseCount, *sampleCount;
  double* nextSample;
  // run control
  double tMax;
  long long maxSteps;          // steps per instance per launch
  std::int32_t firstLaunch;
  RetireRule rule;
  // the reference's calm rule: after 1,800 s, stop once |inflow| < 0.02, |pitch rate| < 1e-5 and |heave rate| < 1e-3
  // have held for more than 1,200 s; exclusive with `rule` (both keep their timer in state slot 7)
  std::int32_t stopWhenStable;
  std::int32_t* queue;         // work-queue head (atomic), reset to 0 before each launch
  std::int32_t* error;         // HealthBit flags of the run (0 = none), or-ed by the kernels and read back by the host
  // 1: every block first copies the model's column table (the arrays the buoyancy reads, in the arithmetic's type)
  // into its shared memory after its slots, by bulk asynchronous copies, and the buoyancy reads it from there
  std::int32_t stageColumns;
  // adaptive team size: instances not yet stopped (atomic, set to count before the first launch); a launch with
  // yieldBelow > 0 pauses its instances and stops claiming new ones once at most yieldBelow remain, so that the
  // next launch resumes them with larger teams (shorter steps)
  std::int32_t* remaining;
  std::int32_t yieldBelow;
  // when not null: the steps this launch took, summed over its instances (the per-phase work figure of the timing)
  unsigned long long* phaseSteps;
  // when not null: queue position k claims instance order[k] (k < *orderCount) instead of instance k. Launch phases
  // after the first take the unfinished instances with the fewest steps done first, so that the runs with the most
  // work left to do are the first to get the larger teams.
  const std::int32_t* order;
  const std::int32_t* orderCount;
  // A fleet (instances of several models in one launch): instance i steps models[model[i]], and its per-node,
  // per-connection, event, monitor and mark arrays start at the offsets below instead of i x the model's size.
  // Null for a batch of one model, which the kernel's model parameter describes.
  const DevModel* models;
  const std::int32_t* model;
  const long long *nodeOff, *connOff, *evOff, *monOff, *markOff;
};

// Pose R = Ry(pitch) Rx(roll) and translation (kernel/frame.hpp:9-21), with the single-precision copies the
// portable32 column arithmetic uses (kernel/reduce.hpp:86-98). A team keeps the pose of its current step in its slot.
struct Pose {
  double R00, R01, R02, R10, R11, R12, R20, R21, R22, tx, ty, tz, cth, iR;
  float fR20, fR21, fR22, ftz, fiR;
};

// The buoyancy pass's result: displaced volume, its centroid in the ship frame, the highest hull point in the world.
struct Buoy {
  double V, x, y, z, top;
};

// The run's values that the hydrostatic phases of a step do not read: a team parks them in its slot while those
// phases run, so that their registers serve the level solve (every thread of the team holds the same values).
struct Parked {
  double t, zO, pitch, roll, vz, wth, wph, calm, inflow, Vb, hullTop, mw, bx, by, bz, founderT;
  int foundered;
};

// Lanes that solve one group of nodes' free-surface levels together (8, 16 or 32), per numerics: a warp works on
// 32 / kLevelLanes groups at once. Each lane forms the partials of 32 / kLevelLanes lanes of the 32-lane node-pass tree
// and combines them in the tree's order, so the results do not depend on this choice. Fewer lanes per group give more
// groups in flight but more partials per lane (registers); on B200 (titanic64 batches) 16 was the fastest for double
// precision partials and 8 for single precision ones.
#ifndef SSB_LEVEL_LANES_F64
#define SSB_LEVEL_LANES_F64 16
#endif
#ifndef SSB_LEVEL_LANES_F32
#define SSB_LEVEL_LANES_F32 8
#endif
template <bool MIXED>
constexpr int kLevelLanes = MIXED ? SSB_LEVEL_LANES_F32 : SSB_LEVEL_LANES_F64;
static_assert(kLevelLanes<false> == 8 || kLevelLanes<false> == 16 || kLevelLanes<false> == 32, "level lanes must be 8, 16 or 32");
static_assert(kLevelLanes<true> == 8 || kLevelLanes<true> == 16 || kLevelLanes<true> == 32, "level lanes must be 8, 16 or 32");
// the slot's node-pass buffers are sized for the numerics with the most groups per warp
constexpr int kMaxLevelGroupsPerWarp = 32 / (kLevelLanes<false> < kLevelLanes<true> ? kLevelLanes<false> : kLevelLanes<true>);

// Byte offsets of one simulation slot (one team of warps) in dynamic shared memory; `bytes` is the slot stride.
// passes holds maxGroup node-pass results per level lane group of the team (up to kMaxLevelGroupsPerWarp per warp); hydro the
// eight buoyancy tree results; misc two ints the team broadcasts (the claimed instance, the yield decision); pose and
// buoy the step's pose and buoyancy result, which every phase reads (kept here rather than in each thread's registers);
// parked the run's values during the hydrostatic phases; model (fleets only) the team's copy of its instance's model.
// tmp is the sixth column of the loads' per-node terms (the other five reuse area, zmax, hEff, aEff and acc, which
// are dead by then); kSlotAliasDV places it on dV when there are at least as many connections as nodes.
struct SlotLayout {
  std::uint32_t vol, level, cx, cy, cz, area, zmax, hEff, aEff, acc, deg, dV, q, tmp, passes, hydro, misc, merged, pose, buoy, parked, model, bytes;
};
constexpr std::uint32_t kSlotAliasDV = 0xFFFFFFFFu;

}  // namespace ssb
