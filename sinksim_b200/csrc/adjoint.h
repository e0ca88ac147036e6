// The adjoint engine: objective and gradient of a trajectory misfit with respect to every connection area, for many
// instances of one compiled model on one GPU, by the discrete adjoint of the time step (adjoint_kernel.cu) with FP64
// checkpoints every K steps and recomputation in between. No counterpart in the reference, which has no gradients
// (docs/adr/0001-single-source-cpp-kernel.md:25-26); the instances are set up as the reference's cuda::Batch sets up
// its own (engine/cuda/batch.cu:217-243: connection areas and enabled flags per instance).
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "model.h"

namespace ssb {

struct AdjointOptions {
  std::int32_t count = 1;
  double tMax = 7920;             // s: the runs stop here or at their founder
  std::int32_t checkpointEvery = 256;
  std::int32_t teamWarps = 0;     // warps per instance, 4, 8 or 16; 0: chosen from the count
  int device = 0;
};

class AdjointBatch {
 public:
  AdjointBatch(std::shared_ptr<const CompiledShip> ship, const CompiledSim& sim, const AdjointOptions& opt);
  ~AdjointBatch();
  AdjointBatch(const AdjointBatch&) = delete;
  AdjointBatch& operator=(const AdjointBatch&) = delete;

  void set_connection_enabled(std::int32_t inst, std::int32_t c, bool en);
  // area of connection conns[j] of instance first + i = areas[i * nConns + j], every index checked first
  void set_connection_areas(std::int32_t first, std::int32_t count, std::int32_t nConns, const std::int32_t* conns, const double* areas);
  // the objective: sample times (ascending) and per instance the target trim (degrees) and heave at them, row-major
  // count x n
  void set_objective(std::int32_t n, const double* times, const double* trim, const double* heave);
  // Runs every instance forward and back; returns the device time in milliseconds (CUDA events on the launching
  // stream). Inputs go to the device in the call, results come back before it returns.
  float run();

  std::int32_t count() const { return opt_.count; }
  std::int32_t connections() const;
  std::int32_t nodes() const;
  int team_warps() const { return teamWarps_; }
  int teams() const { return teams_; }
  double objective(std::int32_t inst) const;
  const double* gradient(std::int32_t inst) const;     // [connections]
  const double* samples_trim(std::int32_t inst) const;  // the run's trim at the sample times
  const double* samples_heave(std::int32_t inst) const;
  std::int64_t steps(std::int32_t inst) const;
  std::int32_t error(std::int32_t inst) const;
  // the team's time on the instance in the last run, ns: forward, recomputation of the segments, reverse steps
  const long long* phase_ns(std::int32_t inst) const;
  std::int64_t recomputed_steps(std::int32_t inst) const;  // steps recomputed from checkpoints in the last run
  // The order in which the teams claim the instances (a permutation of 0 .. count-1; null or n = 0: by index). Longest
  // runs first lets the others fill in around them when there are more instances than teams; the results do not
  // depend on it.
  void set_claim_order(const std::int32_t* order, std::int32_t n);
  // Bytes of step records all teams together may keep (0: a whole run's with two passes per node, within half the
  // device memory free at the next run). With room for a whole run the reverse recomputes nothing; the least is one
  // segment of K records per team, every segment then recomputed.
  void set_tape_budget(std::uint64_t bytes);
  std::size_t ring_bytes() const;  // per team, as the last run used
  std::size_t upload_bytes() const;
  std::size_t download_bytes() const;

 private:
  struct Impl;
  std::unique_ptr<Impl> I_;
  AdjointOptions opt_;
  int teamWarps_ = 0, teams_ = 0;
};

}  // namespace ssb
