// The batch engine: many instances of one compiled ship and sim on one GPU. The host-side counterpart of the
// reference's cuda::Batch (engine/include/sinksim/cuda/batch.hpp:27-87): per-instance setters staged on the host,
// run() to completion, then results, curves, final readouts and traces.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "batch_kernel.h"
#include "device_model.h"
#include "model.h"
#include "sweep.h"

namespace ssb {

struct BatchOptions {
  std::int32_t count = 1;
  bool mixedPrecision = true;      // portable32 numerics; false: portable (double precision)
  std::int32_t tracedInstances = 1;
  std::int32_t denseSteps = 400;
  double sampleEvery = 60;
  double curveEvery = 0;           // s between readout-curve records (0: none)
  double tMax = 5 * 3600;
  std::int64_t stepsPerLaunch = 0; // 0: one launch runs every instance to its end; > 0: bounded launches
  std::int32_t teamWarps = 0;      // warps per simulation in the main phase (1, 2, 4, 8); 0: chosen from the batch size
  std::int32_t tailTeamWarps = -1; // warps per simulation once few instances remain; 0: no tail phase; -1: chosen
  std::int32_t teamsPerBlock = 0;  // simulations per block in the main phase; 0: chosen from the slot size
  std::int32_t yieldBelow = -1;    // main phase pauses once at most this many instances remain; -1: from handoverFactor
  double handoverFactor = 2.0;     // a phase hands over once the unfinished instances number at most this multiple of
                                   // the next phase's resident teams (the surplus waits in the next phase's queue)
  std::int32_t blocks = 0;         // 0: persistent grid sized to the device
  RetireRule rule{};
  bool stopWhenStable = false;     // the reference's calm rule (a sweep's "stopWhenStable"); exclusive with `rule`
  bool claimByIndex = false;       // phases after the first claim by index instead of fewest steps done first
  bool stageColumns = false;       // every block copies the column table into its shared memory (single-model batches;
                                   // a phase whose blocks lack the room takes simulations off its blocks to make it)
  int device = 0;
};

struct DeviceInfo {
  std::string name;
  int major = 0, minor = 0, multiprocessors = 0;
  std::size_t globalMemory = 0, sharedPerBlockOptIn = 0, sharedPerSM = 0;
  int runtimeVersion = 0, driverVersion = 0;
};

bool cuda_available(std::string* why);
DeviceInfo device_info(int device);

// One launch phase: teams of teamWarps warps, teamsPerBlock per block, a persistent grid of `blocks`.
struct PhaseConfig {
  int teamWarps = 0, teamsPerBlock = 0, blocks = 0, blocksPerSM = 0;
  int yieldBelow = 0;  // the phase pauses its instances once at most this many remain (0: never)
  bool stageColumns = false;  // its blocks hold the column table in shared memory
  SlotLayout layout{};
};

// Launch phases in order. Each phase's teams are twice the size of the previous phase's; a phase hands its
// unfinished instances to the next once they fit in the next phase's resident teams.
struct LaunchConfig {
  std::vector<PhaseConfig> phases;
  std::size_t slotBytes = 0;
  const PhaseConfig& main() const { return phases.front(); }
  PhaseConfig tail() const { return phases.size() > 1 ? phases.back() : PhaseConfig{}; }
};

// Does launch phase k claim its instances fewest steps done first (launch_order_unfinished) rather than by index?
// Phases after the first of a run that goes to the end in one graph, unless opt.claimByIndex.
bool ordered_phase(const BatchOptions& opt, const LaunchConfig& cfg, std::size_t k);

// The kernels of one run that goes to the end in one graph, in launch order: the counters' reset (start_run), then per
// phase its claim-order kernels (compact_unfinished + rank_unfinished, only where ordered_phase holds) and the phase's
// batch kernel. A caller's claim order for the first phase adds no kernel (it is uploaded, not computed). Batch::launch
// captures exactly this list, and kernels_per_run counts it, so the two cannot disagree.
struct PlanStep {
  enum Kind { kStartRun = 0, kClaimOrder = 1, kPhase = 2 } kind;
  int phase;  // the launch phase the step belongs to (-1 for kStartRun)
};
std::vector<PlanStep> run_plan(const BatchOptions& opt, const LaunchConfig& cfg);
// Kernel launches of one run that goes to the end in one graph: start_run 1, each claim order 2, each phase 1.
int kernels_per_run(const BatchOptions& opt, const LaunchConfig& cfg);

class Batch {
 public:
  Batch(std::shared_ptr<const CompiledShip> ship, const CompiledSim& sim, const BatchOptions& opt);
  // A fleet: instance i steps models[instanceModel[i]] (opt.count is the number of instances). Every instance of every
  // model runs in the same launches; per-instance setters and results work as for one model, except sweeps, traces,
  // batch-results files and the no-allocation run, which hold one model.
  Batch(std::vector<std::pair<std::shared_ptr<const CompiledShip>, CompiledSim>> models, std::vector<std::int32_t> instanceModel,
        const BatchOptions& opt);
  ~Batch();
  Batch(const Batch&) = delete;
  Batch& operator=(const Batch&) = delete;

  // Per-instance setup before run(): a state record (10 + 5 N values, the trace record layout) and connection fields.
  void restore(std::int32_t inst, const double* record);
  void set_connection_enabled(std::int32_t inst, std::int32_t c, bool en);
  void set_connection_area(std::int32_t inst, std::int32_t c, double area);
  void set_connection_activation(std::int32_t inst, std::int32_t c, double tOn);
  // set_connection_area over a block: area of connection conns[j] of instance first + i = areas[i * nConns + j]. Every
  // index is checked before anything is written, so a call that throws changes nothing.
  void set_connection_areas(std::int32_t first, std::int32_t count, std::int32_t nConns, const std::int32_t* conns, const double* areas);
  // The first launch phase claims the instances in this order (a permutation of 0 .. count-1) instead of by index:
  // a caller who knows which runs are long (an earlier evaluation of similar points) lists them first, so that they
  // do not start last and end the batch late. The results do not depend on it.
  void set_claim_order(const std::int32_t* order, std::int32_t n);
  // Instance i takes sweep instance first + i (a shard of a larger sweep when first > 0 or the sweep is longer);
  // results() then names the instances by those sweep instances' ids.
  void apply_sweep(const Sweep& sw, std::int32_t first = 0);
  std::int32_t sweep_first() const { return sweepFirst_; }

  // run() = upload() + launch() + download(); returns the wall seconds of all three.
  double run();
  // Makes the batch runnable again from its staged inputs (the setters' values persist); the last results stay
  // readable until the next download().
  void reset();
  void upload();
  // Runs every instance to its end on the device; returns the device time in milliseconds (CUDA events on the
  // launching stream).
  float launch();
  void download();

  const BatchOptions& options() const { return opt_; }
  const LaunchConfig& launch_config() const { return cfg_; }
  std::int64_t total_steps() const;
  // HealthBit flags of the last launch() (0: nothing to report): kHealthNonFinite when an instance's state went NaN or
  // infinite. Read back with the run's timing; the results themselves are unchanged.
  std::int32_t health() const;
  // The last launch() by phase: its team size, device time (CUDA events around its kernel launches) and the steps its
  // kernels took.
  struct PhaseStats {
    int teamWarps;
    float deviceMs;
    std::int64_t steps;
  };
  std::vector<PhaseStats> phase_stats() const;
  std::size_t slot_bytes() const;
  std::int32_t nodes() const;        // of the first model
  std::int32_t connections() const;  // of the first model
  std::int32_t models() const;
  struct InstanceShape {
    std::int32_t model, nodes, connections;
  };
  InstanceShape instance_shape(std::int32_t inst) const;
  // h2d and d2h bytes of one run() (the per-instance inputs and the results that download() reads back)
  std::size_t upload_bytes() const;
  std::size_t download_bytes() const;

  struct Summary {
    bool foundered;
    double founderT, tEnd;
    std::int64_t steps;
    std::int32_t stop;
    double outputs[7];  // inflow, Vb, hullTop, mw, bx, by, bz
  };
  Summary summary(std::int32_t inst) const;
  void state(std::int32_t inst, double* record) const;
  std::vector<EventRecord> events(std::int32_t inst) const;
  std::vector<int> event_kinds(std::int32_t inst) const;
  std::vector<int> event_ids(std::int32_t inst) const;  // monitor or mark index, -1 for the founder
  const CompiledSim& sim() const;

  // Runs `count` instances of this batch's model with the caller's device buffers and the library's fixed scratch
  // array: nothing is allocated on the device (see run_batch_noalloc). Numerics, tMax and the retire rule are the
  // batch's; one launch of single- or multi-warp teams chosen from count, no curves or traces.
  void run_noalloc(const NoAllocRun& run, cudaStream_t stream) const;
  std::vector<CurveRecord> curve(std::int32_t inst) const;  // the device records closed by the final readouts
  CurveRecord final_readouts(std::int32_t inst) const;
  Trace trace(std::int32_t inst) const;
  Results results(const Sweep* sw) const;
  std::string engine_name() const;

 private:
  void init(std::vector<std::pair<std::shared_ptr<const CompiledShip>, CompiledSim>> models, std::vector<std::int32_t> instanceModel);
  struct Impl;
  std::unique_ptr<Impl> I_;
  BatchOptions opt_;
  LaunchConfig cfg_;
  std::int32_t sweepFirst_ = 0;
};

}  // namespace ssb
