// sinksim_cuda_run: the GPU batch runner, a drop-in for the reference's tool of the same name
// (apps/sinksim_cuda_run.cpp of the reference), with its options, defaults and outputs:
//   sinksim_cuda_run <ship.json> <sim.json> [--count N] [--precision mixed|double] [--tmax S] [--trace out.json]
//                    [--dense N] [--sample-every S] [--steps-per-launch K] [--perturb]
//   sinksim_cuda_run <ship.json> <sim.json> --sweep sweep.json [--results out.json] [--precision mixed|double]
// --precision mixed (the default) computes the portable32 numerics, double the portable numerics; --numerics
// portable|portable32 names them directly. --perturb scales the breach connections of instance i >= 1 by
// 1 + 0.02 i / count. --steps-per-launch bounds the steps of one launch (2000 by default, as in the reference; results do
// not depend on it); 0 runs every instance to its end in one persistent launch. Sweeps with stopWhenStable, which
// the reference's GPU runner refused, run here with the calm rule.
#include <algorithm>
#include <cstdio>
#include <exception>
#include <string>

#include "tool.h"

using namespace ssb;

namespace {

const char* const kUsage =
    "usage: sinksim_cuda_run <ship.json> <sim.json> [--count N] [--precision mixed|double] [--tmax S] [--trace out.json] [--dense N]\n"
    "                        [--sample-every S] [--steps-per-launch K] [--perturb]\n"
    "       sinksim_cuda_run <ship.json> <sim.json> --sweep sweep.json [--results out.json] [--precision mixed|double]\n";

// mixed (portable32) or double (portable), from --precision or --numerics
bool mixed_precision(const tool::CommandLine& cl) {
  if (cl.given("numerics")) {
    const std::string n = cl.text("numerics");
    if (n == "portable") return false;
    if (n == "portable32") return true;
    cl.usage_error("numerics " + n + " is not available on the GPU (use portable or portable32)");
  }
  const std::string p = cl.text("precision");
  if (p != "mixed" && p != "double") cl.usage_error("unknown --precision " + p + " (use mixed or double)");
  return p == "mixed";
}

int sweep_mode(const tool::CommandLine& cl, std::shared_ptr<const CompiledShip> ship, const CompiledSim& sim, bool mixed) {
  const Sweep sw = load_sweep(cl.text("sweep"), sim);
  std::printf("sweep of %zu instances on %s / %s, numerics %s, tMax %s, curve every %g s\n", sw.instances.size(), ship->id.c_str(), sim.id.c_str(),
              mixed ? "portable32" : "portable", tool::minutes(sw.tMax).c_str(), sw.every);
  const tool::SweepRun run = tool::run_sweep_file(ship, sim, sw, mixed, static_cast<std::int64_t>(cl.number("steps-per-launch")));
  std::printf("%lld steps in %.2f s (%.0f steps/s aggregate)\n", static_cast<long long>(run.steps), run.seconds, run.steps / run.seconds);
  std::printf("%d of %zu instances foundered\n", tool::foundered_count(run.results), run.results.instances.size());
  tool::print_instances(run.results);
  if (cl.given("results")) {
    save_results(run.results, cl.text("results"));
    std::printf("wrote %s\n", cl.text("results").c_str());
  }
  return 0;
}

// The breach connections of instance i >= 1 scaled by 1 + 0.02 i / count.
void perturb(Batch& batch, const CompiledSim& sim, std::int32_t count) {
  const std::int32_t breach = sim.kindIndex("breach");
  if (breach < 0) return;
  for (std::int32_t c = 0; c < sim.connections(); ++c) {
    if (sim.cKind[static_cast<std::size_t>(c)] != static_cast<std::uint8_t>(breach)) continue;
    for (std::int32_t i = 1; i < count; ++i)
      batch.set_connection_area(i, c, sim.cArea[static_cast<std::size_t>(c)] * (1 + 0.02 * static_cast<double>(i) / static_cast<double>(count)));
  }
}

int batch_mode(const tool::CommandLine& cl, std::shared_ptr<const CompiledShip> ship, const CompiledSim& sim, bool mixed) {
  BatchOptions opt;
  opt.count = static_cast<std::int32_t>(cl.number("count"));
  opt.mixedPrecision = mixed;
  opt.tMax = cl.number("tmax");
  opt.tracedInstances = cl.given("trace") ? 1 : 0;
  opt.denseSteps = static_cast<std::int32_t>(cl.number("dense"));
  opt.sampleEvery = cl.number("sample-every");
  opt.stepsPerLaunch = static_cast<std::int64_t>(cl.number("steps-per-launch"));
  std::printf("ship %s: %d columns, %d segments, %d nodes; sim %s: %d groups, %d connections; batch of %d\n", ship->id.c_str(), ship->columns(),
              ship->segments(), ship->nodes(), sim.id.c_str(), sim.groups(), sim.connections(), opt.count);
  Batch batch(ship, sim, opt);
  const LaunchConfig& lc = batch.launch_config();
  std::printf("numerics %s; shared memory per simulation %zu bytes; %d-warp simulations, %d per block, %d blocks",
              mixed ? "portable32 (mixed precision)" : "portable (double precision)", batch.slot_bytes(), lc.main().teamWarps, lc.main().teamsPerBlock,
              lc.main().blocks);
  for (std::size_t k = 1; k < lc.phases.size(); ++k) std::printf("; the last %d in %d-warp simulations", lc.phases[k - 1].yieldBelow, lc.phases[k].teamWarps);
  std::printf("\n");
  if (cl.given("perturb")) perturb(batch, sim, opt.count);
  const double seconds = batch.run();
  const std::int64_t steps = batch.total_steps();
  const double rate = steps / seconds;
  const double first = static_cast<double>(std::max<std::int64_t>(batch.summary(0).steps, 1));
  std::printf("%lld steps over %d instances in %.3f s: %.0f steps/s aggregate, %.1f simulated hours per wall second, %.0f full sinkings per minute at this length\n",
              static_cast<long long>(steps), opt.count, seconds, rate, steps * sim.dt / 3600.0 / seconds, rate / first * 60.0);
  double earliest = 1e300, latest = -1;
  int foundered = 0;
  for (std::int32_t i = 0; i < opt.count; ++i) {
    const Batch::Summary s = batch.summary(i);
    if (!s.foundered) continue;
    ++foundered;
    earliest = std::min(earliest, s.founderT);
    latest = std::max(latest, s.founderT);
  }
  if (foundered)
    std::printf("%d of %d instances foundered, between %s and %s\n", foundered, opt.count, tool::minutes(earliest).c_str(), tool::minutes(latest).c_str());
  else
    std::printf("no instance foundered within %s\n", tool::minutes(opt.tMax).c_str());
  for (const EventRecord& e : batch.events(0)) std::printf("  %9.2f min  %s\n", e.t / 60, e.label.c_str());
  if (cl.given("trace")) {
    const Trace tr = batch.trace(0);
    save_trace(tr, cl.text("trace"));
    std::printf("wrote %s with %d dense and %d sampled records\n", cl.text("trace").c_str(), tr.dense.n, tr.samples.n);
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  const tool::CommandLine cl(argc, argv,
                             {{"count", true, "1"}, {"precision", true, "mixed"}, {"numerics", true, nullptr}, {"tmax", true, "18000"},
                              {"trace", true, nullptr}, {"dense", true, "400"}, {"sample-every", true, "60"}, {"steps-per-launch", true, "2000"},
                              {"perturb", false, nullptr}, {"sweep", true, nullptr}, {"results", true, nullptr}},
                             kUsage);
  if (cl.positional().size() < 2) cl.usage_error();
  const bool mixed = mixed_precision(cl);
  for (const char* numeric : {"count", "tmax", "dense", "sample-every", "steps-per-launch"}) cl.number(numeric);  // usage errors first
  if (cl.number("count") < 1) cl.usage_error("--count must be at least 1");
  try {
    std::string why;
    if (!cuda_available(&why)) {
      std::fprintf(stderr, "sinksim_cuda_run: no usable CUDA device (%s)\n", why.c_str());
      return 1;
    }
    const DeviceInfo info = device_info(0);
    const auto ship = load_ship(cl.positional()[0]);
    const CompiledSim sim = load_sim(cl.positional()[1]);
    check_pairing(*ship, sim);
    std::printf("device %s (sm_%d%d, %d SMs, %.1f GiB); runtime %d, driver %d\n", info.name.c_str(), info.major, info.minor, info.multiprocessors,
                info.globalMemory / 1073741824.0, info.runtimeVersion, info.driverVersion);
    return cl.given("sweep") ? sweep_mode(cl, ship, sim, mixed) : batch_mode(cl, ship, sim, mixed);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "sinksim_cuda_run: %s\n", e.what());
    return 1;
  }
}
