// sinksim_cuda_run: the B200 batch runner, a drop-in for the reference's tool of the same name
// (apps/sinksim_cuda_run.cpp of the reference) with the same options and outputs:
//   sinksim_cuda_run <ship.json> <sim.json> [--count N] [--precision mixed|double] [--tmax S] [--trace out.json]
//                    [--dense N] [--sample-every S] [--steps-per-launch K] [--perturb]
//   sinksim_cuda_run <ship.json> <sim.json> --sweep sweep.json --results out.json [--precision mixed|double]
// --precision mixed (default) computes the portable32 numerics, double the portable numerics; --numerics
// portable|portable32 is accepted as well. --perturb scales the breach kind of instance i >= 1 by 1 + 0.02 i / count.
// --steps-per-launch 0 (the default here) runs every instance to its end in one persistent launch.
#include <algorithm>
#include <cstdio>
#include <exception>
#include <string>

#include "../batch.h"
#include "../model.h"
#include "../sweep.h"
#include "cli.h"

using namespace ssb;

namespace {

int run_sweep(const cli::Args& args, std::shared_ptr<const CompiledShip> ship, const CompiledSim& sim, bool mixed, const DeviceInfo& info) {
  const Sweep sw = load_sweep(args.get("sweep", ""), sim);
  if (sw.instances.empty()) throw std::runtime_error("the sweep has no instances");
  BatchOptions opt;
  opt.stopWhenStable = sw.stopWhenStable;  // the reference's GPU runner refused these sweeps; this engine runs them
  opt.count = static_cast<std::int32_t>(sw.instances.size());
  opt.mixedPrecision = mixed;
  opt.tracedInstances = 0;
  opt.tMax = sw.tMax;
  opt.curveEvery = sw.every;
  opt.stepsPerLaunch = static_cast<std::int64_t>(args.num("steps-per-launch", 0));
  std::printf("sweep of %zu instances on %s / %s, numerics %s, tMax %s, curve every %g s\n", sw.instances.size(), ship->id.c_str(), sim.id.c_str(),
              mixed ? "portable32" : "portable", cli::minutes(sw.tMax).c_str(), sw.every);
  Batch batch(ship, sim, opt);
  batch.apply_sweep(sw);
  const double seconds = batch.run();
  const std::int64_t steps = batch.total_steps();
  std::printf("%lld steps in %.2f s (%.0f steps/s aggregate)\n", static_cast<long long>(steps), seconds, steps / seconds);
  Results r = batch.results(&sw);
  r.tMax = sw.tMax;
  r.every = sw.every;
  int foundered = 0;
  for (const InstanceResult& in : r.instances) foundered += in.foundered ? 1 : 0;
  std::printf("%d of %d instances foundered\n", foundered, opt.count);
  for (std::size_t i = 0; i < std::min<std::size_t>(r.instances.size(), 12); ++i) {
    const InstanceResult& in = r.instances[i];
    std::printf("  %-16s %s  trim %.2f  list %.2f  water %.0f t\n", in.id.c_str(),
                in.foundered ? ("founders at " + cli::minutes(in.founderT)).c_str() : "afloat", in.fTrim, in.fList, in.fWater);
  }
  if (r.instances.size() > 12) std::printf("  ... %zu more\n", r.instances.size() - 12);
  (void)info;
  if (args.has("results")) {
    save_results(r, args.get("results", ""));
    std::printf("wrote %s\n", args.get("results", "").c_str());
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  const cli::Args args = cli::Args::parse(argc, argv, {"perturb"});
  if (args.positional.size() < 2) {
    std::fprintf(stderr,
                 "usage: sinksim_cuda_run <ship.json> <sim.json> [--count N] [--precision mixed|double] [--tmax S] [--trace out.json] [--dense N] "
                 "[--sample-every S] [--steps-per-launch K] [--perturb]\n"
                 "       sinksim_cuda_run <ship.json> <sim.json> --sweep sweep.json --results out.json [--precision mixed|double]\n");
    return 2;
  }
  std::string precision = args.get("precision", "mixed");
  if (args.has("numerics")) {
    const std::string n = args.get("numerics", "");
    if (n == "portable") precision = "double";
    else if (n == "portable32") precision = "mixed";
    else {
      std::fprintf(stderr, "numerics %s is not available on the GPU (use portable or portable32)\n", n.c_str());
      return 2;
    }
  }
  if (precision != "mixed" && precision != "double") {
    std::fprintf(stderr, "unknown --precision %s (use mixed or double)\n", precision.c_str());
    return 2;
  }
  try {
    std::string why;
    if (!cuda_available(&why)) {
      std::fprintf(stderr, "sinksim_cuda_run: no usable CUDA device (%s)\n", why.c_str());
      return 1;
    }
    const DeviceInfo info = device_info(0);
    const auto ship = load_ship(args.positional[0]);
    const CompiledSim sim = load_sim(args.positional[1]);
    check_pairing(*ship, sim);
    std::printf("device %s (sm_%d%d, %d SMs, %.1f GiB); runtime %d, driver %d\n", info.name.c_str(), info.major, info.minor, info.multiprocessors,
                info.globalMemory / 1073741824.0, info.runtimeVersion, info.driverVersion);
    if (args.has("sweep")) return run_sweep(args, ship, sim, precision == "mixed", info);

    BatchOptions opt;
    opt.count = static_cast<std::int32_t>(args.num("count", 1));
    opt.mixedPrecision = precision == "mixed";
    opt.tMax = args.num("tmax", 5 * 3600);
    opt.tracedInstances = args.has("trace") ? 1 : 0;
    opt.denseSteps = static_cast<std::int32_t>(args.num("dense", 400));
    opt.sampleEvery = args.num("sample-every", 60);
    opt.stepsPerLaunch = static_cast<std::int64_t>(args.num("steps-per-launch", 0));
    std::printf("ship %s: %d columns, %d segments, %d nodes; sim %s: %d groups, %d connections; batch of %d\n", ship->id.c_str(), ship->columns(),
                ship->segments(), ship->nodes(), sim.id.c_str(), sim.groups(), sim.connections(), opt.count);
    Batch batch(ship, sim, opt);
    const LaunchConfig& lc = batch.launch_config();
    std::printf("numerics %s; shared memory per simulation %zu bytes; %d-warp simulations, %d per block, %d blocks",
                opt.mixedPrecision ? "portable32 (mixed precision)" : "portable (double precision)", batch.slot_bytes(), lc.main().teamWarps,
                lc.main().teamsPerBlock, lc.main().blocks);
    for (std::size_t k = 1; k < lc.phases.size(); ++k)
      std::printf("; the last %d in %d-warp simulations", lc.phases[k - 1].yieldBelow, lc.phases[k].teamWarps);
    std::printf("\n");
    if (args.flag("perturb")) {
      const std::int32_t breachKind = sim.kindIndex("breach");
      for (std::int32_t i = 1; i < opt.count; ++i) {
        const double scale = 1 + 0.02 * static_cast<double>(i) / static_cast<double>(opt.count);
        for (std::int32_t c = 0; c < sim.connections(); ++c)
          if (breachKind >= 0 && sim.cKind[static_cast<std::size_t>(c)] == static_cast<std::uint8_t>(breachKind))
            batch.set_connection_area(i, c, sim.cArea[static_cast<std::size_t>(c)] * scale);
      }
    }
    const double seconds = batch.run();
    const std::int64_t steps = batch.total_steps();
    const Batch::Summary s0 = batch.summary(0);
    std::printf("%lld steps over %d instances in %.3f s: %.0f steps/s aggregate, %.1f simulated hours per wall second, %.0f full sinkings per minute at this length\n",
                static_cast<long long>(steps), opt.count, seconds, steps / seconds, steps * sim.dt / 3600.0 / seconds,
                (steps / seconds) / (s0.steps > 0 ? static_cast<double>(s0.steps) : 1.0) * 60.0);
    double tMin = 1e9, tMaxF = -1;
    int foundered = 0;
    for (std::int32_t i = 0; i < opt.count; ++i) {
      const Batch::Summary s = batch.summary(i);
      if (s.foundered) { ++foundered; tMin = std::min(tMin, s.founderT); tMaxF = std::max(tMaxF, s.founderT); }
    }
    if (foundered) std::printf("%d of %d instances foundered, between %s and %s\n", foundered, opt.count, cli::minutes(tMin).c_str(), cli::minutes(tMaxF).c_str());
    else std::printf("no instance foundered within %s\n", cli::minutes(opt.tMax).c_str());
    for (const EventRecord& e : batch.events(0)) std::printf("  %9.2f min  %s\n", e.t / 60, e.label.c_str());
    if (args.has("trace")) {
      const Trace tr = batch.trace(0);
      save_trace(tr, args.get("trace", "cuda.trace.json"));
      std::printf("wrote %s with %d dense and %d sampled records\n", args.get("trace", "cuda.trace.json").c_str(), tr.dense.n, tr.samples.n);
    }
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "sinksim_cuda_run: %s\n", e.what());
    return 1;
  }
}
