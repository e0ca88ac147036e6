// sinksim_sweep: run a sweep file on the B200 and write its results, or compare two results files exactly; a
// drop-in for the reference's CPU sweep runner (apps/sinksim_sweep.cpp of the reference) with the same options:
//   sinksim_sweep <ship.json> <sim.json> <sweep.json> [--numerics portable|portable32] [--threads N] [--results out.json]
//   sinksim_sweep --compare a.results.json b.results.json
// The GPU computes the portable numerics; "oracle" and "std" exist on the reference's CPU engine only. --threads is
// accepted and ignored. Without --numerics the portable numerics are used (the reference's CPU default is oracle).
#include <algorithm>
#include <cstdio>
#include <exception>
#include <string>

#include "../batch.h"
#include "../model.h"
#include "../sweep.h"
#include "cli.h"

using namespace ssb;

int main(int argc, char** argv) {
  const cli::Args args = cli::Args::parse(argc, argv, {});
  try {
    if (args.has("compare")) {
      if (args.positional.size() < 1) {
        std::fprintf(stderr, "usage: sinksim_sweep --compare a.results.json b.results.json\n");
        return 2;
      }
      const Results a = load_results(args.get("compare", ""));
      const Results b = load_results(args.positional[0]);
      const Diff d = compare_results(a, b);
      std::printf("compared %zu values over %zu instances: %zu differ", d.compared, a.instances.size(), d.differing);
      if (d.differing) std::printf("; largest |diff| %.3e; first: %s", d.maxAbs, d.first.c_str());
      std::printf("\nRESULT: %s\n", d.differing == 0 ? "IDENTICAL" : "DIFFERENT");
      return d.differing == 0 ? 0 : 1;
    }
    if (args.positional.size() < 3) {
      std::fprintf(stderr,
                   "usage: sinksim_sweep <ship.json> <sim.json> <sweep.json> [--numerics portable|portable32] [--threads N] [--results out.json]\n"
                   "       sinksim_sweep --compare a.results.json b.results.json\n");
      return 2;
    }
    const std::string numerics = args.get("numerics", "portable");
    if (numerics == "oracle" || numerics == "std") {
      std::fprintf(stderr, "numerics %s runs on the reference CPU engine only; the GPU engine computes portable or portable32\n", numerics.c_str());
      return 2;
    }
    if (numerics != "portable" && numerics != "portable32") {
      std::fprintf(stderr, "unknown --numerics %s (use portable or portable32)\n", numerics.c_str());
      return 2;
    }
    const auto ship = load_ship(args.positional[0]);
    const CompiledSim sim = load_sim(args.positional[1]);
    check_pairing(*ship, sim);
    const Sweep sw = load_sweep(args.positional[2], sim);
    if (sw.instances.empty()) throw std::runtime_error("the sweep has no instances");
    std::printf("sweep of %zu instances on %s / %s, numerics %s, tMax %s, curve every %g s, GPU\n", sw.instances.size(), ship->id.c_str(), sim.id.c_str(),
                numerics.c_str(), cli::minutes(sw.tMax).c_str(), sw.every);
    BatchOptions opt;
    opt.count = static_cast<std::int32_t>(sw.instances.size());
    opt.mixedPrecision = numerics == "portable32";
    opt.tracedInstances = 0;
    opt.tMax = sw.tMax;
    opt.curveEvery = sw.every;
    opt.stopWhenStable = sw.stopWhenStable;
    Batch batch(ship, sim, opt);
    batch.apply_sweep(sw);
    const double s = batch.run();
    const std::int64_t steps = batch.total_steps();
    Results r = batch.results(&sw);
    r.tMax = sw.tMax;
    r.every = sw.every;
    int foundered = 0;
    for (const InstanceResult& in : r.instances) foundered += in.foundered ? 1 : 0;
    std::printf("%lld steps in %.2f s (%.0f steps/s aggregate); %d of %zu instances foundered\n", static_cast<long long>(steps), s, steps / s, foundered,
                r.instances.size());
    for (std::size_t i = 0; i < std::min<std::size_t>(r.instances.size(), 12); ++i) {
      const InstanceResult& in = r.instances[i];
      std::printf("  %-16s %s  trim %.2f  list %.2f  water %.0f t\n", in.id.c_str(),
                  in.foundered ? ("founders at " + cli::minutes(in.founderT)).c_str() : "afloat", in.fTrim, in.fList, in.fWater);
    }
    if (r.instances.size() > 12) std::printf("  ... %zu more\n", r.instances.size() - 12);
    if (args.has("results")) {
      save_results(r, args.get("results", ""));
      std::printf("wrote %s\n", args.get("results", "").c_str());
    }
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "sinksim_sweep: %s\n", e.what());
    return 1;
  }
}
