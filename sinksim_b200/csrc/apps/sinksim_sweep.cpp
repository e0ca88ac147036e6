// sinksim_sweep: runs a sweep file on the GPU and writes its batch-results, or compares two batch-results files value
// for value. A drop-in for the reference's CPU sweep runner (apps/sinksim_sweep.cpp of the reference):
//   sinksim_sweep <ship.json> <sim.json> <sweep.json> --numerics portable|portable32 [--threads N] [--results out.json]
//   sinksim_sweep --compare a.results.json b.results.json
// The GPU computes the portable numerics. The reference's default numerics, oracle (and std), exist on its CPU engine
// only, so --numerics must be given: without it, or with oracle or std, the tool stops with exit code 2 instead of
// silently computing other numbers. --threads sizes the reference's CPU pool; here every instance runs at once and
// the value is only reported.
#include <cstdio>
#include <exception>
#include <string>

#include "tool.h"

using namespace ssb;

namespace {

const char* const kUsage =
    "usage: sinksim_sweep <ship.json> <sim.json> <sweep.json> --numerics portable|portable32 [--threads N] [--results out.json]\n"
    "       sinksim_sweep --compare a.results.json b.results.json\n";

int compare(const tool::CommandLine& cl) {
  if (cl.positional().empty()) cl.usage_error();
  const Results a = load_results(cl.text("compare"));
  const Results b = load_results(cl.positional()[0]);
  const Diff d = compare_results(a, b);
  std::printf("compared %zu values over %zu instances: %zu differ", d.compared, a.instances.size(), d.differing);
  if (d.differing) std::printf("; largest |diff| %.3e; first: %s", d.maxAbs, d.first.c_str());
  std::printf("\nRESULT: %s\n", d.differing == 0 ? "IDENTICAL" : "DIFFERENT");
  return d.differing == 0 ? 0 : 1;
}

}  // namespace

int main(int argc, char** argv) {
  const tool::CommandLine cl(argc, argv,
                             {{"numerics", true, nullptr}, {"threads", true, "0"}, {"results", true, nullptr}, {"compare", true, nullptr}}, kUsage);
  try {
    if (cl.given("compare")) return compare(cl);
    if (cl.positional().size() < 3) cl.usage_error();
    if (!cl.given("numerics"))
      cl.usage_error("sinksim_sweep: give --numerics portable or portable32 (the reference's default, oracle, runs on its CPU engine only)");
    const std::string numerics = cl.text("numerics");
    if (numerics == "oracle" || numerics == "std")
      cl.usage_error("sinksim_sweep: numerics " + numerics + " runs on the reference's CPU engine only; the GPU computes portable or portable32");
    if (numerics != "portable" && numerics != "portable32") cl.usage_error("unknown --numerics " + numerics + " (use portable or portable32)");
    const auto ship = load_ship(cl.positional()[0]);
    const CompiledSim sim = load_sim(cl.positional()[1]);
    check_pairing(*ship, sim);
    const Sweep sw = load_sweep(cl.positional()[2], sim);
    std::printf("sweep of %zu instances on %s / %s, numerics %s, tMax %s, curve every %g s, GPU (--threads %d not used)\n", sw.instances.size(),
                ship->id.c_str(), sim.id.c_str(), numerics.c_str(), tool::minutes(sw.tMax).c_str(), sw.every, static_cast<int>(cl.number("threads")));
    const tool::SweepRun run = tool::run_sweep_file(ship, sim, sw, numerics == "portable32", 0);
    std::printf("%lld steps in %.2f s (%.0f steps/s aggregate); %d of %zu instances foundered\n", static_cast<long long>(run.steps), run.seconds,
                run.steps / run.seconds, tool::foundered_count(run.results), run.results.instances.size());
    tool::print_instances(run.results);
    if (cl.given("results")) {
      save_results(run.results, cl.text("results"));
      std::printf("wrote %s\n", cl.text("results").c_str());
    }
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "sinksim_sweep: %s\n", e.what());
    return 1;
  }
}
