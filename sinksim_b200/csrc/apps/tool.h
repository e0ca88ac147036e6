// What the two drop-in tools share: an option table and its parser, the sweep run both of them offer, and the
// summaries they print. The option names, their defaults, the exit codes (2 for a usage error, 1 for a failure) and the
// summary lines that scripts read ("N steps in S s (R steps/s aggregate)", "RESULT: IDENTICAL|DIFFERENT") are the
// reference tools' (apps/sinksim_sweep.cpp, apps/sinksim_cuda_run.cpp, apps/cli.hpp of the reference); the
// table-driven parser and the shared runner are this project's.
#pragma once

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../batch.h"
#include "../model.h"
#include "../sweep.h"

namespace ssb::tool {

// One option a tool declares: --name followed by a value, or a switch.
struct Option {
  const char* name;
  bool takesValue;
  const char* fallback;  // the value when the option is absent (nullptr: none)
};

// The parsed command line: positional arguments and the declared options that were given. An option missing its value
// is a usage error (exit 2); an option the tool does not declare is reported on stderr and ignored, as the reference
// tools ignore options they do not read.
class CommandLine {
 public:
  CommandLine(int argc, char** argv, const std::vector<Option>& table, const char* usage) : usage_(usage) {
    for (const Option& o : table) declared_[o.name] = o;
    for (int i = 1; i < argc; ++i) {
      const std::string arg = argv[i];
      if (arg.rfind("--", 0) != 0 || arg.size() <= 2) {
        positional_.push_back(arg);
        continue;
      }
      const std::string name = arg.substr(2);
      const auto it = declared_.find(name);
      const bool takesValue = it == declared_.end() || it->second.takesValue;
      if (takesValue && i + 1 >= argc) {
        std::fprintf(stderr, "option --%s needs a value\n", name.c_str());
        std::exit(2);
      }
      const std::string value = takesValue ? argv[++i] : "";
      if (it == declared_.end()) std::fprintf(stderr, "ignoring option --%s (this tool does not read it)\n", name.c_str());
      else given_[name] = value;
    }
  }
  [[noreturn]] void usage_error(const std::string& why = "") const {
    if (!why.empty()) std::fprintf(stderr, "%s\n", why.c_str());
    std::fprintf(stderr, "%s", usage_);
    std::exit(2);
  }
  const std::vector<std::string>& positional() const { return positional_; }
  bool given(const std::string& name) const { return given_.count(name) != 0; }
  std::string text(const std::string& name) const {
    const auto g = given_.find(name);
    if (g != given_.end()) return g->second;
    const auto d = declared_.find(name);
    return d != declared_.end() && d->second.fallback ? d->second.fallback : "";
  }
  double number(const std::string& name) const {
    const std::string s = text(name);
    char* end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    if (s.empty() || (end && *end)) usage_error("option --" + name + " needs a number, got \"" + s + "\"");
    return v;
  }

 private:
  const char* usage_;
  std::map<std::string, Option> declared_;
  std::map<std::string, std::string> given_;
  std::vector<std::string> positional_;
};

inline std::string minutes(double seconds) {
  char buf[32];
  std::snprintf(buf, sizeof buf, "%.2f min", seconds / 60.0);
  return buf;
}

inline int foundered_count(const Results& r) {
  return static_cast<int>(std::count_if(r.instances.begin(), r.instances.end(), [](const InstanceResult& in) { return in.foundered; }));
}

// The per-instance lines both tools print (the first twelve instances).
inline void print_instances(const Results& r) {
  const std::size_t shown = std::min<std::size_t>(r.instances.size(), 12);
  for (std::size_t i = 0; i < shown; ++i) {
    const InstanceResult& in = r.instances[i];
    const std::string fate = in.foundered ? "founders at " + minutes(in.founderT) : "afloat";
    std::printf("  %-16s %s  trim %.2f  list %.2f  water %.0f t\n", in.id.c_str(), fate.c_str(), in.fTrim, in.fList, in.fWater);
  }
  if (r.instances.size() > shown) std::printf("  ... %zu more\n", r.instances.size() - shown);
}

// A sweep file run on the GPU: one batch of all its instances, the calm rule when the sweep asks for it.
struct SweepRun {
  Results results;
  std::int64_t steps = 0;
  double seconds = 0;
};

inline SweepRun run_sweep_file(std::shared_ptr<const CompiledShip> ship, const CompiledSim& sim, const Sweep& sw, bool mixed,
                               std::int64_t stepsPerLaunch) {
  if (sw.instances.empty()) throw std::runtime_error("the sweep has no instances");
  BatchOptions opt;
  opt.count = static_cast<std::int32_t>(sw.instances.size());
  opt.mixedPrecision = mixed;
  opt.tracedInstances = 0;
  opt.tMax = sw.tMax;
  opt.curveEvery = sw.every;
  opt.stopWhenStable = sw.stopWhenStable;
  opt.stepsPerLaunch = stepsPerLaunch;
  Batch batch(std::move(ship), sim, opt);
  batch.apply_sweep(sw);
  SweepRun run;
  run.seconds = batch.run();
  run.steps = batch.total_steps();
  run.results = batch.results(&sw);
  run.results.tMax = sw.tMax;
  run.results.every = sw.every;
  return run;
}

}  // namespace ssb::tool
