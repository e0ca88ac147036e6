// Sweeps ("sinksim.sweep"), their application to instances, and batch results ("sinksim.batch-results"): the
// file formats and semantics of the reference's sweep module (engine/include/sinksim/sweep.hpp:20-108,
// engine/src/sweep.cpp:30-281), and traces ("sinksim.trace", engine/src/trace.cpp:272-308).
#pragma once

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "model.h"

namespace ssb {

struct ConnectionOverride {
  std::int32_t conn = -1;
  std::uint8_t kind = 255;
  std::int32_t idx = -1;  // -1: every connection of the kind
  bool hasEnabled = false, enabled = false;
  bool hasTOn = false;
  double tOn = 0;
  bool hasArea = false;
  double area = 0;
};

struct SweepInstance {
  std::string id;
  std::vector<std::pair<std::uint8_t, double>> kindScale;  // multiply the compiled area of every connection of the kind
  std::vector<ConnectionOverride> overrides;
};

struct Sweep {
  std::string ship, sim;
  double tMax = 5 * 3600;
  double every = 30;
  bool stopWhenStable = false;
  std::vector<SweepInstance> instances;
};

Sweep load_sweep(const std::string& path, const CompiledSim& sim);
void save_sweep(const Sweep& sw, const std::string& path, const CompiledSim& sim);

// Applies an instance to per-connection arrays (length nc each): kind scales first, each the single product
// compiled area x factor; then the overrides in the order written (sweep.hpp:49-65 of the reference).
void apply_instance(const SweepInstance& in, const CompiledSim& base, std::uint8_t* en, double* area, double* tOn);

struct CurveRecord {
  double t, trim, list, water, inflow, dF, dA;
};

struct EventRecord {
  double t;
  std::string id, label;
};

struct InstanceResult {
  std::string id;
  bool foundered = false;
  double founderT = -1;
  double tEnd = 0;
  std::int64_t steps = 0;
  double fTrim = 0, fList = 0, fWater = 0, fDraftF = 0, fDraftA = 0, fInflow = 0;
  std::vector<EventRecord> events;
  std::vector<CurveRecord> curve;
};

struct Results {
  std::string ship, sim, numerics, engine;
  double tMax = 0, every = 0;
  std::vector<InstanceResult> instances;
};

void save_results(const Results& r, const std::string& path);
Results load_results(const std::string& path);

struct Diff {
  std::size_t differing = 0, compared = 0;
  double maxAbs = 0;
  std::string first;
};
// Exact comparison of two results, value for value (engine/src/sweep.cpp:234-281 of the reference).
Diff compare_results(const Results& a, const Results& b);

struct TraceColumns {
  std::int32_t n = 0;
  std::vector<double> t, zO, pitch, roll, vz, wth, wph, inflow, Vb, hullTop;
  std::vector<double> vol, level, cx, cy, cz;  // flat, n * nodes
  // Appends one record in the device layout: 10 scalars then vol, level, cx, cy, cz per node.
  void push_record(const double* rec, std::int32_t nodes);
};

struct TraceEvent {
  double t;
  std::string id, label;
};

struct Trace {
  std::string role = "trace", ship, sim, title, producer, engine;
  double dt = 0;
  std::int32_t nodes = 0, denseSteps = 0;
  double sampleEvery = 0;
  std::int64_t steps = 0;
  double tEnd = 0;
  bool foundered = false;
  double founderT = -1;
  std::vector<TraceEvent> events;
  TraceColumns dense, samples;
};

void save_trace(const Trace& tr, const std::string& path);

}  // namespace ssb
