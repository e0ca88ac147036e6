// The extern "C" boundary (include/sinksim_b200.h): exceptions become status codes and a thread-local message.
#include "sinksim_b200.h"

#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>

#include <cuda_runtime.h>

#include "adjoint.h"
#include "batch.h"
#include "model.h"
#include "sweep.h"

namespace ssb {
void portable_math_host(int op, const double* x, const double* y, double* out, std::int64_t n);
cudaError_t portable_math_device(int op, const double* x, const double* y, double* out, std::int64_t n);
double measure_add_mul_peak(bool fp64, int device);
}  // namespace ssb

struct ssb_adjoint {
  std::unique_ptr<ssb::AdjointBatch> adj;
  std::int32_t nsamples = 0;
};

struct ssb_batch {
  std::shared_ptr<ssb::Batch> batch;
  std::unique_ptr<ssb::Sweep> sweep;  // the sweep applied by ssb_batch_apply_sweep, for instance ids
};

namespace {

thread_local std::string g_error;

struct Unsupported : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct NoDevice : std::runtime_error {
  using std::runtime_error::runtime_error;
};

template <class F>
int guard(F&& f) {
  try {
    f();
    return SSB_OK;
  } catch (const Unsupported& e) {
    g_error = e.what();
    return SSB_EUNSUPPORTED;
  } catch (const NoDevice& e) {
    g_error = e.what();
    return SSB_ENODEVICE;
  } catch (const std::invalid_argument& e) {
    g_error = e.what();
    return SSB_EINVAL;
  } catch (const std::out_of_range& e) {
    g_error = e.what();
    return SSB_EINVAL;
  } catch (const std::logic_error& e) {
    g_error = e.what();
    return SSB_ESTATE;
  } catch (const std::exception& e) {
    g_error = e.what();
    return SSB_ERUNTIME;
  } catch (...) {
    g_error = "unknown error";
    return SSB_ERUNTIME;
  }
}

void need(const void* p, const char* what) {
  if (!p) throw std::invalid_argument(std::string(what) + " is NULL");
}

ssb::BatchOptions to_options(const ssb_batch_options& o) {
  if (o.numerics != 0 && o.numerics != 1) throw Unsupported("numerics " + std::to_string(o.numerics) + " is not available on the GPU (0 portable, 1 portable32)");
  ssb::BatchOptions b;
  b.count = o.count;
  b.mixedPrecision = o.numerics == 1;
  b.tracedInstances = o.traced_instances;
  b.denseSteps = o.dense_steps;
  b.sampleEvery = o.sample_every;
  b.curveEvery = o.curve_every;
  b.tMax = o.t_max;
  b.stepsPerLaunch = o.steps_per_launch;
  b.teamWarps = o.team_warps;
  b.tailTeamWarps = o.tail_team_warps;
  b.teamsPerBlock = o.teams_per_block;
  b.yieldBelow = o.yield_below;
  b.blocks = o.blocks;
  b.device = o.device;
  b.rule.enabled = o.rule_enabled;
  b.rule.pitchLimit = o.rule_pitch;
  b.rule.xDeck = o.rule_x; b.rule.yDeck = o.rule_y; b.rule.zDeck = o.rule_z;
  b.rule.wthLimit = o.rule_wth;
  b.rule.settleTime = o.rule_settle;
  b.stopWhenStable = o.stop_when_stable != 0;
  if (o.handover_factor > 0) b.handoverFactor = o.handover_factor;
  b.claimByIndex = o.claim_by_index != 0;
  b.stageColumns = o.stage_columns != 0;
  return b;
}

void need_device() {
  std::string why;
  if (!ssb::cuda_available(&why)) throw NoDevice("no usable CUDA device (" + why + ")");
}

}  // namespace

extern "C" {

const char* ssb_last_error(void) { return g_error.c_str(); }
const char* ssb_version(void) { return "sinksim-b200 0.1.0"; }

int ssb_available(char* why, size_t cap) {
  std::string w;
  const bool ok = ssb::cuda_available(&w);
  if (why && cap) {
    std::strncpy(why, w.c_str(), cap - 1);
    why[cap - 1] = 0;
  }
  return ok ? 1 : 0;
}

int ssb_get_device_info(int32_t device, ssb_device_info* out) {
  return guard([&] {
    need(out, "out");
    need_device();
    const ssb::DeviceInfo d = ssb::device_info(device);
    std::memset(out, 0, sizeof *out);
    std::strncpy(out->name, d.name.c_str(), sizeof out->name - 1);
    out->major = d.major; out->minor = d.minor; out->multiprocessors = d.multiprocessors;
    out->global_memory = d.globalMemory; out->shared_per_block_optin = d.sharedPerBlockOptIn;
    out->runtime_version = d.runtimeVersion; out->driver_version = d.driverVersion;
  });
}

void ssb_batch_options_init(ssb_batch_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->count = 1;
  o->numerics = 1;
  o->traced_instances = 1;
  o->dense_steps = 400;
  o->sample_every = 60;
  o->curve_every = 0;
  o->t_max = 5 * 3600;
  o->tail_team_warps = -1;
  o->yield_below = -1;
}

int ssb_batch_create(const char* ship_path, const char* sim_path, const ssb_batch_options* opt, ssb_batch** out) {
  return guard([&] {
    need(ship_path, "ship_path"); need(sim_path, "sim_path"); need(opt, "opt"); need(out, "out");
    *out = nullptr;
    const ssb::BatchOptions bo = to_options(*opt);
    auto ship = ssb::load_ship(ship_path);
    const ssb::CompiledSim sim = ssb::load_sim(sim_path);
    ssb::check_pairing(*ship, sim);
    need_device();
    auto h = std::make_unique<ssb_batch>();
    h->batch = std::make_shared<ssb::Batch>(ship, sim, bo);
    *out = h.release();
  });
}

int ssb_fleet_create(int32_t n_models, const char* const* ship_paths, const char* const* sim_paths, const int32_t* instance_model,
                     const ssb_batch_options* opt, ssb_batch** out) {
  return guard([&] {
    need(ship_paths, "ship_paths"); need(sim_paths, "sim_paths"); need(instance_model, "instance_model"); need(opt, "opt"); need(out, "out");
    *out = nullptr;
    if (n_models < 1) throw std::invalid_argument("a fleet needs at least one model");
    if (opt->count < 1) throw std::invalid_argument("count must be at least 1");
    const ssb::BatchOptions bo = to_options(*opt);
    need_device();
    std::vector<std::pair<std::shared_ptr<const ssb::CompiledShip>, ssb::CompiledSim>> models;
    for (int32_t m = 0; m < n_models; ++m) {
      need(ship_paths[m], "ship path"); need(sim_paths[m], "sim path");
      auto ship = ssb::load_ship(ship_paths[m]);
      ssb::CompiledSim sim = ssb::load_sim(sim_paths[m]);
      ssb::check_pairing(*ship, sim);
      models.emplace_back(std::move(ship), std::move(sim));
    }
    std::vector<std::int32_t> im(instance_model, instance_model + opt->count);
    auto h = std::make_unique<ssb_batch>();
    h->batch = std::make_shared<ssb::Batch>(std::move(models), std::move(im), bo);
    *out = h.release();
  });
}

int ssb_batch_instance_shape(const ssb_batch* b, int32_t instance, int32_t* model, int32_t* nodes, int32_t* connections) {
  return guard([&] {
    need(b, "batch");
    const ssb::Batch::InstanceShape s = b->batch->instance_shape(instance);
    if (model) *model = s.model;
    if (nodes) *nodes = s.nodes;
    if (connections) *connections = s.connections;
  });
}

void ssb_batch_destroy(ssb_batch* b) { delete b; }

int ssb_batch_nodes(const ssb_batch* b, int32_t* nodes, int32_t* connections) {
  return guard([&] {
    need(b, "batch");
    if (nodes) *nodes = b->batch->nodes();
    if (connections) *connections = b->batch->connections();
  });
}

int ssb_batch_launch_info(const ssb_batch* b, ssb_launch_info* out) {
  return guard([&] {
    need(b, "batch"); need(out, "out");
    const ssb::LaunchConfig& c = b->batch->launch_config();
    const ssb::PhaseConfig m = c.main(), t = c.tail();
    out->team_warps = m.teamWarps; out->teams_per_block = m.teamsPerBlock; out->blocks = m.blocks;
    out->blocks_per_sm = m.blocksPerSM; out->yield_below = m.yieldBelow;
    out->tail_team_warps = t.teamWarps; out->tail_teams_per_block = t.teamsPerBlock; out->tail_blocks = t.blocks;
    out->tail_blocks_per_sm = t.blocksPerSM;
    out->slot_bytes = c.slotBytes;
    out->phases = static_cast<int32_t>(c.phases.size());
    out->kernels = ssb::kernels_per_run(b->batch->options(), c);
    out->staged_phases = 0;
    for (const ssb::PhaseConfig& p : c.phases) out->staged_phases += p.stageColumns ? 1 : 0;
  });
}

int ssb_launch_plan(const ssb_batch_options* opt, int32_t n_phases, const int32_t* yield_below, int32_t* kinds, int32_t* phases,
                    int32_t cap, int32_t* n) {
  return guard([&] {
    need(opt, "opt"); need(yield_below, "yield_below"); need(n, "n");
    if (n_phases < 1) throw std::invalid_argument("ssb_launch_plan: n_phases must be at least 1");
    ssb::LaunchConfig c;
    for (int32_t k = 0; k < n_phases; ++k) {
      ssb::PhaseConfig p;
      p.yieldBelow = yield_below[k];
      c.phases.push_back(p);
    }
    const std::vector<ssb::PlanStep> plan = ssb::run_plan(to_options(*opt), c);
    *n = static_cast<int32_t>(plan.size());
    if (static_cast<int32_t>(plan.size()) > cap) throw std::invalid_argument("ssb_launch_plan: cap is below the plan's length");
    for (std::size_t i = 0; i < plan.size(); ++i) {
      if (kinds) kinds[i] = static_cast<int32_t>(plan[i].kind);
      if (phases) phases[i] = plan[i].phase;
    }
  });
}

int ssb_batch_restore(ssb_batch* b, int32_t instance, const double* record) {
  return guard([&] { need(b, "batch"); need(record, "record"); b->batch->restore(instance, record); });
}

int ssb_batch_set_connection_enabled(ssb_batch* b, int32_t instance, int32_t c, int32_t enabled) {
  return guard([&] { need(b, "batch"); b->batch->set_connection_enabled(instance, c, enabled != 0); });
}

int ssb_batch_set_connection_area(ssb_batch* b, int32_t instance, int32_t c, double area) {
  return guard([&] { need(b, "batch"); b->batch->set_connection_area(instance, c, area); });
}

int ssb_batch_set_connection_areas(ssb_batch* b, int32_t first, int32_t count, int32_t n_connections, const int32_t* connections,
                                   const double* areas) {
  return guard([&] {
    need(b, "batch");
    b->batch->set_connection_areas(first, count, n_connections, connections, areas);
  });
}

int ssb_batch_set_claim_order(ssb_batch* b, const int32_t* order, int32_t n) {
  return guard([&] {
    need(b, "batch");
    b->batch->set_claim_order(order, n);
  });
}

int ssb_batch_set_connection_activation(ssb_batch* b, int32_t instance, int32_t c, double t_on) {
  return guard([&] { need(b, "batch"); b->batch->set_connection_activation(instance, c, t_on); });
}

int ssb_batch_apply_sweep(ssb_batch* b, const char* sweep_path) {
  return guard([&] {
    need(b, "batch"); need(sweep_path, "sweep_path");
    auto sw = std::make_unique<ssb::Sweep>(ssb::load_sweep(sweep_path, b->batch->sim()));
    if (static_cast<std::int32_t>(sw->instances.size()) != b->batch->options().count)
      throw std::invalid_argument("the sweep has " + std::to_string(sw->instances.size()) + " instances, the batch " +
                                  std::to_string(b->batch->options().count));
    b->batch->apply_sweep(*sw);
    b->sweep = std::move(sw);
  });
}

int ssb_batch_apply_sweep_range(ssb_batch* b, const char* sweep_path, int32_t first) {
  return guard([&] {
    need(b, "batch"); need(sweep_path, "sweep_path");
    auto sw = std::make_unique<ssb::Sweep>(ssb::load_sweep(sweep_path, b->batch->sim()));
    b->batch->apply_sweep(*sw, first);
    b->sweep = std::move(sw);
  });
}

int ssb_batch_run(ssb_batch* b, double* seconds) {
  return guard([&] {
    need(b, "batch");
    const double s = b->batch->run();
    if (seconds) *seconds = s;
  });
}

int ssb_batch_reset(ssb_batch* b) {
  return guard([&] { need(b, "batch"); b->batch->reset(); });
}

int ssb_batch_upload(ssb_batch* b) {
  return guard([&] { need(b, "batch"); b->batch->upload(); });
}

int ssb_batch_launch(ssb_batch* b, float* device_ms) {
  return guard([&] {
    need(b, "batch");
    const float ms = b->batch->launch();
    if (device_ms) *device_ms = ms;
  });
}

int ssb_batch_download(ssb_batch* b) {
  return guard([&] { need(b, "batch"); b->batch->download(); });
}

int ssb_batch_transfer_bytes(const ssb_batch* b, uint64_t* h2d, uint64_t* d2h) {
  return guard([&] {
    need(b, "batch");
    if (h2d) *h2d = b->batch->upload_bytes();
    if (d2h) *d2h = b->batch->download_bytes();
  });
}

int ssb_batch_phase_stats(const ssb_batch* b, int32_t phase, int32_t* team_warps, float* device_ms, int64_t* steps) {
  return guard([&] {
    need(b, "batch");
    const auto v = b->batch->phase_stats();
    if (v.empty()) throw std::logic_error("phase statistics before the first launch");
    if (phase < 0 || static_cast<std::size_t>(phase) >= v.size()) throw std::out_of_range("phase " + std::to_string(phase) + " out of range");
    if (team_warps) *team_warps = v[phase].teamWarps;
    if (device_ms) *device_ms = v[phase].deviceMs;
    if (steps) *steps = v[phase].steps;
  });
}

int ssb_batch_total_steps(const ssb_batch* b, int64_t* steps) {
  return guard([&] { need(b, "batch"); need(steps, "steps"); *steps = b->batch->total_steps(); });
}

int ssb_batch_summary(const ssb_batch* b, int32_t instance, ssb_instance_summary* out) {
  return guard([&] {
    need(b, "batch"); need(out, "out");
    const ssb::Batch::Summary s = b->batch->summary(instance);
    out->foundered = s.foundered ? 1 : 0;
    out->stop_reason = s.stop;
    out->founder_t = s.founderT;
    out->t_end = s.tEnd;
    out->steps = s.steps;
    out->event_count = static_cast<int32_t>(b->batch->events(instance).size());
    out->curve_count = b->batch->options().curveEvery > 0 ? static_cast<int32_t>(b->batch->curve(instance).size()) : 0;
    for (int k = 0; k < 7; ++k) out->outputs[k] = s.outputs[k];
  });
}

int ssb_batch_state(const ssb_batch* b, int32_t instance, double* record) {
  return guard([&] { need(b, "batch"); need(record, "record"); b->batch->state(instance, record); });
}

int ssb_batch_events(const ssb_batch* b, int32_t instance, double* t, int32_t* id, int32_t* kind, int32_t cap, int32_t* count) {
  return guard([&] {
    need(b, "batch");
    const auto ev = b->batch->events(instance);
    const auto kinds = b->batch->event_kinds(instance);
    const auto ids = b->batch->event_ids(instance);
    for (int32_t k = 0; k < static_cast<int32_t>(ev.size()) && k < cap; ++k) {
      const auto i = static_cast<std::size_t>(k);
      if (t) t[k] = ev[i].t;
      if (kind) kind[k] = kinds[i];
      if (id) id[k] = kinds[i] == 2 ? -1 : ids[i];
    }
    if (count) *count = static_cast<int32_t>(ev.size());
  });
}

int ssb_batch_curve(const ssb_batch* b, int32_t instance, double* records, int32_t cap, int32_t* count) {
  return guard([&] {
    need(b, "batch");
    const auto c = b->batch->curve(instance);
    for (int32_t k = 0; k < static_cast<int32_t>(c.size()) && k < cap; ++k) {
      const ssb::CurveRecord& r = c[static_cast<std::size_t>(k)];
      double* p = records + 7 * k;
      p[0] = r.t; p[1] = r.trim; p[2] = r.list; p[3] = r.water; p[4] = r.inflow; p[5] = r.dF; p[6] = r.dA;
    }
    if (count) *count = static_cast<int32_t>(c.size());
  });
}

int ssb_batch_final_readouts(const ssb_batch* b, int32_t instance, double* r7) {
  return guard([&] {
    need(b, "batch"); need(r7, "record7");
    const ssb::CurveRecord r = b->batch->final_readouts(instance);
    r7[0] = r.t; r7[1] = r.trim; r7[2] = r.list; r7[3] = r.water; r7[4] = r.inflow; r7[5] = r.dF; r7[6] = r.dA;
  });
}

int ssb_batch_save_trace(const ssb_batch* b, int32_t instance, const char* path) {
  return guard([&] { need(b, "batch"); need(path, "path"); ssb::save_trace(b->batch->trace(instance), path); });
}

int ssb_batch_save_results(const ssb_batch* b, const char* sweep_path, const char* results_path) {
  return guard([&] {
    need(b, "batch"); need(results_path, "results_path");
    std::unique_ptr<ssb::Sweep> own;
    const ssb::Sweep* sw = b->sweep.get();
    if (sweep_path) {
      own = std::make_unique<ssb::Sweep>(ssb::load_sweep(sweep_path, b->batch->sim()));
      sw = own.get();
    }
    if (sw && static_cast<std::size_t>(b->batch->sweep_first()) + static_cast<std::size_t>(b->batch->options().count) > sw->instances.size())
      throw std::invalid_argument("the sweep has fewer instances than the batch's range of it");
    ssb::Results r = b->batch->results(sw);
    if (sw) { r.tMax = sw->tMax; r.every = sw->every; }
    ssb::save_results(r, results_path);
  });
}

namespace {

// sinksim_cuda_run --sweep on instances [first, first + count) of the sweep (count < 0: to its end).
void run_sweep_range(const char* ship_path, const char* sim_path, const char* sweep_path, const char* numerics, std::int32_t first,
                     std::int32_t count, int device, const char* results_path, int64_t* steps, double* seconds) {
  need(ship_path, "ship_path"); need(sim_path, "sim_path"); need(sweep_path, "sweep_path"); need(numerics, "numerics");
  const std::string nm = numerics;
  if (nm != "portable" && nm != "portable32")
    throw Unsupported("numerics " + nm + " is not available on the GPU engine (use portable or portable32)");
  need_device();
  auto ship = ssb::load_ship(ship_path);
  const ssb::CompiledSim sim = ssb::load_sim(sim_path);
  ssb::check_pairing(*ship, sim);
  const ssb::Sweep sw = ssb::load_sweep(sweep_path, sim);
  const auto total = static_cast<std::int32_t>(sw.instances.size());
  if (count < 0) count = total - first;
  if (first < 0 || count < 1 || first + count > total)
    throw std::invalid_argument("sweep instances " + std::to_string(first) + " .. " + std::to_string(first + count - 1) + " do not exist (the sweep has " +
                                std::to_string(total) + ")");
  ssb::BatchOptions opt;
  opt.stopWhenStable = sw.stopWhenStable;
  opt.count = count;
  opt.mixedPrecision = nm == "portable32";
  opt.tracedInstances = 0;
  opt.tMax = sw.tMax;
  opt.curveEvery = sw.every;
  opt.device = device;
  ssb::Batch batch(ship, sim, opt);
  batch.apply_sweep(sw, first);
  const double s = batch.run();
  if (steps) *steps = batch.total_steps();
  if (seconds) *seconds = s;
  if (results_path) {
    ssb::Results r = batch.results(&sw);
    r.tMax = sw.tMax;
    r.every = sw.every;
    ssb::save_results(r, results_path);
  }
}

}  // namespace

int ssb_run_sweep(const char* ship_path, const char* sim_path, const char* sweep_path, const char* numerics, const char* results_path,
                  int64_t* steps, double* seconds) {
  return guard([&] { run_sweep_range(ship_path, sim_path, sweep_path, numerics, 0, -1, 0, results_path, steps, seconds); });
}

int ssb_run_sweep_range(const char* ship_path, const char* sim_path, const char* sweep_path, const char* numerics, int32_t first,
                        int32_t count, int32_t device, const char* results_path, int64_t* steps, double* seconds) {
  return guard([&] { run_sweep_range(ship_path, sim_path, sweep_path, numerics, first, count, device, results_path, steps, seconds); });
}

int ssb_compare_results(const char* a_path, const char* b_path, uint64_t* compared, uint64_t* differing, char* first, size_t first_cap) {
  return guard([&] {
    need(a_path, "a_path"); need(b_path, "b_path");
    const ssb::Diff d = ssb::compare_results(ssb::load_results(a_path), ssb::load_results(b_path));
    if (compared) *compared = d.compared;
    if (differing) *differing = d.differing;
    if (first && first_cap) {
      std::strncpy(first, d.first.c_str(), first_cap - 1);
      first[first_cap - 1] = 0;
    }
  });
}

int ssb_portable_math_host(int32_t op, const double* x, const double* y, double* out, int64_t n) {
  return guard([&] {
    need(x, "x"); need(out, "out");
    if (op < 0 || op > 3) throw std::invalid_argument("op must be 0..3");
    ssb::portable_math_host(op, x, y, out, n);
  });
}

int ssb_portable_math_device(int32_t op, const double* x, const double* y, double* out, int64_t n) {
  return guard([&] {
    need(x, "x"); need(out, "out");
    if (op < 0 || op > 3) throw std::invalid_argument("op must be 0..3");
    need_device();
    const cudaError_t e = ssb::portable_math_device(op, x, y, out, n);
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e));
  });
}

int ssb_batch_run_noalloc(const ssb_batch* b, int32_t count, const uint8_t* en, const double* area, const double* t_on, double* state,
                          double* vol, double* level, double* cx, double* cy, double* cz, double* final_readouts, int64_t* steps,
                          int32_t* stop_reason, void* stream) {
  return guard([&] {
    need(b, "batch");
    ssb::NoAllocRun r{};
    r.count = count;
    r.en = en; r.area = area; r.tOn = t_on;
    r.state = state; r.vol = vol; r.level = level; r.cx = cx; r.cy = cy; r.cz = cz;
    r.finalRec = final_readouts;
    r.steps = reinterpret_cast<long long*>(steps);
    r.stop = stop_reason;
    b->batch->run_noalloc(r, static_cast<cudaStream_t>(stream));
  });
}

int ssb_measure_add_mul_peak(int32_t fp64, int32_t device, double* ops_per_s) {
  return guard([&] {
    need(ops_per_s, "ops_per_s");
    need_device();
    const double v = ssb::measure_add_mul_peak(fp64 != 0, device);
    if (v < 0) throw std::runtime_error("the peak probe failed");
    *ops_per_s = v;
  });
}

uint64_t ssb_fnv1a64(uint64_t state, const void* data, size_t n) {
  const auto* p = static_cast<const unsigned char*>(data);
  for (size_t i = 0; i < n; ++i) {
    state ^= p[i];
    state *= 1099511628211ULL;
  }
  return state;
}

}  // extern "C"

int ssb_adjoint_create(const char* ship_path, const char* sim_path, int32_t count, double t_max, int32_t checkpoint_every, int32_t team_warps,
                       int32_t device, ssb_adjoint** out) {
  return guard([&] {
    need(ship_path, "ship_path"); need(sim_path, "sim_path"); need(out, "out");
    *out = nullptr;
    ssb::AdjointOptions o;
    o.count = count;
    o.tMax = t_max;
    o.checkpointEvery = checkpoint_every ? checkpoint_every : 256;
    o.teamWarps = team_warps;
    o.device = device;
    if (count < 1) throw std::invalid_argument("count must be at least 1");
    need_device();
    auto ship = ssb::load_ship(ship_path);
    const ssb::CompiledSim sim = ssb::load_sim(sim_path);
    ssb::check_pairing(*ship, sim);
    auto h = std::make_unique<ssb_adjoint>();
    h->adj = std::make_unique<ssb::AdjointBatch>(ship, sim, o);
    *out = h.release();
  });
}

void ssb_adjoint_destroy(ssb_adjoint* a) { delete a; }

int ssb_adjoint_set_connection_enabled(ssb_adjoint* a, int32_t instance, int32_t connection, int32_t enabled) {
  return guard([&] { need(a, "adjoint"); a->adj->set_connection_enabled(instance, connection, enabled != 0); });
}

int ssb_adjoint_set_connection_areas(ssb_adjoint* a, int32_t first, int32_t count, int32_t n_connections, const int32_t* connections,
                                     const double* areas) {
  return guard([&] {
    need(a, "adjoint");
    if (count > 0 && n_connections > 0) { need(connections, "connections"); need(areas, "areas"); }
    a->adj->set_connection_areas(first, count, n_connections, connections, areas);
  });
}

int ssb_adjoint_set_objective(ssb_adjoint* a, int32_t n, const double* times, const double* trim, const double* heave) {
  return guard([&] {
    need(a, "adjoint"); need(times, "times"); need(trim, "trim"); need(heave, "heave");
    a->adj->set_objective(n, times, trim, heave);
    a->nsamples = n;
  });
}

int ssb_adjoint_set_claim_order(ssb_adjoint* a, const int32_t* order, int32_t n) {
  return guard([&] {
    need(a, "adjoint");
    a->adj->set_claim_order(order, n);
  });
}

int ssb_adjoint_set_tape_budget(ssb_adjoint* a, uint64_t bytes) {
  return guard([&] {
    need(a, "adjoint");
    a->adj->set_tape_budget(bytes);
  });
}

int ssb_adjoint_ring_bytes(const ssb_adjoint* a, uint64_t* bytes) {
  return guard([&] {
    need(a, "adjoint"); need(bytes, "bytes");
    *bytes = a->adj->ring_bytes();
  });
}

int ssb_adjoint_run(ssb_adjoint* a, double* J, double* grad, int64_t* steps, int32_t* error, float* device_ms) {
  return guard([&] {
    need(a, "adjoint");
    const float ms = a->adj->run();
    if (device_ms) *device_ms = ms;
    const int32_t n = a->adj->count(), nc = a->adj->connections();
    for (int32_t i = 0; i < n; ++i) {
      if (J) J[i] = a->adj->objective(i);
      if (grad) std::memcpy(grad + static_cast<std::size_t>(i) * nc, a->adj->gradient(i), sizeof(double) * nc);
      if (steps) steps[i] = a->adj->steps(i);
      if (error) error[i] = a->adj->error(i);
    }
  });
}

int ssb_adjoint_samples(const ssb_adjoint* a, double* trim, double* heave) {
  return guard([&] {
    need(a, "adjoint");
    const int32_t n = a->adj->count(), k = a->nsamples;
    for (int32_t i = 0; i < n; ++i) {
      if (trim) std::memcpy(trim + static_cast<std::size_t>(i) * k, a->adj->samples_trim(i), sizeof(double) * k);
      if (heave) std::memcpy(heave + static_cast<std::size_t>(i) * k, a->adj->samples_heave(i), sizeof(double) * k);
    }
  });
}

int ssb_adjoint_info(const ssb_adjoint* a, int32_t* connections, int32_t* team_warps, int32_t* teams, uint64_t* h2d_bytes, uint64_t* d2h_bytes) {
  return guard([&] {
    need(a, "adjoint");
    if (connections) *connections = a->adj->connections();
    if (team_warps) *team_warps = a->adj->team_warps();
    if (teams) *teams = a->adj->teams();
    if (h2d_bytes) *h2d_bytes = a->adj->upload_bytes();
    if (d2h_bytes) *d2h_bytes = a->adj->download_bytes();
  });
}

int ssb_adjoint_phase_times(const ssb_adjoint* a, int64_t* ns) {
  return guard([&] {
    need(a, "adjoint"); need(ns, "ns");
    const int32_t n = a->adj->count();
    for (int32_t i = 0; i < n; ++i) std::memcpy(ns + 3 * static_cast<std::size_t>(i), a->adj->phase_ns(i), 3 * sizeof(int64_t));
  });
}

int ssb_adjoint_recomputed_steps(const ssb_adjoint* a, int64_t* steps) {
  return guard([&] {
    need(a, "adjoint"); need(steps, "steps");
    for (int32_t i = 0; i < a->adj->count(); ++i) steps[i] = a->adj->recomputed_steps(i);
  });
}

int ssb_check_model(const char* ship_path, const char* sim_path) {
  return guard([&] {
    need(ship_path, "ship_path"); need(sim_path, "sim_path");
    const auto ship = ssb::load_ship(ship_path);
    const ssb::CompiledSim sim = ssb::load_sim(sim_path);
    ssb::check_pairing(*ship, sim);
  });
}

int ssb_check_sweep(const char* ship_path, const char* sim_path, const char* sweep_path) {
  return guard([&] {
    need(ship_path, "ship_path"); need(sim_path, "sim_path"); need(sweep_path, "sweep_path");
    const auto ship = ssb::load_ship(ship_path);
    const ssb::CompiledSim sim = ssb::load_sim(sim_path);
    ssb::check_pairing(*ship, sim);
    ssb::load_sweep(sweep_path, sim);
  });
}

int ssb_batch_health(const ssb_batch* b, int32_t* flags) {
  return guard([&] {
    need(b, "batch"); need(flags, "flags");
    *flags = b->batch->health();
  });
}
