// A C ABI over the reference CPU engine (sinksim::Simulation), compiled by oracle/Makefile together with the
// reference's own engine sources into oracle/_ref/libsinksim_ref.so. Test infrastructure only: the parity tests
// and the CPU leg of bench.py load it through ctypes as the checker. The sinksim_b200 package never links it.
//
// Every entry point returns 0 on success and a negative value on failure; ssref_last_error() holds the message.
// The record layout of ssref_state/ssref_restore is the trace record of the reference
// (engine/src/trace.cpp:140-150): t, zO, pitch, roll, vz, wth, wph, inflow, Vb, hullTop, then vol, level, cx, cy,
// cz per node (10 + 5 N values).
#include <atomic>
#include <chrono>
#include <functional>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "sinksim/io/compiled.hpp"
#include "sinksim/simulation.hpp"
#include "sinksim/sweep.hpp"

using namespace sinksim;

namespace {

thread_local std::string g_error;

struct Handle {
  std::shared_ptr<const CompiledShip> ship;
  CompiledSim sim;
  std::unique_ptr<Simulation> S;
};

template <class F>
int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return -1;
  }
}

bool numerics_of(const char* name, Numerics& n) { return name && parse_numerics(name, n); }

// The extra retire predicate of the batching workloads, evaluated after every step through Simulation::run's
// onStep hook (engine/src/simulation.cpp:183). A run also ends at the reference's own founder rule and at tMax.
//   sink:   |pitch| > pitchLimit and the world height of the deck edge at (xDeck, +-yDeck, zDeck) below the sea
//   settle: |wth| < wthLimit held for settleTime seconds of simulated time
struct Retire {
  double pitchLimit, xDeck, yDeck, zDeck, wthLimit, settleTime;
};

}  // namespace

extern "C" {

const char* ssref_last_error() { return g_error.c_str(); }

void* ssref_open(const char* shipPath, const char* simPath, const char* numerics) {
  auto h = std::make_unique<Handle>();
  const int rc = guard([&] {
    Numerics n;
    if (!numerics_of(numerics, n)) throw std::invalid_argument(std::string("unknown numerics ") + (numerics ? numerics : "(null)"));
    h->ship = io::load_ship(shipPath);
    h->sim = io::load_sim(simPath);
    io::check_pairing(*h->ship, h->sim);
    h->S = std::make_unique<Simulation>(h->ship, h->sim, n);
  });
  return rc == 0 ? h.release() : nullptr;
}

void ssref_close(void* p) { delete static_cast<Handle*>(p); }

int ssref_nodes(void* p) { return static_cast<Handle*>(p)->S->nodes(); }
int ssref_connections(void* p) { return static_cast<Handle*>(p)->sim.connections(); }

int ssref_set_connection(void* p, int c, int enabled, double area, double tOn) {
  Handle& h = *static_cast<Handle*>(p);
  return guard([&] {
    if (c < 0 || c >= h.sim.connections()) throw std::out_of_range("connection");
    if (enabled >= 0) h.S->set_connection_enabled(c, enabled != 0);
    if (!std::isnan(area)) h.S->set_connection_area(c, area);
    if (!std::isnan(tOn)) h.S->set_connection_activation(c, tOn);
  });
}

// Apply one instance of a sweep file (by index) to the simulation: kind scales, then overrides in order.
int ssref_apply_sweep_instance(void* p, const char* sweepPath, int instance) {
  Handle& h = *static_cast<Handle*>(p);
  return guard([&] {
    const sweep::Sweep sw = sweep::load_sweep(sweepPath, h.sim);
    if (instance < 0 || static_cast<std::size_t>(instance) >= sw.instances.size()) throw std::out_of_range("sweep instance");
    sweep::apply(sw.instances[static_cast<std::size_t>(instance)], h.sim, *h.S);
  });
}

int ssref_step(void* p, long long n) {
  Handle& h = *static_cast<Handle*>(p);
  return guard([&] { for (long long i = 0; i < n; ++i) h.S->step(); });
}

int ssref_state(void* p, double* rec) {
  Handle& h = *static_cast<Handle*>(p);
  const State& st = h.S->state();
  const Outputs& o = h.S->outputs();
  const Scratch& sc = h.S->scratch();
  const Index N = h.S->nodes();
  rec[0] = st.t; rec[1] = st.zO; rec[2] = st.pitch; rec[3] = st.roll; rec[4] = st.vz; rec[5] = st.wth; rec[6] = st.wph;
  rec[7] = o.inflow; rec[8] = o.Vb; rec[9] = o.hullTop;
  for (Index n = 0; n < N; ++n) {
    rec[10 + n] = st.vol[n];
    rec[10 + N + n] = st.level[n];
    rec[10 + 2 * N + n] = sc.cx[n];
    rec[10 + 3 * N + n] = sc.cy[n];
    rec[10 + 4 * N + n] = sc.cz[n];
  }
  return 0;
}

int ssref_restore(void* p, const double* rec) {
  Handle& h = *static_cast<Handle*>(p);
  const Index N = h.S->nodes();
  const StateSnapshot s{rec[0], rec[1], rec[2], rec[3], rec[4], rec[5], rec[6], rec + 10, rec + 10 + N, rec + 10 + 2 * N, rec + 10 + 3 * N, rec + 10 + 4 * N};
  return guard([&] { h.S->restore(s); });
}

int ssref_evaluate_hydro(void* p) {
  Handle& h = *static_cast<Handle*>(p);
  return guard([&] { h.S->evaluate_hydro(); });
}

// Per-step flows and scratch of the last step: q per connection (nc values), then area, hEff, aEff, acc, excess per node.
int ssref_scratch(void* p, double* q, double* perNode) {
  Handle& h = *static_cast<Handle*>(p);
  const Index N = h.S->nodes();
  const Scratch& sc = h.S->scratch();
  const std::vector<Real>& f = h.S->flows();
  for (std::size_t c = 0; c < f.size(); ++c) q[c] = f[c];
  for (Index n = 0; n < N; ++n) {
    perNode[n] = sc.area[n]; perNode[N + n] = sc.hEff[n]; perNode[2 * N + n] = sc.aEff[n];
    perNode[3 * N + n] = sc.acc[n]; perNode[4 * N + n] = sc.excess[n];
  }
  return 0;
}

// Events so far: up to cap triples (t, id, kind). Returns the count, or a negative value on error.
int ssref_events(void* p, double* out, int cap) {
  Handle& h = *static_cast<Handle*>(p);
  const std::vector<Event> ev = h.S->events();
  const int n = static_cast<int>(ev.size());
  for (int i = 0; i < n && i < cap; ++i) {
    out[3 * i] = ev[static_cast<std::size_t>(i)].t;
    out[3 * i + 1] = ev[static_cast<std::size_t>(i)].id;
    out[3 * i + 2] = static_cast<double>(ev[static_cast<std::size_t>(i)].kind);
  }
  return n;
}

int ssref_foundered(void* p, double* founderT) {
  Handle& h = *static_cast<Handle*>(p);
  *founderT = h.S->founderT();
  return h.S->foundered() ? 1 : 0;
}

// Readouts at the current state (engine/include/sinksim/kernel/readouts.hpp): t, trim, list, water t, inflow t/min, dF, dA.
int ssref_readouts(void* p, double* r7) {
  Handle& h = *static_cast<Handle*>(p);
  const kernel::Readouts r = h.S->readouts();
  r7[0] = r.t; r7[1] = r.trimDeg; r7[2] = r.listDeg; r7[3] = r.waterT; r7[4] = r.inflowTpm; r7[5] = r.draftF; r7[6] = r.draftA;
  return 0;
}

// Simulation::run with the extra retire predicate (rule != nullptr) or without it. Writes steps, foundered flag,
// founderT, tEnd, and whether the extra predicate ended the run (0 none, 1 sink, 2 settle) into summary[5]; the
// readout curve (7 values per record, at most curveCap records) into curve; returns the record count.
int ssref_run(void* p, double tMax, double every, int stopWhenStable, const double* rule, double* summary, double* curve, int curveCap) {
  Handle& h = *static_cast<Handle*>(p);
  int records = -1;
  const int rc = guard([&] {
    RunOptions opt;
    opt.tMax = tMax;
    opt.every = every;
    opt.stopWhenStable = stopWhenStable != 0;
    int why = 0;
    double calm = 0;
    std::function<bool(Simulation&)> onStep;
    if (rule) {
      const Retire R{rule[0], rule[1], rule[2], rule[3], rule[4], rule[5]};
      onStep = [&, R](Simulation& S) {
        const State& st = S.state();
        const Frame F = kernel::pose_frame<PortableMath>(S.sim_view().body, st.zO, st.pitch, st.roll);
        const Real zp = kernel::world_z(F, R.xDeck, R.yDeck, R.zDeck), zs = kernel::world_z(F, R.xDeck, -R.yDeck, R.zDeck);
        if (ss_abs(st.pitch) > R.pitchLimit && (zp < 0 || zs < 0)) { why = 1; return false; }
        calm = ss_abs(st.wth) < R.wthLimit ? calm + S.sim_view().dt : 0;
        if (calm >= R.settleTime) { why = 2; return false; }
        return true;
      };
    }
    const RunResult r = h.S->run(opt, onStep);
    summary[0] = static_cast<double>(r.steps);
    summary[1] = r.foundered ? 1 : 0;
    summary[2] = r.founderT;
    summary[3] = r.tEnd;
    summary[4] = why;
    records = static_cast<int>(r.hist.size());
    for (int i = 0; i < records && i < curveCap; ++i) {
      const HistoryRecord& k = r.hist[static_cast<std::size_t>(i)];
      double* o = curve + 7 * i;
      o[0] = k.t; o[1] = k.trim; o[2] = k.list; o[3] = k.water; o[4] = k.inflow; o[5] = k.dF; o[6] = k.dA;
    }
  });
  return rc == 0 ? records : rc;
}

// Time the reference CPU engine over a bounded sample: `count` instances (instance i scales the breach kind by
// 1 + 0.02 i / count, the reference GPU runner's --perturb rule, apps/sinksim_cuda_run.cpp:126-135), each stepped
// maxSteps steps or to its founder, on `threads` std::threads pulling instances from an atomic counter (the
// scheduling of sweep::run_cpu, engine/src/sweep.cpp:121-160). Returns the total steps taken; seconds gets the
// wall time.
long long ssref_time_steps(const char* shipPath, const char* simPath, const char* numerics, int count, long long maxSteps, int threads, double* seconds) {
  long long total = -1;
  guard([&] {
    Numerics n;
    if (!numerics_of(numerics, n)) throw std::invalid_argument("unknown numerics");
    const auto ship = io::load_ship(shipPath);
    const CompiledSim sim = io::load_sim(simPath);
    io::check_pairing(*ship, sim);
    const Index breach = sim.kindIndex("breach");
    std::atomic<int> next{0};
    std::atomic<long long> steps{0};
    const auto t0 = std::chrono::steady_clock::now();
    auto worker = [&] {
      for (;;) {
        const int i = next.fetch_add(1);
        if (i >= count) return;
        Simulation S(ship, sim, n);
        const Real scale = 1 + 0.02 * static_cast<Real>(i) / static_cast<Real>(count);
        if (i > 0 && breach >= 0)
          for (Index c = 0; c < sim.connections(); ++c)
            if (sim.cKind[static_cast<std::size_t>(c)] == static_cast<Byte>(breach)) S.set_connection_area(c, sim.cArea[static_cast<std::size_t>(c)] * scale);
        long long s = 0;
        while (s < maxSteps && !S.foundered()) { S.step(); ++s; }
        steps += s;
      }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    total = steps.load();
  });
  return total;
}

// Times the reference CPU engine on whole runs of chosen sweep instances: instance instances[k] of the sweep file, each
// run by Simulation::run from the compiled initial state to its founder, tMax or the extra retire predicate (rule,
// may be null), as the GPU batch runs them; `threads` std::threads pull the instances from an atomic counter (the
// scheduling of sweep::run_cpu, engine/src/sweep.cpp:121-160). Returns the total steps; seconds gets the wall time of
// the runs (the models are loaded before the clock starts).
long long ssref_time_sweep_runs(const char* shipPath, const char* simPath, const char* sweepPath, const char* numerics, const int* instances, int n,
                                double tMax, const double* rule, int threads, double* seconds) {
  long long total = -1;
  guard([&] {
    Numerics num;
    if (!numerics_of(numerics, num)) throw std::invalid_argument("unknown numerics");
    const auto ship = io::load_ship(shipPath);
    const CompiledSim sim = io::load_sim(simPath);
    io::check_pairing(*ship, sim);
    const sweep::Sweep sw = sweep::load_sweep(sweepPath, sim);
    for (int k = 0; k < n; ++k)
      if (instances[k] < 0 || static_cast<std::size_t>(instances[k]) >= sw.instances.size()) throw std::out_of_range("sweep instance");
    std::atomic<int> next{0};
    std::atomic<long long> steps{0};
    const auto t0 = std::chrono::steady_clock::now();
    auto worker = [&] {
      for (;;) {
        const int k = next.fetch_add(1);
        if (k >= n) return;
        Simulation S(ship, sim, num);
        sweep::apply(sw.instances[static_cast<std::size_t>(instances[k])], sim, S);
        RunOptions opt;
        opt.tMax = tMax;
        opt.every = 1e9;  // no readout curve beyond the first record
        std::function<bool(Simulation&)> onStep;
        double calm = 0;
        if (rule) {
          const Retire R{rule[0], rule[1], rule[2], rule[3], rule[4], rule[5]};
          onStep = [&calm, R](Simulation& Sm) {
            const State& st = Sm.state();
            const Frame F = kernel::pose_frame<PortableMath>(Sm.sim_view().body, st.zO, st.pitch, st.roll);
            const Real zp = kernel::world_z(F, R.xDeck, R.yDeck, R.zDeck), zs = kernel::world_z(F, R.xDeck, -R.yDeck, R.zDeck);
            if (ss_abs(st.pitch) > R.pitchLimit && (zp < 0 || zs < 0)) return false;
            calm = ss_abs(st.wth) < R.wthLimit ? calm + Sm.sim_view().dt : 0;
            return calm < R.settleTime;
          };
        }
        steps += S.run(opt, onStep).steps;
      }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    total = steps.load();
  });
  return total;
}

}  // extern "C"
