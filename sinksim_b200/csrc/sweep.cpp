// Sweep files, their application to instances, batch-results files and traces: the formats "sinksim.sweep",
// "sinksim.batch-results" and "sinksim.trace" of the reference (engine/include/sinksim/sweep.hpp:20-108,
// engine/src/sweep.cpp, engine/src/trace.cpp:272-308). The member names, their order and the numbers' text are the
// formats'; the code is organised around tables: the columns of a readout curve, the final readouts and the trace
// columns are each declared once and drive the writer, the reader and the exact comparison alike.
#include "sweep.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "json.h"

namespace ssb {

using json::Value;

namespace {

// ----------------------------------------------------------------------------- the tables

// The seven columns of a readout curve, in the file's order.
struct CurveColumn {
  const char* name;
  double CurveRecord::*field;
};
constexpr CurveColumn kCurve[] = {{"t", &CurveRecord::t},         {"trim", &CurveRecord::trim},     {"list", &CurveRecord::list},
                                  {"water", &CurveRecord::water}, {"inflow", &CurveRecord::inflow}, {"draftF", &CurveRecord::dF},
                                  {"draftA", &CurveRecord::dA}};

// The final readouts of an instance, in the file's order, with the short name the comparison reports.
struct FinalField {
  const char* name;
  const char* shortName;
  double InstanceResult::*field;
};
constexpr FinalField kFinal[] = {{"trimDeg", "trim", &InstanceResult::fTrim},    {"listDeg", "list", &InstanceResult::fList},
                                 {"waterT", "water", &InstanceResult::fWater},   {"draftF", "draftF", &InstanceResult::fDraftF},
                                 {"draftA", "draftA", &InstanceResult::fDraftA}, {"inflowTpm", "inflow", &InstanceResult::fInflow}};
// the comparison checks every final field but the inflow (the reference's sweep::compare does the same)
constexpr int kComparedFinal = 5;

// The columns of a trace block, in the file's (and the hash chain's) order.
struct TraceField {
  const char* name;
  std::vector<double> TraceColumns::*field;
};
constexpr TraceField kTrace[] = {{"t", &TraceColumns::t},         {"zO", &TraceColumns::zO},       {"pitch", &TraceColumns::pitch},
                                 {"roll", &TraceColumns::roll},   {"vz", &TraceColumns::vz},       {"wth", &TraceColumns::wth},
                                 {"wph", &TraceColumns::wph},     {"inflow", &TraceColumns::inflow}, {"Vb", &TraceColumns::Vb},
                                 {"hullTop", &TraceColumns::hullTop}, {"vol", &TraceColumns::vol},   {"level", &TraceColumns::level},
                                 {"cx", &TraceColumns::cx},       {"cy", &TraceColumns::cy},       {"cz", &TraceColumns::cz}};

Value header(const char* format) {
  Value doc = Value::object();
  doc.set("format", Value::string(format));
  doc.set("formatVersion", Value::integer(1));
  return doc;
}

// A sweep must state its formatVersion; a results file may omit it.
void expect_format(const Value& doc, const std::string& path, const char* format, bool versionRequired) {
  if (json::string_or(doc, "format", "") != format) throw std::runtime_error(path + ": not a " + format + " file");
  if ((versionRequired || doc.contains("formatVersion")) && json::integer(doc, "formatVersion", path) != 1)
    throw std::runtime_error(path + ": " + format + " formatVersion " + std::to_string(json::integer(doc, "formatVersion", path)) +
                             " cannot be read (version 1 can)");
}

// ----------------------------------------------------------------------------- sweeps

std::uint8_t kind_of(const CompiledSim& sim, const std::string& name, const std::string& where) {
  const std::int32_t k = sim.kindIndex(name);
  if (k < 0) throw std::runtime_error(where + ": the sim has no connection kind \"" + name + "\"");
  return static_cast<std::uint8_t>(k);
}

std::string kind_label(const CompiledSim& sim, std::uint8_t kind) {
  return kind < sim.kindNames.size() ? sim.kindNames[kind] : std::to_string(kind);
}

// One entry of an instance's "connections" list: a selector (one connection, or a kind with an optional index
// within the kind) and the fields it sets.
ConnectionOverride read_override(const Value& o, const CompiledSim& sim, const std::string& where) {
  if (!o.is_object()) throw std::runtime_error(where + ": a connection override must be an object");
  ConnectionOverride ov;
  if (o.contains("conn")) {
    ov.conn = static_cast<std::int32_t>(json::integer(o, "conn", where));  // a connection that does not exist matches nothing
  } else {
    ov.kind = kind_of(sim, json::string(o, "kind", where), where);
    if (o.contains("idx")) ov.idx = static_cast<std::int32_t>(json::integer(o, "idx", where));
  }
  if ((ov.hasEnabled = o.contains("enabled"))) ov.enabled = json::boolean(o, "enabled", where);
  if ((ov.hasTOn = o.contains("tOn"))) ov.tOn = json::number(o, "tOn", where);
  if ((ov.hasArea = o.contains("area"))) ov.area = json::number(o, "area", where);
  return ov;
}

SweepInstance read_instance(const Value& j, std::size_t index, const CompiledSim& sim, const std::string& path) {
  SweepInstance in;
  in.id = json::string_or(j, "id", "instance" + std::to_string(index));
  const std::string where = path + ", instance " + in.id;
  if (const Value* s = j.find("scale")) {
    if (!s->is_object()) throw std::runtime_error(where + ": scale must map connection kinds to factors");
    for (const auto& [kind, factor] : s->members()) {
      if (!factor.is_number()) throw std::runtime_error(where + ": the scale of " + kind + " is not a number");
      in.kindScale.emplace_back(kind_of(sim, kind, where), factor.as_double());
    }
  }
  if (const Value* list = j.find("connections")) {
    if (!list->is_array()) throw std::runtime_error(where + ": connections must be a list of overrides");
    for (const Value& o : list->items()) in.overrides.push_back(read_override(o, sim, where));
  }
  return in;
}

}  // namespace

Sweep load_sweep(const std::string& path, const CompiledSim& sim) {
  const Value doc = json::read_file(path);
  expect_format(doc, path, "sinksim.sweep", true);
  Sweep sw;
  sw.ship = json::string_or(doc, "ship", "");
  sw.sim = json::string_or(doc, "sim", "");
  sw.tMax = json::number_or(doc, "tMax", sw.tMax);
  sw.every = json::number_or(doc, "every", sw.every);
  const Value* stable = doc.find("stopWhenStable");
  sw.stopWhenStable = stable && stable->is_bool() && stable->as_bool();
  const Value& list = json::member(doc, "instances", path);
  if (!list.is_array()) throw std::runtime_error(path + ": instances must be a list");
  for (std::size_t i = 0; i < list.items().size(); ++i) sw.instances.push_back(read_instance(list.items()[i], i, sim, path));
  return sw;
}

void save_sweep(const Sweep& sw, const std::string& path, const CompiledSim& sim) {
  Value doc = header("sinksim.sweep");
  doc.set("ship", Value::string(sw.ship));
  doc.set("sim", Value::string(sw.sim));
  doc.set("tMax", Value::number(sw.tMax));
  doc.set("every", Value::number(sw.every));
  doc.set("stopWhenStable", Value::boolean(sw.stopWhenStable));
  Value list = Value::array();
  for (const SweepInstance& in : sw.instances) {
    Value j = Value::object();
    j.set("id", Value::string(in.id));
    if (!in.kindScale.empty()) {
      Value s = Value::object();
      for (const auto& [kind, factor] : in.kindScale) s.set(kind_label(sim, kind), Value::number(factor));
      j.set("scale", std::move(s));
    }
    if (!in.overrides.empty()) {
      Value ovs = Value::array();
      for (const ConnectionOverride& o : in.overrides) {
        Value x = Value::object();
        if (o.conn >= 0) {
          x.set("conn", Value::integer(o.conn));
        } else {
          x.set("kind", Value::string(kind_label(sim, o.kind)));
          if (o.idx >= 0) x.set("idx", Value::integer(o.idx));
        }
        if (o.hasEnabled) x.set("enabled", Value::boolean(o.enabled));
        if (o.hasTOn) x.set("tOn", Value::number(o.tOn));
        if (o.hasArea) x.set("area", Value::number(o.area));
        ovs.push(std::move(x));
      }
      j.set("connections", std::move(ovs));
    }
    list.push(std::move(j));
  }
  doc.set("instances", std::move(list));
  json::write_file(path, doc, 2);
}

void apply_instance(const SweepInstance& in, const CompiledSim& base, std::uint8_t* en, double* area, double* tOn) {
  // The connections a selector names: one connection, every connection of a kind, or the one(s) of a kind with the
  // given index within the kind.
  const std::int32_t nc = base.connections();
  auto selected = [&](const ConnectionOverride& o, std::int32_t c) {
    if (o.conn >= 0) return c == o.conn;
    const auto i = static_cast<std::size_t>(c);
    return base.cKind[i] == o.kind && (o.idx < 0 || base.cIdx[i] == o.idx);
  };
  // kind scales first, each the single product compiled area x factor (sweep.hpp:49-57 of the reference), so that
  // a scale set here and the same product computed anywhere else give the same bits
  for (const auto& [kind, factor] : in.kindScale)
    for (std::int32_t c = 0; c < nc; ++c)
      if (base.cKind[static_cast<std::size_t>(c)] == kind) area[c] = base.cArea[static_cast<std::size_t>(c)] * factor;
  // then the overrides, in the order written (sweep.hpp:58-65), a later one winning over an earlier one
  for (const ConnectionOverride& o : in.overrides)
    for (std::int32_t c = 0; c < nc; ++c) {
      if (!selected(o, c)) continue;
      if (o.hasEnabled) en[c] = o.enabled ? 1 : 0;
      if (o.hasArea) area[c] = o.area;
      if (o.hasTOn) tOn[c] = o.tOn;
    }
}

// ----------------------------------------------------------------------------- batch results

void save_results(const Results& r, const std::string& path) {
  Value doc = header("sinksim.batch-results");
  doc.set("ship", Value::string(r.ship));
  doc.set("sim", Value::string(r.sim));
  doc.set("numerics", Value::string(r.numerics));
  doc.set("engine", Value::string(r.engine));
  doc.set("tMax", Value::number(r.tMax));
  doc.set("every", Value::number(r.every));
  Value list = Value::array();
  for (const InstanceResult& in : r.instances) {
    Value j = Value::object();
    j.set("id", Value::string(in.id));
    j.set("foundered", Value::boolean(in.foundered));
    j.set("founderT", Value::number(in.founderT));
    j.set("tEnd", Value::number(in.tEnd));
    j.set("steps", Value::integer(in.steps));
    Value fin = Value::object();
    for (const FinalField& f : kFinal) fin.set(f.name, Value::number(in.*f.field));
    j.set("final", std::move(fin));
    Value events = Value::array();
    for (const EventRecord& e : in.events) {
      Value x = Value::object();
      x.set("t", Value::number(e.t));
      x.set("id", Value::string(e.id));
      x.set("label", Value::string(e.label));
      events.push(std::move(x));
    }
    j.set("events", std::move(events));
    Value curve = Value::object();
    for (const CurveColumn& col : kCurve) {
      std::vector<double> v(in.curve.size());
      std::transform(in.curve.begin(), in.curve.end(), v.begin(), [&](const CurveRecord& k) { return k.*col.field; });
      curve.set(col.name, Value::numbers(v));
    }
    j.set("curve", std::move(curve));
    list.push(std::move(j));
  }
  doc.set("instances", std::move(list));
  json::write_file(path, doc, 2);
}

Results load_results(const std::string& path) {
  const Value doc = json::read_file(path);
  expect_format(doc, path, "sinksim.batch-results", false);
  Results r;
  r.ship = json::string_or(doc, "ship", "");
  r.sim = json::string_or(doc, "sim", "");
  r.numerics = json::string_or(doc, "numerics", "");
  r.engine = json::string_or(doc, "engine", "");
  r.tMax = json::number_or(doc, "tMax", 0);
  r.every = json::number_or(doc, "every", 0);
  for (const Value& j : json::member(doc, "instances", path).items()) {
    InstanceResult in;
    in.id = json::string_or(j, "id", "");
    const std::string where = path + ", instance " + in.id;
    in.foundered = json::boolean(j, "foundered", where);
    in.founderT = json::number(j, "founderT", where);
    in.tEnd = json::number(j, "tEnd", where);
    in.steps = json::integer(j, "steps", where);
    const Value& fin = json::member(j, "final", where);
    for (const FinalField& f : kFinal) in.*f.field = json::number(fin, f.name, where);
    for (const Value& e : json::member(j, "events", where).items())
      in.events.push_back(EventRecord{json::number(e, "t", where), json::string(e, "id", where), json::string_or(e, "label", "")});
    const Value& curve = json::member(j, "curve", where);
    const std::size_t n = json::member(curve, "t", where).size();
    in.curve.assign(n, CurveRecord{});
    for (const CurveColumn& col : kCurve) {
      const Value& v = json::member(curve, col.name, where);
      if (v.size() != n) throw std::runtime_error(where + ": curve column " + col.name + " has " + std::to_string(v.size()) + " values, t has " + std::to_string(n));
      for (std::size_t k = 0; k < n; ++k) in.curve[k].*col.field = v.items()[k].as_double();
    }
    r.instances.push_back(std::move(in));
  }
  return r;
}

Diff compare_results(const Results& a, const Results& b) {
  // Value for value, bit for bit: two NaNs agree, everything else must be equal. The first difference is reported by
  // its place ("instance <id> curve[k] trim").
  Diff d;
  auto same = [&](const std::string& where, double x, double y) {
    ++d.compared;
    if (x == y || (std::isnan(x) && std::isnan(y))) return;
    ++d.differing;
    d.maxAbs = std::max(d.maxAbs, std::fabs(x - y));
    if (d.first.empty()) d.first = where + ": " + json::format_number(x) + " vs " + json::format_number(y);
  };
  if (a.instances.size() != b.instances.size()) {
    d.differing = 1;
    d.first = "instance count " + std::to_string(a.instances.size()) + " vs " + std::to_string(b.instances.size());
    return d;
  }
  for (std::size_t i = 0; i < a.instances.size(); ++i) {
    const InstanceResult &x = a.instances[i], &y = b.instances[i];
    const std::string w = "instance " + x.id;
    same(w + " foundered", x.foundered, y.foundered);
    same(w + " founderT", x.founderT, y.founderT);
    same(w + " tEnd", x.tEnd, y.tEnd);
    same(w + " steps", static_cast<double>(x.steps), static_cast<double>(y.steps));
    for (int f = 0; f < kComparedFinal; ++f) same(w + " " + kFinal[f].shortName, x.*kFinal[f].field, y.*kFinal[f].field);
    same(w + " events", static_cast<double>(x.events.size()), static_cast<double>(y.events.size()));
    for (std::size_t k = 0; k < std::min(x.events.size(), y.events.size()); ++k) {
      same(w + " event " + x.events[k].id + " t", x.events[k].t, y.events[k].t);
      if (x.events[k].id == y.events[k].id) continue;
      ++d.differing;
      if (d.first.empty()) d.first = w + " event id " + x.events[k].id + " vs " + y.events[k].id;
    }
    same(w + " curve length", static_cast<double>(x.curve.size()), static_cast<double>(y.curve.size()));
    for (std::size_t k = 0; k < std::min(x.curve.size(), y.curve.size()); ++k)
      for (const CurveColumn& col : kCurve)
        same(w + " curve[" + std::to_string(k) + "] " + col.name, x.curve[k].*col.field, y.curve[k].*col.field);
  }
  return d;
}

// ----------------------------------------------------------------------------- traces

void TraceColumns::push_record(const double* rec, std::int32_t nodes) {
  // the record layout of the device: ten scalars, then vol, level, cx, cy, cz per node
  ++n;
  for (int f = 0; f < 10; ++f) (this->*kTrace[f].field).push_back(rec[f]);
  for (int f = 10; f < 15; ++f) {
    const double* p = rec + 10 + (f - 10) * nodes;
    (this->*kTrace[f].field).insert((this->*kTrace[f].field).end(), p, p + nodes);
  }
}

void save_trace(const Trace& tr, const std::string& path) {
  Value doc = header("sinksim.trace");
  doc.set("role", Value::string(tr.role));
  doc.set("ship", Value::string(tr.ship));
  doc.set("sim", Value::string(tr.sim));
  Value meta = Value::object();
  meta.set("title", Value::string(tr.title));
  meta.set("producer", Value::string(tr.producer));
  meta.set("engine", Value::string(tr.engine));
  doc.set("meta", std::move(meta));
  doc.set("dt", Value::number(tr.dt));
  doc.set("nodes", Value::integer(tr.nodes));
  doc.set("denseSteps", Value::integer(tr.denseSteps));
  doc.set("sampleEvery", Value::number(tr.sampleEvery));
  doc.set("steps", Value::integer(tr.steps));
  doc.set("tEnd", Value::number(tr.tEnd));
  doc.set("foundered", Value::boolean(tr.foundered));
  doc.set("founderT", Value::number(tr.founderT));
  Value events = Value::array();
  for (const TraceEvent& e : tr.events) {
    Value x = Value::object();
    x.set("t", Value::number(e.t));
    x.set("id", Value::string(e.id));
    x.set("label", Value::string(e.label));
    events.push(std::move(x));
  }
  doc.set("events", std::move(events));
  // both blocks column by column, each column hashed alone and into the chain of all of them (dense, then samples)
  Value hash = Value::object();
  Fnv1a64 chain;
  const std::pair<const char*, const TraceColumns*> blocks[] = {{"dense", &tr.dense}, {"samples", &tr.samples}};
  for (const auto& [name, cols] : blocks) {
    Value block = Value::object();
    block.set("n", Value::integer(cols->n));
    for (const TraceField& f : kTrace) {
      const std::vector<double>& v = cols->*f.field;
      block.set(f.name, Value::numbers(v));
      Fnv1a64 own;
      own.f64(v.data(), v.size());
      chain.f64(v.data(), v.size());
      hash.set(std::string(name) + "." + f.name, Value::string(own.hex()));
    }
    doc.set(name, std::move(block));
  }
  hash.set("all", Value::string(chain.hex()));
  doc.set("hash", std::move(hash));
  json::write_file(path, doc, 2);
}

}  // namespace ssb
