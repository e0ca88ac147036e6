#include "sweep.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "json.h"

namespace ssb {

using json::Value;

namespace {

std::uint8_t kind_byte(const CompiledSim& sim, const std::string& name, const std::string& where) {
  const std::int32_t k = sim.kindIndex(name);
  if (k < 0) throw std::runtime_error(where + ": unknown connection kind \"" + name + "\"");
  return static_cast<std::uint8_t>(k);
}

std::string kind_name(const CompiledSim& sim, std::uint8_t kind) {
  const auto i = static_cast<std::size_t>(kind);
  return i < sim.kindNames.size() ? sim.kindNames[i] : std::to_string(kind);
}

}  // namespace

Sweep load_sweep(const std::string& path, const CompiledSim& sim) {
  const Value doc = json::read_file(path);
  if (json::string_or(doc, "format", "") != "sinksim.sweep") throw std::runtime_error(path + ": format is not sinksim.sweep");
  if (json::integer(doc, "formatVersion", path) != 1) throw std::runtime_error(path + ": unsupported sweep formatVersion");
  Sweep sw;
  sw.ship = json::string_or(doc, "ship", "");
  sw.sim = json::string_or(doc, "sim", "");
  sw.tMax = json::number_or(doc, "tMax", 5 * 3600);
  sw.every = json::number_or(doc, "every", 30);
  const Value* sws = doc.find("stopWhenStable");
  sw.stopWhenStable = sws && sws->is_bool() && sws->as_bool();
  const Value& list = json::member(doc, "instances", path);
  if (!list.is_array()) throw std::runtime_error(path + ": instances must be an array");
  std::size_t k = 0;
  for (const Value& j : list.items()) {
    SweepInstance in;
    in.id = json::string_or(j, "id", "instance" + std::to_string(k));
    const std::string where = path + " instance " + in.id;
    if (const Value* s = j.find("scale")) {
      if (!s->is_object()) throw std::runtime_error(where + ": scale must be an object of kind -> factor");
      for (const auto& kv : s->members()) {
        if (!kv.second.is_number()) throw std::runtime_error(where + ": scale factor for " + kv.first + " is not a number");
        in.kindScale.emplace_back(kind_byte(sim, kv.first, where), kv.second.as_double());
      }
    }
    if (const Value* l2 = j.find("connections")) {
      if (!l2->is_array()) throw std::runtime_error(where + ": connections must be an array");
      for (const Value& o : l2->items()) {
        ConnectionOverride ov;
        if (o.contains("conn")) {
          ov.conn = static_cast<std::int32_t>(json::integer(o, "conn", where));
        } else {
          ov.kind = kind_byte(sim, json::string(o, "kind", where), where);
          if (o.contains("idx")) ov.idx = static_cast<std::int32_t>(json::integer(o, "idx", where));
        }
        if (o.contains("enabled")) { ov.hasEnabled = true; ov.enabled = json::boolean(o, "enabled", where); }
        if (o.contains("tOn")) { ov.hasTOn = true; ov.tOn = json::number(o, "tOn", where); }
        if (o.contains("area")) { ov.hasArea = true; ov.area = json::number(o, "area", where); }
        in.overrides.push_back(ov);
      }
    }
    sw.instances.push_back(std::move(in));
    ++k;
  }
  return sw;
}

void save_sweep(const Sweep& sw, const std::string& path, const CompiledSim& sim) {
  Value doc = Value::object();
  doc.set("format", Value::string("sinksim.sweep"));
  doc.set("formatVersion", Value::integer(1));
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
      for (const auto& [kind, factor] : in.kindScale) s.set(kind_name(sim, kind), Value::number(factor));
      j.set("scale", s);
    }
    if (!in.overrides.empty()) {
      Value l2 = Value::array();
      for (const ConnectionOverride& o : in.overrides) {
        Value x = Value::object();
        if (o.conn >= 0) x.set("conn", Value::integer(o.conn));
        else {
          x.set("kind", Value::string(kind_name(sim, o.kind)));
          if (o.idx >= 0) x.set("idx", Value::integer(o.idx));
        }
        if (o.hasEnabled) x.set("enabled", Value::boolean(o.enabled));
        if (o.hasTOn) x.set("tOn", Value::number(o.tOn));
        if (o.hasArea) x.set("area", Value::number(o.area));
        l2.push(x);
      }
      j.set("connections", l2);
    }
    list.push(j);
  }
  doc.set("instances", list);
  json::write_file(path, doc, 2);
}

void apply_instance(const SweepInstance& in, const CompiledSim& base, std::uint8_t* en, double* area, double* tOn) {
  const std::int32_t nc = base.connections();
  for (const auto& [kind, factor] : in.kindScale)
    for (std::int32_t c = 0; c < nc; ++c)
      if (base.cKind[static_cast<std::size_t>(c)] == kind) area[c] = base.cArea[static_cast<std::size_t>(c)] * factor;
  for (const ConnectionOverride& o : in.overrides) {
    for (std::int32_t c = 0; c < nc; ++c) {
      const auto i = static_cast<std::size_t>(c);
      const bool match = o.conn >= 0 ? c == o.conn : (base.cKind[i] == o.kind && (o.idx < 0 || base.cIdx[i] == o.idx));
      if (!match) continue;
      if (o.hasEnabled) en[c] = o.enabled ? 1 : 0;
      if (o.hasArea) area[c] = o.area;
      if (o.hasTOn) tOn[c] = o.tOn;
    }
  }
}

void save_results(const Results& r, const std::string& path) {
  Value doc = Value::object();
  doc.set("format", Value::string("sinksim.batch-results"));
  doc.set("formatVersion", Value::integer(1));
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
    Value f = Value::object();
    f.set("trimDeg", Value::number(in.fTrim));
    f.set("listDeg", Value::number(in.fList));
    f.set("waterT", Value::number(in.fWater));
    f.set("draftF", Value::number(in.fDraftF));
    f.set("draftA", Value::number(in.fDraftA));
    f.set("inflowTpm", Value::number(in.fInflow));
    j.set("final", f);
    Value ev = Value::array();
    for (const EventRecord& e : in.events) {
      Value x = Value::object();
      x.set("t", Value::number(e.t));
      x.set("id", Value::string(e.id));
      x.set("label", Value::string(e.label));
      ev.push(x);
    }
    j.set("events", ev);
    std::vector<double> t, trim, lst, water, inflow, dF, dA;
    for (const CurveRecord& k : in.curve) {
      t.push_back(k.t); trim.push_back(k.trim); lst.push_back(k.list); water.push_back(k.water);
      inflow.push_back(k.inflow); dF.push_back(k.dF); dA.push_back(k.dA);
    }
    Value c = Value::object();
    c.set("t", Value::numbers(t));
    c.set("trim", Value::numbers(trim));
    c.set("list", Value::numbers(lst));
    c.set("water", Value::numbers(water));
    c.set("inflow", Value::numbers(inflow));
    c.set("draftF", Value::numbers(dF));
    c.set("draftA", Value::numbers(dA));
    j.set("curve", c);
    list.push(j);
  }
  doc.set("instances", list);
  json::write_file(path, doc, 2);
}

Results load_results(const std::string& path) {
  const Value doc = json::read_file(path);
  if (json::string_or(doc, "format", "") != "sinksim.batch-results") throw std::runtime_error(path + ": format is not sinksim.batch-results");
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
    in.foundered = json::boolean(j, "foundered", path);
    in.founderT = json::number(j, "founderT", path);
    in.tEnd = json::number(j, "tEnd", path);
    in.steps = json::integer(j, "steps", path);
    const Value& f = json::member(j, "final", path);
    in.fTrim = json::number(f, "trimDeg", path); in.fList = json::number(f, "listDeg", path); in.fWater = json::number(f, "waterT", path);
    in.fDraftF = json::number(f, "draftF", path); in.fDraftA = json::number(f, "draftA", path); in.fInflow = json::number(f, "inflowTpm", path);
    for (const Value& e : json::member(j, "events", path).items())
      in.events.push_back(EventRecord{json::number(e, "t", path), json::string(e, "id", path), json::string_or(e, "label", "")});
    const Value& c = json::member(j, "curve", path);
    auto col = [&](const char* k) {
      std::vector<double> v;
      for (const Value& x : json::member(c, k, path).items()) v.push_back(x.as_double());
      return v;
    };
    const auto t = col("t"), trim = col("trim"), lst = col("list"), water = col("water"), inflow = col("inflow"), dF = col("draftF"), dA = col("draftA");
    for (std::size_t i = 0; i < t.size(); ++i) in.curve.push_back(CurveRecord{t[i], trim[i], lst[i], water[i], inflow[i], dF[i], dA[i]});
    r.instances.push_back(std::move(in));
  }
  return r;
}

Diff compare_results(const Results& a, const Results& b) {
  Diff d;
  auto note = [&](const std::string& where, double x, double y) {
    ++d.compared;
    if (x != y && !(std::isnan(x) && std::isnan(y))) {
      ++d.differing;
      const double ad = std::fabs(x - y);
      if (ad > d.maxAbs) d.maxAbs = ad;
      if (d.first.empty()) d.first = where + ": " + json::format_number(x) + " vs " + json::format_number(y);
    }
  };
  if (a.instances.size() != b.instances.size()) {
    d.differing++;
    d.first = "instance count " + std::to_string(a.instances.size()) + " vs " + std::to_string(b.instances.size());
    return d;
  }
  for (std::size_t i = 0; i < a.instances.size(); ++i) {
    const InstanceResult& x = a.instances[i];
    const InstanceResult& y = b.instances[i];
    const std::string w = "instance " + x.id;
    note(w + " foundered", x.foundered, y.foundered);
    note(w + " founderT", x.founderT, y.founderT);
    note(w + " tEnd", x.tEnd, y.tEnd);
    note(w + " steps", static_cast<double>(x.steps), static_cast<double>(y.steps));
    note(w + " trim", x.fTrim, y.fTrim);
    note(w + " list", x.fList, y.fList);
    note(w + " water", x.fWater, y.fWater);
    note(w + " draftF", x.fDraftF, y.fDraftF);
    note(w + " draftA", x.fDraftA, y.fDraftA);
    note(w + " events", static_cast<double>(x.events.size()), static_cast<double>(y.events.size()));
    for (std::size_t k = 0; k < std::min(x.events.size(), y.events.size()); ++k) {
      note(w + " event " + x.events[k].id + " t", x.events[k].t, y.events[k].t);
      if (x.events[k].id != y.events[k].id) {
        ++d.differing;
        if (d.first.empty()) d.first = w + " event id " + x.events[k].id + " vs " + y.events[k].id;
      }
    }
    note(w + " curve length", static_cast<double>(x.curve.size()), static_cast<double>(y.curve.size()));
    for (std::size_t k = 0; k < std::min(x.curve.size(), y.curve.size()); ++k) {
      const std::string c = w + " curve[" + std::to_string(k) + "]";
      note(c + " t", x.curve[k].t, y.curve[k].t);
      note(c + " trim", x.curve[k].trim, y.curve[k].trim);
      note(c + " list", x.curve[k].list, y.curve[k].list);
      note(c + " water", x.curve[k].water, y.curve[k].water);
      note(c + " inflow", x.curve[k].inflow, y.curve[k].inflow);
      note(c + " draftF", x.curve[k].dF, y.curve[k].dF);
      note(c + " draftA", x.curve[k].dA, y.curve[k].dA);
    }
  }
  return d;
}

// ----------------------------------------------------------------------------- traces

void TraceColumns::push_record(const double* rec, std::int32_t nodes) {
  ++n;
  t.push_back(rec[0]); zO.push_back(rec[1]); pitch.push_back(rec[2]); roll.push_back(rec[3]);
  vz.push_back(rec[4]); wth.push_back(rec[5]); wph.push_back(rec[6]);
  inflow.push_back(rec[7]); Vb.push_back(rec[8]); hullTop.push_back(rec[9]);
  const double* p = rec + 10;
  vol.insert(vol.end(), p, p + nodes); p += nodes;
  level.insert(level.end(), p, p + nodes); p += nodes;
  cx.insert(cx.end(), p, p + nodes); p += nodes;
  cy.insert(cy.end(), p, p + nodes); p += nodes;
  cz.insert(cz.end(), p, p + nodes);
}

namespace {

const char* const kTraceFields[] = {"t", "zO", "pitch", "roll", "vz", "wth", "wph", "inflow", "Vb", "hullTop", "vol", "level", "cx", "cy", "cz"};

const std::vector<double>& trace_field(const TraceColumns& c, int i) {
  const std::vector<double>* f[] = {&c.t, &c.zO, &c.pitch, &c.roll, &c.vz, &c.wth, &c.wph, &c.inflow, &c.Vb, &c.hullTop,
                                    &c.vol, &c.level, &c.cx, &c.cy, &c.cz};
  return *f[i];
}

Value trace_columns(const TraceColumns& c, Fnv1a64& chain, Value& hash, const std::string& name) {
  Value v = Value::object();
  v.set("n", Value::integer(c.n));
  for (int i = 0; i < 15; ++i) {
    const std::vector<double>& src = trace_field(c, i);
    v.set(kTraceFields[i], Value::numbers(src));
    Fnv1a64 one;
    one.f64(src.data(), src.size());
    chain.f64(src.data(), src.size());
    hash.set(name + "." + kTraceFields[i], Value::string(one.hex()));
  }
  return v;
}

}  // namespace

void save_trace(const Trace& tr, const std::string& path) {
  Value doc = Value::object();
  doc.set("format", Value::string("sinksim.trace"));
  doc.set("formatVersion", Value::integer(1));
  doc.set("role", Value::string(tr.role));
  doc.set("ship", Value::string(tr.ship));
  doc.set("sim", Value::string(tr.sim));
  Value meta = Value::object();
  meta.set("title", Value::string(tr.title));
  meta.set("producer", Value::string(tr.producer));
  meta.set("engine", Value::string(tr.engine));
  doc.set("meta", meta);
  doc.set("dt", Value::number(tr.dt));
  doc.set("nodes", Value::integer(tr.nodes));
  doc.set("denseSteps", Value::integer(tr.denseSteps));
  doc.set("sampleEvery", Value::number(tr.sampleEvery));
  doc.set("steps", Value::integer(tr.steps));
  doc.set("tEnd", Value::number(tr.tEnd));
  doc.set("foundered", Value::boolean(tr.foundered));
  doc.set("founderT", Value::number(tr.founderT));
  Value ev = Value::array();
  for (const TraceEvent& e : tr.events) {
    Value x = Value::object();
    x.set("t", Value::number(e.t));
    x.set("id", Value::string(e.id));
    x.set("label", Value::string(e.label));
    ev.push(x);
  }
  doc.set("events", ev);
  Value hash = Value::object();
  Fnv1a64 chain;
  doc.set("dense", trace_columns(tr.dense, chain, hash, "dense"));
  doc.set("samples", trace_columns(tr.samples, chain, hash, "samples"));
  hash.set("all", Value::string(chain.hex()));
  doc.set("hash", hash);
  json::write_file(path, doc, 2);
}

}  // namespace ssb
