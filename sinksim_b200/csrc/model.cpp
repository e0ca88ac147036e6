// Loading compiled ships and sims ("sinksim.compiled-ship" / "sinksim.compiled-sim", the reference's docs/FORMATS.md).
//
// A compiled file is a set of named arrays ("columns.x", "connections.area", ...) plus a few scalars. Each loader here
// is a declaration: a table of the arrays it reads, in the order the format hashes them, each with its element type,
// the length it must have and, for integers, the range it must fall in. One generic reader walks the table: it reads
// and checks every array, then re-hashes each one (FNV-1a over its little-endian bytes, -0 as 0) and the chain of all
// of them, and refuses the file when any hash differs from the one the file states: a value that did not survive the
// JSON round trip, or a hand-edited file. The hash order and the verdicts are the format's (the reference's loader,
// engine/src/compiled.cpp:82-279, reads the same files with the same outcome); the table-driven reader is this
// project's own.
#include "model.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <stdexcept>

#include "json.h"

namespace ssb {

// ----------------------------------------------------------------------------- FNV-1a

namespace {
template <class Word>
void feed_words(Fnv1a64& h, const Word* v, std::size_t n) {
  unsigned char b[sizeof(Word)];
  for (std::size_t i = 0; i < n; ++i) {
    Word w = v[i];
    for (std::size_t k = 0; k < sizeof(Word); ++k) { b[k] = static_cast<unsigned char>(w & 0xffu); w >>= 8; }
    h.update(b, sizeof(Word));
  }
}
}  // namespace

void Fnv1a64::f64(const double* v, std::size_t n) {
  std::vector<std::uint64_t> w(n);
  for (std::size_t i = 0; i < n; ++i) {
    const double d = v[i] == 0 ? 0.0 : v[i];  // -0 and +0 hash alike
    std::memcpy(&w[i], &d, 8);
  }
  feed_words(*this, w.data(), n);
}

void Fnv1a64::i32(const std::int32_t* v, std::size_t n) {
  std::vector<std::uint32_t> w(n);
  std::memcpy(w.data(), v, n * 4);
  feed_words(*this, w.data(), n);
}

std::string Fnv1a64::hex() const {
  char buf[17];
  for (int i = 0; i < 16; ++i) buf[i] = "0123456789abcdef"[(h_ >> (60 - 4 * i)) & 0xfu];
  buf[16] = 0;
  return buf;
}

std::int32_t CompiledSim::maxGroupSize() const {
  return gNodeCount.empty() ? 1 : std::max<std::int32_t>(1, *std::max_element(gNodeCount.begin(), gNodeCount.end()));
}

std::int32_t CompiledSim::kindIndex(const std::string& name) const {
  const auto it = std::find(kindNames.begin(), kindNames.end(), name);
  return it == kindNames.end() ? -1 : static_cast<std::int32_t>(it - kindNames.begin());
}

// ----------------------------------------------------------------------------- the table-driven reader

namespace {

using json::Value;

// A compiled document: the parsed JSON, its file name for the messages, and lookups by dotted path.
class Document {
 public:
  Document(const std::string& file, const char* format) : file_(file), doc_(json::read_file(file)) {
    if (json::string_or(doc_, "format", "") != format) fail(std::string("not a ") + format + " file");
    const long long v = json::integer(doc_, "formatVersion", file_);
    if (v != 1) fail("formatVersion " + std::to_string(v) + " cannot be read (this engine reads version 1)");
  }
  [[noreturn]] void fail(const std::string& why) const { throw std::runtime_error(file_ + ": " + why); }
  const Value& at(const std::string& path) const {
    const Value* v = find(path);
    if (!v) fail("missing " + path);
    return *v;
  }
  const Value* find(const std::string& path) const {
    const Value* v = &doc_;
    std::size_t from = 0;
    while (v) {
      const std::size_t dot = path.find('.', from);
      v = v->find(path.substr(from, dot == std::string::npos ? std::string::npos : dot - from));
      if (dot == std::string::npos) break;
      from = dot + 1;
    }
    return v;
  }
  double scalar(const std::string& path) const {
    const Value& v = at(path);
    if (!v.is_number()) fail(path + " is not a number");
    return v.as_double();
  }
  std::size_t count(const std::string& path) const {
    const double d = scalar(path);
    if (!(d >= 0) || d != std::floor(d)) fail(path + " is not a count");
    return static_cast<std::size_t>(d);
  }
  std::string text(const std::string& path) const {
    const Value& v = at(path);
    if (!v.is_string()) fail(path + " is not a string");
    return v.as_string();
  }
  std::string text_or(const std::string& path, const std::string& fallback) const {
    const Value* v = find(path);
    return v && v->is_string() ? v->as_string() : fallback;
  }
  // length of the array at path (the arrays whose length defines a count)
  std::size_t length(const std::string& path) const {
    const Value& v = at(path);
    if (!v.is_array()) fail(path + " is not an array");
    return v.size();
  }
  const std::string& file() const { return file_; }

 private:
  std::string file_;
  Value doc_;
};

constexpr std::size_t kAnyLength = static_cast<std::size_t>(-1);

// One array of a compiled file: its path, where it goes, the length it must have, the integer range (for Int and
// Byte) and whether the format hashes it.
struct ArraySpec {
  enum Kind { Real, Int, Byte, Text } kind;
  const char* path;
  void* out;  // std::vector<double> / <std::int32_t> / <std::uint8_t> / <std::string>
  std::size_t length;
  long long lo, hi;
  bool hashed;
};

ArraySpec reals(const char* path, std::vector<double>& out, std::size_t length) { return {ArraySpec::Real, path, &out, length, 0, 0, true}; }
ArraySpec ints(const char* path, std::vector<std::int32_t>& out, std::size_t length, long long lo, long long hi) {
  return {ArraySpec::Int, path, &out, length, lo, hi, true};
}
ArraySpec bytes(const char* path, std::vector<std::uint8_t>& out, std::size_t length) { return {ArraySpec::Byte, path, &out, length, 0, 255, true}; }
ArraySpec texts(const char* path, std::vector<std::string>& out, std::size_t length) { return {ArraySpec::Text, path, &out, length, 0, 0, false}; }

void read_one(const Document& d, const ArraySpec& s) {
  const Value& a = d.at(s.path);
  if (!a.is_array()) d.fail(std::string(s.path) + " is not an array");
  if (s.length != kAnyLength && a.size() != s.length)
    d.fail(std::string(s.path) + ": " + std::to_string(a.size()) + " values where the file declares " + std::to_string(s.length));
  const std::vector<Value>& items = a.items();
  if (s.kind == ArraySpec::Text) {
    auto& out = *static_cast<std::vector<std::string>*>(s.out);
    out.clear();
    for (const Value& v : items) {
      if (!v.is_string()) d.fail(std::string(s.path) + " holds a value that is not a string");
      out.push_back(v.as_string());
    }
    return;
  }
  std::vector<double> vals(items.size());
  for (std::size_t i = 0; i < items.size(); ++i) {
    if (!items[i].is_number()) d.fail(std::string(s.path) + "[" + std::to_string(i) + "] is not a number");
    vals[i] = items[i].as_double();
  }
  if (s.kind == ArraySpec::Real) {
    *static_cast<std::vector<double>*>(s.out) = std::move(vals);
    return;
  }
  for (std::size_t i = 0; i < vals.size(); ++i)
    if (vals[i] != std::floor(vals[i]) || vals[i] < static_cast<double>(s.lo) || vals[i] > static_cast<double>(s.hi))
      d.fail(std::string(s.path) + "[" + std::to_string(i) + "] = " + json::format_number(vals[i]) + " is outside the integers " +
             std::to_string(s.lo) + " .. " + std::to_string(s.hi));
  if (s.kind == ArraySpec::Int) {
    auto& out = *static_cast<std::vector<std::int32_t>*>(s.out);
    out.assign(vals.size(), 0);
    std::transform(vals.begin(), vals.end(), out.begin(), [](double x) { return static_cast<std::int32_t>(x); });
  } else {
    auto& out = *static_cast<std::vector<std::uint8_t>*>(s.out);
    out.assign(vals.size(), 0);
    std::transform(vals.begin(), vals.end(), out.begin(), [](double x) { return static_cast<std::uint8_t>(x); });
  }
}

void hash_into(Fnv1a64& h, const ArraySpec& s) {
  switch (s.kind) {
    case ArraySpec::Real: { const auto& v = *static_cast<const std::vector<double>*>(s.out); h.f64(v.data(), v.size()); break; }
    case ArraySpec::Int: { const auto& v = *static_cast<const std::vector<std::int32_t>*>(s.out); h.i32(v.data(), v.size()); break; }
    case ArraySpec::Byte: { const auto& v = *static_cast<const std::vector<std::uint8_t>*>(s.out); h.u8(v.data(), v.size()); break; }
    case ArraySpec::Text: break;
  }
}

// Reads every array of the table, then checks the file's per-array hashes and the chained hash over the hashed arrays
// in table order; returns the chained hash.
std::string read_arrays(const Document& d, const std::vector<ArraySpec>& table) {
  for (const ArraySpec& s : table) read_one(d, s);
  // the "hash" block names each array by its dotted path as one key ("columns.x"), plus "all" for the chain
  const Value& stated_hashes = d.at("hash");
  auto stated_hash = [&](const std::string& key) {
    const Value* v = stated_hashes.find(key);
    if (!v || !v->is_string()) d.fail("the hash block has no " + key);
    return v->as_string();
  };
  Fnv1a64 chain;
  for (const ArraySpec& s : table) {
    if (!s.hashed) continue;
    Fnv1a64 own;
    hash_into(own, s);
    hash_into(chain, s);
    const std::string stated = stated_hash(s.path);
    if (own.hex() != stated)
      d.fail(std::string("hash mismatch on ") + s.path + ": the values hash to " + own.hex() + ", the file states " + stated);
  }
  const std::string stated = stated_hash("all");
  if (chain.hex() != stated) d.fail("hash mismatch on the chain of all arrays: " + chain.hex() + ", the file states " + stated);
  return chain.hex();
}

}  // namespace

// ----------------------------------------------------------------------------- the two formats

std::shared_ptr<CompiledShip> load_ship(const std::string& file) {
  const Document d(file, "sinksim.compiled-ship");
  auto S = std::make_shared<CompiledShip>();
  S->id = d.text("id");
  S->title = d.text_or("meta.title", "");
  const std::size_t nc = d.count("columns.n"), nn = d.count("nodes.n"), ns = d.count("segments.n");
  const auto ns_ll = static_cast<long long>(ns), nc_ll = static_cast<long long>(nc);
  // the hash order of the format: columns, nodes, segments
  S->hashAll = read_arrays(d, {
      reals("columns.x", S->x, nc), reals("columns.y", S->y, nc), reals("columns.dxdy", S->dxdy, nc),
      reals("columns.zlo", S->zlo, nc), reals("columns.zhi", S->zhi, nc),
      ints("columns.zone", S->zone, nc, 0, 1 << 30), ints("columns.side", S->side, nc, 0, 1),
      reals("nodes.mu", S->mu, nn), reals("nodes.vmax", S->vmax, nn), reals("nodes.amin", S->amin, nn), reals("nodes.aov", S->aov, nn),
      ints("nodes.segStart", S->segStart, nn, 0, ns_ll), ints("nodes.segCount", S->segCount, nn, 0, ns_ll),
      ints("segments.col", S->segCol, ns, 0, nc_ll - 1), reals("segments.a", S->segA, ns), reals("segments.e", S->segE, ns),
      texts("nodes.label", S->nodeLabel, nn),
  });
  for (std::size_t n = 0; n < nn; ++n)
    if (static_cast<std::size_t>(S->segStart[n]) + static_cast<std::size_t>(S->segCount[n]) > ns)
      d.fail("the segments of node " + std::to_string(n) + " run past the segment table");
  return S;
}

CompiledSim load_sim(const std::string& file) {
  const Document d(file, "sinksim.compiled-sim");
  CompiledSim M;
  M.id = d.text("id");
  M.shipId = d.text("ship");
  M.shipHash = d.text("shipHash");
  M.title = d.text_or("meta.title", "");
  M.rho = d.scalar("constants.rho");
  M.g = d.scalar("constants.g");
  M.dt = d.scalar("scheme.dt");
  M.t0 = d.scalar("state0.t"); M.zO0 = d.scalar("state0.zO"); M.pitch0 = d.scalar("state0.pitch"); M.roll0 = d.scalar("state0.roll");
  M.vz0 = d.scalar("state0.vz"); M.wth0 = d.scalar("state0.wth"); M.wph0 = d.scalar("state0.wph");
  M.gMargin = d.scalar("groups.margin");
  M.monitorThreshold = d.scalar("monitors.threshold");
  M.hullTopBelow = d.scalar("founder.hullTopBelow"); M.pitchAbsAbove = d.scalar("founder.pitchAbsAbove");
  M.buoyancyBelow = d.scalar("founder.buoyancyBelow"); M.minT = d.scalar("founder.minT");
  M.xFP = d.scalar("readout.xFP"); M.xAP = d.scalar("readout.xAP");
  // the body: ms, KG, g0 (three values), then XO .. qph
  M.body[0] = d.scalar("body.ms");
  M.body[1] = d.scalar("body.KG");
  std::vector<double> g0;
  read_one(d, reals("body.g0", g0, 3));
  std::copy(g0.begin(), g0.end(), M.body + 2);
  const char* tail[] = {"XO", "YO", "mh0", "Ith0", "Iph0", "cDz", "cDth", "cDph", "qz", "qth", "qph"};
  for (int k = 0; k < 11; ++k) M.body[5 + k] = d.scalar(std::string("body.") + tail[k]);

  // counts: nodes from the initial volumes, the rest declared or from their id lists
  const std::size_t nn = d.length("state0.vol"), ng = d.count("groups.n"), nk = d.count("connections.n");
  const std::size_t members = d.length("groups.nodes"), nmon = d.length("monitors.id"), nmark = d.length("marks.id");
  const auto nn_ll = static_cast<long long>(nn), ng_ll = static_cast<long long>(ng);
  // the hash order of the format: groups, connections, marks, initial state
  M.hashAll = read_arrays(d, {
      ints("groups.nodeStart", M.gNodeStart, ng, 0, static_cast<long long>(members)), ints("groups.nodeCount", M.gNodeCount, ng, 1, 1 << 20),
      ints("groups.nodes", M.gNodes, kAnyLength, 0, nn_ll - 1), bytes("groups.mode", M.gMode, ng),
      reals("groups.px", M.gpx, ng), reals("groups.py", M.gpy, ng), reals("groups.pz", M.gpz, ng),
      ints("connections.a", M.ca, nk, -1, nn_ll - 1), ints("connections.b", M.cb, nk, 0, nn_ll - 1), bytes("connections.type", M.cLaw, nk),
      reals("connections.x", M.cx, nk), reals("connections.y", M.cy, nk), reals("connections.z", M.cz, nk),
      reals("connections.area", M.cArea, nk), reals("connections.coef", M.cCoef, nk), bytes("connections.kind", M.cKind, nk),
      ints("connections.idx", M.cIdx, nk, -1, 1 << 30), bytes("connections.en", M.cEn, nk), reals("connections.tOn", M.cTOn, nk),
      ints("connections.skipGroup", M.cSkipGroup, nk, -1, ng_ll - 1), ints("connections.monitor", M.cMonitor, nk, -1, static_cast<long long>(nmon) - 1),
      reals("marks.x", M.mkx, nmark), reals("marks.y", M.mky, nmark), reals("marks.z", M.mkz, nmark), bytes("marks.when", M.mkWhen, nmark),
      reals("state0.vol", M.vol0, nn), reals("state0.level", M.level0, nn), reals("state0.cx", M.cx0, nn), reals("state0.cy", M.cy0, nn),
      reals("state0.cz", M.cz0, nn),
      texts("monitors.id", M.monitorId, nmon), texts("monitors.label", M.monitorLabel, nmon),
      texts("marks.id", M.markId, nmark), texts("marks.label", M.markLabel, nmark),
  });
  if (d.find("connections.kindNames")) read_one(d, texts("connections.kindNames", M.kindNames, kAnyLength));
  for (std::size_t g = 0; g < ng; ++g)
    if (static_cast<std::size_t>(M.gNodeStart[g]) + static_cast<std::size_t>(M.gNodeCount[g]) > members)
      d.fail("the members of group " + std::to_string(g) + " run past the member table");
  return M;
}

void check_pairing(const CompiledShip& ship, const CompiledSim& sim) {
  // the sim names the ship it was compiled for and the chained hash of that ship's arrays
  // (engine/src/compiled.cpp:275-279 of the reference makes the same three checks)
  if (sim.shipId != ship.id) throw std::runtime_error("simulation " + sim.id + " belongs to ship " + sim.shipId + ", not to " + ship.id);
  if (sim.shipHash != ship.hashAll)
    throw std::runtime_error("simulation " + sim.id + " was compiled against another build of ship " + ship.id + " (its ship hash " + sim.shipHash +
                             ", the ship's " + ship.hashAll + ")");
  if (sim.nodes() != ship.nodes())
    throw std::runtime_error("simulation " + sim.id + " describes " + std::to_string(sim.nodes()) + " nodes, ship " + ship.id + " has " +
                             std::to_string(ship.nodes()));
}

// ----------------------------------------------------------------------------- derived tables

Incidence build_incidence(const CompiledSim& sim) {
  // Every connection touches its b node (+dV) and, unless it opens to the sea, its a node (-dV). Listing those
  // touches in connection order and sorting them stably by node gives each node its connections in increasing
  // order: the order in which a scatter over the connections would have added them (engine/src/model.cpp:26-56 of
  // the reference builds the same lists).
  struct Touch {
    std::int32_t node, conn;
    std::uint8_t side;
  };
  std::vector<Touch> touches;
  Incidence inc;
  for (std::int32_t c = 0; c < sim.connections(); ++c) {
    if (sim.ca[c] >= 0) touches.push_back({sim.ca[c], c, 0});
    else inc.sea.push_back(c);
    touches.push_back({sim.cb[c], c, 1});
  }
  std::stable_sort(touches.begin(), touches.end(), [](const Touch& x, const Touch& y) { return x.node < y.node; });
  const auto nn = static_cast<std::size_t>(sim.nodes());
  inc.count.assign(nn, 0);
  for (const Touch& t : touches) {
    inc.count[static_cast<std::size_t>(t.node)]++;
    inc.conn.push_back(t.conn);
    inc.side.push_back(t.side);
  }
  inc.start.assign(nn, 0);
  std::partial_sum(inc.count.begin(), inc.count.end() - (nn ? 1 : 0), inc.start.begin() + (nn ? 1 : 0));
  return inc;
}

MonitorLists build_monitor_lists(const CompiledSim& sim) {
  // per monitor the connections that report to it, in increasing order (the monitor sums of the event pass)
  MonitorLists L;
  const auto nm = static_cast<std::size_t>(sim.monitors());
  std::vector<std::vector<std::int32_t>> lists(nm);
  for (std::int32_t c = 0; c < sim.connections(); ++c)
    if (sim.cMonitor[static_cast<std::size_t>(c)] >= 0) lists[static_cast<std::size_t>(sim.cMonitor[static_cast<std::size_t>(c)])].push_back(c);
  for (const auto& l : lists) {
    L.start.push_back(static_cast<std::int32_t>(L.conn.size()));
    L.count.push_back(static_cast<std::int32_t>(l.size()));
    L.conn.insert(L.conn.end(), l.begin(), l.end());
  }
  return L;
}

}  // namespace ssb
