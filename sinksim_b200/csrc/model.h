// Compiled ship and sim (the reference's on-disk formats "sinksim.compiled-ship" and "sinksim.compiled-sim",
// docs/FORMATS.md of the reference) as host containers, their loaders with FNV-1a verification, and the derived
// tables the device needs.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace ssb {

// FNV-1a 64 over little-endian bytes; -0 is hashed as 0 (engine/include/sinksim/hash.hpp:15-56 of the reference).
class Fnv1a64 {
 public:
  void update(const void* data, std::size_t n) {
    const auto* p = static_cast<const unsigned char*>(data);
    for (std::size_t i = 0; i < n; ++i) { h_ ^= p[i]; h_ *= 1099511628211ULL; }
  }
  void f64(const double* v, std::size_t n);
  void i32(const std::int32_t* v, std::size_t n);
  void u8(const std::uint8_t* v, std::size_t n) { update(v, n); }
  std::uint64_t value() const { return h_; }
  std::string hex() const;

 private:
  std::uint64_t h_ = 14695981039346656037ULL;
};

struct CompiledShip {
  std::string id, title, hashAll;
  std::vector<double> x, y, dxdy, zlo, zhi;
  std::vector<std::int32_t> zone, side;
  std::vector<std::string> nodeLabel;
  std::vector<double> mu, vmax, amin, aov;
  std::vector<std::int32_t> segStart, segCount, segCol;
  std::vector<double> segA, segE;
  std::int32_t columns() const { return static_cast<std::int32_t>(x.size()); }
  std::int32_t nodes() const { return static_cast<std::int32_t>(mu.size()); }
  std::int32_t segments() const { return static_cast<std::int32_t>(segCol.size()); }
};

struct CompiledSim {
  std::string id, title, shipId, shipHash, hashAll;
  double rho = 0, g = 0, dt = 0;
  std::vector<std::int32_t> gNodeStart, gNodeCount, gNodes;
  std::vector<std::uint8_t> gMode;
  std::vector<double> gpx, gpy, gpz;
  double gMargin = 0;
  std::vector<std::int32_t> ca, cb;
  std::vector<std::uint8_t> cLaw;
  std::vector<double> cx, cy, cz, cArea, cCoef;
  std::vector<std::uint8_t> cKind;
  std::vector<std::int32_t> cIdx;
  std::vector<std::uint8_t> cEn;
  std::vector<double> cTOn;
  std::vector<std::int32_t> cSkipGroup, cMonitor;
  std::vector<std::string> kindNames;
  double monitorThreshold = 0;
  std::vector<std::string> monitorId, monitorLabel, markId, markLabel;
  std::vector<double> mkx, mky, mkz;
  std::vector<std::uint8_t> mkWhen;
  double hullTopBelow = 0, pitchAbsAbove = 0, buoyancyBelow = 0, minT = 0;
  // ms, KG, g0x, g0y, g0z, XO, YO, mh0, Ith0, Iph0, cDz, cDth, cDph, qz, qth, qph
  double body[16] = {};
  double xFP = 0, xAP = 0;
  double t0 = 0, zO0 = 0, pitch0 = 0, roll0 = 0, vz0 = 0, wth0 = 0, wph0 = 0;
  std::vector<double> vol0, level0, cx0, cy0, cz0;

  std::int32_t groups() const { return static_cast<std::int32_t>(gNodeCount.size()); }
  std::int32_t connections() const { return static_cast<std::int32_t>(ca.size()); }
  std::int32_t monitors() const { return static_cast<std::int32_t>(monitorId.size()); }
  std::int32_t marks() const { return static_cast<std::int32_t>(mkx.size()); }
  std::int32_t nodes() const { return static_cast<std::int32_t>(vol0.size()); }
  std::int32_t maxGroupSize() const;
  std::int32_t kindIndex(const std::string& name) const;  // -1 when the kind is not defined
};

std::shared_ptr<CompiledShip> load_ship(const std::string& path);
CompiledSim load_sim(const std::string& path);
// Throws unless the sim was compiled against this ship (engine/src/compiled.cpp:275-279 of the reference).
void check_pairing(const CompiledShip& ship, const CompiledSim& sim);

// Per node its connections in increasing order (side 1 at the b end) and the sea connections in order: the
// gather that reproduces a scatter in connection order (engine/src/model.cpp:26-56 of the reference).
struct Incidence {
  std::vector<std::int32_t> start, count, conn, sea;
  std::vector<std::uint8_t> side;
};
Incidence build_incidence(const CompiledSim& sim);

// Per monitor its connections in increasing order: the monitor sums of the event pass in the reference's order.
struct MonitorLists {
  std::vector<std::int32_t> start, count, conn;
};
MonitorLists build_monitor_lists(const CompiledSim& sim);

}  // namespace ssb
