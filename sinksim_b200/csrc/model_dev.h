// Device memory of one compiled model and of the buffers the engines own: DevBuf (an owning device array) and ModelDev
// (a compiled ship and sim in the kernels' layout, DevModel pointing into it). Shared by the batch engine (batch.cpp)
// and the adjoint engine (adjoint.cpp).
#pragma once

#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "device_model.h"
#include "model.h"

namespace ssb {

inline void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + what + ": " + cudaGetErrorString(e));
}


// A device array that owns its allocation.
template <class T>
class DevBuf {
 public:
  DevBuf() = default;
  ~DevBuf() { release(); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  void alloc(std::size_t n) {
    if (p_ && n == n_) return;  // same size: keep the allocation (a re-run reuses every buffer)
    release();
    n_ = n;
    if (n) check(cudaMalloc(reinterpret_cast<void**>(&p_), n * sizeof(T)), "cudaMalloc");
  }
  void upload(const std::vector<T>& v, cudaStream_t s) {
    if (v.size() != n_) alloc(v.size());
    if (n_) check(cudaMemcpyAsync(p_, v.data(), n_ * sizeof(T), cudaMemcpyHostToDevice, s), "copy to device");
  }
  void download(std::vector<T>& v, cudaStream_t s) const {
    v.resize(n_);
    if (n_) check(cudaMemcpyAsync(v.data(), p_, n_ * sizeof(T), cudaMemcpyDeviceToHost, s), "copy to host");
  }
  T* get() const { return p_; }
  std::size_t size() const { return n_; }
  std::size_t bytes() const { return n_ * sizeof(T); }

 private:
  T* p_ = nullptr;
  std::size_t n_ = 0;
  void release() {
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = 0;
  }
};


inline std::uint32_t take(std::uint32_t& off, std::size_t bytes) {
  const std::uint32_t at = off;
  off = static_cast<std::uint32_t>((off + bytes + 15) & ~static_cast<std::size_t>(15));
  return at;
}

// One compiled model on the device: its geometry in the kernel's layout (paired fields, the segment -> column gather
// resolved, float copies), its node, group, connection, incidence, monitor and mark tables, and the DevModel that
// points into them.
struct ModelDev {
  std::shared_ptr<const CompiledShip> ship;
  CompiledSim sim;
  Incidence inc;
  MonitorLists mons;
  std::int32_t NN = 0, NC = 0, NG = 0, nmon = 0, nmark = 0, evCap = 0, maxGroup = 0;
  DevBuf<double2> colXY, colLH, segXY, segLH;
  DevBuf<float2> colXYf, colLHf, segXYf, segLHf;
  DevBuf<float> colAf, segArf;
  DevBuf<double> colA, segAr, mu, vmax, amin, aov;
  DevBuf<std::int32_t> segStart, segCount, gStart, gCount, gNodes, ca, cb, skip, incStart, incCount, incConn, sea, monStart, monCount, monConn;
  DevBuf<std::uint8_t> gMode, law, incSide, mkWhen;
  DevBuf<double> gpx, gpy, gpz, kx, ky, kz, coef, mkx, mky, mkz;
  DevModel dm{};

  ModelDev(std::shared_ptr<const CompiledShip> s, const CompiledSim& m) : ship(std::move(s)), sim(m) {
    if (!ship) throw std::invalid_argument("Batch: null ship");
    check_pairing(*ship, sim);
    inc = build_incidence(sim);
    mons = build_monitor_lists(sim);
    NN = ship->nodes(); NC = sim.connections(); NG = sim.groups();
    nmon = sim.monitors(); nmark = sim.marks(); evCap = nmon + nmark + 1; maxGroup = sim.maxGroupSize();
  }

  void upload(cudaStream_t s) {
    const CompiledShip& S = *ship;
    const CompiledSim& M = sim;
    {
      const std::size_t nc = S.x.size(), ns = S.segCol.size();
      std::vector<double2> cxy(nc), clh(nc), sxy(ns), slh(ns);
      std::vector<float2> cxyf(nc), clhf(nc), sxyf(ns), slhf(ns);
      std::vector<double> sa(ns);
      std::vector<float> caf(nc), saf(ns);
      for (std::size_t i = 0; i < nc; ++i) {
        cxy[i] = double2{S.x[i], S.y[i]};
        clh[i] = double2{S.zlo[i], S.zhi[i]};
        cxyf[i] = float2{static_cast<float>(S.x[i]), static_cast<float>(S.y[i])};
        clhf[i] = float2{static_cast<float>(S.zlo[i]), static_cast<float>(S.zhi[i])};
        caf[i] = static_cast<float>(S.dxdy[i]);
      }
      for (std::size_t j = 0; j < ns; ++j) {
        const auto c = static_cast<std::size_t>(S.segCol[j]);
        sxy[j] = double2{S.x[c], S.y[c]};
        slh[j] = double2{S.segA[j], S.segE[j]};
        sa[j] = S.dxdy[c];
        sxyf[j] = float2{static_cast<float>(S.x[c]), static_cast<float>(S.y[c])};
        slhf[j] = float2{static_cast<float>(S.segA[j]), static_cast<float>(S.segE[j])};
        saf[j] = static_cast<float>(S.dxdy[c]);
      }
      colXY.upload(cxy, s); colLH.upload(clh, s); colA.upload(S.dxdy, s);
      colXYf.upload(cxyf, s); colLHf.upload(clhf, s); colAf.upload(caf, s);
      segXY.upload(sxy, s); segLH.upload(slh, s); segAr.upload(sa, s);
      segXYf.upload(sxyf, s); segLHf.upload(slhf, s); segArf.upload(saf, s);
      check(cudaStreamSynchronize(s), "stream sync");
    }
    mu.upload(S.mu, s); vmax.upload(S.vmax, s); amin.upload(S.amin, s); aov.upload(S.aov, s);
    segStart.upload(S.segStart, s); segCount.upload(S.segCount, s);
    gStart.upload(M.gNodeStart, s); gCount.upload(M.gNodeCount, s); gNodes.upload(M.gNodes, s); gMode.upload(M.gMode, s);
    gpx.upload(M.gpx, s); gpy.upload(M.gpy, s); gpz.upload(M.gpz, s);
    ca.upload(M.ca, s); cb.upload(M.cb, s); skip.upload(M.cSkipGroup, s); law.upload(M.cLaw, s);
    kx.upload(M.cx, s); ky.upload(M.cy, s); kz.upload(M.cz, s); coef.upload(M.cCoef, s);
    incStart.upload(inc.start, s); incCount.upload(inc.count, s); incConn.upload(inc.conn, s); incSide.upload(inc.side, s);
    sea.upload(inc.sea.empty() ? std::vector<std::int32_t>{0} : inc.sea, s);
    monStart.upload(mons.start.empty() ? std::vector<std::int32_t>{0} : mons.start, s);
    monCount.upload(mons.count.empty() ? std::vector<std::int32_t>{0} : mons.count, s);
    monConn.upload(mons.conn.empty() ? std::vector<std::int32_t>{0} : mons.conn, s);
    mkx.upload(M.mkx.empty() ? std::vector<double>{0} : M.mkx, s);
    mky.upload(M.mky.empty() ? std::vector<double>{0} : M.mky, s);
    mkz.upload(M.mkz.empty() ? std::vector<double>{0} : M.mkz, s);
    mkWhen.upload(M.mkWhen.empty() ? std::vector<std::uint8_t>{0} : M.mkWhen, s);
    check(cudaStreamSynchronize(s), "model upload");

    DevModel& d = dm;
    d.ncol = S.columns();
    d.colXY = colXY.get(); d.colLH = colLH.get(); d.colA = colA.get();
    d.colXYf = colXYf.get(); d.colLHf = colLHf.get(); d.colAf = colAf.get();
    d.nseg = S.segments();
    d.segXY = segXY.get(); d.segLH = segLH.get(); d.segAr = segAr.get();
    d.segXYf = segXYf.get(); d.segLHf = segLHf.get(); d.segArf = segArf.get();
    d.nn = NN;
    d.mu = mu.get(); d.vmax = vmax.get(); d.amin = amin.get(); d.aov = aov.get();
    d.segStart = segStart.get(); d.segCount = segCount.get();
    d.ng = NG;
    d.gStart = gStart.get(); d.gCount = gCount.get(); d.gNodes = gNodes.get(); d.gMode = gMode.get();
    d.gpx = gpx.get(); d.gpy = gpy.get(); d.gpz = gpz.get(); d.gMargin = M.gMargin; d.maxGroup = maxGroup;
    d.nc = NC;
    d.ca = ca.get(); d.cb = cb.get(); d.skip = skip.get(); d.law = law.get();
    d.kx = kx.get(); d.ky = ky.get(); d.kz = kz.get(); d.coef = coef.get();
    d.incStart = incStart.get(); d.incCount = incCount.get(); d.incConn = incConn.get(); d.incSide = incSide.get();
    d.nsea = static_cast<std::int32_t>(inc.sea.size()); d.sea = sea.get();
    d.nmon = nmon; d.monThreshold = M.monitorThreshold;
    d.monStart = monStart.get(); d.monCount = monCount.get(); d.monConn = monConn.get();
    d.nmark = nmark; d.mkx = mkx.get(); d.mky = mky.get(); d.mkz = mkz.get(); d.mkWhen = mkWhen.get();
    d.hullTopBelow = M.hullTopBelow; d.pitchAbsAbove = M.pitchAbsAbove; d.buoyancyBelow = M.buoyancyBelow; d.minT = M.minT;
    d.rho = M.rho; d.g = M.g; d.sq2g = std::sqrt(2 * M.g); d.dt = M.dt;
    d.ms = M.body[0]; d.g0x = M.body[2]; d.g0y = M.body[3]; d.g0z = M.body[4]; d.XO = M.body[5]; d.YO = M.body[6];
    d.mh0 = M.body[7]; d.Ith0 = M.body[8]; d.Iph0 = M.body[9]; d.cDz = M.body[10]; d.cDth = M.body[11]; d.cDph = M.body[12];
    d.qz = M.body[13]; d.qth = M.body[14]; d.qph = M.body[15];
    d.xFP = M.xFP; d.xAP = M.xAP;
    d.evCap = evCap;
  }
};

}  // namespace ssb
