#include "batch.h"

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <stdexcept>

#include <cuda_runtime.h>

#include "batch_kernel.h"
#include "model_dev.h"

namespace ssb {

bool cuda_available(std::string* why) {
  int n = 0;
  const cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    if (why) *why = cudaGetErrorString(e);
    return false;
  }
  if (n == 0) {
    if (why) *why = "no CUDA device";
    return false;
  }
  return true;
}

DeviceInfo device_info(int device) {
  DeviceInfo d;
  cudaDeviceProp p{};
  check(cudaGetDeviceProperties(&p, device), "cudaGetDeviceProperties");
  d.name = p.name;
  d.major = p.major; d.minor = p.minor; d.multiprocessors = p.multiProcessorCount;
  d.globalMemory = p.totalGlobalMem; d.sharedPerBlockOptIn = p.sharedMemPerBlockOptin; d.sharedPerSM = p.sharedMemPerMultiprocessor;
  cudaRuntimeGetVersion(&d.runtimeVersion);
  cudaDriverGetVersion(&d.driverVersion);
  return d;
}

struct Batch::Impl {
  // The models of the batch (one, or several for a fleet), the model of every instance and where each instance's
  // per-node, per-connection, event, monitor and mark values start in the per-instance arrays (count + 1 prefix sums).
  std::vector<std::unique_ptr<ModelDev>> models;
  std::vector<std::int32_t> instModel;
  std::vector<long long> nodeOff, connOff, evOff, monOff, markOff;
  DevBuf<DevModel> dModels;
  DevBuf<std::int32_t> dInstModel;
  DevBuf<long long> dNodeOff, dConnOff, dEvOff, dMonOff, dMarkOff;
  DeviceInfo info;
  // the largest sizes over the models (the slot is laid out for them) and the trace/curve record counts
  std::int32_t NN = 0, NC = 0, NG = 0, maxGroup = 0, recSize = 0, maxSamples = 0, curveMax = 0;

  bool fleet() const { return models.size() > 1; }
  const ModelDev& m0() const { return *models.front(); }
  const ModelDev& model(std::size_t inst) const { return *models[static_cast<std::size_t>(instModel[inst])]; }

  // The shared-memory slot of one simulation stepped by a team of W warps: per-node state and scratch, per-connection
  // dV and q, the group-pass buffers, the buoyancy tree results, the pose, buoyancy result and parked run values, and
  // in a fleet the team's copy of its instance's model. The loads' sixth scratch column reuses dV when there are at
  // least as many connections as nodes.
  SlotLayout layout_for(int W) const {
    SlotLayout L{};
    std::uint32_t off = 0;
    const std::size_t nb = sizeof(double) * static_cast<std::size_t>(NN);
    L.vol = take(off, nb); L.level = take(off, nb); L.cx = take(off, nb); L.cy = take(off, nb); L.cz = take(off, nb);
    L.area = take(off, nb); L.zmax = take(off, nb); L.hEff = take(off, nb); L.aEff = take(off, nb); L.acc = take(off, nb);
    L.deg = take(off, sizeof(std::int32_t) * static_cast<std::size_t>(NN));
    L.dV = take(off, sizeof(double) * static_cast<std::size_t>(std::max(NC, 1)));
    L.q = take(off, sizeof(double) * static_cast<std::size_t>(std::max(NC, 1)));
    L.tmp = NC >= NN ? kSlotAliasDV : take(off, nb);
    L.passes = take(off, 7 * sizeof(double) * static_cast<std::size_t>(maxGroup) * static_cast<std::size_t>(W * kMaxLevelGroupsPerWarp));
    L.hydro = take(off, 8 * 5 * sizeof(double));
    L.misc = take(off, 4 * sizeof(std::int32_t));
    L.merged = take(off, static_cast<std::size_t>(std::max(NG, 1)));
    L.pose = take(off, sizeof(Pose));
    L.buoy = take(off, sizeof(Buoy));
    L.parked = take(off, sizeof(Parked));
    L.model = fleet() ? take(off, sizeof(DevModel)) : 0u;
    L.bytes = off;
    return L;
  }
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> phaseEv;           // launch phase k ends at phaseEv[k + 1]; phaseEv[0] starts a round
  // one run's launch chain as a CUDA graph (runs to the end in one launch per phase), captured at the first launch;
  // graphKey holds the kernel arguments it was captured with, so that a moved buffer captures it again
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graphExec = nullptr;
  std::vector<unsigned char> graphKey;
  DevBuf<unsigned long long> phaseSteps;      // steps per launch phase in the last launch()
  // claim order of the phases after the first (launch_order_unfinished): unfinished instances, their order, its length
  DevBuf<std::int32_t> orderList, order, orderCount;
  // the caller's claim order of the first phase (set_claim_order; empty: by index) and its device copy
  std::vector<std::int32_t> hOrder0;
  DevBuf<std::int32_t> order0, order0Count;
  std::vector<float> lastPhaseMs;
  std::vector<std::int32_t> lastHealth;       // the error word (HealthBit flags) of the last launch()
  std::vector<unsigned long long> lastPhaseSteps;


  // per instance (device)
  DevBuf<std::uint8_t> en;
  DevBuf<double> area, tOn, st, out, vol, level, cx, cy, cz, evT, overT, markT, founderT, curveRec, nextCurve, finalRec, denseRec,
      sampleRec, nextSample;
  DevBuf<std::int32_t> evId, evKind, evCount, foundered, stop, curveCount, denseCount, sampleCount, queue, error, remaining;
  DevBuf<long long> steps;

  // host staging
  std::vector<std::uint8_t> hEn;
  std::vector<double> hArea, hTOn, hSt, hVol, hLevel, hCx, hCy, hCz;
  // host results
  struct {
    std::vector<double> st, out, vol, level, cx, cy, cz, evT, founderT, curveRec, finalRec, denseRec, sampleRec;
    std::vector<std::int32_t> evId, evKind, evCount, foundered, stop, curveCount, denseCount, sampleCount;
    std::vector<long long> steps;
  } r;
  bool uploaded = false, launched = false, downloaded = false;

  DevBatch devBatch(const BatchOptions& opt, long long maxSteps, int firstLaunch) {
    DevBatch b{};
    b.count = opt.count;
    b.en = en.get(); b.area = area.get(); b.tOn = tOn.get();
    b.st = st.get(); b.out = out.get();
    b.vol = vol.get(); b.level = level.get(); b.cx = cx.get(); b.cy = cy.get(); b.cz = cz.get();
    b.evT = evT.get(); b.evId = evId.get(); b.evKind = evKind.get(); b.evCount = evCount.get();
    b.overT = overT.get(); b.markT = markT.get(); b.foundered = foundered.get(); b.founderT = founderT.get();
    b.steps = steps.get(); b.stop = stop.get();
    b.curveEvery = opt.curveEvery; b.curveMax = curveMax;
    b.curveRec = curveRec.get(); b.curveCount = curveCount.get(); b.nextCurve = nextCurve.get();
    b.finalRec = finalRec.get();
    b.traced = opt.tracedInstances; b.denseSteps = opt.denseSteps; b.maxSamples = maxSamples; b.recSize = recSize;
    b.sampleEvery = opt.sampleEvery;
    b.denseRec = denseRec.get(); b.sampleRec = sampleRec.get();
    b.denseCount = denseCount.get(); b.sampleCount = sampleCount.get(); b.nextSample = nextSample.get();
    b.tMax = opt.tMax;
    b.maxSteps = maxSteps;
    b.firstLaunch = firstLaunch;
    b.rule = opt.rule;
    b.stopWhenStable = opt.stopWhenStable ? 1 : 0;
    b.queue = queue.get();
    b.error = error.get();
    b.remaining = remaining.get();
    b.yieldBelow = 0;
    if (fleet()) {
      b.models = dModels.get(); b.model = dInstModel.get();
      b.nodeOff = dNodeOff.get(); b.connOff = dConnOff.get(); b.evOff = dEvOff.get(); b.monOff = dMonOff.get(); b.markOff = dMarkOff.get();
    }
    return b;
  }
};

Batch::Batch(std::shared_ptr<const CompiledShip> ship, const CompiledSim& sim, const BatchOptions& opt) : I_(new Impl), opt_(opt) {
  std::vector<std::pair<std::shared_ptr<const CompiledShip>, CompiledSim>> models;
  models.emplace_back(std::move(ship), sim);
  init(std::move(models), std::vector<std::int32_t>(static_cast<std::size_t>(std::max(opt.count, 0)), 0));
}

Batch::Batch(std::vector<std::pair<std::shared_ptr<const CompiledShip>, CompiledSim>> models, std::vector<std::int32_t> instanceModel,
             const BatchOptions& opt)
    : I_(new Impl), opt_(opt) {
  opt_.count = static_cast<std::int32_t>(instanceModel.size());
  init(std::move(models), std::move(instanceModel));
}

void Batch::init(std::vector<std::pair<std::shared_ptr<const CompiledShip>, CompiledSim>> models, std::vector<std::int32_t> instanceModel) {
  Impl& I = *I_;
  if (models.empty()) throw std::invalid_argument("Batch: no model");
  if (opt_.count < 1) throw std::invalid_argument("Batch: count must be at least 1");
  if (!(opt_.tMax > 0)) throw std::invalid_argument("Batch: tMax must be positive");
  if (models.size() > 1 && opt_.tracedInstances > 0) throw std::invalid_argument("Batch: a fleet of several models records no traces");
  if (models.size() > 1 && opt_.stepsPerLaunch > 0) throw std::invalid_argument("Batch: a fleet of several models runs in one launch per phase");
  if (opt_.tracedInstances > opt_.count) opt_.tracedInstances = opt_.count;
  if (opt_.tracedInstances < 0) opt_.tracedInstances = 0;
  if (opt_.tracedInstances > 0 && !(opt_.sampleEvery > 0)) throw std::invalid_argument("Batch: sampleEvery must be positive");
  if (opt_.stopWhenStable && opt_.rule.enabled) throw std::invalid_argument("Batch: stopWhenStable and the retire rule are exclusive");
  std::string why;
  if (!cuda_available(&why)) throw std::runtime_error("Batch: " + why);
  check(cudaSetDevice(opt_.device), "cudaSetDevice");
  for (auto& m : models) I.models.push_back(std::make_unique<ModelDev>(std::move(m.first), m.second));
  I.instModel = std::move(instanceModel);
  const auto count = static_cast<std::size_t>(opt_.count);
  I.nodeOff.assign(count + 1, 0); I.connOff.assign(count + 1, 0); I.evOff.assign(count + 1, 0);
  I.monOff.assign(count + 1, 0); I.markOff.assign(count + 1, 0);
  for (std::size_t i = 0; i < count; ++i) {
    const std::int32_t m = I.instModel[i];
    if (m < 0 || static_cast<std::size_t>(m) >= I.models.size())
      throw std::out_of_range("Batch: instance " + std::to_string(i) + " refers to model " + std::to_string(m) + " of " + std::to_string(I.models.size()));
    const ModelDev& d = *I.models[static_cast<std::size_t>(m)];
    I.nodeOff[i + 1] = I.nodeOff[i] + d.NN; I.connOff[i + 1] = I.connOff[i] + d.NC; I.evOff[i + 1] = I.evOff[i] + d.evCap;
    I.monOff[i + 1] = I.monOff[i] + d.nmon; I.markOff[i + 1] = I.markOff[i] + d.nmark;
  }
  for (const auto& d : I.models) {
    I.NN = std::max(I.NN, d->NN); I.NC = std::max(I.NC, d->NC); I.NG = std::max(I.NG, d->NG); I.maxGroup = std::max(I.maxGroup, d->maxGroup);
  }
  I.info = device_info(opt_.device);
  I.recSize = 10 + 5 * I.m0().NN;
  I.maxSamples = opt_.tracedInstances > 0 ? static_cast<std::int32_t>(std::floor(opt_.tMax / opt_.sampleEvery)) + 2 : 0;
  I.curveMax = opt_.curveEvery > 0 ? static_cast<std::int32_t>(std::floor(opt_.tMax / opt_.curveEvery)) + 2 : 0;

  // launch shape. Teams of W warps; a slot of shared memory per team; persistent grids sized to the device.
  // Main phase: single-warp teams when the batch fills the device (the most simulations per SM), larger teams when it
  // does not. Later phases: when the unfinished instances fit the resident teams of twice the size, they resume there.
  const bool fleet = I.fleet();
  const std::size_t optin = I.info.sharedPerBlockOptIn;
  const int sms = I.info.multiprocessors;
  cfg_.slotBytes = I.layout_for(1).bytes;
  if (cfg_.slotBytes > optin)
    throw std::runtime_error("Batch: one simulation needs " + std::to_string(cfg_.slotBytes) + " bytes of shared memory, the device allows " +
                             std::to_string(optin) + " per block");
  auto plan = [&](int W, int teamsReq, int count) {
    PhaseConfig p;
    if (!valid_team_size(W)) throw std::invalid_argument("Batch: warps per simulation must be 1, 2, 4, 8 or 16");
    p.teamWarps = W;
    p.layout = I.layout_for(W);
    const SlotLayout& L = p.layout;
    if (L.bytes > optin) throw std::runtime_error("Batch: a " + std::to_string(W) + "-warp simulation needs more shared memory than a block has");
    // the column table beside the slots when asked for and one simulation still fits beside it
    const std::size_t table = opt_.stageColumns && !fleet ? column_stage_bytes(opt_.mixedPrecision, I.m0().ship->columns()) : 0;
    p.stageColumns = table > 0 && table + L.bytes <= optin;
    const std::size_t room = p.stageColumns ? optin - table : optin;
    const int maxTeams = std::min(static_cast<int>(room / L.bytes), kMaxWarpsPerBlock / W);
    int tpb = teamsReq > 0 ? teamsReq : std::max(1, std::min(maxTeams, (count + sms - 1) / sms));
    tpb = std::max(1, std::min(tpb, maxTeams));
    p.teamsPerBlock = tpb;
    const std::size_t smem = static_cast<std::size_t>(tpb) * L.bytes + (p.stageColumns ? table : 0);
    check(configure_batch_kernel(opt_.mixedPrecision, W, smem, fleet), "cudaFuncSetAttribute");
    check(batch_kernel_occupancy(opt_.mixedPrecision, W, tpb, smem, &p.blocksPerSM, fleet), "occupancy");
    if (p.blocksPerSM < 1) throw std::runtime_error("Batch: the kernel cannot be resident with " + std::to_string(tpb) + " simulations per block");
    p.blocks = std::min((count + tpb - 1) / tpb, p.blocksPerSM * sms);
    return p;
  };
  int W1 = opt_.teamWarps;
  if (W1 <= 0) {
    // About 16 warps per SM in all. A batch that all fits at once in single-warp teams runs there; a larger one
    // starts in two-warp teams: with 16 slots per SM the slots leave too little of the SM's shared storage to L1 for
    // the geometry that every simulation reads (uneven titanic64 batches of 4096 and 8192 instances on B200: 7.3 and
    // 7.8 M steps/s in two-warp teams, 6.4 and 5.5 M in single-warp teams).
    const int fit = (sms * 16) / std::max(opt_.count, 1);
    W1 = fit >= 8 ? 8 : fit >= 4 ? 4 : fit >= 2 ? 2 : fit >= 1 ? 1 : 2;
    // Large slots (a fleet's largest hull sets the slot) fit few simulations per SM: start with teams big enough that
    // the simulations that fit carry about 16 warps (a fleet of 2,048 hulls up to 256 spaces: 5 slots of 41.7 KB
    // per SM, so 4-warp teams).
    const int slotsPerSM = std::max(1, static_cast<int>(optin / cfg_.slotBytes));
    while (W1 < 8 && W1 * slotsPerSM < 16) W1 *= 2;
  }
  cfg_.phases.push_back(plan(W1, opt_.teamsPerBlock, opt_.count));
  if (opt_.blocks > 0) cfg_.phases[0].blocks = opt_.blocks;
  // the last phase: a whole 16-warp block per simulation (the uneven titanic64 bench batch on B200: 4.12 s against
  // 4.25 s with 8-warp teams last, same bits; the lone simulations of the tail step faster in larger teams)
  const int Wlast = opt_.tailTeamWarps < 0 ? 16 : opt_.tailTeamWarps;
  if (Wlast > W1 && opt_.stepsPerLaunch <= 0) {
    for (int W = W1 * 2; W <= Wlast; W *= 2) {
      PhaseConfig p = plan(W, 0, opt_.count);
      p.blocks = p.blocksPerSM * sms;  // any instance may be left for it
      const double capacity = static_cast<double>(p.blocks) * p.teamsPerBlock;
      cfg_.phases.back().yieldBelow = static_cast<int>(std::min<double>(opt_.count - 1, std::ceil(opt_.handoverFactor * capacity)));
      cfg_.phases.push_back(p);
    }
    if (opt_.yieldBelow >= 0) cfg_.phases[0].yieldBelow = opt_.yieldBelow;
  }

  // model upload
  check(cudaStreamCreateWithFlags(&I.stream, cudaStreamNonBlocking), "cudaStreamCreate");
  check(cudaEventCreate(&I.ev0), "cudaEventCreate");
  check(cudaEventCreate(&I.ev1), "cudaEventCreate");
  I.phaseEv.assign(cfg_.phases.size() + 1, nullptr);
  for (cudaEvent_t& e : I.phaseEv) check(cudaEventCreate(&e), "cudaEventCreate");
  cudaStream_t s = I.stream;
  for (auto& d : I.models) d->upload(s);
  if (fleet) {
    std::vector<DevModel> dms;
    for (const auto& d : I.models) dms.push_back(d->dm);
    I.dModels.upload(dms, s);
    I.dInstModel.upload(I.instModel, s);
    I.dNodeOff.upload(I.nodeOff, s); I.dConnOff.upload(I.connOff, s); I.dEvOff.upload(I.evOff, s);
    I.dMonOff.upload(I.monOff, s); I.dMarkOff.upload(I.markOff, s);
    check(cudaStreamSynchronize(s), "fleet tables upload");
  }

  // per-instance staging: the compiled connection table and initial state of every instance's model
  I.hEn.resize(static_cast<std::size_t>(I.connOff[count])); I.hArea.resize(I.hEn.size()); I.hTOn.resize(I.hEn.size());
  const auto nodesTotal = static_cast<std::size_t>(I.nodeOff[count]);
  I.hVol.resize(nodesTotal); I.hLevel.resize(nodesTotal); I.hCx.resize(nodesTotal); I.hCy.resize(nodesTotal); I.hCz.resize(nodesTotal);
  I.hSt.resize(count * 8);
  for (std::size_t i = 0; i < count; ++i) {
    const CompiledSim& M = I.model(i).sim;
    double* p = &I.hSt[i * 8];
    p[0] = M.t0; p[1] = M.zO0; p[2] = M.pitch0; p[3] = M.roll0; p[4] = M.vz0; p[5] = M.wth0; p[6] = M.wph0; p[7] = 0;
    std::copy(M.cEn.begin(), M.cEn.end(), I.hEn.begin() + I.connOff[i]);
    std::copy(M.cArea.begin(), M.cArea.end(), I.hArea.begin() + I.connOff[i]);
    std::copy(M.cTOn.begin(), M.cTOn.end(), I.hTOn.begin() + I.connOff[i]);
    std::copy(M.vol0.begin(), M.vol0.end(), I.hVol.begin() + I.nodeOff[i]);
    std::copy(M.level0.begin(), M.level0.end(), I.hLevel.begin() + I.nodeOff[i]);
    std::copy(M.cx0.begin(), M.cx0.end(), I.hCx.begin() + I.nodeOff[i]);
    std::copy(M.cy0.begin(), M.cy0.end(), I.hCy.begin() + I.nodeOff[i]);
    std::copy(M.cz0.begin(), M.cz0.end(), I.hCz.begin() + I.nodeOff[i]);
  }
}

Batch::~Batch() {
  if (I_) {
    if (I_->stream) cudaStreamSynchronize(I_->stream);
    if (I_->ev0) cudaEventDestroy(I_->ev0);
    if (I_->ev1) cudaEventDestroy(I_->ev1);
    for (cudaEvent_t e : I_->phaseEv) if (e) cudaEventDestroy(e);
    if (I_->graphExec) cudaGraphExecDestroy(I_->graphExec);
    if (I_->graph) cudaGraphDestroy(I_->graph);
    if (I_->stream) cudaStreamDestroy(I_->stream);
  }
}

std::int32_t Batch::nodes() const { return I_->m0().NN; }
std::int32_t Batch::connections() const { return I_->m0().NC; }
std::int32_t Batch::models() const { return static_cast<std::int32_t>(I_->models.size()); }

Batch::InstanceShape Batch::instance_shape(std::int32_t inst) const {
  if (inst < 0 || inst >= opt_.count) throw std::out_of_range("Batch: instance " + std::to_string(inst) + " out of range");
  const ModelDev& d = I_->model(static_cast<std::size_t>(inst));
  return InstanceShape{I_->instModel[static_cast<std::size_t>(inst)], d.NN, d.NC};
}
std::size_t Batch::slot_bytes() const { return cfg_.slotBytes; }

static void check_inst(const BatchOptions& o, std::int32_t inst) {
  if (inst < 0 || inst >= o.count) throw std::out_of_range("Batch: instance " + std::to_string(inst) + " out of range");
}

void Batch::restore(std::int32_t inst, const double* rec) {
  Impl& I = *I_;
  if (I.uploaded) throw std::logic_error("Batch: restore after run");
  check_inst(opt_, inst);
  const auto i = static_cast<std::size_t>(inst);
  const auto N = static_cast<std::size_t>(I.model(i).NN);
  const auto o = static_cast<std::size_t>(I.nodeOff[i]);
  for (int k = 0; k < 7; ++k) I.hSt[i * 8 + static_cast<std::size_t>(k)] = rec[k];
  I.hSt[i * 8 + 7] = 0;
  for (std::size_t n = 0; n < N; ++n) {
    I.hVol[o + n] = rec[10 + n];
    I.hLevel[o + n] = rec[10 + N + n];
    I.hCx[o + n] = rec[10 + 2 * N + n];
    I.hCy[o + n] = rec[10 + 3 * N + n];
    I.hCz[o + n] = rec[10 + 4 * N + n];
  }
}

void Batch::set_connection_enabled(std::int32_t inst, std::int32_t c, bool en) {
  if (I_->uploaded) throw std::logic_error("Batch: set after run");
  check_inst(opt_, inst);
  if (c < 0 || c >= I_->model(static_cast<std::size_t>(inst)).NC) throw std::out_of_range("Batch: connection " + std::to_string(c));
  I_->hEn[static_cast<std::size_t>(I_->connOff[static_cast<std::size_t>(inst)] + c)] = en ? 1 : 0;
}

void Batch::set_connection_area(std::int32_t inst, std::int32_t c, double area) {
  if (I_->uploaded) throw std::logic_error("Batch: set after run");
  check_inst(opt_, inst);
  if (c < 0 || c >= I_->model(static_cast<std::size_t>(inst)).NC) throw std::out_of_range("Batch: connection " + std::to_string(c));
  I_->hArea[static_cast<std::size_t>(I_->connOff[static_cast<std::size_t>(inst)] + c)] = area;
}

void Batch::set_connection_activation(std::int32_t inst, std::int32_t c, double tOn) {
  if (I_->uploaded) throw std::logic_error("Batch: set after run");
  check_inst(opt_, inst);
  if (c < 0 || c >= I_->model(static_cast<std::size_t>(inst)).NC) throw std::out_of_range("Batch: connection " + std::to_string(c));
  I_->hTOn[static_cast<std::size_t>(I_->connOff[static_cast<std::size_t>(inst)] + c)] = tOn;
}

void Batch::set_connection_areas(std::int32_t first, std::int32_t count, std::int32_t nConns, const std::int32_t* conns,
                                 const double* areas) {
  Impl& I = *I_;
  if (I.uploaded) throw std::logic_error("Batch: set after run");
  if (count < 0 || nConns < 0) throw std::invalid_argument("Batch: negative instance or connection count");
  if (count == 0 || nConns == 0) return;
  if (conns == nullptr || areas == nullptr) throw std::invalid_argument("Batch: null connection or area array");
  if (first < 0 || static_cast<std::int64_t>(first) + count > opt_.count)
    throw std::out_of_range("Batch: instances " + std::to_string(first) + " .. " +
                            std::to_string(static_cast<std::int64_t>(first) + count - 1) + " out of range");
  for (std::int32_t i = first; i < first + count; ++i) {
    const std::int32_t nc = I.model(static_cast<std::size_t>(i)).NC;
    for (std::int32_t j = 0; j < nConns; ++j)
      if (conns[j] < 0 || conns[j] >= nc) throw std::out_of_range("Batch: connection " + std::to_string(conns[j]));
  }
  for (std::int32_t i = 0; i < count; ++i) {
    const auto o = static_cast<std::size_t>(I.connOff[static_cast<std::size_t>(first + i)]);
    const double* row = areas + static_cast<std::size_t>(i) * static_cast<std::size_t>(nConns);
    for (std::int32_t j = 0; j < nConns; ++j) I.hArea[o + static_cast<std::size_t>(conns[j])] = row[j];
  }
}

void Batch::set_claim_order(const std::int32_t* order, std::int32_t n) {
  Impl& I = *I_;
  if (I.uploaded) throw std::logic_error("Batch: set after run");
  if (n != opt_.count) throw std::invalid_argument("Batch: a claim order lists every instance once (" + std::to_string(opt_.count) + ")");
  if (order == nullptr) throw std::invalid_argument("Batch: null claim order");
  std::vector<char> seen(static_cast<std::size_t>(n), 0);
  for (std::int32_t k = 0; k < n; ++k) {
    if (order[k] < 0 || order[k] >= n || seen[static_cast<std::size_t>(order[k])])
      throw std::invalid_argument("Batch: the claim order is not a permutation of the instances (position " + std::to_string(k) + ")");
    seen[static_cast<std::size_t>(order[k])] = 1;
  }
  I.hOrder0.assign(order, order + n);
}

void Batch::apply_sweep(const Sweep& sw, std::int32_t first) {
  Impl& I = *I_;
  if (I.uploaded) throw std::logic_error("Batch: set after run");
  if (I.fleet()) throw std::invalid_argument("Batch: a sweep applies to a batch of one model");
  if (first < 0 || static_cast<std::size_t>(first) + static_cast<std::size_t>(opt_.count) > sw.instances.size())
    throw std::invalid_argument("Batch: sweep instances " + std::to_string(first) + " .. " + std::to_string(first + opt_.count - 1) +
                                " do not exist (the sweep has " + std::to_string(sw.instances.size()) + ")");
  for (std::int32_t i = 0; i < opt_.count; ++i) {
    const auto o = static_cast<std::size_t>(I.connOff[static_cast<std::size_t>(i)]);
    apply_instance(sw.instances[static_cast<std::size_t>(first + i)], I.m0().sim, I.hEn.data() + o, I.hArea.data() + o, I.hTOn.data() + o);
  }
  sweepFirst_ = first;
}

void Batch::upload() {
  Impl& I = *I_;
  if (I.uploaded) throw std::logic_error("Batch: run twice");
  I.uploaded = true;
  check(cudaSetDevice(opt_.device), "cudaSetDevice");
  cudaStream_t s = I.stream;
  const auto count = static_cast<std::size_t>(opt_.count);
  I.en.upload(I.hEn, s); I.area.upload(I.hArea, s); I.tOn.upload(I.hTOn, s);
  I.st.upload(I.hSt, s);
  I.vol.upload(I.hVol, s); I.level.upload(I.hLevel, s); I.cx.upload(I.hCx, s); I.cy.upload(I.hCy, s); I.cz.upload(I.hCz, s);
  // outputs and bookkeeping start at zero / -1 on the device
  I.out.alloc(count * 7); check(cudaMemsetAsync(I.out.get(), 0, I.out.bytes(), s), "memset");
  const auto events = static_cast<std::size_t>(I.evOff[count]);
  I.evT.alloc(events); I.evId.alloc(events); I.evKind.alloc(events);
  I.evCount.alloc(count); check(cudaMemsetAsync(I.evCount.get(), 0, I.evCount.bytes(), s), "memset");
  I.overT.upload(std::vector<double>(std::max<std::size_t>(static_cast<std::size_t>(I.monOff[count]), 1), -1), s);
  I.markT.upload(std::vector<double>(std::max<std::size_t>(static_cast<std::size_t>(I.markOff[count]), 1), -1), s);
  I.foundered.alloc(count); check(cudaMemsetAsync(I.foundered.get(), 0, I.foundered.bytes(), s), "memset");
  I.founderT.upload(std::vector<double>(count, -1), s);
  I.steps.alloc(count); check(cudaMemsetAsync(I.steps.get(), 0, I.steps.bytes(), s), "memset");
  I.stop.alloc(count); check(cudaMemsetAsync(I.stop.get(), 0, I.stop.bytes(), s), "memset");
  I.finalRec.alloc(count * 7);
  const auto traced = static_cast<std::size_t>(opt_.tracedInstances);
  const auto rec = static_cast<std::size_t>(I.recSize);
  I.denseRec.alloc(std::max<std::size_t>(traced * static_cast<std::size_t>(opt_.denseSteps + 1) * rec, 1));
  I.sampleRec.alloc(std::max<std::size_t>(traced * static_cast<std::size_t>(I.maxSamples) * rec, 1));
  I.denseCount.alloc(std::max<std::size_t>(traced, 1)); check(cudaMemsetAsync(I.denseCount.get(), 0, I.denseCount.bytes(), s), "memset");
  I.sampleCount.alloc(std::max<std::size_t>(traced, 1)); check(cudaMemsetAsync(I.sampleCount.get(), 0, I.sampleCount.bytes(), s), "memset");
  I.nextSample.upload(std::vector<double>(std::max<std::size_t>(traced, 1), opt_.sampleEvery), s);
  I.curveRec.alloc(std::max<std::size_t>(count * static_cast<std::size_t>(I.curveMax) * 7, 1));
  I.curveCount.alloc(count); check(cudaMemsetAsync(I.curveCount.get(), 0, I.curveCount.bytes(), s), "memset");
  I.nextCurve.alloc(count); check(cudaMemsetAsync(I.nextCurve.get(), 0, I.nextCurve.bytes(), s), "memset");
  I.queue.alloc(1);
  I.remaining.alloc(1);
  I.phaseSteps.alloc(cfg_.phases.size());
  I.orderList.alloc(count); I.order.alloc(count); I.orderCount.alloc(1);
  if (!I.hOrder0.empty()) {
    I.order0.upload(I.hOrder0, s);
    I.order0Count.upload(std::vector<std::int32_t>{opt_.count}, s);
  }
  I.error.alloc(1); check(cudaMemsetAsync(I.error.get(), 0, I.error.bytes(), s), "memset");
}

namespace {
// Above this bound on the unfinished instances a phase claims by index: ranking them takes O(n^2) compares.
constexpr int kMaxOrderedInstances = 16384;
}  // namespace

bool ordered_phase(const BatchOptions& opt, const LaunchConfig& cfg, std::size_t k) {
  // a phase after the first of a run that goes to the end in one graph; the phase before hands over once at most
  // yieldBelow instances remain, which bounds the instances to rank
  if (k == 0 || k >= cfg.phases.size() || opt.claimByIndex || opt.stepsPerLaunch > 0) return false;
  const int bound = cfg.phases[k - 1].yieldBelow;
  return bound > 0 && bound <= kMaxOrderedInstances;
}

std::vector<PlanStep> run_plan(const BatchOptions& opt, const LaunchConfig& cfg) {
  std::vector<PlanStep> plan{{PlanStep::kStartRun, -1}};
  for (std::size_t k = 0; k < cfg.phases.size(); ++k) {
    if (ordered_phase(opt, cfg, k)) plan.push_back({PlanStep::kClaimOrder, static_cast<int>(k)});
    plan.push_back({PlanStep::kPhase, static_cast<int>(k)});
  }
  return plan;
}

int kernels_per_run(const BatchOptions& opt, const LaunchConfig& cfg) {
  int n = 0;
  for (const PlanStep& p : run_plan(opt, cfg)) n += p.kind == PlanStep::kClaimOrder ? 2 : 1;
  return n;
}

float Batch::launch() {
  Impl& I = *I_;
  if (!I.uploaded) throw std::logic_error("Batch: launch before upload");
  if (I.launched) throw std::logic_error("Batch: launch twice");
  I.launched = true;
  check(cudaSetDevice(opt_.device), "cudaSetDevice");
  cudaStream_t s = I.stream;
  const long long maxSteps = opt_.stepsPerLaunch > 0 ? opt_.stepsPerLaunch : LLONG_MAX;
  const std::size_t nph = cfg_.phases.size();
  I.lastPhaseMs.assign(nph, 0.0f);
  if (opt_.stepsPerLaunch <= 0) {
    // the whole run in one CUDA graph: the counters, then per phase the queue reset, the kernel and its end event
    std::vector<DevBatch> dbs(nph);
    for (std::size_t k = 0; k < nph; ++k) {
      dbs[k] = I.devBatch(opt_, maxSteps, k == 0 ? 1 : 0);
      dbs[k].yieldBelow = cfg_.phases[k].yieldBelow;
      dbs[k].stageColumns = cfg_.phases[k].stageColumns ? 1 : 0;
      dbs[k].phaseSteps = I.phaseSteps.get() + k;
      if (ordered_phase(opt_, cfg_, k)) { dbs[k].order = I.order.get(); dbs[k].orderCount = I.orderCount.get(); }
      if (k == 0 && !I.hOrder0.empty()) { dbs[k].order = I.order0.get(); dbs[k].orderCount = I.order0Count.get(); }
    }
    const auto* kb = reinterpret_cast<const unsigned char*>(dbs.data());
    std::vector<unsigned char> key(kb, kb + dbs.size() * sizeof(DevBatch));
    if (!I.graphExec || key != I.graphKey) {
      if (I.graphExec) { cudaGraphExecDestroy(I.graphExec); I.graphExec = nullptr; }
      if (I.graph) { cudaGraphDestroy(I.graph); I.graph = nullptr; }
      check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
      cudaError_t e = cudaSuccess;
      for (const PlanStep& step : run_plan(opt_, cfg_)) {
        if (e != cudaSuccess) break;
        if (step.kind == PlanStep::kStartRun) {
          e = launch_start_run(I.remaining.get(), opt_.count, I.phaseSteps.get(), static_cast<int>(nph), s);
          // the phase events are recorded by the graph itself (external records), so the phases stay timed one by one
          if (e == cudaSuccess) e = cudaEventRecordWithFlags(I.phaseEv[0], s, cudaEventRecordExternal);
          continue;
        }
        const auto k = static_cast<std::size_t>(step.phase);
        if (step.kind == PlanStep::kClaimOrder) {
          // the previous phase's hand-over bound (k >= 1 here: ordered_phase never holds for the first phase)
          e = launch_order_unfinished(I.stop.get(), I.steps.get(), opt_.count, cfg_.phases[k - 1].yieldBelow, I.orderList.get(),
                                      I.order.get(), I.orderCount.get(), s);
          continue;
        }
        const PhaseConfig& p = cfg_.phases[k];
        e = cudaMemsetAsync(I.queue.get(), 0, sizeof(std::int32_t), s);
        if (e == cudaSuccess) e = launch_batch_kernel(opt_.mixedPrecision, p.teamWarps, I.m0().dm, dbs[k], p.layout, p.blocks, p.teamsPerBlock, s);
        if (e == cudaSuccess) e = cudaEventRecordWithFlags(I.phaseEv[k + 1], s, cudaEventRecordExternal);
      }
      cudaGraph_t g = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(s, &g);  // always ends the capture, also after a failed step
      if (e == cudaSuccess) e = ec;
      if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        check(e, "capturing the run's launches");
      }
      I.graph = g;
      check(cudaGraphInstantiate(&I.graphExec, I.graph, 0), "cudaGraphInstantiate");
      I.graphKey = std::move(key);
    }
    check(cudaEventRecord(I.ev0, s), "cudaEventRecord");
    check(cudaGraphLaunch(I.graphExec, s), "cudaGraphLaunch");
    check(cudaEventRecord(I.ev1, s), "cudaEventRecord");
    check(cudaEventSynchronize(I.ev1), "kernel execution");
    for (std::size_t k = 0; k < nph; ++k) {
      float pm = 0;
      check(cudaEventElapsedTime(&pm, I.phaseEv[k], I.phaseEv[k + 1]), "cudaEventElapsedTime");
      I.lastPhaseMs[k] = pm;
    }
    float ms = 0;
    check(cudaEventElapsedTime(&ms, I.ev0, I.ev1), "cudaEventElapsedTime");
    I.phaseSteps.download(I.lastPhaseSteps, s);
    I.error.download(I.lastHealth, s);
    check(cudaStreamSynchronize(s), "copy to host");
    return ms;
  }
  // bounded launches: every round launches the phases again until no instance runs
  check(launch_start_run(I.remaining.get(), opt_.count, I.phaseSteps.get(), static_cast<int>(nph), s), "kernel launch");
  check(cudaEventRecord(I.ev0, s), "cudaEventRecord");
  int first = 1;
  for (;;) {
    // phase by phase: the instances a phase paused (and any it did not reach) resume in the next phase's larger teams
    check(cudaEventRecord(I.phaseEv[0], s), "cudaEventRecord");
    for (std::size_t k = 0; k < nph; ++k) {
      const PhaseConfig& p = cfg_.phases[k];
      check(cudaMemsetAsync(I.queue.get(), 0, sizeof(std::int32_t), s), "memset");
      DevBatch db = I.devBatch(opt_, maxSteps, first);
      db.yieldBelow = p.yieldBelow;
      db.stageColumns = p.stageColumns ? 1 : 0;
      db.phaseSteps = I.phaseSteps.get() + k;
      if (k == 0 && !I.hOrder0.empty()) { db.order = I.order0.get(); db.orderCount = I.order0Count.get(); }
      check(launch_batch_kernel(opt_.mixedPrecision, p.teamWarps, I.m0().dm, db, p.layout, p.blocks, p.teamsPerBlock, s), "kernel launch");
      check(cudaEventRecord(I.phaseEv[k + 1], s), "cudaEventRecord");
      first = 0;
    }
    check(cudaEventSynchronize(I.phaseEv[nph]), "kernel execution");
    for (std::size_t k = 0; k < nph; ++k) {
      float pm = 0;
      check(cudaEventElapsedTime(&pm, I.phaseEv[k], I.phaseEv[k + 1]), "cudaEventElapsedTime");
      I.lastPhaseMs[k] += pm;
    }
    std::vector<std::int32_t> stops;
    I.stop.download(stops, s);
    check(cudaStreamSynchronize(s), "kernel execution");
    bool active = false;
    for (const std::int32_t v : stops) if (v == kRunning) { active = true; break; }
    if (!active) break;
  }
  check(cudaEventRecord(I.ev1, s), "cudaEventRecord");
  check(cudaEventSynchronize(I.ev1), "kernel execution");
  float ms = 0;
  check(cudaEventElapsedTime(&ms, I.ev0, I.ev1), "cudaEventElapsedTime");
  I.phaseSteps.download(I.lastPhaseSteps, s);
  I.error.download(I.lastHealth, s);
  check(cudaStreamSynchronize(s), "copy to host");
  return ms;
}

void Batch::download() {
  Impl& I = *I_;
  if (!I.launched) throw std::logic_error("Batch: download before launch");
  cudaStream_t s = I.stream;
  auto& r = I.r;
  I.st.download(r.st, s); I.out.download(r.out, s);
  I.vol.download(r.vol, s); I.level.download(r.level, s); I.cx.download(r.cx, s); I.cy.download(r.cy, s); I.cz.download(r.cz, s);
  I.evT.download(r.evT, s); I.evId.download(r.evId, s); I.evKind.download(r.evKind, s); I.evCount.download(r.evCount, s);
  I.foundered.download(r.foundered, s); I.founderT.download(r.founderT, s); I.steps.download(r.steps, s); I.stop.download(r.stop, s);
  I.finalRec.download(r.finalRec, s);
  if (opt_.curveEvery > 0) { I.curveRec.download(r.curveRec, s); I.curveCount.download(r.curveCount, s); }
  if (opt_.tracedInstances > 0) {
    I.denseRec.download(r.denseRec, s); I.sampleRec.download(r.sampleRec, s);
    I.denseCount.download(r.denseCount, s); I.sampleCount.download(r.sampleCount, s);
  }
  check(cudaStreamSynchronize(s), "copy to host");
  I.downloaded = true;
}

void Batch::reset() {
  Impl& I = *I_;
  if (I.uploaded && !I.launched) throw std::logic_error("Batch: reset between upload and launch");
  check(cudaStreamSynchronize(I.stream), "stream sync");
  I.uploaded = false;
  I.launched = false;
}

double Batch::run() {
  const auto t0 = std::chrono::steady_clock::now();
  upload();
  launch();
  download();
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

std::size_t Batch::upload_bytes() const {
  const Impl& I = *I_;
  return I.hEn.size() + sizeof(double) * (I.hArea.size() + I.hTOn.size() + I.hSt.size() + I.hVol.size() + I.hLevel.size() + I.hCx.size() +
                                          I.hCy.size() + I.hCz.size());
}

std::size_t Batch::download_bytes() const {
  const Impl& I = *I_;
  std::size_t b = I.st.bytes() + I.out.bytes() + I.vol.bytes() + I.level.bytes() + I.cx.bytes() + I.cy.bytes() + I.cz.bytes() + I.evT.bytes() +
                  I.evId.bytes() + I.evKind.bytes() + I.evCount.bytes() + I.foundered.bytes() + I.founderT.bytes() + I.steps.bytes() +
                  I.stop.bytes() + I.finalRec.bytes();
  if (opt_.curveEvery > 0) b += I.curveRec.bytes() + I.curveCount.bytes();
  if (opt_.tracedInstances > 0) b += I.denseRec.bytes() + I.sampleRec.bytes() + I.denseCount.bytes() + I.sampleCount.bytes();
  return b;
}

std::vector<Batch::PhaseStats> Batch::phase_stats() const {
  const Impl& I = *I_;
  std::vector<PhaseStats> v;
  for (std::size_t k = 0; k < I.lastPhaseMs.size() && k < I.lastPhaseSteps.size(); ++k)
    v.push_back({cfg_.phases[k].teamWarps, I.lastPhaseMs[k], static_cast<std::int64_t>(I.lastPhaseSteps[k])});
  return v;
}

std::int32_t Batch::health() const { return I_->lastHealth.empty() ? 0 : I_->lastHealth.front(); }

std::int64_t Batch::total_steps() const {
  if (!I_->downloaded) throw std::logic_error("Batch: results before run");
  std::int64_t t = 0;
  for (const long long s : I_->r.steps) t += s;
  return t;
}

Batch::Summary Batch::summary(std::int32_t inst) const {
  const Impl& I = *I_;
  if (!I.downloaded) throw std::logic_error("Batch: result before run");
  check_inst(opt_, inst);
  const auto i = static_cast<std::size_t>(inst);
  Summary s{};
  s.foundered = I.r.foundered[i] != 0;
  s.founderT = I.r.founderT[i];
  s.tEnd = I.r.st[i * 8];
  s.steps = I.r.steps[i];
  s.stop = I.r.stop[i];
  for (int k = 0; k < 7; ++k) s.outputs[k] = I.r.out[i * 7 + static_cast<std::size_t>(k)];
  return s;
}

void Batch::state(std::int32_t inst, double* rec) const {
  const Impl& I = *I_;
  if (!I.downloaded) throw std::logic_error("Batch: result before run");
  check_inst(opt_, inst);
  const auto i = static_cast<std::size_t>(inst);
  const auto N = static_cast<std::size_t>(I.model(i).NN);
  const auto o = static_cast<std::size_t>(I.nodeOff[i]);
  for (int k = 0; k < 7; ++k) rec[k] = I.r.st[i * 8 + static_cast<std::size_t>(k)];
  rec[7] = I.r.out[i * 7]; rec[8] = I.r.out[i * 7 + 1]; rec[9] = I.r.out[i * 7 + 2];
  for (std::size_t n = 0; n < N; ++n) {
    rec[10 + n] = I.r.vol[o + n];
    rec[10 + N + n] = I.r.level[o + n];
    rec[10 + 2 * N + n] = I.r.cx[o + n];
    rec[10 + 3 * N + n] = I.r.cy[o + n];
    rec[10 + 4 * N + n] = I.r.cz[o + n];
  }
}

std::vector<int> Batch::event_kinds(std::int32_t inst) const {
  const Impl& I = *I_;
  const auto i = static_cast<std::size_t>(inst);
  std::vector<int> out;
  for (std::int32_t k = 0; k < I.r.evCount[i]; ++k) out.push_back(I.r.evKind[static_cast<std::size_t>(I.evOff[i] + k)]);
  return out;
}

std::vector<int> Batch::event_ids(std::int32_t inst) const {
  const Impl& I = *I_;
  const auto i = static_cast<std::size_t>(inst);
  std::vector<int> out;
  for (std::int32_t k = 0; k < I.r.evCount[i]; ++k) out.push_back(I.r.evId[static_cast<std::size_t>(I.evOff[i] + k)]);
  return out;
}

const CompiledSim& Batch::sim() const { return I_->m0().sim; }

void Batch::run_noalloc(const NoAllocRun& run, cudaStream_t stream) const {
  const Impl& I = *I_;
  if (I.fleet()) throw std::invalid_argument("run_noalloc: a batch of one model only");
  if (run.count < 1) throw std::invalid_argument("run_noalloc: count must be at least 1");
  const std::size_t need = noalloc_scratch_bytes(I.m0().dm, run.count), cap = noalloc_scratch_capacity();
  if (need > cap) {
    // the largest count that fits: the scratch grows with the count, so bisect on [0, run.count)
    std::int32_t lo = 0, hi = run.count;
    while (hi - lo > 1) {
      const std::int32_t mid = lo + (hi - lo) / 2;
      (noalloc_scratch_bytes(I.m0().dm, mid) <= cap ? lo : hi) = mid;
    }
    throw std::invalid_argument("run_noalloc: " + std::to_string(run.count) + " instances of this model need " + std::to_string(need) +
                                " bytes of scratch; the fixed scratch array holds " + std::to_string(cap) + " (at most " +
                                std::to_string(lo) + " instances)");
  }
  if (!run.en || !run.area || !run.tOn || !run.state || !run.vol || !run.level || !run.cx || !run.cy || !run.cz || !run.finalRec || !run.steps ||
      !run.stop)
    throw std::invalid_argument("run_noalloc: a device pointer is NULL");
  check(cudaSetDevice(opt_.device), "cudaSetDevice");
  NoAllocRun r = run;
  r.tMax = opt_.tMax;
  r.rule = opt_.rule;
  r.stopWhenStable = opt_.stopWhenStable;
  // one launch, teams sized so that about 16 warps per SM carry the instances
  const int sms = I.info.multiprocessors;
  const int fit = std::max(1, (sms * 16) / r.count);
  r.teamWarps = fit >= 8 ? 8 : fit >= 4 ? 4 : fit >= 2 ? 2 : 1;
  const SlotLayout L = I.layout_for(r.teamWarps);
  const int maxTeams = std::min(static_cast<int>(I.info.sharedPerBlockOptIn / L.bytes), kMaxWarpsPerBlock / r.teamWarps);
  r.teamsPerBlock = std::max(1, std::min(maxTeams, (r.count + sms - 1) / sms));
  const std::size_t smem = static_cast<std::size_t>(r.teamsPerBlock) * L.bytes;
  check(configure_batch_kernel(opt_.mixedPrecision, r.teamWarps, smem), "cudaFuncSetAttribute");
  int perSM = 0;
  check(batch_kernel_occupancy(opt_.mixedPrecision, r.teamWarps, r.teamsPerBlock, smem, &perSM), "occupancy");
  if (perSM < 1) throw std::runtime_error("run_noalloc: the kernel cannot be resident");
  r.blocks = std::min((r.count + r.teamsPerBlock - 1) / r.teamsPerBlock, perSM * sms);
  check(run_batch_noalloc(opt_.mixedPrecision, I.m0().dm, L, r, stream), "kernel launch");
}

std::vector<EventRecord> Batch::events(std::int32_t inst) const {
  const Impl& I = *I_;
  if (!I.downloaded) throw std::logic_error("Batch: result before run");
  check_inst(opt_, inst);
  const auto i = static_cast<std::size_t>(inst);
  std::vector<EventRecord> out;
  const CompiledSim& sim = I.model(i).sim;
  for (std::int32_t k = 0; k < I.r.evCount[i]; ++k) {
    const auto j = static_cast<std::size_t>(I.evOff[i] + k);
    const std::int32_t id = I.r.evId[j];
    switch (I.r.evKind[j]) {
      case 0: out.push_back(EventRecord{I.r.evT[j], sim.monitorId[static_cast<std::size_t>(id)], sim.monitorLabel[static_cast<std::size_t>(id)]}); break;
      case 1: out.push_back(EventRecord{I.r.evT[j], sim.markId[static_cast<std::size_t>(id)], sim.markLabel[static_cast<std::size_t>(id)]}); break;
      default: out.push_back(EventRecord{I.r.evT[j], "founder", "Foundered"}); break;
    }
  }
  return out;
}

CurveRecord Batch::final_readouts(std::int32_t inst) const {
  const Impl& I = *I_;
  if (!I.downloaded) throw std::logic_error("Batch: result before run");
  check_inst(opt_, inst);
  const double* p = &I.r.finalRec[static_cast<std::size_t>(inst) * 7];
  return CurveRecord{p[0], p[1], p[2], p[3], p[4], p[5], p[6]};
}

std::vector<CurveRecord> Batch::curve(std::int32_t inst) const {
  const Impl& I = *I_;
  if (!I.downloaded) throw std::logic_error("Batch: curve before run");
  if (opt_.curveEvery <= 0) throw std::logic_error("Batch: curves were not recorded (curveEvery is 0)");
  check_inst(opt_, inst);
  const auto i = static_cast<std::size_t>(inst);
  std::vector<CurveRecord> out;
  for (std::int32_t k = 0; k < I.r.curveCount[i]; ++k) {
    const double* p = &I.r.curveRec[(i * static_cast<std::size_t>(I.curveMax) + static_cast<std::size_t>(k)) * 7];
    out.push_back(CurveRecord{p[0], p[1], p[2], p[3], p[4], p[5], p[6]});
  }
  out.push_back(final_readouts(inst));
  return out;
}

std::string Batch::engine_name() const { return "sinksim-b200 CUDA engine on " + I_->info.name; }

Trace Batch::trace(std::int32_t inst) const {
  const Impl& I = *I_;
  if (!I.downloaded) throw std::logic_error("Batch: trace before run");
  if (inst < 0 || inst >= opt_.tracedInstances) throw std::out_of_range("Batch: instance was not traced");
  const auto i = static_cast<std::size_t>(inst);
  Trace tr;
  tr.ship = I.m0().ship->id; tr.sim = I.m0().sim.id; tr.title = I.m0().sim.title;
  tr.producer = opt_.mixedPrecision ? "sinksim-b200 CUDA engine, numerics portable32" : "sinksim-b200 CUDA engine, numerics portable";
  tr.engine = "sinksim-b200 0.1.0 on " + I.info.name;
  tr.dt = I.m0().sim.dt; tr.nodes = I.m0().NN; tr.denseSteps = opt_.denseSteps; tr.sampleEvery = opt_.sampleEvery;
  const Summary s = summary(inst);
  tr.steps = s.steps; tr.tEnd = s.tEnd; tr.foundered = s.foundered; tr.founderT = s.founderT;
  for (const EventRecord& e : events(inst)) tr.events.push_back(TraceEvent{e.t, e.id, e.label});
  const auto rec = static_cast<std::size_t>(I.recSize);
  const std::size_t db = i * static_cast<std::size_t>(opt_.denseSteps + 1) * rec, sb = i * static_cast<std::size_t>(I.maxSamples) * rec;
  for (std::int32_t k = 0; k < I.r.denseCount[i]; ++k) tr.dense.push_record(&I.r.denseRec[db + static_cast<std::size_t>(k) * rec], I.m0().NN);
  for (std::int32_t k = 0; k < I.r.sampleCount[i]; ++k) tr.samples.push_record(&I.r.sampleRec[sb + static_cast<std::size_t>(k) * rec], I.m0().NN);
  return tr;
}

Results Batch::results(const Sweep* sw) const {
  const Impl& I = *I_;
  if (I.fleet()) throw std::logic_error("Batch: batch-results hold one model; read a fleet's instances one by one");
  Results r;
  r.ship = I.m0().ship->id;
  r.sim = I.m0().sim.id;
  r.numerics = opt_.mixedPrecision ? "portable32" : "portable";
  r.engine = engine_name();
  r.tMax = opt_.tMax;
  r.every = opt_.curveEvery;
  for (std::int32_t i = 0; i < opt_.count; ++i) {
    InstanceResult in;
    in.id = sw ? sw->instances[static_cast<std::size_t>(sweepFirst_ + i)].id : "instance" + std::to_string(i);
    const Summary s = summary(i);
    in.foundered = s.foundered; in.founderT = s.founderT; in.tEnd = s.tEnd; in.steps = s.steps;
    const CurveRecord f = final_readouts(i);
    in.fTrim = f.trim; in.fList = f.list; in.fWater = f.water; in.fInflow = f.inflow; in.fDraftF = f.dF; in.fDraftA = f.dA;
    in.events = events(i);
    if (opt_.curveEvery > 0) in.curve = curve(i);
    r.instances.push_back(std::move(in));
  }
  return r;
}

}  // namespace ssb
