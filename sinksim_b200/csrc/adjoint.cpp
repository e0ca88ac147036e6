#include "adjoint.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>

#include <cuda_runtime.h>

#include "adjoint_kernel.h"
#include "batch.h"
#include "model_dev.h"

namespace ssb {

struct AdjointBatch::Impl {
  std::unique_ptr<ModelDev> model;
  DeviceInfo info;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // host staging
  std::vector<std::uint8_t> hEn;
  std::vector<double> hArea, hTOn, hSt, hVol, hLevel, hCx, hCy, hCz, hTimes, hTrimT, hHeaveT;
  std::int32_t nsamples = 0;
  // device
  DevBuf<std::uint8_t> en;
  DevBuf<double> area, tOn, st, vol, level, cx, cy, cz, times, trimT, heaveT, trim, heave, J, grad, ckpt, sink;
  DevBuf<unsigned char> arena;
  DevBuf<long long> steps, phase, stepOff, recomputed;
  DevBuf<std::int32_t> recBytes;
  DevBuf<std::int32_t> error, queue, isink, order;
  std::vector<std::int32_t> hOrder;  // the caller's claim order (empty: by index)
  // results
  std::vector<double> rJ, rGrad, rTrim, rHeave;
  std::vector<long long> rSteps, rPhase, rRecomputed;
  std::vector<std::int32_t> rError;
  bool ran = false;
  std::size_t up = 0, down = 0;
  std::uint64_t tapeBudget = 0;   // bytes of the rings of all teams; 0: chosen at the first run
  std::size_t ringBytes = 0;      // per team, as chosen
  int ringTeams = 0;

  SlotLayout slot_for(int W) const {
    // the forward slot of a team of W warps, as the batch kernel lays it out for one model
    const ModelDev& m = *model;
    SlotLayout L{};
    std::uint32_t off = 0;
    const std::size_t nb = sizeof(double) * static_cast<std::size_t>(m.NN);
    L.vol = take(off, nb); L.level = take(off, nb); L.cx = take(off, nb); L.cy = take(off, nb); L.cz = take(off, nb);
    L.area = take(off, nb); L.zmax = take(off, nb); L.hEff = take(off, nb); L.aEff = take(off, nb); L.acc = take(off, nb);
    L.deg = take(off, sizeof(std::int32_t) * static_cast<std::size_t>(m.NN));
    L.dV = take(off, sizeof(double) * static_cast<std::size_t>(std::max(m.NC, 1)));
    L.q = take(off, sizeof(double) * static_cast<std::size_t>(std::max(m.NC, 1)));
    L.tmp = m.NC >= m.NN ? kSlotAliasDV : take(off, nb);
    L.passes = take(off, 7 * sizeof(double) * static_cast<std::size_t>(m.maxGroup) * static_cast<std::size_t>(W * kMaxLevelGroupsPerWarp));
    L.hydro = take(off, 8 * 5 * sizeof(double));
    L.misc = take(off, 4 * sizeof(std::int32_t));
    L.merged = take(off, static_cast<std::size_t>(std::max(m.NG, 1)));
    L.pose = take(off, sizeof(Pose));
    L.buoy = take(off, sizeof(Buoy));
    L.parked = take(off, sizeof(Parked));
    L.model = 0;
    L.bytes = off;
    return L;
  }
};

AdjointBatch::AdjointBatch(std::shared_ptr<const CompiledShip> ship, const CompiledSim& sim, const AdjointOptions& opt)
    : I_(new Impl), opt_(opt) {
  if (opt_.count < 1) throw std::invalid_argument("AdjointBatch: count must be at least 1");
  if (opt_.checkpointEvery < 1) throw std::invalid_argument("AdjointBatch: checkpointEvery must be at least 1");
  if (!(opt_.tMax > 0)) throw std::invalid_argument("AdjointBatch: tMax must be positive");
  if (opt_.teamWarps != 0 && opt_.teamWarps != 4 && opt_.teamWarps != 8 && opt_.teamWarps != 16)
    throw std::invalid_argument("AdjointBatch: teamWarps must be 4, 8 or 16");
  std::string why;
  if (!cuda_available(&why)) throw std::runtime_error("AdjointBatch: " + why);
  Impl& I = *I_;
  check(cudaSetDevice(opt_.device), "cudaSetDevice");
  I.info = device_info(opt_.device);
  check(cudaStreamCreateWithFlags(&I.stream, cudaStreamNonBlocking), "cudaStreamCreate");
  check(cudaEventCreate(&I.ev0), "cudaEventCreate");
  check(cudaEventCreate(&I.ev1), "cudaEventCreate");
  I.model = std::make_unique<ModelDev>(std::move(ship), sim);
  I.model->upload(I.stream);
  const ModelDev& m = *I.model;
  const auto count = static_cast<std::size_t>(opt_.count);
  const auto nc = static_cast<std::size_t>(m.NC), nn = static_cast<std::size_t>(m.NN);
  I.hEn.resize(count * nc); I.hArea.resize(count * nc); I.hTOn.resize(count * nc);
  I.hSt.resize(count * 7); I.hVol.resize(count * nn); I.hLevel.resize(count * nn); I.hCx.resize(count * nn); I.hCy.resize(count * nn);
  I.hCz.resize(count * nn);
  const CompiledSim& M = m.sim;
  for (std::size_t i = 0; i < count; ++i) {
    std::copy(M.cEn.begin(), M.cEn.end(), I.hEn.begin() + i * nc);
    std::copy(M.cArea.begin(), M.cArea.end(), I.hArea.begin() + i * nc);
    std::copy(M.cTOn.begin(), M.cTOn.end(), I.hTOn.begin() + i * nc);
    const double s0[7] = {M.t0, M.zO0, M.pitch0, M.roll0, M.vz0, M.wth0, M.wph0};
    std::copy(s0, s0 + 7, I.hSt.begin() + i * 7);
    std::copy(M.vol0.begin(), M.vol0.end(), I.hVol.begin() + i * nn);
    std::copy(M.level0.begin(), M.level0.end(), I.hLevel.begin() + i * nn);
    std::copy(M.cx0.begin(), M.cx0.end(), I.hCx.begin() + i * nn);
    std::copy(M.cy0.begin(), M.cy0.end(), I.hCy.begin() + i * nn);
    std::copy(M.cz0.begin(), M.cz0.end(), I.hCz.begin() + i * nn);
  }
  // team size: a whole 16-warp block per instance while the instances number at most two per SM, 8 warps beyond
  // (the liner's gradient workload on B200: 256 points 2.24 s per call in 16-warp teams against 2.40 s in 8-warp
  // teams; 512 points 4.68 s in 8-warp teams against 5.88 s in 16-warp and 6.18 s in 4-warp teams, measured before
  // the reverse's rework; the evaluator's claim order, longest runs first, in every case)
  teamWarps_ = opt_.teamWarps ? opt_.teamWarps : (opt_.count <= 2 * I.info.multiprocessors ? 16 : 8);
}

AdjointBatch::~AdjointBatch() {
  if (I_) {
    if (I_->stream) cudaStreamSynchronize(I_->stream);
    if (I_->ev0) cudaEventDestroy(I_->ev0);
    if (I_->ev1) cudaEventDestroy(I_->ev1);
    if (I_->stream) cudaStreamDestroy(I_->stream);
  }
}

std::int32_t AdjointBatch::connections() const { return I_->model->NC; }
std::int32_t AdjointBatch::nodes() const { return I_->model->NN; }

static void check_inst(std::int32_t count, std::int32_t inst) {
  if (inst < 0 || inst >= count) throw std::out_of_range("AdjointBatch: instance " + std::to_string(inst) + " out of range");
}

void AdjointBatch::set_connection_enabled(std::int32_t inst, std::int32_t c, bool en) {
  check_inst(opt_.count, inst);
  if (c < 0 || c >= I_->model->NC) throw std::out_of_range("AdjointBatch: connection " + std::to_string(c) + " out of range");
  I_->hEn[static_cast<std::size_t>(inst) * I_->model->NC + c] = en ? 1 : 0;
}

void AdjointBatch::set_connection_areas(std::int32_t first, std::int32_t count, std::int32_t nConns, const std::int32_t* conns, const double* areas) {
  const std::int32_t NC = I_->model->NC;
  if (count < 0 || nConns < 0 || first < 0 || first + count > opt_.count) throw std::out_of_range("AdjointBatch: instance block out of range");
  for (std::int32_t j = 0; j < nConns; ++j)
    if (conns[j] < 0 || conns[j] >= NC) throw std::out_of_range("AdjointBatch: connection " + std::to_string(conns[j]) + " out of range");
  for (std::int32_t i = 0; i < count; ++i)
    for (std::int32_t j = 0; j < nConns; ++j)
      I_->hArea[static_cast<std::size_t>(first + i) * NC + conns[j]] = areas[static_cast<std::size_t>(i) * nConns + j];
}

void AdjointBatch::set_objective(std::int32_t n, const double* times, const double* trim, const double* heave) {
  if (n < 1) throw std::invalid_argument("AdjointBatch: the objective needs at least one sample time");
  for (std::int32_t k = 1; k < n; ++k)
    if (!(times[k] >= times[k - 1])) throw std::invalid_argument("AdjointBatch: sample times must ascend");
  Impl& I = *I_;
  I.nsamples = n;
  I.hTimes.assign(times, times + n);
  const auto total = static_cast<std::size_t>(opt_.count) * n;
  I.hTrimT.assign(trim, trim + total);
  I.hHeaveT.assign(heave, heave + total);
}

float AdjointBatch::run() {
  Impl& I = *I_;
  if (I.nsamples < 1) throw std::logic_error("AdjointBatch: set_objective before run");
  check(cudaSetDevice(opt_.device), "cudaSetDevice");
  cudaStream_t s = I.stream;
  const ModelDev& m = *I.model;
  const int W = teamWarps_;
  const SlotLayout SL = I.slot_for(W);
  AdjLayout AL = adjoint_layout(m.NN, m.NC, m.NG, I.nsamples, W);
  std::size_t smem = static_cast<std::size_t>(SL.bytes) + AL.bytes;
  if (smem > I.info.sharedPerBlockOptIn)
    throw std::runtime_error("AdjointBatch: a team needs " + std::to_string(smem) + " bytes of shared memory, the device allows " +
                             std::to_string(I.info.sharedPerBlockOptIn));
  check(configure_adjoint_kernel(W, smem), "cudaFuncSetAttribute");
  int perSM = 0;
  check(adjoint_occupancy(W, smem, &perSM), "occupancy");
  if (perSM < 1) throw std::runtime_error("AdjointBatch: the adjoint kernel cannot be resident");
  // a buffer for the next step's record (copied while the current step is reversed) when it costs no team per SM
  bool stageRecords = false;
  {
    const AdjLayout AR = adjoint_layout(m.NN, m.NC, m.NG, I.nsamples, W, true);
    const std::size_t smemR = static_cast<std::size_t>(SL.bytes) + AR.bytes;
    int perSMR = 0;
    if (smemR <= I.info.sharedPerBlockOptIn) {
      check(configure_adjoint_kernel(W, smemR), "cudaFuncSetAttribute");
      check(adjoint_occupancy(W, smemR, &perSMR), "occupancy");
    }
    if (perSMR >= perSM) {
      AL = AR;
      smem = smemR;
      stageRecords = true;
    } else {
      check(configure_adjoint_kernel(W, smem), "cudaFuncSetAttribute");
    }
  }
  teams_ = std::min(opt_.count, perSM * I.info.multiprocessors);
  const auto count = static_cast<std::size_t>(opt_.count);
  const auto NS = static_cast<std::size_t>(I.nsamples);
  const double dt = m.sim.dt;
  const long long maxSteps = static_cast<long long>(std::ceil((opt_.tMax - m.sim.t0) / dt)) + 2;
  const int K = opt_.checkpointEvery;
  const int maxCkpt = static_cast<int>(maxSteps / K) + 2;
  const std::size_t recSize = 7 + 5 * static_cast<std::size_t>(m.NN);
  const std::size_t tapeBytes = adjoint_tape_bytes(m.NN, m.NG);
  // inputs
  I.en.upload(I.hEn, s); I.area.upload(I.hArea, s); I.tOn.upload(I.hTOn, s);
  I.st.upload(I.hSt, s); I.vol.upload(I.hVol, s); I.level.upload(I.hLevel, s);
  I.cx.upload(I.hCx, s); I.cy.upload(I.hCy, s); I.cz.upload(I.hCz, s);
  I.times.upload(I.hTimes, s); I.trimT.upload(I.hTrimT, s); I.heaveT.upload(I.hHeaveT, s);
  I.up = I.hEn.size() + sizeof(double) * (I.hArea.size() + I.hTOn.size() + I.hSt.size() + I.hVol.size() * 5 + I.hTimes.size() +
                                          I.hTrimT.size() + I.hHeaveT.size());
  // outputs and per-team memory
  I.trim.alloc(count * NS); I.heave.alloc(count * NS); I.J.alloc(count); I.grad.alloc(count * static_cast<std::size_t>(m.NC));
  I.steps.alloc(count); I.phase.alloc(3 * count); I.recomputed.alloc(count);
  I.error.alloc(count); check(cudaMemsetAsync(I.error.get(), 0, I.error.bytes(), s), "memset");
  I.queue.alloc(1); check(cudaMemsetAsync(I.queue.get(), 0, I.queue.bytes(), s), "memset");
  I.ckpt.alloc(static_cast<std::size_t>(teams_) * maxCkpt * recSize);
  I.stepOff.alloc(static_cast<std::size_t>(teams_) * (static_cast<std::size_t>(maxSteps) + 1));
  I.recBytes.alloc(static_cast<std::size_t>(teams_) * (static_cast<std::size_t>(maxSteps) + 1));
  // the rings: at least K records of the largest size per team (one segment); up to a whole run of them when memory
  // allows. Unless the caller set a budget: a whole run of records with two passes per node (nodes take about 1.2 on
  // average), within half the device memory free at the first run; the ring is kept for later runs.
  const std::size_t minRing = static_cast<std::size_t>(K) * tapeBytes;
  if (I.ringBytes == 0 || I.ringTeams != teams_) {
    std::size_t perTeam = 0;
    if (I.tapeBudget != 0) {
      perTeam = static_cast<std::size_t>(I.tapeBudget / static_cast<std::uint64_t>(teams_));
    } else {
      std::size_t freeB = 0, totalB = 0;
      check(cudaMemGetInfo(&freeB, &totalB), "cudaMemGetInfo");
      const std::size_t usual = (static_cast<std::size_t>(maxSteps) + 1) * adjoint_record_bytes(m.NN, m.NG, 2 * m.NN);
      perTeam = std::min(usual, (freeB + I.arena.bytes()) / 2 / static_cast<std::size_t>(teams_));
    }
    I.ringBytes = std::max(minRing, perTeam) & ~static_cast<std::size_t>(15);
    I.ringTeams = teams_;
  }
  I.arena.alloc(static_cast<std::size_t>(teams_) * I.ringBytes);
  I.sink.alloc(static_cast<std::size_t>(teams_) * (m.evCap + m.nmon + m.nmark + 1));
  I.isink.alloc(static_cast<std::size_t>(teams_) * (m.evCap + 1));
  AdjRun R{};
  R.count = opt_.count;
  R.en = I.en.get(); R.area = I.area.get(); R.tOn = I.tOn.get();
  R.st0 = I.st.get(); R.vol0 = I.vol.get(); R.level0 = I.level.get(); R.cx0 = I.cx.get(); R.cy0 = I.cy.get(); R.cz0 = I.cz.get();
  R.tMax = opt_.tMax;
  R.maxSteps = maxSteps;
  R.nsamples = I.nsamples;
  R.sampleT = I.times.get(); R.trimT = I.trimT.get(); R.heaveT = I.heaveT.get();
  R.trim = I.trim.get(); R.heave = I.heave.get(); R.J = I.J.get(); R.grad = I.grad.get(); R.steps = I.steps.get();
  R.error = I.error.get(); R.queue = I.queue.get();
  if (!I.hOrder.empty()) I.order.upload(I.hOrder, s);
  R.order = I.hOrder.empty() ? nullptr : I.order.get();
  R.K = K; R.maxCkpt = maxCkpt; R.ckpt = I.ckpt.get();
  R.arena = I.arena.get(); R.arenaBytes = I.ringBytes; R.stepOff = I.stepOff.get(); R.recBytes = I.recBytes.get();
  R.stageRecords = stageRecords ? 1 : 0;
  R.tapeForward = I.ringBytes > minRing ? 1 : 0; R.sink = I.sink.get(); R.isink = I.isink.get();
  R.phaseNs = I.phase.get();
  R.recomputed = I.recomputed.get();
  check(cudaEventRecord(I.ev0, s), "cudaEventRecord");
  check(launch_adjoint_kernel(W, m.dm, R, SL, AL, teams_, s), "adjoint kernel launch");
  check(cudaEventRecord(I.ev1, s), "cudaEventRecord");
  check(cudaEventSynchronize(I.ev1), "adjoint kernel execution");
  float ms = 0;
  check(cudaEventElapsedTime(&ms, I.ev0, I.ev1), "cudaEventElapsedTime");
  I.J.download(I.rJ, s); I.grad.download(I.rGrad, s); I.trim.download(I.rTrim, s); I.heave.download(I.rHeave, s);
  I.steps.download(I.rSteps, s); I.error.download(I.rError, s); I.phase.download(I.rPhase, s); I.recomputed.download(I.rRecomputed, s);
  check(cudaStreamSynchronize(s), "copy to host");
  I.down = I.J.bytes() + I.grad.bytes() + I.trim.bytes() + I.heave.bytes() + I.steps.bytes() + I.error.bytes() + I.phase.bytes() + I.recomputed.bytes();
  I.ran = true;
  return ms;
}

double AdjointBatch::objective(std::int32_t inst) const {
  if (!I_->ran) throw std::logic_error("AdjointBatch: results before run");
  check_inst(opt_.count, inst);
  return I_->rJ[static_cast<std::size_t>(inst)];
}

const double* AdjointBatch::gradient(std::int32_t inst) const {
  if (!I_->ran) throw std::logic_error("AdjointBatch: results before run");
  check_inst(opt_.count, inst);
  return &I_->rGrad[static_cast<std::size_t>(inst) * I_->model->NC];
}

const double* AdjointBatch::samples_trim(std::int32_t inst) const {
  if (!I_->ran) throw std::logic_error("AdjointBatch: results before run");
  check_inst(opt_.count, inst);
  return &I_->rTrim[static_cast<std::size_t>(inst) * I_->nsamples];
}

const double* AdjointBatch::samples_heave(std::int32_t inst) const {
  if (!I_->ran) throw std::logic_error("AdjointBatch: results before run");
  check_inst(opt_.count, inst);
  return &I_->rHeave[static_cast<std::size_t>(inst) * I_->nsamples];
}

std::int64_t AdjointBatch::steps(std::int32_t inst) const {
  if (!I_->ran) throw std::logic_error("AdjointBatch: results before run");
  check_inst(opt_.count, inst);
  return I_->rSteps[static_cast<std::size_t>(inst)];
}

std::int32_t AdjointBatch::error(std::int32_t inst) const {
  if (!I_->ran) throw std::logic_error("AdjointBatch: results before run");
  check_inst(opt_.count, inst);
  return I_->rError[static_cast<std::size_t>(inst)];
}

const long long* AdjointBatch::phase_ns(std::int32_t inst) const {
  if (!I_->ran) throw std::logic_error("AdjointBatch: results before run");
  check_inst(opt_.count, inst);
  return &I_->rPhase[3 * static_cast<std::size_t>(inst)];
}

std::int64_t AdjointBatch::recomputed_steps(std::int32_t inst) const {
  if (!I_->ran) throw std::logic_error("AdjointBatch: results before run");
  check_inst(opt_.count, inst);
  return I_->rRecomputed[static_cast<std::size_t>(inst)];
}

void AdjointBatch::set_claim_order(const std::int32_t* order, std::int32_t n) {
  if (order == nullptr || n == 0) {
    I_->hOrder.clear();
    return;
  }
  if (n != opt_.count) throw std::invalid_argument("AdjointBatch: a claim order lists every instance once (" + std::to_string(opt_.count) + ")");
  std::vector<char> seen(static_cast<std::size_t>(n), 0);
  for (std::int32_t k = 0; k < n; ++k) {
    if (order[k] < 0 || order[k] >= n || seen[static_cast<std::size_t>(order[k])])
      throw std::invalid_argument("AdjointBatch: the claim order is not a permutation of the instances (position " + std::to_string(k) + ")");
    seen[static_cast<std::size_t>(order[k])] = 1;
  }
  I_->hOrder.assign(order, order + n);
}

void AdjointBatch::set_tape_budget(std::uint64_t bytes) {
  I_->tapeBudget = bytes;
  I_->ringBytes = 0;
}

std::size_t AdjointBatch::ring_bytes() const { return I_->ringBytes; }

std::size_t AdjointBatch::upload_bytes() const { return I_->up; }
std::size_t AdjointBatch::download_bytes() const { return I_->down; }

}  // namespace ssb
