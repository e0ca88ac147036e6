// The batch kernel: a persistent grid whose warps each run one simulation at a time. A warp takes the next
// instance index from a device work queue (one atomicAdd), loads that instance's state into its shared-memory
// slot and registers, steps it until it founders, reaches tMax, meets the optional retire rule or uses up the
// launch's step budget, stores the state back and takes the next instance. Instances of uneven run length thus
// retire and admit new ones without any host round trip; the reference instead launched one 256-thread block per
// instance in fixed-size chunks (engine/cuda/device_step.cuh:323-434, engine/cuda/batch.cu:287-302).
//
// There are no waits between warps: the only inter-warp operation is the queue's atomicAdd.
#include <cuda_runtime.h>

#include "batch_kernel.h"
#include "warp_step.cuh"

namespace ssb {

namespace {

__device__ __forceinline__ void write_record(double* rec, const SimRegs& R, const Slot& S, int nn, int lane) {
  if (lane == 0) {
    rec[0] = R.t; rec[1] = R.zO; rec[2] = R.pitch; rec[3] = R.roll; rec[4] = R.vz; rec[5] = R.wth; rec[6] = R.wph;
    rec[7] = R.inflow; rec[8] = R.Vb; rec[9] = R.hullTop;
  }
  double* p = rec + 10;
  for (int n = lane; n < nn; n += kLanes) {
    p[n] = S.vol[n];
    p[nn + n] = S.level[n];
    p[2 * nn + n] = S.cx[n];
    p[3 * nn + n] = S.cy[n];
    p[4 * nn + n] = S.cz[n];
  }
}

template <bool MIXED>
__device__ void run_instance(const DevModel& M, const DevBatch& B, Slot& S, int inst, int lane) {
  if (B.stop[inst] != kRunning) return;
  const std::size_t iN = static_cast<std::size_t>(inst) * M.nn;
  const std::size_t iC = static_cast<std::size_t>(inst) * M.nc;
  SimRegs R;
  {
    const double* st = B.st + static_cast<std::size_t>(inst) * 8;
    R.t = st[0]; R.zO = st[1]; R.pitch = st[2]; R.roll = st[3]; R.vz = st[4]; R.wth = st[5]; R.wph = st[6]; R.calm = st[7];
    const double* o = B.out + static_cast<std::size_t>(inst) * 7;
    R.inflow = o[0]; R.Vb = o[1]; R.hullTop = o[2]; R.mw = o[3]; R.bx = o[4]; R.by = o[5]; R.bz = o[6];
    R.foundered = B.foundered[inst];
    R.founderT = B.founderT[inst];
    R.evCount = B.evCount[inst];
  }
  InstPtrs I;
  I.en = B.en + iC; I.area = B.area + iC; I.tOn = B.tOn + iC;
  I.evT = B.evT + static_cast<std::size_t>(inst) * M.evCap;
  I.evId = B.evId + static_cast<std::size_t>(inst) * M.evCap;
  I.evKind = B.evKind + static_cast<std::size_t>(inst) * M.evCap;
  I.overT = B.overT + static_cast<std::size_t>(inst) * M.nmon;
  I.markT = B.markT + static_cast<std::size_t>(inst) * M.nmark;
  for (int n = lane; n < M.nn; n += kLanes) {
    S.vol[n] = B.vol[iN + n]; S.level[n] = B.level[iN + n];
    S.cx[n] = B.cx[iN + n]; S.cy[n] = B.cy[iN + n]; S.cz[n] = B.cz[iN + n];
    S.area[n] = 0; S.zmax[n] = 0; S.hEff[n] = 0; S.aEff[n] = 0; S.acc[n] = 0; S.deg[n] = 0;
  }
  for (int g = lane; g < M.ng; g += kLanes) S.merged[g] = 0;
  for (int c = lane; c < M.nc; c += kLanes) { S.dV[c] = 0; S.q[c] = 0; }
  __syncwarp();

  long long done = B.steps[inst];
  const bool traced = inst < B.traced;
  int denseCount = 0, sampleCount = 0, curveCount = 0;
  double nextSample = 0, nextCurve = 0;
  double* denseBase = nullptr;
  double* sampleBase = nullptr;
  if (traced) {
    denseBase = B.denseRec + static_cast<std::size_t>(inst) * (B.denseSteps + 1) * B.recSize;
    sampleBase = B.sampleRec + static_cast<std::size_t>(inst) * B.maxSamples * B.recSize;
    denseCount = B.denseCount[inst]; sampleCount = B.sampleCount[inst]; nextSample = B.nextSample[inst];
  }
  if (B.curveEvery > 0) { curveCount = B.curveCount[inst]; nextCurve = B.nextCurve[inst]; }

  if (B.firstLaunch && traced && done == 0) {
    // the initial record: buoyancy at the initial pose and no inflow (the reference's Simulation::record_trace)
    const Pose F0 = make_pose(M, R.zO, R.pitch, R.roll);
    const Buoy hb = buoyancy<MIXED>(M, F0, lane);
    R.inflow = 0; R.Vb = hb.V; R.hullTop = hb.top; R.bx = hb.x; R.by = hb.y; R.bz = hb.z;
    write_record(denseBase, R, S, M.nn, lane);
    write_record(sampleBase, R, S, M.nn, lane);
    denseCount = 1; sampleCount = 1; nextSample = B.sampleEvery;
  }

  int stop = kRunning;
  Pose F = make_pose(M, R.zO, R.pitch, R.roll);
  for (long long s = 0; s < B.maxSteps; ++s) {
    if (R.foundered || R.t >= B.tMax) break;
    if (B.curveEvery > 0 && R.t >= nextCurve && curveCount < B.curveMax) {
      double r7[7];
      readouts(M, R, S, r7);
      if (lane == 0) {
        double* rec = B.curveRec + (static_cast<std::size_t>(inst) * B.curveMax + curveCount) * 7;
        for (int k = 0; k < 7; ++k) rec[k] = r7[k];
      }
      ++curveCount;
      nextCurve += B.curveEvery;
    }
    warp_step<MIXED>(M, F, R, S, I, lane);
    ++done;
    F = make_pose(M, R.zO, R.pitch, R.roll);
    if (traced) {
      if (done <= B.denseSteps) write_record(denseBase + static_cast<std::size_t>(denseCount++) * B.recSize, R, S, M.nn, lane);
      if (R.t >= nextSample - 1e-9 && sampleCount < B.maxSamples) {
        write_record(sampleBase + static_cast<std::size_t>(sampleCount++) * B.recSize, R, S, M.nn, lane);
        nextSample += B.sampleEvery;
      }
    }
    if (B.rule.enabled) {
      const double zp = world_z(F, B.rule.xDeck, B.rule.yDeck, B.rule.zDeck);
      const double zs = world_z(F, B.rule.xDeck, -B.rule.yDeck, B.rule.zDeck);
      if (fabs(R.pitch) > B.rule.pitchLimit && (zp < 0 || zs < 0)) { stop = kSinkRule; break; }
      R.calm = fabs(R.wth) < B.rule.wthLimit ? R.calm + M.dt : 0;
      if (R.calm >= B.rule.settleTime) { stop = kSettleRule; break; }
    }
  }
  if (stop == kRunning) {
    if (R.foundered) stop = kFoundered;
    else if (R.t >= B.tMax) stop = kTimeLimit;
  }

  // store the instance
  __syncwarp();
  for (int n = lane; n < M.nn; n += kLanes) {
    B.vol[iN + n] = S.vol[n]; B.level[iN + n] = S.level[n];
    B.cx[iN + n] = S.cx[n]; B.cy[iN + n] = S.cy[n]; B.cz[iN + n] = S.cz[n];
  }
  if (lane == 0) {
    double* st = B.st + static_cast<std::size_t>(inst) * 8;
    st[0] = R.t; st[1] = R.zO; st[2] = R.pitch; st[3] = R.roll; st[4] = R.vz; st[5] = R.wth; st[6] = R.wph; st[7] = R.calm;
    double* o = B.out + static_cast<std::size_t>(inst) * 7;
    o[0] = R.inflow; o[1] = R.Vb; o[2] = R.hullTop; o[3] = R.mw; o[4] = R.bx; o[5] = R.by; o[6] = R.bz;
    B.foundered[inst] = R.foundered;
    B.founderT[inst] = R.founderT;
    B.evCount[inst] = R.evCount;
    B.steps[inst] = done;
    B.stop[inst] = stop;
    if (traced) { B.denseCount[inst] = denseCount; B.sampleCount[inst] = sampleCount; B.nextSample[inst] = nextSample; }
    if (B.curveEvery > 0) { B.curveCount[inst] = curveCount; B.nextCurve[inst] = nextCurve; }
  }
  if (stop != kRunning) {
    double r7[7];
    readouts(M, R, S, r7);
    if (lane == 0)
      for (int k = 0; k < 7; ++k) B.finalRec[static_cast<std::size_t>(inst) * 7 + k] = r7[k];
  }
  __syncwarp();
}

template <bool MIXED>
__global__ void __launch_bounds__(kMaxWarpsPerBlock * 32) run_batch(DevModel M, DevBatch B, SlotLayout L) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  Slot S = carve_slot(smem + static_cast<std::size_t>(warp) * L.bytes, L);
  for (;;) {
    int inst = 0;
    if (lane == 0) inst = atomicAdd(B.queue, 1);
    inst = __shfl_sync(kFull, inst, 0);
    if (inst >= B.count) return;
    run_instance<MIXED>(M, B, S, inst, lane);
  }
}

}  // namespace

cudaError_t configure_batch_kernel(bool mixed, std::size_t smemBytes) {
  if (mixed) return cudaFuncSetAttribute(run_batch<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smemBytes));
  return cudaFuncSetAttribute(run_batch<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smemBytes));
}

cudaError_t launch_batch_kernel(bool mixed, const DevModel& M, const DevBatch& B, const SlotLayout& L, int grid, int warpsPerBlock,
                                cudaStream_t stream) {
  const std::size_t smem = static_cast<std::size_t>(warpsPerBlock) * L.bytes;
  if (mixed) run_batch<true><<<grid, warpsPerBlock * 32, smem, stream>>>(M, B, L);
  else run_batch<false><<<grid, warpsPerBlock * 32, smem, stream>>>(M, B, L);
  return cudaGetLastError();
}

cudaError_t batch_kernel_occupancy(bool mixed, int warpsPerBlock, std::size_t smemBytes, int* blocksPerSM) {
  if (mixed) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocksPerSM, run_batch<true>, warpsPerBlock * 32, smemBytes);
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocksPerSM, run_batch<false>, warpsPerBlock * 32, smemBytes);
}

}  // namespace ssb
