// The batch kernel: a persistent grid whose teams (W warps each) run one simulation at a time. A team takes the
// next instance index from a device work queue (one atomicAdd), loads that instance into its shared-memory slot and
// registers, steps it until it founders, reaches tMax, meets the optional retire rule or uses up the launch's step
// budget, stores it back and takes the next one. Instances of uneven run length thus retire and admit new ones
// without a host round trip; the reference instead launched one 256-thread block per instance in fixed-size chunks
// (engine/cuda/device_step.cuh:323-434, engine/cuda/batch.cu:287-302).
//
// Adaptive team size: a launch of single-warp teams gives the most simulations per SM, but a lone simulation then
// steps slowly. When at most `yieldBelow` instances remain unfinished, the teams pause their instances and stop
// claiming; the next launch resumes them with larger teams, whose steps are several times shorter.
//
// Teams never wait on each other: the only inter-team operations are the queue's atomicAdd and the count of
// unfinished instances (atomicSub when one stops, a plain load every 64 steps).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <mutex>

#include "batch_kernel.h"
#include "warp_step.cuh"

namespace ssb {

namespace {

constexpr int kYieldCheckEvery = 64;
// try_wait rounds a block waits for its column table to arrive before it reads the table from global memory instead
constexpr int kStageWaitLimit = 1 << 20;

// Copies the column table (xy, lh, area: ncol entries each) into the block's shared memory at dst, laid out as
// staged_columns<T>: thread 0 starts one bulk asynchronous copy per array (the part that is a whole number of 16-byte
// units; the rest, under 16 bytes, by plain copies) completing on an mbarrier after the table, and every thread waits
// for the barrier's phase with a bounded number of try_wait rounds. Returns dst, or null when the wait ran out (the
// health bit kHealthStageTimeout is set and the block reads the table from global memory). Every thread of the block
// calls it once, before the teams diverge. The sources are cudaMalloc'd arrays, so 256-byte aligned.
template <class T>
__device__ const unsigned char* stage_column_table(const typename Vec2<T>::type* xy, const typename Vec2<T>::type* lh, const T* area, int ncol,
                                                   unsigned char* dst, std::int32_t* error) {
  using V2 = typename Vec2<T>::type;
  const StagedColumns<T> c = staged_columns<T>(ncol);
  const auto bar = static_cast<unsigned>(__cvta_generic_to_shared(dst + c.bytes));
  const std::size_t n = static_cast<std::size_t>(ncol);
  const std::size_t size[3] = {n * sizeof(V2), n * sizeof(V2), n * sizeof(T)};
  const unsigned char* src[3] = {reinterpret_cast<const unsigned char*>(xy), reinterpret_cast<const unsigned char*>(lh),
                                 reinterpret_cast<const unsigned char*>(area)};
  const std::size_t off[3] = {c.xy, c.lh, c.area};
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned total = 0;
    for (int k = 0; k < 3; ++k) total += static_cast<unsigned>(size[k] & ~static_cast<std::size_t>(15));
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(total) : "memory");
    for (int k = 0; k < 3; ++k) {
      const auto bulk = static_cast<unsigned>(size[k] & ~static_cast<std::size_t>(15));
      const auto to = static_cast<unsigned>(__cvta_generic_to_shared(dst + off[k]));
      if (bulk)
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(to), "l"(src[k]),
                     "r"(bulk), "r"(bar)
                     : "memory");
      for (std::size_t b = bulk; b < size[k]; ++b) dst[off[k] + b] = src[k][b];
    }
  }
  bool done = false;
  for (int it = 0; it < kStageWaitLimit && !done; ++it) {
    unsigned ready;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ready)
        : "r"(bar)
        : "memory");
    done = ready != 0;
  }
  if (!__syncthreads_and(done ? 1 : 0)) {
    if (threadIdx.x == 0) atomicOr(error, kHealthStageTimeout);
    return nullptr;
  }
  return dst;
}

template <int W>
__device__ __forceinline__ void write_record(double* rec, const SimRegs& R, const Slot& S, int nn, const Team<W>& T) {
  if (T.warp != 0) return;
  const int lane = T.lane;
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

// Runs one instance; returns true when the team paused it (yield) and must stop claiming.
template <bool MIXED, int W, bool FLEET>
__device__ bool run_instance(const DevModel& M, const DevBatch& B, Slot& S, int inst, const Team<W>& T) {
  constexpr int kStride = 32 * W;
  if (B.stop[inst] != kRunning) return false;
  const int rank = T.rank;
  const InstPtrs<FLEET> I{M, B, inst};
  const std::size_t iN = I.perNode();
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
  for (int n = rank; n < M.nn; n += kStride) {
    S.vol[n] = B.vol[iN + n]; S.level[n] = B.level[iN + n];
    S.cx[n] = B.cx[iN + n]; S.cy[n] = B.cy[iN + n]; S.cz[n] = B.cz[iN + n];
    S.area[n] = 0; S.zmax[n] = 0; S.hEff[n] = 0; S.aEff[n] = 0; S.acc[n] = 0; S.deg[n] = 0;
  }
  for (int g = rank; g < M.ng; g += kStride) S.merged[g] = 0;
  for (int c = rank; c < M.nc; c += kStride) { S.dV[c] = 0; S.q[c] = 0; }
  T.sync();

  long long done = B.steps[inst];
  const long long done0 = done;
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

  if (traced && done == 0 && denseCount == 0) {
    // the initial record: buoyancy at the initial pose and no inflow (the reference's Simulation::record_trace)
    const Pose F0 = make_pose(M, R.zO, R.pitch, R.roll);
    const Buoy hb = buoyancy<MIXED, W>(M, F0, T, S.hydro, S.cols);
    R.inflow = 0; R.Vb = hb.V; R.hullTop = hb.top; R.bx = hb.x; R.by = hb.y; R.bz = hb.z;
    write_record(denseBase, R, S, M.nn, T);
    write_record(sampleBase, R, S, M.nn, T);
    denseCount = 1; sampleCount = 1; nextSample = B.sampleEvery;
    T.sync();
  }

  int stop = kRunning;
  bool paused = false;
  // every thread of the team stores the same pose; no thread reads the previous one after the step's last barrier
  Pose& F = *S.pose;
  F = make_pose(M, R.zO, R.pitch, R.roll);
  for (long long s = 0; s < B.maxSteps; ++s) {
    if (R.foundered || R.t >= B.tMax) break;
    if (B.yieldBelow > 0 && s > 0 && (s % kYieldCheckEvery) == 0) {
      if (T.leader()) S.misc[1] = *reinterpret_cast<volatile int*>(B.remaining) <= B.yieldBelow ? 1 : 0;
      T.sync();
      const bool y = S.misc[1] != 0;
      T.sync();
      if (y) { paused = true; break; }
    }
    if (B.curveEvery > 0 && R.t >= nextCurve && curveCount < B.curveMax) {
      if (T.warp == 0) {
        double r7[7];
        readouts(M, R, S, r7);
        if (T.lane == 0) {
          double* rec = B.curveRec + (static_cast<std::size_t>(inst) * B.curveMax + curveCount) * 7;
          for (int k = 0; k < 7; ++k) rec[k] = r7[k];
        }
      }
      ++curveCount;
      nextCurve += B.curveEvery;
    }
    team_step<MIXED, W>(M, F, R, S, I, T);
    ++done;
    F = make_pose(M, R.zO, R.pitch, R.roll);
    if (traced) {
      if (done <= B.denseSteps) write_record(denseBase + static_cast<std::size_t>(denseCount++) * B.recSize, R, S, M.nn, T);
      if (R.t >= nextSample - 1e-9 && sampleCount < B.maxSamples) {
        write_record(sampleBase + static_cast<std::size_t>(sampleCount++) * B.recSize, R, S, M.nn, T);
        nextSample += B.sampleEvery;
      }
    }
    if (B.stopWhenStable && R.t > 1800) {
      R.calm = (fabs(R.inflow) < 0.02 && fabs(R.wth) < 1e-5 && fabs(R.vz) < 1e-3) ? R.calm + M.dt : 0;
      if (R.calm > 1200) { stop = kStable; break; }
    }
    if (B.rule.enabled) {
      const double zp = world_z(F, B.rule.xDeck, B.rule.yDeck, B.rule.zDeck);
      const double zs = world_z(F, B.rule.xDeck, -B.rule.yDeck, B.rule.zDeck);
      if (fabs(R.pitch) > B.rule.pitchLimit && (zp < 0 || zs < 0)) { stop = kSinkRule; break; }
      R.calm = fabs(R.wth) < B.rule.wthLimit ? R.calm + M.dt : 0;
      if (R.calm >= B.rule.settleTime) { stop = kSettleRule; break; }
    }
  }
  if (stop == kRunning && !paused) {
    if (R.foundered) stop = kFoundered;
    else if (R.t >= B.tMax) stop = kTimeLimit;
  }

  // store the instance
  T.sync();
  for (int n = rank; n < M.nn; n += kStride) {
    B.vol[iN + n] = S.vol[n]; B.level[iN + n] = S.level[n];
    B.cx[iN + n] = S.cx[n]; B.cy[iN + n] = S.cy[n]; B.cz[iN + n] = S.cz[n];
  }
  if (T.leader()) {
    double* st = B.st + static_cast<std::size_t>(inst) * 8;
    st[0] = R.t; st[1] = R.zO; st[2] = R.pitch; st[3] = R.roll; st[4] = R.vz; st[5] = R.wth; st[6] = R.wph; st[7] = R.calm;
    double* o = B.out + static_cast<std::size_t>(inst) * 7;
    o[0] = R.inflow; o[1] = R.Vb; o[2] = R.hullTop; o[3] = R.mw; o[4] = R.bx; o[5] = R.by; o[6] = R.bz;
    B.foundered[inst] = R.foundered;
    B.founderT[inst] = R.founderT;
    B.evCount[inst] = R.evCount;  // the leader is lane 0 of warp 0, which keeps the event log
    B.steps[inst] = done;
    B.stop[inst] = stop;
    if (!(isfinite(R.zO) && isfinite(R.pitch) && isfinite(R.roll) && isfinite(R.vz) && isfinite(R.wth) && isfinite(R.wph)))
      atomicOr(B.error, kHealthNonFinite);
    if (traced) { B.denseCount[inst] = denseCount; B.sampleCount[inst] = sampleCount; B.nextSample[inst] = nextSample; }
    if (B.curveEvery > 0) { B.curveCount[inst] = curveCount; B.nextCurve[inst] = nextCurve; }
    if (stop != kRunning) atomicSub(B.remaining, 1);
    if (B.phaseSteps) atomicAdd(B.phaseSteps, static_cast<unsigned long long>(done - done0));
  }
  if (stop != kRunning && T.warp == 0) {
    double r7[7];
    readouts(M, R, S, r7);
    if (T.lane == 0)
      for (int k = 0; k < 7; ++k) B.finalRec[static_cast<std::size_t>(inst) * 7 + k] = r7[k];
  }
  T.sync();
  return paused;
}

// The persistent batch kernel: teams claim instances from the work queue until it runs dry (or the phase yields). In a
// fleet (FLEET), a team first copies its instance's model description into its slot and steps the instance with it.
template <bool MIXED, int W, bool FLEET>
__global__ void __launch_bounds__(kMaxWarpsPerBlock * 32, kMinBlocksPerSM) run_batch(DevModel M, DevBatch B, SlotLayout L) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int warpInBlock = threadIdx.x >> 5;
  const int team = warpInBlock / W;
  Team<W> T;
  T.warp = warpInBlock % W;
  T.lane = threadIdx.x & 31;
  T.rank = T.warp * 32 + T.lane;
  T.bar = team + 1;
  unsigned char* const slot = smem + static_cast<std::size_t>(team) * L.bytes;
  Slot S = carve_slot(slot, L);
  if constexpr (!FLEET) {
    if (B.stageColumns) {
      // the column table after the block's slots (one copy per block for the whole launch)
      unsigned char* const table = smem + static_cast<std::size_t>(blockDim.x / (32 * W)) * L.bytes;
      if constexpr (MIXED) S.cols = stage_column_table<float>(M.colXYf, M.colLHf, M.colAf, M.ncol, table, B.error);
      else S.cols = stage_column_table<double>(M.colXY, M.colLH, M.colA, M.ncol, table, B.error);
    }
  }
  for (;;) {
    if (T.leader()) {
      const int q = atomicAdd(B.queue, 1);
      S.misc[0] = B.order == nullptr ? q : (q < *B.orderCount ? B.order[q] : B.count);
      S.misc[2] = W * (32 / kLevelLanes<MIXED>);  // the level solve's group counter for the first step (team_step resets it)
    }
    T.sync();
    const int inst = S.misc[0];
    T.sync();
    if (inst >= B.count) return;
    if constexpr (FLEET) {
      static_assert(sizeof(DevModel) % sizeof(unsigned) == 0, "the model description is copied in 32-bit words");
      DevModel* const own = reinterpret_cast<DevModel*>(slot + L.model);
      const unsigned* src = reinterpret_cast<const unsigned*>(B.models + B.model[inst]);
      unsigned* dst = reinterpret_cast<unsigned*>(own);
      for (int k = T.rank; k < static_cast<int>(sizeof(DevModel) / sizeof(unsigned)); k += 32 * W) dst[k] = src[k];
      T.sync();
      // run_instance ends with a team barrier, so no thread still reads this copy when the next claim overwrites it
      if (run_instance<MIXED, W, true>(*own, B, S, inst, T)) return;
    } else {
      if (run_instance<MIXED, W, false>(M, B, S, inst, T)) return;
    }
  }
}

template <bool MIXED, bool FLEET>
cudaError_t set_smem(int W, std::size_t bytes) {
  const int b = static_cast<int>(bytes);
  switch (W) {
    case 1: return cudaFuncSetAttribute(run_batch<MIXED, 1, FLEET>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    case 2: return cudaFuncSetAttribute(run_batch<MIXED, 2, FLEET>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    case 4: return cudaFuncSetAttribute(run_batch<MIXED, 4, FLEET>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    case 8: return cudaFuncSetAttribute(run_batch<MIXED, 8, FLEET>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    case 16: return cudaFuncSetAttribute(run_batch<MIXED, 16, FLEET>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  }
  return cudaErrorInvalidValue;
}

template <bool MIXED, bool FLEET>
cudaError_t occupancy(int W, int threads, std::size_t bytes, int* perSM) {
  switch (W) {
    case 1: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(perSM, run_batch<MIXED, 1, FLEET>, threads, bytes);
    case 2: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(perSM, run_batch<MIXED, 2, FLEET>, threads, bytes);
    case 4: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(perSM, run_batch<MIXED, 4, FLEET>, threads, bytes);
    case 8: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(perSM, run_batch<MIXED, 8, FLEET>, threads, bytes);
    case 16: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(perSM, run_batch<MIXED, 16, FLEET>, threads, bytes);
  }
  return cudaErrorInvalidValue;
}

template <bool MIXED, bool FLEET>
void launch(int W, const DevModel& M, const DevBatch& B, const SlotLayout& L, int grid, int threads, std::size_t smem, cudaStream_t s) {
  switch (W) {
    case 1: run_batch<MIXED, 1, FLEET><<<grid, threads, smem, s>>>(M, B, L); break;
    case 2: run_batch<MIXED, 2, FLEET><<<grid, threads, smem, s>>>(M, B, L); break;
    case 4: run_batch<MIXED, 4, FLEET><<<grid, threads, smem, s>>>(M, B, L); break;
    case 8: run_batch<MIXED, 8, FLEET><<<grid, threads, smem, s>>>(M, B, L); break;
    case 16: run_batch<MIXED, 16, FLEET><<<grid, threads, smem, s>>>(M, B, L); break;
  }
}

}  // namespace

bool valid_team_size(int W) { return W == 1 || W == 2 || W == 4 || W == 8 || W == 16; }

std::size_t column_stage_bytes(bool mixed, int ncol) {
  // the table, then its 8-byte mbarrier (kept at a 16-byte boundary)
  return (mixed ? staged_columns<float>(ncol).bytes : staged_columns<double>(ncol).bytes) + 16;
}

cudaError_t configure_batch_kernel(bool mixed, int teamWarps, std::size_t smemBytes, bool fleet) {
  if (!valid_team_size(teamWarps)) return cudaErrorInvalidValue;
  if (fleet) return mixed ? set_smem<true, true>(teamWarps, smemBytes) : set_smem<false, true>(teamWarps, smemBytes);
  return mixed ? set_smem<true, false>(teamWarps, smemBytes) : set_smem<false, false>(teamWarps, smemBytes);
}

cudaError_t launch_batch_kernel(bool mixed, int teamWarps, const DevModel& M, const DevBatch& B, const SlotLayout& L, int grid,
                                int teamsPerBlock, cudaStream_t stream) {
  if (!valid_team_size(teamWarps) || teamsPerBlock * teamWarps > kMaxWarpsPerBlock) return cudaErrorInvalidValue;
  const bool fleet = B.models != nullptr;
  const std::size_t smem = static_cast<std::size_t>(teamsPerBlock) * L.bytes + (B.stageColumns && !fleet ? column_stage_bytes(mixed, M.ncol) : 0);
  const int threads = teamsPerBlock * teamWarps * 32;
  if (fleet) {
    if (mixed) launch<true, true>(teamWarps, M, B, L, grid, threads, smem, stream);
    else launch<false, true>(teamWarps, M, B, L, grid, threads, smem, stream);
  } else {
    if (mixed) launch<true, false>(teamWarps, M, B, L, grid, threads, smem, stream);
    else launch<false, false>(teamWarps, M, B, L, grid, threads, smem, stream);
  }
  return cudaGetLastError();
}

namespace {
__global__ void start_run(std::int32_t* remaining, std::int32_t count, unsigned long long* phaseSteps, int phases) {
  if (threadIdx.x == 0) *remaining = count;
  for (int k = static_cast<int>(threadIdx.x); k < phases; k += blockDim.x) phaseSteps[k] = 0;
}
}  // namespace

cudaError_t launch_start_run(std::int32_t* remaining, std::int32_t count, unsigned long long* phaseSteps, int phases, cudaStream_t stream) {
  start_run<<<1, 32, 0, stream>>>(remaining, count, phaseSteps, phases);
  return cudaGetLastError();
}

// Claim order of a launch phase after the first. The phase before paused its instances; the one with the most work
// left should get a larger team first, or it waits behind others for a free one and ends last. The work left is not
// known, but a run's length is bounded (tMax, and in practice the founder/settle times), so the fewer steps an
// instance has done, the more it has left: the order is by steps done, ascending, ties by index.
namespace {
constexpr int kOrderThreads = 256;

__global__ void compact_unfinished(const std::int32_t* stop, std::int32_t count, std::int32_t* list, std::int32_t* n) {
  for (std::int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    if (stop[i] == kRunning) list[atomicAdd(n, 1)] = i;
}

// order[rank of (steps[i], i) among the listed instances] = i: ranks of distinct keys, so a permutation of 0 .. n-1
// whatever order the compaction listed them in.
__global__ void __launch_bounds__(kOrderThreads) rank_unfinished(const long long* steps, const std::int32_t* list, const std::int32_t* n,
                                                                 std::int32_t* order) {
  __shared__ long long keyS[kOrderThreads];
  __shared__ std::int32_t keyI[kOrderThreads];
  const std::int32_t R = *n;
  for (std::int32_t base = blockIdx.x * kOrderThreads; base < R; base += gridDim.x * kOrderThreads) {
    const std::int32_t k = base + static_cast<std::int32_t>(threadIdx.x);
    const bool mine = k < R;
    const std::int32_t me = mine ? list[k] : 0;
    const long long ms = mine ? steps[me] : 0;
    std::int32_t rank = 0;
    for (std::int32_t t0 = 0; t0 < R; t0 += kOrderThreads) {
      __syncthreads();
      const std::int32_t m = t0 + static_cast<std::int32_t>(threadIdx.x);
      if (m < R) {
        const std::int32_t j = list[m];
        keyI[threadIdx.x] = j;
        keyS[threadIdx.x] = steps[j];
      }
      __syncthreads();
      const std::int32_t lim = min(kOrderThreads, R - t0);
      if (mine)
        for (std::int32_t j = 0; j < lim; ++j) rank += (keyS[j] < ms || (keyS[j] == ms && keyI[j] < me)) ? 1 : 0;
    }
    if (mine) order[rank] = me;
  }
}
}  // namespace

cudaError_t launch_order_unfinished(const std::int32_t* stop, const long long* steps, std::int32_t count, std::int32_t bound,
                                    std::int32_t* list, std::int32_t* order, std::int32_t* n, cudaStream_t stream) {
  if (count < 1 || bound < 1) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(n, 0, sizeof(std::int32_t), stream);
  if (e != cudaSuccess) return e;
  const int compactBlocks = static_cast<int>(std::min<std::int64_t>((static_cast<std::int64_t>(count) + 255) / 256, 1024));
  compact_unfinished<<<compactBlocks, 256, 0, stream>>>(stop, count, list, n);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const int rankBlocks = static_cast<int>(std::min<std::int64_t>((static_cast<std::int64_t>(std::min(bound, count)) + kOrderThreads - 1) / kOrderThreads, 1024));
  rank_unfinished<<<rankBlocks, kOrderThreads, 0, stream>>>(steps, list, n, order);
  return cudaGetLastError();
}

cudaError_t batch_kernel_occupancy(bool mixed, int teamWarps, int teamsPerBlock, std::size_t smemBytes, int* blocksPerSM, bool fleet) {
  if (!valid_team_size(teamWarps)) return cudaErrorInvalidValue;
  const int threads = teamsPerBlock * teamWarps * 32;
  if (fleet) return mixed ? occupancy<true, true>(teamWarps, threads, smemBytes, blocksPerSM) : occupancy<false, true>(teamWarps, threads, smemBytes, blocksPerSM);
  return mixed ? occupancy<true, false>(teamWarps, threads, smemBytes, blocksPerSM) : occupancy<false, false>(teamWarps, threads, smemBytes, blocksPerSM);
}

// ----------------------------------------------------------------------------- the batch run without device allocation
// Some callers cannot call cudaMalloc when they run a batch: a host application that owns every device allocation
// through its own pool (a calibration or control loop embedded in a larger program), or code that must not allocate
// once it is running. For them the batch kernel's scratch, the memory it needs beyond the caller's inputs and outputs
// (the work-queue head, the count of unfinished instances, and each instance's outputs, event log, overflow and mark
// times), lives in this fixed array instead of in buffers the engine allocates. Every GPU that loads the library
// holds it until the process exits. All calls share it and it keeps the last call's contents, so each call clears
// what must start at zero; two calls that overlap on the GPU (on different streams) would race on it.

namespace {

constexpr std::size_t kNoAllocScratchBytes = std::size_t(4) << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void* g_scratch_address[kMaxDevices] = {};

// The device address of g_noalloc_scratch on the current device. The array's name in host code is a host-side stand-in,
// not a device address, so the first call on a device looks the address up (cudaGetSymbolAddress, with that device
// current). Later calls look it up again and replace the cached value if it moved: the query is cheap and allocates
// nothing, and a cudaDeviceReset between calls reloads the module at a possibly different address. The mutex keeps host
// threads that call at the same time from racing on the cache.
cudaError_t scratch_address(int device, void** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  g_scratch_address[device] = p;
  *out = p;
  return cudaSuccess;
}

// The per-instance fields the batch kernel expects to find set before its first launch.
__global__ void clear_noalloc_scratch(DevBatch B, int nmon, int nmark) {
  const std::int32_t stride = gridDim.x * blockDim.x;
  for (std::int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < B.count; i += stride) {
    for (int k = 0; k < 7; ++k) B.out[static_cast<std::size_t>(i) * 7 + k] = 0;
    B.evCount[i] = 0;
    B.foundered[i] = 0;
    B.founderT[i] = -1;
    B.steps[i] = 0;
    B.stop[i] = kRunning;
    for (int m = 0; m < nmon; ++m) B.overT[static_cast<std::size_t>(i) * nmon + m] = -1;
    for (int m = 0; m < nmark; ++m) B.markT[static_cast<std::size_t>(i) * nmark + m] = -1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *B.queue = 0;
    *B.remaining = B.count;
    *B.error = 0;
  }
}

std::size_t align256(std::size_t x) { return (x + 255) & ~static_cast<std::size_t>(255); }

}  // namespace

std::size_t noalloc_scratch_capacity() { return kNoAllocScratchBytes; }

std::size_t noalloc_scratch_bytes(const DevModel& M, int count) {
  const auto c = static_cast<std::size_t>(count);
  std::size_t b = align256(3 * sizeof(std::int32_t));                         // queue, remaining, error
  b += align256(c * 7 * sizeof(double));                                        // outputs
  b += 2 * align256(c * sizeof(std::int32_t)) + align256(c * sizeof(double));   // evCount, foundered, founderT
  b += align256(c * M.evCap * sizeof(double)) + 2 * align256(c * M.evCap * sizeof(std::int32_t));  // event log
  b += align256(c * std::max(M.nmon, 1) * sizeof(double)) + align256(c * std::max(M.nmark, 1) * sizeof(double));
  return b;
}

cudaError_t run_batch_noalloc(bool mixed, const DevModel& M, const SlotLayout& L, const NoAllocRun& r, cudaStream_t stream) {
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  if (noalloc_scratch_bytes(M, r.count) > kNoAllocScratchBytes) return cudaErrorMemoryAllocation;
  void* address = nullptr;
  e = scratch_address(device, &address);
  if (e != cudaSuccess) return e;
  auto* base = static_cast<unsigned char*>(address);
  std::size_t off = 0;
  auto carve = [&](std::size_t bytes) { unsigned char* p = base + off; off += align256(bytes); return p; };
  const auto c = static_cast<std::size_t>(r.count);
  DevBatch B{};
  B.count = r.count;
  B.queue = reinterpret_cast<std::int32_t*>(carve(3 * sizeof(std::int32_t)));
  B.remaining = B.queue + 1;
  B.error = B.queue + 2;
  B.out = reinterpret_cast<double*>(carve(c * 7 * sizeof(double)));
  B.evCount = reinterpret_cast<std::int32_t*>(carve(c * sizeof(std::int32_t)));
  B.foundered = reinterpret_cast<std::int32_t*>(carve(c * sizeof(std::int32_t)));
  B.founderT = reinterpret_cast<double*>(carve(c * sizeof(double)));
  B.evT = reinterpret_cast<double*>(carve(c * M.evCap * sizeof(double)));
  B.evId = reinterpret_cast<std::int32_t*>(carve(c * M.evCap * sizeof(std::int32_t)));
  B.evKind = reinterpret_cast<std::int32_t*>(carve(c * M.evCap * sizeof(std::int32_t)));
  B.overT = reinterpret_cast<double*>(carve(c * std::max(M.nmon, 1) * sizeof(double)));
  B.markT = reinterpret_cast<double*>(carve(c * std::max(M.nmark, 1) * sizeof(double)));
  // the caller's inputs and outputs
  B.en = r.en; B.area = r.area; B.tOn = r.tOn;
  B.st = r.state; B.vol = r.vol; B.level = r.level; B.cx = r.cx; B.cy = r.cy; B.cz = r.cz;
  B.finalRec = r.finalRec; B.steps = r.steps; B.stop = r.stop;
  B.curveEvery = 0; B.traced = 0;
  B.tMax = r.tMax;
  B.maxSteps = LLONG_MAX;
  B.firstLaunch = 1;
  B.rule = r.rule;
  B.stopWhenStable = r.stopWhenStable ? 1 : 0;
  B.yieldBelow = 0;
  clear_noalloc_scratch<<<64, 256, 0, stream>>>(B, M.nmon, M.nmark);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_batch_kernel(mixed, r.teamWarps, M, B, L, r.blocks, r.teamsPerBlock, stream);
}

}  // namespace ssb
