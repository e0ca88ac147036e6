// Host-side entry points of the batch kernel (batch_kernel.cu).
#pragma once

#include <cstddef>

#include <cuda_runtime.h>

#include "device_model.h"

namespace ssb {

// Warps per block at most (teams of 1, 2, 4 or 8 warps; teams per block x warps per team <= kMaxWarpsPerBlock) and the
// blocks of that size the kernel is compiled to fit on one SM (which sets its register budget: 65,536 registers
// over kMaxWarpsPerBlock x 32 x kMinBlocksPerSM threads).
#ifndef SSB_BLOCK_WARPS
#define SSB_BLOCK_WARPS 16
#endif
#ifndef SSB_MIN_BLOCKS
#define SSB_MIN_BLOCKS 1
#endif
constexpr int kMaxWarpsPerBlock = SSB_BLOCK_WARPS;
constexpr int kMinBlocksPerSM = SSB_MIN_BLOCKS;
static_assert(kMaxWarpsPerBlock >= 8, "a block must hold an eight-warp team");

bool valid_team_size(int teamWarps);
cudaError_t configure_batch_kernel(bool mixed, int teamWarps, std::size_t smemBytes, bool fleet = false);
// Shared memory a block needs beyond its slots to hold the column table (DevBatch::stageColumns).
std::size_t column_stage_bytes(bool mixed, int ncol);
cudaError_t launch_batch_kernel(bool mixed, int teamWarps, const DevModel& M, const DevBatch& B, const SlotLayout& L, int grid,
                                int teamsPerBlock, cudaStream_t stream);
cudaError_t batch_kernel_occupancy(bool mixed, int teamWarps, int teamsPerBlock, std::size_t smemBytes, int* blocksPerSM, bool fleet = false);
// The counters a run starts from: `remaining` = count, the phases' step counters zero (a kernel, so that the run's
// whole launch chain can be captured in a CUDA graph).
cudaError_t launch_start_run(std::int32_t* remaining, std::int32_t count, unsigned long long* phaseSteps, int phases, cudaStream_t stream);
// The claim order of a launch phase after the first (DevBatch::order): the unfinished instances (stop == running),
// fewest steps done first, ties by index, into order[0 .. *n). list and order hold count entries. `bound` is an upper
// bound on the unfinished instances (it sizes the ranking grid; the ranking takes O(n^2) compares).
cudaError_t launch_order_unfinished(const std::int32_t* stop, const long long* steps, std::int32_t count, std::int32_t bound,
                                    std::int32_t* list, std::int32_t* order, std::int32_t* n, cudaStream_t stream);

// A batch run whose scratch lives in a fixed device array of the library (see batch_kernel.cu); every pointer here
// is the caller's device memory. state is count x 8 (t, zO, pitch, roll, vz, wth, wph, and the settle timer, which
// must start at 0); vol .. cz are count x nodes; en, area, tOn count x connections; finalRec count x 7; steps and
// stop count (cleared by the call). In and out: state, vol, level, cx, cy, cz.
struct NoAllocRun {
  std::int32_t count;
  const std::uint8_t* en;
  const double *area, *tOn;
  double *state, *vol, *level, *cx, *cy, *cz, *finalRec;
  long long* steps;
  std::int32_t* stop;
  double tMax;
  RetireRule rule;
  bool stopWhenStable;  // the reference's calm rule (stop reason 5), as in the batch's own runs
  int teamWarps, teamsPerBlock, blocks;
};
std::size_t noalloc_scratch_capacity();
std::size_t noalloc_scratch_bytes(const DevModel& M, int count);
// cudaErrorMemoryAllocation when count instances need more scratch than the fixed array holds.
cudaError_t run_batch_noalloc(bool mixed, const DevModel& M, const SlotLayout& L, const NoAllocRun& run, cudaStream_t stream);

}  // namespace ssb
