// Host-side entry points of the batch kernel (batch_kernel.cu).
#pragma once

#include <cstddef>

#include <cuda_runtime.h>

#include "device_model.h"

namespace ssb {

// Warps per block at most (teams of 1, 2, 4 or 8 warps; teams per block x warps per team <= 16).
constexpr int kMaxWarpsPerBlock = 16;

bool valid_team_size(int teamWarps);
cudaError_t configure_batch_kernel(bool mixed, int teamWarps, std::size_t smemBytes);
cudaError_t launch_batch_kernel(bool mixed, int teamWarps, const DevModel& M, const DevBatch& B, const SlotLayout& L, int grid,
                                int teamsPerBlock, cudaStream_t stream);
cudaError_t batch_kernel_occupancy(bool mixed, int teamWarps, int teamsPerBlock, std::size_t smemBytes, int* blocksPerSM);

}  // namespace ssb
