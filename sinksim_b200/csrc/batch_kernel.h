// Host-side entry points of the batch kernel (batch_kernel.cu).
#pragma once

#include <cstddef>

#include <cuda_runtime.h>

#include "device_model.h"

namespace ssb {

// Simulations (warps) per block at most; the launcher picks fewer when a slot's shared memory is large.
constexpr int kMaxWarpsPerBlock = 16;

cudaError_t configure_batch_kernel(bool mixed, std::size_t smemBytes);
cudaError_t launch_batch_kernel(bool mixed, const DevModel& M, const DevBatch& B, const SlotLayout& L, int grid, int warpsPerBlock,
                                cudaStream_t stream);
cudaError_t batch_kernel_occupancy(bool mixed, int warpsPerBlock, std::size_t smemBytes, int* blocksPerSM);

}  // namespace ssb
