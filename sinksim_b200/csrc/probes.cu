// Peak probes: the denominators of the roofline this engine reports. The step is bound by FP64 (portable) or FP32
// (portable32) arithmetic issued without fused multiply-add (the bits require separately rounded products and sums)
// and by on-chip memory latency, not by HBM or tensor cores, so its roofline is the measured rate of separately
// rounded FP64 (or FP32) adds and multiplies.
//
// Each thread runs kChains independent dependency chains of alternating add and multiply for `iters` iterations; the
// result is stored so the work cannot be removed. Counted operations: 2 * kChains * iters per thread.
#include <cuda_runtime.h>

#include <cstdint>

namespace ssb {

namespace {

constexpr int kChains = 8;

template <class T>
__global__ void __launch_bounds__(256) add_mul_chains(T* out, T a, T m, int iters) {
  T v[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) v[k] = static_cast<T>(threadIdx.x + k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) {
      v[k] = v[k] + a;
      v[k] = v[k] * m;
    }
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += v[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

// Returns the achieved operations per second (adds + multiplies) of one burst, or a negative value on error.
double measure_add_mul_peak(bool fp64, int device) {
  if (cudaSetDevice(device) != cudaSuccess) return -1;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int blocks = sms * 8, threads = 256, iters = 4096;
  void* out = nullptr;
  if (cudaMalloc(&out, static_cast<std::size_t>(blocks) * threads * 8) != cudaSuccess) return -1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0);
    if (fp64) add_mul_chains<double><<<blocks, threads>>>(static_cast<double*>(out), 1e-9, 0.999999, iters);
    else add_mul_chains<float><<<blocks, threads>>>(static_cast<float*>(out), 1e-6f, 0.9999f, iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;  // the first launch is a warm-up
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return -1;
  const double ops = 2.0 * kChains * static_cast<double>(iters) * blocks * threads;
  return ops / (best * 1e-3);
}

}  // namespace ssb
