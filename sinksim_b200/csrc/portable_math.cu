// Elementwise evaluation of the portable math on the device and on the host, for the parity tests of the device
// code against the reference's fdlibm (op 0 sin, 1 cos, 2 pow, 3 scalbn).
#include <cuda_runtime.h>

#include <cstdint>

#include "portable_math.cuh"

namespace ssb {

namespace {

__host__ __device__ inline double eval(int op, double x, double y) {
  switch (op) {
    case 0: return pm::sin(x);
    case 1: return pm::cos(x);
    case 2: return pm::pow(x, y);
    default: return pm::scale2(x, static_cast<int>(y));
  }
}

__global__ void portable_math_kernel(int op, const double* x, const double* y, double* out, std::int64_t n) {
  const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
  for (std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = eval(op, x[i], y ? y[i] : 0.0);
}

}  // namespace

void portable_math_host(int op, const double* x, const double* y, double* out, std::int64_t n) {
  for (std::int64_t i = 0; i < n; ++i) out[i] = eval(op, x[i], y ? y[i] : 0.0);
}

cudaError_t portable_math_device(int op, const double* x, const double* y, double* out, std::int64_t n) {
  if (n <= 0) return cudaSuccess;
  const std::size_t bytes = static_cast<std::size_t>(n) * sizeof(double);
  double *dx = nullptr, *dy = nullptr, *dout = nullptr;
  cudaError_t e = cudaMalloc(&dx, bytes);
  if (e == cudaSuccess && y) e = cudaMalloc(&dy, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&dout, bytes);
  if (e == cudaSuccess) e = cudaMemcpy(dx, x, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && y) e = cudaMemcpy(dy, y, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const int threads = 256;
    const std::int64_t want = (n + threads - 1) / threads;
    const int blocks = static_cast<int>(want < 148 * 16 ? want : 148 * 16);
    portable_math_kernel<<<blocks, threads>>>(op, dx, dy, dout, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, bytes, cudaMemcpyDeviceToHost);
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(dout);
  return e;
}

}  // namespace ssb
