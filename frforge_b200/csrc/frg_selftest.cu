// Internal self-check of device arithmetic that the stage kernels use in
// place of CUDA's own operations, for the test suite; not part of the public
// C ABI (include/frforge_cuda.h declares nothing from this file).
//
//   frg_internal_reciprocal_check: the Newton reciprocal frcp (frg_device.cuh)
//   and CUDA's correctly rounded 1.0 / x on the same inputs.
//   frg_internal_sqrt_check: the Goldschmidt square root fsqrt and CUDA's
//   correctly rounded sqrt on the same inputs.
#include <cuda_runtime.h>

#include <cstddef>

#include "frg_device.cuh"

namespace frg {
namespace {

__global__ void reciprocal_check_kernel(const double* x, double* y, double* q, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    y[i] = frcp(x[i]);
    q[i] = 1.0 / x[i];
  }
}

__global__ void sqrt_check_kernel(const double* x, double* y, double* q, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    y[i] = fsqrt(x[i]);
    q[i] = sqrt(x[i]);
  }
}

// x (host, n values) -> ours and CUDA's (host) through one of the kernels
int run_check(int which, const double* x, double* ours, double* cuda, size_t n) {
  if (!x || !ours || !cuda) return (int)cudaErrorInvalidValue;
  if (n == 0) return 0;
  double* d = nullptr;
  cudaError_t e = cudaMalloc(&d, 3 * n * sizeof(double));
  if (e != cudaSuccess) return (int)e;
  e = cudaMemcpy(d, x, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const int blocks = (int)((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024);
    if (which == 0)
      reciprocal_check_kernel<<<blocks, 256>>>(d, d + n, d + 2 * n, n);
    else
      sqrt_check_kernel<<<blocks, 256>>>(d, d + n, d + 2 * n, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(ours, d + n, n * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(cuda, d + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return (int)e;
}

}  // namespace
}  // namespace frg

// x (host, n values) -> frcp(x) and 1.0 / x (host); returns 0 or a CUDA error
// code.  Runs on the current device with its own short-lived buffers.
extern "C" int frg_internal_reciprocal_check(const double* x, double* frcp_out, double* div_out, size_t n) {
  return frg::run_check(0, x, frcp_out, div_out, n);
}

// x (host, n values) -> fsqrt(x) and sqrt(x) (host), as above.
extern "C" int frg_internal_sqrt_check(const double* x, double* fsqrt_out, double* sqrt_out, size_t n) {
  return frg::run_check(1, x, fsqrt_out, sqrt_out, n);
}
