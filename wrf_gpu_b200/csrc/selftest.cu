// Device self-checks of numerical helpers, built as a separate test library
// (libwrfgpu_selftest.so) so the product library exports only its C ABI.
#include <cuda_runtime.h>

#include "dycore_common.cuh"

namespace {

__global__ void k_div_check(const double *a, const double *b, const double *rb, double *q_rcp, double *q_div,
                            long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  q_rcp[i] = wg::div_rcp(a[i], b[i], rb[i]);
  q_div[i] = a[i] / b[i];
}

}  // namespace

// q_rcp[i] = div_rcp(a[i], b[i], rb[i]) and q_div[i] = a[i] / b[i] (CUDA's
// IEEE division) on device arrays of n doubles.
extern "C" int wrfgpu_selftest_div_rcp(const double *a, const double *b, const double *rb, double *q_rcp,
                                       double *q_div, long n, cudaStream_t stream) {
  if (n <= 0) return 0;
  const int threads = 256;
  const long blocks = (n + threads - 1) / threads;
  k_div_check<<<(unsigned)blocks, threads, 0, stream>>>(a, b, rb, q_rcp, q_div, n);
  return cudaGetLastError() == cudaSuccess ? 0 : 3;
}
