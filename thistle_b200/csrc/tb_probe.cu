// FP64 FMA throughput probe: the denominator of the Bessel-sum roofline.
// Sixteen independent register-resident FMA chains per thread, enough warps
// per SM to cover the FMA latency; nothing touches memory inside the loop.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "thistle_b200.h"

namespace {

__global__ void __launch_bounds__(256) fma_probe_kernel(double *out, int iters) {
  double a[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) a[k] = 1e-3 * (threadIdx.x + k);
  const double b = 0.9999999, c = 1e-9;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) a[k] = fma(a[k], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 16; ++k) s += a[k];
  if (s == -1.0) out[blockIdx.x] = s;  // keeps the chains alive
}

}  // namespace

extern "C" int thistle_probe_fp64_peak(int32_t reps, double *tflops) {
  if (!tflops || reps <= 0) return THISTLE_ERR_ARG;
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return THISTLE_ERR_CUDA;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return THISTLE_ERR_CUDA;
  double *out = nullptr;
  if (cudaMalloc(&out, sizeof(double) * nsm * 8) != cudaSuccess) return THISTLE_ERR_NOMEM;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int iters = 1 << 16, blocks = nsm * 8, threads = 256;
  double best = 0.0;
  for (int r = 0; r < reps + 1; ++r) {
    cudaEventRecord(e0);
    fma_probe_kernel<<<blocks, threads>>>(out, iters);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess) break;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    double fl = 2.0 * 16.0 * iters * (double)blocks * threads;
    if (r > 0 && ms > 0) best = std::max(best, fl / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  *tflops = best;
  return cudaGetLastError() == cudaSuccess && best > 0 ? THISTLE_OK : THISTLE_ERR_CUDA;
}
