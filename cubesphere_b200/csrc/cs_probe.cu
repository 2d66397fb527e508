// Measured FP64 FMA rate of the current device: the denominator of the
// FP64 roofline the bench reports beside the HBM one (the stage kernels are
// FP64-arithmetic and latency bound).  No counterpart in the reference.
#include <cuda_runtime.h>

#include "cubesphere_b200.h"

namespace {

constexpr int kChains = 8;   // independent FMA chains per thread
constexpr int kUnroll = 16;  // FMAs per chain per loop trip

// Every thread runs kChains independent dependency chains a = a * b + c
// (|b| < 1, so the values stay bounded); the sum is stored only when it is
// non-finite, which never happens, so the loop is not removed.
__global__ void __launch_bounds__(256) k_dfma_rate(int iters, double b, double c, double* sink) {
  double a[kChains];
#pragma unroll
  for (int q = 0; q < kChains; ++q) a[q] = (threadIdx.x + 1) * 1e-3 + q;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
      for (int q = 0; q < kChains; ++q) a[q] = fma(a[q], b, c);
    }
  }
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < kChains; ++q) s += a[q];
  if (!isfinite(s)) *sink = s;
}

}  // namespace

extern "C" int cs_fp64_fma_rate(int32_t iters, double* tflops) {
  if (!tflops || iters < 1) return CS_ERR_ARG;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return CS_ERR_CUDA;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return CS_ERR_CUDA;
  double* sink = nullptr;
  if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess) return CS_ERR_CUDA;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8, threads = 256;
  k_dfma_rate<<<blocks, threads>>>(iters / 4 + 1, 0.999999, 1e-6, sink);  // warm-up
  cudaEventRecord(e0);
  k_dfma_rate<<<blocks, threads>>>(iters, 0.999999, 1e-6, sink);
  cudaEventRecord(e1);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (e != cudaSuccess || !(ms > 0.0f)) return CS_ERR_CUDA;
  const double flops = 2.0 * kChains * kUnroll * (double)iters * blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return CS_OK;
}
