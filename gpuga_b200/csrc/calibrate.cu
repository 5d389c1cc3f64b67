// Measured FP32 CUDA-core peak of the current GPU: a grid of independent FMA
// chains (no memory traffic in the timed loop), timed with CUDA events.  Used
// as the denominator of the FP32 roofline of the batched kernels.
#include "engine.hpp"

namespace gpuga {

__global__ void ffma_chains(int iters, float seed, float* sink) {
  float a0 = seed + threadIdx.x, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
  float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
  const float m = 0.999999f, c = 1e-7f;
  for (int k = 0; k < iters; ++k) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
      a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
    }
  }
  const float s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
  if (s == 1234.5f) sink[threadIdx.x] = s;  // keeps the chains alive
}

}  // namespace gpuga

extern "C" int gpuga_calibrate_fp32(int device, double* tflops) {
  using namespace gpuga;
  if (!tflops) {
    set_error("gpuga_calibrate_fp32: null output");
    return GPUGA_ERR_ARG;
  }
  GPUGA_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  GPUGA_CUDA(cudaGetDeviceProperties(&prop, device));
  float* sink = nullptr;
  GPUGA_CUDA(cudaMalloc(&sink, 1024 * sizeof(float)));
  const int threads = 256, blocks = prop.multiProcessorCount * 8, iters = 4096;
  cudaEvent_t a, b;
  GPUGA_CUDA(cudaEventCreate(&a));
  GPUGA_CUDA(cudaEventCreate(&b));
  ffma_chains<<<blocks, threads>>>(iters / 8, 1.0f, sink);  // warm-up
  GPUGA_CUDA(cudaGetLastError());
  double best = 0.0;
  for (int rep = 0; rep < 5; ++rep) {
    GPUGA_CUDA(cudaEventRecord(a));
    ffma_chains<<<blocks, threads>>>(iters, 1.0f + rep, sink);
    GPUGA_CUDA(cudaEventRecord(b));
    GPUGA_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    GPUGA_CUDA(cudaEventElapsedTime(&ms, a, b));
    const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    best = std::max(best, flops / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(sink);
  *tflops = best;
  return GPUGA_OK;
}
