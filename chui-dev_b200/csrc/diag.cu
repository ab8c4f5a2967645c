// Diagnostics for the roofline of the residual walk, which is bound by the FP32
// pipes rather than HBM or tensor cores: a measured FP32 FMA throughput of this
// GPU (independent FFMA chains across all SMs, timed with CUDA events).
#include <cuda_runtime.h>

#include "../../include/chui_treepm_diag.h"
#include "context.cuh"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 8192;

__global__ void __launch_bounds__(256) ffmaKernel(float b, float c, float* sink) {
  float a[kChains];
  for (int k = 0; k < kChains; ++k) a[k] = threadIdx.x * 1e-7f + k;
#pragma unroll 4
  for (int i = 0; i < kIters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = fmaf(a[k], b, c);
  }
  float s = 0.f;
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (s == 1.2345f) sink[threadIdx.x] = s;  // keeps the chains live
}

}  // namespace

extern "C" int chui_treepm_probe_fp32_peak(int device, double* tflops) {
  if (!tflops) return CHUI_TREEPM_EINVAL;
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return CHUI_TREEPM_EDEVICE;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  float* sink = nullptr;
  if (cudaMalloc(&sink, 256 * sizeof(float)) != cudaSuccess) return CHUI_TREEPM_ENOMEM;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8;
  { chui::noteLaunch(); ffmaKernel<<<blocks, 256>>>(0.999999f, 1e-7f, sink); }
  cudaEventRecord(e0);
  const int reps = 5;
  for (int r = 0; r < reps; ++r) { chui::noteLaunch(); ffmaKernel<<<blocks, 256>>>(0.999999f, 1e-7f, sink); }
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  const double flops = 2.0 * kChains * static_cast<double>(kIters) * 256.0 * blocks * reps;
  *tflops = flops / (ms * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  cudaSetDevice(prev);
  return cudaGetLastError() == cudaSuccess ? 0 : CHUI_TREEPM_EDEVICE;
}
