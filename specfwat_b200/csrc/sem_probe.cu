// FP32 FMA throughput of the device, the denominator of the element
// kernels' FP32 roofline fraction.
//
// Every thread runs 8 independent fmaf chains (x = x * a + b with a, b > 0,
// so x stays in (0, 1] and never denormalises) for `iters` x 16 rounds.  The
// grid fills every SM with 2,048 resident threads, enough warps to cover the
// FMA pipe's latency.  The chain results are kept live by a store that only
// runs if their sum is negative, which it never is.

#include <cuda_runtime.h>

#include "sem_b200.h"
#include "sem_internal.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kChains = 8;
constexpr int kUnroll = 16;

__global__ void __launch_bounds__(kThreads) k_fma_peak(float* sink, int iters, float a, float b) {
  float x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) x[k] = 1e-3f * (float)((threadIdx.x + k) & 63);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < kUnroll; ++r)
#pragma unroll
      for (int k = 0; k < kChains; ++k) x[k] = fmaf(x[k], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += x[k];
  if (s < 0.f) sink[0] = s;
}

}  // namespace

extern "C" int sem_fp32_fma_peak(double* tflops, double* ms) {
  if (!tflops) return sem::report_error(SEM_ERR_ARG, "null output");
  int dev = 0, sms = 0, maxthr = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return sem::report_error(SEM_ERR_NODEVICE, "no CUDA device: %s", cudaGetErrorString(e));
  }
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&maxthr, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
  if (sms < 1 || maxthr < kThreads)
    return sem::report_error(SEM_ERR_UNSUPPORTED, "device reports %d SMs, %d threads per SM", sms,
                             maxthr);
  const int blocks = sms * (maxthr / kThreads);
  const int iters = 4096;
  float* sink = nullptr;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  e = cudaMalloc(&sink, sizeof(float));
  if (e == cudaSuccess) e = cudaEventCreate(&t0);
  if (e == cudaSuccess) e = cudaEventCreate(&t1);
  float best = 0.f;
  if (e == cudaSuccess) {
    k_fma_peak<<<blocks, kThreads>>>(sink, iters, 0.999f, 1e-3f);  // warm-up
    for (int rep = 0; rep < 5 && e == cudaSuccess; ++rep) {
      cudaEventRecord(t0);
      k_fma_peak<<<blocks, kThreads>>>(sink, iters, 0.999f, 1e-3f);
      cudaEventRecord(t1);
      e = cudaEventSynchronize(t1);
      float m = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&m, t0, t1);
      if (e == cudaSuccess && (best == 0.f || m < best)) best = m;
    }
  }
  if (t0) cudaEventDestroy(t0);
  if (t1) cudaEventDestroy(t1);
  if (sink) cudaFree(sink);
  if (e != cudaSuccess || !(best > 0.f)) {
    cudaGetLastError();
    return sem::report_error(SEM_ERR_CUDA, "FMA peak probe failed: %s", cudaGetErrorString(e));
  }
  const double fmas = (double)blocks * kThreads * iters * kUnroll * kChains;
  *tflops = 2.0 * fmas / (best * 1e-3) / 1e12;
  if (ms) *ms = best;
  return SEM_OK;
}
