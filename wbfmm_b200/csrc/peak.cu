// Measured FP32 FMA throughput of the current GPU, the denominator of the
// roofline fractions of the engine's SIMT kernels (the M2L, P2P, P2M and
// L2P arithmetic runs on the FP32 / FP64 pipes, not on the tensor cores).
// Eight independent FMA chains per thread keep every FP32 lane issuing; the
// grid fills each SM several times over.
#include <cuda_runtime.h>

#include "../../include/wbfmm_b200.h"
#include "engine.h"

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) k_fma_peak(float* out, int iters, float a, float b) {
  float x[kChains];
#pragma unroll
  for (int j = 0; j < kChains; j++) x[j] = (float)(threadIdx.x + j) * 1e-3f;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int j = 0; j < kChains; j++) x[j] = fmaf(x[j], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < kChains; j++) s += x[j];
  if (s == 1234.5f) out[blockIdx.x] = s;   // keeps the chains live; never true here
}

}  // namespace

using namespace wbfmm;

extern "C" int wbfmm_b200_fp32_fma_peak(double* tflops) {
  if (!tflops) return set_error(WBFMM_B200_E_ARG, "null output");
  if (wbfmm_b200_device_count() < 1) return set_error(WBFMM_B200_E_NOGPU, "no CUDA device is available");
  int dev = 0, sms = 0;
  WBFMM_CUDA(cudaGetDevice(&dev));
  WBFMM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = sms * 8, threads = 256, iters = 1 << 15;
  float* out = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = 0;
  float best = 0.f;
  if (cudaMalloc(&out, sizeof(float) * blocks) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    rc = set_error(WBFMM_B200_E_NOMEM, "peak measurement setup failed");
  }
  for (int r = 0; r < 4 && !rc; r++) {   // the first launch warms up
    cudaEventRecord(e0, s);
    k_fma_peak<<<blocks, threads, 0, s>>>(out, iters, 0.999f, 1e-4f);
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      rc = set_error(WBFMM_B200_E_STATE, "peak measurement kernel failed");
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && (best == 0.f || ms < best)) best = ms;
  }
  cudaGetLastError();
  if (!rc) {
    const double flops = 2.0 * kChains * (double)iters * blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  if (out) cudaFree(out);
  return rc;
}
