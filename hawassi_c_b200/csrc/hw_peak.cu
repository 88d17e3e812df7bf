// hw_peak.cu -- FP64 fused multiply-add throughput of this GPU, the denominator of
// the FP64 roofline the benchmark reports next to the HBM one.  Every thread runs
// eight independent FMA chains (x = a x + b, |a| < 1 keeps x bounded and normal);
// the grid fills every SM to full occupancy, so the issue rate of the FP64 pipe,
// not latency, sets the time.  Best of five event-timed launches after a warm-up.
#include <cuda_runtime.h>

#include <cfloat>

#include "../../include/hawassi_b200.h"

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_dfma(double* __restrict__ out, int iters, double a, double b) {
  double x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) x[k] = 1e-3 * (double)(threadIdx.x + k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = fma(x[k], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += x[k];
  out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" double hw_fp64_peak_tflops(int device) {
  if (cudaSetDevice(device) != cudaSuccess) return -1.0;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0) return -1.0;
  const int blocks = sms * 8, iters = 4096;
  double* out = nullptr;
  if (cudaMalloc(&out, (size_t)blocks * kThreads * sizeof(double)) != cudaSuccess) return -1.0;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  double result = -1.0;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess && cudaEventCreate(&e0) == cudaSuccess &&
      cudaEventCreate(&e1) == cudaSuccess) {
    const double a = 0.999999, b = 1e-7;
    k_dfma<<<blocks, kThreads, 0, s>>>(out, iters, a, b);
    float best = FLT_MAX;
    bool ok = cudaGetLastError() == cudaSuccess;
    for (int rep = 0; ok && rep < 5; ++rep) {
      cudaEventRecord(e0, s);
      k_dfma<<<blocks, kThreads, 0, s>>>(out, iters, a, b);
      cudaEventRecord(e1, s);
      float ms = 0.0f;
      ok = cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && ms > 0.0f;
      if (ok && ms < best) best = ms;
    }
    if (ok) {
      const double flops = 2.0 * kChains * (double)iters * (double)blocks * kThreads;
      result = flops / (best * 1e-3) / 1e12;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  cudaFree(out);
  return result;
}
