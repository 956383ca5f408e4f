// peaks.cu -- the FP64 arithmetic peak of the device, measured with an FMA loop.
//
// The stencil kernels are graded against the binding roof of the device: the HBM copy
// bandwidth, measured elsewhere, and the FP64 rate, measured here.  k_fma_loop runs
// kChains independent dependency chains of fused multiply-adds per thread (enough to
// cover the FMA latency), on a grid of 8 blocks of 256 threads per SM, and writes one value
// per thread so that nothing is optimised away.  FLOPs = 2 per FMA.
#include <cuda_runtime.h>

#include "../../include/inductioneq.h"

namespace {

constexpr int kThreads = 256;
constexpr int kChains = 8;

__global__ void __launch_bounds__(kThreads) k_fma_loop(double *out, int iters, double a, double b) {
  double x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = (double)(threadIdx.x + c) * 1e-3;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  out[blockIdx.x * (long long)kThreads + threadIdx.x] = s;
}

}  // namespace

extern "C" ieq_status ieq_fp64_fma_rate(int device, int iterations, double *gflops) {
  if (!gflops || iterations < 1) return IEQ_ERR_ARG;
  *gflops = 0.0;
  if (cudaSetDevice(device) != cudaSuccess) return IEQ_ERR_CUDA;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return IEQ_ERR_CUDA;
  const int blocks = 8 * sms;
  double *out = nullptr;
  if (cudaMalloc(&out, (size_t)blocks * kThreads * sizeof(double)) != cudaSuccess) return IEQ_ERR_CUDA;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // a = 1 - 2^-20, b = 2^-30: the chains stay finite and normal
  const double a = 1.0 - 9.5367431640625e-07, b = 9.313225746154785e-10;
  k_fma_loop<<<blocks, kThreads>>>(out, iterations / 10 + 1, a, b);   // warm-up
  cudaEventRecord(e0);
  k_fma_loop<<<blocks, kThreads>>>(out, iterations, a, b);
  cudaEventRecord(e1);
  ieq_status st = IEQ_OK;
  float ms = 0.f;
  if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || ms <= 0.f)
    st = IEQ_ERR_CUDA;
  else
    *gflops = 2.0 * kChains * (double)iterations * blocks * kThreads / (ms * 1e-3) / 1e9;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return st;
}
