// noalloc.cu -- an FP64 dot product that allocates no device memory.
//
// Every other reduction of this library keeps its block partials in scratch memory that
// ieq_create allocates.  Some callers cannot allow that: hosts whose device memory is
// owned by their own pool (a framework's caching allocator, a MATLAB mex working within a
// fixed budget) and time loops that must not allocate once they run.  For them this entry
// point keeps its scratch -- one FP64 partial per block -- in a file-scope __device__ array
// of fixed size, so it needs no context and calls no cudaMalloc, cudaFree or allocating
// library routine.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/inductioneq.h"

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 8;
constexpr long long kPerBlock = (long long)kThreads * kPerThread;   // 2048 elements per block
constexpr int kMaxBlocks = IEQ_NOALLOC_DOT_MAX_ELEMENTS / kPerBlock;  // 4096 partials = 32 KiB

// the scratch: one partial per block; every GPU that loads the library holds it until exit
__device__ __align__(256) double g_noalloc_partials[kMaxBlocks];

// host-side stand-in names are not device addresses: the address is looked up once per
// device with that device current
constexpr int kMaxDevices = 64;
double *g_partials_addr[kMaxDevices] = {nullptr};
std::mutex g_setup_mutex;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sm[kThreads / 32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kThreads / 32; ++w) s += sm[w];
  return s;
}

// block k adds elements [k*2048, (k+1)*2048) in a fixed order
__global__ void __launch_bounds__(kThreads) k_dot_partials(const double *__restrict__ a, const double *__restrict__ b,
                                                           long long n, double *partials) {
  const long long base = blockIdx.x * kPerBlock;
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < kPerThread; ++k) {
    const long long i = base + (long long)k * kThreads + threadIdx.x;
    if (i < n) acc += a[i] * b[i];
  }
  const double s = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) k_dot_final(const double *partials, int nblocks, double *result) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < nblocks; i += kThreads) acc += partials[i];
  const double s = block_sum(acc);
  if (threadIdx.x == 0) result[0] = s;
}

}  // namespace

extern "C" ieq_status ieq_dot_product_noalloc(const double *a, const double *b, uint64_t n, double *result,
                                              void *stream) {
  if (!result || (n > 0 && (!a || !b))) return IEQ_ERR_ARG;
  if (n > (uint64_t)IEQ_NOALLOC_DOT_MAX_ELEMENTS) return IEQ_ERR_SHAPE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return IEQ_ERR_CUDA;
  double *partials = nullptr;
  {
    // set-up on the first call on this device (no allocation: only the symbol's address)
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_partials_addr[dev]) {
      void *p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) return IEQ_ERR_CUDA;
      g_partials_addr[dev] = static_cast<double *>(p);
    }
    partials = g_partials_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nblocks = (int)((n + kPerBlock - 1) / kPerBlock);
  if (nblocks > 0) k_dot_partials<<<nblocks, kThreads, 0, s>>>(a, b, (long long)n, partials);
  k_dot_final<<<1, kThreads, 0, s>>>(partials, nblocks, result);
  return cudaGetLastError() == cudaSuccess ? IEQ_OK : IEQ_ERR_CUDA;
}
