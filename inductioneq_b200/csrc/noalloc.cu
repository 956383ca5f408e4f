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

// In host code the array's name is a host-side stand-in, not a device address: the address
// is looked up with cudaGetSymbolAddress (which allocates nothing) on every call, with the
// calling thread's current device, so a module reloaded after a device reset is found again.
// The lock serialises the lookups (the first one on a device loads the library's device image).
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
  double *partials = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) return IEQ_ERR_CUDA;
    partials = static_cast<double *>(p);
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  long long nn = (long long)n;
  int nblocks = (int)((nn + kPerBlock - 1) / kPerBlock);
  // each launch's own status (not an error left behind by an earlier, unrelated launch)
  if (nblocks > 0) {
    void *args[] = {(void *)&a, (void *)&b, (void *)&nn, (void *)&partials};
    if (cudaLaunchKernel((const void *)k_dot_partials, dim3(nblocks), dim3(kThreads), args, 0, s) != cudaSuccess)
      return IEQ_ERR_CUDA;
  }
  void *fargs[] = {(void *)&partials, (void *)&nblocks, (void *)&result};
  if (cudaLaunchKernel((const void *)k_dot_final, dim3(1), dim3(kThreads), fargs, 0, s) != cudaSuccess)
    return IEQ_ERR_CUDA;
  return IEQ_OK;
}
