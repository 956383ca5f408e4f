// diag.cuh -- the per-step diagnostics of the time loop in one pass.
//
// compute_numerical_solution.m:153-173 (save_integrals_over_time) records before every
// step the energy norm2(b), the divergence norm sqrt(norm2_S(calc_div(b))) and the error
// sqrt(norm2_diff(b, analytical_b(time))) -- four kernels, three reductions and a host
// sum each.  k_diag_partials evaluates the three per-node terms in one pass over b (the
// divergence with the SBP rows of calc_div, the exact field at time[0]) and writes one
// partial per block and quantity; k_diag_final adds them in a fixed order and appends
// the three totals to a device series.  The per-node terms and the summation order are
// those of the stand-alone reductions (k_reduce_partials / k_reduce_final), so each entry
// equals what ieq_norm2_value, ieq_norm2_S_value of calc_div and ieq_norm2_diff_value of
// analytical_b return for the same field (up to the compiler's FMA contraction).
#pragma once
#include "misc_kernels.cuh"
#include "stage_kernel.cuh"

namespace ieq {

template <typename R, typename F>
struct DiagArgs {
  Mesh m;
  F b;
  long long n;
  const R *wx, *wy, *wz;   // per-axis mass weights (norm2 of kernel_operator.cl)
  const R *D;              // derivative rows [2nb+1][sw]
  int nb, sw, periodic;
  R dS[3];                 // (REAL)DX ...
  int tc;                  // testcase of analytical_b
  const R *time;           // analytical_b at time[0]
};

// the three terms of node i: energy, divergence, error (each as its reduction kernel forms it)
template <typename R, typename F>
__device__ __forceinline__ void diag_terms(const DiagArgs<R, F> &a, long long i, double &e, double &dv, double &er) {
  const int ix = (int)(i % a.m.nx);
  const long long r = i / a.m.nx;
  const int iy = (int)(r % a.m.ny);
  const int iz = (int)(r / a.m.ny);
  const R fac = (a.wx[ix] * a.wy[iy]) * a.wz[iz];
  const V3<R> B = ldf(a.b, i);
  e += (double)(fac * ((B.x * B.x + B.y * B.y) + B.z * B.z));
  // calc_div (kernel_operator.cl:145): sum over the axes of d/d(axis) of that component
  const int ii[3] = {ix, iy, iz};
  const int nn[3] = {a.m.nx, a.m.ny, a.m.nz};
  const long long st[3] = {1, a.m.nx, (long long)a.m.nx * a.m.ny};
  const int c0 = (a.sw - 1) / 2;
  R d[3];
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    const int row = a.periodic ? a.nb : sbp_row(ii[ax], nn[ax], a.nb);
    R v = 0;
    for (int c = 0; c < a.sw; ++c) {
      const R cf = a.D[row * a.sw + c];
      if (cf == (R)0) continue;
      const long long j = i + (long long)(nbr_rt<R>(ii[ax], c - c0, nn[ax], a.periodic) - ii[ax]) * st[ax];
      v += cf * ldc<R, F>(a.b, j, ax);
    }
    d[ax] = v / a.dS[ax];
  }
  const R dvg = (d[0] + d[1]) + d[2];
  dv += (double)((fac * dvg) * dvg);
  const V3<R> A = b_analytical<R>(a.tc, a.m, ix, iy, iz, a.time[0]);
  const V3<R> w = {B.x - A.x, B.y - A.y, B.z - A.z};
  er += (double)(fac * ((w.x * w.x + w.y * w.y) + w.z * w.z));
}

// partials[k * gridDim.x + block], k = 0 energy, 1 divergence, 2 error
template <typename R, typename F>
__global__ void __launch_bounds__(256) k_diag_partials(const DiagArgs<R, F> a, double *partials) {
  __shared__ double sm[3][8];
  double acc[3] = {0.0, 0.0, 0.0};
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.n; i += stride)
    diag_terms(a, i, acc[0], acc[1], acc[2]);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double v = warp_sum(acc[k]);
    if ((threadIdx.x & 31) == 0) sm[k][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double v = threadIdx.x < (blockDim.x >> 5) ? sm[k][threadIdx.x] : 0.0;
      v = warp_sum(v);
      if (threadIdx.x == 0) partials[k * gridDim.x + blockIdx.x] = v;
    }
  }
}

// the three totals of `np` partials each, in the order of k_reduce_final, appended to
// series[3 * pos .. 3 * pos + 2] (pos = *count, then incremented; nothing is written past
// `capacity` entries)
static __global__ void __launch_bounds__(256) k_diag_final(const double *partials, int np, double *series, int *count,
                                                    int capacity) {
  __shared__ double sm[8];
  const int pos = *count;
  for (int k = 0; k < 3; ++k) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) acc += partials[k * np + i];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double v = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += sm[w];
      if (pos < capacity) series[3 * pos + k] = v;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *count = pos + 1;
}

}  // namespace ieq
