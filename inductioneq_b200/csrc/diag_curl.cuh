// diag_curl.cuh -- the per-step diagnostics of the time loop folded into the step's first
// curl kernel.
//
// compute_numerical_solution.m:153-173 (save_integrals_over_time) records before every step
// the energy norm2(b), the divergence norm sqrt(norm2_S(calc_div(b))) and the error
// sqrt(norm2_diff(b, analytical_b(time))).  The first kernel of a Hall step, the curl kernel
// of stage 1, reads exactly that state -- b at every node and its stencil neighbours -- so
// k_curl_e_diag forms J = curl(B)/rho, E = J x B (and the dissipation sum) as k_curl_e_hod /
// k_curl_e do, adds each node's three diagnostic terms (diag_terms: the terms of the stand-
// alone reductions) into per-block partials, and the last block to finish (ticket counter)
// adds the partials in a fixed order and appends the three totals to the device series.  The
// step graph then has no launch for the diagnostics.
#pragma once
#include "diag.cuh"
#include "stage_col.cuh"

namespace ieq {

// where the diagnostics of one step go
struct DiagOut {
  double *partials;    // [3][gridDim] block partials
  unsigned *counter;   // last-block ticket
  double *series;      // 3 totals per step
  int *count;          // steps recorded so far
  int capacity;
};

template <typename R, int OP, bool PER, bool HODS>
__global__ void __launch_bounds__(kColThreads) k_curl_e_diag(const __grid_constant__ CurlArgs<R, SoA<R>> a,
                                                             const __grid_constant__ DiagArgs<R, SoA<R>> d,
                                                             const DiagOut o) {
  pdl_enter();
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z;
  double acc[3] = {0.0, 0.0, 0.0};
  if (ix < nx && iy < ny && iz < nz) {
    const long long idx = ix + (long long)nx * (iy + (long long)ny * iz);
    const int ii[3] = {ix, iy, iz};
    const int nn[3] = {nx, ny, nz};
    const long long st[3] = {1, nx, (long long)nx * ny};
    const V3<R> Bm = ldf(a.b, idx);
    R g[3][3];
    V3<R> hod = {0, 0, 0};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      const int c1 = (ax + 1) % 3, c2 = (ax + 2) % 3;
      R v1, v2;
      V3<R> ho;
      curl_axis_node<R, OP, PER, HODS>(a, ax, ii[ax], nn[ax], idx, st[ax], Bm, v1, v2, ho);
      g[ax][c1] = v1 * a.inv_d[ax];
      g[ax][c2] = v2 * a.inv_d[ax];
      if (HODS) {
        hod.x += ho.x; hod.y += ho.y; hod.z += ho.z;
      }
    }
    V3<R> J = {g[1][2] - g[2][1], g[2][0] - g[0][2], g[0][1] - g[1][0]};
    if (a.rho) {
      const R r = (R)1 / a.rho[idx];
      J = {J.x * r, J.y * r, J.z * r};
    }
    stf(a.out, idx, V3<R>{J.x * Bm.y - J.y * Bm.x, J.x * Bm.z - J.z * Bm.x, J.y * Bm.z - J.z * Bm.y});
    if (HODS) stf(a.hout, idx, hod);
    if (!PER && (ix == 0 || iy == 0 || iz == 0 || ix == nx - 1 || iy == ny - 1 || iz == nz - 1))
      stf(a.jface, idx, J);
    diag_terms(d, idx, acc[0], acc[1], acc[2]);
  }
  // block partials (whole warps: the launcher gives 128-thread blocks), then the last block
  // adds them in a fixed order
  __shared__ double sm[3][kColThreads / 32];
  __shared__ bool last;
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
  const unsigned blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double v = warp_sum(acc[k]);
    if ((t & 31) == 0) sm[k][t >> 5] = v;
  }
  __syncthreads();
  if (t == 0) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double s = 0.0;
      for (int w = 0; w < nt >> 5; ++w) s += sm[k][w];
      o.partials[k * nb + blk] = s;
    }
    __threadfence();
    last = atomicAdd(o.counter, 1u) == nb - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int pos = *o.count;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double s = 0.0;
    for (unsigned i = t; i < nb; i += nt) s += o.partials[k * nb + i];
    s = warp_sum(s);
    __syncthreads();
    if ((t & 31) == 0) sm[0][t >> 5] = s;
    __syncthreads();
    if (t == 0) {
      double v = 0.0;
      for (int w = 0; w < nt >> 5; ++w) v += sm[0][w];
      if (pos < o.capacity) o.series[3 * pos + k] = v;
    }
  }
  if (t == 0) {
    *o.count = pos + 1;
    *o.counter = 0u;
  }
}

// explicit launcher, instantiated per (R, OP) in stage_<r>_o<op>.cu
template <typename R, int OP>
void launch_curl_e_diag(const CurlArgs<R, SoA<R>> &a, const DiagArgs<R, SoA<R>> &d, const DiagOut &o, bool per,
                        bool hod, dim3 grid, dim3 block, bool pdl, cudaStream_t s);

}  // namespace ieq
