// misc_kernels.cuh -- the non-stage kernels: testcase evaluation, time bookkeeping,
// pointwise Runge-Kutta updates, reductions (norms, dot products), divergence/gradient
// operators and the conjugate-gradient pieces of divergence cleaning.
#pragma once
#include "ieq_common.cuh"

namespace ieq {

// ---------------------------------------------------------------- testcase evaluation
enum InitKind : int { INIT_B = 0, INIT_U = 1, INIT_RHO = 2, ANALYTICAL_B = 3, CALC_U = 4 };

// kernel_init.cl:3-48 and kernel_time_integrator.cl:93-125 (u = u_analytical(time[1]))
// vout: REAL4 AoS (vstride = 0) or SoA with component stride vstride
template <typename R>
__device__ __forceinline__ void st_any(R *base, long long vstride, long long idx, V3<R> v) {
  if (vstride == 0) {
    st3(reinterpret_cast<R4<R> *>(base) + idx, v);
  } else {
    base[idx] = v.x;
    base[idx + vstride] = v.y;
    base[idx + 2 * vstride] = v.z;
  }
}

// u of hall_periodic at time t (a sum of one-dimensional terms): the block evaluates the
// terms once per x, y and z index of its tile in shared memory (blockDim.x + y + z cosine and
// sine pairs instead of six per node), then adds them per node
template <typename R>
__device__ void hall_periodic_u_block(const Mesh &m, R *vout, long long vstride, R t) {
  __shared__ R tc[3][32], ts[3][32];   // [axis][index within the tile]
  const int dim[3] = {(int)blockDim.x, (int)blockDim.y, (int)blockDim.z};
  const int base[3] = {(int)(blockIdx.x * blockDim.x), (int)(blockIdx.y * blockDim.y), (int)(blockIdx.z * blockDim.z)};
  const int lin = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  int ax = -1, k = lin;
  for (int a = 0; a < 3 && ax < 0; ++a) {
    if (k < dim[a]) ax = a;
    else k -= dim[a];
  }
  if (ax >= 0) {
    int ii[3] = {0, 0, 0};
    ii[ax] = base[ax] + k;
    R q[3];
    coords<R>(m, ii[0], ii[1], ii[2], q[0], q[1], q[2]);
    tc_hall_periodic_terms(q[ax], t, tc[ax][k], ts[ax][k]);
  }
  __syncthreads();
  const int ix = base[0] + threadIdx.x, iy = base[1] + threadIdx.y, iz = base[2] + threadIdx.z;
  if (ix >= m.nx || iy >= m.ny || iz >= m.nz) return;
  const long long idx = ix + (long long)m.nx * (iy + (long long)m.ny * iz);
  const int x = threadIdx.x, y = threadIdx.y, z = threadIdx.z;
  st_any(vout, vstride, idx, V3<R>{tc[1][y] + ts[2][z], tc[2][z] + ts[0][x], tc[0][x] + ts[1][y]});
}

template <typename R>
__global__ void k_init(Mesh m, int tc, int kind, R *vout, long long vstride, R *sout, const R *time) {
  if (kind == CALC_U && tc == TC_HALL_PERIODIC && blockDim.x <= 32 && blockDim.y <= 32 && blockDim.z <= 32 &&
      blockDim.x * blockDim.y * blockDim.z >= blockDim.x + blockDim.y + blockDim.z) {
    hall_periodic_u_block<R>(m, vout, vstride, time[1]);
    return;
  }
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z;
  if (ix >= m.nx || iy >= m.ny || iz >= m.nz) return;
  const long long idx = ix + (long long)m.nx * (iy + (long long)m.ny * iz);
  switch (kind) {
    case INIT_B: st_any(vout, vstride, idx, b_analytical<R>(tc, m, ix, iy, iz, (R)0)); break;
    case INIT_U: st_any(vout, vstride, idx, u_analytical<R>(tc, m, ix, iy, iz, (R)0)); break;
    case INIT_RHO: sout[idx] = (R)1; break;
    case ANALYTICAL_B: st_any(vout, vstride, idx, b_analytical<R>(tc, m, ix, iy, iz, time[0])); break;
    case CALC_U: st_any(vout, vstride, idx, u_analytical<R>(tc, m, ix, iy, iz, time[1])); break;
  }
}

// ---------------------------------------------------------------- time bookkeeping
// the idx == 0 branches of the "a" kernels and calc_time_*: one thread
template <typename R>
__global__ void k_time(R *time, int kind, R K, R DT) {
  if (kind == 1) {
    time[1] = time[0] + K;
  } else if (kind == 2) {
    const R t0 = time[0] + DT;
    time[0] = t0;
    time[1] = t0;
  }
}

// ---------------------------------------------------------------- pointwise RK updates
enum PointwiseMode : int {
  PW_AXPY = 0,        // P = P + c1*Q                     (2N "b" kernels: b1 += B*b2)
  PW_2R = 1,          // P = P + c1*D; Q = P + c2*D       (2R "b" kernels)
  PW_SSP104_06 = 2,   // b3 = 0.04 b1 + 0.36 b2; b2 = 0.6 b1 + 0.4 b2
};

template <typename R>
__global__ void k_pointwise(long long n, int mode, R4<R> *P, R4<R> *Q, R4<R> *Dd, R c1, R c2, R *time,
                            int tkind, R tK, unsigned *counter) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) {
    if (mode == PW_AXPY) {
      const V3<R> p = ld3_plain(P + i), q = ld3_plain(Q + i);
      st3(P + i, V3<R>{p.x + c1 * q.x, p.y + c1 * q.y, p.z + c1 * q.z});
    } else if (mode == PW_2R) {
      const V3<R> p = ld3_plain(P + i), d = ld3_plain(Dd + i);
      const V3<R> pn = {p.x + c1 * d.x, p.y + c1 * d.y, p.z + c1 * d.z};
      st3(P + i, pn);
      st3(Q + i, V3<R>{pn.x + c2 * d.x, pn.y + c2 * d.y, pn.z + c2 * d.z});
    } else {
      // P = b1, Q = b2, Dd = b3
      const V3<R> b1 = ld3_plain(P + i), b2 = ld3_plain(Q + i);
      st3(Dd + i, V3<R>{(R)0.04 * b1.x + (R)0.36 * b2.x, (R)0.04 * b1.y + (R)0.36 * b2.y,
                        (R)0.04 * b1.z + (R)0.36 * b2.z});
      st3(Q + i, V3<R>{(R)0.60 * b1.x + (R)0.40 * b2.x, (R)0.60 * b1.y + (R)0.40 * b2.y,
                       (R)0.60 * b1.z + (R)0.40 * b2.z});
    }
  }
  if (tkind != 0) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      if (atomicAdd(counter, 1u) == gridDim.x - 1) {
        if (tkind == 1) {
          time[1] = time[0] + tK;
        }
        __threadfence();
        *counter = 0u;
      }
    }
  }
}

// ---------------------------------------------------------------- reductions
// Deterministic two-pass sums: a fixed grid of blocks writes one FP64 partial each (fixed
// element-to-thread assignment, warp-shuffle tree), then one block adds the partials in a
// fixed order.  Reruns are bitwise identical.
enum ReduceKind : int { RED_NORM2 = 0, RED_NORM2_DIFF = 1, RED_NORM2_S = 2, RED_DOT = 3 };

template <typename T>
struct ReduceArgs {
  int kind;
  long long n;          // nodes (padding entries are zero and skipped)
  int nx, ny;
  const R4<T> *va, *vb;
  const T *sa, *sb;
  const T *wx, *wy, *wz;  // per-axis mass weights (REAL)D/M_INV[row] (kernel_operator.cl:26-28)
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <typename T>
__device__ __forceinline__ double reduce_term(const ReduceArgs<T> &a, long long i) {
  if (a.kind == RED_DOT) return (double)(a.sa[i] * a.sb[i]);
  const int ix = (int)(i % a.nx);
  const long long r = i / a.nx;
  const int iy = (int)(r % a.ny);
  const int iz = (int)(r / a.ny);
  const T fac = (a.wx[ix] * a.wy[iy]) * a.wz[iz];
  if (a.kind == RED_NORM2_S) return (double)((fac * a.sa[i]) * a.sa[i]);
  V3<T> v = ld3(a.va + i);
  if (a.kind == RED_NORM2_DIFF) {
    const V3<T> w = ld3(a.vb + i);
    v = {v.x - w.x, v.y - w.y, v.z - w.z};
  }
  return (double)(fac * ((v.x * v.x + v.y * v.y) + v.z * v.z));
}

template <typename T>
__global__ void __launch_bounds__(256) k_reduce_partials(const ReduceArgs<T> a, double *partials) {
  __shared__ double sm[8];
  double acc = 0.0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.n; i += stride)
    acc += reduce_term(a, i);
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
    v = warp_sum(v);
    if (threadIdx.x == 0) partials[blockIdx.x] = v;
  }
}

// sum of `np` partials in a fixed order by one block; the total goes to *total (FP64) and,
// if out_real is given, to out_real[0] with zeros in out_real[1..n_zero-1]
template <typename T>
__global__ void __launch_bounds__(256) k_reduce_final(const double *partials, int np, double *total, T *out_real,
                                                      long long n_zero, int accumulate) {
  __shared__ double sm[8];
  double acc = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) acc += partials[i];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += sm[w];
    if (total) *total = v;
    if (out_real) out_real[0] = accumulate ? (T)((double)out_real[0] + v) : (T)v;
  }
  if (out_real && !accumulate)
    for (long long i = 1 + threadIdx.x; i < n_zero; i += blockDim.x) out_real[i] = (T)0;
}

// ---------------------------------------------------------------- operators
// Generic-row SBP operators for the diagnostics and divergence cleaning.  R is the
// precision of the vector field, S the precision of scalar fields and arithmetic.
struct OpDesc {
  int nb, sw;          // derivative rows
  int periodic;
};

template <typename R, typename S>
struct OpArgs {
  Mesh m;
  OpDesc op;
  int off;                  // BNODES offset of the CG interior range
  int gx, gy, gz;           // NDRange
  const R4<R> *v;           // vector input
  const S *s;               // scalar input
  R4<R> *vout;
  S *sout;
  const S *D;               // derivative rows [2nb+1][sw] in S
  const S *Dadj;
  S dS[3];                  // (S)DX ...
  int adjoint;              // projector with the least-norm Laplacian
};

template <typename S>
__device__ __forceinline__ int nbr_rt(int i, int o, int n, int periodic) {
  int j = i + o;
  if (periodic) {
    j += (j < 0) ? n : 0;
    j -= (j >= n) ? n : 0;
  } else if (j < 0 || j >= n) {
    j = i;
  }
  return j;
}

// d/d(axis) of one component (comp < 0: scalar field) with rows `tab`, divided by (S)d
template <typename R, typename S>
__device__ S diff_rt(const OpArgs<R, S> &a, const S *tab, int ax, int comp, int ix, int iy, int iz) {
  const int ii[3] = {ix, iy, iz};
  const int nn[3] = {a.m.nx, a.m.ny, a.m.nz};
  const long long st[3] = {1, a.m.nx, (long long)a.m.nx * a.m.ny};
  const long long idx = ix + (long long)a.m.nx * (iy + (long long)a.m.ny * iz);
  const int row = a.op.periodic ? a.op.nb : sbp_row(ii[ax], nn[ax], a.op.nb);
  const int c0 = (a.op.sw - 1) / 2;
  S v = 0;
  for (int c = 0; c < a.op.sw; ++c) {
    const S cf = tab[row * a.op.sw + c];
    if (cf == (S)0) continue;
    const long long j = idx + (long long)(nbr_rt<S>(ii[ax], c - c0, nn[ax], a.op.periodic) - ii[ax]) * st[ax];
    S f;
    if (comp < 0) f = a.s[j];
    else {
      const R *p = reinterpret_cast<const R *>(a.v + j);
      f = (S)p[comp];
    }
    v += cf * f;
  }
  return v / a.dS[ax];
}

// div (kernel_operator.cl:145, kernel_div_cleaning.cl:60 with off = BNODES)
template <typename R, typename S>
__global__ void k_div(const OpArgs<R, S> a) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x + a.off;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y + a.off;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z + a.off;
  if (ix >= a.gx + a.off || iy >= a.gy + a.off || iz >= a.gz + a.off) return;
  const long long idx = ix + (long long)a.m.nx * (iy + (long long)a.m.ny * iz);
  a.sout[idx] = (diff_rt(a, a.D, 0, 0, ix, iy, iz) + diff_rt(a, a.D, 1, 1, ix, iy, iz)) +
                diff_rt(a, a.D, 2, 2, ix, iy, iz);
}

// grad (kernel_operator.cl:170) and the projector (kernel_div_cleaning.cl:96-109):
// mode 0 writes grad(s) to vout; mode 1 adds it to vout.xyz; mode 2 subtracts grad_adj
template <typename R, typename S>
__global__ void k_grad(const OpArgs<R, S> a, int mode) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z;
  if (ix >= a.gx || iy >= a.gy || iz >= a.gz) return;
  const long long idx = ix + (long long)a.m.nx * (iy + (long long)a.m.ny * iz);
  const S *tab = mode == 2 ? a.Dadj : a.D;
  const S gx = diff_rt(a, tab, 0, -1, ix, iy, iz);
  const S gy = diff_rt(a, tab, 1, -1, ix, iy, iz);
  const S gz = diff_rt(a, tab, 2, -1, ix, iy, iz);
  if (mode == 0) {
    st3(a.vout + idx, V3<R>{(R)gx, (R)gy, (R)gz});
  } else {
    V3<R> b = ld3_plain(a.vout + idx);
    if (mode == 1) b = {(R)((S)b.x + gx), (R)((S)b.y + gy), (R)((S)b.z + gz)};
    else b = {(R)((S)b.x - gx), (R)((S)b.y - gy), (R)((S)b.z - gz)};
    R *p = reinterpret_cast<R *>(a.vout + idx);
    p[0] = b.x; p[1] = b.y; p[2] = b.z;   // .w untouched, as the reference's .xyz store
  }
}

// ---------------------------------------------------------------- conjugate gradients
template <typename S>
struct LapArgs {
  Mesh m;
  int nb, w, periodic, off, gx, gy, gz;
  const S *L;          // rows [2nb+1][w]
  S dd[3];             // (S)DX*(S)DX ...
  const S *in;
  S *out;
  double *partials;    // CG: block partials of <in, out>
};

// (-Laplace) of kernel_div_cleaning.cl:11-56 at one node, in the reference's order
template <typename S>
__device__ __forceinline__ S laplace_at(const LapArgs<S> &a, int ix, int iy, int iz, long long idx) {
  const int ii[3] = {ix, iy, iz};
  const int nn[3] = {a.m.nx, a.m.ny, a.m.nz};
  const long long st[3] = {1, a.m.nx, (long long)a.m.nx * a.m.ny};
  int row[3];
  for (int ax = 0; ax < 3; ++ax) row[ax] = a.periodic ? a.nb : sbp_row(ii[ax], nn[ax], a.nb);
  const int c0 = (a.w - 1) / 2;
  S val = 0;
  for (int c = 0; c < a.w; ++c) {
    S t[3];
    for (int ax = 0; ax < 3; ++ax) {
      const S cf = a.L[row[ax] * a.w + c];
      const long long j = idx + (long long)(nbr_rt<S>(ii[ax], c - c0, nn[ax], a.periodic) - ii[ax]) * st[ax];
      t[ax] = (cf * a.in[j]) / a.dd[ax];
    }
    val = ((val + t[0]) + t[1]) + t[2];
  }
  return val;
}

// calc_laplace_divcleaning over the CG interior (kernel_div_cleaning.cl:75-84)
template <typename S>
__global__ void __launch_bounds__(256) k_laplace(const LapArgs<S> a) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x + a.off;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y + a.off;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z + a.off;
  if (ix >= a.gx + a.off || iy >= a.gy + a.off || iz >= a.gz + a.off) return;
  const long long idx = ix + (long long)a.m.nx * (iy + (long long)a.m.ny * iz);
  a.out[idx] = laplace_at(a, ix, iy, iz, idx);
}

// x = a*x + y (calc_axpy, kernel_CG.cl:8) or x = x + a*y (calc_xpay, kernel_CG.cl:21) over
// the interior; `a` is a device scalar as in the reference
template <typename S>
__global__ void k_axpy_interior(Mesh m, int off, int gx, int gy, int gz, S *x, const S *y, const S *a, int xpay,
                                S sign) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x + off;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y + off;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z + off;
  if (ix >= gx + off || iy >= gy + off || iz >= gz + off) return;
  const long long idx = ix + (long long)m.nx * (iy + (long long)m.ny * iz);
  const S av = sign * a[0];
  x[idx] = xpay ? x[idx] + av * y[idx] : av * x[idx] + y[idx];
}

// ---- device-resident CG loop (matlab/+induction_eq/clean_div.m:47-73).  The scalars live
// in CgState; every kernel returns at once when `done` is set, so a fixed-length chunk of
// iterations can be replayed from a CUDA graph and stops exactly where the host loop would.
// The dot products are fused into the stencil/update kernels: each block writes a partial,
// and the last block to finish (ticket counter) adds the partials in a fixed order.
struct CgState {
  double rr;         // residual_norm2
  double old;        // old_residual_norm2
  double tol;        // absolute_error_threshold^2
  double alpha;
  int it;            // iterations
  int max_it;
  int done;
  int pad;
};

// sum of np partials in a fixed order by the calling block (all threads get the total)
__device__ __forceinline__ double block_sum_partials(const double *partials, int np) {
  __shared__ double sm[32];
  __shared__ double total;
  const int tx = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  double acc = 0.0;
  for (int i = tx; i < np; i += nt) acc += partials[i];
  acc = warp_sum(acc);
  if ((tx & 31) == 0) sm[tx >> 5] = acc;
  __syncthreads();
  if (tx == 0) {
    double v = 0.0;
    for (int w = 0; w < nt >> 5; ++w) v += sm[w];
    total = v;
  }
  __syncthreads();
  return total;
}

// block partial of v, written to partials[block]; returns true in the last block to finish
__device__ __forceinline__ bool block_partial_and_ticket(double v, double *partials, unsigned *counter) {
  __shared__ double sm[32];
  __shared__ bool last;
  const int tx = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  v = warp_sum(v);
  if ((tx & 31) == 0) sm[tx >> 5] = v;
  __syncthreads();
  if (tx == 0) {
    double s = 0.0;
    for (int w = 0; w < nt >> 5; ++w) s += sm[w];
    partials[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = s;
    __threadfence();
    const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
    last = atomicAdd(counter, 1u) == nb - 1;
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// The same operator for the device-resident CG loop, with the row width W fixed at compile
// time and the coefficients pre-divided by DX^2, DY^2, DZ^2 (Ls[axis][row][c] = L[row][c] /
// dd[axis]; Li: the interior row of each axis): a multiply per term instead of the
// reference's division (cf * u) / dd.  Every term differs from the reference's by at most
// a rounding of the scaled coefficient; the sum runs in the reference's order.
template <int W>
struct LapFastArgs {
  double Li[3][W];
  const double *Ls;   // [3][2nb+1][W]
};
// ---- the two passes of one CG iteration inside a graph loop (a conditional WHILE node
// whose condition the last block of pass B sets; no host round trip per iteration).
//
// Pass A (clean_div.m:50-56): the search direction u = beta*u + r (calc_axpy) is formed at
// every stencil point as it is loaded -- u and r are read, the new direction is written at the
// node into the other buffer of a ping-pong pair (iteration parity) -- and lap = (-Laplace) u,
// <u, lap> and alpha = rr / <u, lap> (last block) follow in the same pass.  The direction value
// at a point is __fma_rn(beta, u, r) wherever it is formed, so every node's u is one value.
// Non-periodic grids: a node whose y and z rows are interior (warp-uniform for x-rows of
// threads) takes fixed y/z offsets and only its x coefficient from the row table (boundary
// rows in x no longer send a warp down a second path).
template <int W>
__device__ __forceinline__ double cg_dir(const double *uo, const double *r, double beta, long long j) {
  return __fma_rn(beta, __ldg(uo + j), __ldg(r + j));
}
template <int W>
__device__ __forceinline__ double laplace_dir_at(const LapArgs<double> &a, const LapFastArgs<W> &f, const double *uo,
                                                 const double *r, double beta, int ix, int iy, int iz, long long idx) {
  constexpr int C0 = (W - 1) / 2;
  const int ii[3] = {ix, iy, iz};
  const int nn[3] = {a.m.nx, a.m.ny, a.m.nz};
  const long long st[3] = {1, a.m.nx, (long long)a.m.nx * a.m.ny};
  const int rows = 2 * a.nb + 1;
  int row[3];
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) row[ax] = a.periodic ? a.nb : sbp_row(ii[ax], nn[ax], a.nb);
  double val = 0;
  if (!a.periodic && row[1] == a.nb && row[2] == a.nb) {
    const double *lx = f.Ls + (long long)row[0] * W;   // axis 0 rows come first in Ls
#pragma unroll
    for (int c = 0; c < W; ++c) {
      int jx = ix + c - C0;
      jx = (jx < 0 || jx >= nn[0]) ? ix : jx;   // clamp-to-self: its coefficient is zero
      const double t0 = cg_dir<W>(uo, r, beta, idx + (jx - ix)) * lx[c];
      const double t1 = cg_dir<W>(uo, r, beta, idx + (long long)(c - C0) * st[1]) * f.Li[1][c];
      const double t2 = cg_dir<W>(uo, r, beta, idx + (long long)(c - C0) * st[2]) * f.Li[2][c];
      val = ((val + t0) + t1) + t2;
    }
    return val;
  }
#pragma unroll
  for (int c = 0; c < W; ++c) {
    double t[3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      const double cf = f.Ls[(ax * rows + row[ax]) * W + c];
      const long long j = idx + (long long)(nbr_rt<double>(ii[ax], c - C0, nn[ax], a.periodic) - ii[ax]) * st[ax];
      t[ax] = cg_dir<W>(uo, r, beta, j) * cf;
    }
    val = ((val + t[0]) + t[1]) + t[2];
  }
  return val;
}

template <int W>
__global__ void __launch_bounds__(256) k_cg_pass_a(const LapArgs<double> a, const LapFastArgs<W> f, const double *r,
                                                   double *u0, double *u1, CgState *cs, unsigned *counter) {
  if (cs->done) return;   // (host-driven iterations past convergence)
  const int it = cs->it;
  const double *uo = (it & 1) ? u1 : u0;
  double *un = (it & 1) ? u0 : u1;
  const double beta = cs->rr / cs->old;
  const int ix = blockIdx.x * blockDim.x + threadIdx.x + a.off;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y + a.off;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z + a.off;
  double prod = 0.0;
  if (ix < a.gx + a.off && iy < a.gy + a.off && iz < a.gz + a.off) {
    const long long idx = ix + (long long)a.m.nx * (iy + (long long)a.m.ny * iz);
    const double val = laplace_dir_at<W>(a, f, uo, r, beta, ix, iy, iz, idx);
    const double uc = cg_dir<W>(uo, r, beta, idx);
    un[idx] = uc;
    a.out[idx] = val;
    prod = uc * val;
  }
  if (block_partial_and_ticket(prod, a.partials, counter)) {
    const int np = gridDim.x * gridDim.y * gridDim.z;
    const double ul = block_sum_partials(a.partials, np);
    if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
      cs->alpha = cs->rr / ul;
      *counter = 0u;
    }
  }
}

// Pass A as a 2.5D kernel: a CTA of kCgTX x kCgTY threads owns a tile of x-y columns of the
// CG interior and marches through a chunk of z planes.  Every thread keeps the direction
// values of its column at planes z - C0 .. z + C0 in a register queue (the z terms), and the
// plane z of the tile with its x and y halos (C0 deep) sits in shared memory (the x and y
// terms), so each direction value is formed (__fma_rn(beta, u, r)) and loaded from global
// memory about once per node instead of once per stencil point.  Values outside the grid are
// 0 (their coefficient is 0, where the reference reads the node itself); periodic grids wrap.
// The terms are summed in the order of laplace_dir_at: per row entry c, ((val + x) + y) + z.
constexpr int kCgTX = 32, kCgTY = 8;

// the direction value at global node (x, y, z): 0 outside the grid (non-periodic)
__device__ __forceinline__ double cg_dir_at(const LapArgs<double> &a, const double *uo, const double *r, double beta,
                                            int x, int y, int z) {
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  if (a.periodic) {
    x += x < 0 ? nx : 0; x -= x >= nx ? nx : 0;
    y += y < 0 ? ny : 0; y -= y >= ny ? ny : 0;
    z += z < 0 ? nz : 0; z -= z >= nz ? nz : 0;
  } else if (x < 0 || x >= nx || y < 0 || y >= ny || z < 0 || z >= nz) {
    return 0.0;
  }
  const long long j = x + (long long)nx * (y + (long long)ny * z);
  return __fma_rn(beta, __ldg(uo + j), __ldg(r + j));
}

template <int W>
__global__ void __launch_bounds__(kCgTX * kCgTY) k_cg_pass_a_z(const LapArgs<double> a, const LapFastArgs<W> f,
                                                                const double *r, double *u0, double *u1, CgState *cs,
                                                                unsigned *counter, int tz) {
  if (cs->done) return;   // (host-driven iterations past convergence)
  constexpr int C0 = (W - 1) / 2;
  constexpr int SX = kCgTX + 2 * C0, SY = kCgTY + 2 * C0;
  __shared__ double pl[SY][SX];
  const int it = cs->it;
  const double *uo = (it & 1) ? u1 : u0;
  double *un = (it & 1) ? u0 : u1;
  const double beta = cs->rr / cs->old;
  const int tx = threadIdx.x % kCgTX, ty = threadIdx.x / kCgTX;
  const int x0 = a.off + blockIdx.x * kCgTX, y0 = a.off + blockIdx.y * kCgTY;
  const int zb = a.off + blockIdx.z * tz;
  const int ze = min(zb + tz, a.off + a.gz);
  const int ix = x0 + tx, iy = y0 + ty;
  const bool mine = ix < a.off + a.gx && iy < a.off + a.gy;
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const int rows = 2 * a.nb + 1;
  const int rx = a.periodic ? a.nb : sbp_row(ix, nx, a.nb);
  const int ry = a.periodic ? a.nb : sbp_row(iy, ny, a.nb);
  const double *lx = f.Ls + ((long long)0 * rows + rx) * W;
  const double *ly = f.Ls + ((long long)1 * rows + ry) * W;
  double q[W];
#pragma unroll
  for (int k = 0; k < W - 1; ++k) q[k + 1] = mine ? cg_dir_at(a, uo, r, beta, ix, iy, zb - C0 + k) : 0.0;
  double prod = 0.0;
  for (int z = zb; z < ze; ++z) {
#pragma unroll
    for (int k = 0; k < W - 1; ++k) q[k] = q[k + 1];
    q[W - 1] = mine ? cg_dir_at(a, uo, r, beta, ix, iy, z + C0) : 0.0;
    // the tile of plane z (own column: the queue centre) and its x / y halos
    // (a thread past the interior holds the value of its own grid position: 0 on a box, the
    // wrapped value on a periodic grid)
    pl[ty + C0][tx + C0] = mine ? q[C0] : cg_dir_at(a, uo, r, beta, ix, iy, z);
    for (int h = threadIdx.x; h < 2 * C0 * kCgTY + 2 * C0 * kCgTX; h += kCgTX * kCgTY) {
      int px, py;
      if (h < 2 * C0 * kCgTY) {   // x halo: C0 columns on each side of every tile row
        const int side = h / (C0 * kCgTY), rem = h % (C0 * kCgTY);
        py = C0 + rem / C0;
        px = side ? kCgTX + C0 + rem % C0 : rem % C0;
      } else {                     // y halo: C0 rows above and below the tile's columns
        const int g = h - 2 * C0 * kCgTY;
        const int side = g / (C0 * kCgTX), rem = g % (C0 * kCgTX);
        px = C0 + rem % kCgTX;
        py = side ? kCgTY + C0 + rem / kCgTX : rem / kCgTX;
      }
      pl[py][px] = cg_dir_at(a, uo, r, beta, x0 - C0 + px, y0 - C0 + py, z);
    }
    __syncthreads();
    if (mine) {
      const int rz = a.periodic ? a.nb : sbp_row(z, nz, a.nb);
      const double *lz = f.Ls + ((long long)2 * rows + rz) * W;
      double val = 0.0;
#pragma unroll
      for (int c = 0; c < W; ++c) {
        const double t0 = pl[ty + C0][tx + c] * lx[c];
        const double t1 = pl[ty + c][tx + C0] * ly[c];
        const double t2 = q[c] * lz[c];
        val = ((val + t0) + t1) + t2;
      }
      const long long idx = ix + (long long)nx * (iy + (long long)ny * z);
      un[idx] = q[C0];
      a.out[idx] = val;
      prod += q[C0] * val;
    }
    __syncthreads();
  }
  if (block_partial_and_ticket(prod, a.partials, counter)) {
    const int np = gridDim.x * gridDim.y * gridDim.z;
    const double ul = block_sum_partials(a.partials, np);
    if (threadIdx.x == 0) {
      cs->alpha = cs->rr / ul;
      *counter = 0u;
    }
  }
}

// Pass B (clean_div.m:57-66): phi += alpha*u (calc_xpay), r -= alpha*lap, rr = <r, r> (last
// block), then the loop condition of clean_div.m:47, written to the graph loop's condition.
// NPT nodes per thread, blockDim.x apart along x (independent loads in flight per thread).
template <typename S, int NPT>
__global__ void __launch_bounds__(256) k_cg_pass_b(Mesh m, int off, int gx, int gy, int gz, S *phi, S *r,
                                                   const S *u0, const S *u1, const S *lap, double *partials,
                                                   CgState *cs, unsigned *counter, double *history,
                                                   cudaGraphConditionalHandle loop, int in_loop) {
  if (cs->done) return;                  // (host-driven iterations past convergence)
  const S *u = (cs->it & 1) ? u0 : u1;   // the direction pass A of this iteration wrote
  const S alpha = (S)cs->alpha;
  const int ix0 = blockIdx.x * blockDim.x * NPT + threadIdx.x + off;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y + off;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z + off;
  double rr = 0.0;
  if (iy < gy + off && iz < gz + off) {
    const long long row = (long long)m.nx * (iy + (long long)m.ny * iz);
#pragma unroll
    for (int k = 0; k < NPT; ++k) {
      const int ix = ix0 + k * (int)blockDim.x;
      if (ix < gx + off) {
        const long long idx = ix + row;
        phi[idx] = phi[idx] + alpha * u[idx];
        const S rn = r[idx] + (-alpha) * lap[idx];
        r[idx] = rn;
        rr += (double)rn * (double)rn;
      }
    }
  }
  if (block_partial_and_ticket(rr, partials, counter)) {
    const int np = gridDim.x * gridDim.y * gridDim.z;
    const double tot = block_sum_partials(partials, np);
    if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
      cs->old = cs->rr;
      cs->rr = tot;
      cs->it += 1;
      if (history) history[cs->it] = tot;
      cs->done = !(tot > cs->tol && cs->it < cs->max_it);
      if (in_loop) cudaGraphSetConditional(loop, cs->done ? 0u : 1u);
      *counter = 0u;
    }
  }
}

// the loop state of one cleaning: tolerance and cap (set on the device, so that a captured
// cleaning needs no host copy)
static __global__ void k_cg_init(CgState *cs, double tol, int max_it) {
  if (threadIdx.x == 0) {
    CgState s{};
    s.tol = tol;
    s.max_it = max_it;
    *cs = s;
  }
}

// initial residual r = div B: rr = <r, r> from reduction partials, the loop condition, and
// the graph loop's condition (no iteration when the field is already clean)
static __global__ void k_cg_start_loop(const double *partials_rr, int np, CgState *cs, double *history,
                                       cudaGraphConditionalHandle loop, int in_loop) {
  const double rr = block_sum_partials(partials_rr, np);
  if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
    cs->rr = rr;
    cs->old = 1.0;
    cs->it = 0;
    if (history) history[0] = rr;
    cs->done = !(rr > cs->tol && cs->it < cs->max_it);
    if (in_loop) cudaGraphSetConditional(loop, cs->done ? 0u : 1u);
  }
}

// any non-zero x/y/z component (decides whether the convection terms can vanish)
template <typename R>
__global__ void k_any_nonzero(long long n, const R4<R> *v, int *flag) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const V3<R> x = ld3(v + i);
  if (x.x != (R)0 || x.y != (R)0 || x.z != (R)0) *flag = 1;
}

// finiteness check of a vector field (sets *flag if any x/y/z is not finite)
template <typename R>
__global__ void k_check_finite(long long n, const R4<R> *v, int *flag) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const V3<R> x = ld3(v + i);
  if (!isfinite(x.x) || !isfinite(x.y) || !isfinite(x.z)) *flag = 1;
}

}  // namespace ieq
