// stage_x2.cuh -- the column kernels with several x-adjacent nodes per thread.
//
// The kernels of a stage (the curl kernel J = curl(B)/rho, E = J x B and the dissipation
// sum H; the stage kernel gathering the flux rows) are bound by load issue and load latency,
// not by DRAM bandwidth, at the sizes of this path: the FP32 build, with half the bytes, was
// only a few per cent faster with one node per thread.  Here each thread owns K nodes
// (ix .. ix + K - 1, ix a multiple of K; K = 2 in FP64 and FP32, K = 4 in FP32 on large
// grids).  Every y and z stencil point of the K nodes comes from one vector load (16 bytes),
// and their x stencils from 2*QL+1 vector loads covering ix-K*QL .. ix+K*QL+K-1
// (QL = ceil(RI/K)), instead of one scalar load per point and node: about half the load
// instructions and address arithmetic per node with pairs.
//
//   k_curl_e_x2     curl, E and (HODS) H                              periodic grids; FP32 boxes
//   k_stage_hall_x2 Hall stage without convection, H precomputed    every grid
//   k_stage_col_x2  general stage (convection; flux mask fixed at    periodic Hall; Hall +
//                   compile time for the default forms)               convection, rotation: every grid
//   k_stage_xband / k_curl_xband   the x boundary columns of a box, one node per thread,
//                   beside the pair kernels launched over the interior x range (XBAND)
//
// Each node's sums are formed term by term in the order of the one-node kernels
// (k_curl_e, k_curl_e_hod, k_stage_col); the results agree with them up to the compiler's
// choice of fused multiply-adds.
//
// A launcher uses these kernels only where every vector load is aligned and stays in one row
// (nx a multiple of K, each field's component stride a multiple of K, bases aligned to K
// elements) and where they measured faster (stage_inst.cuh).  Without XBAND, x-boundary rows
// of a box (and groups whose x window would leave the row) take the one-node code per node.
#pragma once
#include "stage_col.cuh"

namespace ieq {

template <typename R>
struct Pair2;
template <>
struct Pair2<double> {
  using T = double2;
};
template <>
struct Pair2<float> {
  using T = float2;
};

// the values at j and j + 1 (j even) through the read-only path
template <typename R>
__device__ __forceinline__ void ld_pair(const R *p, R &v0, R &v1) {
  const typename Pair2<R>::T v = __ldg(reinterpret_cast<const typename Pair2<R>::T *>(p));
  v0 = v.x;
  v1 = v.y;
}
// the same through the ordinary path (fields the kernel also writes)
template <typename R>
__device__ __forceinline__ void ld_pair_plain(const R *p, R &v0, R &v1) {
  const typename Pair2<R>::T v = *reinterpret_cast<const typename Pair2<R>::T *>(p);
  v0 = v.x;
  v1 = v.y;
}
template <typename R>
__device__ __forceinline__ void st_pair(R *p, R v0, R v1) {
  typename Pair2<R>::T v;
  v.x = v0;
  v.y = v1;
  *reinterpret_cast<typename Pair2<R>::T *>(p) = v;
}
template <typename R>
__device__ __forceinline__ void ldf_pair(const SoA<R> &f, long long j, V3<R> &a, V3<R> &b) {
  ld_pair(f.p + j, a.x, b.x);
  ld_pair(f.p + j + f.s, a.y, b.y);
  ld_pair(f.p + j + 2 * f.s, a.z, b.z);
}
template <typename R>
__device__ __forceinline__ void ldf_pair_plain(const SoA<R> &f, long long j, V3<R> &a, V3<R> &b) {
  ld_pair_plain(f.p + j, a.x, b.x);
  ld_pair_plain(f.p + j + f.s, a.y, b.y);
  ld_pair_plain(f.p + j + 2 * f.s, a.z, b.z);
}
template <typename R>
__device__ __forceinline__ void stf_pair(const SoA<R> &f, long long j, const V3<R> &a, const V3<R> &b) {
  st_pair(f.p + j, a.x, b.x);
  st_pair(f.p + j + f.s, a.y, b.y);
  st_pair(f.p + j + 2 * f.s, a.z, b.z);
}
template <typename R>
__device__ __forceinline__ R &cref(V3<R> &v, int c) {
  return c == 0 ? v.x : (c == 1 ? v.y : v.z);
}

// K consecutive values (K = 2: FP64 or FP32 pairs; K = 4: FP32 quads) in one vector load
template <typename R, int K>
struct VecK;
template <>
struct VecK<double, 2> {
  using T = double2;
};
template <>
struct VecK<float, 2> {
  using T = float2;
};
template <>
struct VecK<float, 4> {
  using T = float4;
};
template <typename R, int K>
__device__ __forceinline__ void unpack_k(const typename VecK<R, K>::T &v, R (&o)[K]) {
  o[0] = v.x;
  o[1] = v.y;
  if constexpr (K == 4) {
    o[2] = v.z;
    o[3] = v.w;
  }
}
// the values at j .. j + K - 1 (j a multiple of K) through the read-only path
template <typename R, int K>
__device__ __forceinline__ void ld_k(const R *p, R (&o)[K]) {
  unpack_k<R, K>(__ldg(reinterpret_cast<const typename VecK<R, K>::T *>(p)), o);
}
template <typename R, int K>
__device__ __forceinline__ void ld_k_plain(const R *p, R (&o)[K]) {
  unpack_k<R, K>(*reinterpret_cast<const typename VecK<R, K>::T *>(p), o);
}
template <typename R, int K>
__device__ __forceinline__ void st_k(R *p, const R (&o)[K]) {
  typename VecK<R, K>::T v;
  v.x = o[0];
  v.y = o[1];
  if constexpr (K == 4) {
    v.z = o[2];
    v.w = o[3];
  }
  *reinterpret_cast<typename VecK<R, K>::T *>(p) = v;
}
template <typename R, int K, bool PLAIN = false>
__device__ __forceinline__ void ldf_k(const SoA<R> &f, long long j, V3<R> (&a)[K]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    R t[K];
    if (PLAIN) ld_k_plain<R, K>(f.p + j + c * f.s, t);
    else ld_k<R, K>(f.p + j + c * f.s, t);
#pragma unroll
    for (int k = 0; k < K; ++k) cref(a[k], c) = t[k];
  }
}
template <typename R, int K>
__device__ __forceinline__ void stf_k(const SoA<R> &f, long long j, const V3<R> (&a)[K]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    R t[K];
#pragma unroll
    for (int k = 0; k < K; ++k) t[k] = cmp(a[k], c);
    st_k<R, K>(f.p + j + c * f.s, t);
  }
}

// the x window of one component for the K nodes row0 + ix .. row0 + ix + K - 1:
// w[m] = f[row0 + ix - K*QL + m], m = 0 .. K*(2QL+1) - 1, periodic wrap of the group starts
template <typename R, int K, int QL, bool PER>
__device__ __forceinline__ void x_window_k(const R *f, long long row0, int ix, int nx, R (&w)[K * (2 * QL + 1)]) {
#pragma unroll
  for (int q = -QL; q <= QL; ++q) {
    int xx = ix + K * q;
    if (PER) {
      xx += xx < 0 ? nx : 0;
      xx -= xx >= nx ? nx : 0;
    }
    R t[K];
    ld_k<R, K>(f + row0 + xx, t);
#pragma unroll
    for (int k = 0; k < K; ++k) w[K * (q + QL) + k] = t[k];
  }
}

// whether the group's x stencils may use the window (all K nodes on the interior row and
// the window inside the row; always with periodic wrap)
template <int OP, bool PER, int K>
__device__ __forceinline__ bool x_group_interior(int ix, int nx) {
  constexpr int NB = Op<OP>::NB, QL = (Op<OP>::RI + K - 1) / K;
  if (PER) return true;
  return sbp_row(ix, nx, NB) == NB && sbp_row(ix + K - 1, nx, NB) == NB && ix - K * QL >= 0 &&
         ix + K * QL + K - 1 < nx;
}

// whether the pair's x stencils may use the window (both nodes on the interior row and
// the window inside the row; always with periodic wrap)
template <int OP, bool PER>
__device__ __forceinline__ bool x_pair_interior(int ix, int nx) {
  constexpr int NB = Op<OP>::NB, QL = (Op<OP>::RI + 1) / 2;
  if (PER) return true;
  return sbp_row(ix, nx, NB) == NB && sbp_row(ix + 1, nx, NB) == NB && ix - 2 * QL >= 0 && ix + 2 * QL + 1 < nx;
}

// Boxes: the x boundary columns in a band of their own.  A pair kernel launched with XBAND
// covers only the nodes xband(OP) <= ix < nx - xband(OP), whose x stencils are all interior
// rows inside the row (no per-node fallback, no SAT on the x faces in its warps); the 2 *
// xband(OP) boundary columns of every row run one node per thread in k_stage_xband, which
// also does the stage's time bookkeeping.  xband is even, >= NUM_BOUNDS and >= the pair
// window's reach 2*ceil(RI/2).
template <int OP>
__host__ __device__ constexpr int xband() {
  constexpr int nb = Op<OP>::NB + (Op<OP>::NB & 1), w = 2 * ((Op<OP>::RI + 1) / 2);
  return nb > w ? nb : w;
}

// resident 128-thread blocks per SM the register allocation targets (measured on B200 at
// 64^3 and 128^3, FP64: the curl kernel is fastest with 4 blocks of <= 128 registers and
// no spills, 15-25 % ahead of 5 or 6 blocks with spills; the stage kernel with 7 blocks of
// <= 72 registers, 3-7 % ahead of 8 blocks of 64 -- at 64^3 its 1024 blocks then fit in one
// wave of 148 x 7)
#ifndef IEQ_CURL_X2_MIN_BLOCKS
#define IEQ_CURL_X2_MIN_BLOCKS 4
#endif
#ifndef IEQ_CURL_X2_PLAIN_MIN_BLOCKS
#define IEQ_CURL_X2_PLAIN_MIN_BLOCKS 8
#endif
#ifndef IEQ_STAGE_X2_MIN_BLOCKS
#define IEQ_STAGE_X2_MIN_BLOCKS 7
#endif
// FP32 with four nodes per thread (float4 loads; measured at 128^3: curl 4 blocks of <= 128
// registers, stage 7 blocks of <= 72: 22.9 / 29.5 us against 29.0 / 35.3 with pairs)
#ifndef IEQ_CURL_X4_MIN_BLOCKS
#define IEQ_CURL_X4_MIN_BLOCKS 4
#endif
#ifndef IEQ_STAGE_X4_MIN_BLOCKS
#define IEQ_STAGE_X4_MIN_BLOCKS 7
#endif

// whether FP32 runs four nodes per thread: only where a quarter of the nodes still fills
// the GPU (>= 2^20 nodes; at 64^3 the quads leave about 14 warps per SM and measured slower
// than pairs)
inline bool quads_fill(long long nodes) { return nodes >= (1ll << 20); }

// J = curl(B)/rho, E = J x B and (HODS) the dissipation sum H of B at K x-adjacent nodes
template <typename R, int OP, bool PER, bool HODS, int K = 2, bool XBAND = false>
__global__ void __launch_bounds__(kColThreads, HODS ? (K == 4 ? IEQ_CURL_X4_MIN_BLOCKS : IEQ_CURL_X2_MIN_BLOCKS)
                                                   : IEQ_CURL_X2_PLAIN_MIN_BLOCKS)
    k_curl_e_x2(const __grid_constant__ CurlArgs<R, SoA<R>> a) {
  constexpr int NB = Op<OP>::NB, SW = Op<OP>::SW, C0 = (SW - 1) / 2, WH = Op<OP>::WH, RI = Op<OP>::RI;
  constexpr int RB = HODS ? ((C0 > WH - 1) ? C0 : WH - 1) : C0;
  constexpr int QL = (RI + K - 1) / K;
  constexpr int X0 = XBAND ? xband<OP>() : 0;
  pdl_enter();
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const int ix = X0 + K * (blockIdx.x * blockDim.x + threadIdx.x);
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z;
  if (ix >= nx - X0 || iy >= ny || iz >= nz) return;
  const long long row0 = (long long)nx * (iy + (long long)ny * iz);
  const long long idx = row0 + ix;
  const long long cs = a.b.s;
  const V3<R> zero = {0, 0, 0};
  V3<R> Bm[K];
  ldf_k<R, K>(a.b, idx, Bm);
  R g[K][3][3];
  V3<R> hod[K];
#pragma unroll
  for (int k = 0; k < K; ++k) hod[k] = zero;

  // x
  {
    R v1[K], v2[K];
    V3<R> ho[K];
    if (XBAND || x_group_interior<OP, PER, K>(ix, nx)) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        v1[k] = 0;
        v2[k] = 0;
        ho[k] = zero;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (!HODS && c == 0) continue;   // the x derivatives of By and Bz only
        R w[K * (2 * QL + 1)];
        x_window_k<R, K, QL, PER>(a.b.p + c * cs, row0, ix, nx, w);
#pragma unroll
        for (int k = 0; k < K; ++k) {
#pragma unroll
          for (int o = -RI; o <= RI; ++o) {
            const R val = w[K * QL + k + o];
            if (o != 0) {
              if (c == 1) v1[k] += a.Dint[o + RI] * val;
              if (c == 2) v2[k] += a.Dint[o + RI] * val;
            }
            if (HODS) cref(ho[k], c) += a.Hint[o + RI] * val;
          }
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < K; ++k)
        curl_axis_node<R, OP, PER, HODS>(a, 0, ix + k, nx, idx + k, 1, Bm[k], v1[k], v2[k], ho[k]);
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      g[k][0][1] = v1[k] * a.inv_d[0];
      g[k][0][2] = v2[k] * a.inv_d[0];
      if (HODS) {
        hod[k].x += ho[k].x; hod[k].y += ho[k].y; hod[k].z += ho[k].z;
      }
    }
  }

  // y and z: all K nodes on the same row of the axis
  const int ii[3] = {ix, iy, iz};
  const int nn[3] = {nx, ny, nz};
  const long long st[3] = {1, nx, (long long)nx * ny};
#pragma unroll
  for (int ax = 1; ax < 3; ++ax) {
    const int c1 = (ax + 1) % 3, c2 = (ax + 2) % 3;
    const int i = ii[ax], n = nn[ax];
    R v1[K], v2[K];
    V3<R> ho[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      v1[k] = 0;
      v2[k] = 0;
      ho[k] = zero;
    }
    const int row = PER ? NB : sbp_row(i, n, NB);
    if (row == NB) {
      const bool wrap = PER && (i < RI || i >= n - RI);
#pragma unroll
      for (int o = -RI; o <= RI; ++o) {
        const R cH = a.Hint[o + RI];
        if (o == 0) {
          if (HODS) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
              ho[k].x += cH * Bm[k].x; ho[k].y += cH * Bm[k].y; ho[k].z += cH * Bm[k].z;
            }
          }
          continue;
        }
        const long long j = wrap ? idx + (long long)(nbr<true>(i, o, n) - i) * st[ax] : idx + (long long)o * st[ax];
        const R c = a.Dint[o + RI];
        if (HODS) {
          V3<R> B[K];
          ldf_k<R, K>(a.b, j, B);
#pragma unroll
          for (int k = 0; k < K; ++k) {
            v1[k] += c * cmp(B[k], c1);
            v2[k] += c * cmp(B[k], c2);
            ho[k].x += cH * B[k].x; ho[k].y += cH * B[k].y; ho[k].z += cH * B[k].z;
          }
        } else {
          R p1[K], p2[K];
          ld_k<R, K>(a.b.p + j + c1 * cs, p1);
          ld_k<R, K>(a.b.p + j + c2 * cs, p2);
#pragma unroll
          for (int k = 0; k < K; ++k) {
            v1[k] += c * p1[k];
            v2[k] += c * p2[k];
          }
        }
      }
    } else {
      for (int o = -RB; o <= RB; ++o) {
        const R cD = (o >= -C0 && o <= C0) ? a.tab->D[row][o + C0] : (R)0;
        const R cH = (HODS && o >= -(WH - 1) && o <= WH - 1) ? a.tab->H[row][o + WH - 1] : (R)0;
        if (cD == (R)0 && cH == (R)0) continue;
        const long long j = idx + (long long)(nbr<PER>(i, o, n) - i) * st[ax];
        if (HODS) {
          V3<R> B[K];
          ldf_k<R, K>(a.b, j, B);
#pragma unroll
          for (int k = 0; k < K; ++k) {
            if (cD != (R)0) {
              v1[k] += cD * cmp(B[k], c1);
              v2[k] += cD * cmp(B[k], c2);
            }
            if (cH != (R)0) {
              ho[k].x += cH * B[k].x; ho[k].y += cH * B[k].y; ho[k].z += cH * B[k].z;
            }
          }
        } else {
          R p1[K], p2[K];
          ld_k<R, K>(a.b.p + j + c1 * cs, p1);
          ld_k<R, K>(a.b.p + j + c2 * cs, p2);
#pragma unroll
          for (int k = 0; k < K; ++k) {
            v1[k] += cD * p1[k];
            v2[k] += cD * p2[k];
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      g[k][ax][c1] = v1[k] * a.inv_d[ax];
      g[k][ax][c2] = v2[k] * a.inv_d[ax];
      if (HODS) {
        hod[k].x += ho[k].x; hod[k].y += ho[k].y; hod[k].z += ho[k].z;
      }
    }
  }

  R r[K];
  if (a.rho) ld_k<R, K>(a.rho + idx, r);
  V3<R> E[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    V3<R> J = {g[k][1][2] - g[k][2][1], g[k][2][0] - g[k][0][2], g[k][0][1] - g[k][1][0]};
    if (a.rho) {
      const R ri = (R)1 / r[k];
      J = {J.x * ri, J.y * ri, J.z * ri};
    }
    const V3<R> &B = Bm[k];
    E[k] = V3<R>{J.x * B.y - J.y * B.x, J.x * B.z - J.z * B.x, J.y * B.z - J.z * B.y};
    if (!PER && (ix + k == 0 || iy == 0 || iz == 0 || ix + k == nx - 1 || iy == ny - 1 || iz == nz - 1))
      stf(a.jface, idx + k, J);
  }
  stf_k<R, K>(a.out, idx, E);
  if (HODS) stf_k<R, K>(a.hout, idx, hod);
}

// the stage update of K nodes from DB (epilogue modes of stage_kernel.cuh), with vector loads
// and stores of the fields it combines
template <typename R, int K>
__device__ __forceinline__ void epilogue_load_k(const StageArgs<R, SoA<R>> &a, long long idx, EpIn<R> (&e)[K]) {
  const V3<R> zero = {0, 0, 0};
  V3<R> x[K], y[K];
#pragma unroll
  for (int k = 0; k < K; ++k) x[k] = y[k] = zero;
  switch (a.mode) {
    case EP_X_PLUS_HF:
    case EP_AX_HF:
    case EP_2R_FUSED:
      ldf_k<R, K, true>(a.X, idx, x);
      break;
    case EP_PX_QYHF:
      ldf_k<R, K, true>(a.X, idx, x);
      ldf_k<R, K, true>(a.Y, idx, y);
      break;
    case EP_2N_FUSED:
      ldf_k<R, K, true>(a.X, idx, x);
      ldf_k<R, K, true>(a.Z, idx, y);
      break;
    case EP_2N_FUSED_FIRST:
      ldf_k<R, K, true>(a.Z, idx, y);
      break;
    default:
      break;
  }
#pragma unroll
  for (int k = 0; k < K; ++k) e[k] = EpIn<R>{x[k], y[k]};
}
template <typename R, int K>
__device__ __forceinline__ void epilogue_store_k(const StageArgs<R, SoA<R>> &a, long long idx, const V3<R> (&d)[K],
                                                 const EpIn<R> (&e)[K]) {
  V3<R> o1[K], o2[K], o3[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const EpOut<R> o = epilogue_values(a, d[k], e[k]);
    o1[k] = o.o1;
    o2[k] = o.o2;
    o3[k] = o.o3;
  }
  stf_k<R, K>(a.out, idx, o1);
  if (epilogue_writes_out2(a.mode)) stf_k<R, K>(a.out2, idx, o2);
  if (a.mode == EP_2R_FUSED && a.out3.p) stf_k<R, K>(a.out3, idx, o3);
}
template <typename R, int K>
__device__ __forceinline__ void stage_epilogue_k(const StageArgs<R, SoA<R>> &a, long long idx, const V3<R> (&d)[K]) {
  EpIn<R> e[K];
  epilogue_load_k<R, K>(a, idx, e);
  epilogue_store_k<R, K>(a, idx, d, e);
}
template <typename R>
__device__ __forceinline__ void stage_epilogue_pair(const StageArgs<R, SoA<R>> &a, long long idx, const V3<R> &d0,
                                                    const V3<R> &d1) {
  const V3<R> d[2] = {d0, d1};
  stage_epilogue_k<R, 2>(a, idx, d);
}

// DB of a Hall stage without convection terms at K x-adjacent nodes, with the dissipation
// sum precomputed (HODP, read from a.Hpre) or absent, and the stage update
template <typename R, int OP, bool PER, bool HODP, int K = 2, bool XBAND = false>
__global__ void __launch_bounds__(kColThreads, K == 4 ? IEQ_STAGE_X4_MIN_BLOCKS : IEQ_STAGE_X2_MIN_BLOCKS)
    k_stage_hall_x2(const __grid_constant__ StageArgs<R, SoA<R>> a) {
  constexpr int NB = Op<OP>::NB, SW = Op<OP>::SW, C0 = (SW - 1) / 2, RI = Op<OP>::RI;
  constexpr int QL = (RI + K - 1) / K;
  constexpr int X0 = XBAND ? xband<OP>() : 0;
  pdl_enter();
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const int ix = X0 + K * (blockIdx.x * blockDim.x + threadIdx.x);
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z;
  if (ix < nx - X0 && iy < ny && iz < nz) {
    const long long row0 = (long long)nx * (iy + (long long)ny * iz);
    const long long idx = row0 + ix;
    const long long es = a.E.s;
    const V3<R> zero = {0, 0, 0};
    V3<R> db[K];
#pragma unroll
    for (int k = 0; k < K; ++k) db[k] = zero;

    // x: DB_y += D[Exy], DB_z += D[Exz]
    {
      ColSums<R> s[K];
#pragma unroll
      for (int k = 0; k < K; ++k) s[k] = ColSums<R>{};
      if (XBAND || x_group_interior<OP, PER, K>(ix, nx)) {
#pragma unroll
        for (int ci = 0; ci < 2; ++ci) {
          R w[K * (2 * QL + 1)];
          x_window_k<R, K, QL, PER>(a.E.p + (ci == 0 ? e_comp1(0) : e_comp2(0)) * es, row0, ix, nx, w);
#pragma unroll
          for (int k = 0; k < K; ++k) {
#pragma unroll
            for (int o = -RI; o <= RI; ++o) {
              if (o == 0) continue;
              if (ci == 0) s[k].h1 += a.Dint[o + RI] * w[K * QL + k + o];
              else s[k].h2 += a.Dint[o + RI] * w[K * QL + k + o];
            }
          }
        }
      } else {
#pragma unroll
        for (int k = 0; k < K; ++k)
          col_axis<R, OP, PER, true, false, 0>(s[k], a, 0, ix + k, nx, idx + k, 1, zero);
      }
#pragma unroll
      for (int k = 0; k < K; ++k) col_combine<R, true, false, 0>(a, 0, s[k], zero, zero, db[k], db[k]);
    }

    // y and z
    const int ii[3] = {ix, iy, iz};
    const int nn[3] = {nx, ny, nz};
    const long long st[3] = {1, nx, (long long)nx * ny};
#pragma unroll
    for (int ax = 1; ax < 3; ++ax) {
      const int i = ii[ax], n = nn[ax];
      const R *e1p = a.E.p + e_comp1(ax) * es, *e2p = a.E.p + e_comp2(ax) * es;
      ColSums<R> s[K];
#pragma unroll
      for (int k = 0; k < K; ++k) s[k] = ColSums<R>{};
      const int row = PER ? NB : sbp_row(i, n, NB);
      if (row == NB) {
        const bool wrap = PER && (i < RI || i >= n - RI);
#pragma unroll
        for (int o = -RI; o <= RI; ++o) {
          if (o == 0) continue;
          const long long j = wrap ? idx + (long long)(nbr<true>(i, o, n) - i) * st[ax] : idx + (long long)o * st[ax];
          R p1[K], p2[K];
          ld_k<R, K>(e1p + j, p1);
          ld_k<R, K>(e2p + j, p2);
          const R c = a.Dint[o + RI];
#pragma unroll
          for (int k = 0; k < K; ++k) {
            s[k].h1 += c * p1[k];
            s[k].h2 += c * p2[k];
          }
        }
      } else {
        for (int o = -C0; o <= C0; ++o) {
          const R cD = a.tab->D[row][o + C0];
          if (cD == (R)0) continue;
          const long long j = idx + (long long)(nbr<PER>(i, o, n) - i) * st[ax];
          R p1[K], p2[K];
          ld_k<R, K>(e1p + j, p1);
          ld_k<R, K>(e2p + j, p2);
#pragma unroll
          for (int k = 0; k < K; ++k) {
            s[k].h1 += cD * p1[k];
            s[k].h2 += cD * p2[k];
          }
        }
      }
#pragma unroll
      for (int k = 0; k < K; ++k) col_combine<R, true, false, 0>(a, ax, s[k], zero, zero, db[k], db[k]);
    }

    V3<R> hv[K];
#pragma unroll
    for (int k = 0; k < K; ++k) hv[k] = zero;
    if (HODP) ldf_k<R, K>(a.Hpre, idx, hv);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!PER) {
        const int iik[3] = {ix + k, iy, iz};
        stage_sat<R, SoA<R>, true>(a, iik, nn, idx + k, ldf(a.bk, idx + k), zero, 0, db[k]);
      }
      if (HODP) {
        db[k].x += a.hod_factor * hv[k].x;
        db[k].y += a.hod_factor * hv[k].y;
        db[k].z += a.hod_factor * hv[k].z;
      }
    }
    stage_epilogue_k<R, K>(a, idx, db);
  }
  stage_time_post(a);
}

// ---------------------------------------------------------------------------------------
// The general column stage kernel (convection sums, dissipation gathered here or
// precomputed, first-order / adaptive dissipation) with two x-adjacent nodes per thread.
// The x stencils stream through the pairs at ix + 2q, q = -QL .. QL: the pair's first value
// is offset 2q of node ix and offset 2q - 1 of node ix + 1, its second offsets 2q + 1 and 2q,
// so each node meets its offsets in ascending order -- the order of col_axis -- without a
// window kept in registers.  Every term goes through col_acc / col_combine, as in k_stage_col.

// the stencil-point values col_load reads, for both nodes of a pair at j, j + 1
template <typename R, bool HALL, bool HOD, int CONV>
__device__ __forceinline__ void col_load_pair(const StageArgs<R, SoA<R>> &a, int ax, long long j, V3<R> (&B)[2],
                                              V3<R> (&U)[2], R (&e1)[2], R (&e2)[2]) {
  if (CONV || HOD) ldf_pair(a.bk, j, B[0], B[1]);
  if (CONV) ldf_pair(a.u, j, U[0], U[1]);
  if (HALL) {
    ld_pair(a.E.p + j + e_comp1(ax) * a.E.s, e1[0], e1[1]);
    ld_pair(a.E.p + j + e_comp2(ax) * a.E.s, e2[0], e2[1]);
  }
}

// the x sums of the pair (ix, ix + 1) on the interior row (or with periodic wrap)
template <typename R, int OP, bool PER, bool HALL, bool HOD, int CONV, int NEED = -1, bool FOF = false>
__device__ __forceinline__ void col_x_pair(ColSums<R> (&s)[2], const StageArgs<R, SoA<R>> &a, long long row0, int ix,
                                           int nx, const V3<R> (*Bm)[2] = nullptr, const V3<R> (*Um)[2] = nullptr) {
  constexpr int RI = Op<OP>::RI, QL = (RI + 1) / 2;
  const int need = NEED >= 0 ? NEED : a.need;
  const V3<R> zero = {0, 0, 0};
#pragma unroll
  for (int q = -QL; q <= QL; ++q) {
    int xx = ix + 2 * q;
    if (PER) {
      xx += xx < 0 ? nx : 0;
      xx -= xx >= nx ? nx : 0;
    }
    V3<R> B[2] = {zero, zero}, U[2] = {zero, zero};
    R e1[2] = {0, 0}, e2[2] = {0, 0};
    col_load_pair<R, HALL, HOD, CONV>(a, 0, row0 + xx, B, U, e1, e2);
#pragma unroll
    for (int e = 0; e < 2; ++e) {
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int o = 2 * q + e - k;
        if (o < -RI || o > RI) continue;
        if (o == 0) {
          // the interior derivative rows have a zero centre (the value is the node's own B)
          if (HOD) col_acc<R, false, HOD, 0>(s[k], 0, 0, (R)0, a.Hint[RI], false, true, B[e], zero, (R)0, (R)0);
          continue;
        }
        col_acc<R, HALL, HOD, CONV>(s[k], 0, need, a.Dint[o + RI], a.Hint[o + RI], true, true, B[e], U[e], e1[e],
                                    e2[e]);
        if (FOF) fo_acc(s[k], a.Dint[o + RI], B[e], U[e], (*Bm)[k], (*Um)[k]);
      }
    }
  }
}

// the y or z sums of the pair (both nodes on the same row of the axis)
template <typename R, int OP, bool PER, bool HALL, bool HOD, int CONV, int NEED = -1, bool FOF = false>
__device__ __forceinline__ void col_yz_pair(ColSums<R> (&s)[2], const StageArgs<R, SoA<R>> &a, int ax, int i, int n,
                                            long long idx, long long st, const V3<R> (&Bm)[2],
                                            const V3<R> (*Um)[2] = nullptr) {
  constexpr int NB = Op<OP>::NB, SW = Op<OP>::SW, C0 = (SW - 1) / 2, WH = Op<OP>::WH, RI = Op<OP>::RI;
  constexpr int RB = (C0 > WH - 1) ? C0 : WH - 1;
  const int need = NEED >= 0 ? NEED : a.need;
  const V3<R> zero = {0, 0, 0};
  const int row = PER ? NB : sbp_row(i, n, NB);
  if (row == NB) {
    const bool wrap = PER && (i < RI || i >= n - RI);
#pragma unroll
    for (int o = -RI; o <= RI; ++o) {
      if (o == 0) {
        if (HOD) {
#pragma unroll
          for (int k = 0; k < 2; ++k)
            col_acc<R, false, HOD, 0>(s[k], ax, 0, (R)0, a.Hint[RI], false, true, Bm[k], zero, (R)0, (R)0);
        }
        continue;
      }
      const long long j = wrap ? idx + (long long)(nbr<true>(i, o, n) - i) * st : idx + (long long)o * st;
      V3<R> B[2] = {zero, zero}, U[2] = {zero, zero};
      R e1[2] = {0, 0}, e2[2] = {0, 0};
      col_load_pair<R, HALL, HOD, CONV>(a, ax, j, B, U, e1, e2);
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        col_acc<R, HALL, HOD, CONV>(s[k], ax, need, a.Dint[o + RI], a.Hint[o + RI], true, true, B[k], U[k], e1[k],
                                    e2[k]);
        if (FOF) fo_acc(s[k], a.Dint[o + RI], B[k], U[k], Bm[k], (*Um)[k]);
      }
    }
  } else {
    for (int o = -RB; o <= RB; ++o) {
      const R cD = (o >= -C0 && o <= C0) ? a.tab->D[row][o + C0] : (R)0;
      const R cH = (HOD && o >= -(WH - 1) && o <= WH - 1) ? a.tab->H[row][o + WH - 1] : (R)0;
      if (cD == (R)0 && cH == (R)0) continue;
      const long long j = idx + (long long)(nbr<PER>(i, o, n) - i) * st;
      V3<R> B[2] = {zero, zero}, U[2] = {zero, zero};
      R e1[2] = {0, 0}, e2[2] = {0, 0};
      col_load_pair<R, HALL, HOD, CONV>(a, ax, j, B, U, e1, e2);
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        col_acc<R, HALL, HOD, CONV>(s[k], ax, need, cD, cH, cD != (R)0, cH != (R)0, B[k], U[k], e1[k], e2[k]);
        if (FOF) fo_acc(s[k], cD, B[k], U[k], Bm[k], (*Um)[k]);
      }
    }
  }
}

#ifndef IEQ_COL_X2_MIN_BLOCKS
#define IEQ_COL_X2_MIN_BLOCKS 4
#endif
#ifndef IEQ_COL_X2_CONV_MIN_BLOCKS
#define IEQ_COL_X2_CONV_MIN_BLOCKS 4
#endif
// resident blocks the pair kernel with fused first-order dissipation (FOF) is compiled for,
// measured on B200 (Hall periodic 64^3 with variable u and the confined 64^3 box, CK2N54):
// boxes 4 (4th / 6th order 1.80e10 / 1.30e10 DOF/s against 1.67e10 / 1.25e10 with 3), periodic
// grids 3 at radius <= 2 (2.21e10 against 2.07e10 with 4 and 2.13e10 with 2) and 2 at radius 3
// (1.83e10 against 1.59e10 with 3 and 1.34e10 with 4): the periodic x window of a pair is
// loaded whole, and at radius 3 the first-order sums of both nodes spilled below 255 registers
#ifndef IEQ_COL_X2_FO_MIN_BLOCKS
#define IEQ_COL_X2_FO_MIN_BLOCKS 4
#endif
// resident blocks of the convection pair kernel with a compile-time flux-form mask: masks of
// three or four sums per axis (7, 13, 14, 15) get more registers (3 blocks of <= 168)
template <int NEED>
__host__ __device__ constexpr int conv_min_blocks() {
  return (NEED >= 0 && ((NEED & 1) + ((NEED >> 1) & 1) + ((NEED >> 2) & 1) + ((NEED >> 3) & 1)) >= 3)
             ? 3
             : IEQ_COL_X2_CONV_MIN_BLOCKS;
}
template <int OP, bool PER>
__host__ __device__ constexpr int fo_min_blocks() {
  return PER ? (Op<OP>::RI >= 3 ? 2 : 3) : IEQ_COL_X2_FO_MIN_BLOCKS;
}

// DB (volume, Hall, SAT, dissipation) and the stage update at the pair; template
// arguments as k_stage_col (CONV = 1: the convection sums; HODP: the dissipation sum read
// from a.Hpre; FOAD: first-order / adaptive dissipation; FOF: first-order dissipation with
// its terms summed in the gathers of the volume terms, which load the same B and u)
template <typename R, int OP, bool PER, bool HALL, bool HOD_, int CONV, bool HODP = false, bool FOAD = false,
          int NEED = -1, bool XBAND = false, bool FOF = false>
__global__ void __launch_bounds__(kColThreads, FOF ? fo_min_blocks<OP, PER>()
                                                   : (CONV ? conv_min_blocks<NEED>() : IEQ_COL_X2_MIN_BLOCKS))
    k_stage_col_x2(const __grid_constant__ StageArgs<R, SoA<R>> a) {
  static_assert(!FOF || (CONV && !FOAD), "the fused first-order terms need the convection loads");
  constexpr bool HOD = HOD_ && !HODP;   // the dissipation rows gathered in this kernel
  constexpr int X0 = XBAND ? xband<OP>() : 0;
  pdl_enter();
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const int ix = X0 + 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z;
  if (ix < nx - X0 && iy < ny && iz < nz) {
    const long long row0 = (long long)nx * (iy + (long long)ny * iz);
    const long long idx = row0 + ix;
    const V3<R> zero = {0, 0, 0};
    V3<R> Bm[2], um[2] = {zero, zero}, db[2] = {zero, zero}, hod[2] = {zero, zero}, fo[2] = {zero, zero};
    ldf_pair(a.bk, idx, Bm[0], Bm[1]);
    if (CONV) ldf_pair(a.u, idx, um[0], um[1]);
    {
      ColSums<R> s[2] = {ColSums<R>{}, ColSums<R>{}};
      if (XBAND || x_pair_interior<OP, PER>(ix, nx)) {
        col_x_pair<R, OP, PER, HALL, HOD, CONV, NEED, FOF>(s, a, row0, ix, nx, &Bm, &um);
      } else {
#pragma unroll
        for (int k = 0; k < 2; ++k)
          col_axis<R, OP, PER, HALL, HOD, CONV, SoA<R>, NEED, FOF>(s[k], a, 0, ix + k, nx, idx + k, 1, Bm[k], &um[k]);
      }
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        col_combine<R, HALL, HOD, CONV>(a, 0, s[k], Bm[k], um[k], db[k], hod[k]);
        if (FOF) fo_combine(a.dR, 0, s[k], fo[k]);
      }
    }
    const int nn[3] = {nx, ny, nz};
    const long long st[3] = {1, nx, (long long)nx * ny};
#pragma unroll
    for (int ax = 1; ax < 3; ++ax) {
      ColSums<R> s[2] = {ColSums<R>{}, ColSums<R>{}};
      col_yz_pair<R, OP, PER, HALL, HOD, CONV, NEED, FOF>(s, a, ax, ax == 1 ? iy : iz, nn[ax], idx, st[ax], Bm, &um);
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        col_combine<R, HALL, HOD, CONV>(a, ax, s[k], Bm[k], um[k], db[k], hod[k]);
        if (FOF) fo_combine(a.dR, ax, s[k], fo[k]);
      }
    }
    V3<R> hv[2] = {hod[0], hod[1]};
    if (HODP) ldf_pair(a.Hpre, idx, hv[0], hv[1]);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int ii[3] = {ix + k, iy, iz};
      if (!PER) stage_sat<R, SoA<R>, HALL>(a, ii, nn, idx + k, Bm[k], um[k], CONV, db[k]);
      if (HOD_) {
        db[k].x += a.hod_factor * hv[k].x;
        db[k].y += a.hod_factor * hv[k].y;
        db[k].z += a.hod_factor * hv[k].z;
      }
      if (FOAD) {
        const V3<R> ds = fo_ad_dissipation<R, SoA<R>, OP, PER>(a, ii, nn, st, idx + k, Bm[k], um[k]);
        db[k].x += ds.x; db[k].y += ds.y; db[k].z += ds.z;
      }
      if (FOF) {
        db[k].x += fo[k].x; db[k].y += fo[k].y; db[k].z += fo[k].z;
      }
    }
    stage_epilogue_pair(a, idx, db[0], db[1]);
  }
  stage_time_post(a);
}

// One node of a box's stage in the order of operations of k_stage_col (one node per thread)
template <typename R, int OP, bool HALL, bool HOD_, int CONV, int NEED, bool HODP, bool FOAD, bool FOF = false>
__device__ __forceinline__ void col_stage_node(const StageArgs<R, SoA<R>> &a, int ix, int iy, int iz) {
  constexpr bool HOD = HOD_ && !HODP;
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const long long idx = ix + (long long)nx * (iy + (long long)ny * iz);
  const int ii[3] = {ix, iy, iz};
  const int nn[3] = {nx, ny, nz};
  const long long st[3] = {1, nx, (long long)nx * ny};
  const V3<R> zero = {0, 0, 0};
  const V3<R> Bm = ldf(a.bk, idx);
  const V3<R> um = CONV ? ldf(a.u, idx) : zero;
  V3<R> db = zero, hod = zero, fo = zero;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    ColSums<R> s{};
    col_axis<R, OP, false, HALL, HOD, CONV, SoA<R>, NEED, FOF>(s, a, ax, ii[ax], nn[ax], idx, st[ax], Bm, &um);
    col_combine<R, HALL, HOD, CONV>(a, ax, s, Bm, um, db, hod);
    if (FOF) fo_combine(a.dR, ax, s, fo);
  }
  stage_sat<R, SoA<R>, HALL>(a, ii, nn, idx, Bm, um, CONV, db);
  if (HOD_) {
    const V3<R> hv = HODP ? ldf(a.Hpre, idx) : hod;
    db.x += a.hod_factor * hv.x;
    db.y += a.hod_factor * hv.y;
    db.z += a.hod_factor * hv.z;
  }
  if (FOAD) {
    const V3<R> ds = fo_ad_dissipation<R, SoA<R>, OP, false>(a, ii, nn, st, idx, Bm, um);
    db.x += ds.x; db.y += ds.y; db.z += ds.z;
  }
  if (FOF) {
    db.x += fo.x; db.y += fo.y; db.z += fo.z;
  }
  stage_epilogue<R, SoA<R>>(a, idx, db);
}

// the x boundary columns of a box (2 * xband nodes per row, one per thread), and the stage's
// time bookkeeping
template <typename R, int OP, bool HALL, bool HOD_, int CONV, int NEED, bool HODP, bool FOAD, bool FOF = false>
__global__ void __launch_bounds__(kColThreads) k_stage_xband(const __grid_constant__ StageArgs<R, SoA<R>> a) {
  constexpr int XB = xband<OP>();
  pdl_enter();
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long rows = (long long)a.m.ny * a.m.nz;
  if (i < rows * 2 * XB) {
    const int slot = (int)(i % (2 * XB));
    const long long row = i / (2 * XB);
    const int ix = slot < XB ? slot : a.m.nx - 2 * XB + slot;
    col_stage_node<R, OP, HALL, HOD_, CONV, NEED, HODP, FOAD, FOF>(a, ix, (int)(row % a.m.ny), (int)(row / a.m.ny));
  }
  stage_time_post(a);
}

// J = curl(B)/rho, E = J x B, (HODS) the dissipation sum and J on the faces at one node of a
// box's x boundary columns (2 * xband per row, one per thread; the order of k_curl_e_hod)
template <typename R, int OP, bool HODS>
__global__ void __launch_bounds__(kColThreads) k_curl_xband(const __grid_constant__ CurlArgs<R, SoA<R>> a) {
  constexpr int XB = xband<OP>();
  pdl_enter();
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  if (i >= (long long)ny * nz * 2 * XB) return;
  const int slot = (int)(i % (2 * XB));
  const long long row = i / (2 * XB);
  const int ix = slot < XB ? slot : nx - 2 * XB + slot, iy = (int)(row % ny), iz = (int)(row / ny);
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
    curl_axis_node<R, OP, false, HODS>(a, ax, ii[ax], nn[ax], idx, st[ax], Bm, v1, v2, ho);
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
  if (ix == 0 || iy == 0 || iz == 0 || ix == nx - 1 || iy == ny - 1 || iz == nz - 1) stf(a.jface, idx, J);
}

// whether every K-wide load or store of a field is aligned (K elements, stride a multiple of K)
template <int K, typename R>
inline bool group_ok(const SoA<R> &f) {
  return f.p == nullptr || ((reinterpret_cast<uintptr_t>(f.p) % (K * sizeof(R))) == 0 && f.s % K == 0);
}

// whether a launch may use the pair kernels: nx even and every pair load or store aligned
template <typename R>
inline bool pair_ok(const SoA<R> &f) {
  return f.p == nullptr || ((reinterpret_cast<uintptr_t>(f.p) % (2 * sizeof(R))) == 0 && f.s % 2 == 0);
}

}  // namespace ieq
