// stage_brick.cuh -- TMA-staged brick kernels of the fused path (u = 0 stages).
//
// A CTA owns a brick of 16 x 8 x 4 nodes.  One thread loads the brick's star-shaped halo
// region of each field it needs -- the x slab (brick + 4 columns on each side), two y
// slabs and two z slabs of radius 3 -- with cp.async.bulk.tensor into shared memory,
// completing on one mbarrier; all 256 threads then evaluate the derivative rows from
// shared memory (two nodes each) and write the stage update.  The fields enter as 4-D
// tensor maps (NX, NY, NZ, component) over the structure-of-arrays state, so one TMA
// instruction moves all three components of a slab.
//
//   k_stage_brick: Hall flux rows on E = J x B and dissipation rows on B, then the
//                  stage epilogue (as k_stage_col);
//   k_curl_brick:  J = curl(B)/rho from the B slabs, writes E (and J on box faces).
//
// Bricks whose nodes use an SBP boundary row (non-periodic box) take the per-node global
// path instead (block-uniform branch).  Periodic boxes need NX, NY, NZ to be multiples of
// the brick; the x wrap columns are loaded as separate boxes and copied into place.
#pragma once
#include "stage_col.cuh"
#include "tma.cuh"

namespace ieq {

// one node through the global-memory column path (per-node gathers on E), used by the
// boundary bricks
template <typename R, int OP, bool PER, bool HALL, bool HOD>
__device__ __forceinline__ void stage_node_e(const StageArgs<R, SoA<R>> &a, int ix, int iy, int iz) {
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const long long idx = ix + (long long)nx * (iy + (long long)ny * iz);
  const V3<R> zero = {0, 0, 0};
  const V3<R> Bm = ldf(a.bk, idx);
  V3<R> db = zero, hod = zero;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    ColSums<R> s{};
    const int i = ax == 0 ? ix : (ax == 1 ? iy : iz);
    const int n = ax == 0 ? nx : (ax == 1 ? ny : nz);
    const long long st = ax == 0 ? 1 : (ax == 1 ? (long long)nx : (long long)nx * ny);
    col_axis<R, OP, PER, HALL, HOD, 0>(s, a, ax, i, n, idx, st, Bm);
    col_combine<R, HALL, HOD, 0>(a, ax, s, Bm, zero, db, hod);
  }
  const int ii[3] = {ix, iy, iz};
  const int nn[3] = {nx, ny, nz};
  if (!PER) stage_sat<R, SoA<R>, HALL>(a, ii, nn, idx, Bm, zero, 0, db);
  if (HOD) {
    db.x += a.hod_factor * hod.x;
    db.y += a.hod_factor * hod.y;
    db.z += a.hod_factor * hod.z;
  }
  stage_epilogue<R, SoA<R>>(a, idx, db);
}

template <int OP, bool PER>
__device__ __forceinline__ bool brick_interior(int x0, int y0, int z0, int nx, int ny, int nz) {
  constexpr int NB = Op<OP>::NB;
  return PER || (x0 >= NB && x0 + kBX <= nx - NB && y0 >= NB && y0 + kBY <= ny - NB && z0 >= NB &&
                 z0 + kBZ <= nz - NB);
}

template <typename R, int OP, bool PER, bool HALL, bool HOD>
__global__ void __launch_bounds__(kBrickThreads, 2)
    k_stage_brick(const __grid_constant__ StageArgs<R, SoA<R>> a, const __grid_constant__ TmaStageMaps maps,
                  int *err) {
  constexpr int RI = Op<OP>::RI;
  using L = BrickLayout<sizeof(R)>;
  constexpr int NF = (HOD ? 1 : 0) + (HALL ? 1 : 0);
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + NF * L::BYTES);
  int *ok = reinterpret_cast<int *>(bar + 1);
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const int x0 = blockIdx.x * kBX, y0 = blockIdx.y * kBY, z0 = blockIdx.z * kBZ;
  const int t = threadIdx.x;
  const int lx = t % kBX, ly = (t / kBX) % kBY, lz0 = t / (kBX * kBY);
  const bool aligned = (smem_u32(smem) & 127u) == 0;
  if (!brick_interior<OP, PER>(x0, y0, z0, nx, ny, nz) || !aligned) {
    if (!aligned && t == 0) atomicMax(err, kBrickErrMisaligned);   // no copy is issued into a misaligned buffer
#pragma unroll
    for (int k = 0; k < kBrickNodesPerThread; ++k) {
      const int ix = x0 + lx, iy = y0 + ly, iz = z0 + lz0 + kBrickZPerPass * k;
      if (ix < nx && iy < ny && iz < nz) stage_node_e<R, OP, PER, HALL, HOD>(a, ix, iy, iz);
    }
    stage_time_post(a);
    return;
  }
  unsigned char *sB = smem;
  unsigned char *sE = smem + (HOD ? L::BYTES : 0);
  if (t == 0) {
    mbar_init(bar, 1);
    // the barrier expects the bytes of every box before any copy is issued
    mbar_arrive_expect_tx(bar, NF * brick_tx_bytes<R, PER>(x0, nx));
    if (HOD) brick_issue<R, PER>(sB, maps.B, bar, x0, y0, z0, nx, ny, nz);
    if (HALL) brick_issue<R, PER>(sE, maps.E, bar, x0, y0, z0, nx, ny, nz);
    *ok = 1;
  }
  // the epilogue's own fields do not depend on the copies: load them while they fly
  EpIn<R> ein[kBrickNodesPerThread];
#pragma unroll
  for (int k = 0; k < kBrickNodesPerThread; ++k) {
    const int iz = z0 + lz0 + kBrickZPerPass * k;
    ein[k] = epilogue_load(a, (x0 + lx) + (long long)nx * ((y0 + ly) + (long long)ny * iz));
  }
  __syncthreads();
  if (!brick_first_wait(bar, err)) *ok = 0;
  __syncthreads();
  if (!*ok) {
    // leave only after the copies stopped writing into this CTA's shared memory
    brick_drain(bar, err);
    stage_time_post(a);
    return;
  }
  if (PER && (x0 == 0 || x0 + kBX == nx)) {
    if (HOD) brick_fix_x_wrap<R>(sB, x0, nx);
    if (HALL) brick_fix_x_wrap<R>(sE, x0, nx);
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < kBrickNodesPerThread; ++k) {
    const int lz = lz0 + kBrickZPerPass * k;
    const int ix = x0 + lx, iy = y0 + ly, iz = z0 + lz;
    const long long idx = ix + (long long)nx * (iy + (long long)ny * iz);
    V3<R> db = {0, 0, 0}, hod = {0, 0, 0};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      R h1 = 0, h2 = 0;
      V3<R> ho = {0, 0, 0};
      const int c1 = e_comp1(ax), c2 = e_comp2(ax);
#pragma unroll
      for (int o = -RI; o <= RI; ++o) {
        if (HOD) {
          const R cH = a.Hint[o + RI];
          ho.x += cH * *brick_at<R>(sB, ax, o, 0, lx, ly, lz);
          ho.y += cH * *brick_at<R>(sB, ax, o, 1, lx, ly, lz);
          ho.z += cH * *brick_at<R>(sB, ax, o, 2, lx, ly, lz);
        }
        if (HALL && o != 0) {
          const R cD = a.Dint[o + RI];
          h1 += cD * *brick_at<R>(sE, ax, o, c1, lx, ly, lz);
          h2 += cD * *brick_at<R>(sE, ax, o, c2, lx, ly, lz);
        }
      }
      if (HALL) {
        const R f1 = a.inv_d[ax] * h1, f2 = a.inv_d[ax] * h2;
        if (ax == 0) {
          db.y += f1; db.z += f2;
        } else if (ax == 1) {
          db.x -= f1; db.z += f2;
        } else {
          db.x -= f1; db.y -= f2;
        }
      }
      if (HOD) {
        hod.x += ho.x; hod.y += ho.y; hod.z += ho.z;
      }
    }
    if (HOD) {
      db.x += a.hod_factor * hod.x;
      db.y += a.hod_factor * hod.y;
      db.z += a.hod_factor * hod.z;
    }
    epilogue_store<R, SoA<R>>(a, idx, db, ein[k]);
  }
  stage_time_post(a);
}

template <typename R, int OP, bool PER>
__global__ void __launch_bounds__(kBrickThreads, 2)
    k_curl_brick(const __grid_constant__ CurlArgs<R, SoA<R>> a, const __grid_constant__ TmaStageMaps maps, int *err) {
  constexpr int NB = Op<OP>::NB, SW = Op<OP>::SW, C0 = (SW - 1) / 2, RI = Op<OP>::RI;
  using L = BrickLayout<sizeof(R)>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L::BYTES);
  int *ok = reinterpret_cast<int *>(bar + 1);
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const int x0 = blockIdx.x * kBX, y0 = blockIdx.y * kBY, z0 = blockIdx.z * kBZ;
  const int t = threadIdx.x;
  const int lx = t % kBX, ly = (t / kBX) % kBY, lz0 = t / (kBX * kBY);
  const bool aligned = (smem_u32(smem) & 127u) == 0;
  const int nn[3] = {nx, ny, nz};
  const long long st[3] = {1, nx, (long long)nx * ny};
  auto finish = [&](int ix, int iy, int iz, long long idx, R g[3][3]) {
    V3<R> J = {g[1][2] - g[2][1], g[2][0] - g[0][2], g[0][1] - g[1][0]};
    if (a.rho) {
      const R r = (R)1 / a.rho[idx];
      J = {J.x * r, J.y * r, J.z * r};
    }
    const V3<R> B = ldf(a.b, idx);
    stf(a.out, idx, V3<R>{J.x * B.y - J.y * B.x, J.x * B.z - J.z * B.x, J.y * B.z - J.z * B.y});
    if (!PER && (ix == 0 || iy == 0 || iz == 0 || ix == nx - 1 || iy == ny - 1 || iz == nz - 1))
      stf(a.jface, idx, J);
  };
  if (!brick_interior<OP, PER>(x0, y0, z0, nx, ny, nz) || !aligned) {
    if (!aligned && t == 0) atomicMax(err, kBrickErrMisaligned);
#pragma unroll
    for (int k = 0; k < kBrickNodesPerThread; ++k) {
      const int ix = x0 + lx, iy = y0 + ly, iz = z0 + lz0 + kBrickZPerPass * k;
      if (ix >= nx || iy >= ny || iz >= nz) continue;
      const long long idx = ix + (long long)nx * (iy + (long long)ny * iz);
      const int ii[3] = {ix, iy, iz};
      R g[3][3];
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        const int c1 = (ax + 1) % 3, c2 = (ax + 2) % 3;
        R v1 = 0, v2 = 0;
        const int row = PER ? NB : sbp_row(ii[ax], nn[ax], NB);
        if (row == NB) {
          const bool wrap = PER && (ii[ax] < RI || ii[ax] >= nn[ax] - RI);
#pragma unroll
          for (int o = -RI; o <= RI; ++o) {
            if (o == 0) continue;
            const R c = a.Dint[o + RI];
            const long long j = wrap ? idx + (long long)(nbr<true>(ii[ax], o, nn[ax]) - ii[ax]) * st[ax]
                                     : idx + (long long)o * st[ax];
            v1 += c * __ldg(a.b.p + j + c1 * a.b.s);
            v2 += c * __ldg(a.b.p + j + c2 * a.b.s);
          }
        } else {
          for (int o = -C0; o <= C0; ++o) {
            const R c = a.tab->D[row][o + C0];
            if (c == (R)0) continue;
            const long long j = idx + (long long)(nbr<PER>(ii[ax], o, nn[ax]) - ii[ax]) * st[ax];
            v1 += c * __ldg(a.b.p + j + c1 * a.b.s);
            v2 += c * __ldg(a.b.p + j + c2 * a.b.s);
          }
        }
        g[ax][c1] = v1 * a.inv_d[ax];
        g[ax][c2] = v2 * a.inv_d[ax];
      }
      finish(ix, iy, iz, idx, g);
    }
    return;
  }
  if (t == 0) {
    mbar_init(bar, 1);
    mbar_arrive_expect_tx(bar, brick_tx_bytes<R, PER>(x0, nx));
    brick_issue<R, PER>(smem, maps.B, bar, x0, y0, z0, nx, ny, nz);
    *ok = 1;
  }
  __syncthreads();
  if (!brick_first_wait(bar, err)) *ok = 0;
  __syncthreads();
  if (!*ok) {
    brick_drain(bar, err);
    return;
  }
  if (PER && (x0 == 0 || x0 + kBX == nx)) {
    brick_fix_x_wrap<R>(smem, x0, nx);
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < kBrickNodesPerThread; ++k) {
    const int lz = lz0 + kBrickZPerPass * k;
    const int ix = x0 + lx, iy = y0 + ly, iz = z0 + lz;
    const long long idx = ix + (long long)nx * (iy + (long long)ny * iz);
    R g[3][3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      const int c1 = (ax + 1) % 3, c2 = (ax + 2) % 3;
      R v1 = 0, v2 = 0;
#pragma unroll
      for (int o = -RI; o <= RI; ++o) {
        if (o == 0) continue;
        const R c = a.Dint[o + RI];
        v1 += c * *brick_at<R>(smem, ax, o, c1, lx, ly, lz);
        v2 += c * *brick_at<R>(smem, ax, o, c2, lx, ly, lz);
      }
      g[ax][c1] = v1 * a.inv_d[ax];
      g[ax][c2] = v2 * a.inv_d[ax];
    }
    finish(ix, iy, iz, idx, g);
  }
}

template <typename R, int OP>
void launch_stage_brick(const StageArgs<R, SoA<R>> &a, const TmaStageMaps &maps, int *err, bool per, bool hall,
                        bool hod, cudaStream_t s);
template <typename R, int OP>
void launch_curl_brick(const CurlArgs<R, SoA<R>> &a, const TmaStageMaps &maps, int *err, bool per, cudaStream_t s);

// dynamic shared memory of a brick kernel with nf fields (the barrier and a flag follow
// the field buffers)
template <typename R>
constexpr int brick_smem_bytes(int nf) {
  return nf * BrickLayout<sizeof(R)>::BYTES + 16;
}

inline dim3 brick_grid(int nx, int ny, int nz) {
  return dim3((unsigned)((nx + kBX - 1) / kBX), (unsigned)((ny + kBY - 1) / kBY), (unsigned)((nz + kBZ - 1) / kBZ));
}

}  // namespace ieq
