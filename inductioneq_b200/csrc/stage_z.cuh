// stage_z.cuh -- the one-pass Hall stage: J = curl(B)/rho, E = J x B, the dissipation sum and
// the stage update in one kernel that marches through z (periodic grids, u = 0).
//
// The two-kernel stage (k_curl_e_x2 writes E and H, k_stage_hall_x2 reads them back) moves
// 224 B per node and stage; the stage's compulsory traffic is 136 B (read b1, b2, rho; write
// b1', b2).  Here a CTA owns a tile of kZTX x kZTY nodes of the x-y plane and a chunk of z
// planes, two x-adjacent nodes per thread.  E never leaves the SM:
//   * E of the tile is computed RI planes ahead of the plane being updated and kept in a ring
//     of 2*RI + 1 planes in shared memory (the z derivative of E reads the ring);
//   * E on the tile's x and y halo strips (RI deep; x strips 4 columns so that pairs stay
//     aligned) is recomputed for the plane being updated, just in time, and the x strips are
//     written into the padding columns of that plane's ring slot, the y strips into a buffer
//     of their own;
//   * the dissipation sum H of the updated plane is formed by the thread that updates it;
//   * the Hall flux rows then read E from shared memory only.
// B, rho and the epilogue's fields are read through the read-only path: every neighbour
// value of B is an L1/L2 hit after the first touch, so DRAM sees the compulsory bytes (plus
// the halo and z-prologue re-reads that L2 does not catch).
//
// Every node's sums are formed term by term in the order of k_curl_e_x2 (J, E, H) and
// k_stage_hall_x2 (the Hall rows, then the dissipation sum), so the result equals the
// two-kernel stage up to the compiler's choice of fused multiply-adds.
//
// Requirements (checked by the launcher): periodic grid, nx a multiple of kZTX, ny a
// multiple of kZTY, nz >= 2*RI + 1 (a stencil wraps once), every field 16-byte aligned
// with an even component stride.
#pragma once
#include "stage_x2.cuh"

namespace ieq {

constexpr int kZTX = 32;                      // tile nodes in x (16 pairs)
constexpr int kZTY = 16;                      // tile rows in y
constexpr int kZThreads = (kZTX / 2) * kZTY;  // 256: one pair per thread
constexpr int kZPad = 4;                      // x halo columns on each side of a ring row
constexpr int kZRow = kZTX + 2 * kZPad;       // 40 elements per ring row

template <typename R, int RI>
struct ZLayout {
  static constexpr int W = 2 * RI + 1;                    // ring slots (planes)
  static constexpr int SLOT = 3 * kZTY * kZRow;           // [comp][row][pad + tile + pad]
  static constexpr int RING = W * SLOT;
  static constexpr int YS = 2 * 2 * RI * kZTX;            // y strips [side][Exy, Eyz][row][col]
  static constexpr int ELEMS = RING + YS;
  static constexpr size_t BYTES = (size_t)ELEMS * sizeof(R);
};

// J = curl(B)/rho and E = J x B at the pair (ix, ix + 1) of plane iz (periodic interior
// rows; the order of operations of k_curl_e_x2)
template <typename R, int OP>
__device__ __forceinline__ void zm_e_pair(const StageArgs<R, SoA<R>> &a, const R *rho, int ix, int iy, int iz,
                                          V3<R> (&E)[2]) {
  constexpr int RI = Op<OP>::RI, QL = (RI + 1) / 2;
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const long long row0 = (long long)nx * (iy + (long long)ny * iz);
  const long long idx = row0 + ix;
  const long long cs = a.bk.s;
  V3<R> Bm[2];
  ldf_k<R, 2>(a.bk, idx, Bm);
  R g[2][3][3];
  {
    R v1[2] = {0, 0}, v2[2] = {0, 0};
#pragma unroll
    for (int c = 1; c < 3; ++c) {
      R w[2 * (2 * QL + 1)];
      x_window_k<R, 2, QL, true>(a.bk.p + c * cs, row0, ix, nx, w);
#pragma unroll
      for (int k = 0; k < 2; ++k) {
#pragma unroll
        for (int o = -RI; o <= RI; ++o) {
          if (o == 0) continue;
          const R val = w[2 * QL + k + o];
          if (c == 1) v1[k] += a.Dint[o + RI] * val;
          else v2[k] += a.Dint[o + RI] * val;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      g[k][0][1] = v1[k] * a.inv_d[0];
      g[k][0][2] = v2[k] * a.inv_d[0];
    }
  }
  const int ii[3] = {ix, iy, iz};
  const int nn[3] = {nx, ny, nz};
  const long long st[3] = {1, nx, (long long)nx * ny};
#pragma unroll
  for (int ax = 1; ax < 3; ++ax) {
    const int c1 = (ax + 1) % 3, c2 = (ax + 2) % 3;
    const int i = ii[ax], n = nn[ax];
    R v1[2] = {0, 0}, v2[2] = {0, 0};
    const bool wrap = i < RI || i >= n - RI;
#pragma unroll
    for (int o = -RI; o <= RI; ++o) {
      if (o == 0) continue;
      const long long j = wrap ? idx + (long long)(nbr<true>(i, o, n) - i) * st[ax] : idx + (long long)o * st[ax];
      R p1[2], p2[2];
      ld_k<R, 2>(a.bk.p + j + c1 * cs, p1);
      ld_k<R, 2>(a.bk.p + j + c2 * cs, p2);
      const R c = a.Dint[o + RI];
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        v1[k] += c * p1[k];
        v2[k] += c * p2[k];
      }
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      g[k][ax][c1] = v1[k] * a.inv_d[ax];
      g[k][ax][c2] = v2[k] * a.inv_d[ax];
    }
  }
  R r[2];
  if (rho) ld_k<R, 2>(rho + idx, r);
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    V3<R> J = {g[k][1][2] - g[k][2][1], g[k][2][0] - g[k][0][2], g[k][0][1] - g[k][1][0]};
    if (rho) {
      const R ri = (R)1 / r[k];
      J = {J.x * ri, J.y * ri, J.z * ri};
    }
    const V3<R> &B = Bm[k];
    E[k] = V3<R>{J.x * B.y - J.y * B.x, J.x * B.z - J.z * B.x, J.y * B.z - J.z * B.y};
  }
}

// the dissipation sum of B at the pair (the HODS part of k_curl_e_x2, in its order)
template <typename R, int OP>
__device__ __forceinline__ void zm_h_pair(const StageArgs<R, SoA<R>> &a, int ix, int iy, int iz, V3<R> (&hod)[2]) {
  constexpr int RI = Op<OP>::RI, QL = (RI + 1) / 2;
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const long long row0 = (long long)nx * (iy + (long long)ny * iz);
  const long long idx = row0 + ix;
  const long long cs = a.bk.s;
  const V3<R> zero = {0, 0, 0};
  V3<R> Bm[2];
  ldf_k<R, 2>(a.bk, idx, Bm);
  hod[0] = hod[1] = zero;
  {
    V3<R> ho[2] = {zero, zero};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      R w[2 * (2 * QL + 1)];
      x_window_k<R, 2, QL, true>(a.bk.p + c * cs, row0, ix, nx, w);
#pragma unroll
      for (int k = 0; k < 2; ++k) {
#pragma unroll
        for (int o = -RI; o <= RI; ++o) cref(ho[k], c) += a.Hint[o + RI] * w[2 * QL + k + o];
      }
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      hod[k].x += ho[k].x; hod[k].y += ho[k].y; hod[k].z += ho[k].z;
    }
  }
  const int ii[3] = {ix, iy, iz};
  const int nn[3] = {nx, ny, nz};
  const long long st[3] = {1, nx, (long long)nx * ny};
#pragma unroll
  for (int ax = 1; ax < 3; ++ax) {
    const int i = ii[ax], n = nn[ax];
    const bool wrap = i < RI || i >= n - RI;
    V3<R> ho[2] = {zero, zero};
#pragma unroll
    for (int o = -RI; o <= RI; ++o) {
      const R cH = a.Hint[o + RI];
      if (o == 0) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          ho[k].x += cH * Bm[k].x; ho[k].y += cH * Bm[k].y; ho[k].z += cH * Bm[k].z;
        }
        continue;
      }
      const long long j = wrap ? idx + (long long)(nbr<true>(i, o, n) - i) * st[ax] : idx + (long long)o * st[ax];
      V3<R> B[2];
      ldf_k<R, 2>(a.bk, j, B);
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        ho[k].x += cH * B[k].x; ho[k].y += cH * B[k].y; ho[k].z += cH * B[k].z;
      }
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      hod[k].x += ho[k].x; hod[k].y += ho[k].y; hod[k].z += ho[k].z;
    }
  }
}

__device__ __forceinline__ int zm_wrap(int i, int n) {
  i += i < 0 ? n : 0;
  return i >= n ? i - n : i;
}

// grid: x = tile (nx/kZTX * ny/kZTY tiles), y = z chunk of tz planes; block: kZThreads
template <typename R, int OP, bool HOD>
__global__ void __launch_bounds__(kZThreads, 2)
    k_stage_hall_z(const __grid_constant__ StageArgs<R, SoA<R>> a, const R *__restrict__ rho, int tz) {
  constexpr int RI = Op<OP>::RI;
  using L = ZLayout<R, RI>;
  constexpr int W = L::W;
  extern __shared__ __align__(16) unsigned char zsm_raw[];
  R *ring = reinterpret_cast<R *>(zsm_raw);
  R *ys = ring + L::RING;
  pdl_enter();
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const int ntx = nx / kZTX;
  const int x0 = (blockIdx.x % ntx) * kZTX, y0 = (blockIdx.x / ntx) * kZTY;
  const int z0 = blockIdx.y * tz;
  const int z1 = min(z0 + tz, nz);
  const int t = threadIdx.x;
  const int px = t % (kZTX / 2), ly = t / (kZTX / 2);
  const int lx = 2 * px;
  const int ix = x0 + lx, iy = y0 + ly;
  // ring slot of plane e (z0 - RI <= e): e - z0 + RI >= 0
  auto slot = [&](int e) -> R * { return ring + ((e - z0 + RI) % W) * L::SLOT; };
  auto at = [&](R *s, int c, int row, int col) -> R * { return s + (c * kZTY + row) * kZRow + kZPad + col; };

  for (int e = z0 - RI; e < z1 + RI; ++e) {
    const int p = e - RI;
    // (1) E of the tile on plane e, RI planes ahead of the plane it updates
    {
      V3<R> E[2];
      zm_e_pair<R, OP>(a, rho, ix, iy, zm_wrap(e, nz), E);
      R *s = slot(e);
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        *at(s, 0, ly, lx + k) = E[k].x;
        *at(s, 1, ly, lx + k) = E[k].y;
        *at(s, 2, ly, lx + k) = E[k].z;
      }
    }
    const bool out = p >= z0;
    V3<R> hv[2];
    if (out) {
      const int pz = zm_wrap(p, nz);
      // (2) E on the halo strips of plane p: x strips (4 columns a side, into the padding of
      // the plane's ring slot: Exy, Exz) and y strips (RI rows a side: Exy, Eyz)
      constexpr int NXS = 2 * 2 * kZTY;              // x-strip pairs
      constexpr int NYS = 2 * RI * (kZTX / 2);       // y-strip pairs
      if (t < NXS) {
        const int side = t / (2 * kZTY), rem = t % (2 * kZTY);
        const int row = rem / 2, q = rem % 2;
        const int col = side ? kZTX + 2 * q : -kZPad + 2 * q;   // tile-relative
        V3<R> E[2];
        zm_e_pair<R, OP>(a, rho, zm_wrap(x0 + col, nx), y0 + row, pz, E);
        R *s = slot(p);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          *at(s, 0, row, col + k) = E[k].x;
          *at(s, 1, row, col + k) = E[k].y;
        }
      } else if (t < NXS + NYS) {
        const int u = t - NXS;
        const int side = u / (RI * (kZTX / 2)), rem = u % (RI * (kZTX / 2));
        const int row = rem / (kZTX / 2), q = rem % (kZTX / 2);
        const int yy = side ? y0 + kZTY + row : y0 - RI + row;
        V3<R> E[2];
        zm_e_pair<R, OP>(a, rho, x0 + 2 * q, zm_wrap(yy, ny), pz, E);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          ys[((side * 2 + 0) * RI + row) * kZTX + 2 * q + k] = E[k].x;
          ys[((side * 2 + 1) * RI + row) * kZTX + 2 * q + k] = E[k].z;
        }
      }
      // (3) the dissipation sum of the tile pair on plane p
      if (HOD) zm_h_pair<R, OP>(a, ix, iy, pz, hv);
    }
    __syncthreads();
    if (out) {
      // (4) DB on plane p from shared memory, then the stage update (k_stage_hall_x2's order)
      const int pz = zm_wrap(p, nz);
      const V3<R> zero = {0, 0, 0};
      V3<R> db[2] = {zero, zero};
      R *s = slot(p);
      {
        // x: DB_y += D[Exy], DB_z += D[Exz]
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          R h1 = 0, h2 = 0;
#pragma unroll
          for (int o = -RI; o <= RI; ++o) {
            if (o == 0) continue;
            h1 += a.Dint[o + RI] * *at(s, 0, ly, lx + k + o);
            h2 += a.Dint[o + RI] * *at(s, 1, ly, lx + k + o);
          }
          db[k].y += a.inv_d[0] * h1;
          db[k].z += a.inv_d[0] * h2;
        }
      }
      {
        // y: DB_x -= D[Exy], DB_z += D[Eyz]
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          R h1 = 0, h2 = 0;
#pragma unroll
          for (int o = -RI; o <= RI; ++o) {
            if (o == 0) continue;
            const int yy = ly + o;
            const R *pxy = yy < 0 ? ys + ((0 * 2 + 0) * RI + yy + RI) * kZTX + lx + k
                           : yy >= kZTY ? ys + ((1 * 2 + 0) * RI + yy - kZTY) * kZTX + lx + k
                                        : at(s, 0, yy, lx + k);
            const R *pyz = yy < 0 ? ys + ((0 * 2 + 1) * RI + yy + RI) * kZTX + lx + k
                           : yy >= kZTY ? ys + ((1 * 2 + 1) * RI + yy - kZTY) * kZTX + lx + k
                                        : at(s, 2, yy, lx + k);
            h1 += a.Dint[o + RI] * *pxy;
            h2 += a.Dint[o + RI] * *pyz;
          }
          db[k].x -= a.inv_d[1] * h1;
          db[k].z += a.inv_d[1] * h2;
        }
      }
      {
        // z: DB_x -= D[Exz], DB_y -= D[Eyz]
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          R h1 = 0, h2 = 0;
#pragma unroll
          for (int o = -RI; o <= RI; ++o) {
            if (o == 0) continue;
            R *so = slot(p + o);
            h1 += a.Dint[o + RI] * *at(so, 1, ly, lx + k);
            h2 += a.Dint[o + RI] * *at(so, 2, ly, lx + k);
          }
          db[k].x -= a.inv_d[2] * h1;
          db[k].y -= a.inv_d[2] * h2;
        }
      }
      if (HOD) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          db[k].x += a.hod_factor * hv[k].x;
          db[k].y += a.hod_factor * hv[k].y;
          db[k].z += a.hod_factor * hv[k].z;
        }
      }
      const long long idx = ix + (long long)nx * (iy + (long long)ny * pz);
      stage_epilogue_k<R, 2>(a, idx, db);
    }
    // the next plane overwrites the ring slot of plane p - RI and the halo strips
    __syncthreads();
  }
  stage_time_post(a);
}

// explicit launcher, instantiated per (R, OP) in stage_<r>_o<op>.cu: one stage on the
// periodic grid of a.m (the caller checked zm_eligible)
template <typename R, int OP>
void launch_stage_zmarch(const StageArgs<R, SoA<R>> &a, const R *rho, bool hod, bool pdl, int tz, cudaStream_t s);

// whether the one-pass stage can run on this grid and these fields
template <typename R>
inline bool zm_eligible(const StageArgs<R, SoA<R>> &a, const R *rho, int ri) {
  const auto al = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
  return a.m.nx % kZTX == 0 && a.m.ny % kZTY == 0 && a.m.nz >= 2 * ri + 1 && al(a.bk.p) && a.bk.s % 2 == 0 &&
         pair_ok(a.X) && pair_ok(a.Y) && pair_ok(a.Z) && pair_ok(a.out) && pair_ok(a.out2) && pair_ok(a.out3) &&
         (rho == nullptr || al(rho));
}

// chunk length in z: the number of chunks minimises (waves of `resident` CTAs) x (planes a
// CTA marches, its 2*RI prologue planes of tile E included)
inline int zm_chunk(int nx, int ny, int nz, int ri, int resident) {
  const long long tiles = (long long)(nx / kZTX) * (ny / kZTY);
  long long best_cost = -1;
  int best_tz = nz;
  for (int chunks = 1; chunks <= nz; ++chunks) {
    const int tz = (nz + chunks - 1) / chunks;
    const long long ctas = tiles * ((nz + tz - 1) / tz);
    const long long waves = (ctas + resident - 1) / resident;
    const long long cost = waves * (tz + 2 * ri);
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      best_tz = tz;
    }
  }
  return best_tz;
}

}  // namespace ieq

namespace ieq {

// ---------------------------------------------------------------------------------------
// The curl kernel as a 2.5D z march (periodic grids): J = curl(B)/rho, E = J x B and (HODS)
// the dissipation sum of B, the outputs of k_curl_e_x2 / k_curl_e_hod, with each value of B
// loaded from global memory about once.  A CTA of kCzTX x kCzTY threads owns a tile of x-y
// columns and a chunk of z planes; every thread keeps the three components of B of its
// column at planes z - RI .. z + RI in registers (the z terms) and plane z of the tile with
// its x and y halos (RI deep) sits in shared memory (the x and y terms).  The march is
// software-pipelined: the column's queue values (B at plane z + RI, the only loads that
// come from DRAM rather than from a neighbour's recent loads in L2) are copied kCzAhead
// planes ahead into a per-thread shared-memory ring by cp.async (each thread reads back only
// what it copied, so the ring needs no barrier), while the next plane's halo points and rho
// are loaded into registers during the current plane's compute; the halo'd plane is
// double-buffered in shared memory, so one barrier per plane suffices (a thread writes
// buffer (z + 1) & 1 only after every thread passed the barrier of plane z, i.e. finished
// plane z - 1, the last reader of that buffer).  The sums run in the order of k_curl_e_hod
// (axis by axis, offsets ascending), so the outputs equal the one-node kernels' up to the
// compiler's fused multiply-adds.  Registers are capped for kCzBlocks resident CTAs per SM
// (80 in FP64, no spills; 2 CTAs of 120 registers measured 7 % slower at 256^3).
constexpr int kCzTX = 32, kCzTY = 8, kCzBlocks = 3;
constexpr int kCzAhead = 3;   // planes of the column's B loads in flight ahead of the march
// ring slots: one more than the look-ahead, so that the slot refilled at plane z was last
// read at plane z - 1, before the barrier of plane z
constexpr int kCzSlots = kCzAhead + 1;
// dynamic shared memory of k_curl_e_z: the ring of the column's B, kCzSlots x 3 x threads
template <typename R>
constexpr int cz_ring_bytes() { return kCzSlots * 3 * kCzTX * kCzTY * (int)sizeof(R); }

// per-thread asynchronous copies (cp.async, L1-allocating) of one element into shared memory
template <typename R>
__device__ __forceinline__ void cz_async(R *dst, const R *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(R) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cz_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cz_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <typename R, int OP, bool HODS>
__global__ void __launch_bounds__(kCzTX * kCzTY, kCzBlocks)
    k_curl_e_z(const __grid_constant__ CurlArgs<R, SoA<R>> a, int tz) {
  constexpr int RI = Op<OP>::RI, W = 2 * RI + 1;
  constexpr int SX = kCzTX + 2 * RI, SY = kCzTY + 2 * RI;
  constexpr int NT = kCzTX * kCzTY;
  constexpr int NHALO = 2 * RI * (kCzTX + kCzTY);   // x halos of the tile rows, y halos of its columns
  constexpr int HPT = (NHALO + NT - 1) / NT;         // halo points per thread
  __shared__ R pl[2][3][SY][SX];
  extern __shared__ __align__(16) unsigned char cz_dyn[];
  R(*qr)[3][NT] = reinterpret_cast<R(*)[3][NT]>(cz_dyn);   // ring of the column's B at plane z + RI
  pdl_enter();
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const int tx = threadIdx.x % kCzTX, ty = threadIdx.x / kCzTX;
  const int x0 = blockIdx.x * kCzTX, y0 = blockIdx.y * kCzTY;
  const int zb = blockIdx.z * tz, ze = min(zb + tz, nz);
  const int ix = x0 + tx, iy = y0 + ty;
  const bool own = ix < nx && iy < ny;
  const long long sz = (long long)nx * ny;
  const long long cs = a.b.s;
  const R *bp = a.b.p;
  auto wrap = [](int i, int n) { i %= n; return i < 0 ? i + n : i; };
  // the column of (ix, iy) wrapped into the grid (threads past the edge hold the periodic image)
  const long long col = wrap(ix, nx) + (long long)nx * wrap(iy, ny);
  // this thread's halo points: offset within a shared component plane and grid column
  int hpos[HPT];
  long long hcol[HPT];
#pragma unroll
  for (int k = 0; k < HPT; ++k) {
    const int h = threadIdx.x + k * NT;
    hpos[k] = -1;
    hcol[k] = 0;
    if (h < NHALO) {
      int px, py;
      if (h < 2 * RI * kCzTY) {
        const int side = h / (RI * kCzTY), rem = h % (RI * kCzTY);
        py = RI + rem / RI;
        px = side ? kCzTX + RI + rem % RI : rem % RI;
      } else {
        const int g = h - 2 * RI * kCzTY;
        const int side = g / (RI * kCzTX), rem = g % (RI * kCzTX);
        px = RI + rem % kCzTX;
        py = side ? kCzTY + RI + rem / kCzTX : rem / kCzTX;
      }
      hpos[k] = py * SX + px;
      hcol[k] = wrap(x0 - RI + px, nx) + (long long)nx * wrap(y0 - RI + py, ny);
    }
  }
  R q[3][W];
#pragma unroll
  for (int k = 0; k < W - 1; ++k) {
    const long long j = col + sz * wrap(zb - RI + k, nz);
#pragma unroll
    for (int c = 0; c < 3; ++c) q[c][k + 1] = __ldg(bp + j + c * cs);
  }
  // the column's B at plane z + RI into ring slot (z - zb) % kCzSlots, one commit group per
  // plane (empty past the chunk, so that every plane waits for the same group count)
  auto issue = [&](int z) {
    if (z < ze) {
      int zq = z + RI;
      if (zq >= nz) zq -= nz;
      const long long jq = col + sz * zq;
      const int slot = (z - zb) % kCzSlots;
#pragma unroll
      for (int c = 0; c < 3; ++c) cz_async(&qr[slot][c][threadIdx.x], bp + jq + c * cs);
    }
    cz_commit();
  };
#pragma unroll
  for (int k = 0; k < kCzAhead; ++k) issue(zb + k);
  // registers of the next plane: halo points, rho
  R nh[HPT][3], nr = (R)1;
  auto fetch = [&](int z) {
    const long long zo = sz * z;
#pragma unroll
    for (int k = 0; k < HPT; ++k)
      if (hpos[k] >= 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) nh[k][c] = __ldg(bp + hcol[k] + zo + c * cs);
      }
    if (a.rho && own) nr = __ldg(a.rho + ix + (long long)nx * iy + zo);
  };
  fetch(zb);
  for (int z = zb; z < ze; ++z) {
    R(*P)[SY][SX] = pl[(z - zb) & 1];
    cz_wait<kCzAhead - 1>();
    const int slot = (z - zb) % kCzSlots;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
      for (int k = 0; k < W - 1; ++k) q[c][k] = q[c][k + 1];
      q[c][W - 1] = qr[slot][c][threadIdx.x];
      P[c][ty + RI][tx + RI] = q[c][RI];
    }
#pragma unroll
    for (int k = 0; k < HPT; ++k)
      if (hpos[k] >= 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) (&P[c][0][0])[hpos[k]] = nh[k][c];
      }
    const R rz = nr;
    __syncthreads();
    issue(z + kCzAhead);
    if (z + 1 < ze) fetch(z + 1);
    if (own) {
      const V3<R> Bm = {q[0][RI], q[1][RI], q[2][RI]};
      R g[3][3];
      V3<R> hod = {0, 0, 0};
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        const int c1 = (ax + 1) % 3, c2 = (ax + 2) % 3;
        R v1 = 0, v2 = 0;
        V3<R> ho = {0, 0, 0};
#pragma unroll
        for (int o = -RI; o <= RI; ++o) {
          // the three components of B at offset o along the axis
          R b3[3];
#pragma unroll
          for (int c = 0; c < 3; ++c)
            b3[c] = ax == 0 ? P[c][ty + RI][tx + RI + o] : (ax == 1 ? P[c][ty + RI + o][tx + RI] : q[c][RI + o]);
          const R cH = a.Hint[o + RI];
          if (o == 0) {
            if (HODS) {
              ho.x += cH * Bm.x; ho.y += cH * Bm.y; ho.z += cH * Bm.z;
            }
            continue;
          }
          const R cD = a.Dint[o + RI];
          v1 += cD * b3[c1];
          v2 += cD * b3[c2];
          if (HODS) {
            ho.x += cH * b3[0]; ho.y += cH * b3[1]; ho.z += cH * b3[2];
          }
        }
        g[ax][c1] = v1 * a.inv_d[ax];
        g[ax][c2] = v2 * a.inv_d[ax];
        if (HODS) {
          hod.x += ho.x; hod.y += ho.y; hod.z += ho.z;
        }
      }
      const long long idx = ix + (long long)nx * iy + sz * z;
      V3<R> J = {g[1][2] - g[2][1], g[2][0] - g[0][2], g[0][1] - g[1][0]};
      if (a.rho) {
        const R r = (R)1 / rz;
        J = {J.x * r, J.y * r, J.z * r};
      }
      stf(a.out, idx, V3<R>{J.x * Bm.y - J.y * Bm.x, J.x * Bm.z - J.z * Bm.x, J.y * Bm.z - J.z * Bm.y});
      if (HODS) stf(a.hout, idx, hod);
    }
  }
}

// z planes per CTA of k_curl_e_z: about `per_sm` CTAs per SM, at least 4 planes
inline int cz_chunk(int nx, int ny, int nz, int nsm, int per_sm) {
  const long long tiles = (long long)((nx + kCzTX - 1) / kCzTX) * ((ny + kCzTY - 1) / kCzTY);
  const long long chunks = ((long long)per_sm * nsm + tiles - 1) / tiles;
  int tz = (int)((nz + chunks - 1) / chunks);
  return tz < 4 ? 4 : tz;
}

template <typename R, int OP>
void launch_curl_e_z(const CurlArgs<R, SoA<R>> &a, bool hod, int tz, bool pdl, cudaStream_t s);

}  // namespace ieq
