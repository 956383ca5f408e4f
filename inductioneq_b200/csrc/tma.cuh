// tma.cuh -- Tensor Memory Accelerator loads and mbarriers (sm_100a inline PTX) for the
// brick kernels, and the brick geometry they share with the host.
//
// Rules the kernels and the host keep (checked on the host before a tensor map is made):
//   * a tiled copy's innermost coordinate x times the element size is a multiple of 16
//     bytes: every x passed here is a multiple of 4 elements (bricks start at multiples of
//     TX = 16; the halo starts 4 before the brick; wrap boxes start at 0 and NX - 4);
//   * the global base is 16-byte aligned and every global stride (NX, NX*NY, component
//     stride) is a multiple of 16 bytes;
//   * every shared-memory destination is 128-byte aligned;
//   * no multicast: each CTA loads its own boxes.
// Waits on an mbarrier are bounded; on time-out the kernel records it in an error word and
// skips the computation.
#pragma once
#include <cuda.h>
#include <stdint.h>

namespace ieq {

// brick of nodes per CTA and its halo slabs (radius <= 3; the x slab is 4 wider on each
// side so that it starts on a 16-byte boundary)
constexpr int kBX = 16, kBY = 8, kBZ = 4;
constexpr int kHX = 4, kH = 3;
constexpr int kSX = kBX + 2 * kHX;
#ifndef IEQ_BRICK_THREADS
#define IEQ_BRICK_THREADS 256
#endif
constexpr int kBrickThreads = IEQ_BRICK_THREADS;                        // 256 or 512
constexpr int kBrickNodesPerThread = kBX * kBY * kBZ / kBrickThreads;   // 2 or 1
constexpr int kBrickZPerPass = kBrickThreads / (kBX * kBY);             // z planes per pass
constexpr long long kTmaWaitLimit = 1 << 20;

// element counts of the slabs of one 3-component field (layouts [c][z][y][x], x fastest)
constexpr int kElX = 3 * kBZ * kBY * kSX;   // core + x halo
constexpr int kElY = 3 * kBZ * kH * kBX;    // one y halo slab
constexpr int kElZ = 3 * kH * kBY * kBX;    // one z halo slab
constexpr int kElW = 3 * kBZ * kBY * kHX;   // one periodic x wrap box

template <int ES>
struct BrickLayout {
  static constexpr int up(int bytes) { return (bytes + 127) / 128 * 128; }
  static constexpr int X = 0;
  static constexpr int YLO = X + up(kElX * ES);
  static constexpr int YHI = YLO + up(kElY * ES);
  static constexpr int ZLO = YHI + up(kElY * ES);
  static constexpr int ZHI = ZLO + up(kElZ * ES);
  static constexpr int WLO = ZHI + up(kElZ * ES);
  static constexpr int WHI = WLO + up(kElW * ES);
  static constexpr int BYTES = WHI + up(kElW * ES);   // one field
};

// the four tensor maps of one SoA field (dims NX, NY, NZ, 3): boxes of the x slab, a y
// slab, a z slab and an x wrap piece
struct TmaField {
  CUtensorMap x, y, z, w;
};
struct TmaStageMaps {
  TmaField B, E;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait for phase `parity` of the barrier
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity) {
  for (long long it = 0; it < kTmaWaitLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// The brick kernels' error word err[0] (the highest code wins): 1 a brick's first wait
// for its halo copies gave up (the brick skipped its computation; its copies completed
// before it left), 2 a misaligned shared-memory buffer (the brick ran on the global path),
// 3 copies still outstanding when a brick left after its second wait (they may have
// written into the shared memory of a later CTA: the context's results are undefined).
// err[kBrickHookSlot] is a test hook: non-zero makes every first wait give up at once.
constexpr int kBrickErrLate = 1, kBrickErrMisaligned = 2, kBrickErrOutstanding = 3;
constexpr int kBrickHookSlot = 6;

// the first bounded wait of a brick for phase 0; false (recorded in err) if it gave up
__device__ __forceinline__ bool brick_first_wait(uint64_t *bar, int *err) {
  const bool give_up = *reinterpret_cast<volatile int *>(err + kBrickHookSlot) != 0;
  if (!give_up && mbar_wait_bounded(bar, 0)) return true;
  atomicMax(err, kBrickErrLate);
  return false;
}

// after a brick gave up: wait (production limit) until its copies stopped writing into
// its shared memory before it leaves; record the case where they did not
__device__ __forceinline__ void brick_drain(uint64_t *bar, int *err) {
  if (!mbar_wait_bounded(bar, 0)) atomicMax(err, kBrickErrOutstanding);
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z,
                                            int c) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(c), "r"(smem_u32(bar))
      : "memory");
}

// bytes the boxes of one field for the brick starting at x0 deliver (brick_issue)
template <typename R, bool PER>
__device__ __forceinline__ unsigned brick_tx_bytes(int x0, int nx) {
  unsigned n = kElX + 2 * kElY + 2 * kElZ;
  if (PER) n += ((x0 == 0) + (x0 + kBX == nx)) * kElW;
  return n * (unsigned)sizeof(R);
}

// Issue the halo loads of one field for the brick at (x0, y0, z0) into `base` (layout
// BrickLayout).  Periodic boxes wrap: the y/z slabs start at the wrapped row, the x wrap
// pieces land in WLO/WHI and are copied into the x slab after the wait
// (brick_fix_x_wrap).  Requires NX % kBX == 0 etc. when periodic.
template <typename R, bool PER>
__device__ __forceinline__ void brick_issue(unsigned char *base, const TmaField &f, uint64_t *bar, int x0, int y0,
                                            int z0, int nx, int ny, int nz) {
  using L = BrickLayout<sizeof(R)>;
  tma_load_4d(base + L::X, &f.x, bar, x0 - kHX, y0, z0, 0);
  int ylo = y0 - kH, yhi = y0 + kBY, zlo = z0 - kH, zhi = z0 + kBZ;
  if (PER) {
    ylo += ylo < 0 ? ny : 0;
    yhi -= yhi >= ny ? ny : 0;
    zlo += zlo < 0 ? nz : 0;
    zhi -= zhi >= nz ? nz : 0;
  }
  tma_load_4d(base + L::YLO, &f.y, bar, x0, ylo, z0, 0);
  tma_load_4d(base + L::YHI, &f.y, bar, x0, yhi, z0, 0);
  tma_load_4d(base + L::ZLO, &f.z, bar, x0, y0, zlo, 0);
  tma_load_4d(base + L::ZHI, &f.z, bar, x0, y0, zhi, 0);
  if (PER) {
    if (x0 == 0) tma_load_4d(base + L::WLO, &f.w, bar, nx - kHX, y0, z0, 0);
    if (x0 + kBX == nx) tma_load_4d(base + L::WHI, &f.w, bar, 0, y0, z0, 0);
  }
}

// periodic x: copy the wrap pieces into the halo columns of the x slab (all threads)
template <typename R>
__device__ __forceinline__ void brick_fix_x_wrap(unsigned char *base, int x0, int nx) {
  using L = BrickLayout<sizeof(R)>;
  R *X = reinterpret_cast<R *>(base + L::X);
  const R *wlo = reinterpret_cast<const R *>(base + L::WLO);
  const R *whi = reinterpret_cast<const R *>(base + L::WHI);
  const bool lo = x0 == 0, hi = x0 + kBX == nx;
  for (int i = threadIdx.x; i < 3 * kBZ * kBY * kHX; i += blockDim.x) {
    const int k = i % kHX, row = i / kHX;   // row = (c*BZ + z)*BY + y
    if (lo) X[row * kSX + k] = wlo[i];
    if (hi) X[row * kSX + kHX + kBX + k] = whi[i];
  }
}

// shared-memory address of component c of the neighbour at offset o along axis ax of the
// brick-local node (lx, ly, lz)
template <typename R>
__device__ __forceinline__ const R *brick_at(const unsigned char *base, int ax, int o, int c, int lx, int ly, int lz) {
  using L = BrickLayout<sizeof(R)>;
  const R *X = reinterpret_cast<const R *>(base + L::X);
  if (ax == 0) return X + ((c * kBZ + lz) * kBY + ly) * kSX + kHX + lx + o;
  if (ax == 1) {
    const int d = ly + o;
    if (d < 0) return reinterpret_cast<const R *>(base + L::YLO) + ((c * kBZ + lz) * kH + d + kH) * kBX + lx;
    if (d >= kBY) return reinterpret_cast<const R *>(base + L::YHI) + ((c * kBZ + lz) * kH + d - kBY) * kBX + lx;
    return X + ((c * kBZ + lz) * kBY + d) * kSX + kHX + lx;
  }
  const int d = lz + o;
  if (d < 0) return reinterpret_cast<const R *>(base + L::ZLO) + ((c * kH + d + kH) * kBY + ly) * kBX + lx;
  if (d >= kBZ) return reinterpret_cast<const R *>(base + L::ZHI) + ((c * kH + d - kBZ) * kBY + ly) * kBX + lx;
  return X + ((c * kBZ + d) * kBY + ly) * kSX + kHX + lx;
}

}  // namespace ieq
