// stage_col.cuh -- the column form of the fused stage kernel and of curl(B)/rho, used by
// the time stepping on the structure-of-arrays state.
//
// Each thread advances a column of NZ nodes adjacent in z (IEQ_COL_NODES).  The x and y
// derivative rows are gathered per node as in k_stage; along z the nodes of a column share
// their stencil planes: the planes iz0-RI .. iz0+NZ-1+RI are loaded once and each is
// accumulated into every node's sums with its own coefficient.  A column that meets the
// SBP boundary rows in z (non-periodic box) falls back to per-node gathers.
//
// Hall term.  The Hall volume flux of axis a at a stencil point k is J_a B_i - J_i B_a
// (induction_Eq_volume.cl Hall_volume), an entry of the antisymmetric tensor of J and B
// whose three independent entries are E = (Jx By - Jy Bx, Jx Bz - Jz Bx, Jy Bz - Jz By).
// k_curl_e computes J = curl(B)/rho and writes E (and J itself on the faces of a
// non-periodic box, where the outflow SAT needs it), so the stage kernel reads two values
// per stencil point and axis instead of six and forms no products there.
#pragma once
#include "stage_kernel.cuh"

namespace ieq {

// Nodes per thread along z and the register cap (via resident blocks of 128 threads).
// Measured on B200 for the 6th-order Hall + HOD stage (64^3 .. 128^3): one node per thread
// at <= 64 registers (8 blocks per SM) beats two- and four-node columns, whose extra
// registers cost more latency hiding than the shared z planes save.
#ifndef IEQ_COL_NODES
#define IEQ_COL_NODES 1
#endif
#ifndef IEQ_COL_MIN_BLOCKS
#define IEQ_COL_MIN_BLOCKS 8
#endif
#ifndef IEQ_COL_CONV_MIN_BLOCKS
#define IEQ_COL_CONV_MIN_BLOCKS 8
#endif
#ifndef IEQ_CURL_NODES
#define IEQ_CURL_NODES 1
#endif
// every column kernel runs 128-thread blocks; their x-y-z shape is a run-time choice
// (ColShape), since the kernels index with blockDim
constexpr int kColThreads = 128;
constexpr int kColNodes = IEQ_COL_NODES;     // nodes per thread along z (stage kernel)
constexpr int kCurlNodes = IEQ_CURL_NODES;   // nodes per thread along z (curl kernel)
// the convection terms keep twelve sums per node and axis: one node per thread there
__host__ __device__ constexpr int col_nodes(int conv) { return conv ? 1 : kColNodes; }

template <typename R>
__device__ __forceinline__ R cmp(const V3<R> &v, int ax) {
  return ax == 0 ? v.x : (ax == 1 ? v.y : v.z);
}

// Programmatic dependent launch: the curl and stage kernels of consecutive stages depend on
// each other's complete output.  Launched with programmatic stream serialization (launch_pdl), a kernel may be scheduled while its predecessor still runs; each block first
// waits for the predecessor grid to complete and its writes to be visible (griddepcontrol.wait,
// a hardware dependency wait that ends when the predecessor ends) and only then allows its own
// dependents to be scheduled (griddepcontrol.launch_dependents).  No block reads or writes
// fields before its wait, and a kernel never runs more than one launch ahead.  Launched
// without the attribute both instructions return at once.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename Kern, typename... Args>
inline void launch_pdl(Kern kernel, dim3 grid, dim3 block, cudaStream_t s, bool pdl, const Args &...a) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kernel, a...);
}

template <typename R>
struct ColSums {
  V3<R> SuiBa, SU, SB, SuaB, SHo;
  R h1, h2;   // sum_k c_k E_c1(k), sum_k c_k E_c2(k) (see e_comp*)
  V3<R> SFo;  // (FOF) sum_k (|c_k| max(|u_k|, |u_m|)) (B_k - B_m) of first-order dissipation
};

// one stencil point of the first-order dissipation of the axis (artificial_dissipation.cl
// :36-78, the terms of fo_ad_dissipation in the same order): skipped where the derivative
// coefficient is zero, as there
template <typename R>
__device__ __forceinline__ void fo_acc(ColSums<R> &s, R cD, const V3<R> &B, const V3<R> &U, const V3<R> &Bm,
                                       const V3<R> &Um) {
  const R cd = fabs(cD);
  if (cd == (R)0) return;
  s.SFo.x += (cd * fmax(fabs(U.x), fabs(Um.x))) * (B.x - Bm.x);
  s.SFo.y += (cd * fmax(fabs(U.y), fabs(Um.y))) * (B.y - Bm.y);
  s.SFo.z += (cd * fmax(fabs(U.z), fabs(Um.z))) * (B.z - Bm.z);
}
// the axis' first-order term into the node's sum: acc += tmp / DX (fo_ad_dissipation's order)
template <typename R>
__device__ __forceinline__ void fo_combine(const R *dR, int ax, const ColSums<R> &s, V3<R> &fo) {
  fo.x += s.SFo.x / dR[ax];
  fo.y += s.SFo.y / dR[ax];
  fo.z += s.SFo.z / dR[ax];
}

// The two entries of E the Hall flux of axis ax needs, and their signs in DB:
//   ax 0: DB_y += D[Exy], DB_z += D[Exz];  ax 1: DB_x -= D[Exy], DB_z += D[Eyz];
//   ax 2: DB_x -= D[Exz], DB_y -= D[Eyz]
__host__ __device__ constexpr int e_comp1(int ax) { return ax == 2 ? 1 : 0; }
__host__ __device__ constexpr int e_comp2(int ax) { return ax == 0 ? 1 : 2; }

// one stencil point: dterm adds the derivative-row terms (conv, Hall), hterm the dissipation
template <typename R, bool HALL, bool HOD, int CONV>
__device__ __forceinline__ void col_acc(ColSums<R> &s, int ax, int need, R cD, R cH, bool dterm, bool hterm,
                                        const V3<R> &B, const V3<R> &U, R e1, R e2) {
  if (CONV && dterm) {
    const R Ba = cmp(B, ax), Ua = cmp(U, ax);
    if (need & 1) {
      s.SuiBa.x += cD * (U.x * Ba); s.SuiBa.y += cD * (U.y * Ba); s.SuiBa.z += cD * (U.z * Ba);
    }
    if (need & 2) { s.SU.x += cD * U.x; s.SU.y += cD * U.y; s.SU.z += cD * U.z; }
    if (need & 4) { s.SB.x += cD * B.x; s.SB.y += cD * B.y; s.SB.z += cD * B.z; }
    if (need & 8) {
      s.SuaB.x += cD * (Ua * B.x); s.SuaB.y += cD * (Ua * B.y); s.SuaB.z += cD * (Ua * B.z);
    }
  }
  if (HALL && dterm) {
    s.h1 += cD * e1;
    s.h2 += cD * e2;
  }
  if (HOD && hterm) {
    s.SHo.x += cH * B.x; s.SHo.y += cH * B.y; s.SHo.z += cH * B.z;
  }
}

template <typename R, bool HALL, bool HOD, int CONV, typename F = SoA<R>>
__device__ __forceinline__ void col_load(const StageArgs<R, F> &a, int ax, long long j, V3<R> &B, V3<R> &U,
                                         R &e1, R &e2) {
  if (CONV || HOD) B = ldf(a.bk, j);
  if (CONV) U = ldf(a.u, j);
  if (HALL) {
    e1 = __ldg(a.E.p + j + e_comp1(ax) * a.E.s);
    e2 = __ldg(a.E.p + j + e_comp2(ax) * a.E.s);
  }
}

// the sums of one axis at one node (interior row, periodic wrap or SBP boundary row);
// NEED >= 0 fixes the flux-form mask (StageArgs::need) at compile time
// FOF: also the first-order dissipation terms of the axis (*Um: u at the node)
template <typename R, int OP, bool PER, bool HALL, bool HOD, int CONV, typename F = SoA<R>, int NEED = -1,
          bool FOF = false>
__device__ __forceinline__ void col_axis(ColSums<R> &s, const StageArgs<R, F> &a, int ax, int i, int n,
                                         long long idx, long long st, const V3<R> &Bm,
                                         const V3<R> *Um = nullptr) {
  const int need = NEED >= 0 ? NEED : a.need;
  constexpr int NB = Op<OP>::NB, SW = Op<OP>::SW, C0 = (SW - 1) / 2, WH = Op<OP>::WH, RI = Op<OP>::RI;
  constexpr int RB = (C0 > WH - 1) ? C0 : WH - 1;
  const V3<R> zero = {0, 0, 0};
  const int row = PER ? NB : sbp_row(i, n, NB);
  if (row == NB) {
    const bool wrap = PER && (i < RI || i >= n - RI);
#pragma unroll
    for (int o = -RI; o <= RI; ++o) {
      if (o == 0) {
        // the interior derivative rows have a zero centre
        if (HOD) col_acc<R, false, HOD, 0>(s, ax, 0, (R)0, a.Hint[RI], false, true, Bm, zero, (R)0, (R)0);
        continue;
      }
      const long long j = wrap ? idx + (long long)(nbr<true>(i, o, n) - i) * st : idx + (long long)o * st;
      V3<R> B = zero, U = zero;
      R e1 = 0, e2 = 0;
      col_load<R, HALL, HOD, CONV, F>(a, ax, j, B, U, e1, e2);
      col_acc<R, HALL, HOD, CONV>(s, ax, need, a.Dint[o + RI], a.Hint[o + RI], true, true, B, U, e1, e2);
      if (FOF) fo_acc(s, a.Dint[o + RI], B, U, Bm, *Um);
    }
  } else {
    for (int o = -RB; o <= RB; ++o) {
      const R cD = (o >= -C0 && o <= C0) ? a.tab->D[row][o + C0] : (R)0;
      const R cH = (HOD && o >= -(WH - 1) && o <= WH - 1) ? a.tab->H[row][o + WH - 1] : (R)0;
      if (cD == (R)0 && cH == (R)0) continue;
      const long long j = idx + (long long)(nbr<PER>(i, o, n) - i) * st;
      V3<R> B = zero, U = zero;
      R e1 = 0, e2 = 0;
      col_load<R, HALL, HOD, CONV, F>(a, ax, j, B, U, e1, e2);
      col_acc<R, HALL, HOD, CONV>(s, ax, need, cD, cH, cD != (R)0, cH != (R)0, B, U, e1, e2);
      if (FOF) fo_acc(s, cD, B, U, Bm, *Um);
    }
  }
}

// add one axis' sums into DB (volume and Hall terms) and the dissipation sum
template <typename R, bool HALL, bool HOD, int CONV, typename F = SoA<R>>
__device__ __forceinline__ void col_combine(const StageArgs<R, F> &a, int ax, const ColSums<R> &s,
                                            const V3<R> &Bm, const V3<R> &um, V3<R> &db, V3<R> &hod) {
  if (CONV) {
    const R Ba = cmp(Bm, ax), Ua = cmp(um, ax);
    const R SBa = cmp(s.SB, ax), SUa = cmp(s.SU, ax);
    const R *w = a.w;
    V3<R> vol;
    vol.x = w[0] * s.SuiBa.x + w[1] * Ba * s.SU.x + w[2] * um.x * SBa -
            (w[3] * s.SuaB.x + w[4] * Ua * s.SB.x + w[5] * Bm.x * SUa);
    vol.y = w[0] * s.SuiBa.y + w[1] * Ba * s.SU.y + w[2] * um.y * SBa -
            (w[3] * s.SuaB.y + w[4] * Ua * s.SB.y + w[5] * Bm.y * SUa);
    vol.z = w[0] * s.SuiBa.z + w[1] * Ba * s.SU.z + w[2] * um.z * SBa -
            (w[3] * s.SuaB.z + w[4] * Ua * s.SB.z + w[5] * Bm.z * SUa);
    db.x += a.two_inv_d[ax] * vol.x;
    db.y += a.two_inv_d[ax] * vol.y;
    db.z += a.two_inv_d[ax] * vol.z;
  }
  if (HALL) {
    const R f1 = a.inv_d[ax] * s.h1, f2 = a.inv_d[ax] * s.h2;
    if (ax == 0) {
      db.y += f1; db.z += f2;
    } else if (ax == 1) {
      db.x -= f1; db.z += f2;
    } else {
      db.x -= f1; db.y -= f2;
    }
  }
  if (HOD) {
    hod.x += s.SHo.x; hod.y += s.SHo.y; hod.z += s.SHo.z;
  }
}

// HODP: the dissipation sum comes precomputed (a.Hpre, written by k_curl_e_hod in the
// same order of operations) instead of being gathered here
// FOAD: first-order or adaptive dissipation (fo_ad_dissipation, after the SAT terms)
template <typename R, int OP, bool PER, bool HALL, bool HOD_, int CONV, int NEED = -1, bool HODP = false,
          bool FOAD = false>
__global__ void __launch_bounds__(kColThreads, (CONV ? IEQ_COL_CONV_MIN_BLOCKS : IEQ_COL_MIN_BLOCKS) * 128 / kColThreads) k_stage_col(const __grid_constant__ StageArgs<R, SoA<R>> a) {
  constexpr int NB = Op<OP>::NB, RI = Op<OP>::RI;
  pdl_enter();
  constexpr bool HOD = HOD_ && !HODP;   // the dissipation rows gathered in this kernel
  const int need = NEED >= 0 ? NEED : a.need;
  constexpr int NZ = col_nodes(CONV);
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz0 = (blockIdx.z * blockDim.z + threadIdx.z) * NZ;
  if (ix < nx && iy < ny && iz0 < nz) {
    const int cnt = nz - iz0 < NZ ? nz - iz0 : NZ;
    const long long sz = (long long)nx * ny;
    const long long base = ix + (long long)nx * iy;
    const V3<R> zero = {0, 0, 0};
    V3<R> Bm[NZ], um[NZ], db[NZ], hod[NZ];
#pragma unroll
    for (int k = 0; k < NZ; ++k) {
      db[k] = zero;
      hod[k] = zero;
      Bm[k] = zero;
      um[k] = zero;
      if (k < cnt) {
        const long long idx = base + (long long)(iz0 + k) * sz;
        Bm[k] = ldf(a.bk, idx);
        if (CONV) um[k] = ldf(a.u, idx);
      }
    }
    // x and y: per-node gathers
#pragma unroll
    for (int k = 0; k < NZ; ++k) {
      if (k < cnt) {
        const long long idx = base + (long long)(iz0 + k) * sz;
#pragma unroll
        for (int ax = 0; ax < 2; ++ax) {
          ColSums<R> s{};
          col_axis<R, OP, PER, HALL, HOD, CONV, SoA<R>, NEED>(s, a, ax, ax == 0 ? ix : iy, ax == 0 ? nx : ny, idx,
                                                             ax == 0 ? 1 : nx, Bm[k]);
          col_combine<R, HALL, HOD, CONV>(a, ax, s, Bm[k], um[k], db[k], hod[k]);
        }
      }
    }
    // z: shared stencil planes when the whole column uses the interior row
    const bool stream = cnt == NZ && (PER || (sbp_row(iz0, nz, NB) == NB && sbp_row(iz0 + NZ - 1, nz, NB) == NB));
    if (stream) {
      ColSums<R> s[NZ];
#pragma unroll
      for (int k = 0; k < NZ; ++k) s[k] = ColSums<R>{};
#pragma unroll
      for (int p = -RI; p <= NZ - 1 + RI; ++p) {
        int zz = iz0 + p;
        if (PER) {
          zz += zz < 0 ? nz : 0;
          zz -= zz >= nz ? nz : 0;
        }
        const long long j = base + (long long)zz * sz;
        V3<R> B = zero, U = zero;
        R e1 = 0, e2 = 0;
        if (p >= 0 && p < NZ) {
          B = Bm[p];
          U = um[p];
          if (HALL) {
            e1 = __ldg(a.E.p + j + e_comp1(2) * a.E.s);
            e2 = __ldg(a.E.p + j + e_comp2(2) * a.E.s);
          }
        } else {
          col_load<R, HALL, HOD, CONV>(a, 2, j, B, U, e1, e2);
        }
#pragma unroll
        for (int k = 0; k < NZ; ++k) {
          const int o = p - k;
          if (o < -RI || o > RI) continue;
          if (o == 0) {
            if (HOD) col_acc<R, false, HOD, 0>(s[k], 2, 0, (R)0, a.Hint[RI], false, true, B, zero, (R)0, (R)0);
          } else {
            col_acc<R, HALL, HOD, CONV>(s[k], 2, need, a.Dint[o + RI], a.Hint[o + RI], true, true, B, U, e1, e2);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < NZ; ++k) col_combine<R, HALL, HOD, CONV>(a, 2, s[k], Bm[k], um[k], db[k], hod[k]);
    } else {
#pragma unroll
      for (int k = 0; k < NZ; ++k) {
        if (k < cnt) {
          const long long idx = base + (long long)(iz0 + k) * sz;
          ColSums<R> s{};
          col_axis<R, OP, PER, HALL, HOD, CONV, SoA<R>, NEED>(s, a, 2, iz0 + k, nz, idx, sz, Bm[k]);
          col_combine<R, HALL, HOD, CONV>(a, 2, s, Bm[k], um[k], db[k], hod[k]);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < NZ; ++k) {
      if (k < cnt) {
        const int ii[3] = {ix, iy, iz0 + k};
        const int nn[3] = {nx, ny, nz};
        const long long idx = base + (long long)(iz0 + k) * sz;
        V3<R> d = db[k];
        if (!PER) stage_sat<R, SoA<R>, HALL>(a, ii, nn, idx, Bm[k], um[k], CONV, d);
        if (HOD_) {
          const V3<R> hv = HODP ? ldf(a.Hpre, idx) : hod[k];
          d.x += a.hod_factor * hv.x;
          d.y += a.hod_factor * hv.y;
          d.z += a.hod_factor * hv.z;
        }
        if (FOAD) {
          const long long st[3] = {1, nx, sz};
          const V3<R> ds = fo_ad_dissipation<R, SoA<R>, OP, PER>(a, ii, nn, st, idx, Bm[k], um[k]);
          d.x += ds.x; d.y += ds.y; d.z += ds.z;
        }
        stage_epilogue<R, SoA<R>>(a, idx, d);
      }
    }
  }
  stage_time_post(a);
}

// J = curl(B)/rho and E = J x B, two nodes per thread along z (see the file comment)
template <typename R, int OP, bool PER>
__global__ void __launch_bounds__(kColThreads) k_curl_e(const __grid_constant__ CurlArgs<R, SoA<R>> a) {
  constexpr int NB = Op<OP>::NB, SW = Op<OP>::SW, C0 = (SW - 1) / 2, RI = Op<OP>::RI;
  pdl_enter();
  constexpr int NZ = kCurlNodes;
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz0 = (blockIdx.z * blockDim.z + threadIdx.z) * NZ;
  if (ix >= nx || iy >= ny || iz0 >= nz) return;
  const int cnt = nz - iz0 < NZ ? nz - iz0 : NZ;
  const long long sz = (long long)nx * ny;
  const long long base = ix + (long long)nx * iy;
  const int nn[3] = {nx, ny, nz};
  const long long st[3] = {1, nx, sz};
  R g[NZ][3][3];   // g[node][axis][component]
  // one axis at one node: the derivatives of the two components orthogonal to it
  auto axis = [&](int ax, int i, long long idx, R &v1, R &v2) {
    const int c1 = (ax + 1) % 3, c2 = (ax + 2) % 3;
    v1 = 0;
    v2 = 0;
    const int row = PER ? NB : sbp_row(i, nn[ax], NB);
    if (row == NB) {
      const bool wrap = PER && (i < RI || i >= nn[ax] - RI);
#pragma unroll
      for (int o = -RI; o <= RI; ++o) {
        if (o == 0) continue;
        const R c = a.Dint[o + RI];
        const long long j = wrap ? idx + (long long)(nbr<true>(i, o, nn[ax]) - i) * st[ax] : idx + (long long)o * st[ax];
        v1 += c * __ldg(a.b.p + j + c1 * a.b.s);
        v2 += c * __ldg(a.b.p + j + c2 * a.b.s);
      }
    } else {
      for (int o = -C0; o <= C0; ++o) {
        const R c = a.tab->D[row][o + C0];
        if (c == (R)0) continue;
        const long long j = idx + (long long)(nbr<PER>(i, o, nn[ax]) - i) * st[ax];
        v1 += c * __ldg(a.b.p + j + c1 * a.b.s);
        v2 += c * __ldg(a.b.p + j + c2 * a.b.s);
      }
    }
  };
#pragma unroll
  for (int k = 0; k < NZ; ++k) {
    if (k < cnt) {
      const long long idx = base + (long long)(iz0 + k) * sz;
#pragma unroll
      for (int ax = 0; ax < 2; ++ax) {
        R v1, v2;
        axis(ax, ax == 0 ? ix : iy, idx, v1, v2);
        g[k][ax][(ax + 1) % 3] = v1 * a.inv_d[ax];
        g[k][ax][(ax + 2) % 3] = v2 * a.inv_d[ax];
      }
    }
  }
  const bool stream = cnt == NZ && (PER || (sbp_row(iz0, nz, NB) == NB && sbp_row(iz0 + NZ - 1, nz, NB) == NB));
  if (stream) {
    R v1[NZ], v2[NZ];
#pragma unroll
    for (int k = 0; k < NZ; ++k) v1[k] = v2[k] = 0;
#pragma unroll
    for (int p = -RI; p <= NZ - 1 + RI; ++p) {
      // the plane is used by some node at a non-zero offset
      bool used = false;
#pragma unroll
      for (int k = 0; k < NZ; ++k) used |= (p - k >= -RI && p - k <= RI && p != k);
      if (!used) continue;
      int zz = iz0 + p;
      if (PER) {
        zz += zz < 0 ? nz : 0;
        zz -= zz >= nz ? nz : 0;
      }
      const long long j = base + (long long)zz * sz;
      const R bx = __ldg(a.b.p + j), by = __ldg(a.b.p + j + a.b.s);
#pragma unroll
      for (int k = 0; k < NZ; ++k) {
        const int o = p - k;
        if (o < -RI || o > RI || o == 0) continue;
        v1[k] += a.Dint[o + RI] * bx;
        v2[k] += a.Dint[o + RI] * by;
      }
    }
#pragma unroll
    for (int k = 0; k < NZ; ++k) {
      g[k][2][0] = v1[k] * a.inv_d[2];
      g[k][2][1] = v2[k] * a.inv_d[2];
    }
  } else {
#pragma unroll
    for (int k = 0; k < NZ; ++k) {
      if (k < cnt) {
        R v1, v2;
        axis(2, iz0 + k, base + (long long)(iz0 + k) * sz, v1, v2);
        g[k][2][0] = v1 * a.inv_d[2];
        g[k][2][1] = v2 * a.inv_d[2];
      }
    }
  }
#pragma unroll
  for (int k = 0; k < NZ; ++k) {
    if (k < cnt) {
      const int iz = iz0 + k;
      const long long idx = base + (long long)iz * sz;
      V3<R> J = {g[k][1][2] - g[k][2][1], g[k][2][0] - g[k][0][2], g[k][0][1] - g[k][1][0]};
      if (a.rho) {
        const R r = (R)1 / a.rho[idx];
        J = {J.x * r, J.y * r, J.z * r};
      }
      const V3<R> B = ldf(a.b, idx);
      stf(a.out, idx, V3<R>{J.x * B.y - J.y * B.x, J.x * B.z - J.z * B.x, J.y * B.z - J.z * B.y});
      if (!PER && (ix == 0 || iy == 0 || iz == 0 || ix == nx - 1 || iy == ny - 1 || iz == nz - 1))
        stf(a.jface, idx, J);
    }
  }
}

// one axis of the curl at one node: the derivatives v1, v2 of the two components of B
// orthogonal to the axis and, with HODS, the dissipation-row sum ho of all three (interior
// row, periodic wrap or SBP boundary rows; each sum term by term in stencil order)
template <typename R, int OP, bool PER, bool HODS>
__device__ __forceinline__ void curl_axis_node(const CurlArgs<R, SoA<R>> &a, int ax, int i, int n, long long idx,
                                               long long st, const V3<R> &Bm, R &v1, R &v2, V3<R> &ho) {
  constexpr int NB = Op<OP>::NB, SW = Op<OP>::SW, C0 = (SW - 1) / 2, WH = Op<OP>::WH, RI = Op<OP>::RI;
  constexpr int RB = HODS ? ((C0 > WH - 1) ? C0 : WH - 1) : C0;
  const int c1 = (ax + 1) % 3, c2 = (ax + 2) % 3;
  v1 = 0;
  v2 = 0;
  ho = {0, 0, 0};
  const int row = PER ? NB : sbp_row(i, n, NB);
  if (row == NB) {
    const bool wrap = PER && (i < RI || i >= n - RI);
#pragma unroll
    for (int o = -RI; o <= RI; ++o) {
      const R cH = a.Hint[o + RI];
      if (o == 0) {
        if (HODS) {
          ho.x += cH * Bm.x; ho.y += cH * Bm.y; ho.z += cH * Bm.z;
        }
        continue;
      }
      const long long j = wrap ? idx + (long long)(nbr<true>(i, o, n) - i) * st : idx + (long long)o * st;
      const R c = a.Dint[o + RI];
      if (HODS) {
        const V3<R> B = ldf(a.b, j);
        v1 += c * cmp(B, c1);
        v2 += c * cmp(B, c2);
        ho.x += cH * B.x; ho.y += cH * B.y; ho.z += cH * B.z;
      } else {
        v1 += c * __ldg(a.b.p + j + c1 * a.b.s);
        v2 += c * __ldg(a.b.p + j + c2 * a.b.s);
      }
    }
  } else {
    for (int o = -RB; o <= RB; ++o) {
      const R cD = (o >= -C0 && o <= C0) ? a.tab->D[row][o + C0] : (R)0;
      const R cH = (HODS && o >= -(WH - 1) && o <= WH - 1) ? a.tab->H[row][o + WH - 1] : (R)0;
      if (cD == (R)0 && cH == (R)0) continue;
      const long long j = idx + (long long)(nbr<PER>(i, o, n) - i) * st;
      if (HODS) {
        const V3<R> B = ldf(a.b, j);
        if (cD != (R)0) {
          v1 += cD * cmp(B, c1);
          v2 += cD * cmp(B, c2);
        }
        if (cH != (R)0) {
          ho.x += cH * B.x; ho.y += cH * B.y; ho.z += cH * B.z;
        }
      } else {
        v1 += cD * __ldg(a.b.p + j + c1 * a.b.s);
        v2 += cD * __ldg(a.b.p + j + c2 * a.b.s);
      }
    }
  }
}

// J = curl(B)/rho, E = J x B and, for the dissipation of the next stage kernel, the sum over
// the axes of the dissipation rows of B (one node per thread).  Every axis loads all three
// components of B at its stencil points once: the two orthogonal components feed the curl,
// all three the dissipation rows, in the order k_stage_col gathers them (so the stored sum
// equals the one the stage kernel would form).
// register cap of k_curl_e_hod (measured: <= 64 registers, 8 CTAs of 128 threads per SM,
// is 4-23 % faster than the uncapped 60-register build at 64^3 .. 128^3)
#ifndef IEQ_CURL_MIN_BLOCKS
#define IEQ_CURL_MIN_BLOCKS 8
#endif
template <typename R, int OP, bool PER>
__global__ void __launch_bounds__(kColThreads, IEQ_CURL_MIN_BLOCKS * 128 / kColThreads)
    k_curl_e_hod(const __grid_constant__ CurlArgs<R, SoA<R>> a) {
  pdl_enter();
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z;
  if (ix >= nx || iy >= ny || iz >= nz) return;
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
    curl_axis_node<R, OP, PER, true>(a, ax, ii[ax], nn[ax], idx, st[ax], Bm, v1, v2, ho);
    g[ax][c1] = v1 * a.inv_d[ax];
    g[ax][c2] = v2 * a.inv_d[ax];
    hod.x += ho.x; hod.y += ho.y; hod.z += ho.z;
  }
  V3<R> J = {g[1][2] - g[2][1], g[2][0] - g[0][2], g[0][1] - g[1][0]};
  if (a.rho) {
    const R r = (R)1 / a.rho[idx];
    J = {J.x * r, J.y * r, J.z * r};
  }
  stf(a.out, idx, V3<R>{J.x * Bm.y - J.y * Bm.x, J.x * Bm.z - J.z * Bm.x, J.y * Bm.z - J.z * Bm.y});
  stf(a.hout, idx, hod);
  if (!PER && (ix == 0 || iy == 0 || iz == 0 || ix == nx - 1 || iy == ny - 1 || iz == nz - 1))
    stf(a.jface, idx, J);
}

// SSPRK104_06 (kernel_time_integrator.cl, between stages 5 and 7) on the SoA state:
// b3 = 0.04 b1 + 0.36 b2; b2 = 0.6 b1 + 0.4 b2; the last block sets time[1] = time[0] + tK
template <typename R>
__global__ void k_soa_ssp104_06(long long n, SoA<R> b1, SoA<R> b2, SoA<R> b3, R *time, R tK, unsigned *counter) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) {
    const V3<R> p = ldf_plain(b1, i), q = ldf_plain(b2, i);
    stf(b3, i, V3<R>{(R)0.04 * p.x + (R)0.36 * q.x, (R)0.04 * p.y + (R)0.36 * q.y, (R)0.04 * p.z + (R)0.36 * q.z});
    stf(b2, i, V3<R>{(R)0.60 * p.x + (R)0.40 * q.x, (R)0.60 * p.y + (R)0.40 * q.y, (R)0.60 * p.z + (R)0.40 * q.z});
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(counter, 1u) == gridDim.x - 1) {
      time[1] = time[0] + tK;
      __threadfence();
      *counter = 0u;
    }
  }
}

// launch shape of the column kernels: x * y * z == kColThreads threads, each `nodes` nodes
// in z.  32 x 4 x 1 keeps every warp on one x row (two full 128-byte lines per FP64 load).
// pairs: the Hall kernels that have the form (stage_x2.cuh) give each thread two
// x-adjacent nodes where the fields allow it.
struct ColShape {
  int x = 32, y = 4, z = 1;
  bool pairs = true;
  bool pdl = true;     // programmatic dependent launch of the column kernels
  bool given = false;  // the shape was set explicitly (else the kernels' defaults apply)
  bool quads = false;  // FP32 Hall kernels: four nodes per thread on every grid that allows it
  int band = 1;        // boxes: x boundary columns in a launch of their own (stage_x2.cuh):
                       // 0 never, 1 where measured faster, 2 wherever the rows allow
};
// the default shape of the pair kernels, measured on B200 (Hall whistler, 6th order + HOD):
// the curl kernel 32 x 2 x 2 (64^3: 6.24 us against 6.46 for 32 x 4 x 1; 128^3: equal); the
// stage kernel 32 x 2 x 2 while the fields stay L2 resident (<= 2^20 nodes; 64^3: 7.20
// against 7.32 us) and 32 x 4 x 1 above (128^3: 53.1 against 53.7 us)
// Rows that are not a multiple of 32 threads long (nxe = nodes, or node pairs, per x row)
// get a block x extent that divides them evenly: ceil(nxe / ceil(nxe / 32)) threads, the
// other dimensions refilled towards 128 threads (a 16-node row as 32 threads would leave
// half the lanes idle; the batched form's small grids are of this kind).
inline ColShape fit_rows(ColShape sh, int nxe) {
  if (sh.given || nxe % 32 == 0) return sh;
  const int nbx = (nxe + 31) / 32;
  sh.x = (nxe + nbx - 1) / nbx;
  const int yz = kColThreads / sh.x;
  sh.z = sh.z > 1 && yz >= 2 ? 2 : 1;
  sh.y = yz / sh.z > 0 ? yz / sh.z : 1;
  return sh;
}
inline ColShape pair_shape(ColShape sh, bool curl, long long nodes, int nx, int K = 2) {
  if (!sh.given && (curl || nodes <= (1ll << 20))) {
    sh.x = 32;
    sh.y = 2;
    sh.z = 2;
  }
  return fit_rows(sh, nx / K);
}
inline dim3 col_block(ColShape sh) { return dim3((unsigned)sh.x, (unsigned)sh.y, (unsigned)sh.z); }
inline dim3 col_grid(ColShape sh, int nx, int ny, int nz, int nodes) {
  const int zb = sh.z * nodes;
  return dim3((unsigned)((nx + sh.x - 1) / sh.x), (unsigned)((ny + sh.y - 1) / sh.y), (unsigned)((nz + zb - 1) / zb));
}

template <typename R, int OP>
void launch_stage_col(const StageArgs<R, SoA<R>> &a, bool per, bool hall, bool hod, int conv, bool hodp,
                      bool foad, ColShape sh, cudaStream_t s);
template <typename R, int OP>
void launch_curl_e(const CurlArgs<R, SoA<R>> &a, bool per, bool hod, ColShape sh, cudaStream_t s);

}  // namespace ieq
