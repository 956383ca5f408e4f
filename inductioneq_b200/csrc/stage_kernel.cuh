// stage_kernel.cuh -- the fused Runge-Kutta stage kernel and the curl(B)/rho kernel.
//
// One thread per node.  For every node the kernel evaluates the time derivative DB of
// kernel/kernel_time_integrator.cl:9-31 -- volume terms (induction_Eq_volume.cl),
// Hall volume term, SAT surface terms (induction_Eq_surface.cl) and artificial
// dissipation (artificial_dissipation.cl) -- and applies the stage update of the
// integrator in the same pass (epilogue modes below), so the stage derivative never
// touches memory.
//
// Volume term.  The reference sums the split-form flux F(B_m,u_m,B_k,u_k) over the
// stencil points k of each derivative row.  Every flux form is bilinear in (m, k)
// quantities, so with D applied to the pointwise products the sum factors into
//     sum_k c_k F = w1 D[u_i B_a] + w2 B_a,m D[u_i] + w3 u_i,m D[B_a]
//                 - (v1 D[u_a B_i] + v2 u_a,m D[B_i] + v3 B_i,m D[u_a])
// (plus terms proportional to sum_k c_k, which is zero for every derivative row);
// w and v come from the USE_UIBJ_* / USE_SOURCE_* / USE_UJBI_* switches.  This cuts the
// flops per stencil point from ~40 to 9-21 and changes only the rounding order.
//
// Interior nodes of every axis use the interior row (radius RI = ORDER/2, coefficients
// in kernel parameters); the SBP boundary closures read their rows from a table.
#pragma once
#include "ieq_common.cuh"

namespace ieq {

// ---- field layouts: REAL4 array-of-structs (the reference's layout, used by the per-kernel
// entry points) and structure-of-arrays (x, y, z planes of one allocation, component stride s;
// used by the fused time stepping: a warp's neighbour load is 256 contiguous bytes).
template <typename R>
struct AoS {
  R4<R> *p;
};
template <typename R>
struct SoA {
  R *p;
  long long s;
  int ro;     // (used by SoAcg only) the field is never written during the launch
};
// SoA for a persistent kernel that reads, in a later stage, data other blocks wrote in an
// earlier stage of the same launch.  Such data must not go through the non-coherent
// read-only path (ld.global.nc); ordinary loads (ld.global.ca) issued after the fenced grid
// barrier observe the other blocks' writes.  A field marked `ro` (never written during the
// launch) keeps the read-only path.
template <typename R>
struct SoAcg {
  R *p;
  long long s;
  int ro;
};
template <typename R>
__device__ __forceinline__ V3<R> ldf(const AoS<R> &f, long long j) { return ld3(f.p + j); }
template <typename R>
__device__ __forceinline__ V3<R> ldf(const SoAcg<R> &f, long long j) {
  if (f.ro) return {__ldg(f.p + j), __ldg(f.p + j + f.s), __ldg(f.p + j + 2 * f.s)};
  return {__ldca(f.p + j), __ldca(f.p + j + f.s), __ldca(f.p + j + 2 * f.s)};
}
template <typename R>
__device__ __forceinline__ V3<R> ldf_plain(const SoAcg<R> &f, long long j) {
  return {__ldca(f.p + j), __ldca(f.p + j + f.s), __ldca(f.p + j + 2 * f.s)};
}
template <typename R>
__device__ __forceinline__ void stf(const SoAcg<R> &f, long long j, V3<R> v) {
  f.p[j] = v.x;
  f.p[j + f.s] = v.y;
  f.p[j + 2 * f.s] = v.z;
}
template <typename R>
__device__ __forceinline__ V3<R> ldf(const SoA<R> &f, long long j) {
  return {__ldg(f.p + j), __ldg(f.p + j + f.s), __ldg(f.p + j + 2 * f.s)};
}
template <typename R>
__device__ __forceinline__ V3<R> ldf_plain(const AoS<R> &f, long long j) { return ld3_plain(f.p + j); }
template <typename R>
__device__ __forceinline__ V3<R> ldf_plain(const SoA<R> &f, long long j) {
  return {f.p[j], f.p[j + f.s], f.p[j + 2 * f.s]};
}
template <typename R>
__device__ __forceinline__ void stf(const AoS<R> &f, long long j, V3<R> v) { st3(f.p + j, v); }
template <typename R>
__device__ __forceinline__ void stf(const SoA<R> &f, long long j, V3<R> v) {
  f.p[j] = v.x;
  f.p[j + f.s] = v.y;
  f.p[j + 2 * f.s] = v.z;
}

enum EpilogueMode : int {
  EP_X_PLUS_HF = 0,   // out = X + h*F                 SSPRK33_1, SSPRK104, KCL_5, CFR_6
  EP_PX_QYHF = 1,     // out = p*X + q*(Y + h*F)       SSPRK33_2b/3b, SSPRK104_11b
  EP_HF = 2,          // out = h*F                     *_1a, KCL/CFR "a" kernels
  EP_AX_HF = 3,       // out = A*X + h*F               CarpenterKennedy/ToulorgeDesmet "a"
  EP_2N_FUSED = 4,    // t = A*X + h*F; out = t; out2 = Z + Bc*t     ("a" and "b" fused)
  EP_2N_FUSED_FIRST = 5,  // t = h*F; out = t; out2 = Z + Bc*t
  EP_2R_FUSED = 6,    // t = h*F; out = X + A*t; out2 = out + Bc*t; out3 = t (if set)   (2R "a" + "b")
};

enum TimePost : int {
  TP_NONE = 0,
  TP_SET_STAGE = 1,   // time[1] = time[0] + K
  TP_ADVANCE = 2,     // time[0] = time[0] + DT; time[1] = time[0]
};

enum DissKind : int { DISS_NONE = 0, DISS_HO = 1, DISS_FO_OR_AD = 2 };

template <typename R, typename F = AoS<R>>
struct StageArgs {
  Mesh m;
  F bk;                 // field the derivative is taken of
  F J;                  // curl(B)/rho (Hall; the column kernel reads it on faces only)
  F E;                  // (column kernel, Hall) J x B as (Jx By - Jy Bx, Jx Bz - Jz Bx, Jy Bz - Jz By)
  F Hpre;               // (column kernel) the dissipation sum of bk, precomputed by k_curl_e_hod
  F u;
  F X, Y, Z;
  F out, out2, out3;
  const Tables<R> *tab;
  R *time;
  unsigned *counter;    // last-block ticket for the time post-update
  R Dint[7];            // interior derivative row, offsets -RI..RI
  R Hint[7];            // interior dissipation row, offsets -RI..RI
  R two_inv_d[3];       // (REAL)(2.0/DX) ...
  R inv_d[3];           // (REAL)(1.0/DX) ...
  R sat_s[3];           // (REAL)(M_INV[0]/DX) ...
  R dR[3];              // (REAL)DX ...
  R w[6];               // flux-form weights w1 w2 w3 v1 v2 v3
  int need;             // 1: D[u_i B_a], 2: D[u], 4: D[B], 8: D[u_a B_i]
  int conv;             // convection terms present (u not identically zero) ...
  const int *conv_flag; // ... or, if set, read from device memory at kernel start
  int tc;               // testcase (b_boundary of the inflow SAT)
  int diss_form;        // 2 first order, 3 adaptive (DISS_FO_OR_AD)
  R hod_factor;
  double mp2min, mp2max, cmin, cmax;
  int mode;
  R p, q, h, A, Bc;
  int tpost;
  R tK, tDT;
};

// neighbour index along one axis: periodic wrap, or clamp-to-self outside the grid
// (include/utils.h:89-168; the coefficient of a clamped point is zero)
template <bool PER>
__device__ __forceinline__ int nbr(int i, int o, int n) {
  int j = i + o;
  if (PER) {
    j += (j < 0) ? n : 0;
    j -= (j >= n) ? n : 0;
  } else {
    j = (j < 0 || j >= n) ? i : j;
  }
  return j;
}

template <typename R>
struct AxisSums {
  V3<R> SuiBa, SU, SB, SuaB, SH, SHo;
};

// CHK: test the coefficients for zero at run time (boundary rows); the interior rows call
// this with compile-time knowledge instead (only the centre derivative coefficient is zero)
template <typename R, typename F, bool HALL, bool HOD, bool CHK>
__device__ __forceinline__ void accumulate(AxisSums<R> &s, const StageArgs<R, F> &a, int conv, int axis, R cD, R cH,
                                           long long j) {
  const V3<R> B = ldf(a.bk, j);
  if (conv && (!CHK || cD != (R)0)) {
    const V3<R> U = ldf(a.u, j);
    const R Ba = axis == 0 ? B.x : (axis == 1 ? B.y : B.z);
    const R Ua = axis == 0 ? U.x : (axis == 1 ? U.y : U.z);
    if (a.need & 1) {
      s.SuiBa.x += cD * (U.x * Ba); s.SuiBa.y += cD * (U.y * Ba); s.SuiBa.z += cD * (U.z * Ba);
    }
    if (a.need & 2) { s.SU.x += cD * U.x; s.SU.y += cD * U.y; s.SU.z += cD * U.z; }
    if (a.need & 4) { s.SB.x += cD * B.x; s.SB.y += cD * B.y; s.SB.z += cD * B.z; }
    if (a.need & 8) {
      s.SuaB.x += cD * (Ua * B.x); s.SuaB.y += cD * (Ua * B.y); s.SuaB.z += cD * (Ua * B.z);
    }
  }
  if (HALL && (!CHK || cD != (R)0)) {
    // Hall_volume: D[J_a B - J B_a]; the a-component is J_a B_a - J_a B_a = 0
    const V3<R> Jk = ldf(a.J, j);
    const R Ja = axis == 0 ? Jk.x : (axis == 1 ? Jk.y : Jk.z);
    const R Ba = axis == 0 ? B.x : (axis == 1 ? B.y : B.z);
    if (axis != 0) s.SH.x += cD * (Ja * B.x - Jk.x * Ba);
    if (axis != 1) s.SH.y += cD * (Ja * B.y - Jk.y * Ba);
    if (axis != 2) s.SH.z += cD * (Ja * B.z - Jk.z * Ba);
  }
  if (HOD && (!CHK || cH != (R)0)) {
    s.SHo.x += cH * B.x; s.SHo.y += cH * B.y; s.SHo.z += cH * B.z;
  }
}

// first-order / adaptive dissipation (artificial_dissipation.cl:36-160), evaluated as in
// the reference per stencil point; used only by the DISS_FO_OR_AD instantiation.
template <typename R, typename F, int OP, bool PER>
__device__ V3<R> fo_ad_dissipation(const StageArgs<R, F> &a, const int ii[3], const int nn[3],
                                   const long long st[3], long long idx, V3<R> Bm, V3<R> um) {
  constexpr int NB = Op<OP>::NB, SW = Op<OP>::SW, C0 = (SW - 1) / 2, WH = Op<OP>::WH;
  V3<R> acc = {0, 0, 0};
  const bool adaptive = a.diss_form == 3;
  auto kap = [&](unsigned k, R dx, R b1, R b2, R u1, R u2) -> R {
    // include/artificial_dissipation.h:23-45 (k*k of the unsigned argument)
    R s = (fmax(fabs(u1), fabs(u2)) * (b1 - b2)) * (b1 - b2);
    k = k + (k == 0);
    double kk = (double)(k * k);
    double lo = ((kk * a.mp2min) * a.cmin) * (double)dx;
    double hi = ((kk * a.mp2max) * a.cmax) * (double)dx;
    double sd = (double)s;
    double v = ((lo < sd) && (sd < hi)) * sqrt(fabs(sd - lo) / fabs(hi - lo)) + (double)(sd >= hi);
    return (R)v;
  };
  for (int ax = 0; ax < 3; ++ax) {
    const int row = PER ? NB : sbp_row(ii[ax], nn[ax], NB);
    V3<R> tmp = {0, 0, 0};
    for (int c = 0; c < SW; ++c) {
      const int o = c - C0;
      const R cd = fabs(a.tab->D[row][c]);
      if (cd == (R)0) continue;   // a zero coefficient adds a zero term: skip its loads
      const long long j = idx + (long long)(nbr<PER>(ii[ax], o, nn[ax]) - ii[ax]) * st[ax];
      const V3<R> Bk = ldf(a.bk, j);
      const V3<R> uk = ldf(a.u, j);
      V3<R> sg = {fmax(fabs(uk.x), fabs(um.x)), fmax(fabs(uk.y), fabs(um.y)), fmax(fabs(uk.z), fabs(um.z))};
      if (adaptive) {
        const unsigned k = (unsigned)(o < 0 ? -o : o);
        tmp.x += ((cd * kap(k, a.dR[ax], Bk.x, Bm.x, uk.x, um.x)) * sg.x) * (Bk.x - Bm.x);
        tmp.y += ((cd * kap(k, a.dR[ax], Bk.y, Bm.y, uk.y, um.y)) * sg.y) * (Bk.y - Bm.y);
        tmp.z += ((cd * kap(k, a.dR[ax], Bk.z, Bm.z, uk.z, um.z)) * sg.z) * (Bk.z - Bm.z);
      } else {
        tmp.x += (cd * sg.x) * (Bk.x - Bm.x);
        tmp.y += (cd * sg.y) * (Bk.y - Bm.y);
        tmp.z += (cd * sg.z) * (Bk.z - Bm.z);
      }
    }
    acc.x += tmp.x / a.dR[ax]; acc.y += tmp.y / a.dR[ax]; acc.z += tmp.z / a.dR[ax];
  }
  if (adaptive) {
    // high-order part weighted by (1 - kappa) of the neighbouring pair
    for (int term = -WH + 1; term <= 0; ++term) {
      for (int ax = 0; ax < 3; ++ax) {
        const int row = PER ? NB : sbp_row(ii[ax], nn[ax], NB);
        const long long j1 = idx + (long long)(nbr<PER>(ii[ax], term + WH - 1, nn[ax]) - ii[ax]) * st[ax];
        const long long j2 = idx + (long long)(nbr<PER>(ii[ax], term + WH - 2, nn[ax]) - ii[ax]) * st[ax];
        const V3<R> b1 = ldf(a.bk, j1), b2 = ldf(a.bk, j2), u1 = ldf(a.u, j1), u2 = ldf(a.u, j2);
        // diff_HOD (artificial_dissipation.h:58-101) for this start offset
        const R sgn = (Op<OP>::ORDER / 2 + 1) % 2 ? (R)-1 : (R)1;
        V3<R> hod = {0, 0, 0};
        for (int i = 0; i < WH; ++i) {
          const R coef = ((a.tab->Minv[row] * a.tab->DHO[row][term + WH - 1]) * a.tab->DHO[NB][i]) * sgn;
          const long long j = idx + (long long)(nbr<PER>(ii[ax], i + term, nn[ax]) - ii[ax]) * st[ax];
          const V3<R> Bk = ldf(a.bk, j);
          hod.x += coef * Bk.x; hod.y += coef * Bk.y; hod.z += coef * Bk.z;
        }
        acc.x += (((R)1 - kap(1, a.dR[ax], b1.x, b2.x, u1.x, u2.x)) * a.hod_factor) * hod.x;
        acc.y += (((R)1 - kap(1, a.dR[ax], b1.y, b2.y, u1.y, u2.y)) * a.hod_factor) * hod.y;
        acc.z += (((R)1 - kap(1, a.dR[ax], b1.z, b2.z, u1.z, u2.z)) * a.hod_factor) * hod.z;
      }
    }
  }
  return acc;
}

// SAT surface terms on the faces of a non-periodic box (added into db)
template <typename R, typename F, bool HALL>
__device__ __forceinline__ void stage_sat(const StageArgs<R, F> &a, const int ii[3], const int nn[3], long long idx,
                                          const V3<R> &Bm, const V3<R> &um, int conv, V3<R> &db) {
  const int ix = ii[0], iy = ii[1], iz = ii[2], nx = nn[0], ny = nn[1], nz = nn[2];
  const bool face = ix == 0 || iy == 0 || iz == 0 || ix == nx - 1 || iy == ny - 1 || iz == nz - 1;
  if (face) {
    if (HALL) {
      // induction_Eq_surface.cl:35-81 (outflow, directional do-nothing)
      const V3<R> Jm = ldf(a.J, idx);
      const V3<R> tv = {(R)0.5 * um.x - Jm.x, (R)0.5 * um.y - Jm.y, (R)0.5 * um.z - Jm.z};
      for (int ax = 0; ax < 3; ++ax) {
        const bool l = ii[ax] == 0, r = ii[ax] == nn[ax] - 1;
        if (!l && !r) continue;
        const R tva = ax == 0 ? tv.x : (ax == 1 ? tv.y : tv.z);
        const R Ba = ax == 0 ? Bm.x : (ax == 1 ? Bm.y : Bm.z);
        const R c1 = (l && tva > (R)0 ? (R)-1 : (R)0) + (r && tva < (R)0 ? (R)1 : (R)0);
        const R c2 = (l ? (R)-1 : (R)0) + (r ? (R)1 : (R)0);
        const R f1 = c1 * tva, f2 = c2 * Ba;
        db.x += a.sat_s[ax] * (f1 * Bm.x + f2 * Jm.x);
        db.y += a.sat_s[ax] * (f1 * Bm.y + f2 * Jm.y);
        db.z += a.sat_s[ax] * (f1 * Bm.z + f2 * Jm.z);
      }
    } else if (conv) {
      // induction_Eq_surface.cl:7-33 (upwind inflow against b_boundary(t))
      const R t = a.time[1];
      const V3<R> bb = b_boundary<R>(a.tc, a.m, ix, iy, iz, t);
      const V3<R> df = {Bm.x - bb.x, Bm.y - bb.y, Bm.z - bb.z};
      for (int ax = 0; ax < 3; ++ax) {
        const bool l = ii[ax] == 0, r = ii[ax] == nn[ax] - 1;
        const R ua = ax == 0 ? um.x : (ax == 1 ? um.y : um.z);
        const R c = (l && ua > (R)0 ? (R)-1 : (R)0) + (r && ua < (R)0 ? (R)1 : (R)0);
        if (c == (R)0) continue;
        const R f = (a.sat_s[ax] * c) * ua;
        db.x += f * df.x; db.y += f * df.y; db.z += f * df.z;
      }
    }
  }
}

// the stage update of the integrator (EpilogueMode) at one node, split into the loads of
// the fields it combines (which do not depend on DB, so a kernel may issue them early) and
// the arithmetic and stores
template <typename R>
struct EpIn {
  V3<R> X, Y;   // X; Y (EP_PX_QYHF) or Z (the fused 2N modes)
};

template <typename R, typename F>
__device__ __forceinline__ EpIn<R> epilogue_load(const StageArgs<R, F> &a, long long idx) {
  EpIn<R> e = {{0, 0, 0}, {0, 0, 0}};
  switch (a.mode) {
    case EP_X_PLUS_HF:
    case EP_AX_HF:
    case EP_2R_FUSED:
      e.X = ldf_plain(a.X, idx);
      break;
    case EP_PX_QYHF:
      e.X = ldf_plain(a.X, idx);
      e.Y = ldf_plain(a.Y, idx);
      break;
    case EP_2N_FUSED:
      e.X = ldf_plain(a.X, idx);
      e.Y = ldf_plain(a.Z, idx);
      break;
    case EP_2N_FUSED_FIRST:
      e.Y = ldf_plain(a.Z, idx);
      break;
    default:
      break;
  }
  return e;
}

// the values a mode stores: o1 into out, o2 into out2 (fused 2N / 2R modes), o3 into out3
// (EP_2R_FUSED, if set)
template <typename R>
struct EpOut {
  V3<R> o1, o2, o3;
};
__host__ __device__ constexpr bool epilogue_writes_out2(int mode) {
  return mode == EP_2N_FUSED || mode == EP_2N_FUSED_FIRST || mode == EP_2R_FUSED;
}

template <typename R, typename F>
__device__ __forceinline__ EpOut<R> epilogue_values(const StageArgs<R, F> &a, const V3<R> &db, const EpIn<R> &e) {
  const V3<R> &X = e.X, &Y = e.Y;
  EpOut<R> r = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  switch (a.mode) {
    case EP_X_PLUS_HF:
      r.o1 = V3<R>{X.x + a.h * db.x, X.y + a.h * db.y, X.z + a.h * db.z};
      break;
    case EP_PX_QYHF:
      r.o1 = V3<R>{a.p * X.x + a.q * (Y.x + a.h * db.x), a.p * X.y + a.q * (Y.y + a.h * db.y),
                   a.p * X.z + a.q * (Y.z + a.h * db.z)};
      break;
    case EP_HF:
      r.o1 = V3<R>{a.h * db.x, a.h * db.y, a.h * db.z};
      break;
    case EP_AX_HF:
      r.o1 = V3<R>{a.A * X.x + a.h * db.x, a.A * X.y + a.h * db.y, a.A * X.z + a.h * db.z};
      break;
    case EP_2N_FUSED:
    case EP_2N_FUSED_FIRST: {
      V3<R> t;
      if (a.mode == EP_2N_FUSED) t = {a.A * X.x + a.h * db.x, a.A * X.y + a.h * db.y, a.A * X.z + a.h * db.z};
      else t = {a.h * db.x, a.h * db.y, a.h * db.z};
      r.o1 = t;
      r.o2 = V3<R>{Y.x + a.Bc * t.x, Y.y + a.Bc * t.y, Y.z + a.Bc * t.z};
      break;
    }
    case EP_2R_FUSED: {
      const V3<R> t = {a.h * db.x, a.h * db.y, a.h * db.z};
      const V3<R> o = {X.x + a.A * t.x, X.y + a.A * t.y, X.z + a.A * t.z};
      r.o1 = o;
      r.o2 = V3<R>{o.x + a.Bc * t.x, o.y + a.Bc * t.y, o.z + a.Bc * t.z};
      r.o3 = t;
      break;
    }
  }
  return r;
}

template <typename R, typename F>
__device__ __forceinline__ void epilogue_store(const StageArgs<R, F> &a, long long idx, const V3<R> &db,
                                               const EpIn<R> &e) {
  const EpOut<R> r = epilogue_values(a, db, e);
  stf(a.out, idx, r.o1);
  if (epilogue_writes_out2(a.mode)) stf(a.out2, idx, r.o2);
  if (a.mode == EP_2R_FUSED && a.out3.p) stf(a.out3, idx, r.o3);
}

template <typename R, typename F>
__device__ __forceinline__ void stage_epilogue(const StageArgs<R, F> &a, long long idx, const V3<R> &db) {
  epilogue_store(a, idx, db, epilogue_load(a, idx));
}

// DB and the stage update at one node (ix, iy, iz) inside the grid.
template <typename R, typename F, int OP, bool PER, bool HALL, int DISS, int CONV>
__device__ __forceinline__ void stage_node(const StageArgs<R, F> &a, int ix, int iy, int iz) {
  constexpr int NB = Op<OP>::NB, SW = Op<OP>::SW, C0 = (SW - 1) / 2, WH = Op<OP>::WH;
  constexpr int RI = Op<OP>::RI;
  constexpr int RB = (C0 > WH - 1) ? C0 : WH - 1;
  constexpr bool HOD = DISS == DISS_HO;
  const int nx = a.m.nx, ny = a.m.ny, nz = a.m.nz;
  {
    const long long idx = ix + (long long)nx * (iy + (long long)ny * iz);
    const int ii[3] = {ix, iy, iz};
    const int nn[3] = {nx, ny, nz};
    const long long st[3] = {1, nx, (long long)nx * ny};
    const int conv = CONV >= 0 ? CONV : (a.conv_flag ? *a.conv_flag : a.conv);
    const V3<R> Bm = ldf(a.bk, idx);
    V3<R> um = {0, 0, 0};
    if (conv) um = ldf(a.u, idx);
    V3<R> db = {0, 0, 0};
    V3<R> hod = {0, 0, 0};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      AxisSums<R> s{};
      const int row = PER ? NB : sbp_row(ii[ax], nn[ax], NB);
      if (row == NB) {
        // periodic neighbours wrap only within RI of the ends of the axis
        const bool wrap = PER && (ii[ax] < RI || ii[ax] >= nn[ax] - RI);
#pragma unroll
        for (int o = -RI; o <= RI; ++o) {
          const R cD = a.Dint[o + RI];
          const R cH = a.Hint[o + RI];
          long long j = idx;
          if (o != 0) {
            if (wrap) j = idx + (long long)(nbr<true>(ii[ax], o, nn[ax]) - ii[ax]) * st[ax];
            else j = idx + (long long)o * st[ax];
            accumulate<R, F, HALL, HOD, false>(s, a, conv, ax, cD, cH, j);
          } else if (HOD) {
            // the interior derivative rows have a zero centre
            accumulate<R, F, false, HOD, false>(s, a, 0, ax, cD, cH, j);
          }
        }
      } else {
        for (int o = -RB; o <= RB; ++o) {
          const R cD = (o >= -C0 && o <= C0) ? a.tab->D[row][o + C0] : (R)0;
          const R cH = (HOD && o >= -(WH - 1) && o <= WH - 1) ? a.tab->H[row][o + WH - 1] : (R)0;
          if (cD == (R)0 && cH == (R)0) continue;
          const long long j = idx + (long long)(nbr<PER>(ii[ax], o, nn[ax]) - ii[ax]) * st[ax];
          accumulate<R, F, HALL, HOD, true>(s, a, conv, ax, cD, cH, j);
        }
      }
      if (conv) {
        const R Ba = ax == 0 ? Bm.x : (ax == 1 ? Bm.y : Bm.z);
        const R Ua = ax == 0 ? um.x : (ax == 1 ? um.y : um.z);
        const R SBa = ax == 0 ? s.SB.x : (ax == 1 ? s.SB.y : s.SB.z);
        const R SUa = ax == 0 ? s.SU.x : (ax == 1 ? s.SU.y : s.SU.z);
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
        db.x += a.inv_d[ax] * s.SH.x;
        db.y += a.inv_d[ax] * s.SH.y;
        db.z += a.inv_d[ax] * s.SH.z;
      }
      if (HOD) {
        hod.x += s.SHo.x; hod.y += s.SHo.y; hod.z += s.SHo.z;
      }
    }
    if (!PER) stage_sat<R, F, HALL>(a, ii, nn, idx, Bm, um, conv, db);
    if (HOD) {
      db.x += a.hod_factor * hod.x;
      db.y += a.hod_factor * hod.y;
      db.z += a.hod_factor * hod.z;
    }
    if (DISS == DISS_FO_OR_AD) {
      const V3<R> ds = fo_ad_dissipation<R, F, OP, PER>(a, ii, nn, st, idx, Bm, um);
      db.x += ds.x; db.y += ds.y; db.z += ds.z;
    }
    stage_epilogue<R, F>(a, idx, db);
  }
}

// time bookkeeping of the folded "a"/calc_time kernels, done by the last block to finish
// (every thread of the block must call this)
template <typename R, typename F>
__device__ __forceinline__ void stage_time_post(const StageArgs<R, F> &a) {
  if (a.tpost != TP_NONE) {
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
      __threadfence();
      const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
      const unsigned ticket = atomicAdd(a.counter, 1u);
      if (ticket == nblocks - 1) {
        if (a.tpost == TP_SET_STAGE) {
          a.time[1] = a.time[0] + a.tK;
        } else {
          const R t0 = a.time[0] + a.tDT;
          a.time[0] = t0;
          a.time[1] = t0;
        }
        __threadfence();
        *a.counter = 0u;
      }
    }
  }
}

template <typename R, typename F, int OP, bool PER, bool HALL, int DISS, int CONV = -1>
__global__ void __launch_bounds__(256) k_stage(const __grid_constant__ StageArgs<R, F> a) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z;
  if (ix < a.m.nx && iy < a.m.ny && iz < a.m.nz) stage_node<R, F, OP, PER, HALL, DISS, CONV>(a, ix, iy, iz);
  stage_time_post(a);
}

// curl(b)/rho (kernel_time_integrator.cl:136-208 via SBP_operator.cl:126-135), with the
// same interior/boundary row split; diff_* divide by (REAL)DX as the reference does.
template <typename R, typename F = AoS<R>>
struct CurlArgs {
  Mesh m;
  F b;
  const R *rho;       // nullptr: plain curl (kernel_operator.cl:158 calc_curl)
  F out;
  F jface;      // (k_curl_e) J on the faces of a non-periodic box
  F hout;       // (k_curl_e_hod) the dissipation sum of b (sum over the axes of the H rows)
  R Hint[7];    // (k_curl_e_hod) interior dissipation row, offsets -RI..RI
  const Tables<R> *tab;
  R dR[3];
  R inv_d[3];   // (REAL)(1.0/DX) ...
  R Dint[7];
};

template <typename R, typename F>
__device__ __forceinline__ R ldc(const F &f, long long j, int comp);
template <>
__device__ __forceinline__ double ldc<double, SoA<double>>(const SoA<double> &f, long long j, int comp) {
  return __ldg(f.p + j + comp * f.s);
}
template <>
__device__ __forceinline__ float ldc<float, SoA<float>>(const SoA<float> &f, long long j, int comp) {
  return __ldg(f.p + j + comp * f.s);
}
template <>
__device__ __forceinline__ double ldc<double, AoS<double>>(const AoS<double> &f, long long j, int comp) {
  return __ldg(reinterpret_cast<const double *>(f.p + j) + comp);
}
template <>
__device__ __forceinline__ float ldc<float, AoS<float>>(const AoS<float> &f, long long j, int comp) {
  return __ldg(reinterpret_cast<const float *>(f.p + j) + comp);
}

// curl(b)/rho.  Each axis contributes the derivatives of the two components orthogonal to
// it; the derivative rows are multiplied by (REAL)(1/DX) and the curl by 1/rho (within one
// rounding of the reference's divisions).
template <typename R, typename F, int OP, bool PER>
__global__ void __launch_bounds__(256) k_curl_rho(const __grid_constant__ CurlArgs<R, F> a) {
  constexpr int NB = Op<OP>::NB, SW = Op<OP>::SW, C0 = (SW - 1) / 2, RI = Op<OP>::RI;
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z;
  if (ix >= a.m.nx || iy >= a.m.ny || iz >= a.m.nz) return;
  const long long idx = ix + (long long)a.m.nx * (iy + (long long)a.m.ny * iz);
  const int ii[3] = {ix, iy, iz};
  const int nn[3] = {a.m.nx, a.m.ny, a.m.nz};
  const long long st[3] = {1, a.m.nx, (long long)a.m.nx * a.m.ny};
  R g[3][3];   // g[axis][component]
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    const int c1 = (ax + 1) % 3, c2 = (ax + 2) % 3;
    R v1 = 0, v2 = 0;
    const int row = PER ? NB : sbp_row(ii[ax], nn[ax], NB);
    if (row == NB) {
      const bool wrap = PER && (ii[ax] < RI || ii[ax] >= nn[ax] - RI);
#pragma unroll
      for (int o = -RI; o <= RI; ++o) {
        if (o == 0) continue;   // the interior row has a zero centre
        const R c = a.Dint[o + RI];
        long long j;
        if (wrap) j = idx + (long long)(nbr<true>(ii[ax], o, nn[ax]) - ii[ax]) * st[ax];
        else j = idx + (long long)o * st[ax];
        v1 += c * ldc<R, F>(a.b, j, c1);
        v2 += c * ldc<R, F>(a.b, j, c2);
      }
    } else {
      for (int o = -C0; o <= C0; ++o) {
        const R c = a.tab->D[row][o + C0];
        if (c == (R)0) continue;
        const long long j = idx + (long long)(nbr<PER>(ii[ax], o, nn[ax]) - ii[ax]) * st[ax];
        v1 += c * ldc<R, F>(a.b, j, c1);
        v2 += c * ldc<R, F>(a.b, j, c2);
      }
    }
    g[ax][c1] = v1 * a.inv_d[ax];
    g[ax][c2] = v2 * a.inv_d[ax];
  }
  V3<R> c = {g[1][2] - g[2][1], g[2][0] - g[0][2], g[0][1] - g[1][0]};
  if (a.rho) {
    const R r = (R)1 / a.rho[idx];
    c = {c.x * r, c.y * r, c.z * r};
  }
  stf(a.out, idx, c);
}

// explicit launchers, instantiated per (R, OP) in stage_<r>_o<op>.cu
// conv: -1 decides per launch from StageArgs (conv / conv_flag); 0/1 fixes it at compile time
template <typename R, typename F, int OP>
void launch_stage(const StageArgs<R, F> &a, bool per, bool hall, int diss, int conv, dim3 grid, dim3 block,
                  cudaStream_t s);
template <typename R, typename F, int OP>
void launch_curl(const CurlArgs<R, F> &a, bool per, dim3 grid, dim3 block, cudaStream_t s);

// layout conversion of a vector field between REAL4 AoS and SoA (fused path entry/exit)
template <typename R>
__global__ void k_aos_to_soa(long long n, const R4<R> *in, R *out, long long s) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const V3<R> v = ld3_plain(in + i);
  out[i] = v.x;
  out[i + s] = v.y;
  out[i + 2 * s] = v.z;
}
template <typename R>
__global__ void k_soa_to_aos(long long n, const R *in, long long s, R4<R> *out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  st3(out + i, V3<R>{in[i], in[i + s], in[i + 2 * s]});
}

}  // namespace ieq
