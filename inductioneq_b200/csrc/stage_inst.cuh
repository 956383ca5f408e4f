// stage_inst.cuh -- instantiates the stage and curl kernels for one (REAL, operator) pair in
// both field layouts.  Included by stage_<real>_o<op>.cu with IEQ_R and IEQ_OP defined, so
// the instantiations compile in parallel.
#include "stage_brick.cuh"
#include "stage_x2.cuh"
#include "stage_z.cuh"
#include "diag_curl.cuh"

namespace ieq {

template <typename F, int C>
static void launch_stage_layout(const StageArgs<IEQ_R, F> &a, bool per, bool hall, int diss, dim3 grid,
                                dim3 block, cudaStream_t s) {
#define IEQ_L(P, H, D) k_stage<IEQ_R, F, IEQ_OP, P, H, D, C><<<grid, block, 0, s>>>(a)
  if (per) {
    if (hall) {
      if (diss == DISS_NONE) IEQ_L(true, true, DISS_NONE);
      else if (diss == DISS_HO) IEQ_L(true, true, DISS_HO);
      else IEQ_L(true, true, DISS_FO_OR_AD);
    } else {
      if (diss == DISS_NONE) IEQ_L(true, false, DISS_NONE);
      else if (diss == DISS_HO) IEQ_L(true, false, DISS_HO);
      else IEQ_L(true, false, DISS_FO_OR_AD);
    }
  } else {
    if (hall) {
      if (diss == DISS_NONE) IEQ_L(false, true, DISS_NONE);
      else if (diss == DISS_HO) IEQ_L(false, true, DISS_HO);
      else IEQ_L(false, true, DISS_FO_OR_AD);
    } else {
      if (diss == DISS_NONE) IEQ_L(false, false, DISS_NONE);
      else if (diss == DISS_HO) IEQ_L(false, false, DISS_HO);
      else IEQ_L(false, false, DISS_FO_OR_AD);
    }
  }
#undef IEQ_L
}

// the per-kernel entry points (AoS) decide the convection switch at run time; the fused
// path (SoA) knows it before capturing its graph
template <>
void launch_stage<IEQ_R, AoS<IEQ_R>, IEQ_OP>(const StageArgs<IEQ_R, AoS<IEQ_R>> &a, bool per, bool hall, int diss,
                                             int conv, dim3 grid, dim3 block, cudaStream_t s) {
  (void)conv;
  launch_stage_layout<AoS<IEQ_R>, -1>(a, per, hall, diss, grid, block, s);
}
template <>
void launch_stage<IEQ_R, SoA<IEQ_R>, IEQ_OP>(const StageArgs<IEQ_R, SoA<IEQ_R>> &a, bool per, bool hall, int diss,
                                             int conv, dim3 grid, dim3 block, cudaStream_t s) {
  if (conv == 0) launch_stage_layout<SoA<IEQ_R>, 0>(a, per, hall, diss, grid, block, s);
  else launch_stage_layout<SoA<IEQ_R>, 1>(a, per, hall, diss, grid, block, s);
}

template <>
void launch_curl<IEQ_R, AoS<IEQ_R>, IEQ_OP>(const CurlArgs<IEQ_R, AoS<IEQ_R>> &a, bool per, dim3 grid, dim3 block,
                                            cudaStream_t s) {
  if (per) k_curl_rho<IEQ_R, AoS<IEQ_R>, IEQ_OP, true><<<grid, block, 0, s>>>(a);
  else k_curl_rho<IEQ_R, AoS<IEQ_R>, IEQ_OP, false><<<grid, block, 0, s>>>(a);
}
template <>
void launch_curl<IEQ_R, SoA<IEQ_R>, IEQ_OP>(const CurlArgs<IEQ_R, SoA<IEQ_R>> &a, bool per, dim3 grid, dim3 block,
                                            cudaStream_t s) {
  if (per) k_curl_rho<IEQ_R, SoA<IEQ_R>, IEQ_OP, true><<<grid, block, 0, s>>>(a);
  else k_curl_rho<IEQ_R, SoA<IEQ_R>, IEQ_OP, false><<<grid, block, 0, s>>>(a);
}

// the column kernels of the fused path (no first-order / adaptive dissipation)
template <bool P, bool H>
static void launch_col_ph(const StageArgs<IEQ_R, SoA<IEQ_R>> &a, bool hod, int conv, bool hodp, bool foad, dim3 g,
                          dim3 b, bool pdl, cudaStream_t s) {
  // (a flux-form mask compiled in for the default forms measured 3-10 % slower for orders
  // 4 and 6 on B200: the mask stays a run-time value)
  if (foad) {
    if (conv) launch_pdl(k_stage_col<IEQ_R, IEQ_OP, P, H, false, 1, -1, false, true>, g, b, s, pdl, a);
    else launch_pdl(k_stage_col<IEQ_R, IEQ_OP, P, H, false, 0, -1, false, true>, g, b, s, pdl, a);
  } else if (hod && hodp) {
    if (conv) launch_pdl(k_stage_col<IEQ_R, IEQ_OP, P, H, true, 1, -1, true>, g, b, s, pdl, a);
    else launch_pdl(k_stage_col<IEQ_R, IEQ_OP, P, H, true, 0, -1, true>, g, b, s, pdl, a);
  } else if (hod) {
    if (conv) launch_pdl(k_stage_col<IEQ_R, IEQ_OP, P, H, true, 1>, g, b, s, pdl, a);
    else launch_pdl(k_stage_col<IEQ_R, IEQ_OP, P, H, true, 0>, g, b, s, pdl, a);
  } else {
    if (conv) launch_pdl(k_stage_col<IEQ_R, IEQ_OP, P, H, false, 1>, g, b, s, pdl, a);
    else launch_pdl(k_stage_col<IEQ_R, IEQ_OP, P, H, false, 0>, g, b, s, pdl, a);
  }
}

// a box's stage as two launches: the pair kernel `kint` over the interior x range
// [xband, nx - xband) (no time bookkeeping) and the one-node kernel `kband` over the 2 *
// xband boundary columns of every row (with it)
template <typename KI, typename KB>
static void launch_banded(KI kint, KB kband, const StageArgs<IEQ_R, SoA<IEQ_R>> &a, ColShape sh, cudaStream_t s) {
  constexpr int XB = xband<IEQ_OP>();
  StageArgs<IEQ_R, SoA<IEQ_R>> ai = a;
  ai.tpost = TP_NONE;
  const int np = (a.m.nx - 2 * XB) / 2;
  const ColShape ps = pair_shape(sh, false, (long long)a.m.nx * a.m.ny * a.m.nz, 2 * np);
  launch_pdl(kint, col_grid(ps, np, a.m.ny, a.m.nz, 1), col_block(ps), s, sh.pdl, ai);
  const long long nb = 2ll * XB * a.m.ny * a.m.nz;
  launch_pdl(kband, dim3((unsigned)((nb + kColThreads - 1) / kColThreads)), dim3(kColThreads), s, sh.pdl, a);
}
// whether a box's stage splits off its x boundary columns: even rows in which the band is at
// most a tenth of the row, and for a band of two columns a side (2nd order) rows of at least
// 96 (measured on B200: rotation 2nd order 96^3 +10 %, 6th order 128^3 +23 %, confined Hall
// 4th order 128^3 +12 % FP64 / +20 % FP32; 4th order 64^3, a band of 8 of 64 columns, 14 %
// slower; rotation, SSPRK33, 40 steps: 2nd order banded 5-43 % slower at 40^3 .. 80^3 and 12 %
// faster at 96^3 -- its one boundary row a side costs the pair kernel little, the band's
// launch more -- 4th order banded faster from 80^3 (+8 %), 6th order from 120^3 (+29 %))
inline int band_min_nx(int xb) { return xb <= 2 ? 96 : 20 * xb; }
static bool banded(const StageArgs<IEQ_R, SoA<IEQ_R>> &a, bool per, ColShape sh) {
  if (per || sh.band == 0 || a.m.nx % 2 != 0 || a.m.nx < 2 * xband<IEQ_OP>() + 2) return false;
  return sh.band == 2 || a.m.nx >= band_min_nx(xband<IEQ_OP>());
}

// the Hall stage kernel without convection, K x-adjacent nodes per thread
template <int K>
static void launch_stage_hall_k(const StageArgs<IEQ_R, SoA<IEQ_R>> &a, bool per, bool hodp, ColShape sh,
                                cudaStream_t s) {
  if constexpr (K == 4 && sizeof(IEQ_R) != 4) {
    return;   // (quads are FP32 only; the caller never asks for them in FP64)
  } else {
    const ColShape ps = pair_shape(sh, false, (long long)a.m.nx * a.m.ny * a.m.nz, a.m.nx, K);
    const dim3 g = col_grid(ps, a.m.nx / K, a.m.ny, a.m.nz, 1), b = col_block(ps);
    if (per) {
      if (hodp) launch_pdl(k_stage_hall_x2<IEQ_R, IEQ_OP, true, true, K>, g, b, s, sh.pdl, a);
      else launch_pdl(k_stage_hall_x2<IEQ_R, IEQ_OP, true, false, K>, g, b, s, sh.pdl, a);
    } else {
      if (hodp) launch_pdl(k_stage_hall_x2<IEQ_R, IEQ_OP, false, true, K>, g, b, s, sh.pdl, a);
      else launch_pdl(k_stage_hall_x2<IEQ_R, IEQ_OP, false, false, K>, g, b, s, sh.pdl, a);
    }
  }
}

// the same with two x-adjacent nodes per thread (k_stage_col_x2)
template <bool P, bool H>
static void launch_col_x2_ph(const StageArgs<IEQ_R, SoA<IEQ_R>> &a, bool hod, int conv, bool hodp, dim3 g, dim3 b,
                             bool pdl, cudaStream_t s) {
  if (hod && hodp) {
    if (conv) launch_pdl(k_stage_col_x2<IEQ_R, IEQ_OP, P, H, true, 1, true>, g, b, s, pdl, a);
    else launch_pdl(k_stage_col_x2<IEQ_R, IEQ_OP, P, H, true, 0, true>, g, b, s, pdl, a);
  } else if (hod) {
    if (conv) launch_pdl(k_stage_col_x2<IEQ_R, IEQ_OP, P, H, true, 1>, g, b, s, pdl, a);
    else launch_pdl(k_stage_col_x2<IEQ_R, IEQ_OP, P, H, true, 0>, g, b, s, pdl, a);
  } else {
    if (conv) launch_pdl(k_stage_col_x2<IEQ_R, IEQ_OP, P, H, false, 1>, g, b, s, pdl, a);
    else launch_pdl(k_stage_col_x2<IEQ_R, IEQ_OP, P, H, false, 0>, g, b, s, pdl, a);
  }
}

// the Hall + convection pair kernels with the flux-form mask N (high-order dissipation, if
// any, precomputed by the curl kernel: HODP)
template <int N>
static void launch_hall_conv_pairs(const StageArgs<IEQ_R, SoA<IEQ_R>> &a, bool per, bool hodp, ColShape sh,
                                   cudaStream_t s) {
  if (banded(a, per, sh)) {
    if (hodp)
      launch_banded(k_stage_col_x2<IEQ_R, IEQ_OP, false, true, true, 1, true, false, N, true>,
                    k_stage_xband<IEQ_R, IEQ_OP, true, true, 1, N, true, false>, a, sh, s);
    else
      launch_banded(k_stage_col_x2<IEQ_R, IEQ_OP, false, true, false, 1, false, false, N, true>,
                    k_stage_xband<IEQ_R, IEQ_OP, true, false, 1, N, false, false>, a, sh, s);
    return;
  }
  const ColShape ps = pair_shape(sh, false, (long long)a.m.nx * a.m.ny * a.m.nz, a.m.nx);
  const dim3 g2 = col_grid(ps, a.m.nx / 2, a.m.ny, a.m.nz, 1), b2 = col_block(ps);
  if (per) {
    if (hodp) launch_pdl(k_stage_col_x2<IEQ_R, IEQ_OP, true, true, true, 1, true, false, N>, g2, b2, s, sh.pdl, a);
    else launch_pdl(k_stage_col_x2<IEQ_R, IEQ_OP, true, true, false, 1, false, false, N>, g2, b2, s, sh.pdl, a);
  } else {
    if (hodp) launch_pdl(k_stage_col_x2<IEQ_R, IEQ_OP, false, true, true, 1, true, false, N>, g2, b2, s, sh.pdl, a);
    else launch_pdl(k_stage_col_x2<IEQ_R, IEQ_OP, false, true, false, 1, false, false, N>, g2, b2, s, sh.pdl, a);
  }
}

// the convection pair kernels (no Hall term, no dissipation) with the flux-form mask N
template <int N>
static void launch_conv_pairs(const StageArgs<IEQ_R, SoA<IEQ_R>> &a, bool per, ColShape sh, cudaStream_t s) {
  if (banded(a, per, sh)) {
    launch_banded(k_stage_col_x2<IEQ_R, IEQ_OP, false, false, false, 1, false, false, N, true>,
                  k_stage_xband<IEQ_R, IEQ_OP, false, false, 1, N, false, false>, a, sh, s);
    return;
  }
  const ColShape ps = pair_shape(sh, false, (long long)a.m.nx * a.m.ny * a.m.nz, a.m.nx);
  const dim3 g2 = col_grid(ps, a.m.nx / 2, a.m.ny, a.m.nz, 1), b2 = col_block(ps);
  if (per) launch_pdl(k_stage_col_x2<IEQ_R, IEQ_OP, true, false, false, 1, false, false, N>, g2, b2, s, sh.pdl, a);
  else launch_pdl(k_stage_col_x2<IEQ_R, IEQ_OP, false, false, false, 1, false, false, N>, g2, b2, s, sh.pdl, a);
}

// the pair kernels with first-order dissipation summed in their gathers (FOF)
template <bool H>
static void launch_fo_pairs(const StageArgs<IEQ_R, SoA<IEQ_R>> &a, bool per, ColShape sh, cudaStream_t s) {
  if (banded(a, per, sh)) {
    launch_banded(k_stage_col_x2<IEQ_R, IEQ_OP, false, H, false, 1, false, false, 10, true, true>,
                  k_stage_xband<IEQ_R, IEQ_OP, H, false, 1, 10, false, false, true>, a, sh, s);
    return;
  }
  const ColShape ps = pair_shape(sh, false, (long long)a.m.nx * a.m.ny * a.m.nz, a.m.nx);
  const dim3 g2 = col_grid(ps, a.m.nx / 2, a.m.ny, a.m.nz, 1), b2 = col_block(ps);
  if (per) launch_pdl(k_stage_col_x2<IEQ_R, IEQ_OP, true, H, false, 1, false, false, 10, false, true>, g2, b2, s, sh.pdl, a);
  else launch_pdl(k_stage_col_x2<IEQ_R, IEQ_OP, false, H, false, 1, false, false, 10, false, true>, g2, b2, s, sh.pdl, a);
}

template <>
void launch_stage_col<IEQ_R, IEQ_OP>(const StageArgs<IEQ_R, SoA<IEQ_R>> &a, bool per, bool hall, bool hod, int conv,
                                     bool hodp, bool foad, ColShape sh, cudaStream_t s) {
  const ColShape s1 = fit_rows(sh, a.m.nx);
  const dim3 g = col_grid(s1, a.m.nx, a.m.ny, a.m.nz, col_nodes(conv)), b = col_block(s1);
  // the precomputed dissipation sum comes with the Hall curl kernel only
  hodp = hodp && hall && hod && !foad;
  if (sh.pairs && hall && !conv && !foad && (hodp || !hod) && a.m.nx % 2 == 0 && pair_ok(a.E) &&
      pair_ok(a.Hpre) && pair_ok(a.X) && pair_ok(a.Y) && pair_ok(a.Z) && pair_ok(a.out) && pair_ok(a.out2) &&
      pair_ok(a.out3)) {
    // FP32: four nodes per thread (float4) where the fields allow it
    if (sizeof(IEQ_R) == 4 && (sh.quads || quads_fill((long long)a.m.nx * a.m.ny * a.m.nz)) && a.m.nx % 4 == 0 &&
        group_ok<4>(a.E) && group_ok<4>(a.Hpre) && group_ok<4>(a.X) &&
        group_ok<4>(a.Y) && group_ok<4>(a.Z) && group_ok<4>(a.out) && group_ok<4>(a.out2) && group_ok<4>(a.out3)) {
      launch_stage_hall_k<4>(a, per, hodp, sh, s);
      return;
    }
    if (banded(a, per, sh)) {
      if (hodp)
        launch_banded(k_stage_hall_x2<IEQ_R, IEQ_OP, false, true, 2, true>,
                      k_stage_xband<IEQ_R, IEQ_OP, true, true, 0, -1, true, false>, a, sh, s);
      else
        launch_banded(k_stage_hall_x2<IEQ_R, IEQ_OP, false, false, 2, true>,
                      k_stage_xband<IEQ_R, IEQ_OP, true, false, 0, -1, false, false>, a, sh, s);
      return;
    }
    launch_stage_hall_k<2>(a, per, hodp, sh, s);
    return;
  }
  // convection (with or without the Hall term) + first-order dissipation with the default
  // flux forms: two nodes per thread, the first-order terms summed in the gathers of the
  // volume terms (FOF), which load the same B and u -- the one-node kernel gathers them a
  // second time (measured on B200, CK2N54, 64^3, Hall: periodic with variable u 4th / 6th order
  // 2.21e10 / 1.83e10 DOF/s against 1.12e10 / 8.2e9, confined box 1.80e10 / 1.30e10 against
  // 1.17e10 / 7.4e9)
  if (sh.pairs && conv && foad && a.diss_form == 2 && a.need == 10 && a.m.nx % 2 == 0 && pair_ok(a.bk) &&
      pair_ok(a.u) && pair_ok(a.E) && pair_ok(a.X) && pair_ok(a.Y) && pair_ok(a.Z) && pair_ok(a.out) &&
      pair_ok(a.out2) && pair_ok(a.out3)) {
    if (hall) launch_fo_pairs<true>(a, per, sh, s);
    else launch_fo_pairs<false>(a, per, sh, s);
    return;
  }
  // Hall + convection with the flux-form mask compiled in (the default forms' two
  // convection sums per axis, mask 10, and every other mask of the split forms): two nodes
  // per thread on every grid -- with the default mask measured 24-27 % faster on periodic
  // grids than the run-time-masked pair kernel below and 6 % faster than one node per thread
  // on boxes (confined Hall 128^3)
  if (sh.pairs && hall && conv && !foad && (hodp || !hod) &&
      (a.need == 10 || a.need == 9 || a.need == 6 || a.need == 7 || a.need == 13 || a.need == 14 ||
       a.need == 15) &&
      a.m.nx % 2 == 0 && pair_ok(a.bk) && pair_ok(a.u) && pair_ok(a.E) && pair_ok(a.Hpre) && pair_ok(a.X) &&
      pair_ok(a.Y) && pair_ok(a.Z) && pair_ok(a.out) && pair_ok(a.out2) && pair_ok(a.out3)) {
    switch (a.need) {
      case 9: launch_hall_conv_pairs<9>(a, per, hodp, sh, s); break;
      case 6: launch_hall_conv_pairs<6>(a, per, hodp, sh, s); break;
      case 7: launch_hall_conv_pairs<7>(a, per, hodp, sh, s); break;
      case 13: launch_hall_conv_pairs<13>(a, per, hodp, sh, s); break;
      case 14: launch_hall_conv_pairs<14>(a, per, hodp, sh, s); break;
      case 15: launch_hall_conv_pairs<15>(a, per, hodp, sh, s); break;
      default: launch_hall_conv_pairs<10>(a, per, hodp, sh, s); break;
    }
    return;
  }
  // the general pair kernel: periodic Hall runs with convection and other flux forms
  // (measured 25-35 % faster there than one node per thread, whose Hall + convection build
  // spills at 64 registers; first-order / adaptive dissipation keeps one node per thread:
  // 64^3 whistler 1.68e10 against 1.53e10 DOF/s).  On boxes and without the Hall term the
  // one-node kernels measured faster (the x boundary rows run per node, and the
  // convection sums of two nodes exceed the registers).
  if (sh.pairs && per && hall && !foad && a.m.nx % 2 == 0 && pair_ok(a.bk) && pair_ok(a.u) && pair_ok(a.E) &&
      pair_ok(a.Hpre) && pair_ok(a.X) && pair_ok(a.Y) && pair_ok(a.Z) && pair_ok(a.out) && pair_ok(a.out2) &&
      pair_ok(a.out3)) {
    const ColShape ps = pair_shape(sh, false, (long long)a.m.nx * a.m.ny * a.m.nz, a.m.nx);
    launch_col_x2_ph<true, true>(a, hod, conv, hodp, col_grid(ps, a.m.nx / 2, a.m.ny, a.m.nz, 1), col_block(ps), sh.pdl,
                                 s);
    return;
  }
  // convection without the Hall term, with the reference's default flux forms (product
  // u_i B_j, central source and u_j B_i: the sums D[u] and D[u_a B_i] only, fixed at compile
  // time, which keeps two nodes' sums in 128 registers): measured 2-10 % faster than one node
  // per thread (rotation, orders 2/4/6, 64^3 .. 128^3).  Every other mask of the split forms
  // takes the same kernel with its own mask compiled in (two sums per axis: central u_i B_j
  // and u_j B_i with zero source, mask 9; product u_i B_j and u_j B_i with central source,
  // mask 6; three or four sums, masks 7, 13, 14, 15, at 3 blocks of <= 168 registers): measured
  // 1.06-1.43x faster than one node per thread at 80^3 and 160^3 (rotation 3D, orders 2/4/6)
  if (sh.pairs && !hall && conv && !hod && !foad &&
      (a.need == 10 || a.need == 9 || a.need == 6 || a.need == 7 || a.need == 13 || a.need == 14 ||
       a.need == 15) &&
      a.m.nx % 2 == 0 && pair_ok(a.bk) && pair_ok(a.u) && pair_ok(a.X) && pair_ok(a.Y) && pair_ok(a.Z) &&
      pair_ok(a.out) && pair_ok(a.out2) && pair_ok(a.out3)) {
    switch (a.need) {
      case 9: launch_conv_pairs<9>(a, per, sh, s); break;
      case 6: launch_conv_pairs<6>(a, per, sh, s); break;
      case 7: launch_conv_pairs<7>(a, per, sh, s); break;
      case 13: launch_conv_pairs<13>(a, per, sh, s); break;
      case 14: launch_conv_pairs<14>(a, per, sh, s); break;
      case 15: launch_conv_pairs<15>(a, per, sh, s); break;
      default: launch_conv_pairs<10>(a, per, sh, s); break;
    }
    return;
  }
  if (per) {
    if (hall) launch_col_ph<true, true>(a, hod, conv, hodp, foad, g, b, sh.pdl, s);
    else launch_col_ph<true, false>(a, hod, conv, false, foad, g, b, sh.pdl, s);
  } else {
    if (hall) launch_col_ph<false, true>(a, hod, conv, hodp, foad, g, b, sh.pdl, s);
    else launch_col_ph<false, false>(a, hod, conv, false, foad, g, b, sh.pdl, s);
  }
}

template <>
void launch_curl_e<IEQ_R, IEQ_OP>(const CurlArgs<IEQ_R, SoA<IEQ_R>> &a, bool per, bool hod, ColShape sh,
                                  cudaStream_t s) {
  const ColShape s1 = fit_rows(sh, a.m.nx);
  const dim3 b = col_block(s1);
  // pairs on periodic grids only (on boxes the x boundary rows run per node and the
  // one-node kernels measured faster)
  if (sh.pairs && per && a.m.nx % 2 == 0 && pair_ok(a.b) && pair_ok(a.out) && pair_ok(a.hout) &&
      (a.rho == nullptr || reinterpret_cast<uintptr_t>(a.rho) % (2 * sizeof(IEQ_R)) == 0)) {
    if constexpr (sizeof(IEQ_R) == 4) {
      // FP32: four nodes per thread (float4) where the fields allow it
      if ((sh.quads || quads_fill((long long)a.m.nx * a.m.ny * a.m.nz)) && a.m.nx % 4 == 0 && group_ok<4>(a.b) &&
          group_ok<4>(a.out) && group_ok<4>(a.hout) &&
          (a.rho == nullptr || reinterpret_cast<uintptr_t>(a.rho) % 16 == 0)) {
        const ColShape ps = pair_shape(sh, true, (long long)a.m.nx * a.m.ny * a.m.nz, a.m.nx, 4);
        const dim3 g4 = col_grid(ps, a.m.nx / 4, a.m.ny, a.m.nz, 1), b4 = col_block(ps);
        if (hod) launch_pdl(k_curl_e_x2<IEQ_R, IEQ_OP, true, true, 4>, g4, b4, s, sh.pdl, a);
        else launch_pdl(k_curl_e_x2<IEQ_R, IEQ_OP, true, false, 4>, g4, b4, s, sh.pdl, a);
        return;
      }
    }
    const ColShape ps = pair_shape(sh, true, (long long)a.m.nx * a.m.ny * a.m.nz, a.m.nx);
    const dim3 g2 = col_grid(ps, a.m.nx / 2, a.m.ny, a.m.nz, 1), b2 = col_block(ps);
    if (hod) launch_pdl(k_curl_e_x2<IEQ_R, IEQ_OP, true, true>, g2, b2, s, sh.pdl, a);
    else launch_pdl(k_curl_e_x2<IEQ_R, IEQ_OP, true, false>, g2, b2, s, sh.pdl, a);
    return;
  }
  // FP32 boxes: the pair kernel over the interior x range and the x boundary columns apart
  // (the rule of the stage kernels; confined Hall 128^3: 23.7 against 27.0 us).  In FP64 the
  // one-node kernels stay faster on boxes (128^3: 37.5 / 69 us against 39.2 / 86 us without
  // / with the dissipation sum), the pair kernel's y and z boundary rows then running at 4
  // blocks per SM.
  if (sizeof(IEQ_R) == 4 && !per && sh.pairs && sh.band != 0 && a.m.nx % 2 == 0 && a.m.nx >= 2 * xband<IEQ_OP>() + 2 &&
      (sh.band == 2 || a.m.nx >= 20 * xband<IEQ_OP>()) && pair_ok(a.b) && pair_ok(a.out) && pair_ok(a.hout) &&
      (a.rho == nullptr || reinterpret_cast<uintptr_t>(a.rho) % (2 * sizeof(IEQ_R)) == 0)) {
    constexpr int XB = xband<IEQ_OP>();
    const int np = (a.m.nx - 2 * XB) / 2;
    const ColShape ps = pair_shape(sh, true, (long long)a.m.nx * a.m.ny * a.m.nz, 2 * np);
    const dim3 gi = col_grid(ps, np, a.m.ny, a.m.nz, 1), bi = col_block(ps);
    const long long nb = 2ll * XB * a.m.ny * a.m.nz;
    const dim3 gb((unsigned)((nb + kColThreads - 1) / kColThreads)), bb(kColThreads);
    if (hod) {
      launch_pdl(k_curl_e_x2<IEQ_R, IEQ_OP, false, true, 2, true>, gi, bi, s, sh.pdl, a);
      launch_pdl(k_curl_xband<IEQ_R, IEQ_OP, true>, gb, bb, s, sh.pdl, a);
    } else {
      launch_pdl(k_curl_e_x2<IEQ_R, IEQ_OP, false, false, 2, true>, gi, bi, s, sh.pdl, a);
      launch_pdl(k_curl_xband<IEQ_R, IEQ_OP, false>, gb, bb, s, sh.pdl, a);
    }
    return;
  }
  if (hod) {
    const dim3 g = col_grid(s1, a.m.nx, a.m.ny, a.m.nz, 1);
    if (per) launch_pdl(k_curl_e_hod<IEQ_R, IEQ_OP, true>, g, b, s, sh.pdl, a);
    else launch_pdl(k_curl_e_hod<IEQ_R, IEQ_OP, false>, g, b, s, sh.pdl, a);
    return;
  }
  const dim3 g = col_grid(s1, a.m.nx, a.m.ny, a.m.nz, kCurlNodes);
  if (per) launch_pdl(k_curl_e<IEQ_R, IEQ_OP, true>, g, b, s, sh.pdl, a);
  else launch_pdl(k_curl_e<IEQ_R, IEQ_OP, false>, g, b, s, sh.pdl, a);
}

// the TMA brick kernels (u = 0 stages); the dynamic shared memory limit of each
// instantiation is raised once, before its first launch
template <bool P, bool H, bool D>
static void launch_brick_phd(const StageArgs<IEQ_R, SoA<IEQ_R>> &a, const TmaStageMaps &maps, int *err,
                             cudaStream_t s) {
  constexpr int smem = brick_smem_bytes<IEQ_R>((H ? 1 : 0) + (D ? 1 : 0));
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_stage_brick<IEQ_R, IEQ_OP, P, H, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    attr = true;
  }
  k_stage_brick<IEQ_R, IEQ_OP, P, H, D>
      <<<brick_grid(a.m.nx, a.m.ny, a.m.nz), kBrickThreads, smem, s>>>(a, maps, err);
}

template <>
void launch_stage_brick<IEQ_R, IEQ_OP>(const StageArgs<IEQ_R, SoA<IEQ_R>> &a, const TmaStageMaps &maps, int *err,
                                       bool per, bool hall, bool hod, cudaStream_t s) {
  if (per) {
    if (hall) {
      if (hod) launch_brick_phd<true, true, true>(a, maps, err, s);
      else launch_brick_phd<true, true, false>(a, maps, err, s);
    } else if (hod) {
      launch_brick_phd<true, false, true>(a, maps, err, s);
    }
  } else {
    if (hall) {
      if (hod) launch_brick_phd<false, true, true>(a, maps, err, s);
      else launch_brick_phd<false, true, false>(a, maps, err, s);
    } else if (hod) {
      launch_brick_phd<false, false, true>(a, maps, err, s);
    }
  }
}

template <bool P>
static void launch_curl_brick_p(const CurlArgs<IEQ_R, SoA<IEQ_R>> &a, const TmaStageMaps &maps, int *err,
                                cudaStream_t s) {
  constexpr int smem = brick_smem_bytes<IEQ_R>(1);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_curl_brick<IEQ_R, IEQ_OP, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    attr = true;
  }
  k_curl_brick<IEQ_R, IEQ_OP, P><<<brick_grid(a.m.nx, a.m.ny, a.m.nz), kBrickThreads, smem, s>>>(a, maps, err);
}

template <>
void launch_curl_brick<IEQ_R, IEQ_OP>(const CurlArgs<IEQ_R, SoA<IEQ_R>> &a, const TmaStageMaps &maps, int *err,
                                      bool per, cudaStream_t s) {
  if (per) launch_curl_brick_p<true>(a, maps, err, s);
  else launch_curl_brick_p<false>(a, maps, err, s);
}

// the one-pass Hall stage (stage_z.cuh): dynamic shared memory above 48 KB is opted into
// once per instantiation; resident CTAs per SM from the occupancy calculator
template <bool HOD>
static void launch_zmarch_h(const StageArgs<IEQ_R, SoA<IEQ_R>> &a, const IEQ_R *rho, bool pdl, int tz_set,
                            cudaStream_t s) {
  constexpr int RI = Op<IEQ_OP>::RI;
  constexpr size_t smem = ZLayout<IEQ_R, RI>::BYTES;
  auto kern = k_stage_hall_z<IEQ_R, IEQ_OP, HOD>;
  static int resident = 0;
  if (resident == 0) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0, nsm = 0, dev = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kZThreads, smem);
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    resident = per_sm * nsm > 0 ? per_sm * nsm : 1;
  }
  const int tz = tz_set > 0 ? (tz_set < a.m.nz ? tz_set : a.m.nz) : zm_chunk(a.m.nx, a.m.ny, a.m.nz, RI, resident);
  const dim3 g((a.m.nx / kZTX) * (a.m.ny / kZTY), (a.m.nz + tz - 1) / tz, 1);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = g;
  cfg.blockDim = dim3(kZThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kern, a, rho, tz);
}

template <>
void launch_stage_zmarch<IEQ_R, IEQ_OP>(const StageArgs<IEQ_R, SoA<IEQ_R>> &a, const IEQ_R *rho, bool hod, bool pdl,
                                        int tz, cudaStream_t s) {
  if (hod) launch_zmarch_h<true>(a, rho, pdl, tz, s);
  else launch_zmarch_h<false>(a, rho, pdl, tz, s);
}

template <>
void launch_curl_e_diag<IEQ_R, IEQ_OP>(const CurlArgs<IEQ_R, SoA<IEQ_R>> &a, const DiagArgs<IEQ_R, SoA<IEQ_R>> &d,
                                       const DiagOut &o, bool per, bool hod, dim3 g, dim3 b, bool pdl,
                                       cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = g;
  cfg.blockDim = b;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  if (per) {
    if (hod) cudaLaunchKernelEx(&cfg, k_curl_e_diag<IEQ_R, IEQ_OP, true, true>, a, d, o);
    else cudaLaunchKernelEx(&cfg, k_curl_e_diag<IEQ_R, IEQ_OP, true, false>, a, d, o);
  } else {
    if (hod) cudaLaunchKernelEx(&cfg, k_curl_e_diag<IEQ_R, IEQ_OP, false, true>, a, d, o);
    else cudaLaunchKernelEx(&cfg, k_curl_e_diag<IEQ_R, IEQ_OP, false, false>, a, d, o);
  }
}

// one launch of k_curl_e_z<R, OP, H>; its ring is dynamic shared memory beside the static
// plane buffers, allowed once per device for each instantiation
template <typename R, int OP, bool H>
void launch_cz(const CurlArgs<R, SoA<R>> &a, dim3 g, int tz, bool pdl, cudaStream_t s) {
  constexpr int dyn = cz_ring_bytes<R>();
  static bool ring_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || !ring_set[dev]) {
    cudaFuncSetAttribute(k_curl_e_z<R, OP, H>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    if (dev >= 0 && dev < 64) ring_set[dev] = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = g;
  cfg.blockDim = dim3(kCzTX * kCzTY);
  cfg.dynamicSmemBytes = dyn;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k_curl_e_z<R, OP, H>, a, tz);
}

template <>
void launch_curl_e_z<IEQ_R, IEQ_OP>(const CurlArgs<IEQ_R, SoA<IEQ_R>> &a, bool hod, int tz, bool pdl, cudaStream_t s) {
  const dim3 g((a.m.nx + kCzTX - 1) / kCzTX, (a.m.ny + kCzTY - 1) / kCzTY, (a.m.nz + tz - 1) / tz);
  if (hod) launch_cz<IEQ_R, IEQ_OP, true>(a, g, tz, pdl, s);
  else launch_cz<IEQ_R, IEQ_OP, false>(a, g, tz, pdl, s);
}

}  // namespace ieq
