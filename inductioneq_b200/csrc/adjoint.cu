// adjoint.cu -- discrete adjoint of the semi-discretisation and of the SSPRK33 and 2N
// low-storage steps.
//
// F(b) is the time derivative DB of kernel/kernel_time_integrator.cl:9-31 (volume terms,
// Hall term with J = curl(b)/rho, artificial dissipation, inflow SAT) at fixed u and rho.
// The operators, all FP64:
//   jvp:  F'(b0) v    (tangent linear; used by the transpose tests)
//   vjp:  F'(b0)^T w  (the adjoint of the spatial operator)
//   step adjoints: lambda_n = (d b_{n+1} / d b_n)^T lambda_{n+1} from the stage states
//   (SSPRK33; CarpenterKennedy2N54 and ToulorgeDesmet2N84F from the input of every stage),
//   and the checkpointed sweep over many steps, whose forward passes run the fused stage
//   kernels of the time stepping with the stage states written out per stage
// The transposes are written out per term (see the notes at k_vjp_pass1); D^T is applied as
// a gather over the neighbours j = k + p with the coefficient of row(j) at offset -p.
// The Hall outflow SAT (a switch on the sign of 0.5u - J) is differentiated away from the
// switch (tv_a = 0); first-order dissipation is linear in b at fixed u; adaptive dissipation
// (weights that depend on b through a square root and thresholds) has no adjoint.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ieq_host.h"

#include "stage_kernel.cuh"

namespace ieq {

struct AdjArgs {
  Mesh m;
  const Tables<double> *tab;
  int nb, sw, wh, periodic;
  int conv, hall, hod, fo;   // fo: first-order dissipation (linear in b at fixed u)
  int ad;                    // adaptive dissipation (its weights depend on b: linearised at b0)
  double mp2min, mp2max, cmin, cmax, hsgn;   // the adaptive form's thresholds; (-1)^(p/2+1)
  double hod_factor;
  double w[6];           // flux-form weights (see stage_kernel.cuh)
  double inv_d[3], two_inv_d[3], sat_s[3];
  const R4<double> *b0, *J0, *u, *v, *dJ;   // v: tangent direction or adjoint input w
  const double *rho;
  R4<double> *out;
  R4<double> *gJr;       // vjp pass 1 -> pass 2: (Hall adjoint source for J) / rho
  // epilogue of the vjp's last kernel (dst != nullptr): dst = eal ex + ebe ey + ega z instead
  // of out = z (ex, ey may be null; dst may be ex or ey, never v)
  R4<double> *dst;
  const R4<double> *ex, *ey;
  double eal, ebe, ega;
};

__device__ __forceinline__ V3<double> ld(const R4<double> *p, long long j) { return ld3(p + j); }
__device__ __forceinline__ double comp(V3<double> v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }
__device__ __forceinline__ void addc(V3<double> &v, int c, double x) {
  if (c == 0) v.x += x;
  else if (c == 1) v.y += x;
  else v.z += x;
}
__device__ __forceinline__ V3<double> axpy3(double a, V3<double> x, V3<double> y) {
  return {a * x.x + y.x, a * x.y + y.y, a * x.z + y.z};
}
__device__ __forceinline__ double dot3(V3<double> a, V3<double> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

struct Node {
  int i[3], n[3];
  long long st[3], idx;
};

__device__ __forceinline__ int row_of(const AdjArgs &a, int i, int n) {
  return a.periodic ? a.nb : sbp_row(i, n, a.nb);
}

// neighbour j = node + o along axis; false if outside a non-periodic grid
__device__ __forceinline__ bool nbr_idx(const AdjArgs &a, const Node &nd, int ax, int o, long long &j, int &jj) {
  int t = nd.i[ax] + o;
  if (a.periodic) {
    t += (t < 0) ? nd.n[ax] : 0;
    t -= (t >= nd.n[ax]) ? nd.n[ax] : 0;
  } else if (t < 0 || t >= nd.n[ax]) {
    return false;
  }
  jj = t;
  j = nd.idx + (long long)(t - nd.i[ax]) * nd.st[ax];
  return true;
}

// forward derivative row at the node: sum_o D[row][o] f(node + o)
template <typename Fn>
__device__ V3<double> dfwd(const AdjArgs &a, const Node &nd, int ax, Fn f) {
  const int c0 = (a.sw - 1) / 2;
  const int r = row_of(a, nd.i[ax], nd.n[ax]);
  V3<double> s = {0, 0, 0};
  for (int o = -c0; o <= c0; ++o) {
    const double c = a.tab->D[r][o + c0];
    if (c == 0.0) continue;
    long long j;
    int jj;
    if (!nbr_idx(a, nd, ax, o, j, jj)) continue;
    s = axpy3(c, f(j), s);
  }
  return s;
}

// transposed derivative at the node: sum_j D[row(j)][node - j] f(j)
template <typename Fn>
__device__ V3<double> dtr(const AdjArgs &a, const Node &nd, int ax, Fn f) {
  const int c0 = (a.sw - 1) / 2;
  V3<double> s = {0, 0, 0};
  for (int p = -c0; p <= c0; ++p) {
    long long j;
    int jj;
    if (!nbr_idx(a, nd, ax, p, j, jj)) continue;
    const double c = a.tab->D[row_of(a, jj, nd.n[ax])][c0 - p];
    if (c == 0.0) continue;
    s = axpy3(c, f(j), s);
  }
  return s;
}

// dissipation row (symmetric use: forward with the row of the node, transpose with rows of j)
template <bool TR>
__device__ V3<double> hod_apply(const AdjArgs &a, const Node &nd, int ax, const R4<double> *x) {
  const int h0 = a.wh - 1;
  V3<double> s = {0, 0, 0};
  for (int p = -h0; p <= h0; ++p) {
    long long j;
    int jj;
    if (!nbr_idx(a, nd, ax, p, j, jj)) continue;
    const double c = TR ? a.tab->H[row_of(a, jj, nd.n[ax])][h0 - p] : a.tab->H[row_of(a, nd.i[ax], nd.n[ax])][h0 + p];
    if (c == 0.0) continue;
    s = axpy3(c, ld(x, j), s);
  }
  return s;
}

__device__ __forceinline__ bool make_node(const AdjArgs &a, Node &nd) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z;
  if (ix >= a.m.nx || iy >= a.m.ny || iz >= a.m.nz) return false;
  nd.i[0] = ix; nd.i[1] = iy; nd.i[2] = iz;
  nd.n[0] = a.m.nx; nd.n[1] = a.m.ny; nd.n[2] = a.m.nz;
  nd.st[0] = 1; nd.st[1] = a.m.nx; nd.st[2] = (long long)a.m.nx * a.m.ny;
  nd.idx = ix + (long long)a.m.nx * (iy + (long long)a.m.ny * iz);
  return true;
}

// first-order dissipation (artificial_dissipation.cl:36-80) along ax, linear in b at fixed u:
// forward  sum_o |D[row k][o]| sigma(u_{k+o}, u_k) (x_{k+o} - x_k)
// transpose sum_p |D[row (k+p)][-p]| sigma(u_k, u_{k+p}) x_{k+p} - (sum_o |D[row k][o]| sigma(u_{k+o}, u_k)) x_k
// (sigma: the componentwise larger |u|; the caller multiplies by 1/d)
__device__ __forceinline__ V3<double> sigma3(V3<double> p, V3<double> q) {
  return {fmax(fabs(p.x), fabs(q.x)), fmax(fabs(p.y), fabs(q.y)), fmax(fabs(p.z), fabs(q.z))};
}
template <bool TR>
__device__ V3<double> fo_apply(const AdjArgs &a, const Node &nd, int ax, const R4<double> *x) {
  const int c0 = (a.sw - 1) / 2;
  const int rk = row_of(a, nd.i[ax], nd.n[ax]);
  const V3<double> uk = ld(a.u, nd.idx), xk = ld(x, nd.idx);
  V3<double> s = {0, 0, 0}, diag = {0, 0, 0};
  for (int o = -c0; o <= c0; ++o) {
    long long j;
    int jj;
    if (!nbr_idx(a, nd, ax, o, j, jj)) continue;
    const V3<double> uj = ld(a.u, j);
    const double cf = fabs(a.tab->D[rk][o + c0]);
    if (!TR) {
      if (cf == 0.0) continue;
      const V3<double> sg = sigma3(uj, uk), xj = ld(x, j);
      s.x += cf * sg.x * (xj.x - xk.x);
      s.y += cf * sg.y * (xj.y - xk.y);
      s.z += cf * sg.z * (xj.z - xk.z);
    } else {
      const V3<double> sg = sigma3(uj, uk);
      if (cf != 0.0) diag = {diag.x + cf * sg.x, diag.y + cf * sg.y, diag.z + cf * sg.z};
      const double ct = fabs(a.tab->D[row_of(a, jj, nd.n[ax])][c0 - o]);
      if (ct == 0.0) continue;
      const V3<double> xj = ld(x, j);
      s.x += ct * sg.x * xj.x;
      s.y += ct * sg.y * xj.y;
      s.z += ct * sg.z * xj.z;
    }
  }
  if (TR) s = {s.x - diag.x * xk.x, s.y - diag.y * xk.y, s.z - diag.z * xk.z};
  return s;
}

// Adaptive dissipation (artificial_dissipation.cl:82-160 with kappa of
// include/artificial_dissipation.h:23-45), per component, along axis a with d = DX_a:
//   first-order part  sum_o |D[row k][o]| kappa_|o|(s) sigma (b_{k+o} - b_k) / d,
//   high-order part   sum_t hf (1 - kappa_1(s'_t)) sum_i c(row k, t, i) b_{k+t+i},
// sigma = max(|u_j|, |u_k|) of the pair, s = (sigma delta) delta with delta the pair's
// difference of b, and s'_t that of the pair (k+t+WH-1, k+t+WH-2).  kappa_m(s) is
// sqrt(|s - lo| / |hi - lo|) on (lo, hi), 0 below, 1 above (lo, hi = m^2 MP2MIN CMIN d,
// m^2 MP2MAX CMAX d); linearised at b0 its derivative is 1 / (2 |hi - lo| kappa) on (lo, hi)
// and 0 elsewhere (it has none at s = lo and s = hi).  So along a pair, d(kappa sigma delta) =
// sigma (kappa + 2 s kappa') d(delta), and d((1 - kappa_1(s')) H) = (1 - kappa_1) dH -
// kappa_1' 2 sigma' delta' d(delta') H.
struct KapLin {
  double k, dk;
};
__device__ __forceinline__ KapLin kap_lin(const AdjArgs &a, unsigned m, double d, double s) {
  m = m + (m == 0);
  const double kk = (double)(m * m);
  const double lo = ((kk * a.mp2min) * a.cmin) * d;
  const double hi = ((kk * a.mp2max) * a.cmax) * d;
  if (lo < s && s < hi) {
    const double den = fabs(hi - lo);
    const double k = sqrt(fabs(s - lo) / den);
    return {k, k > 0.0 ? 0.5 / (den * k) : 0.0};
  }
  return {s >= hi ? 1.0 : 0.0, 0.0};
}
// sigma (kappa + 2 s kappa') of the pair (p, q) per component: the first-order part's
// linearised weight (symmetric in the pair)
__device__ __forceinline__ V3<double> ad_pair_weight(const AdjArgs &a, unsigned m, double d, V3<double> bp,
                                                     V3<double> bq, V3<double> up, V3<double> uq) {
  const V3<double> sg = sigma3(up, uq);
  const double dl[3] = {bp.x - bq.x, bp.y - bq.y, bp.z - bq.z};
  const double sgc[3] = {sg.x, sg.y, sg.z};
  double w[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double sv = (sgc[c] * dl[c]) * dl[c];
    const KapLin K = kap_lin(a, m, d, sv);
    w[c] = sgc[c] * (K.k + 2.0 * sv * K.dk);
  }
  return {w[0], w[1], w[2]};
}

// the first-order part along ax (times 1/d by the caller): the tangent, or its transpose as
// fo_apply<true> with the pair weights
template <bool TR>
__device__ V3<double> ad_fo_apply(const AdjArgs &a, const Node &nd, int ax, const R4<double> *x) {
  const int c0 = (a.sw - 1) / 2;
  const int rk = row_of(a, nd.i[ax], nd.n[ax]);
  const double d = a.m.d[ax];
  const V3<double> uk = ld(a.u, nd.idx), bk = ld(a.b0, nd.idx), xk = ld(x, nd.idx);
  V3<double> s = {0, 0, 0}, diag = {0, 0, 0};
  for (int o = -c0; o <= c0; ++o) {
    long long j;
    int jj;
    if (!nbr_idx(a, nd, ax, o, j, jj)) continue;
    const double cf = fabs(a.tab->D[rk][o + c0]);
    const double ct = TR ? fabs(a.tab->D[row_of(a, jj, nd.n[ax])][c0 - o]) : 0.0;
    if (cf == 0.0 && ct == 0.0) continue;
    const V3<double> w = ad_pair_weight(a, (unsigned)(o < 0 ? -o : o), d, ld(a.b0, j), bk, ld(a.u, j), uk);
    const V3<double> xj = ld(x, j);
    if (!TR) {
      s.x += cf * w.x * (xj.x - xk.x);
      s.y += cf * w.y * (xj.y - xk.y);
      s.z += cf * w.z * (xj.z - xk.z);
    } else {
      diag = {diag.x + cf * w.x, diag.y + cf * w.y, diag.z + cf * w.z};
      s.x += ct * w.x * xj.x;
      s.y += ct * w.y * xj.y;
      s.z += ct * w.z * xj.z;
    }
  }
  if (TR) s = {s.x - diag.x * xk.x, s.y - diag.y * xk.y, s.z - diag.z * xk.z};
  return s;
}

// position of node + o along ax with the reference's neighbour rule: periodic wrap, or the
// node itself outside a box (include/utils.h:89-168)
__device__ __forceinline__ int ad_pos(const AdjArgs &a, int i, int o, int n) {
  int t = i + o;
  if (a.periodic) {
    t += (t < 0) ? n : 0;
    t -= (t >= n) ? n : 0;
  } else if (t < 0 || t >= n) {
    t = i;
  }
  return t;
}

// one high-order term t of node k (position ik along ax, grid index kidx): the pair weight
// kappa_1 and its derivative factor 2 kappa_1' sigma' delta' per component, the pair's
// positions, and the dissipation row applied to b0 (only where that factor is non-zero)
struct AdTerm {
  int p1, p2;
  V3<double> one_minus_k, dfac, h0;
};
__device__ AdTerm ad_term(const AdjArgs &a, const Node &nd, int ax, int ik, long long kidx, int rk, int t) {
  const int n = nd.n[ax];
  const long long st = nd.st[ax];
  AdTerm r;
  r.p1 = ad_pos(a, ik, t + a.wh - 1, n);
  r.p2 = ad_pos(a, ik, t + a.wh - 2, n);
  const long long j1 = kidx + (long long)(r.p1 - ik) * st, j2 = kidx + (long long)(r.p2 - ik) * st;
  const V3<double> b1 = ld(a.b0, j1), b2 = ld(a.b0, j2);
  const V3<double> sg = sigma3(ld(a.u, j1), ld(a.u, j2));
  const double dl[3] = {b1.x - b2.x, b1.y - b2.y, b1.z - b2.z}, sgc[3] = {sg.x, sg.y, sg.z};
  double om[3], df[3];
  bool any = false;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double sv = (sgc[c] * dl[c]) * dl[c];
    const KapLin K = kap_lin(a, 1, a.m.d[ax], sv);
    om[c] = 1.0 - K.k;
    df[c] = 2.0 * K.dk * sgc[c] * dl[c];
    any = any || df[c] != 0.0;
  }
  r.one_minus_k = {om[0], om[1], om[2]};
  r.dfac = {df[0], df[1], df[2]};
  r.h0 = {0, 0, 0};
  if (any) {
    for (int i = 0; i < a.wh; ++i) {
      const double cf = ((a.tab->Minv[rk] * a.tab->DHO[rk][t + a.wh - 1]) * a.tab->DHO[a.nb][i]) * a.hsgn;
      const int pi = ad_pos(a, ik, i + t, n);
      r.h0 = axpy3(cf, ld(a.b0, kidx + (long long)(pi - ik) * st), r.h0);
    }
  }
  return r;
}

// the high-order part along ax (times hod_factor by the caller): the tangent at the node, or
// its transpose gathered from every node k whose terms reach the node (k within WH-1 along ax)
template <bool TR>
__device__ V3<double> ad_ho_apply(const AdjArgs &a, const Node &nd, int ax, const R4<double> *x) {
  const int n = nd.n[ax], im = nd.i[ax];
  const long long st = nd.st[ax];
  V3<double> out = {0, 0, 0};
  if (!TR) {
    const int rk = row_of(a, im, n);
    for (int t = -a.wh + 1; t <= 0; ++t) {
      const AdTerm T = ad_term(a, nd, ax, im, nd.idx, rk, t);
      V3<double> hv = {0, 0, 0};
      for (int i = 0; i < a.wh; ++i) {
        const double cf = ((a.tab->Minv[rk] * a.tab->DHO[rk][t + a.wh - 1]) * a.tab->DHO[a.nb][i]) * a.hsgn;
        const int pi = ad_pos(a, im, i + t, n);
        hv = axpy3(cf, ld(x, nd.idx + (long long)(pi - im) * st), hv);
      }
      const V3<double> x1 = ld(x, nd.idx + (long long)(T.p1 - im) * st), x2 = ld(x, nd.idx + (long long)(T.p2 - im) * st);
      out.x += T.one_minus_k.x * hv.x - T.dfac.x * (x1.x - x2.x) * T.h0.x;
      out.y += T.one_minus_k.y * hv.y - T.dfac.y * (x1.y - x2.y) * T.h0.y;
      out.z += T.one_minus_k.z * hv.z - T.dfac.z * (x1.z - x2.z) * T.h0.z;
    }
    return out;
  }
  for (int off = -(a.wh - 1); off <= a.wh - 1; ++off) {
    // node k = m + off along ax (a box has no node beyond its faces)
    int ik = im + off;
    if (a.periodic) {
      ik += (ik < 0) ? n : 0;
      ik -= (ik >= n) ? n : 0;
    } else if (ik < 0 || ik >= n) {
      continue;
    }
    const long long kidx = nd.idx + (long long)(ik - im) * st;
    const int rk = row_of(a, ik, n);
    const V3<double> wk = ld(x, kidx);
    for (int t = -a.wh + 1; t <= 0; ++t) {
      const AdTerm T = ad_term(a, nd, ax, ik, kidx, rk, t);
      for (int i = 0; i < a.wh; ++i) {
        if (ad_pos(a, ik, i + t, n) != im) continue;
        const double cf = ((a.tab->Minv[rk] * a.tab->DHO[rk][t + a.wh - 1]) * a.tab->DHO[a.nb][i]) * a.hsgn;
        out.x += T.one_minus_k.x * cf * wk.x;
        out.y += T.one_minus_k.y * cf * wk.y;
        out.z += T.one_minus_k.z * cf * wk.z;
      }
      const double sgn = (T.p1 == im ? -1.0 : 0.0) + (T.p2 == im ? 1.0 : 0.0);
      if (sgn != 0.0) {
        out.x += sgn * T.dfac.x * T.h0.x * wk.x;
        out.y += sgn * T.dfac.y * T.h0.y * wk.y;
        out.z += sgn * T.dfac.z * T.h0.z * wk.z;
      }
    }
  }
  return out;
}

// The Hall outflow SAT at a boundary node (induction_Eq_surface.cl:35-81), per face axis a
// with c = M_INV[0]/d_a, tv = 0.5 u - J (J = curl(b)/rho), sw = -[left, tv_a > 0] + [right,
// tv_a < 0], side = -[left] + [right]:  S = c (sw tv_a b + side b_a J).  Away from tv_a = 0
// its tangent is  c (sw (tv_a v - dJ_a b) + side (v_a J + b_a dJ)),  dJ = curl(v)/rho.
struct HallSat {
  double c, tva, sw, side;
};
__device__ __forceinline__ bool hall_sat_axis(const AdjArgs &a, const Node &nd, int ax, V3<double> tv, HallSat &h) {
  const bool l = nd.i[ax] == 0, r = nd.i[ax] == nd.n[ax] - 1;
  if (!l && !r) return false;
  h.c = a.sat_s[ax];
  h.tva = comp(tv, ax);
  h.sw = (l && h.tva > 0 ? -1.0 : 0.0) + (r && h.tva < 0 ? 1.0 : 0.0);
  h.side = (l ? -1.0 : 0.0) + (r ? 1.0 : 0.0);
  return true;
}

// SAT of the inflow boundary (induction_Eq_surface.cl:7-33): linear in b with the diagonal
// coefficient sum_a s_a c_a u_a on the faces
__device__ double sat_diag(const AdjArgs &a, const Node &nd, V3<double> um) {
  if (a.periodic || a.hall || !a.conv) return 0.0;
  double d = 0.0;
  for (int ax = 0; ax < 3; ++ax) {
    const bool l = nd.i[ax] == 0, r = nd.i[ax] == nd.n[ax] - 1;
    const double ua = comp(um, ax);
    const double c = (l && ua > 0 ? -1.0 : 0.0) + (r && ua < 0 ? 1.0 : 0.0);
    d += (a.sat_s[ax] * c) * ua;
  }
  return d;
}

// tangent linear F'(b0) v; dJ = curl(v)/rho precomputed
template <bool AD>
__global__ void k_jvp(const AdjArgs a) {
  Node nd;
  if (!make_node(a, nd)) return;
  const long long k = nd.idx;
  const V3<double> vm = ld(a.v, k), um = a.conv ? ld(a.u, k) : V3<double>{0, 0, 0};
  V3<double> out = {0, 0, 0};
  for (int ax = 0; ax < 3; ++ax) {
    if (a.conv) {
      // the factored split forms with b -> v (linear in b at fixed u)
      const V3<double> DuiBa = dfwd(a, nd, ax, [&](long long j) {
        const V3<double> uu = ld(a.u, j);
        const double va = comp(ld(a.v, j), ax);
        return V3<double>{uu.x * va, uu.y * va, uu.z * va};
      });
      const V3<double> DU = dfwd(a, nd, ax, [&](long long j) { return ld(a.u, j); });
      const V3<double> DV = dfwd(a, nd, ax, [&](long long j) { return ld(a.v, j); });
      const V3<double> DuaB = dfwd(a, nd, ax, [&](long long j) {
        const V3<double> vv = ld(a.v, j);
        const double ua = comp(ld(a.u, j), ax);
        return V3<double>{ua * vv.x, ua * vv.y, ua * vv.z};
      });
      const double va = comp(vm, ax), ua = comp(um, ax), DVa = comp(DV, ax), DUa = comp(DU, ax);
      for (int i = 0; i < 3; ++i) {
        const double vol = a.w[0] * comp(DuiBa, i) + a.w[1] * va * comp(DU, i) + a.w[2] * comp(um, i) * DVa -
                           (a.w[3] * comp(DuaB, i) + a.w[4] * ua * comp(DV, i) + a.w[5] * comp(vm, i) * DUa);
        addc(out, i, a.two_inv_d[ax] * vol);
      }
    }
    if (a.hall) {
      // D_a[dJ_a b0 + J0_a v - dJ b0_a - J0 v_a]
      const V3<double> s = dfwd(a, nd, ax, [&](long long j) {
        const V3<double> b = ld(a.b0, j), J = ld(a.J0, j), v = ld(a.v, j), dJ = ld(a.dJ, j);
        const double dJa = comp(dJ, ax), Ja = comp(J, ax), ba = comp(b, ax), va = comp(v, ax);
        return V3<double>{dJa * b.x + Ja * v.x - dJ.x * ba - J.x * va, dJa * b.y + Ja * v.y - dJ.y * ba - J.y * va,
                          dJa * b.z + Ja * v.z - dJ.z * ba - J.z * va};
      });
      out = axpy3(a.inv_d[ax], s, out);
    }
    if (a.hod) out = axpy3(a.hod_factor, hod_apply<false>(a, nd, ax, a.v), out);
    if (a.fo) out = axpy3(a.inv_d[ax], fo_apply<false>(a, nd, ax, a.v), out);
    if (AD) {
      out = axpy3(a.inv_d[ax], ad_fo_apply<false>(a, nd, ax, a.v), out);
      out = axpy3(a.hod_factor, ad_ho_apply<false>(a, nd, ax, a.v), out);
    }
  }
  out = axpy3(sat_diag(a, nd, um), vm, out);
  if (a.hall && !a.periodic) {
    const V3<double> b0 = ld(a.b0, k), J0 = ld(a.J0, k), dJ = ld(a.dJ, k);
    const V3<double> tv = {0.5 * um.x - J0.x, 0.5 * um.y - J0.y, 0.5 * um.z - J0.z};
    for (int ax = 0; ax < 3; ++ax) {
      HallSat h;
      if (!hall_sat_axis(a, nd, ax, tv, h)) continue;
      const double dJa = comp(dJ, ax), va = comp(vm, ax), ba = comp(b0, ax);
      out.x += h.c * (h.sw * (h.tva * vm.x - dJa * b0.x) + h.side * (va * J0.x + ba * dJ.x));
      out.y += h.c * (h.sw * (h.tva * vm.y - dJa * b0.y) + h.side * (va * J0.y + ba * dJ.y));
      out.z += h.c * (h.sw * (h.tva * vm.z - dJa * b0.z) + h.side * (va * J0.z + ba * dJ.z));
    }
  }
  st3(a.out + k, out);
}

// Nodes on which every derivative row involved is the interior row of half-width RI: every
// node of a periodic grid, and on a box the nodes at least nb + (SW-1)/2 from every face
// (no boundary row of a neighbour reaches them).  There D^T at the node gathers d[-p] f(k+p)
// and D gathers d[p] f(k+p), d the interior row; RI = 0 when the interior row has entries
// beyond the order's half-width (then every node takes the generic row lookups).
template <int RI>
__device__ __forceinline__ bool fast_node(const AdjArgs &a, const Node &nd) {
  if (RI == 0) return false;
  if (a.periodic) return true;
  const int lo = a.nb + (a.sw - 1) / 2;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax)
    if (nd.i[ax] < lo || nd.i[ax] > nd.n[ax] - 1 - lo) return false;
  return true;
}

// neighbour k + o along ax on the fast path (periodic wrap; interior nodes need none)
__device__ __forceinline__ long long fnbr(const AdjArgs &a, const Node &nd, int ax, int o) {
  int t = nd.i[ax] + o;
  if (a.periodic) {
    t += (t < 0) ? nd.n[ax] : 0;
    t -= (t >= nd.n[ax]) ? nd.n[ax] : 0;
  }
  return nd.idx + (long long)(t - nd.i[ax]) * nd.st[ax];
}

// the interior row d[o + RI] = D[nb][(SW-1)/2 + o]
template <int RI>
__device__ __forceinline__ void interior_row(const AdjArgs &a, double (&d)[2 * RI + 1]) {
  const int c0 = (a.sw - 1) / 2;
#pragma unroll
  for (int o = -RI; o <= RI; ++o) d[o + RI] = a.tab->D[a.nb][c0 + o];
}

// the terms of one axis of F'(b0)^T w at the node from q = D_ax^T w, Du = D_ax u,
// S3 = D_ax^T (u . w), S5 = D_ax^T (u_ax w)
__device__ __forceinline__ void pass1_axis(const AdjArgs &a, int ax, V3<double> q, V3<double> Du, double S3,
                                           V3<double> S5, V3<double> wm, V3<double> um, V3<double> b0m,
                                           V3<double> J0m, V3<double> &z, V3<double> &gJ) {
  if (a.conv) {
    const double ua = comp(um, ax), Dua = comp(Du, ax);
    addc(z, ax, a.two_inv_d[ax] * (a.w[0] * dot3(um, q) + a.w[1] * dot3(Du, wm) + a.w[2] * S3));
    for (int i = 0; i < 3; ++i)
      addc(z, i, -a.two_inv_d[ax] * (a.w[3] * ua * comp(q, i) + a.w[4] * comp(S5, i) + a.w[5] * Dua * comp(wm, i)));
  }
  if (a.hall) {
    const V3<double> Q = {q.x * a.inv_d[ax], q.y * a.inv_d[ax], q.z * a.inv_d[ax]};
    const double J0a = comp(J0m, ax), b0a = comp(b0m, ax);
    z = axpy3(J0a, Q, z);
    addc(z, ax, -dot3(J0m, Q));
    addc(gJ, ax, dot3(b0m, Q));
    gJ = axpy3(-b0a, Q, gJ);
  }
}

// the vjp's result at node k: out = z, or the epilogue dst = eal ex + ebe ey + ega z (the
// operation order of k_lincomb)
__device__ __forceinline__ void vjp_store(const AdjArgs &a, long long k, V3<double> z) {
  if (!a.dst) {
    st3(a.out + k, z);
    return;
  }
  V3<double> r = {0, 0, 0};
  if (a.ex) r = axpy3(a.eal, ld3_plain(a.ex + k), r);
  if (a.ey) r = axpy3(a.ebe, ld3_plain(a.ey + k), r);
  r = axpy3(a.ega, z, r);
  st3(a.dst + k, r);
}

// F'(b0)^T w, pass 1.  With q_a = D_a^T w (per component), the forward terms transpose to
//   D_a[u_i b_a]      -> z_a += sum_i u_i q_a,i          b_a D_a[u_i] -> z_a += D_a[u] . w
//   u_i D_a[b_a]      -> z_a += D_a^T[u . w]             D_a[u_a b_i] -> z_i += u_a q_a,i
//   u_a D_a[b_i]      -> z_i += D_a^T[u_a w_i]           b_i D_a[u_a] -> z_i += D_a[u_a] w_i
// (times the flux-form weights and 2/d_a); the Hall term with Q_a = q_a / d_a gives
//   z_i += J0_a Q_a,i,  z_a -= J0 . Q_a,  and the source for dJ: gJ = sum_a (b0.Q_a) e_a - b0_a Q_a,
// whose curl transpose (pass 2) adds C^T (gJ / rho).  On fast nodes the four gathers of an
// axis share one pass over the neighbours (u and w loaded once per neighbour).
template <int RI, bool AD = false>
__global__ void k_vjp_pass1(const AdjArgs a) {
  Node nd;
  if (!make_node(a, nd)) return;
  const long long k = nd.idx;
  const V3<double> wm = ld(a.v, k), um = a.conv ? ld(a.u, k) : V3<double>{0, 0, 0};
  V3<double> z = {0, 0, 0}, gJ = {0, 0, 0};
  V3<double> b0m = {0, 0, 0}, J0m = {0, 0, 0};
  if (a.hall) b0m = ld(a.b0, k);
  if (fast_node<RI>(a, nd)) {
    double d[2 * RI + 1];
    interior_row<RI>(a, d);
    if (a.hall) {
      // J0 = curl(b0) / rho at the node (as k_curl_rho: interior rows times 1/d, then 1/rho)
      double g[3][3];
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        const int c1 = (ax + 1) % 3, c2 = (ax + 2) % 3;
        double v1 = 0, v2 = 0;
#pragma unroll
        for (int o = -RI; o <= RI; ++o) {
          if (o == 0) continue;
          const V3<double> bj = ld(a.b0, fnbr(a, nd, ax, o));
          v1 += d[RI + o] * comp(bj, c1);
          v2 += d[RI + o] * comp(bj, c2);
        }
        g[ax][c1] = v1 * a.inv_d[ax];
        g[ax][c2] = v2 * a.inv_d[ax];
      }
      const double r = 1.0 / a.rho[k];
      J0m = {(g[1][2] - g[2][1]) * r, (g[2][0] - g[0][2]) * r, (g[0][1] - g[1][0]) * r};
    }
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      V3<double> q = {0, 0, 0}, Du = {0, 0, 0}, S5 = {0, 0, 0};
      double S3 = 0.0;
#pragma unroll
      for (int o = -RI; o <= RI; ++o) {
        const double ct = d[RI - o], cf = d[RI + o];
        V3<double> vj = wm, uj = um;
        if (o != 0) {
          const long long j = fnbr(a, nd, ax, o);
          vj = ld(a.v, j);
          if (a.conv) uj = ld(a.u, j);
        }
        q = axpy3(ct, vj, q);
        if (a.conv) {
          Du = axpy3(cf, uj, Du);
          S3 += ct * dot3(uj, vj);
          const double uja = comp(uj, ax);
          S5 = axpy3(ct, V3<double>{uja * vj.x, uja * vj.y, uja * vj.z}, S5);
        }
      }
      pass1_axis(a, ax, q, Du, S3, S5, wm, um, b0m, J0m, z, gJ);
      if (a.hod) z = axpy3(a.hod_factor, hod_apply<true>(a, nd, ax, a.v), z);
      if (a.fo) z = axpy3(a.inv_d[ax], fo_apply<true>(a, nd, ax, a.v), z);
      if (AD) {
        z = axpy3(a.inv_d[ax], ad_fo_apply<true>(a, nd, ax, a.v), z);
        z = axpy3(a.hod_factor, ad_ho_apply<true>(a, nd, ax, a.v), z);
      }
    }
  } else {
    if (a.hall) J0m = ld(a.J0, k);
    for (int ax = 0; ax < 3; ++ax) {
      const V3<double> q = dtr(a, nd, ax, [&](long long j) { return ld(a.v, j); });
      V3<double> Du = {0, 0, 0}, S5 = {0, 0, 0};
      double S3 = 0.0;
      if (a.conv) {
        Du = dfwd(a, nd, ax, [&](long long j) { return ld(a.u, j); });
        S3 = dtr(a, nd, ax, [&](long long j) {
          const double s = dot3(ld(a.u, j), ld(a.v, j));
          return V3<double>{s, 0, 0};
        }).x;
        S5 = dtr(a, nd, ax, [&](long long j) {
          const double ua = comp(ld(a.u, j), ax);
          const V3<double> ww = ld(a.v, j);
          return V3<double>{ua * ww.x, ua * ww.y, ua * ww.z};
        });
      }
      pass1_axis(a, ax, q, Du, S3, S5, wm, um, b0m, J0m, z, gJ);
      if (a.hod) z = axpy3(a.hod_factor, hod_apply<true>(a, nd, ax, a.v), z);
      if (a.fo) z = axpy3(a.inv_d[ax], fo_apply<true>(a, nd, ax, a.v), z);
      if (AD) {
        z = axpy3(a.inv_d[ax], ad_fo_apply<true>(a, nd, ax, a.v), z);
        z = axpy3(a.hod_factor, ad_ho_apply<true>(a, nd, ax, a.v), z);
      }
    }
  }
  z = axpy3(sat_diag(a, nd, um), wm, z);
  if (a.hall && !a.periodic) {
    // transpose of the Hall outflow SAT's tangent: the terms in v at the node, and the source
    // for dJ (transposed through the curl by pass 2 with the Hall volume term's)
    const V3<double> tv = {0.5 * um.x - J0m.x, 0.5 * um.y - J0m.y, 0.5 * um.z - J0m.z};
    const double bw = dot3(b0m, wm), Jw = dot3(J0m, wm);
    for (int ax = 0; ax < 3; ++ax) {
      HallSat h;
      if (!hall_sat_axis(a, nd, ax, tv, h)) continue;
      z = axpy3(h.c * h.sw * h.tva, wm, z);
      addc(z, ax, h.c * h.side * Jw);
      addc(gJ, ax, -h.c * h.sw * bw);
      gJ = axpy3(h.c * h.side * comp(b0m, ax), wm, gJ);
    }
  }
  if (a.hall) {
    st3(a.out + k, z);
    const double r = 1.0 / a.rho[k];
    st3(a.gJr + k, V3<double>{gJ.x * r, gJ.y * r, gJ.z * r});
  } else {
    vjp_store(a, k, z);
  }
}

// pass 2: z += C^T g with C the SBP curl (rows / d), g = gJ / rho
template <int RI>
__global__ void k_vjp_pass2(const AdjArgs a) {
  Node nd;
  if (!make_node(a, nd)) return;
  const long long k = nd.idx;
  V3<double> g[3];
  if (fast_node<RI>(a, nd)) {
    double d[2 * RI + 1];
    interior_row<RI>(a, d);
    const V3<double> gm = ld(a.gJr, k);
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      V3<double> t = {0, 0, 0};
#pragma unroll
      for (int o = -RI; o <= RI; ++o) t = axpy3(d[RI - o], o == 0 ? gm : ld(a.gJr, fnbr(a, nd, ax, o)), t);
      g[ax] = {t.x * a.inv_d[ax], t.y * a.inv_d[ax], t.z * a.inv_d[ax]};
    }
  } else {
    for (int ax = 0; ax < 3; ++ax) {
      const V3<double> t = dtr(a, nd, ax, [&](long long j) { return ld(a.gJr, j); });
      g[ax] = {t.x * a.inv_d[ax], t.y * a.inv_d[ax], t.z * a.inv_d[ax]};   // (D_ax^T g_c) / d_ax
    }
  }
  // (C^T g)_x = Dz^T g_y - Dy^T g_z, (C^T g)_y = Dx^T g_z - Dz^T g_x, (C^T g)_z = Dy^T g_x - Dx^T g_y
  V3<double> z = ld3_plain(a.out + k);
  z.x += g[2].y - g[1].z;
  z.y += g[0].z - g[2].x;
  z.z += g[1].x - g[0].y;
  vjp_store(a, k, z);
}

// out = alpha*x + beta*y (+ gamma*z) over the nodes (x, y, z may be the same array as out)
__global__ void k_lincomb(long long n, R4<double> *out, double al, const R4<double> *x, double be,
                          const R4<double> *y, double ga, const R4<double> *z) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  V3<double> r = {0, 0, 0};
  if (x) r = axpy3(al, ld3_plain(x + i), r);
  if (y) r = axpy3(be, ld3_plain(y + i), r);
  if (z) r = axpy3(ga, ld3_plain(z + i), r);
  st3(out + i, r);
}

}  // namespace ieq

using namespace ieq;

namespace ieq {
// from api.cu
ieq_status adj_run_kernel(ieq_ctx *c, const char *name, void *const *args, int nargs);
void adj_curl(ieq_ctx *c, const void *b, const void *rho, void *out);
void rk2n_coefficients(bool ck, const double **A, const double **B, const double **C, int *stages);
void adj_context(ieq_ctx *c, Mesh &m, const Tables<double> *&tab, double w[6], double inv_d[3], double two_inv_d[3],
                 double sat_s[3]);
// from api_fused.inc
ieq_status adj_fused_steps(ieq_ctx *c, int conv, void *b, void *b2, void *b3, void *cb, void *u, const void *rho,
                           void *time, int nsteps, void *const *keep, int P);
ieq_status adj_read_conv(ieq_ctx *c, const void *u, int &conv);

AdjArgs adj_args(ieq_ctx *c) {
  AdjArgs a;
  std::memset(&a, 0, sizeof(a));
  adj_context(c, a.m, a.tab, a.w, a.inv_d, a.two_inv_d, a.sat_s);
  a.nb = c->op.nb;
  a.sw = c->op.sw;
  a.wh = c->op.w_hod;
  a.periodic = c->s.periodic ? 1 : 0;
  a.conv = 1;
  a.hall = c->s.hall ? 1 : 0;
  a.hod = c->s.diss_form == 1 ? 1 : 0;
  a.fo = c->s.diss_form == 2 ? 1 : 0;
  a.ad = c->s.diss_form == 3 ? 1 : 0;
  a.mp2min = c->s.mp2min;
  a.mp2max = c->s.mp2max;
  a.cmin = c->s.cmin;
  a.cmax = c->s.cmax;
  a.hsgn = ((c->op.order / 2 + 1) % 2) ? -1.0 : 1.0;
  a.hod_factor = c->s.hod_factor;
  return a;
}
}  // namespace ieq

namespace {

ieq_status afail(ieq_ctx *c, ieq_status st, const std::string &m) {
  c->err = m;
  return st;
}

ieq_status check_adjoint_settings(ieq_ctx *c) {
  if (c->s.real_float) return afail(c, IEQ_ERR_SETTINGS, "the adjoint is FP64 only");
  if (c->s.uibj < 0 || c->s.source < 0 || c->s.ujbi < 0) return afail(c, IEQ_ERR_SETTINGS, "no flux forms");
  return IEQ_OK;
}

// half-width of the vjp kernels' interior fast path: order/2 when the interior derivative row
// has no entries beyond it, else 0 (generic row lookups on every node)
int fast_ri(const ieq_ctx *c) {
  const int ri = c->op.order / 2, c0 = (c->op.sw - 1) / 2;
  for (int k = 0; k < c->op.sw; ++k)
    if (std::abs(k - c0) > ri && c->op.D.at(c->op.nb, k) != 0.0) return 0;
  return ri;
}

dim3 ablock() { return dim3(32, 4, 2); }
dim3 agrid(const ieq_ctx *c) {
  return dim3((c->s.nodes[0] + 31) / 32, (c->s.nodes[1] + 3) / 4, (c->s.nodes[2] + 1) / 2);
}

struct Work {
  void *J0 = nullptr, *dJ = nullptr, *gJr = nullptr;
};

ieq_status work_alloc(ieq_ctx *c, std::vector<void *> &bufs, int n, size_t bytes) {
  for (int i = 0; i < n; ++i) {
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return afail(c, IEQ_ERR_CUDA, "adjoint work allocation");
    cudaMemsetAsync(p, 0, bytes, c->stream);
    bufs.push_back(p);
  }
  return IEQ_OK;
}

void free_all(std::vector<void *> &bufs) {
  for (void *p : bufs) cudaFree(p);
  bufs.clear();
}

// out = F'(b)^T w (u at the stage time, rho); J0, gJr: work fields
// optional epilogue of vjp: dst = al x + be y + ga F'(b)^T w (x, y may be null)
struct Epi {
  void *dst = nullptr;
  const void *x = nullptr, *y = nullptr;
  double al = 0, be = 0, ga = 0;
};

ieq_status vjp(ieq_ctx *c, const void *b, const void *w, const void *u, const void *rho, void *out, void *J0,
               void *gJr, const Epi &epi = Epi()) {
  AdjArgs a = adj_args(c);
  a.dst = (R4<double> *)epi.dst;
  a.ex = (const R4<double> *)epi.x;
  a.ey = (const R4<double> *)epi.y;
  a.eal = epi.al;
  a.ebe = epi.be;
  a.ega = epi.ga;
  a.b0 = (const R4<double> *)b;
  a.u = (const R4<double> *)u;
  a.v = (const R4<double> *)w;
  a.rho = (const double *)rho;
  a.out = (R4<double> *)out;
  a.gJr = (R4<double> *)gJr;
  // adaptive dissipation: its own instantiation of pass 1, generic rows on every node (the
  // terms of its linearisation would raise the other instantiations' registers)
  const int ri1 = a.ad ? 0 : fast_ri(c);
  if (c->s.hall && (!c->s.periodic || ri1 == 0)) {   // else pass 1 forms J0 at every node itself
    adj_curl(c, b, rho, J0);
    a.J0 = (const R4<double> *)J0;
  }
  switch (a.ad ? -1 : ri1) {
    case -1: k_vjp_pass1<0, true><<<agrid(c), ablock(), 0, c->stream>>>(a); break;
    case 1: k_vjp_pass1<1><<<agrid(c), ablock(), 0, c->stream>>>(a); break;
    case 2: k_vjp_pass1<2><<<agrid(c), ablock(), 0, c->stream>>>(a); break;
    case 3: k_vjp_pass1<3><<<agrid(c), ablock(), 0, c->stream>>>(a); break;
    default: k_vjp_pass1<0><<<agrid(c), ablock(), 0, c->stream>>>(a);
  }
  if (c->s.hall) {
    switch (fast_ri(c)) {
      case 1: k_vjp_pass2<1><<<agrid(c), ablock(), 0, c->stream>>>(a); break;
      case 2: k_vjp_pass2<2><<<agrid(c), ablock(), 0, c->stream>>>(a); break;
      case 3: k_vjp_pass2<3><<<agrid(c), ablock(), 0, c->stream>>>(a); break;
      default: k_vjp_pass2<0><<<agrid(c), ablock(), 0, c->stream>>>(a);
    }
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? IEQ_OK : afail(c, IEQ_ERR_CUDA, cudaGetErrorString(e));
}

void lincomb(ieq_ctx *c, void *out, double al, const void *x, double be, const void *y, double ga = 0,
             const void *z = nullptr) {
  const long long n = (long long)c->n;
  k_lincomb<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(n, (R4<double> *)out, al, (const R4<double> *)x, be,
                                                               (const R4<double> *)y, ga, (const R4<double> *)z);
}

// u at stage time t (calc_u with time[1] = t) into `uw`, or the caller's u
const void *stage_u(ieq_ctx *c, const void *u, void *uw, double *d_time, double t) {
  if (!c->s.variable_u) return u;
  double tt[2] = {t, t};
  cudaMemcpyAsync(d_time, tt, sizeof(tt), cudaMemcpyHostToDevice, c->stream);
  void *args[7] = {uw, uw, uw, uw, uw, uw, d_time};   // calc_u_3_args reads u (4) and time (6)
  adj_run_kernel(c, "calc_u_3_args", args, 7);
  return uw;
}

// work fields of one SSPRK33 step adjoint, allocated once per call of the public entry
// points (the checkpointed sweep reuses them for every step)
struct VjpWork {
  std::vector<void *> f;   // J0, gJr, z, l1, l2, l3, uw
  double *d_time = nullptr;
};

ieq_status vjp_work_alloc(ieq_ctx *c, VjpWork &w) {
  ieq_status st = work_alloc(c, w.f, 7, c->n_pad * sizeof(R4<double>));
  if (st == IEQ_OK && cudaMalloc(&w.d_time, 2 * sizeof(double)) != cudaSuccess)
    st = afail(c, IEQ_ERR_CUDA, "adjoint work allocation");
  return st;
}

void vjp_work_free(VjpWork &w) {
  free_all(w.f);
  if (w.d_time) cudaFree(w.d_time);
  w.d_time = nullptr;
}

// lambda <- (d step / d s1)^T lambda for the SSPRK33 step with stage states s1, s2, s3 that
// started at time t0; enqueued on the context's stream, no allocation, no synchronisation
ieq_status ssprk33_step_vjp_ws(ieq_ctx *c, const void *s1, const void *s2, const void *s3, double t0, void *lambda,
                               const void *u, const void *rho, const VjpWork &w) {
  void *J0 = w.f[0], *gJr = w.f[1], *z = w.f[2], *l1 = w.f[3], *l2 = w.f[4], *l3 = w.f[5], *uw = w.f[6];
  double *d_time = w.d_time;
  const double h = c->s.dt;
  const double t2 = t0 + h, t3 = t0 + 0.5 * h;   // SSPRK33_2a / _3a
  ieq_status st;
  // the combinations with F'^T are the vjp's epilogue
  Epi e;
  // stage 3: lambda3 = 2/3 (lambda + h F'(s3)^T lambda); lambda1 = 1/3 lambda
  e.dst = l3; e.x = lambda; e.al = 2.0 / 3.0; e.ga = 2.0 / 3.0 * h;
  if ((st = vjp(c, s3, lambda, stage_u(c, u, uw, d_time, t3), rho, z, J0, gJr, e)) != IEQ_OK) return st;
  lincomb(c, l1, 1.0 / 3.0, lambda, 0.0, nullptr);
  // stage 2: lambda2 = 1/4 (lambda3 + h F'(s2)^T lambda3); lambda1 += 3/4 lambda3
  e.dst = l2; e.x = l3; e.al = 0.25; e.ga = 0.25 * h;
  if ((st = vjp(c, s2, l3, stage_u(c, u, uw, d_time, t2), rho, z, J0, gJr, e)) != IEQ_OK) return st;
  lincomb(c, l1, 1.0, l1, 0.75, l3);
  // stage 1: lambda1 += lambda2 + h F'(s1)^T lambda2
  e.dst = lambda; e.x = l1; e.y = l2; e.al = 1.0; e.be = 1.0; e.ga = h;
  return vjp(c, s1, l2, stage_u(c, u, uw, d_time, t0), rho, z, J0, gJr, e);
}

// lambda <- (d step / d b_n)^T lambda for one step of a 2N low-storage scheme
// (kernel_time_integrator.cl:1023-1206 CarpenterKennedy2N54, 1216-1516 ToulorgeDesmet2N84F)
// from the stage inputs x[s] (b1 before stage s) of a step that started at t0:
//   stage s:  b2 = A_s b2 + h F(x[s], t_s);  b1 = x[s] + B_s b2    (t_0 = t0, t_s = t0 + C_{s-1} h)
// reversed with mu1 = lambda (b1 after the step) and mu2 = 0 (the next step's first stage has
// A_0 = 0, so b2 after a step does not reach the next):
//   mu2 += B_s mu1;  mu1 += h F'(x[s], t_s)^T mu2;  mu2 = A_s mu2      (s = S-1 .. 0)
// (the scaling by A_s and the next stage's B_{s-1} mu1 in one pass; mu1 += h F'^T mu2 as the
// vjp's epilogue).  w.f[3] holds mu2; no allocation, no synchronisation
ieq_status rk2n_step_vjp_ws(ieq_ctx *c, bool ck, void *const *x, double t0, void *lambda, const void *u,
                            const void *rho, const VjpWork &w) {
  void *J0 = w.f[0], *gJr = w.f[1], *z = w.f[2], *mu2 = w.f[3], *uw = w.f[6];
  const double *A, *B, *C;
  int S;
  rk2n_coefficients(ck, &A, &B, &C, &S);
  const double h = c->s.dt;
  ieq_status st;
  Epi e;
  e.dst = lambda; e.x = lambda; e.al = 1.0; e.ga = h;
  for (int s = S - 1; s >= 0; --s) {
    const double ts = s == 0 ? t0 : t0 + C[s - 1] * h;
    if (s == S - 1) lincomb(c, mu2, B[s], lambda, 0.0, nullptr);   // mu2 = 0 + B_s mu1
    else lincomb(c, mu2, A[s + 1], mu2, B[s], lambda);             // A_{s+1} mu2 + B_s mu1
    if ((st = vjp(c, x[s], mu2, stage_u(c, u, uw, w.d_time, ts), rho, z, J0, gJr, e)) != IEQ_OK) return st;
  }
  return IEQ_OK;
}

// lambda <- (d step / d b_n)^T lambda for one step given as a register program
// (rk_step_program: every integrator) from the stage inputs x[e] of the e-th evaluating
// stage of a step that started at t0.  Adjoint registers L0 = lambda, L1 = L2 = 0; the stages
// in reverse order, each assignment R[dst] = sum a[r] R[r] + k K transposed newest first
// (t = L[dst]; L[dst] = a[dst] t; L[r] += a[r] t for r != dst; LK += k t), then the stage's
// evaluation K = h F(R[src]) transposed: L[src] += h F'(x)^T LK (the vjp's epilogue).
// No allocation, no synchronisation
ieq_status program_step_vjp_ws(ieq_ctx *c, const RkProgram &prog, void *const *x, double t0, void *lambda,
                               const void *u, const void *rho, const VjpWork &w, void *L1, void *L2, void *LK,
                               void *tmp) {
  void *J0 = w.f[0], *gJr = w.f[1], *z = w.f[2], *uw = w.f[6];
  void *L[3] = {lambda, L1, L2};
  const size_t vb = c->n_pad * sizeof(R4<double>);
  cudaMemsetAsync(L1, 0, vb, c->stream);
  cudaMemsetAsync(L2, 0, vb, c->stream);
  int e = prog.evaluations;
  for (int si = (int)prog.stages.size() - 1; si >= 0; --si) {
    const RkStage &st = prog.stages[si];
    if (st.src >= 0) {
      cudaMemsetAsync(LK, 0, vb, c->stream);
      --e;
    }
    for (int ai = (int)st.as.size() - 1; ai >= 0; --ai) {
      const RkAssign &as = st.as[ai];
      lincomb(c, tmp, 1.0, L[as.dst], 0.0, nullptr);
      lincomb(c, L[as.dst], as.a[as.dst], tmp, 0.0, nullptr);
      for (int r = 0; r < 3; ++r)
        if (r != as.dst && as.a[r] != 0.0) lincomb(c, L[r], 1.0, L[r], as.a[r], tmp);
      if (st.src >= 0 && as.k != 0.0) lincomb(c, LK, 1.0, LK, as.k, tmp);
    }
    if (st.src >= 0) {
      Epi ep;
      ep.dst = L[st.src];
      ep.x = L[st.src];
      ep.al = 1.0;
      ep.ga = st.h;
      const ieq_status r = vjp(c, x[e], LK, stage_u(c, u, uw, w.d_time, t0 + st.t), rho, z, J0, gJr, ep);
      if (r != IEQ_OK) return r;
    }
  }
  return IEQ_OK;
}

}  // namespace

extern "C" {

ieq_status ieq_operator_jvp(ieq_ctx *c, const void *b, const void *v, const void *u, const void *rho, void *out) {
  if (!c || !b || !v || !u || !rho || !out) return IEQ_ERR_ARG;
  ieq_status st = check_adjoint_settings(c);
  if (st != IEQ_OK) return st;
  cudaSetDevice(c->device);
  std::vector<void *> w;
  if ((st = work_alloc(c, w, 2, c->n_pad * sizeof(R4<double>))) != IEQ_OK) return st;
  AdjArgs a = adj_args(c);
  a.b0 = (const R4<double> *)b;
  a.u = (const R4<double> *)u;
  a.v = (const R4<double> *)v;
  a.rho = (const double *)rho;
  a.out = (R4<double> *)out;
  if (c->s.hall) {
    adj_curl(c, b, rho, w[0]);
    adj_curl(c, v, rho, w[1]);
    a.J0 = (const R4<double> *)w[0];
    a.dJ = (const R4<double> *)w[1];
  }
  if (a.ad) k_jvp<true><<<agrid(c), ablock(), 0, c->stream>>>(a);
  else k_jvp<false><<<agrid(c), ablock(), 0, c->stream>>>(a);
  const cudaError_t e = cudaStreamSynchronize(c->stream);
  free_all(w);
  return e == cudaSuccess ? IEQ_OK : afail(c, IEQ_ERR_CUDA, cudaGetErrorString(e));
}

ieq_status ieq_operator_vjp(ieq_ctx *c, const void *b, const void *w, const void *u, const void *rho, void *out) {
  if (!c || !b || !w || !u || !rho || !out) return IEQ_ERR_ARG;
  ieq_status st = check_adjoint_settings(c);
  if (st != IEQ_OK) return st;
  cudaSetDevice(c->device);
  std::vector<void *> bufs;
  if ((st = work_alloc(c, bufs, 2, c->n_pad * sizeof(R4<double>))) != IEQ_OK) return st;
  st = vjp(c, b, w, u, rho, out, bufs[0], bufs[1]);
  const cudaError_t e = cudaStreamSynchronize(c->stream);
  free_all(bufs);
  if (st != IEQ_OK) return st;
  return e == cudaSuccess ? IEQ_OK : afail(c, IEQ_ERR_CUDA, cudaGetErrorString(e));
}

// Adjoint of one SSPRK33 step (kernel_time_integrator.cl:224-303) from its stage states
// s1 = b_n, s2 = b^(2), s3 = b^(3) and the step start time t0: lambda <- (db_{n+1}/db_n)^T lambda.
//   b2 = s1 + h F(s1, t0)            b3 = 3/4 s1 + 1/4 (s2 + h F(s2, t0 + h))
//   b_{n+1} = 1/3 s1 + 2/3 (s3 + h F(s3, t0 + h/2))
ieq_status ieq_ssprk33_step_vjp(ieq_ctx *c, const void *s1, const void *s2, const void *s3, double t0, void *lambda,
                                const void *u, const void *rho) {
  if (!c || !s1 || !s2 || !s3 || !lambda || !u || !rho) return IEQ_ERR_ARG;
  ieq_status st = check_adjoint_settings(c);
  if (st != IEQ_OK) return st;
  cudaSetDevice(c->device);
  VjpWork w;
  if ((st = vjp_work_alloc(c, w)) == IEQ_OK) st = ssprk33_step_vjp_ws(c, s1, s2, s3, t0, lambda, u, rho, w);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess && st == IEQ_OK) st = afail(c, IEQ_ERR_CUDA, "step vjp");
  vjp_work_free(w);
  return st;
}

// Adjoint of num_steps SSPRK33 steps from b0 (time 0): lambda holds dL/db(T) on entry and
// dL/db0 on return.  The forward run is checkpointed every `checkpoint_every` steps; each
// segment is recomputed (stage states kept) and swept backwards.
}  // extern "C"

namespace {
// n zeroed vector fields from the context's adjoint pool (grown on demand, kept until
// ieq_destroy, so repeated sweeps allocate nothing)
ieq_status adj_pool(ieq_ctx *c, size_t n, size_t bytes, std::vector<void *> &out) {
  while (c->adj_bufs.size() < n) {
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return afail(c, IEQ_ERR_CUDA, "adjoint work allocation");
    c->adj_bufs.push_back(p);
  }
  if (!c->adj_time && cudaMalloc(&c->adj_time, 4 * sizeof(double)) != cudaSuccess)
    return afail(c, IEQ_ERR_CUDA, "adjoint work allocation");
  out.assign(c->adj_bufs.begin(), c->adj_bufs.begin() + (long)n);
  for (void *p : out) cudaMemsetAsync(p, 0, bytes, c->stream);
  return IEQ_OK;
}
}  // namespace

extern "C" {

ieq_status ieq_adjoint_steps(ieq_ctx *c, const void *b0, void *lambda, const void *u, const void *rho, int num_steps,
                             int checkpoint_every) {
  if (!c || !b0 || !lambda || !u || !rho || num_steps < 0 || checkpoint_every < 1) return IEQ_ERR_ARG;
  ieq_status st = check_adjoint_settings(c);
  if (st != IEQ_OK) return st;
  const bool ssp = c->s.integrator == "SSPRK33";
  const bool ck2n = c->s.integrator == "CarpenterKennedy2N54", td2n = c->s.integrator == "ToulorgeDesmet2N84F";
  const int integ = integrator_id(c->s.integrator);
  if (integ < 0) return afail(c, IEQ_ERR_SETTINGS, "no time integrator (-DIEQ_INTEGRATOR=...) in the settings");
  // SSPRK33 and the 2N schemes have step adjoints of their own; the other integrators (and
  // every one with IEQ_ADJOINT_PROGRAM=1) reverse the step's register program
  const bool program = !(ssp || ck2n || td2n) || c->s.adjoint_program;
  if (program && c->s.stage_kernel == 4)
    return afail(c, IEQ_ERR_SETTINGS, "the register-program adjoint recomputes the forward with the fused kernels");
  RkProgram prog;
  if (program) rk_step_program(integ, c->s.dt, prog);
  cudaSetDevice(c->device);
  const size_t vb = c->n_pad * sizeof(R4<double>);
  const int K = checkpoint_every;
  const int nseg = (num_steps + K - 1) / K;
  // states kept per step: SSPRK33 its three stage states, a 2N scheme the input of every stage
  const double *A2, *B2, *C2;
  int S2 = 0;
  if (ck2n || td2n) rk2n_coefficients(ck2n, &A2, &B2, &C2, &S2);
  const int P = program ? prog.evaluations : ssp ? 3 : S2;
  // checkpoints (nseg), the stage states of one segment (P K), step work (5), step-adjoint
  // work (7), the program's adjoint registers L1, L2, LK and a temporary (4)
  std::vector<void *> pool;
  if ((st = adj_pool(c, (size_t)nseg + (size_t)P * K + 16, vb, pool)) != IEQ_OK) return st;
  std::vector<void *> ck(pool.begin(), pool.begin() + nseg), seg(pool.begin() + nseg, pool.begin() + nseg + P * K),
      w(pool.begin() + nseg + P * K, pool.begin() + nseg + P * K + 5);
  VjpWork vw;
  vw.f.assign(pool.begin() + nseg + P * K + 5, pool.begin() + nseg + P * K + 12);
  void *const *preg = &pool[(size_t)nseg + (size_t)P * K + 12];   // L1, L2, LK, tmp
  vw.d_time = c->adj_time + 2;
  void *cur = w[0], *b2 = w[1], *b3 = w[2], *cb = w[3], *uw = w[4];
  double *d_time = c->adj_time;
  std::vector<double> t0s(num_steps + 1, 0.0);
  for (int n = 0; n < num_steps; ++n) t0s[n + 1] = t0s[n] + c->s.dt;   // calc_time_3_args / _2_args
  // the forward passes run the fused stage kernels (ieq_time_steps' path) unless the settings
  // ask for the reference kernel lists (IEQ_STAGE_KERNEL=LIST)
  const bool fused = c->s.stage_kernel != 4;
  int conv = 1;
  if (fused && (st = adj_read_conv(c, u, conv)) != IEQ_OK) return st;
  void *ua = c->s.variable_u ? uw : (void *)u;   // u is rewritten only when it varies in time
  auto set_time = [&](double t0) {
    const double tt[2] = {t0, t0};
    cudaMemcpyAsync(d_time, tt, sizeof(tt), cudaMemcpyHostToDevice, c->stream);
  };
  // one step through the reference kernels; keep (optional) receives the P states of the step
  auto step = [&](void *state, void *const *keep) -> ieq_status {
    if (ssp) {
      if (keep) cudaMemcpyAsync(keep[0], state, vb, cudaMemcpyDeviceToDevice, c->stream);
      void *args[7] = {state, b2, b3, cb, ua, (void *)rho, d_time};
      const char *seq[] = {"calc_curlB_rho_1_3args", "calc_u_3_args", "SSPRK33_1", "SSPRK33_2a",
                           "calc_curlB_rho_2_3args", "calc_u_3_args", "SSPRK33_2b", "SSPRK33_3a",
                           "calc_curlB_rho_3_3args", "calc_u_3_args", "SSPRK33_3b", "calc_time_3_args"};
      for (const char *k : seq) {
        if (!c->s.hall && std::strncmp(k, "calc_curlB", 10) == 0) continue;
        if (!c->s.variable_u && std::strncmp(k, "calc_u", 6) == 0) continue;
        ieq_status s = adj_run_kernel(c, k, args, 7);
        if (s != IEQ_OK) return s;
        if (std::strcmp(k, "SSPRK33_1") == 0 && keep) cudaMemcpyAsync(keep[1], b2, vb, cudaMemcpyDeviceToDevice, c->stream);
        if (std::strcmp(k, "SSPRK33_2b") == 0 && keep) cudaMemcpyAsync(keep[2], b3, vb, cudaMemcpyDeviceToDevice, c->stream);
      }
      return IEQ_OK;
    }
    // 2N: for every stage the curl (Hall), the velocity (variable u), the "a" and the "b"
    // kernel, then calc_time_2_args; b1 kept before every "a" kernel
    void *args[6] = {state, b2, cb, ua, (void *)rho, d_time};
    const std::string p = ck2n ? "CarpenterKennedy2N54_" : "ToulorgeDesmet2N84F_";
    for (int s = 0; s < S2; ++s) {
      if (keep) cudaMemcpyAsync(keep[s], state, vb, cudaMemcpyDeviceToDevice, c->stream);
      ieq_status r;
      if (c->s.hall && (r = adj_run_kernel(c, "calc_curlB_rho_1_2args", args, 6)) != IEQ_OK) return r;
      if (c->s.variable_u && (r = adj_run_kernel(c, "calc_u_2_args", args, 6)) != IEQ_OK) return r;
      if ((r = adj_run_kernel(c, (p + std::to_string(s + 1) + "a").c_str(), args, 6)) != IEQ_OK) return r;
      if ((r = adj_run_kernel(c, (p + std::to_string(s + 1) + "b").c_str(), args, 6)) != IEQ_OK) return r;
    }
    return adj_run_kernel(c, "calc_time_2_args", args, 6);
  };
  // nsteps steps of `state` from time t0, the stage states of step k into keep[P k ..] if given
  auto advance = [&](void *state, double t0, int nsteps, void *const *keep) -> ieq_status {
    set_time(t0);
    if (fused) return adj_fused_steps(c, conv, state, b2, b3, cb, ua, rho, d_time, nsteps, keep, P);
    ieq_status r = IEQ_OK;
    for (int k = 0; k < nsteps && r == IEQ_OK; ++k) r = step(state, keep ? keep + (size_t)P * k : nullptr);
    return r;
  };
  // forward sweep: the checkpoints at the start of every segment (the last segment's steps are
  // run by the reverse sweep only)
  cudaMemcpyAsync(cur, b0, vb, cudaMemcpyDeviceToDevice, c->stream);
  for (int s = 0; s < nseg && st == IEQ_OK; ++s) {
    cudaMemcpyAsync(ck[s], cur, vb, cudaMemcpyDeviceToDevice, c->stream);
    if (s + 1 < nseg) st = advance(cur, t0s[(size_t)s * K], K, nullptr);
  }
  // reverse sweep: recompute a segment from its checkpoint keeping the stage states, then
  // apply the step adjoints backwards
  for (int s = nseg - 1; s >= 0 && st == IEQ_OK; --s) {
    const int n0 = s * K, n1 = std::min(num_steps, n0 + K);
    cudaMemcpyAsync(cur, ck[s], vb, cudaMemcpyDeviceToDevice, c->stream);
    st = advance(cur, t0s[n0], n1 - n0, seg.data());
    for (int n = n1 - 1; n >= n0 && st == IEQ_OK; --n) {
      void *const *x = &seg[(size_t)P * (n - n0)];
      if (program)
        st = program_step_vjp_ws(c, prog, x, t0s[n], lambda, u, rho, vw, preg[0], preg[1], preg[2], preg[3]);
      else
        st = ssp ? ssprk33_step_vjp_ws(c, x[0], x[1], x[2], t0s[n], lambda, u, rho, vw)
                 : rk2n_step_vjp_ws(c, ck2n, x, t0s[n], lambda, u, rho, vw);
    }
  }
  if (cudaStreamSynchronize(c->stream) != cudaSuccess && st == IEQ_OK) st = afail(c, IEQ_ERR_CUDA, "adjoint sweep");
  return st;
}

}  // extern "C"
