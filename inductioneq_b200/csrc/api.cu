// api.cu -- the C ABI of include/inductioneq.h: contexts, the name-dispatched reference
// kernels, the fused/graph-captured time stepping, device-resident CG cleaning and norms.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ieq_host.h"
#include "misc_kernels.cuh"
#include "stage_brick.cuh"
#include "stage_z.cuh"
#include "diag.cuh"
#include "diag_curl.cuh"

namespace ieq {
void free_brick_maps(ieq_ctx *c);   // api_fused.inc
}

using namespace ieq;

namespace {

constexpr int kReduceBlocks = 592;   // 4 x 148 SMs; fixed so that sums are reproducible
constexpr int kMaxPartials = 65536;  // least size of the block-partial buffers (CG passes, diagnostics)
// grids from which IEQ_STAGE_KERNEL=AUTO runs the one-pass Hall stage (stage_z.cuh).
// Measured on B200 (whistler, 6th order + HOD, FP64): 1.73 ms per stage at 256^3 against
// 0.78 ms for the curl + stage pair (0.22 / 0.69 ms at 128^3): its shared-memory E ring
// leaves about 23 KB of L1, the B stencil loads hit L1 33 % of the time and the kernel is
// L2-latency bound.  AUTO therefore never takes it; IEQ_STAGE_KERNEL=ZMARCH does.
constexpr long long kZmarchAutoNodes = 1LL << 62;
// IEQ_CURL_Z=2 (the default) runs the 2.5D curl kernel on periodic FP64 grids of more than
// kCurlZAutoNodes nodes, with the dissipation sum and stencil radius 1 or 3.  Measured on B200
// (whistler, CK2N54, step time against the pair curl kernel): 6th order + HOD 160^3 / 192^3 /
// 256^3 +8.5 / +3.5 / +3.2 %, 128^3 -0.9 %; 2nd order + HOD +9 / +2 / +1 %; slower for 4th
// order (-2..-4 % at 192^3 and 256^3), without the dissipation sum (-3 %) and in FP32 (the
// four-node kernels, -6..-14 %).
constexpr long long kCurlZAutoNodes = 1LL << 21;
template <typename R>
inline bool curl_z_auto(const ieq_ctx *c, bool hod) {
  const int ri = c->op.order / 2;
  return sizeof(R) == 8 && hod && (ri == 1 || ri == 3) && (long long)c->n > kCurlZAutoNodes;
}

#define IEQ_CUDA(ctx, call)                                                                    \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) {                                                                   \
      (ctx)->err = std::string(#call) + ": " + cudaGetErrorString(e_);                         \
      return IEQ_ERR_CUDA;                                                                     \
    }                                                                                          \
  } while (0)

#define IEQ_LAUNCHED(ctx)                                                                      \
  do {                                                                                         \
    cudaError_t e_ = cudaGetLastError();                                                       \
    if (e_ != cudaSuccess) {                                                                   \
      (ctx)->err = std::string("kernel launch: ") + cudaGetErrorString(e_);                    \
      return IEQ_ERR_CUDA;                                                                     \
    }                                                                                          \
  } while (0)

ieq_status fail(ieq_ctx *ctx, ieq_status st, const std::string &msg) {
  if (ctx) ctx->err = msg;
  return st;
}

Mesh mesh_of(const ieq_ctx *c) {
  Mesh m;
  m.nx = c->s.nodes[0];
  m.ny = c->s.nodes[1];
  m.nz = c->s.nodes[2];
  for (int a = 0; a < 3; ++a) {
    m.xmin[a] = c->s.xmin[a];
    m.d[a] = c->s.d[a];
  }
  m.omega = c->s.omega;
  m.zoff = c->s.zoff;
  m.nzg = c->s.nzg;
  return m;
}

dim3 block3() { return dim3(32, 4, 2); }
dim3 grid3(int gx, int gy, int gz) {
  dim3 b = block3();
  return dim3((gx + b.x - 1) / b.x, (gy + b.y - 1) / b.y, (gz + b.z - 1) / b.z);
}

// ------------------------------------------------------------------------- table upload
template <typename R>
ieq_status upload_tables(ieq_ctx *c) {
  const SbpOperator &op = c->op;
  Tables<R> t;
  std::memset(&t, 0, sizeof(t));
  const int rows = 2 * op.nb + 1;
  const int WH = op.w_hod;
  const R sgn = ((op.order / 2 + 1) % 2) ? (R)-1 : (R)1;   // pown(-1.0, ORDER/2+1)
  for (int r = 0; r < rows; ++r) {
    for (int k = 0; k < op.sw; ++k) {
      t.D[r][k] = (R)op.D.at(r, k);
      t.Dadj[r][k] = (R)op.Dadj.at(r, k);
    }
    for (int k = 0; k < WH; ++k) t.DHO[r][k] = (R)op.DHO.at(r, k);
    t.Minv[r] = (R)op.minv[r];
    // combined dissipation row: sum over start s and inner i of the reference's
    // M_INV[row] * D_HO[row][s+W-1] * D_HO[NB][i] * (-1)^(ORDER/2+1) at offset s+i
    for (int s = -WH + 1; s <= 0; ++s)
      for (int i = 0; i < WH; ++i) {
        const R term = (((R)op.minv[r] * (R)op.DHO.at(r, s + WH - 1)) * (R)op.DHO.at(op.nb, i)) * sgn;
        t.H[r][s + i + WH - 1] += term;
      }
  }
  IEQ_CUDA(c, cudaMalloc(&c->d_tables, sizeof(Tables<R>)));
  IEQ_CUDA(c, cudaMemcpy(c->d_tables, &t, sizeof(t), cudaMemcpyHostToDevice));
  // flat D / Dadj rows for the generic operators, in R and FP64
  std::vector<R> rr(2 * rows * op.sw);
  std::vector<double> rd(2 * rows * op.sw);
  for (int r = 0; r < rows; ++r)
    for (int k = 0; k < op.sw; ++k) {
      rr[r * op.sw + k] = (R)op.D.at(r, k);
      rr[rows * op.sw + r * op.sw + k] = (R)op.Dadj.at(r, k);
      rd[r * op.sw + k] = op.D.at(r, k);
      rd[rows * op.sw + r * op.sw + k] = op.Dadj.at(r, k);
    }
  IEQ_CUDA(c, cudaMalloc(&c->d_rows_r, rr.size() * sizeof(R)));
  IEQ_CUDA(c, cudaMemcpy(c->d_rows_r, rr.data(), rr.size() * sizeof(R), cudaMemcpyHostToDevice));
  IEQ_CUDA(c, cudaMalloc(&c->d_rows_d, rd.size() * sizeof(double)));
  IEQ_CUDA(c, cudaMemcpy(c->d_rows_d, rd.data(), rd.size() * sizeof(double), cudaMemcpyHostToDevice));
  // Laplacian rows of the selected form
  if (op.has_lap[c->s.laplace]) {
    const SbpRows &L = op.lap[c->s.laplace];
    std::vector<R> lr(L.rows.size());
    for (size_t i = 0; i < L.rows.size(); ++i) lr[i] = (R)L.rows[i];
    IEQ_CUDA(c, cudaMalloc(&c->d_lap_r, lr.size() * sizeof(R)));
    IEQ_CUDA(c, cudaMemcpy(c->d_lap_r, lr.data(), lr.size() * sizeof(R), cudaMemcpyHostToDevice));
    IEQ_CUDA(c, cudaMalloc(&c->d_lap_d, L.rows.size() * sizeof(double)));
    IEQ_CUDA(c, cudaMemcpy(c->d_lap_d, L.rows.data(), L.rows.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  // norm weights (REAL)D / M_INV[row] per axis (kernel_operator.cl:26-28)
  std::vector<R> w;
  for (int a = 0; a < 3; ++a) {
    const int n = c->s.nodes[a];
    for (int i = 0; i < n; ++i) {
      int row = op.nb;
      if (!c->s.periodic) {
        int bound = 0;
        if (i < op.nb) bound -= op.nb - i;
        if (n - 1 - i < op.nb) bound += op.nb - (n - 1 - i);
        row = op.nb + bound;
      }
      w.push_back((R)c->s.d[a] / (R)op.minv[row]);
    }
  }
  IEQ_CUDA(c, cudaMalloc(&c->d_wnorm, w.size() * sizeof(R)));
  IEQ_CUDA(c, cudaMemcpy(c->d_wnorm, w.data(), w.size() * sizeof(R), cudaMemcpyHostToDevice));
  return IEQ_OK;
}

template <typename R>
const Tables<R> *tables(const ieq_ctx *c) {
  return reinterpret_cast<const Tables<R> *>(c->d_tables);
}

// ------------------------------------------------------------------------- stage launch
struct Forms {
  double w[6];
  int need;
};

Forms flux_forms(const Settings &s) {
  // weights of the factored split forms (see stage_kernel.cuh)
  static const double ui[3][3] = {{0.5, 0, 0}, {0.25, 0.25, 0.25}, {0, 0.5, 0.5}};   // C S P
  static const double so[4][3] = {{0, 0, 0.5}, {0.25, -0.25, 0.25}, {0, 0, 0}, {0, 0, 0}};  // C S - Z
  static const double uj[3][3] = {{0.5, 0, 0}, {0.25, 0.25, 0.25}, {0, 0.5, 0.5}};
  Forms f{};
  const int u = s.uibj < 0 ? 2 : s.uibj, r = s.source < 0 ? 0 : s.source, j = s.ujbi < 0 ? 0 : s.ujbi;
  for (int k = 0; k < 3; ++k) {
    f.w[k] = ui[u][k] - so[r][k];
    f.w[3 + k] = uj[j][k];
  }
  f.need = (f.w[0] != 0 ? 1 : 0) | ((f.w[1] != 0 || f.w[5] != 0) ? 2 : 0) |
           ((f.w[2] != 0 || f.w[4] != 0) ? 4 : 0) | (f.w[3] != 0 ? 8 : 0);
  return f;
}

template <typename R, typename F = AoS<R>>
StageArgs<R, F> stage_base(ieq_ctx *c, bool conv) {
  StageArgs<R, F> a;
  std::memset(&a, 0, sizeof(a));
  a.m = mesh_of(c);
  a.tab = tables<R>(c);
  const SbpOperator &op = c->op;
  const int RI = op.order / 2, C0 = (op.sw - 1) / 2, WH = op.w_hod;
  for (int o = -RI; o <= RI; ++o) a.Dint[o + RI] = (R)op.D.at(op.nb, C0 + o);
  // interior dissipation row (M_INV = 1, integer D_HO: exact)
  const R sgn = ((op.order / 2 + 1) % 2) ? (R)-1 : (R)1;
  for (int s = -WH + 1; s <= 0; ++s)
    for (int i = 0; i < WH; ++i)
      a.Hint[s + i + RI] += (((R)op.minv[op.nb] * (R)op.DHO.at(op.nb, s + WH - 1)) * (R)op.DHO.at(op.nb, i)) * sgn;
  for (int ax = 0; ax < 3; ++ax) {
    a.two_inv_d[ax] = (R)(2.0 / c->s.d[ax]);
    a.inv_d[ax] = (R)(1.0 / c->s.d[ax]);
    a.sat_s[ax] = (R)((double)(R)op.minv[0] / c->s.d[ax]);
    a.dR[ax] = (R)c->s.d[ax];
  }
  const Forms f = flux_forms(c->s);
  for (int k = 0; k < 6; ++k) a.w[k] = (R)f.w[k];
  a.need = f.need;
  a.conv = conv ? 1 : 0;
  a.tc = c->s.testcase;
  a.diss_form = c->s.diss_form;
  a.hod_factor = (R)c->s.hod_factor;
  a.mp2min = c->s.mp2min;
  a.mp2max = c->s.mp2max;
  a.cmin = c->s.cmin;
  a.cmax = c->s.cmax;
  a.counter = c->d_counter;
  a.tDT = (R)c->s.dt;
  return a;
}

int diss_kind(const Settings &s) {
  if (s.diss_form == 1) return DISS_HO;
  if (s.diss_form == 2 || s.diss_form == 3) return DISS_FO_OR_AD;
  return DISS_NONE;
}

template <typename R, typename F>
void launch_stage_any(ieq_ctx *c, const StageArgs<R, F> &a, int conv = -1) {
  const dim3 g = grid3(c->s.nodes[0], c->s.nodes[1], c->s.nodes[2]), b = block3();
  const bool per = c->s.periodic, hall = c->s.hall;
  const int d = diss_kind(c->s);
  switch (c->op_id) {
    case 0: launch_stage<R, F, 0>(a, per, hall, d, conv, g, b, c->stream); break;
    case 1: launch_stage<R, F, 1>(a, per, hall, d, conv, g, b, c->stream); break;
    case 2: launch_stage<R, F, 2>(a, per, hall, d, conv, g, b, c->stream); break;
    case 3: launch_stage<R, F, 3>(a, per, hall, d, conv, g, b, c->stream); break;
    case 4: launch_stage<R, F, 4>(a, per, hall, d, conv, g, b, c->stream); break;
    case 5: launch_stage<R, F, 5>(a, per, hall, d, conv, g, b, c->stream); break;
  }
}

// the block shape of a column kernel (x, y, z threads, from IEQ_COL_BLOCK / IEQ_CURL_BLOCK;
// all zero: the kernels' defaults, see pair_shape) and whether the Hall kernels run two
// nodes per thread
static ColShape col_shape(const int (&b)[3], int pairs, bool pdl, int band) {
  ColShape sh;
  if (b[0] > 0) {
    sh = ColShape{b[0], b[1], b[2]};
    sh.given = true;
  }
  sh.pairs = pairs != 0;
  sh.quads = pairs == 4;
  sh.pdl = pdl;
  sh.band = band;
  return sh;
}

template <typename R>
void launch_stage_col_any(ieq_ctx *c, const StageArgs<R, SoA<R>> &a, int conv, bool hodp = false) {
  const bool per = c->s.periodic, hall = c->s.hall, hod = diss_kind(c->s) == DISS_HO;
  const bool foad = diss_kind(c->s) == DISS_FO_OR_AD;
  const ColShape sh = col_shape(c->s.col_block, c->s.col_pairs, c->s.pdl, c->s.xband);
  switch (c->op_id) {
    case 0: launch_stage_col<R, 0>(a, per, hall, hod, conv, hodp, foad, sh, c->stream); break;
    case 1: launch_stage_col<R, 1>(a, per, hall, hod, conv, hodp, foad, sh, c->stream); break;
    case 2: launch_stage_col<R, 2>(a, per, hall, hod, conv, hodp, foad, sh, c->stream); break;
    case 3: launch_stage_col<R, 3>(a, per, hall, hod, conv, hodp, foad, sh, c->stream); break;
    case 4: launch_stage_col<R, 4>(a, per, hall, hod, conv, hodp, foad, sh, c->stream); break;
    case 5: launch_stage_col<R, 5>(a, per, hall, hod, conv, hodp, foad, sh, c->stream); break;
  }
}

// the one-pass Hall stage (stage_z.cuh)
template <typename R>
void launch_stage_zmarch_any(ieq_ctx *c, const StageArgs<R, SoA<R>> &a, const R *rho, bool hod) {
  switch (c->op_id) {
    case 0: launch_stage_zmarch<R, 0>(a, rho, hod, c->s.pdl, c->s.zmarch_tz, c->stream); break;
    case 1: launch_stage_zmarch<R, 1>(a, rho, hod, c->s.pdl, c->s.zmarch_tz, c->stream); break;
    case 2: launch_stage_zmarch<R, 2>(a, rho, hod, c->s.pdl, c->s.zmarch_tz, c->stream); break;
    case 3: launch_stage_zmarch<R, 3>(a, rho, hod, c->s.pdl, c->s.zmarch_tz, c->stream); break;
    case 4: launch_stage_zmarch<R, 4>(a, rho, hod, c->s.pdl, c->s.zmarch_tz, c->stream); break;
    case 5: launch_stage_zmarch<R, 5>(a, rho, hod, c->s.pdl, c->s.zmarch_tz, c->stream); break;
  }
}

template <typename R, typename F>
CurlArgs<R, F> curl_args(ieq_ctx *c, F b, const R *rho, F out);

// E = J x B with J = curl(b)/rho, and J on the faces of a non-periodic box
template <typename R>
void launch_curl_e_any(ieq_ctx *c, SoA<R> b, const R *rho, SoA<R> E, SoA<R> jface, SoA<R> hout = SoA<R>{}) {
  CurlArgs<R, SoA<R>> a = curl_args<R, SoA<R>>(c, b, rho, E);
  a.jface = jface;
  a.hout = hout;
  const bool hod = hout.p != nullptr;
  if (hod) {
    // the interior dissipation row, as stage_base forms it
    const SbpOperator &op = c->op;
    const int RI = op.order / 2, WH = op.w_hod;
    const R sgn = ((op.order / 2 + 1) % 2) ? (R)-1 : (R)1;
    for (int s = -WH + 1; s <= 0; ++s)
      for (int i = 0; i < WH; ++i)
        a.Hint[s + i + RI] += (((R)op.minv[op.nb] * (R)op.DHO.at(op.nb, s + WH - 1)) * (R)op.DHO.at(op.nb, i)) * sgn;
  }
  const bool per = c->s.periodic;
  // the 2.5D curl kernel (stage_z.cuh) on periodic grids: forced by IEQ_CURL_Z=1, or
  // (IEQ_CURL_Z=2, the default) where curl_z_auto measured it faster
  if (per && (c->s.curl_z == 1 || (c->s.curl_z == 2 && curl_z_auto<R>(c, hod)))) {
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
    const int tz = cz_chunk(c->s.nodes[0], c->s.nodes[1], c->s.nodes[2], nsm > 0 ? nsm : 148, 2 * kCzBlocks);
    switch (c->op_id) {
      case 0: launch_curl_e_z<R, 0>(a, hod, tz, c->s.pdl, c->stream); break;
      case 1: launch_curl_e_z<R, 1>(a, hod, tz, c->s.pdl, c->stream); break;
      case 2: launch_curl_e_z<R, 2>(a, hod, tz, c->s.pdl, c->stream); break;
      case 3: launch_curl_e_z<R, 3>(a, hod, tz, c->s.pdl, c->stream); break;
      case 4: launch_curl_e_z<R, 4>(a, hod, tz, c->s.pdl, c->stream); break;
      case 5: launch_curl_e_z<R, 5>(a, hod, tz, c->s.pdl, c->stream); break;
    }
    return;
  }
  const ColShape sh = col_shape(c->s.curl_block, c->s.col_pairs, c->s.pdl, c->s.xband);
  switch (c->op_id) {
    case 0: launch_curl_e<R, 0>(a, per, hod, sh, c->stream); break;
    case 1: launch_curl_e<R, 1>(a, per, hod, sh, c->stream); break;
    case 2: launch_curl_e<R, 2>(a, per, hod, sh, c->stream); break;
    case 3: launch_curl_e<R, 3>(a, per, hod, sh, c->stream); break;
    case 4: launch_curl_e<R, 4>(a, per, hod, sh, c->stream); break;
    case 5: launch_curl_e<R, 5>(a, per, hod, sh, c->stream); break;
  }
}

template <typename R>
void launch_stage_brick_any(ieq_ctx *c, const StageArgs<R, SoA<R>> &a, const TmaStageMaps &maps) {
  const bool per = c->s.periodic, hall = c->s.hall, hod = diss_kind(c->s) == DISS_HO;
  int *err = c->d_flag + 2;
  switch (c->op_id) {
    case 0: launch_stage_brick<R, 0>(a, maps, err, per, hall, hod, c->stream); break;
    case 1: launch_stage_brick<R, 1>(a, maps, err, per, hall, hod, c->stream); break;
    case 2: launch_stage_brick<R, 2>(a, maps, err, per, hall, hod, c->stream); break;
    case 3: launch_stage_brick<R, 3>(a, maps, err, per, hall, hod, c->stream); break;
    case 4: launch_stage_brick<R, 4>(a, maps, err, per, hall, hod, c->stream); break;
    case 5: launch_stage_brick<R, 5>(a, maps, err, per, hall, hod, c->stream); break;
  }
}

template <typename R>
void launch_curl_brick_any(ieq_ctx *c, SoA<R> b, const R *rho, SoA<R> E, SoA<R> jface, const TmaStageMaps &maps) {
  CurlArgs<R, SoA<R>> a = curl_args<R, SoA<R>>(c, b, rho, E);
  a.jface = jface;
  const bool per = c->s.periodic;
  int *err = c->d_flag + 2;
  switch (c->op_id) {
    case 0: launch_curl_brick<R, 0>(a, maps, err, per, c->stream); break;
    case 1: launch_curl_brick<R, 1>(a, maps, err, per, c->stream); break;
    case 2: launch_curl_brick<R, 2>(a, maps, err, per, c->stream); break;
    case 3: launch_curl_brick<R, 3>(a, maps, err, per, c->stream); break;
    case 4: launch_curl_brick<R, 4>(a, maps, err, per, c->stream); break;
    case 5: launch_curl_brick<R, 5>(a, maps, err, per, c->stream); break;
  }
}

template <typename R, typename F>
CurlArgs<R, F> curl_args(ieq_ctx *c, F b, const R *rho, F out) {
  CurlArgs<R, F> a;
  std::memset(&a, 0, sizeof(a));
  a.m = mesh_of(c);
  a.b = b;
  a.rho = rho;
  a.out = out;
  a.tab = tables<R>(c);
  const SbpOperator &op = c->op;
  const int RI = op.order / 2, C0 = (op.sw - 1) / 2;
  for (int o = -RI; o <= RI; ++o) a.Dint[o + RI] = (R)op.D.at(op.nb, C0 + o);
  for (int ax = 0; ax < 3; ++ax) {
    a.dR[ax] = (R)c->s.d[ax];
    a.inv_d[ax] = (R)(1.0 / c->s.d[ax]);
  }
  return a;
}

template <typename R, typename F>
void launch_curl_any(ieq_ctx *c, F b, const R *rho, F out) {
  const CurlArgs<R, F> a = curl_args<R, F>(c, b, rho, out);
  const dim3 g = grid3(c->s.nodes[0], c->s.nodes[1], c->s.nodes[2]), bl = block3();
  const bool per = c->s.periodic;
  switch (c->op_id) {
    case 0: launch_curl<R, F, 0>(a, per, g, bl, c->stream); break;
    case 1: launch_curl<R, F, 1>(a, per, g, bl, c->stream); break;
    case 2: launch_curl<R, F, 2>(a, per, g, bl, c->stream); break;
    case 3: launch_curl<R, F, 3>(a, per, g, bl, c->stream); break;
    case 4: launch_curl<R, F, 4>(a, per, g, bl, c->stream); break;
    case 5: launch_curl<R, F, 5>(a, per, g, bl, c->stream); break;
  }
}

// ------------------------------------------------------------------------- RK coefficients
// kernel/kernel_time_integrator.cl: 2R schemes 630-1007, 2N schemes 1023-1516
const double kKCL[5][3] = {{0.22502245872571303, -0.17379315208537388, 0.22502245872571303},
                           {0.5440433129514047, -0.1630884872250029, 0.5952726195917439},
                           {0.14456824349399464, -0.5179208398863779, NAN},
                           {0.7866643421983568, -0.19416305717199442, 0.8454958781727144},
                           {0, 0.34866717899927996, NAN}};
const int kKCLsrc[5] = {1, 1, 2, 1, 2};
const double kCFR[6][3] = {{0.17985400977138, 0.10893125722541, 0.28878526699679},
                           {0.14081893152111, 0.13201701492152, 0.38176720366804},
                           {0.08255631629428, 0.38911623225517, 0.71262082069639},
                           {0.65804425034331, -0.59203884581148, 0.69606990893393},
                           {0.31862993413251, 0.47385028714844, 0.83050587987157},
                           {0, 0.48812405426094, NAN}};
const int kCFRsrc[6] = {1, 2, 2, 2, 2, 2};
const double kCK_A[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                         -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double kCK_B[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                         1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                         2277821191437.0 / 14882151754819.0};
const double kCK_C[5] = {1432997174477.0 / 9575080441755.0, 2526269341429.0 / 6820363962896.0,
                         2006345519317.0 / 3224310063776.0, 2802321613138.0 / 2924317926251.0, NAN};
const double kTD_A[8] = {0.0, -0.5534431294501569, 0.01065987570203490, -0.5515812888932000,
                         -1.885790377558741, -5.701295742793264, 2.113903965664793, -0.5339578826675280};
const double kTD_B[8] = {0.08037936882736950, 0.5388497458569843, 0.01974974409031960, 0.09911841297339970,
                         0.7466920411064123, 1.679584245618894, 0.2433728067008188, 0.1422730459001373};
const double kTD_C[8] = {0.08037936882736950, 0.3210064250338430, 0.3408501826604660, 0.3850364824285470,
                         0.5040052477534100, 0.6578977561168540, 0.9484087623348481, NAN};

// ------------------------------------------------------------------------- one reference kernel
enum ArgLayout { L_TI3, L_TI2 };

struct Fields {
  void *b[4] = {nullptr, nullptr, nullptr, nullptr};   // b[1], b[2], b[3]
  void *cb = nullptr, *u = nullptr, *rho = nullptr, *time = nullptr;
};

bool split_args(const char *name, void *const *args, int nargs, Fields &f, int &expect) {
  const bool two = std::strstr(name, "2args") || std::strstr(name, "2_args") ||
                   std::strncmp(name, "CarpenterKennedy2N54", 20) == 0 ||
                   std::strncmp(name, "ToulorgeDesmet2N84F", 19) == 0;
  expect = two ? 6 : 7;
  if (nargs != expect) return false;
  f.b[1] = args[0];
  f.b[2] = args[1];
  int k = 2;
  if (!two) f.b[3] = args[k++];
  f.cb = args[k++];
  f.u = args[k++];
  f.rho = args[k++];
  f.time = args[k++];
  return true;
}

template <typename R>
ieq_status launch_time(ieq_ctx *c, void *time, int kind, R K) {
  k_time<R><<<1, 1, 0, c->stream>>>((R *)time, kind, K, (R)c->s.dt);
  IEQ_LAUNCHED(c);
  return IEQ_OK;
}

template <typename R>
ieq_status reduce(ieq_ctx *c, int kind, const void *va, const void *vb, double *d_total, R *out_real,
                  long long n_zero, int accumulate) {
  ReduceArgs<R> a;
  std::memset(&a, 0, sizeof(a));
  a.kind = kind;
  a.n = (long long)c->n;
  a.nx = c->s.nodes[0];
  a.ny = c->s.nodes[1];
  if (kind == RED_DOT || kind == RED_NORM2_S) {
    a.sa = (const R *)va;
    a.sb = (const R *)vb;
  } else {
    a.va = (const R4<R> *)va;
    a.vb = (const R4<R> *)vb;
  }
  const R *w = (const R *)c->d_wnorm;
  a.wx = w;
  a.wy = w + c->s.nodes[0];
  a.wz = w + c->s.nodes[0] + c->s.nodes[1];
  k_reduce_partials<R><<<kReduceBlocks, 256, 0, c->stream>>>(a, c->d_partials);
  IEQ_LAUNCHED(c);
  k_reduce_final<R><<<1, 256, 0, c->stream>>>(c->d_partials, kReduceBlocks, d_total, out_real, n_zero, accumulate);
  IEQ_LAUNCHED(c);
  return IEQ_OK;
}

template <typename R>
OpArgs<R, R> op_args(ieq_ctx *c) {
  OpArgs<R, R> a;
  std::memset(&a, 0, sizeof(a));
  a.m = mesh_of(c);
  a.op.nb = c->op.nb;
  a.op.sw = c->op.sw;
  a.op.periodic = c->s.periodic;
  a.gx = c->s.nodes[0];
  a.gy = c->s.nodes[1];
  a.gz = c->s.nodes[2];
  const int rows = 2 * c->op.nb + 1;
  a.D = (const R *)c->d_rows_r;
  a.Dadj = (const R *)c->d_rows_r + rows * c->op.sw;
  for (int k = 0; k < 3; ++k) a.dS[k] = (R)c->s.d[k];
  return a;
}

template <typename R>
ieq_status run_one(ieq_ctx *c, const char *name, const uint32_t *g, void *const *args, int nargs) {
  const std::string nm(name);
  const Mesh m = mesh_of(c);
  const dim3 grid = grid3(m.nx, m.ny, m.nz), blk = block3();
  const long long n = (long long)c->n;
  const R DT = (R)c->s.dt;
  auto need = [&](int k) -> ieq_status {
    if (nargs != k) return fail(c, IEQ_ERR_ARG, nm + ": expected " + std::to_string(k) + " arguments");
    for (int i = 0; i < k; ++i)
      if (!args[i]) return fail(c, IEQ_ERR_ARG, nm + ": null argument");
    return IEQ_OK;
  };
  ieq_status st;
  // ---- init / analytic (kernel_init.cl)
  if (nm == "init_b" || nm == "init_u" || nm == "init_rho" || nm == "analytical_b") {
    if ((st = need(nm == "analytical_b" ? 2 : 1)) != IEQ_OK) return st;
    const int kind = nm == "init_b" ? INIT_B : nm == "init_u" ? INIT_U : nm == "init_rho" ? INIT_RHO : ANALYTICAL_B;
    k_init<R><<<grid, blk, 0, c->stream>>>(m, c->s.testcase, kind, (R *)args[0], 0, (R *)args[0],
                                           nargs > 1 ? (const R *)args[1] : nullptr);
    IEQ_LAUNCHED(c);
    return IEQ_OK;
  }
  // ---- reductions (kernel_operator.cl:11-137, kernel_dot_product.cl:47-74)
  if (nm == "norm2" || nm == "norm2_S" || nm == "norm2_diff" || nm == "dot_product") {
    const int k = (nm == "norm2" || nm == "norm2_S") ? 2 : 3;
    if ((st = need(k)) != IEQ_OK) return st;
    const int kind = nm == "norm2" ? RED_NORM2 : nm == "norm2_S" ? RED_NORM2_S : nm == "norm2_diff" ? RED_NORM2_DIFF : RED_DOT;
    return reduce<R>(c, kind, args[0], k == 3 ? args[1] : nullptr, nullptr, (R *)args[k - 1],
                     (long long)c->n_groups, c->s.reduce ? 1 : 0);
  }
  // ---- operators (kernel_operator.cl:145-179)
  if (nm == "calc_div" || nm == "calc_grad" || nm == "calc_curl") {
    if ((st = need(2)) != IEQ_OK) return st;
    if (nm == "calc_curl") {
      launch_curl_any<R, AoS<R>>(c, AoS<R>{(R4<R> *)args[0]}, nullptr, AoS<R>{(R4<R> *)args[1]});
      IEQ_LAUNCHED(c);
      return IEQ_OK;
    }
    OpArgs<R, R> a = op_args<R>(c);
    if (nm == "calc_div") {
      a.v = (const R4<R> *)args[0];
      a.sout = (R *)args[1];
      k_div<R, R><<<grid, blk, 0, c->stream>>>(a);
    } else {
      a.s = (const R *)args[0];
      a.vout = (R4<R> *)args[1];
      k_grad<R, R><<<grid, blk, 0, c->stream>>>(a, 0);
    }
    IEQ_LAUNCHED(c);
    return IEQ_OK;
  }
  // ---- divergence cleaning pieces (kernel_div_cleaning.cl, kernel_CG.cl)
  const int B = c->s.bnodes;
  const int gx = (int)g[0], gy = (int)g[1], gz = (int)g[2];
  if (nm == "calc_div_divcleaning" || nm == "calc_laplace_divcleaning" || nm == "calc_axpy" ||
      nm == "calc_xpay") {
    if ((st = need(nm == "calc_axpy" || nm == "calc_xpay" ? 3 : 2)) != IEQ_OK) return st;
    if (gx + 2 * B > m.nx || gy + 2 * B > m.ny || gz + 2 * B > m.nz)
      return fail(c, IEQ_ERR_SHAPE, nm + ": g_range exceeds NODES - 2*BNODES");
    const dim3 gi = grid3(gx, gy, gz);
    if (nm == "calc_div_divcleaning") {
      OpArgs<R, R> a = op_args<R>(c);
      a.off = B;
      a.gx = gx; a.gy = gy; a.gz = gz;
      a.v = (const R4<R> *)args[0];
      a.sout = (R *)args[1];
      k_div<R, R><<<gi, blk, 0, c->stream>>>(a);
    } else if (nm == "calc_laplace_divcleaning") {
      if (!c->d_lap_r) return fail(c, IEQ_ERR_SETTINGS, "no Laplacian of this form for the operator");
      const SbpRows &L = c->op.lap[c->s.laplace];
      LapArgs<R> a;
      std::memset(&a, 0, sizeof(a));
      a.m = m; a.nb = L.nb; a.w = L.width; a.periodic = c->s.periodic; a.off = B;
      a.gx = gx; a.gy = gy; a.gz = gz;
      a.L = (const R *)c->d_lap_r;
      for (int k = 0; k < 3; ++k) a.dd[k] = (R)c->s.d[k] * (R)c->s.d[k];
      a.in = (const R *)args[0];
      a.out = (R *)args[1];
      k_laplace<R><<<gi, blk, 0, c->stream>>>(a);
    } else {
      k_axpy_interior<R><<<gi, blk, 0, c->stream>>>(m, B, gx, gy, gz, (R *)args[0], (const R *)args[1],
                                                    (const R *)args[2], nm == "calc_xpay", (R)1);
    }
    IEQ_LAUNCHED(c);
    return IEQ_OK;
  }
  if (nm == "projector_divcleaning") {
    if ((st = need(2)) != IEQ_OK) return st;
    OpArgs<R, R> a = op_args<R>(c);
    a.s = (const R *)args[1];
    a.vout = (R4<R> *)args[0];
    k_grad<R, R><<<grid, blk, 0, c->stream>>>(a, c->s.laplace == 2 ? 2 : 1);
    IEQ_LAUNCHED(c);
    return IEQ_OK;
  }
  // ---- time-integrator family (kernel_time_integrator.cl)
  Fields f;
  int expect = 0;
  if (!split_args(name, args, nargs, f, expect))
    return fail(c, IEQ_ERR_ARG, nm + ": expected " + std::to_string(expect) + " arguments");
  for (int i = 0; i < nargs; ++i)
    if (!args[i]) return fail(c, IEQ_ERR_ARG, nm + ": null argument");
  auto vec = [&](int k) { return (R4<R> *)f.b[k]; };
  auto fv = [&](int k) { return AoS<R>{(R4<R> *)f.b[k]}; };
  if (nm == "calc_time_2_args" || nm == "calc_time_3_args") return launch_time<R>(c, f.time, 2, (R)0);
  if (nm == "calc_u_2_args" || nm == "calc_u_3_args") {
    k_init<R><<<grid, blk, 0, c->stream>>>(m, c->s.testcase, CALC_U, (R *)f.u, 0, nullptr, (const R *)f.time);
    IEQ_LAUNCHED(c);
    return IEQ_OK;
  }
  if (nm.rfind("calc_curlB_rho_", 0) == 0) {
    const int k = nm[15] - '0';
    launch_curl_any<R, AoS<R>>(c, fv(k), (const R *)f.rho, AoS<R>{(R4<R> *)f.cb});
    IEQ_LAUNCHED(c);
    return IEQ_OK;
  }
  if (c->s.uibj < 0 || c->s.source < 0 || c->s.ujbi < 0)
    return fail(c, IEQ_ERR_SETTINGS, "no discretization of the volume terms specified (USE_UIBJ_*, USE_SOURCE_*, USE_UJBI_*)");
  StageArgs<R> a = stage_base<R>(c, true);
  a.J = AoS<R>{(R4<R> *)f.cb};
  a.u = AoS<R>{(R4<R> *)f.u};
  a.time = (R *)f.time;
  auto stage = [&](int src, int mode, AoS<R> out) {
    a.bk = fv(src);
    a.mode = mode;
    a.out = out;
    launch_stage_any<R, AoS<R>>(c, a);
  };
  auto pointwise = [&](int mode, R4<R> *P, R4<R> *Q, R4<R> *D, R c1, R c2, int tkind, R tK) -> ieq_status {
    const int nb = (int)((n + 255) / 256);
    k_pointwise<R><<<nb, 256, 0, c->stream>>>(n, mode, P, Q, D, c1, c2, (R *)f.time, tkind, tK, c->d_counter);
    IEQ_LAUNCHED(c);
    return IEQ_OK;
  };
  // SSPRK33 (224-303)
  if (nm == "SSPRK33_1") { a.X = fv(1); a.h = DT; stage(1, EP_X_PLUS_HF, fv(2)); IEQ_LAUNCHED(c); return IEQ_OK; }
  if (nm == "SSPRK33_2a") return launch_time<R>(c, f.time, 1, DT);
  if (nm == "SSPRK33_2b") {
    a.X = fv(1); a.Y = fv(2); a.p = (R)0.75; a.q = (R)0.25; a.h = DT;
    stage(2, EP_PX_QYHF, fv(3)); IEQ_LAUNCHED(c); return IEQ_OK;
  }
  if (nm == "SSPRK33_3a") return launch_time<R>(c, f.time, 1, (R)(0.5 * c->s.dt));
  if (nm == "SSPRK33_3b") {
    a.X = fv(1); a.Y = fv(3); a.p = (R)(1.0 / 3.0); a.q = (R)(2.0 / 3.0); a.h = DT;
    stage(3, EP_PX_QYHF, fv(1)); IEQ_LAUNCHED(c); return IEQ_OK;
  }
  // SSPRK104 (315-621)
  if (nm.rfind("SSPRK104_", 0) == 0) {
    const std::string tag = nm.substr(9);
    const double dt = c->s.dt;
    const R h = (R)(dt / 6.0);
    if (tag == "06") return pointwise(PW_SSP104_06, vec(1), vec(2), vec(3), 0, 0, 1, (R)(dt / 3.0));
    if (tag.size() == 3 && tag[2] == 'a') {
      const std::string s2 = tag.substr(0, 2);
      R K = s2 == "02" ? (R)(dt / 6.0) : s2 == "03" ? (R)(dt / 3.0) : (s2 == "04" || s2 == "08") ? (R)(0.5 * dt)
          : (s2 == "05" || s2 == "09") ? (R)(dt * 2.0 / 3.0) : s2 == "10" ? (R)(dt * 5.0 / 6.0) : (R)dt;
      return launch_time<R>(c, f.time, 1, K);
    }
    const std::string s2 = tag.substr(0, 2);
    if (s2 == "11") {
      a.X = fv(3); a.Y = fv(2); a.p = (R)1; a.q = (R)0.6; a.h = h;
      stage(2, EP_PX_QYHF, fv(1)); IEQ_LAUNCHED(c); return IEQ_OK;
    }
    int src = 0, dst = 0;
    if (s2 == "01") { src = 1; dst = 2; } else if (s2 == "02") { src = 2; dst = 3; }
    else if (s2 == "03") { src = 3; dst = 2; } else if (s2 == "04") { src = 2; dst = 3; }
    else if (s2 == "05") { src = 3; dst = 2; } else if (s2 == "07") { src = 2; dst = 1; }
    else if (s2 == "08") { src = 1; dst = 2; } else if (s2 == "09") { src = 2; dst = 1; }
    else if (s2 == "10") { src = 1; dst = 2; }
    else return fail(c, IEQ_ERR_UNKNOWN_KERNEL, "unknown kernel " + nm);
    a.X = fv(src); a.h = h;
    stage(src, EP_X_PLUS_HF, fv(dst)); IEQ_LAUNCHED(c); return IEQ_OK;
  }
  // 2R schemes (630-1007): the third field is db
  const bool kcl = nm.rfind("KennedyCarpenterLewis2R54C_", 0) == 0;
  const bool cfr = nm.rfind("CalvoFrancoRandez2R64_", 0) == 0;
  if (kcl || cfr) {
    const std::string tag = nm.substr(kcl ? 27 : 22);
    const int sidx = tag[0] - '1';
    const int last = kcl ? 4 : 5;
    if (sidx < 0 || sidx > last) return fail(c, IEQ_ERR_UNKNOWN_KERNEL, "unknown kernel " + nm);
    const double (*tab)[3] = kcl ? kKCL : kCFR;
    const int *src = kcl ? kKCLsrc : kCFRsrc;
    if (sidx == last && tag.size() == 1) {
      // b1 = b1 + coef_B*(REAL)(DT) * DB(b2)
      a.X = fv(1); a.h = (R)tab[sidx][1] * DT;
      stage(2, EP_X_PLUS_HF, fv(1)); IEQ_LAUNCHED(c); return IEQ_OK;
    }
    if (tag.size() != 2) return fail(c, IEQ_ERR_UNKNOWN_KERNEL, "unknown kernel " + nm);
    if (tag[1] == 'a') {
      a.h = DT;
      stage(src[sidx], EP_HF, fv(3)); IEQ_LAUNCHED(c); return IEQ_OK;
    }
    const R A = (R)tab[sidx][0], Bc = (R)tab[sidx][1];
    const double C = tab[sidx][2];
    const int tkind = std::isnan(C) ? 0 : 1;
    const R tK = tkind ? (R)C * DT : (R)0;
    if (kcl) {
      // stages 1,3: b1 = b1 + A db; b2 = b1 + B db.  stages 2,4: b2 = b2 + A db; b1 = b2 + B db
      if (sidx == 0 || sidx == 2) return pointwise(PW_2R, vec(1), vec(2), vec(3), A, Bc, tkind, tK);
      return pointwise(PW_2R, vec(2), vec(1), vec(3), A, Bc, tkind, tK);
    }
    // CFR: b1 = b1 + B db; b2 = b1 + A db
    return pointwise(PW_2R, vec(1), vec(2), vec(3), Bc, A, tkind, tK);
  }
  // 2N schemes (1023-1516)
  const bool ck = nm.rfind("CarpenterKennedy2N54_", 0) == 0;
  const bool td = nm.rfind("ToulorgeDesmet2N84F_", 0) == 0;
  if (ck || td) {
    const std::string tag = nm.substr(ck ? 21 : 20);
    const int ns = ck ? 5 : 8;
    const int sidx = tag[0] - '1';
    if (tag.size() != 2 || sidx < 0 || sidx >= ns) return fail(c, IEQ_ERR_UNKNOWN_KERNEL, "unknown kernel " + nm);
    const double *Atab = ck ? kCK_A : kTD_A, *Btab = ck ? kCK_B : kTD_B, *Ctab = ck ? kCK_C : kTD_C;
    if (tag[1] == 'a') {
      a.h = DT;
      if (sidx == 0) stage(1, EP_HF, fv(2));
      else { a.X = fv(2); a.A = (R)Atab[sidx]; stage(1, EP_AX_HF, fv(2)); }
      IEQ_LAUNCHED(c);
      return IEQ_OK;
    }
    const double C = Ctab[sidx];
    const int tkind = std::isnan(C) ? 0 : 1;
    return pointwise(PW_AXPY, vec(1), vec(2), nullptr, (R)Btab[sidx], 0, tkind, tkind ? (R)C * DT : (R)0);
  }
  return fail(c, IEQ_ERR_UNKNOWN_KERNEL, "unknown kernel " + nm);
}

ieq_status run_one_any(ieq_ctx *c, const char *name, const uint32_t *g, void *const *args, int nargs) {
  if (!c) return IEQ_ERR_ARG;
  if (!name) return fail(c, IEQ_ERR_ARG, "null kernel name");
  IEQ_CUDA(c, cudaSetDevice(c->device));
  return c->s.real_float ? run_one<float>(c, name, g, args, nargs) : run_one<double>(c, name, g, args, nargs);
}

}  // namespace

// ---- helpers of the adjoint (adjoint.cu)
#include "adjoint_args.inc"

namespace ieq {
// the coefficients of the 2N low-storage schemes (CarpenterKennedy2N54: ck = true;
// ToulorgeDesmet2N84F) for adjoint.cu: A, B, C per stage and the stage count
void rk2n_coefficients(bool ck, const double **A, const double **B, const double **C, int *stages) {
  *A = ck ? kCK_A : kTD_A;
  *B = ck ? kCK_B : kTD_B;
  *C = ck ? kCK_C : kTD_C;
  *stages = ck ? 5 : 8;
}
// pieces of a context that adjoint.cu needs to build its kernel arguments
void adj_context(ieq_ctx *c, Mesh &m, const Tables<double> *&tab, double w[6], double inv_d[3], double two_inv_d[3],
                 double sat_s[3]) {
  m = mesh_of(c);
  tab = tables<double>(c);
  const Forms f = flux_forms(c->s);
  for (int k = 0; k < 6; ++k) w[k] = f.w[k];
  for (int a = 0; a < 3; ++a) {
    inv_d[a] = 1.0 / c->s.d[a];
    two_inv_d[a] = 2.0 / c->s.d[a];
    sat_s[a] = c->op.minv[0] / c->s.d[a];
  }
}
}  // namespace ieq

// default NDRange of every reference kernel (used by the typed entry points)
static ieq_status ieq_run_one_default(ieq_ctx *ctx, const char *name, void *const *args, int nargs) {
  if (!ctx) return IEQ_ERR_ARG;
  uint32_t g[3] = {(uint32_t)ctx->s.nodes[0], (uint32_t)ctx->s.nodes[1], (uint32_t)ctx->s.nodes[2]};
  const std::string nm(name);
  if (nm == "calc_div_divcleaning" || nm == "calc_laplace_divcleaning" || nm == "calc_axpy" || nm == "calc_xpay")
    for (int a = 0; a < 3; ++a) g[a] = (uint32_t)(ctx->s.nodes[a] - 2 * ctx->s.bnodes);
  return run_one_any(ctx, name, g, args, nargs);
}

#include "kernel_abi.inc"

// ============================================================================ C ABI
extern "C" {

const char *ieq_status_string(ieq_status s) {
  switch (s) {
    case IEQ_OK: return "ok";
    case IEQ_ERR_SETTINGS: return "invalid settings";
    case IEQ_ERR_SHAPE: return "invalid shape";
    case IEQ_ERR_CUDA: return "CUDA error";
    case IEQ_ERR_NAN: return "non-finite result";
    case IEQ_ERR_NOT_CONVERGED: return "not converged";
    case IEQ_ERR_TIMEOUT: return "timeout";
    case IEQ_ERR_UNKNOWN_KERNEL: return "unknown kernel";
    case IEQ_ERR_ARG: return "invalid argument";
  }
  return "?";
}

static thread_local std::string g_create_error;

ieq_status ieq_create(ieq_ctx **out, const char *settings, const char *const *paths, int n_paths, int device) {
  if (!out) return IEQ_ERR_ARG;
  *out = nullptr;
  ieq_ctx *c = new ieq_ctx();
  c->device = device;
  std::string err;
  if (!parse_settings(settings, paths, n_paths, c->s, err) || !load_operator(c->s.order, c->s.extended, c->op, err)) {
    g_create_error = err;
    delete c;
    return IEQ_ERR_SETTINGS;
  }
  c->op_id = (c->s.order / 2 - 1) + (c->s.extended ? 3 : 0);
  for (int a = 0; a < 3; ++a) {
    if (!c->s.periodic && c->s.nodes[a] < 2 * c->op.nb) {
      g_create_error = "NODES per direction must be at least 2*NUM_BOUNDS = " + std::to_string(2 * c->op.nb);
      delete c;
      return IEQ_ERR_SHAPE;
    }
    // periodic neighbours wrap once: the stencil must not reach around the box twice
    if (c->s.periodic && c->s.nodes[a] < c->op.sw) {
      g_create_error = "periodic NODES per direction must be at least STENCIL_WIDTH = " + std::to_string(c->op.sw);
      delete c;
      return IEQ_ERR_SHAPE;
    }
  }
  c->n = (size_t)c->s.nodes[0] * c->s.nodes[1] * c->s.nodes[2];
  c->n_pad = (c->n + c->s.w_size - 1) / c->s.w_size * c->s.w_size;   // initialize.m:43-44
  c->n_groups = c->n_pad / c->s.w_size;
  ieq_status st = IEQ_OK;
  auto cuda = [&](cudaError_t e, const char *what) {
    if (e != cudaSuccess && st == IEQ_OK) {
      g_create_error = std::string(what) + ": " + cudaGetErrorString(e);
      st = IEQ_ERR_CUDA;
    }
  };
  cuda(cudaSetDevice(device), "cudaSetDevice");
  if (st == IEQ_OK) cuda(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  // one partial per block of the finest grid the one-pass reductions launch (128 threads over
  // 32 x 2 x 2 nodes), three per block for the diagnostics
  {
    const long long bx = (c->s.nodes[0] + 31) / 32, by = (c->s.nodes[1] + 1) / 2, bz = (c->s.nodes[2] + 1) / 2;
    c->partials_cap = std::max<long long>(kMaxPartials, 3 * bx * by * bz);
  }
  if (st == IEQ_OK) cuda(cudaMalloc(&c->d_partials, c->partials_cap * sizeof(double)), "cudaMalloc");
  if (st == IEQ_OK) cuda(cudaMalloc(&c->d_partials2, c->partials_cap * sizeof(double)), "cudaMalloc");
  if (st == IEQ_OK) cuda(cudaMalloc(&c->d_total, 64 * sizeof(double)), "cudaMalloc");
  if (st == IEQ_OK) cuda(cudaMalloc(&c->d_counter, 64 * sizeof(unsigned)), "cudaMalloc");
  if (st == IEQ_OK) cuda(cudaMemset(c->d_counter, 0, 64 * sizeof(unsigned)), "cudaMemset");
  if (st == IEQ_OK) cuda(cudaMalloc(&c->d_flag, 64 * sizeof(int)), "cudaMalloc");
  if (st == IEQ_OK) cuda(cudaMemset(c->d_flag, 0, 64 * sizeof(int)), "cudaMemset");
  if (st == IEQ_OK) cuda(cudaMalloc(&c->d_cg, sizeof(CgState)), "cudaMalloc");
  if (st == IEQ_OK) cuda(cudaEventCreate(&c->ev0), "cudaEventCreate");
  if (st == IEQ_OK) cuda(cudaEventCreate(&c->ev1), "cudaEventCreate");
  if (st == IEQ_OK) {
    st = c->s.real_float ? upload_tables<float>(c) : upload_tables<double>(c);
    if (st != IEQ_OK) g_create_error = c->err;
  }
  if (st != IEQ_OK) {
    ieq_destroy(c);
    return st;
  }
  *out = c;
  return IEQ_OK;
}

void ieq_destroy(ieq_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  ieq::free_brick_maps(c);
  for (auto &kv : c->graphs) {
    if (kv.second.exec1) cudaGraphExecDestroy(kv.second.exec1);
    if (kv.second.exec2) cudaGraphExecDestroy(kv.second.exec2);
  }
  for (auto &kv : c->clean_graphs)
    if (kv.second) cudaGraphExecDestroy(kv.second);
  if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
  for (void *p : c->allocs) cudaFree(p);
  for (void *p : c->adj_bufs) cudaFree(p);
  if (c->adj_time) cudaFree(c->adj_time);
  void *own[] = {c->d_tables, c->d_rows_r, c->d_rows_d, c->d_lap_r, c->d_lap_d, c->d_wnorm, c->d_partials,
                 c->d_partials2, c->d_total, c->d_counter, c->d_flag, c->d_cg, c->d_cg_vec, c->d_cg_hist,
                 c->d_lap_s,
                 c->d_pingpong, c->d_soa};
  for (void *p : own)
    if (p) cudaFree(p);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char *ieq_last_error(const ieq_ctx *c) { return c ? c->err.c_str() : g_create_error.c_str(); }

size_t ieq_num_nodes(const ieq_ctx *c) { return c ? c->n : 0; }
size_t ieq_num_nodes_pad(const ieq_ctx *c) { return c ? c->n_pad : 0; }
size_t ieq_num_groups(const ieq_ctx *c) { return c ? c->n_groups : 0; }
int ieq_real_size(const ieq_ctx *c) { return c ? (c->s.real_float ? 4 : 8) : 0; }
void *ieq_stream(ieq_ctx *c) { return c ? (void *)c->stream : nullptr; }

ieq_status ieq_alloc(ieq_ctx *c, size_t bytes, void **p) {
  if (!c || !p) return IEQ_ERR_ARG;
  IEQ_CUDA(c, cudaSetDevice(c->device));
  IEQ_CUDA(c, cudaMalloc(p, bytes));
  IEQ_CUDA(c, cudaMemsetAsync(*p, 0, bytes, c->stream));
  c->allocs.insert(*p);
  return IEQ_OK;
}

ieq_status ieq_free(ieq_ctx *c, void *p) {
  if (!c) return IEQ_ERR_ARG;
  if (!c->allocs.count(p)) return fail(c, IEQ_ERR_ARG, "pointer not allocated by this context");
  IEQ_CUDA(c, cudaStreamSynchronize(c->stream));
  c->allocs.erase(p);
  IEQ_CUDA(c, cudaFree(p));
  return IEQ_OK;
}

ieq_status ieq_upload(ieq_ctx *c, void *dst, const void *src, size_t bytes) {
  if (!c || !dst || !src) return IEQ_ERR_ARG;
  IEQ_CUDA(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
  IEQ_CUDA(c, cudaStreamSynchronize(c->stream));
  return IEQ_OK;
}

ieq_status ieq_download(ieq_ctx *c, void *dst, const void *src, size_t bytes) {
  if (!c || !dst || !src) return IEQ_ERR_ARG;
  IEQ_CUDA(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
  IEQ_CUDA(c, cudaStreamSynchronize(c->stream));
  return IEQ_OK;
}

ieq_status ieq_memset(ieq_ctx *c, void *dst, int value, size_t bytes) {
  if (!c || !dst) return IEQ_ERR_ARG;
  IEQ_CUDA(c, cudaMemsetAsync(dst, value, bytes, c->stream));
  return IEQ_OK;
}

ieq_status ieq_synchronize(ieq_ctx *c) {
  if (!c) return IEQ_ERR_ARG;
  IEQ_CUDA(c, cudaStreamSynchronize(c->stream));
  return IEQ_OK;
}

ieq_status ieq_run_kernels(ieq_ctx *c, const char *const *names, int n_names, const uint32_t g_range[3],
                           void *const *args, int n_args, double *elapsed) {
  if (!c || !names || !g_range) return IEQ_ERR_ARG;
  IEQ_CUDA(c, cudaSetDevice(c->device));
  if (elapsed) IEQ_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  for (int i = 0; i < n_names; ++i) {
    const ieq_status st = run_one_any(c, names[i], g_range, args, n_args);
    if (st != IEQ_OK) return st;
  }
  if (elapsed) {
    IEQ_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    IEQ_CUDA(c, cudaEventSynchronize(c->ev1));
    float ms = 0;
    IEQ_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    *elapsed = ms * 1e-3;
  }
  return IEQ_OK;
}

ieq_status ieq_run_kernels_host(ieq_ctx *c, const char *const *names, int n_names, const uint32_t g_range[3],
                                void *const *host_args, const size_t *arg_bytes, int n_args, double *elapsed) {
  if (!c || !host_args || !arg_bytes || n_args < 0 || n_args > 16) return IEQ_ERR_ARG;
  IEQ_CUDA(c, cudaSetDevice(c->device));
  void *dev[16] = {nullptr};
  ieq_status st = IEQ_OK;
  for (int i = 0; i < n_args && st == IEQ_OK; ++i) {
    if (cudaMallocAsync(&dev[i], arg_bytes[i], c->stream) != cudaSuccess) st = fail(c, IEQ_ERR_CUDA, "cudaMallocAsync");
    else if (cudaMemcpyAsync(dev[i], host_args[i], arg_bytes[i], cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
      st = fail(c, IEQ_ERR_CUDA, "cudaMemcpyAsync H2D");
  }
  if (st == IEQ_OK) st = ieq_run_kernels(c, names, n_names, g_range, dev, n_args, elapsed);
  for (int i = 0; i < n_args; ++i) {
    if (!dev[i]) continue;
    if (st == IEQ_OK && cudaMemcpyAsync(host_args[i], dev[i], arg_bytes[i], cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
      st = fail(c, IEQ_ERR_CUDA, "cudaMemcpyAsync D2H");
    cudaFreeAsync(dev[i], c->stream);
  }
  if (cudaStreamSynchronize(c->stream) != cudaSuccess && st == IEQ_OK) st = fail(c, IEQ_ERR_CUDA, "sync");
  return st;
}

}  // extern "C"

#include "api_fused.inc"
