// ieq_host.h -- host-side context of the InductionEq library (internal).
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include "../../include/inductioneq.h"

namespace ieq {

// The reference's -D settings (generate_settings.m) in runtime form.
struct Settings {
  int nodes[3] = {0, 0, 0};
  double d[3] = {0, 0, 0};
  double xmin[3] = {0, 0, 0}, xmax[3] = {0, 0, 0};
  bool have_d[3] = {false, false, false};
  double dt = 0.0;
  bool real_float = false;
  int w_size = 1;
  // operator header
  int order = 0;
  bool extended = false;
  // flux forms: 0 CENTRAL, 1 SPLIT, 2 PRODUCT, 3 ZERO; -1 unset
  int uibj = -1, source = -1, ujbi = -1;
  bool hall = false, periodic = false;
  bool dissipation = false;
  int diss_form = 0;   // 0 none, 1 high order, 2 first order, 3 adaptive
  double hod_factor = 1.0, mp2min = 0, mp2max = 0, cmin = 0, cmax = 0;
  int laplace = 0;     // 0 WS_D0, 1 NS_D0, 2 WS_LN
  int bnodes = -1;
  bool reduce = false;
  int testcase = -1;
  double omega = 1.0;
  std::string integrator;
  bool variable_u = false;
  // kernels of the fused time stepping (IEQ_STAGE_KERNEL): 0 AUTO (the column kernels,
  // measured fastest on B200), 1 COLUMN, 2 NODE (the per-node J-based kernels), 3 BRICK
  // (the TMA brick kernels for the u = 0 stages where their rules hold, else COLUMN),
  // 4 LIST (no fusion: the reference's kernel list of each step on the caller's fields),
  // 5 ZMARCH (the one-pass Hall stage of stage_z.cuh wherever it can run, else COLUMN; AUTO
  // takes it on grids of at least kZmarchAutoNodes nodes, which measured slower: never)
  int stage_kernel = 0;
  // thread-block shapes of the column stage kernel (IEQ_COL_BLOCK=XxYxZ) and of the curl
  // kernel (IEQ_CURL_BLOCK); X * Y * Z = 128, all zero for the default 32x4x1
  int col_block[3] = {0, 0, 0};
  int curl_block[3] = {0, 0, 0};
  // IEQ_COL_PAIRS=0: the column kernels keep one node per thread; 1 (default): two
  // x-adjacent nodes per thread where measured faster and the field layout allows it (FP32
  // Hall kernels: four on grids of >= 2^20 nodes); 4: FP32 Hall kernels four on every grid
  int col_pairs = 1;
  // IEQ_PDL=0: launch the column kernels without programmatic dependent launch
  bool pdl = true;
  // IEQ_XBAND: boxes run their x boundary columns in a launch of their own -- 0 never, 1
  // (default) where measured faster (the band at most a tenth of the row), 2 wherever possible
  int xband = 1;
  // IEQ_ZMARCH_TZ: z planes per CTA of the one-pass Hall stage (0: chosen per grid)
  int zmarch_tz = 0;
  // IEQ_Z_OFFSET / IEQ_NZ_GLOBAL: this grid is a z slab of a decomposed periodic grid of
  // IEQ_NZ_GLOBAL planes whose plane 0 is global plane IEQ_Z_OFFSET (testcase coordinates
  // are the global grid's); 0 / 0: the grid is the whole domain
  int zoff = 0, nzg = 0;
  // IEQ_CG_PASS_A: the CG's pass A as the 2.5D kernel (2, the default) or the per-node gather (1)
  int cg_passes = 2;
  // IEQ_CG_LOOP=HOST (profiling): the CG iterations as max_iterations launches in sequence
  // instead of a graph loop node (kernels inside a loop node are invisible to the profiler)
  bool cg_host_loop = false;
  // IEQ_HODP: Hall + high-order dissipation -- 1 the curl kernel forms the dissipation sum and
  // the stage kernel reads it; 0 the stage kernel gathers the dissipation rows itself
  int hodp = 1;
  // IEQ_ADJOINT_PROGRAM: 1 reverses SSPRK33 and the 2N schemes through the generic register
  // program of the step as well (the other integrators always use it)
  int adjoint_program = 0;
  // IEQ_CURL_Z: the curl kernel of periodic Hall stages as the 2.5D z march (stage_z.cuh):
  // 0 never, 1 always, 2 (default) where measured faster (api.cu: curl_z_auto)
  int curl_z = 2;
};

// parse helpers (settings.cpp)
bool parse_settings(const char *settings, const char *const *paths, int n_paths, Settings &out,
                    std::string &err);
int integrator_id(const std::string &name);

struct SbpRows {
  int nb = 0, width = 0;
  std::vector<double> rows;   // (2nb+1) x width
  double at(int r, int c) const { return rows[(size_t)r * width + c]; }
};
struct SbpOperator {
  int order = 0, nb = 0, sw = 0, w_hod = 0;
  SbpRows D, Dadj, DHO, lap[3];
  std::vector<double> minv;
  bool has_lap[3] = {false, false, false};
};
bool load_operator(int order, bool extended, SbpOperator &op, std::string &err);

// One step of a time integrator as a register program (R0 = b1, the solution; R1 = b2;
// R2 = b3 or db): stage s evaluates K = h F(R[src]) at time t0 + t (src < 0: no evaluation),
// then runs its assignments R[dst] = a[0] R0 + a[1] R1 + a[2] R2 + k K in order.  Built from
// the coefficient tables of the fused time step (rk_step_program); the discrete adjoint
// reverses it.
struct RkAssign {
  int dst;
  double a[3];
  double k;
};
struct RkStage {
  int src;
  double h, t;
  std::vector<RkAssign> as;
};
struct RkProgram {
  std::vector<RkStage> stages;
  int evaluations = 0;   // stages with src >= 0 (the stage inputs the adjoint keeps)
};
void rk_step_program(int integ, double dt, RkProgram &p);

}  // namespace ieq

struct ieq_ctx {
  ieq::Settings s;
  ieq::SbpOperator op;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  size_t n = 0, n_pad = 0, n_groups = 0;
  int op_id = 0;
  // device tables
  void *d_tables = nullptr;        // Tables<REAL>
  void *d_rows_r = nullptr;        // D, Dadj rows in REAL  [2][rows*sw]
  double *d_rows_d = nullptr;      // D, Dadj rows in FP64
  void *d_lap_r = nullptr;         // Laplacian rows in REAL
  double *d_lap_d = nullptr;       // Laplacian rows in FP64
  void *d_wnorm = nullptr;         // per-axis norm weights in REAL (nx + ny + nz)
  // scratch
  double *d_partials = nullptr;    // reduction partials
  double *d_partials2 = nullptr;
  long long partials_cap = 0;      // entries of d_partials and d_partials2
  double *d_total = nullptr;       // reduction totals
  unsigned *d_counter = nullptr;   // last-block tickets
  int *d_flag = nullptr;
  void *d_cg = nullptr;            // CgState
  double *d_cg_vec = nullptr;      // FP64 CG vectors: div, phi, r, u, u', lap (6 x n_pad)
  double *d_cg_hist = nullptr;
  double *d_lap_s = nullptr;       // the CG Laplacian's rows divided by DX^2, DY^2, DZ^2
  int cg_hist_len = 0;
  void *d_pingpong = nullptr;      // (unused)
  void *d_soa = nullptr;           // structure-of-arrays state of the fused time stepping
  std::vector<void *> adj_bufs;    // vector fields of the checkpointed adjoint, kept for later calls
  double *adj_time = nullptr;      // its two time pairs
  void *brick_maps = nullptr;      // tensor maps of that state for the TMA brick kernels (host)
  std::set<void *> allocs;
  // fused time-step graphs keyed by the argument pointers
  struct GraphEntry {
    cudaGraphExec_t exec1 = nullptr, exec2 = nullptr;
  };
  std::map<std::vector<uintptr_t>, GraphEntry> graphs;
  // cleaning graphs (div B, CG loop as a conditional WHILE node, projection) keyed by the
  // field and the loop parameters; a second stream on which the loop body is captured
  std::map<std::vector<uintptr_t>, cudaGraphExec_t> clean_graphs;
  cudaStream_t aux_stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // ieq_profile_step: labels of the step's launches, and a gate that lets only the
  // launch with index gate_target through (-1: all launches, -2: none)
  std::vector<std::string> *labels = nullptr;
  int gate_target = -1;
  int gate_count = 0;
  // ieq_stages_*: the fused step enqueued stage by stage.  gate_target == -3 lets only the
  // launches of stage gate_stage through (stage_count: the stage being enqueued); stage_trace
  // receives the state buffers at the start of every stage (b1, b1', b2, b2', last input)
  int gate_stage = -1, stage_count = 0;
  std::vector<std::array<void *, 5>> *stage_trace = nullptr;
  struct Stages {
    bool active = false;
    int integ = -1, conv = 1, count = 0, last = -1, saved_diss = 0;
    std::array<void *, 5> step{};              // buffers at the start of the current step
    std::vector<std::array<void *, 5>> trace;  // buffers at the start of every stage of a step
    std::array<void *, 5> end{};               // buffers at the end of a step
  } stages;
};
