// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY (CPU oracle; never part of the product).
//
// Compiles the reference's OpenCL C sources *in place* (through clshim.hpp) and
// exposes them behind a tiny C ABI so that tests, golden-vector generation and the
// CPU baseline can run the reference's own arithmetic on the host cores.
//
// The include order mirrors the kernel_path_list that the reference host assembles in
// matlab/+induction_eq/compute_numerical_solution_setup.m:57-122:
//   order header, utils.h, testcase header, kernel_init.cl, SBP_operator.cl,
//   kernel_operator.cl, kernel_div_cleaning.cl, kernel_CG.cl,
//   [artificial_dissipation.h, artificial_dissipation.cl], induction_Eq_volume.cl,
//   induction_Eq_surface.cl, kernel_dot_product.cl, kernel_time_integrator.cl
// The discrete switches (order header, testcase, USE_* flags, REAL) are -D flags
// chosen by oracle/refimpl.py; the mesh and time-step values are runtime globals.
#include "clshim.hpp"

#include <cstring>
#include <string>
#include <omp.h>

uint g_NODES_X = 8, g_NODES_Y = 8, g_NODES_Z = 8;
double g_DX = 1, g_DY = 1, g_DZ = 1, g_XMIN = 0, g_XMAX = 1, g_YMIN = 0, g_YMAX = 1, g_ZMIN = 0,
       g_ZMAX = 1;
double g_DT = 0, g_HO_DISSIPATION_FACTOR = 1, g_MP2MIN = 1, g_MP2MAX = 10, g_CMIN = 1, g_CMAX = 10;
uint g_BNODES = 1;
double g_TC_OMEGA = 1.0;
thread_local uint t_gid[3];

#define IEQ_STR2(x) #x
#define IEQ_STR(x) IEQ_STR2(x)

#include IEQ_STR(IEQ_ORDER_HEADER)
#include "utils.h"
#include IEQ_STR(IEQ_TESTCASE_HEADER)
#include "kernel_init.cl"
#include "SBP_operator.cl"
#include "kernel_operator.cl"
#include "kernel_div_cleaning.cl"
#include "kernel_CG.cl"
#ifdef USE_ARTIFICIAL_DISSIPATION
#include "artificial_dissipation.h"
#include "artificial_dissipation.cl"
#endif
#include "induction_Eq_volume.cl"
#include "induction_Eq_surface.cl"
#include "kernel_dot_product.cl"
#include "kernel_time_integrator.cl"

typedef void (*kfn_t)(void **);
struct kentry {
  const char *name;
  kfn_t fn;
  int nargs;
};

#define V4(i) ((REAL4 *)a[i])
#define S(i) ((REAL *)a[i])
#define K3F(n) {#n, [](void **a) { n(V4(0), V4(1), V4(2), V4(3), V4(4), S(5), S(6)); }, 7}
#define K2F(n) {#n, [](void **a) { n(V4(0), V4(1), V4(2), V4(3), S(4), S(5)); }, 6}

static const kentry g_kernels[] = {
    {"init_b", [](void **a) { init_b(V4(0)); }, 1},
    {"init_u", [](void **a) { init_u(V4(0)); }, 1},
    {"init_rho", [](void **a) { init_rho(S(0)); }, 1},
    {"analytical_b", [](void **a) { analytical_b(V4(0), S(1)); }, 2},
    {"norm2", [](void **a) { norm2(V4(0), S(1)); }, 2},
    {"norm2_diff", [](void **a) { norm2_diff(V4(0), V4(1), S(2)); }, 3},
    {"norm2_S", [](void **a) { norm2_S(S(0), S(1)); }, 2},
    {"calc_div", [](void **a) { calc_div(V4(0), S(1)); }, 2},
    {"calc_curl", [](void **a) { calc_curl(V4(0), V4(1)); }, 2},
    {"calc_grad", [](void **a) { calc_grad(S(0), V4(1)); }, 2},
    {"calc_div_divcleaning", [](void **a) { calc_div_divcleaning(V4(0), S(1)); }, 2},
    {"calc_laplace_divcleaning", [](void **a) { calc_laplace_divcleaning(S(0), S(1)); }, 2},
    {"projector_divcleaning", [](void **a) { projector_divcleaning(V4(0), S(1)); }, 2},
    {"calc_axpy", [](void **a) { calc_axpy(S(0), S(1), S(2)); }, 3},
    {"calc_xpay", [](void **a) { calc_xpay(S(0), S(1), S(2)); }, 3},
    {"dot_product", [](void **a) { dot_product(S(0), S(1), S(2)); }, 3},
    K2F(calc_time_2_args),
    K3F(calc_time_3_args),
    K2F(calc_u_2_args),
    K3F(calc_u_3_args),
    K2F(calc_curlB_rho_1_2args),
    K2F(calc_curlB_rho_2_2args),
    K3F(calc_curlB_rho_1_3args),
    K3F(calc_curlB_rho_2_3args),
    K3F(calc_curlB_rho_3_3args),
    K3F(SSPRK33_1),
    K3F(SSPRK33_2a),
    K3F(SSPRK33_2b),
    K3F(SSPRK33_3a),
    K3F(SSPRK33_3b),
    K3F(SSPRK104_01),
    K3F(SSPRK104_02a),
    K3F(SSPRK104_02b),
    K3F(SSPRK104_03a),
    K3F(SSPRK104_03b),
    K3F(SSPRK104_04a),
    K3F(SSPRK104_04b),
    K3F(SSPRK104_05a),
    K3F(SSPRK104_05b),
    K3F(SSPRK104_06),
    K3F(SSPRK104_07),
    K3F(SSPRK104_08a),
    K3F(SSPRK104_08b),
    K3F(SSPRK104_09a),
    K3F(SSPRK104_09b),
    K3F(SSPRK104_10a),
    K3F(SSPRK104_10b),
    K3F(SSPRK104_11a),
    K3F(SSPRK104_11b),
    K3F(KennedyCarpenterLewis2R54C_1a),
    K3F(KennedyCarpenterLewis2R54C_1b),
    K3F(KennedyCarpenterLewis2R54C_2a),
    K3F(KennedyCarpenterLewis2R54C_2b),
    K3F(KennedyCarpenterLewis2R54C_3a),
    K3F(KennedyCarpenterLewis2R54C_3b),
    K3F(KennedyCarpenterLewis2R54C_4a),
    K3F(KennedyCarpenterLewis2R54C_4b),
    K3F(KennedyCarpenterLewis2R54C_5),
    K3F(CalvoFrancoRandez2R64_1a),
    K3F(CalvoFrancoRandez2R64_1b),
    K3F(CalvoFrancoRandez2R64_2a),
    K3F(CalvoFrancoRandez2R64_2b),
    K3F(CalvoFrancoRandez2R64_3a),
    K3F(CalvoFrancoRandez2R64_3b),
    K3F(CalvoFrancoRandez2R64_4a),
    K3F(CalvoFrancoRandez2R64_4b),
    K3F(CalvoFrancoRandez2R64_5a),
    K3F(CalvoFrancoRandez2R64_5b),
    K3F(CalvoFrancoRandez2R64_6),
    K2F(CarpenterKennedy2N54_1a),
    K2F(CarpenterKennedy2N54_1b),
    K2F(CarpenterKennedy2N54_2a),
    K2F(CarpenterKennedy2N54_2b),
    K2F(CarpenterKennedy2N54_3a),
    K2F(CarpenterKennedy2N54_3b),
    K2F(CarpenterKennedy2N54_4a),
    K2F(CarpenterKennedy2N54_4b),
    K2F(CarpenterKennedy2N54_5a),
    K2F(CarpenterKennedy2N54_5b),
    K2F(ToulorgeDesmet2N84F_1a),
    K2F(ToulorgeDesmet2N84F_1b),
    K2F(ToulorgeDesmet2N84F_2a),
    K2F(ToulorgeDesmet2N84F_2b),
    K2F(ToulorgeDesmet2N84F_3a),
    K2F(ToulorgeDesmet2N84F_3b),
    K2F(ToulorgeDesmet2N84F_4a),
    K2F(ToulorgeDesmet2N84F_4b),
    K2F(ToulorgeDesmet2N84F_5a),
    K2F(ToulorgeDesmet2N84F_5b),
    K2F(ToulorgeDesmet2N84F_6a),
    K2F(ToulorgeDesmet2N84F_6b),
    K2F(ToulorgeDesmet2N84F_7a),
    K2F(ToulorgeDesmet2N84F_7b),
    K2F(ToulorgeDesmet2N84F_8a),
    K2F(ToulorgeDesmet2N84F_8b),
};

extern "C" {

// params: DX DY DZ XMIN XMAX YMIN YMAX ZMIN ZMAX DT HO_DISSIPATION_FACTOR MP2MIN MP2MAX CMIN CMAX TC_OMEGA
int ref_configure(const unsigned *nodes, const double *p, unsigned bnodes) {
  g_NODES_X = nodes[0];
  g_NODES_Y = nodes[1];
  g_NODES_Z = nodes[2];
  g_DX = p[0]; g_DY = p[1]; g_DZ = p[2];
  g_XMIN = p[3]; g_XMAX = p[4]; g_YMIN = p[5]; g_YMAX = p[6]; g_ZMIN = p[7]; g_ZMAX = p[8];
  g_DT = p[9];
  g_HO_DISSIPATION_FACTOR = p[10];
  g_MP2MIN = p[11]; g_MP2MAX = p[12]; g_CMIN = p[13]; g_CMAX = p[14];
  g_TC_OMEGA = p[15];
  g_BNODES = bnodes;
  return 0;
}

int ref_real_size(void) { return (int)sizeof(REAL); }

int ref_num_kernels(void) { return (int)(sizeof(g_kernels) / sizeof(g_kernels[0])); }

const char *ref_kernel_name(int i) { return g_kernels[i].name; }

// Runs one kernel over the NDRange grange[0] x grange[1] x grange[2] (work-group size 1),
// with `nthreads` OpenMP threads over the flattened range.  Returns 0, or -1 for an
// unknown name, -2 for a wrong argument count.
int ref_run(const char *name, const unsigned *grange, void **args, int nargs, int nthreads) {
  const kentry *k = nullptr;
  for (const kentry &e : g_kernels)
    if (std::strcmp(e.name, name) == 0) k = &e;
  if (!k) return -1;
  if (k->nargs != nargs) return -2;
  const long g0 = grange[0], g1 = grange[1], g2 = grange[2];
  const long total = g0 * g1 * g2;
  kfn_t fn = k->fn;
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
  for (long i = 0; i < total; ++i) {
    t_gid[0] = (uint)(i % g0);
    t_gid[1] = (uint)((i / g0) % g1);
    t_gid[2] = (uint)(i / (g0 * g1));
    fn(args);
  }
  return 0;
}
}
