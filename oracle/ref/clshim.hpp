// clshim.hpp -- TEST INFRASTRUCTURE ONLY (part of the CPU oracle, never shipped).
//
// Just enough of the OpenCL C 1.x surface for the reference's kernel sources
// (kernel/*.cl, include/*.h of IANW-Projects/InductionEq) to compile unmodified
// as C++ with g++, so that the reference's own arithmetic can run on the host
// cores.  The reference sources are compiled in place from the reference tree;
// nothing of them is copied here.
//
// Semantics kept:
//   * `kernel`, `global`, `local` vanish; `constant` becomes `const`.
//   * REAL4 is a 4-lane vector with .x/.y/.z/.w and an lvalue `.xyz` swizzle;
//     arithmetic is component-wise, scalars broadcast (OpenCL vector rules).
//   * get_global_id() is thread local (set by the NDRange executor); every
//     work-group has size 1, so barrier() is a no-op and the reduction kernels
//     emit one partial per work item -- legal OpenCL semantics.
//   * Mesh sizes, DX/DY/DZ, XMIN..ZMAX, DT, BNODES and the dissipation
//     parameters are runtime globals instead of -D literals; every use in the
//     reference is an arithmetic expression, so the values computed are the
//     same as with the literals (g++ is run with -ffp-contract=off).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstdlib>

#ifndef REAL
#define REAL double
#endif

typedef unsigned int uint;
typedef unsigned long ulong_t;

#define kernel
#define global
#define local
#define constant const
#define CLK_LOCAL_MEM_FENCE 0
static inline void barrier(int) {}

// ---------------------------------------------------------------- runtime "defines"
extern uint g_NODES_X, g_NODES_Y, g_NODES_Z;
extern double g_DX, g_DY, g_DZ, g_XMIN, g_XMAX, g_YMIN, g_YMAX, g_ZMIN, g_ZMAX;
extern double g_DT, g_HO_DISSIPATION_FACTOR, g_MP2MIN, g_MP2MAX, g_CMIN, g_CMAX;
extern uint g_BNODES;
// testcase parameters of the testcase headers written for the oracle
extern double g_TC_OMEGA;

#define NODES_X g_NODES_X
#define NODES_Y g_NODES_Y
#define NODES_Z g_NODES_Z
#define DX g_DX
#define DY g_DY
#define DZ g_DZ
#define XMIN g_XMIN
#define XMAX g_XMAX
#define YMIN g_YMIN
#define YMAX g_YMAX
#define ZMIN g_ZMIN
#define ZMAX g_ZMAX
#define DT g_DT
#define BNODES g_BNODES
#define HO_DISSIPATION_FACTOR g_HO_DISSIPATION_FACTOR
#define MP2MIN g_MP2MIN
#define MP2MAX g_MP2MAX
#define CMIN g_CMIN
#define CMAX g_CMAX
#define W_SIZE 1

// ---------------------------------------------------------------- work-item ids
extern thread_local uint t_gid[3];
static inline uint get_global_id(int d) { return t_gid[d]; }
static inline uint get_local_id(int) { return 0; }
static inline uint get_local_size(int) { return 1; }
static inline uint get_group_id(int d) { return t_gid[d]; }

// ---------------------------------------------------------------- vector types
struct REAL3 {
  REAL x, y, z;
};
union REAL4 {
  struct {
    REAL x, y, z, w;
  };
  REAL3 xyz;
};
union uint4 {
  struct {
    uint x, y, z, w;
  };
};

static inline REAL4 mk4(REAL a, REAL b, REAL c, REAL d) {
  REAL4 r;
  r.x = a; r.y = b; r.z = c; r.w = d;
  return r;
}
static inline REAL3 mk3(REAL a, REAL b, REAL c) {
  REAL3 r;
  r.x = a; r.y = b; r.z = c;
  return r;
}

#define V4OP(op)                                                                          \
  static inline REAL4 operator op(const REAL4 &a, const REAL4 &b) {                       \
    return mk4(a.x op b.x, a.y op b.y, a.z op b.z, a.w op b.w);                           \
  }                                                                                       \
  static inline REAL4 operator op(const REAL4 &a, double s) {                             \
    REAL t = (REAL)s;                                                                     \
    return mk4(a.x op t, a.y op t, a.z op t, a.w op t);                                   \
  }                                                                                       \
  static inline REAL4 operator op(double s, const REAL4 &a) {                             \
    REAL t = (REAL)s;                                                                     \
    return mk4(t op a.x, t op a.y, t op a.z, t op a.w);                                   \
  }                                                                                       \
  static inline REAL3 operator op(const REAL3 &a, const REAL3 &b) {                       \
    return mk3(a.x op b.x, a.y op b.y, a.z op b.z);                                       \
  }                                                                                       \
  static inline REAL3 operator op(const REAL3 &a, double s) {                             \
    REAL t = (REAL)s;                                                                     \
    return mk3(a.x op t, a.y op t, a.z op t);                                             \
  }                                                                                       \
  static inline REAL3 operator op(double s, const REAL3 &a) {                             \
    REAL t = (REAL)s;                                                                     \
    return mk3(t op a.x, t op a.y, t op a.z);                                             \
  }
V4OP(+)
V4OP(-)
V4OP(*)
V4OP(/)
#undef V4OP

static inline REAL4 operator-(const REAL4 &a) { return mk4(-a.x, -a.y, -a.z, -a.w); }
static inline REAL3 operator-(const REAL3 &a) { return mk3(-a.x, -a.y, -a.z); }

// ---------------------------------------------------------------- built-ins
static inline REAL4 fabs(const REAL4 &a) {
  return mk4(std::fabs(a.x), std::fabs(a.y), std::fabs(a.z), std::fabs(a.w));
}
static inline REAL4 fmax(const REAL4 &a, const REAL4 &b) {
  return mk4(std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z), std::fmax(a.w, b.w));
}
static inline REAL dot(const REAL4 &a, const REAL4 &b) {
  return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
}
static inline double pown(double x, int n) {
  double r = 1.0;
  for (int i = 0; i < (n < 0 ? -n : n); ++i) r *= x;
  return n < 0 ? 1.0 / r : r;
}
static inline double sinpi(double x) { return std::sin(M_PI * x); }
static inline double cospi(double x) { return std::cos(M_PI * x); }
using std::abs;
// OpenCL's abs() of an unsigned argument returns it unchanged (kernel code relies on
// k*k of the wrapped value, which equals the square of the true distance mod 2^32).
static inline uint abs(uint x) { return x; }
using std::cos;
using std::exp;
using std::fabs;
using std::fmax;
using std::sin;
using std::sqrt;

// atomic_cmpxchg is only referenced by the REDUCE path, which the oracle does not use;
// these single-threaded versions let the sources compile.
static inline uint atomic_cmpxchg(volatile uint *p, uint cmp, uint val) {
  uint old = *p;
  if (old == cmp) *p = val;
  return old;
}
static inline unsigned long atomic_cmpxchg(volatile unsigned long *p, unsigned long cmp,
                                           unsigned long val) {
  unsigned long old = *p;
  if (old == cmp) *p = val;
  return old;
}
