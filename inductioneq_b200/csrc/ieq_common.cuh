// ieq_common.cuh -- types, operator traits, coefficient tables and testcase plug-ins
// shared by the sm_100a kernels of the InductionEq time-stepping library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ieq {

// --------------------------------------------------------------------------- layout
// REAL4 array-of-structs at the boundary (x, y, z, w with w = 0): one 32-byte (FP64) or
// 16-byte (FP32) record per node, index ix + NX*(iy + NY*iz).
template <typename R>
struct alignas(4 * sizeof(R)) R4 {
  R x, y, z, w;
};
template <typename R>
struct V3 {
  R x, y, z;
};

template <typename R>
__device__ __forceinline__ V3<R> ld3(const R4<R> *p) {
  // 16-byte + 8-byte (FP64) loads: the w lane is never read
  if constexpr (sizeof(R) == 8) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
    const double c = __ldg(reinterpret_cast<const double *>(p) + 2);
    return {(R)a.x, (R)a.y, (R)c};
  } else {
    const float4 a = __ldg(reinterpret_cast<const float4 *>(p));
    return {(R)a.x, (R)a.y, (R)a.z};
  }
}
template <typename R>
__device__ __forceinline__ V3<R> ld3_plain(const R4<R> *p) {
  // for fields written earlier in the same kernel launch (no read-only path)
  if constexpr (sizeof(R) == 8) {
    const double2 a = *reinterpret_cast<const double2 *>(p);
    const double c = reinterpret_cast<const double *>(p)[2];
    return {(R)a.x, (R)a.y, (R)c};
  } else {
    const float4 a = *reinterpret_cast<const float4 *>(p);
    return {(R)a.x, (R)a.y, (R)a.z};
  }
}
template <typename R>
__device__ __forceinline__ void st3(R4<R> *p, V3<R> v) {
  if constexpr (sizeof(R) == 8) {
    reinterpret_cast<double2 *>(p)[0] = make_double2(v.x, v.y);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v.z, 0.0);
  } else {
    *reinterpret_cast<float4 *>(p) = make_float4(v.x, v.y, v.z, 0.f);
  }
}

// --------------------------------------------------------------------------- operators
// Operator ids: 0..2 classical order 2/4/6, 3..5 extended order 2/4/6.
// NB = boundary rows per side, SW = derivative stencil width, WH = width of the
// dissipation factor D_HO, RI = interior radius (ORDER/2) of both D and D_HO^T D_HO.
template <int OP>
struct Op;
template <> struct Op<0> { static constexpr int NB = 1, SW = 3, WH = 2, RI = 1, ORDER = 2; };
template <> struct Op<1> { static constexpr int NB = 4, SW = 7, WH = 3, RI = 2, ORDER = 4; };
template <> struct Op<2> { static constexpr int NB = 6, SW = 11, WH = 4, RI = 3, ORDER = 6; };
template <> struct Op<3> { static constexpr int NB = 3, SW = 5, WH = 2, RI = 1, ORDER = 2; };
template <> struct Op<4> { static constexpr int NB = 6, SW = 11, WH = 3, RI = 2, ORDER = 4; };
template <> struct Op<5> { static constexpr int NB = 8, SW = 15, WH = 4, RI = 3, ORDER = 6; };

constexpr int MAX_ROWS = 17;   // 2*NB+1 of the widest operator (6th extended)
constexpr int MAX_SW = 15;
constexpr int MAX_HW = 7;      // 2*WH-1
constexpr int MAX_LROWS = 23;  // Laplacian rows (6th extended, wide stencil)
constexpr int MAX_LW = 21;

// Coefficient tables of one operator in device memory, in the precision R of the state.
template <typename R>
struct Tables {
  R D[MAX_ROWS][MAX_SW];        // first derivative rows, column c <-> offset c-(SW-1)/2
  R Dadj[MAX_ROWS][MAX_SW];     // adjoint rows (least-norm projection)
  R H[MAX_ROWS][MAX_HW];        // dissipation rows sum_s,i M^-1 D_HO[r][s] D_HO[c][i] (-1)^(p/2+1)
  R DHO[MAX_ROWS][4];           // raw D_HO rows (first-order/adaptive dissipation)
  R Minv[MAX_ROWS];
};

// Laplacian rows for divergence cleaning in the CG precision S.
template <typename S>
struct LapTable {
  int nb, w;
  S L[MAX_LROWS][MAX_LW];
};

// row index of node i along an axis of n nodes (include/utils.h:172-201): the boundary
// closures occupy rows 0..nb-1 (left) and nb+1..2nb (right); interior nodes use row nb.
__device__ __forceinline__ int sbp_row(int i, int n, int nb) {
  int bound = 0;
  if (i < nb) bound -= nb - i;
  if (n - 1 - i < nb) bound += nb - (n - 1 - i);
  return nb + bound;
}

// --------------------------------------------------------------------------- testcases
// Built-in testcase plug-ins (the reference's include/<testcase>.h compile-time headers
// become runtime ids).  Each returns b_analytical / b_boundary / u_analytical / rho.
enum Testcase : int {
  TC_ROTATION_2D = 0,
  TC_ROTATION_3D = 1,
  TC_HALL_PERIODIC = 2,
  TC_HALL_TRAVELLING_WAVE = 3,
  TC_CONFINED_DOMAIN = 4,
  TC_ALFVEN_PERIODIC_2D = 5,
  TC_ROTATION_GAUSSIAN = 6,
  TC_HALL_CIRCULAR_WAVE = 7,
};

struct Mesh {
  int nx, ny, nz;
  double xmin[3];
  double d[3];       // DX, DY, DZ
  double omega;      // rotation rate of TC_ROTATION_GAUSSIAN
  // a z slab of a decomposed periodic grid: local plane iz is global plane iz + zoff (modulo
  // nzg, the global plane count) -- coordinates are those of the global grid; nzg = 0: the
  // grid is the whole domain
  int zoff, nzg;
};

template <typename R>
__device__ __forceinline__ void coords(const Mesh &m, int ix, int iy, int iz, R &x, R &y, R &z) {
  int gz = iz;
  if (m.nzg > 0) {
    gz = (iz + m.zoff) % m.nzg;
    gz += gz < 0 ? m.nzg : 0;
  }
  x = (R)m.xmin[0] + (R)ix * (R)m.d[0];
  y = (R)m.xmin[1] + (R)iy * (R)m.d[1];
  z = (R)m.xmin[2] + (R)gz * (R)m.d[2];
}

// include/rotation_2D.h:7-25
template <typename R>
__device__ V3<R> tc_rotation_2d_b(R x, R y, R t) {
  R s = sin(t), c = cos(t);
  R xx = c * x + s * y, yy = -s * x + c * y;
  R fac = exp((R)-20 * ((xx - (R)0.5) * (xx - (R)0.5) + yy * yy));
  R bx0 = (R)-4 * yy * fac, by0 = ((R)4 * xx - (R)2) * fac;
  return {c * bx0 - s * by0, s * bx0 + c * by0, (R)0};
}

// include/rotation_3D.h:7-34
template <typename R>
__device__ V3<R> tc_rotation_3d_b(R x, R y, R z, R t) {
  const R sqrt3 = (R)1.7320508075688772;
  R s = sin(t), c = cos(t);
  R xx = ((1 + 2 * c) * x + (1 - c + sqrt3 * s) * y + (1 - c - sqrt3 * s) * z) / (R)3.0;
  R yy = ((1 - c - sqrt3 * s) * x + (1 + 2 * c) * y + (1 - c + sqrt3 * s) * z) / (R)3.0;
  R zz = ((1 - c + sqrt3 * s) * x + (1 - c - sqrt3 * s) * y + (1 + 2 * c) * z) / (R)3.0;
  R alpha = exp(-(R)(5.0 / 3.0) * (3 - 2 * (3 + sqrt3) * xx + 12 * xx * xx - 2 * (-3 + sqrt3) * yy +
                                    12 * yy * yy + 4 * sqrt3 * zz + 12 * zz * zz));
  R b0x = alpha * (3 - sqrt3 - 4 * sqrt3 * yy + 4 * sqrt3 * zz) / (R)48.0;
  R b0y = alpha * (-3 - sqrt3 + 4 * sqrt3 * xx - 4 * sqrt3 * zz) / (R)48.0;
  R b0z = alpha * (1 - 2 * xx + 2 * yy) / (8 * sqrt3);
  return {((1 + 2 * c) * b0x + (1 - c - sqrt3 * s) * b0y + (1 - c + sqrt3 * s) * b0z) / (R)3.0,
          ((1 - c + sqrt3 * s) * b0x + (1 + 2 * c) * b0y + (1 - c - sqrt3 * s) * b0z) / (R)3.0,
          ((1 - c - sqrt3 * s) * b0x + (1 - c + sqrt3 * s) * b0y + (1 + 2 * c) * b0z) / (R)3.0};
}

// include/hall_periodic.h:3-34 (b) and 75-92 (u).  u is a sum of one-dimensional terms,
// u1 = c(y) + s(z), u2 = c(z) + s(x), u3 = c(x) + s(y) with c(q) = a cos(k q + al k t n),
// s(q) = a sin(k q + al k t n)
template <typename R>
__device__ __forceinline__ void tc_hall_periodic_terms(R q, R t, R &c, R &s) {
  const R n = (R)0.5773502691896258, a = (R)1, al = (R)0.5;
  const R k = (R)(1.0 - al * al) / al;
  c = a * cos(k * q + al * k * t * n);
  s = a * sin(k * q + al * k * t * n);
}
template <typename R>
__device__ V3<R> tc_hall_periodic_u(R x, R y, R z, R t) {
  R cx, sx, cy, sy, cz, sz;
  tc_hall_periodic_terms(x, t, cx, sx);
  tc_hall_periodic_terms(y, t, cy, sy);
  tc_hall_periodic_terms(z, t, cz, sz);
  return {cy + sz, cz + sx, cx + sy};
}

// include/hall_travelling_wave.h:3-30 (b) and 66-82 (u)
template <typename R>
__device__ V3<R> tc_hall_travelling(R z, R t, bool velocity) {
  const R B0 = 1, Bz = 1, ux = 1, uy = 1, uz = (R)0.1, k = 1, om = 1;
  R xi = k * z - om * t;
  R Om = ((k * uz - om) * (k * uz - om) - k * k * Bz * Bz) / (Bz * (k * uz - om) * k * k);
  if (velocity) {
    R fac = k * Bz / (k * uz - om);
    return {fac * B0 * cos(Om * xi) + ux, fac * B0 * sin(Om * xi) + uy, uz};
  }
  return {B0 * cos(Om * xi), B0 * sin(Om * xi), Bz};
}

// include/confined_domain.h:7-24 (b and u are the same field)
template <typename R>
__device__ V3<R> tc_confined(R x, R y, R z) {
  R sx = sinpi(x), cx = cospi(x), sy = sinpi(y), cy = cospi(y), sz = sinpi(z), cz = cospi(z);
  return {sx * cy * cz, cx * sy * cz, -2 * cx * cy * sz};
}

// include/alfven_periodic_2D.h:3-28 (b) and 49-66 (u)
template <typename R>
__device__ V3<R> tc_alfven(R x, R y, R t, bool velocity) {
  const R A = (R)0.1, al = (R)0.5235987755982988;
  R ca = cos(al), sa = sin(al);
  R phi = (R)6.283185307179586 * (x * ca + y * sa + t);
  R cp = cos(phi), sp = sin(phi);
  if (velocity) return {-A * sa * sp, A * ca * sp, A * cp};
  return {ca - A * sa * sp, sa - A * ca * sp, A * cp};
}

// rotation of a divergence-free Gaussian bump (this project's testcase; width 0.1,
// max |B0| = 1, rotation rate omega): B(x,t) = R(omega t) B0(R(-omega t) x)
template <typename R>
__device__ V3<R> tc_rotation_gaussian_b(R x, R y, R t, R om) {
  const R w2 = (R)0.01;
  const R amp = (R)(0.1 * 1.6487212707001282 / 1.4142135623730951);
  R th = om * t;
  R s = sin(th), c = cos(th);
  R xr = c * x + s * y - (R)0.5, yr = -s * x + c * y;
  R g = amp * exp(-(xr * xr + yr * yr) / w2);
  R b0x = -(R)2 * yr / w2 * g, b0y = (R)2 * xr / w2 * g;
  return {c * b0x - s * b0y, s * b0x + c * b0y, (R)0};
}

// whistler wave of the Hall equation with u = 0, rho = 1 (this project's testcase)
template <typename R>
__device__ V3<R> tc_hall_circular_b(R z, R t) {
  R ph = z - t;
  return {(R)0.1 * sin(ph), (R)0.1 * cos(ph), (R)1};
}

template <typename R>
__device__ V3<R> b_analytical(int tc, const Mesh &m, int ix, int iy, int iz, R t) {
  R x, y, z;
  coords<R>(m, ix, iy, iz, x, y, z);
  switch (tc) {
    case TC_ROTATION_2D: return tc_rotation_2d_b<R>(x, y, t);
    case TC_ROTATION_3D: return tc_rotation_3d_b<R>(x, y, z, t);
    case TC_HALL_PERIODIC: {
      V3<R> u = tc_hall_periodic_u<R>(x, y, z, t);
      const R n = (R)0.5773502691896258, al = (R)0.5;
      return {al * u.x + n, al * u.y + n, al * u.z + n};
    }
    case TC_HALL_TRAVELLING_WAVE: return tc_hall_travelling<R>(z, t, false);
    case TC_CONFINED_DOMAIN: return tc_confined<R>(x, y, z);
    case TC_ALFVEN_PERIODIC_2D: return tc_alfven<R>(x, y, t, false);
    case TC_ROTATION_GAUSSIAN: return tc_rotation_gaussian_b<R>(x, y, t, (R)m.omega);
    case TC_HALL_CIRCULAR_WAVE: return tc_hall_circular_b<R>(z, t);
  }
  return {0, 0, 0};
}

template <typename R>
__device__ V3<R> b_boundary(int tc, const Mesh &m, int ix, int iy, int iz, R t) {
  if (tc == TC_HALL_PERIODIC || tc == TC_HALL_TRAVELLING_WAVE) return {0, 0, 0};
  return b_analytical<R>(tc, m, ix, iy, iz, t);
}

template <typename R>
__device__ V3<R> u_analytical(int tc, const Mesh &m, int ix, int iy, int iz, R t) {
  R x, y, z;
  coords<R>(m, ix, iy, iz, x, y, z);
  switch (tc) {
    case TC_ROTATION_2D: return {-y, x, (R)0};
    case TC_ROTATION_3D: {
      const R sqrt3 = (R)1.7320508075688772;
      return {(z - y) / sqrt3, (x - z) / sqrt3, (y - x) / sqrt3};
    }
    case TC_HALL_PERIODIC: return tc_hall_periodic_u<R>(x, y, z, t);
    case TC_HALL_TRAVELLING_WAVE: return tc_hall_travelling<R>(z, t, true);
    case TC_CONFINED_DOMAIN: return tc_confined<R>(x, y, z);
    case TC_ALFVEN_PERIODIC_2D: return tc_alfven<R>(x, y, t, true);
    case TC_ROTATION_GAUSSIAN: return {-(R)m.omega * y, (R)m.omega * x, (R)0};
    case TC_HALL_CIRCULAR_WAVE: return {0, 0, 0};
  }
  return {0, 0, 0};
}

}  // namespace ieq
