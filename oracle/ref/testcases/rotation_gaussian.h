// rotation_gaussian.h -- TEST INFRASTRUCTURE ONLY: a testcase plug-in for the CPU oracle,
// written for this project in the reference's testcase-header interface
// (b_analytical / b_init / b_boundary / u_init / u_analytical / rho_init, the interface of
// include/rotation_2D.h in the reference).
//
// Rigid rotation u = omega*(-y, x, 0) of a divergence-free Gaussian bump
//   B0 = curl(psi e_z),  psi = A exp(-((x-1/2)^2 + y^2) / w^2),  w = 0.1,
// with A chosen so that max |B0| = 1.  The exact solution is the rotated field
//   B(x, t) = R(omega t) B0(R(-omega t) x).
// omega is the runtime parameter g_TC_OMEGA (1 for the single-solve workload).

inline REAL4 b_analytical(uint ix, uint iy, uint iz, REAL time) {
  REAL x = (REAL)XMIN + ix * (REAL)DX;
  REAL y = (REAL)YMIN + iy * (REAL)DY;
  REAL w2 = (REAL)(0.01);
  REAL amp = (REAL)(0.1 * 1.6487212707001282 / 1.4142135623730951);
  REAL th = (REAL)g_TC_OMEGA * time;
  REAL s = sin(th);
  REAL c = cos(th);
  REAL xr = c * x + s * y - (REAL)(0.5);
  REAL yr = -s * x + c * y;
  REAL g = amp * exp(-(xr * xr + yr * yr) / w2);
  REAL b0x = -(REAL)(2) * yr / w2 * g;
  REAL b0y = (REAL)(2) * xr / w2 * g;
  return (REAL4){c * b0x - s * b0y, s * b0x + c * b0y, (REAL)(0), (REAL)(0)};
}

inline REAL4 b_init(uint ix, uint iy, uint iz) { return b_analytical(ix, iy, iz, (REAL)(0)); }

inline REAL4 b_boundary(uint ix, uint iy, uint iz, REAL time) {
  return b_analytical(ix, iy, iz, time);
}

inline REAL4 u_init(uint ix, uint iy, uint iz) {
  REAL x = (REAL)XMIN + ix * (REAL)DX;
  REAL y = (REAL)YMIN + iy * (REAL)DY;
  REAL om = (REAL)g_TC_OMEGA;
  return (REAL4){-om * y, om * x, (REAL)(0), (REAL)(0)};
}

inline REAL4 u_analytical(uint ix, uint iy, uint iz, REAL time) { return u_init(ix, iy, iz); }

inline REAL rho_init(uint ix, uint iy, uint iz) { return (REAL)(1); }
