// hall_circular_wave.h -- TEST INFRASTRUCTURE ONLY: a testcase plug-in for the CPU oracle,
// written for this project in the reference's testcase-header interface.
//
// Circularly polarised whistler wave of the Hall induction equation with zero ion
// velocity and unit density on the periodic box [0, 2 pi]^3:
//   B = (a sin(z - omega t), a cos(z - omega t), 1),  a = 0.1,  omega = k^2 B_z / rho = 1.
// curl B = (B_x, B_y, 0) here, and -curl((curl B) x B) = dB/dt holds exactly.

inline REAL4 b_analytical(uint ix, uint iy, uint iz, REAL time) {
  REAL z = (REAL)ZMIN + iz * (REAL)DZ;
  REAL ph = z - time;
  return (REAL4){(REAL)(0.1) * sin(ph), (REAL)(0.1) * cos(ph), (REAL)(1), (REAL)(0)};
}

inline REAL4 b_init(uint ix, uint iy, uint iz) { return b_analytical(ix, iy, iz, (REAL)(0)); }

inline REAL4 b_boundary(uint ix, uint iy, uint iz, REAL time) {
  return b_analytical(ix, iy, iz, time);
}

inline REAL4 u_init(uint ix, uint iy, uint iz) { return (REAL4){0, 0, 0, 0}; }

inline REAL4 u_analytical(uint ix, uint iy, uint iz, REAL time) { return u_init(ix, iy, iz); }

inline REAL rho_init(uint ix, uint iy, uint iz) { return (REAL)(1); }
