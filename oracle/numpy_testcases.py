"""TEST INFRASTRUCTURE ONLY -- numpy restatement of the testcase plug-ins.

Each function restates one testcase header's b_analytical / u_analytical / rho_init
(reference include/<testcase>.h, cited per function) on the whole grid, in the header's
order of operations.  ``evaluate(oracle, name, what, t)`` returns a grid-shaped array:
``what`` is "b" (b_analytical(t)), "init" (b_init), "boundary" (b_boundary(t)), "u"
(u_analytical(t)), "u_init" or "rho".  Two testcases of this project are included:
"rotation_gaussian" and "hall_circular_wave" (oracle/ref/testcases/*.h).
"""
from __future__ import annotations

import math

import numpy as np


def _zeros_like_grid(o):
    return np.zeros((o.NZ, o.NY, o.NX), dtype=o.T)


def _bc(o, *arrs):
    sh = (o.NZ, o.NY, o.NX)
    return [np.broadcast_to(a, sh) for a in arrs]


def rotation_2D(o, what, t):
    # include/rotation_2D.h:7-25 (b), 46-57 (u), 62-64 (rho)
    T = o.T
    x, y, z = o.coords()
    if what in ("u", "u_init"):
        return o._v4(*_bc(o, -y + 0 * x, x + 0 * y, _zeros_like_grid(o)))
    t = T(t)
    s, c = np.sin(t), np.cos(t)
    xx = c * x + s * y
    yy = -s * x + c * y
    fac = np.exp(-20 * ((xx - T(0.5)) * (xx - T(0.5)) + yy * yy))
    bx0 = -4 * yy * fac
    by0 = (4 * xx - 2) * fac
    return o._v4(*_bc(o, c * bx0 - s * by0, s * bx0 + c * by0, _zeros_like_grid(o)))


def rotation_3D(o, what, t):
    # include/rotation_3D.h:7-34 (b), 57-69 (u)
    T = o.T
    x, y, z = o.coords()
    sqrt3 = T(math.sqrt(3.0))
    if what in ("u", "u_init"):
        return o._v4(*_bc(o, (z - y) / sqrt3, (x - z) / sqrt3, (y - x) / sqrt3))
    t = T(t)
    s, c = np.sin(t), np.cos(t)
    xx = ((1 + 2 * c) * x + (1 - c + sqrt3 * s) * y + (1 - c - sqrt3 * s) * z) / T(3.0)
    yy = ((1 - c - sqrt3 * s) * x + (1 + 2 * c) * y + (1 - c + sqrt3 * s) * z) / T(3.0)
    zz = ((1 - c + sqrt3 * s) * x + (1 - c - sqrt3 * s) * y + (1 + 2 * c) * z) / T(3.0)
    alpha = np.exp(-T(5.0 / 3.0) * (3 - 2 * (3 + sqrt3) * xx + 12 * xx * xx
                                    - 2 * (-3 + sqrt3) * yy + 12 * yy * yy
                                    + 4 * sqrt3 * zz + 12 * zz * zz))
    b0x = alpha * (3 - sqrt3 - 4 * sqrt3 * yy + 4 * sqrt3 * zz) / T(48.0)
    b0y = alpha * (-3 - sqrt3 + 4 * sqrt3 * xx - 4 * sqrt3 * zz) / T(48.0)
    b0z = alpha * (1 - 2 * xx + 2 * yy) / (8 * sqrt3)
    bx = ((1 + 2 * c) * b0x + (1 - c - sqrt3 * s) * b0y + (1 - c + sqrt3 * s) * b0z) / T(3.0)
    by = ((1 - c + sqrt3 * s) * b0x + (1 + 2 * c) * b0y + (1 - c - sqrt3 * s) * b0z) / T(3.0)
    bz = ((1 - c - sqrt3 * s) * b0x + (1 - c + sqrt3 * s) * b0y + (1 + 2 * c) * b0z) / T(3.0)
    return o._v4(*_bc(o, bx, by, bz))


def hall_periodic(o, what, t):
    # include/hall_periodic.h:3-9 (constants), 15-34 (b), 75-92 (u)
    T = o.T
    x, y, z = o.coords()
    n1 = n2 = n3 = T(0.5773502691896258)
    a = b = c = T(1.0)
    alpha = T(0.5)
    k = T(1.0 - alpha * alpha) / alpha
    if what == "u_init":
        what, t = "u", 0.0
    if what == "init":
        what, t = "b", 0.0
    t = T(t)
    u1 = a * np.cos(k * y + alpha * k * t * n2) + b * np.sin(k * z + alpha * k * t * n3)
    u2 = b * np.cos(k * z + alpha * k * t * n3) + c * np.sin(k * x + alpha * k * t * n1)
    u3 = c * np.cos(k * x + alpha * k * t * n1) + a * np.sin(k * y + alpha * k * t * n2)
    if what == "u":
        return o._v4(*_bc(o, u1, u2, u3))
    if what == "boundary":
        return o._v4(*_bc(o, *(3 * [_zeros_like_grid(o)])))
    return o._v4(*_bc(o, alpha * u1 + n1, alpha * u2 + n2, alpha * u3 + n3))


def hall_travelling_wave(o, what, t):
    # include/hall_travelling_wave.h:3-9 (constants), 15-30 (b), 66-82 (u)
    T = o.T
    x, y, z = o.coords()
    B0, Bz, ux, uy, uz, k, om = (T(1.0), T(1.0), T(1.0), T(1.0), T(0.1), T(1.0), T(1.0))
    if what == "u_init":
        what, t = "u", 0.0
    if what == "init":
        what, t = "b", 0.0
    if what == "boundary":
        return o._v4(*_bc(o, *(3 * [_zeros_like_grid(o)])))
    t = T(t)
    xi = k * z - om * t
    Om = ((k * uz - om) * (k * uz - om) - k * k * Bz * Bz) / (Bz * (k * uz - om) * k * k)
    if what == "u":
        fac = k * Bz / (k * uz - om)
        return o._v4(*_bc(o, fac * B0 * np.cos(Om * xi) + ux, fac * B0 * np.sin(Om * xi) + uy,
                          uz + 0 * xi))
    return o._v4(*_bc(o, B0 * np.cos(Om * xi), B0 * np.sin(Om * xi), Bz + 0 * xi))


def confined_domain(o, what, t):
    # include/confined_domain.h:7-24 (b = u, time independent), 45-62 (u)
    x, y, z = o.coords()
    sx, cx = np.sin(np.pi * x), np.cos(np.pi * x)
    sy, cy = np.sin(np.pi * y), np.cos(np.pi * y)
    sz, cz = np.sin(np.pi * z), np.cos(np.pi * z)
    return o._v4(*_bc(o, sx * cy * cz, cx * sy * cz, -2 * cx * cy * sz))


def alfven_periodic_2D(o, what, t):
    # include/alfven_periodic_2D.h:3-4 (constants), 10-28 (b), 49-66 (u)
    T = o.T
    x, y, z = o.coords()
    A = T(0.1)
    al = T(0.5235987755982988)
    ca, sa = np.cos(al), np.sin(al)
    if what in ("init", "u_init"):
        t = 0.0
    t = T(t)
    phi = T(6.283185307179586) * (x * ca + y * sa + t)
    cp, sp = np.cos(phi), np.sin(phi)
    if what in ("u", "u_init"):
        return o._v4(*_bc(o, -A * sa * sp, A * ca * sp, A * cp))
    return o._v4(*_bc(o, ca - A * sa * sp, sa - A * ca * sp, A * cp))


def rotation_gaussian(o, what, t):
    # oracle/ref/testcases/rotation_gaussian.h
    T = o.T
    x, y, z = o.coords()
    om = T(o.cfg.tc_omega)
    if what in ("u", "u_init"):
        return o._v4(*_bc(o, -om * y + 0 * x, om * x + 0 * y, _zeros_like_grid(o)))
    if what == "init":
        t = 0.0
    w2 = T(0.01)
    amp = T(0.1 * 1.6487212707001282 / 1.4142135623730951)
    th = om * T(t)
    s, c = np.sin(th), np.cos(th)
    xr = c * x + s * y - T(0.5)
    yr = -s * x + c * y
    g = amp * np.exp(-(xr * xr + yr * yr) / w2)
    b0x = -T(2) * yr / w2 * g
    b0y = T(2) * xr / w2 * g
    return o._v4(*_bc(o, c * b0x - s * b0y, s * b0x + c * b0y, _zeros_like_grid(o)))


def hall_circular_wave(o, what, t):
    # oracle/ref/testcases/hall_circular_wave.h
    T = o.T
    x, y, z = o.coords()
    if what in ("u", "u_init"):
        return o._v4(*_bc(o, *(3 * [_zeros_like_grid(o)])))
    if what == "init":
        t = 0.0
    ph = z - T(t)
    return o._v4(*_bc(o, T(0.1) * np.sin(ph), T(0.1) * np.cos(ph), T(1) + 0 * ph))


TESTCASES = {f.__name__: f for f in (rotation_2D, rotation_3D, hall_periodic, hall_travelling_wave,
                                      confined_domain, alfven_periodic_2D, rotation_gaussian,
                                      hall_circular_wave)}


def evaluate(o, name: str, what: str, t):
    if what == "rho":
        return np.ones((o.NZ, o.NY, o.NX), dtype=o.T)
    f = TESTCASES[name]
    if what == "init":
        return f(o, "init", 0.0)
    if what == "boundary" and name in ("rotation_2D", "rotation_3D", "confined_domain",
                                       "alfven_periodic_2D", "rotation_gaussian",
                                       "hall_circular_wave"):
        return f(o, "b", t)
    return f(o, what, t)
