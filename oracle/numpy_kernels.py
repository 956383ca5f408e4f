"""TEST INFRASTRUCTURE ONLY -- the reference's kernel entry points restated over numpy.

``run(oracle, name, grange, *arrays)`` executes the kernel ``name`` with the reference's
argument order (kernel/*.cl).  Time-integrator kernels take
``(b1, b2, [b3 | db,] curlB_rho, u, rho, time)``; the others are cited where defined.
"""
from __future__ import annotations

import numpy as np

# ----------------------------------------------------------------------------- RK tables
# kernel/kernel_time_integrator.cl:224-303 (SSPRK33), 315-621 (SSPRK104),
# 630-792 (KennedyCarpenterLewis2R54C), 801-1007 (CalvoFrancoRandez2R64),
# 1023-1206 (CarpenterKennedy2N54), 1216-1516 (ToulorgeDesmet2N84F)
KCL = {1: (0.22502245872571303, -0.17379315208537388, 0.22502245872571303),
       2: (0.5440433129514047, -0.1630884872250029, 0.5952726195917439),
       3: (0.14456824349399464, -0.5179208398863779, None),
       4: (0.7866643421983568, -0.19416305717199442, 0.8454958781727144)}
KCL_B5 = 0.34866717899927996
KCL_BK = {1: 1, 2: 1, 3: 2, 4: 1}           # which field the "a" kernel differentiates
CFR = {1: (0.17985400977138, 0.10893125722541, 0.28878526699679),
       2: (0.14081893152111, 0.13201701492152, 0.38176720366804),
       3: (0.08255631629428, 0.38911623225517, 0.71262082069639),
       4: (0.65804425034331, -0.59203884581148, 0.69606990893393),
       5: (0.31862993413251, 0.47385028714844, 0.83050587987157)}
CFR_B6 = 0.48812405426094
CFR_BK = {1: 1, 2: 2, 3: 2, 4: 2, 5: 2}
CK_A = {2: -567301805773.0 / 1357537059087.0, 3: -2404267990393.0 / 2016746695238.0,
        4: -3550918686646.0 / 2091501179385.0, 5: -1275806237668.0 / 842570457699.0}
CK_B = {1: 1432997174477.0 / 9575080441755.0, 2: 5161836677717.0 / 13612068292357.0,
        3: 1720146321549.0 / 2090206949498.0, 4: 3134564353537.0 / 4481467310338.0,
        5: 2277821191437.0 / 14882151754819.0}
CK_C = {1: 1432997174477.0 / 9575080441755.0, 2: 2526269341429.0 / 6820363962896.0,
        3: 2006345519317.0 / 3224310063776.0, 4: 2802321613138.0 / 2924317926251.0}
TD_A = {2: -0.5534431294501569, 3: 0.01065987570203490, 4: -0.5515812888932000,
        5: -1.885790377558741, 6: -5.701295742793264, 7: 2.113903965664793, 8: -0.5339578826675280}
TD_B = {1: 0.08037936882736950, 2: 0.5388497458569843, 3: 0.01974974409031960,
        4: 0.09911841297339970, 5: 0.7466920411064123, 6: 1.679584245618894,
        7: 0.2433728067008188, 8: 0.1422730459001373}
TD_C = {1: 0.08037936882736950, 2: 0.3210064250338430, 3: 0.3408501826604660,
        4: 0.3850364824285470, 5: 0.5040052477534100, 6: 0.6578977561168540,
        7: 0.9484087623348481}
# SSPRK104 stage kernels: name -> (time offset factor of the "a" kernel, src field, dst field)
SSP104 = {"01": (None, 1, 2), "02": (1.0 / 6.0, 2, 3), "03": (1.0 / 3.0, 3, 2), "04": (0.5, 2, 3),
          "05": (2.0 / 3.0, 3, 2), "07": (None, 2, 1), "08": (0.5, 1, 2), "09": (2.0 / 3.0, 2, 1),
          "10": (5.0 / 6.0, 1, 2), "11": (1.0, 2, 1)}
# the time value the reference forms for each "a" kernel (as a REAL expression of DT)
_SSP104_TEXPR = {"02": lambda dt: dt / 6.0, "03": lambda dt: dt / 3.0, "04": lambda dt: 0.5 * dt,
                 "05": lambda dt: dt * 2.0 / 3.0, "08": lambda dt: 0.5 * dt,
                 "09": lambda dt: dt * 2.0 / 3.0, "10": lambda dt: dt * 5.0 / 6.0,
                 "11": lambda dt: dt}


def _g(o, a):
    return o.grid(a)


def _DB(o, bk, cb, u, time):
    return o.DB(bk, _g(o, cb), _g(o, u), time[1])


def _interior(o, f):
    """Slice of the (NZ,NY,NX[,4]) grid view covering the CG interior (+BNODES offset)."""
    B = o.cfg.bnodes
    return f[B:o.NZ - B, B:o.NY - B, B:o.NX - B]


def run(o, name: str, grange, *a) -> None:
    T = o.T
    dt = o.cfg.dt
    TDT = T(dt)
    # -------------------------------------------------------------- init / analytic
    if name == "init_b":
        _g(o, a[0])[...] = o._testcase("init", 0.0)
        return
    if name == "init_u":
        _g(o, a[0])[...] = o._testcase("u_init", 0.0)
        return
    if name == "init_rho":
        _g(o, a[0])[...] = o._testcase("rho", 0.0)
        return
    if name == "analytical_b":
        _g(o, a[0])[...] = o._testcase("b", a[1][0])
        return
    # -------------------------------------------------------------- norms (kernel_operator.cl:11-137)
    if name in ("norm2", "norm2_diff", "norm2_S"):
        fac = _norm_fac(o)
        out = a[-1]
        n = int(grange[0])
        out[:n] = 0
        if name == "norm2":
            f = _g(o, a[0])
            val = fac * _dot4(f, f)
        elif name == "norm2_diff":
            dif = _g(o, a[0]) - _g(o, a[1])
            val = fac * _dot4(dif, dif)
        else:
            s = _g(o, a[0])
            val = (fac * s) * s
        out[:o.N] = val.reshape(-1)
        return
    if name == "dot_product":
        # kernel_dot_product.cl:47-74 (one partial per work item)
        n = int(grange[0])
        a[2][:n] = a[0][:n] * a[1][:n]
        return
    # -------------------------------------------------------------- operators
    if name == "calc_div":
        _g(o, a[1])[...] = o.div(_g(o, a[0]))
        return
    if name == "calc_curl":
        _g(o, a[1])[...] = o.curl(_g(o, a[0]))
        return
    if name == "calc_grad":
        _g(o, a[1])[...] = o.grad(_g(o, a[0]))
        return
    # -------------------------------------------------------------- divergence cleaning
    if name == "calc_div_divcleaning":
        _interior(o, _g(o, a[1]))[...] = _interior(o, o.div(_g(o, a[0])))
        return
    if name == "calc_laplace_divcleaning":
        _interior(o, _g(o, a[1]))[...] = _interior(o, _laplace(o, _g(o, a[0])))
        return
    if name == "projector_divcleaning":
        b = _g(o, a[0])
        phi = _g(o, a[1])
        if o.cfg.laplace == "WIDE_STENCIL_LNS":
            b[..., :3] = b[..., :3] - o.grad(phi, adjoint=True)[..., :3]
        else:
            b[..., :3] = b[..., :3] + o.grad(phi)[..., :3]
        return
    if name == "calc_axpy":
        x = _interior(o, _g(o, a[0]))
        x[...] = a[2][0] * x + _interior(o, _g(o, a[1]))
        return
    if name == "calc_xpay":
        x = _interior(o, _g(o, a[0]))
        x[...] = x + a[2][0] * _interior(o, _g(o, a[1]))
        return
    # -------------------------------------------------------------- time-integrator family
    three = len(a) == 7
    if three:
        b1, b2, b3, cb, u, rho, time = a
        b3 = _g(o, b3)
    else:
        b1, b2, cb, u, rho, time = a
        b3 = None
    b1, b2 = _g(o, b1), _g(o, b2)
    fields = {1: b1, 2: b2, 3: b3}
    if name in ("calc_time_2_args", "calc_time_3_args"):
        time[0] = time[0] + TDT
        time[1] = time[0]
        return
    if name in ("calc_u_2_args", "calc_u_3_args"):
        _g(o, u)[...] = o._testcase("u", time[1])
        return
    if name.startswith("calc_curlB_rho_"):
        k = int(name[len("calc_curlB_rho_")])
        _g(o, cb)[...] = o.curl(fields[k]) / _g(o, rho)[..., None]
        return
    if name == "SSPRK33_1":
        b2[...] = b1 + TDT * _DB(o, b1, cb, u, time)
        return
    if name == "SSPRK33_2a":
        time[1] = time[0] + TDT
        return
    if name == "SSPRK33_2b":
        b3[...] = T(0.75) * b1 + T(0.25) * (b2 + TDT * _DB(o, b2, cb, u, time))
        return
    if name == "SSPRK33_3a":
        time[1] = time[0] + T(0.5 * dt)
        return
    if name == "SSPRK33_3b":
        b1[...] = T(1.0 / 3.0) * b1 + T(2.0 / 3.0) * (b3 + TDT * _DB(o, b3, cb, u, time))
        return
    if name.startswith("SSPRK104_"):
        tag = name[len("SSPRK104_"):]
        h = T(dt / 6.0)
        if tag == "06":
            b3[...] = T(0.04) * b1 + T(0.36) * b2
            b2[...] = T(0.60) * b1 + T(0.40) * b2
            time[1] = time[0] + T(dt / 3.0)
            return
        if tag.endswith("a"):
            time[1] = time[0] + T(_SSP104_TEXPR[tag[:2]](dt))
            return
        key = tag[:2]
        _, src, dst = SSP104[key]
        if key == "11":
            b1[...] = b3 + T(0.6) * (b2 + h * _DB(o, b2, cb, u, time))
            return
        s = fields[src]
        fields[dst][...] = s + h * _DB(o, s, cb, u, time)
        return
    if name.startswith("KennedyCarpenterLewis2R54C_"):
        tag = name.split("_")[1]
        db = b3
        if tag == "5":
            b1[...] = b1 + (T(KCL_B5) * TDT) * _DB(o, b2, cb, u, time)
            return
        st = int(tag[0])
        if tag.endswith("a"):
            db[...] = TDT * _DB(o, fields[KCL_BK[st]], cb, u, time)
            return
        A, B, C = KCL[st]
        if st in (1, 3):
            b1[...] = b1 + T(A) * db
            b2[...] = b1 + T(B) * db
        else:
            b2[...] = b2 + T(A) * db
            b1[...] = b2 + T(B) * db
        if C is not None:
            time[1] = time[0] + T(C) * TDT
        return
    if name.startswith("CalvoFrancoRandez2R64_"):
        tag = name.split("_")[1]
        db = b3
        if tag == "6":
            b1[...] = b1 + (T(CFR_B6) * TDT) * _DB(o, b2, cb, u, time)
            return
        st = int(tag[0])
        if tag.endswith("a"):
            db[...] = TDT * _DB(o, fields[CFR_BK[st]], cb, u, time)
            return
        A, B, C = CFR[st]
        b1[...] = b1 + T(B) * db
        b2[...] = b1 + T(A) * db
        time[1] = time[0] + T(C) * TDT
        return
    if name.startswith("CarpenterKennedy2N54_") or name.startswith("ToulorgeDesmet2N84F_"):
        ck = name.startswith("Carpenter")
        Atab, Btab, Ctab = (CK_A, CK_B, CK_C) if ck else (TD_A, TD_B, TD_C)
        tag = name.split("_")[1]
        st = int(tag[0])
        if tag.endswith("a"):
            if st == 1:
                b2[...] = TDT * _DB(o, b1, cb, u, time)
            else:
                b2[...] = T(Atab[st]) * b2 + TDT * _DB(o, b1, cb, u, time)
            return
        b1[...] = b1 + T(Btab[st]) * b2
        if st in Ctab:
            time[1] = time[0] + T(Ctab[st]) * TDT
        return
    raise KeyError(f"unknown kernel {name}")


def _dot4(f, g):
    return ((f[..., 0] * g[..., 0] + f[..., 1] * g[..., 1]) + f[..., 2] * g[..., 2]) + f[..., 3] * g[..., 3]


def _norm_fac(o):
    # kernel_operator.cl:22-28: fac = prod_d (d / M_INV[row_d])
    T = o.T
    nb = o.NB
    fx = T(o.d[0]) / o.MINV[o._rows(0, nb)]
    fy = T(o.d[1]) / o.MINV[o._rows(1, nb)]
    fz = T(o.d[2]) / o.MINV[o._rows(2, nb)]
    return (fx[None, None, :] * fy[None, :, None]) * fz[:, None, None]


def _laplace(o, phi):
    # kernel_div_cleaning.cl:11-56
    from .numpy_oracle import _LAP_KEY
    T = o.T
    L = o.op["laplace"][_LAP_KEY[o.cfg.laplace]].astype(T)
    nb = (L.shape[0] - 1) // 2
    W = L.shape[1]
    c0 = (W - 1) // 2
    dd = [T(o.d[i]) * T(o.d[i]) for i in range(3)]
    val = np.zeros_like(phi)
    for i in range(W):
        tx = (o._coef(L, 0, nb, i, False) * o.shift(phi, 0, i - c0)) / dd[0]
        ty = (o._coef(L, 1, nb, i, False) * o.shift(phi, 1, i - c0)) / dd[1]
        tz = (o._coef(L, 2, nb, i, False) * o.shift(phi, 2, i - c0)) / dd[2]
        val = ((val + tx) + ty) + tz
    return val
