"""TEST INFRASTRUCTURE ONLY -- numpy restatement of InductionEq's kernels (the oracle).

Every reference kernel of the time-stepping path is restated here over whole arrays, in
the reference's own order of floating-point operations, so that this restatement agrees
bit for bit with the reference kernels compiled by ``oracle/refimpl.py`` (g++,
-ffp-contract=off) whenever the inputs agree.  Fields are flat arrays in the reference
layout: a vector field is ``(num_nodes, 4)`` (REAL4, ``.w`` = 0), a scalar field
``(num_nodes,)``, node index ``ix + NX*(iy + NY*iz)`` (include/utils.h:66-68).

Kernel names and argument orders are the reference's; ``NumpyOracle.run(name, grange,
*arrays)`` mirrors MatCL's ``cl_run_kernel`` call.  Reductions return one partial per node
(work-group size 1), so the host sums them, as matlab/+induction_eq/clean_div.m:41 does.

Only tests, ``__graft_entry__.smoke`` and ``bench.py``'s CPU-baseline leg use this module.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass

import numpy as np

_TABLES_JSON = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                            "inductioneq_b200", "sbp_tables.json")


def _expand(tab: dict) -> np.ndarray:
    """Compact table -> full (2*nb+1, width) rows (right rows by mirror symmetry)."""
    rows = [[float.fromhex(x) for x in r] for r in tab["rows"]]
    if not tab["explicit"]:
        nb, s = tab["nb"], tab["sign"]
        for j in range(nb - 1, -1, -1):
            rows.append([s * v if v != 0 else 0.0 for v in rows[j][::-1]])
    return np.array(rows, dtype=np.float64)


def load_operator(order: int, extended: bool) -> dict:
    with open(_TABLES_JSON) as f:
        data = json.load(f)
    e = data[f"{order}{'e' if extended else 'c'}"]
    minv_half = [float.fromhex(x) for x in e["Minv"]]
    minv = np.array(minv_half + minv_half[-2::-1], dtype=np.float64)
    lap = {k: _expand(v) for k, v in e["laplace"].items()}
    return {"ORDER": order, "NUM_BOUNDS": e["nb"], "STENCIL_WIDTH": e["sw"],
            "STENCIL_WIDTH_HOD": e["w_hod"], "SBP_diff": _expand(e["D"]),
            "SBP_diff_adjoint": _expand(e["Dadj"]), "D_HO": _expand(e["DHO"]), "M_INV": minv,
            "laplace": lap}


@dataclass
class OracleConfig:
    """The reference's -D settings (generate_settings.m) in runtime form."""
    nodes: tuple
    xmin: tuple
    xmax: tuple
    order: int = 4
    extended: bool = False
    periodic: bool = False
    hall: bool = False
    dissipation: str = "NONE"            # NONE | HIGH_ORDER | FIRST_ORDER | ADAPTIVE
    uibj: str = "PRODUCT"
    source: str = "CENTRAL"
    ujbi: str = "CENTRAL"
    laplace: str = "WIDE_STENCIL_DIRICHLET"
    testcase: str = "rotation_3D"
    real: str = "double"
    dt: float = 0.0
    hod_factor: float = 1.0
    mp2min: float = 1.0
    mp2max: float = 10.0
    cmin: float = 1.0
    cmax: float = 10.0
    tc_omega: float = 1.0
    bnodes: int = 1
    # a z slab of a decomposed grid of nzg planes whose plane 0 is global plane zoff: testcase
    # coordinates are the global grid's (IEQ_Z_OFFSET / IEQ_NZ_GLOBAL of the CUDA library;
    # not a reference setting -- the reference runs one grid); nzg = 0: the whole domain
    zoff: int = 0
    nzg: int = 0

    def spacing(self):
        # matlab/+induction_eq/initialize.m:12-21
        n = self.nodes
        if self.periodic:
            return tuple(float(self.xmax[i] - self.xmin[i]) / float(n[i]) for i in range(3))
        return tuple(float(self.xmax[i] - self.xmin[i]) / (float(n[i]) - 1) for i in range(3))


_LAP_KEY = {"WIDE_STENCIL_DIRICHLET": "WS_D0", "NARROW_STENCIL_DIRICHLET": "NS_D0",
            "WIDE_STENCIL_LNS": "WS_LN"}


class NumpyOracle:
    def __init__(self, cfg: OracleConfig):
        self.cfg = cfg
        self.T = np.float32 if cfg.real == "float" else np.float64
        self.op = load_operator(cfg.order, cfg.extended)
        self.NX, self.NY, self.NZ = cfg.nodes
        self.N = self.NX * self.NY * self.NZ
        self.d = cfg.spacing()
        T = self.T
        self.D = self.op["SBP_diff"].astype(T)
        self.Dadj = self.op["SBP_diff_adjoint"].astype(T)
        self.DHO = self.op["D_HO"].astype(T)
        self.MINV = self.op["M_INV"].astype(T)
        self.NB = self.op["NUM_BOUNDS"]
        self.SW = self.op["STENCIL_WIDTH"]
        self.WH = self.op["STENCIL_WIDTH_HOD"]
        self._coord = [np.arange(n) for n in (self.NX, self.NY, self.NZ)]

    # ------------------------------------------------------------------ indexing helpers
    def grid(self, f: np.ndarray) -> np.ndarray:
        """Flat (N[,4]) -> (NZ, NY, NX[,4]) view."""
        return f[: self.N].reshape((self.NZ, self.NY, self.NX) + f.shape[1:])

    def _nbr_index(self, axis: int, off: int) -> np.ndarray:
        # include/utils.h:89-121 (periodic wrap) and 142-168 (clamp to the node itself)
        n = (self.NX, self.NY, self.NZ)[axis]
        i = self._coord[axis]
        j = i + off
        if self.cfg.periodic:
            return np.mod(j, n)
        bad = (j < 0) | (j >= n)
        return np.where(bad, i, j)

    def shift(self, g: np.ndarray, axis: int, off: int) -> np.ndarray:
        """g on the (NZ,NY,NX[,4]) grid, fetched at (axis) offset `off`."""
        if off == 0:
            return g
        return np.take(g, self._nbr_index(axis, off), axis=2 - axis)

    def _rows(self, axis: int, nb: int) -> np.ndarray:
        # include/utils.h:125-136 (periodic: always the interior row), 172-201
        n = (self.NX, self.NY, self.NZ)[axis]
        i = self._coord[axis]
        if self.cfg.periodic:
            return np.full(n, nb)
        bound = np.zeros(n, dtype=np.int64)
        for k in range(nb):
            bound += (nb - k) * ((i == n - (k + 1)).astype(np.int64) - (i == k).astype(np.int64))
        return nb + bound

    def _coef(self, table: np.ndarray, axis: int, nb: int, col: int, vec: bool) -> np.ndarray:
        c = table[self._rows(axis, nb), col]
        shape = [1, 1, 1]
        shape[2 - axis] = -1
        if vec:
            shape.append(1)
        return c.reshape(shape)

    def _col_used(self, table: np.ndarray, axis: int, nb: int, col: int) -> bool:
        return bool(np.any(table[np.unique(self._rows(axis, nb)), col] != 0))

    def _bcast(self, v, axis: int, vec: bool):
        shape = [1, 1, 1]
        shape[2 - axis] = -1
        if vec:
            shape.append(1)
        return v.reshape(shape)

    def coords(self):
        c = self.cfg
        T = self.T
        x = (T(c.xmin[0]) + self._coord[0].astype(T) * T(self.d[0]))[None, None, :]
        y = (T(c.xmin[1]) + self._coord[1].astype(T) * T(self.d[1]))[None, :, None]
        gz = self._coord[2] if c.nzg <= 0 else np.mod(self._coord[2] + c.zoff, c.nzg)
        z = (T(c.xmin[2]) + gz.astype(T) * T(self.d[2]))[:, None, None]
        return x, y, z

    def _v4(self, a, b, c, d=None):
        sh = np.broadcast_shapes(np.shape(a), np.shape(b), np.shape(c))
        out = np.zeros(sh + (4,), dtype=self.T)
        out[..., 0] = a
        out[..., 1] = b
        out[..., 2] = c
        if d is not None:
            out[..., 3] = d
        return out

    # ------------------------------------------------------------------ testcases
    def b_analytical(self, t) -> np.ndarray:
        return self._testcase("b", t)

    def _testcase(self, what: str, t) -> np.ndarray:
        from . import numpy_testcases as tc
        return tc.evaluate(self, self.cfg.testcase, what, t)

    # ------------------------------------------------------------------ SBP operator rows
    def diff(self, g: np.ndarray, axis: int, table=None) -> np.ndarray:
        """SBP_operator.cl:12-51 (vector) / 144-183 (scalar): sum_i D[row][i] f(i-c), / d."""
        table = self.D if table is None else table
        vec = g.ndim == 4
        val = np.zeros_like(g)
        c0 = (self.SW - 1) // 2
        for i in range(self.SW):
            if not self._col_used(table, axis, self.NB, i):
                continue
            val = val + self._coef(table, axis, self.NB, i, vec) * self.shift(g, axis, i - c0)
        return val / self.T(self.d[axis])

    def curl(self, g: np.ndarray) -> np.ndarray:
        # SBP_operator.cl:126-135
        dx, dy, dz = (self.diff(g, a) for a in range(3))
        out = np.zeros_like(g)
        out[..., 0] = dy[..., 2] - dz[..., 1]
        out[..., 1] = dz[..., 0] - dx[..., 2]
        out[..., 2] = dx[..., 1] - dy[..., 0]
        return out

    def div(self, g: np.ndarray, adjoint: bool = False) -> np.ndarray:
        # SBP_operator.cl:101-122
        tab = self.Dadj if adjoint else self.D
        return (self.diff(g, 0, tab)[..., 0] + self.diff(g, 1, tab)[..., 1]) + self.diff(g, 2, tab)[..., 2]

    def grad(self, s: np.ndarray, adjoint: bool = False) -> np.ndarray:
        # SBP_operator.cl:233-256
        tab = self.Dadj if adjoint else self.D
        return self._v4(self.diff(s, 0, tab), self.diff(s, 1, tab), self.diff(s, 2, tab), 0)

    # ------------------------------------------------------------------ volume terms
    def _flux(self, a: int, Bm, um, Bk, uk):
        """induction_Eq_volume.cl:13-165 for direction a (0=x, 1=y, 2=z)."""
        T = self.T
        c = self.cfg
        Ba_m, Ba_k = Bm[..., a:a + 1], Bk[..., a:a + 1]
        ua_m, ua_k = um[..., a:a + 1], uk[..., a:a + 1]
        if c.uibj == "CENTRAL":
            f1 = T(0.5) * (um * Ba_m + uk * Ba_k)
        elif c.uibj == "SPLIT":
            f1 = T(0.25) * (Ba_m + Ba_k) * (um + uk)
        else:
            f1 = T(0.5) * (um * Ba_k + uk * Ba_m)
        if c.source == "ZERO":
            f2 = np.zeros_like(Bm)
        elif c.source == "CENTRAL":
            f2 = T(0.5) * um * (Ba_k - Ba_m)
        else:
            f2 = T(0.25) * (um + uk) * (Ba_k - Ba_m)
        if c.ujbi == "CENTRAL":
            f3 = T(0.5) * (ua_m * Bm + ua_k * Bk)
        elif c.ujbi == "SPLIT":
            f3 = T(0.25) * (ua_m + ua_k) * (Bm + Bk)
        else:
            f3 = T(0.5) * (ua_m * Bk + ua_k * Bm)
        return f1 - f2 - f3

    def convec_volume(self, b: np.ndarray, u: np.ndarray) -> np.ndarray:
        # induction_Eq_volume.cl:168-212
        T = self.T
        val = np.zeros_like(b)
        c0 = (self.SW - 1) // 2
        for a in range(3):
            dB = np.zeros_like(b)
            for i in range(self.SW):
                if not self._col_used(self.D, a, self.NB, i):
                    continue
                Bk = self.shift(b, a, i - c0)
                uk = self.shift(u, a, i - c0)
                dB = dB + self._coef(self.D, a, self.NB, i, True) * self._flux(a, b, u, Bk, uk)
            val = val + T(2.0 / self.d[a]) * dB
        return val

    def hall_volume(self, b: np.ndarray, J: np.ndarray) -> np.ndarray:
        # induction_Eq_volume.cl:215-256
        T = self.T
        val = np.zeros_like(b)
        c0 = (self.SW - 1) // 2
        for a in range(3):
            dB = np.zeros_like(b)
            for i in range(self.SW):
                if not self._col_used(self.D, a, self.NB, i):
                    continue
                B = self.shift(b, a, i - c0)
                Jk = self.shift(J, a, i - c0)
                dB = dB + self._coef(self.D, a, self.NB, i, True) * (Jk[..., a:a + 1] * B - Jk * B[..., a:a + 1])
            val = val + T(1.0 / self.d[a]) * dB
        return val

    # ------------------------------------------------------------------ surface terms
    def _face_masks(self, a: int):
        n = (self.NX, self.NY, self.NZ)[a]
        i = self._coord[a]
        return self._bcast((i == 0).astype(self.T), a, False), self._bcast((i == n - 1).astype(self.T), a, False)

    def convec_surface(self, b, u, t) -> np.ndarray:
        # induction_Eq_surface.cl:7-33
        if self.cfg.periodic:
            return np.zeros_like(b)
        T = self.T
        bb = self._testcase("boundary", t)
        diff = b - bb
        terms = []
        for a in range(3):
            left, right = self._face_masks(a)
            ua = u[..., a]
            coef = (left * (ua > 0)) * T(-1) + (right * (ua < 0)) * T(1)
            s = T(self.MINV[0] / self.d[a]) if self.T == np.float64 else T(float(self.MINV[0]) / self.d[a])
            terms.append(((s * coef) * ua)[..., None] * diff)
        return (terms[0] + terms[1]) + terms[2]

    def convec_hall_surface(self, b, J, u) -> np.ndarray:
        # induction_Eq_surface.cl:35-81
        if self.cfg.periodic:
            return np.zeros_like(b)
        T = self.T
        tv = T(0.5) * u - J
        terms = []
        for a in range(3):
            left, right = self._face_masks(a)
            c1 = left * (tv[..., a] > 0) * T(-1) + right * (tv[..., a] < 0) * T(1)
            c2 = left * T(-1) + right * T(1)
            inner = (c1 * tv[..., a])[..., None] * b + (c2 * b[..., a])[..., None] * J
            s = T(float(self.MINV[0]) / self.d[a])
            terms.append(s * inner)
        return (terms[0] + terms[1]) + terms[2]

    # ------------------------------------------------------------------ artificial dissipation
    def _diff_hod(self, g, a: int, start: int) -> np.ndarray:
        # include/artificial_dissipation.h:58-101
        T = self.T
        W = self.WH
        rows = self._rows(a, self.NB)
        sgn = T(math.pow(-1.0, self.op["ORDER"] // 2 + 1))
        HOD = np.zeros_like(g)
        for i in range(W):
            m = self.MINV[rows] * self.DHO[rows, start + W - 1]
            coef = (m * self.DHO[self.NB, i]) * sgn
            HOD = HOD + self._bcast(coef.astype(T), a, True) * self.shift(g, a, i + start)
        return HOD

    def high_order_dissipation(self, b) -> np.ndarray:
        # artificial_dissipation.cl:13-32
        T = self.T
        F = T(self.cfg.hod_factor)
        H = np.zeros_like(b)
        for start in range(-self.WH + 1, 1):
            H = ((H + F * self._diff_hod(b, 0, start)) + F * self._diff_hod(b, 1, start)) + F * self._diff_hod(b, 2, start)
        H[..., 3] = 0
        return H

    def first_order_dissipation(self, b, u) -> np.ndarray:
        # artificial_dissipation.cl:36-79
        T = self.T
        FO = np.zeros_like(b)
        c0 = (self.SW - 1) // 2
        for a in range(3):
            tmp = np.zeros_like(b)
            for i in range(self.SW):
                ck = np.abs(self._coef(self.D, a, self.NB, i, True))
                uk = self.shift(u, a, i - c0)
                Bk = self.shift(b, a, i - c0)
                sig = np.fmax(np.abs(uk), np.abs(u))
                tmp[..., :3] = tmp[..., :3] + (ck * sig[..., :3]) * (Bk[..., :3] - b[..., :3])
            FO = FO + tmp / T(self.d[a])
        return FO

    def _kappa4(self, k: int, dx, b1, b2, u1, u2) -> np.ndarray:
        # include/artificial_dissipation.h:23-45 (k*k of the unsigned argument)
        c = self.cfg
        s = (np.fmax(np.abs(u1), np.abs(u2)) * (b1 - b2)) * (b1 - b2)
        k = k + (k == 0)
        kk = float(k * k)
        lo = ((kk * c.mp2min) * c.cmin) * float(dx)
        hi = ((kk * c.mp2max) * c.cmax) * float(dx)
        sd = s.astype(np.float64)
        inside = (lo < sd) & (sd < hi)
        val = inside * np.sqrt(np.abs(sd - lo) / abs(hi - lo)) + (sd >= hi)
        out = val.astype(self.T)
        out[..., 3] = 0
        return out

    def adaptive_dissipation(self, b, u) -> np.ndarray:
        # artificial_dissipation.cl:83-160
        T = self.T
        AD = np.zeros_like(b)
        c0 = (self.SW - 1) // 2
        F = T(self.cfg.hod_factor)
        for a in range(3):
            tmp = np.zeros_like(b)
            dxa = T(self.d[a])
            for i in range(self.SW):
                ck = np.abs(self._coef(self.D, a, self.NB, i, True))
                Bk = self.shift(b, a, i - c0)
                uk = self.shift(u, a, i - c0)
                kap = self._kappa4(abs(i - c0), dxa, Bk, b, uk, u)
                sig = np.fmax(np.abs(uk), np.abs(u))
                tmp[..., :3] = tmp[..., :3] + ((ck * kap[..., :3]) * sig[..., :3]) * (Bk[..., :3] - b[..., :3])
            AD[..., :3] = AD[..., :3] + tmp[..., :3] / dxa
        W = self.WH
        for term in range(-W + 1, 1):
            acc = AD[..., :3]
            for a in range(3):
                dxa = T(self.d[a])
                k1 = self._kappa4(1, dxa, self.shift(b, a, term + W - 1), self.shift(b, a, term + W - 2),
                                  self.shift(u, a, term + W - 1), self.shift(u, a, term + W - 2))
                acc = acc + ((T(1) - k1[..., :3]) * F) * self._diff_hod(b, a, term)[..., :3]
            AD[..., :3] = acc
        AD[..., 3] = 0
        return AD

    def artificial_dissipation(self, b, u) -> np.ndarray:
        d = self.cfg.dissipation
        if d == "HIGH_ORDER":
            return self.high_order_dissipation(b)
        if d == "FIRST_ORDER":
            return self.first_order_dissipation(b, u)
        if d == "ADAPTIVE":
            return self.adaptive_dissipation(b, u)
        return np.zeros_like(b)

    # ------------------------------------------------------------------ DB
    def DB(self, b, J, u, t) -> np.ndarray:
        """kernel_time_integrator.cl:9-31 on the grid views."""
        db = self.convec_volume(b, u)
        if self.cfg.hall:
            db = (db + self.convec_hall_surface(b, J, u)) + self.hall_volume(b, J)
        else:
            db = db + self.convec_surface(b, u, t)
        if self.cfg.dissipation != "NONE":
            db = db + self.artificial_dissipation(b, u)
        return db

    # ------------------------------------------------------------------ kernel dispatch
    def run(self, name: str, grange, *arrays: np.ndarray) -> None:
        from . import numpy_kernels
        numpy_kernels.run(self, name, grange, *arrays)

    def run_list(self, names, grange, *arrays: np.ndarray) -> None:
        for n in names:
            self.run(n, grange, *arrays)

    def vec(self, n=None) -> np.ndarray:
        return np.zeros((n or self.N, 4), dtype=self.T)

    def scalar(self, n=None, fill=0.0) -> np.ndarray:
        return np.full((n or self.N,), fill, dtype=self.T)
