"""Host-side mirror of the reference's MATLAB driver (matlab/+induction_eq/*.m).

The reference keeps its run description in global maps (prepare_vars.m:29-56) --
I_Mesh, I_TI, I_IEq, I_DC, I_Tech, I_RunOps -- turns the upper-case keys into an OpenCL
"-D" settings string (generate_settings.m) and assembles the kernel path list
(compute_numerical_solution_setup.m:57-122).  ``Maps`` carries the same keys with the same
meanings; ``settings()`` and ``kernel_path_list()`` produce the strings that
``inductioneq_b200.lib.Context`` (the C ABI's ieq_create) accepts, and ``initialize`` /
``compute_numerical_solution`` / ``clean_div`` follow initialize.m,
compute_numerical_solution.m and clean_div.m on the B200 library.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .lib import Context


def generate_settings(m: dict, keys) -> str:
    """generate_settings.m:3-33: USE_* values become -DUSE_*=1, integers -DKEY=%d, reals
    -DKEY=%.16e, the 'optimizations' string is appended verbatim."""
    out = ""
    for k in keys:
        if k not in m:
            continue
        v = m[k]
        if isinstance(v, str):
            if k == "optimizations":
                out += v
            elif "USE" in v:
                out += f" -D{v}=1"
            else:
                out += f" -D{k}={v}"
        elif isinstance(v, bool):
            out += f" -D{k}={int(v)}"
        elif isinstance(v, (int, np.integer)):
            out += f" -D{k}={int(v)}"
        else:
            out += f" -D{k}={float(v):.16e}"
    return out


@dataclass
class Maps:
    """I_Mesh, I_TI, I_IEq, I_DC, I_Tech, I_RunOps with the reference's defaults."""
    I_Mesh: dict = field(default_factory=lambda: {"NODES_X": 0, "NODES_Y": 0, "NODES_Z": 0, "XMIN": 0.0,
                                                  "XMAX": 0.0, "YMIN": 0.0, "YMAX": 0.0, "ZMIN": 0.0,
                                                  "ZMAX": 0.0})
    I_TI: dict = field(default_factory=lambda: {"cfl": 0.0, "final_time": 0.0, "time_integrator": ""})
    I_IEq: dict = field(default_factory=lambda: {"form_uibj": "USE_UIBJ_PRODUCT",
                                                 "form_source": "USE_SOURCE_CENTRAL",
                                                 "form_ujbi": "USE_UJBI_CENTRAL", "hall_term": "NONE",
                                                 "dissipation": "NONE",
                                                 "dissipation_form": "USE_HIGH_ORDER_DISSIPATION",
                                                 "HO_DISSIPATION_FACTOR": 1.0, "MP2MIN": 1.0, "MP2MAX": 10.0,
                                                 "CMIN": 1.0, "CMAX": 10.0})
    I_DC: dict = field(default_factory=lambda: {"divergence_cleaning": False,
                                                "divergence_cleaning_form": "USE_LAPLACE_WIDE_STENCIL_DIRICHLET",
                                                "absolute_error_threshold": 1e-3, "max_iterations": 50})
    I_Tech: dict = field(default_factory=lambda: {"device": 0, "REAL": "double", "W_SIZE": 1,
                                                  "optimizations": " -cl-mad-enable -cl-no-signed-zeros"})
    I_RunOps: dict = field(default_factory=lambda: {"order": 4, "operator_form": "classical",
                                                    "testcase": "rotation_3D", "variable_u": False,
                                                    "periodic": "NONE"})
    tc_omega: float = 1.0
    # (DX, DY, DZ) given instead of derived from the box (a z slab of a decomposed grid keeps
    # the global spacing)
    spacing_override: tuple | None = None

    # initialize.m:12-21
    def spacing(self) -> tuple[float, float, float]:
        m = self.I_Mesh
        per = self.I_RunOps["periodic"] == "USE_PERIODIC"
        out = []
        for a in "XYZ":
            span = float(m[a + "MAX"] - m[a + "MIN"])
            n = float(m["NODES_" + a])
            out.append(span / n if per else span / (n - 1))
        return tuple(out)

    def settings(self) -> str:
        """compute_numerical_solution_setup.m:97-137."""
        m = dict(self.I_Mesh)
        m["DX"], m["DY"], m["DZ"] = self.spacing_override or self.spacing()
        tech = dict(self.I_Tech)
        tech["REAL4"] = tech["REAL"] + "4"
        s = generate_settings(self.I_IEq, ["form_uibj", "form_source", "form_ujbi", "hall_term"])
        s += generate_settings(self.I_TI, ["DT"])
        s += generate_settings(tech, ["REAL", "REAL4", "W_SIZE", "optimizations"])
        s += generate_settings(m, ["DX", "DY", "DZ", "NODES_X", "NODES_Y", "NODES_Z", "XMIN", "XMAX", "YMIN",
                                   "YMAX", "ZMIN", "ZMAX"])
        if self.I_IEq["dissipation"] == "USE_ARTIFICIAL_DISSIPATION":
            s += generate_settings(self.I_IEq, ["dissipation", "dissipation_form", "HO_DISSIPATION_FACTOR"])
            if self.I_IEq["dissipation_form"] == "USE_ADAPTIVE_DISSIPATION":
                s += generate_settings(self.I_IEq, ["MP2MIN", "MP2MAX", "CMIN", "CMAX"])
        dc = self.I_DC
        bn = 0 if dc["divergence_cleaning_form"] == "USE_LAPLACE_WIDE_STENCIL_LNS" else 1
        s += generate_settings({"BNODES": bn, "divergence_cleaning_form": dc["divergence_cleaning_form"]},
                               ["BNODES", "divergence_cleaning_form"])
        s += generate_settings(self.I_RunOps, ["periodic"])
        # keys of this library: integrator, variable velocity, rotation rate of the testcase
        if self.I_TI.get("time_integrator"):
            s += f" -DIEQ_INTEGRATOR={self.I_TI['time_integrator']}"
        if self.I_RunOps.get("variable_u"):
            s += " -DIEQ_VARIABLE_U=1"
        s += f" -DTC_OMEGA={self.tc_omega:.16e}"
        if self.I_Tech.get("stage_kernel", "AUTO") != "AUTO":
            s += f" -DIEQ_STAGE_KERNEL={self.I_Tech['stage_kernel']}"
        for key, name in (("col_block", "IEQ_COL_BLOCK"), ("curl_block", "IEQ_CURL_BLOCK")):
            if self.I_Tech.get(key):   # (x, y, z) threads of that column kernel, x * y * z = 128
                s += f" -D{name}=" + "x".join(str(int(v)) for v in self.I_Tech[key])
        if self.I_Tech.get("col_pairs") is not None:   # nodes per thread of the column kernels: 0, 1, 4
            s += f" -DIEQ_COL_PAIRS={int(self.I_Tech['col_pairs'])}"
        if self.I_Tech.get("pdl") is not None:   # programmatic dependent launch of the column kernels
            s += f" -DIEQ_PDL={int(bool(self.I_Tech['pdl']))}"
        if self.I_Tech.get("xband") is not None:   # boxes: x boundary columns in a launch of their own
            s += f" -DIEQ_XBAND={int(self.I_Tech['xband'])}"
        if self.I_Tech.get("zmarch_tz") is not None:   # z planes per CTA of the one-pass Hall stage
            s += f" -DIEQ_ZMARCH_TZ={int(self.I_Tech['zmarch_tz'])}"
        if self.I_Tech.get("cg_loop"):   # GRAPH (default) or HOST: the CG iterations as a graph loop or host launches
            s += f" -DIEQ_CG_LOOP={self.I_Tech['cg_loop']}"
        if self.I_Tech.get("curl_z") is not None:   # the 2.5D curl kernel on periodic grids: 0 never, 1 always, 2 auto
            s += f" -DIEQ_CURL_Z={int(self.I_Tech['curl_z'])}"
        if self.I_Tech.get("hodp") is not None:   # the dissipation sum formed by the curl kernel (1) or the stage kernel (0)
            s += f" -DIEQ_HODP={int(self.I_Tech['hodp'])}"
        if self.I_Tech.get("cg_pass_a") is not None:   # the CG's pass A: 2 the 2.5D kernel, 1 per-node gathers
            s += f" -DIEQ_CG_PASS_A={int(self.I_Tech['cg_pass_a'])}"
        if self.I_Tech.get("adjoint_program") is not None:   # 1: the register-program step adjoint for every integrator
            s += f" -DIEQ_ADJOINT_PROGRAM={int(self.I_Tech['adjoint_program'])}"
        if self.I_Tech.get("nz_global"):   # a z slab of a decomposed grid (inductioneq_b200.decomp)
            s += f" -DIEQ_Z_OFFSET={int(self.I_Tech['z_offset'])} -DIEQ_NZ_GLOBAL={int(self.I_Tech['nz_global'])}"
        return s

    def kernel_path_list(self) -> list[str]:
        """compute_numerical_solution_setup.m:57-122."""
        o = self.I_RunOps
        order = o["order"]
        hdr = f"../include/{order}{'th' if order > 2 else 'nd'}Order{'Extended' if o['operator_form'] == 'extended' else ''}.h"
        paths = [hdr, "../include/utils.h", f"../include/{o['testcase']}.h", "../kernel/kernel_init.cl",
                 "../kernel/SBP_operator.cl", "../kernel/kernel_operator.cl"]
        if self.I_DC["divergence_cleaning"]:
            paths += ["../kernel/kernel_div_cleaning.cl", "../kernel/kernel_CG.cl"]
        if self.I_IEq["dissipation"] == "USE_ARTIFICIAL_DISSIPATION":
            paths += ["../include/artificial_dissipation.h", "../kernel/artificial_dissipation.cl"]
        paths += ["../kernel/induction_Eq_volume.cl", "../kernel/induction_Eq_surface.cl",
                  "../kernel/kernel_dot_product.cl", "../kernel/kernel_time_integrator.cl"]
        return paths

    def context(self, device: int = 0) -> Context:
        return Context(self.settings(), self.kernel_path_list(), device)


def initialize(maps: Maps, u_max: float | None = None, device: int = 0):
    """initialize.m: spacing, fields b/u/rho from the testcase, dt from the CFL number
    (dt = cfl*min(d)/max|u|, num_steps = ceil(T/dt), dt = T/num_steps, lines 93-99).
    Returns (ctx, b, u, rho) device buffers; u_max overrides max|u| (the Hall cases with
    u = 0 need an explicit step)."""
    maps.I_TI.setdefault("DT", 0.0)
    ctx = maps.context(device)
    b, u, rho = ctx.vec(), ctx.vec(), ctx.scalar()
    ctx.kernel("init_b", b)
    ctx.kernel("init_u", u)
    ctx.kernel("init_rho", rho)
    if u_max is None:
        uh = ctx.get_vec(u)
        u_max = float(np.sqrt((uh[:, :3] ** 2).sum(1)).max())
    dt = maps.I_TI["cfl"] * min(maps.spacing()) / u_max
    num_steps = math.ceil(maps.I_TI["final_time"] / dt)
    maps.I_TI["DT"] = maps.I_TI["final_time"] / num_steps
    maps.I_TI["num_steps"] = num_steps
    ctx.close()
    ctx = maps.context(device)   # recompile with DT, as compute_numerical_solution does
    return ctx


def compute_numerical_solution(ctx: Context, b, u, rho, num_steps: int, t_final: float,
                               save_integrals_over_time: bool = False, dc: dict | None = None) -> dict:
    """compute_numerical_solution.m: the step loop (fused, graph captured) and the results
    (I_Results: runtime, abs_err, rel_err, divergence_norm, energy; lines 197-250).

    save_integrals_over_time (lines 153-173): energy, ||div B|| and the L2 error of B before
    every step, with the final values appended (num_steps + 1 entries each, as
    energy_over_time, L2error_divB_over_time, L2error_B_over_time) and the times
    linspace(0, t_final, num_steps + 1).  dc: the I_DC map; with divergence_cleaning B is
    cleaned after every step (lines 121-129) by the CG of clean_div.m with its
    absolute_error_threshold and max_iterations.  Series and cleaning stay on the device
    (ieq_time_steps_integrals)."""
    import time as _time
    b2, b3, cb = ctx.vec(), ctx.vec(), ctx.vec()
    clock = ctx.scalar(np.zeros(2), n=2)
    clean = bool(dc and dc.get("divergence_cleaning"))
    t0 = _time.perf_counter()
    series = None
    if save_integrals_over_time or clean:
        series = ctx.time_steps_integrals(b, b2, b3, cb, u, rho, clock, num_steps,
                                          int(dc["max_iterations"]) if clean else 0,
                                          float(dc["absolute_error_threshold"]) if clean else 0.0)
    else:
        ctx.time_steps(b, b2, b3, cb, u, rho, clock, num_steps)
    ctx.synchronize()
    runtime = _time.perf_counter() - t0
    wv, ws = ctx.vec(), ctx.scalar()
    res = ctx.results(b, t_final, wv, ws)
    res["runtime"] = runtime
    if save_integrals_over_time:
        res["energy_over_time"] = np.append(series["energy"], res["energy"])
        res["L2error_divB_over_time"] = np.append(series["divergence_norm"], res["divergence_norm"])
        res["L2error_B_over_time"] = np.append(series["l2_error"], res["abs_err"])
        res["time"] = np.linspace(0.0, t_final, num_steps + 1)
    return res


def clean_div(ctx: Context, b, dc: dict) -> dict:
    """clean_div.m: the CG projection of B with I_DC's absolute_error_threshold and
    max_iterations (iterations, final residual, divergence_norm_initial)."""
    return ctx.clean_div(b, int(dc["max_iterations"]), float(dc["absolute_error_threshold"]), check=False)


# ---------------------------------------------------------------- time-series output
# The paper scripts write the series of a run to an HDF5 file (paper/divcleaning_confined_domain.m
# :183-190: datasets /time, /energy, /L2error_B, /L2error_divB) and one summary line per run
# (:197-199).  The same datasets go to an .npz archive here (no HDF5 library is needed).

SERIES_DATASETS = (("time", "time"), ("energy", "energy_over_time"), ("L2error_B", "L2error_B_over_time"),
                   ("L2error_divB", "L2error_divB_over_time"))
_DC_LABELS = {"USE_LAPLACE_WIDE_STENCIL_LNS": "WS_LN", "USE_LAPLACE_WIDE_STENCIL_DIRICHLET": "WS_D0",
              "USE_LAPLACE_NARROW_STENCIL_DIRICHLET": "NS_D0"}


def series_filename(maps: Maps, ext: str = ".npz") -> str:
    """The paper script's file name of a run (divcleaning_confined_domain.m:162-177) with the
    testcase as prefix: <testcase>_N_<N>_order_<p>_<uibj>_<source>_<ujbi>__DC_<0|1>[_<label>]."""
    ieq, dc = maps.I_IEq, maps.I_DC
    forms = "_".join(ieq[k].split("_", 2)[2].lower() for k in ("form_uibj", "form_source", "form_ujbi"))
    name = f"{maps.I_RunOps['testcase']}_N_{int(maps.I_Mesh['NODES_X'])}_order_{int(maps.I_RunOps['order'])}_{forms}"
    if dc.get("divergence_cleaning"):
        name += "__DC_1_" + _DC_LABELS[dc["divergence_cleaning_form"]]
    else:
        name += "__DC_0"
    return name + ext


def write_series(path: str, results: dict) -> None:
    """The series of a run (compute_numerical_solution with save_integrals_over_time) as an
    .npz archive with the paper's dataset names (time, energy, L2error_B, L2error_divB),
    float64; an existing file is replaced."""
    np.savez(path, **{ds: np.asarray(results[key], dtype=np.float64) for ds, key in SERIES_DATASETS})


def read_series(path: str) -> dict:
    with np.load(path) as z:
        return {ds: z[ds].copy() for ds, _ in SERIES_DATASETS}


def summary_row(maps: Maps, results: dict) -> str:
    """The paper script's summary line of a run (divcleaning_confined_domain.m:192-199): N,
    order, the three flux forms, runtime, energy, abs_err, divergence_norm, the cleaning switch
    and its form."""
    ieq, dc = maps.I_IEq, maps.I_DC
    on = bool(dc.get("divergence_cleaning"))
    return "%d, %d, %s, %s, %s, %.15e, %.15e, %.15e, %.15e, %d, %s \n" % (
        int(maps.I_Mesh["NODES_X"]), int(maps.I_RunOps["order"]), ieq["form_uibj"], ieq["form_source"],
        ieq["form_ujbi"], results["runtime"], results["energy"], results["abs_err"], results["divergence_norm"],
        int(on), dc["divergence_cleaning_form"] if on else " ")
