"""Shared helpers of the tests: contexts and oracles built from one case description."""
from __future__ import annotations

import numpy as np

from inductioneq_b200.induction_eq import Maps
from oracle.numpy_oracle import NumpyOracle, OracleConfig
from tests.golden.cases import mesh_args, variant_kwargs

INTEGRATOR_OF = {}


def maps_for(c: dict) -> Maps:
    m = Maps()
    n = c["nodes"]
    lo, hi = c["lo"], c["hi"]
    m.I_Mesh.update({"NODES_X": n[0], "NODES_Y": n[1], "NODES_Z": n[2], "XMIN": lo, "XMAX": hi,
                     "YMIN": lo, "YMAX": hi, "ZMIN": lo, "ZMAX": hi})
    m.I_TI["DT"] = c.get("dt", 0.0)
    m.I_TI["time_integrator"] = c.get("integrator", "")
    m.I_IEq["form_uibj"] = "USE_UIBJ_" + c.get("uibj", "PRODUCT")
    m.I_IEq["form_source"] = "USE_SOURCE_" + c.get("source", "CENTRAL")
    m.I_IEq["form_ujbi"] = "USE_UJBI_" + c.get("ujbi", "CENTRAL")
    m.I_IEq["hall_term"] = "USE_HALL" if c.get("hall") else "NONE"
    d = c.get("dissipation", "NONE")
    if d != "NONE":
        m.I_IEq["dissipation"] = "USE_ARTIFICIAL_DISSIPATION"
        m.I_IEq["dissipation_form"] = f"USE_{d}_DISSIPATION"
    m.I_DC["divergence_cleaning"] = True
    m.I_DC["divergence_cleaning_form"] = "USE_LAPLACE_" + c.get("laplace", "WIDE_STENCIL_DIRICHLET")
    m.I_Tech["REAL"] = c.get("real", "double")
    m.I_Tech["stage_kernel"] = c.get("stage_kernel", "AUTO")
    m.I_Tech["col_block"] = c.get("col_block")
    m.I_Tech["curl_block"] = c.get("curl_block")
    m.I_Tech["col_pairs"] = c.get("col_pairs")
    m.I_Tech["xband"] = c.get("xband")
    m.I_Tech["zmarch_tz"] = c.get("zmarch_tz")
    m.I_Tech["cg_pass_a"] = c.get("cg_pass_a")
    m.I_Tech["curl_z"] = c.get("curl_z")
    m.I_Tech["hodp"] = c.get("hodp")
    m.I_Tech["adjoint_program"] = c.get("adjoint_program")
    m.I_RunOps.update({"order": c.get("order", 4), "operator_form": "extended" if c.get("extended") else "classical",
                       "testcase": c["testcase"], "variable_u": c.get("variable_u", False),
                       "periodic": "USE_PERIODIC" if c.get("periodic") else "NONE"})
    m.tc_omega = c.get("omega", 1.0)
    return m


def oracle_for(c: dict, dt=None) -> NumpyOracle:
    m = mesh_args(c)
    cfg = OracleConfig(nodes=m["nodes"], xmin=m["xmin"], xmax=m["xmax"], periodic=m["periodic"],
                       dt=c.get("dt", 0.0) if dt is None else dt, bnodes=c.get("bnodes", 1),
                       tc_omega=c.get("omega", 1.0),
                       **{k: v for k, v in variant_kwargs(c).items() if k != "periodic"})
    return NumpyOracle(cfg)


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """max |a - b| / max(|b|): the per-stage relative error of a field."""
    scale = float(np.abs(b).max())
    return float(np.abs(a - b).max()) / (scale if scale > 0 else 1.0)


def ref_runner_for(c: dict, dt=None):
    """The reference's kernels compiled in place (the strict parity build of oracle/_ref),
    OpenMP over every host core, for one case description."""
    import os

    from oracle import refimpl
    m = mesh_args(c)
    mesh = refimpl.Mesh(m["nodes"], m["xmin"], m["xmax"], m["periodic"],
                        dt=c.get("dt", 0.0) if dt is None else dt, bnodes=c.get("bnodes", 1),
                        tc_omega=c.get("omega", 1.0))
    return refimpl.RefRunner(refimpl.Variant(**variant_kwargs(c)), mesh, nthreads=os.cpu_count() or 1)


def own_scale_err(got: np.ndarray, ref: np.ndarray) -> float:
    """max |got - ref| / max |ref| over the first len(ref) rows (the device arrays are padded)."""
    return rel_err(np.asarray(got)[: len(ref)].astype(np.float64), ref.astype(np.float64))


def rounding_floor(c: dict, kind: str, max_b: float, max_u: float = 0.0, stages: int = 1) -> float:
    """Absolute forward-error floor of a field that a derivative of the state feeds, for
    comparisons of those fields on their own (small) scale.

    The state carries rounding of eps * |B| (|B| includes a unit mean field in the Hall
    cases); an RK register (b2 of the 2N schemes, b3/db of the 2R schemes) holds DT * F(b),
    and the curl buffer holds curl(B)/rho, so that rounding reaches them through the
    discrete operator F (Lipschitz constant ||F||) once per stage:
        register: stages * eps * DT * |B| * ||F||,  curl: stages * eps * |B| * 3 * sum|D| / dx,
    with ||F|| <= 3 * 3 * 2^order (high-order dissipation: three axes and components,
    interior row sum 2^order times the boundary-row factor 3) + 6 * (sum|D|/dx)^2 * |B| (Hall:
    J = curl B, E = J x B, D[E]) + 12 * (sum|D|/dx) * |u| (convection), sum|D| <= 4 the
    absolute row sum of a derivative row (boundary rows included), dx the smallest spacing.
    A comparison passes at rtol * max|ref| + this floor."""
    eps = float(np.finfo(np.float32 if c.get("real") == "float" else np.float64).eps)
    n = c["nodes"]
    span = c["hi"] - c["lo"]
    dx = min(span / (k if c.get("periodic") else k - 1) for k in n)
    sd = 4.0 / dx
    if kind == "curl":
        return stages * eps * max_b * 3.0 * sd
    op = 0.0
    if c.get("dissipation", "NONE") != "NONE":
        op += 9.0 * 2.0 ** c.get("order", 4)
    if c.get("hall"):
        op += 6.0 * sd * sd * max_b
    op += 12.0 * sd * max_u
    return stages * eps * c.get("dt", 0.0) * max_b * op


def stages_of(c: dict, steps: int) -> int:
    from oracle.sequencing import stages_per_step
    return steps * stages_per_step(c["integrator"])


def field_ok(got, ref, rtol: float, floor: float = 0.0) -> tuple[bool, float]:
    """max |got - ref| <= rtol * max |ref| + floor over the reference rows; returns (ok, the
    error relative to max |ref|)."""
    g = np.asarray(got)[: len(ref)].astype(np.float64)
    r = np.asarray(ref).astype(np.float64)
    d = float(np.abs(g - r).max())
    s = float(np.abs(r).max())
    return d <= rtol * s + floor, d / (s if s > 0 else 1.0)
