"""TEST INFRASTRUCTURE ONLY -- restatement of the reference host loops.

Works with any runner that has ``run(name, grange, *arrays)`` and ``vec()/scalar()``
(``oracle.refimpl.RefRunner`` or ``oracle.numpy_oracle.NumpyOracle``).
"""
from __future__ import annotations

import math

import numpy as np

from .sequencing import NUM_FIELDS, rk_step


def time_loop(runner, integrator: str, hall: bool, variable_u: bool, num_steps: int,
              b, b2, b3, curlB_rho, u, rho, time) -> None:
    """matlab/+induction_eq/compute_numerical_solution.m:111-193 (no cleaning, no integrals)."""
    nodes = runner_nodes(runner)
    seq = rk_step(integrator, hall, variable_u)
    args = (b, b2, b3, curlB_rho, u, rho, time) if NUM_FIELDS[integrator] == 3 else \
        (b, b2, curlB_rho, u, rho, time)
    for _ in range(num_steps):
        for k in seq:
            runner.run(k, nodes, *args)


def runner_nodes(runner):
    if hasattr(runner, "mesh"):
        return runner.mesh.nodes
    return runner.cfg.nodes


def clean_div(runner, b, max_iterations: int, absolute_error_threshold: float, bnodes: int):
    """matlab/+induction_eq/clean_div.m:36-79.  Returns a dict with phi, r, iterations,
    residual_norm2 (sum of per-item dot partials, as the host does) and the initial norm."""
    n = runner_nodes(runner)
    num = n[0] * n[1] * n[2]
    div = runner.scalar()
    phi = runner.scalar()
    lap = runner.scalar()
    r = runner.scalar()
    u = runner.scalar()
    out = runner.scalar()
    T = div.dtype.type
    g_dc = tuple(x - 2 * bnodes for x in n)
    runner.run("calc_div_divcleaning", g_dc, b, div)
    r[:] = div
    out[:] = 0
    runner.run("dot_product", (num, 1, 1), r, r, out)
    residual_norm2 = float(np.sum(out.astype(np.float64)))
    old = 1.0
    initial = math.sqrt(residual_norm2)
    tol = absolute_error_threshold * absolute_error_threshold
    it = 0
    history = [residual_norm2]
    while residual_norm2 > tol and it < max_iterations:
        beta = np.array([residual_norm2 / old], dtype=T)
        runner.run("calc_axpy", g_dc, u, r, beta)
        runner.run("calc_laplace_divcleaning", g_dc, u, lap)
        out[:] = 0
        runner.run("dot_product", (num, 1, 1), u, lap, out)
        alpha = residual_norm2 / float(np.sum(out.astype(np.float64)))
        runner.run("calc_xpay", g_dc, phi, u, np.array([alpha], dtype=T))
        runner.run("calc_xpay", g_dc, r, lap, np.array([-alpha], dtype=T))
        old = residual_norm2
        out[:] = 0
        runner.run("dot_product", (num, 1, 1), r, r, out)
        residual_norm2 = float(np.sum(out.astype(np.float64)))
        history.append(residual_norm2)
        it += 1
    runner.run("projector_divcleaning", n, b, phi)
    return {"phi": phi, "r": r, "div": div, "iterations": it, "residual_norm2": residual_norm2,
            "initial_norm": initial, "history": np.array(history)}


def norms(runner, b, b_ana, divB):
    """matlab/+induction_eq/compute_numerical_solution.m:210-250: abs/rel error, ||div B||, energy."""
    n = runner_nodes(runner)
    num = n[0] * n[1] * n[2]
    out = runner.scalar()
    runner.run("norm2_diff", (num, 1, 1), b, b_ana, out)
    abs_err = math.sqrt(float(np.sum(out.astype(np.float64))))
    out[:] = 0
    runner.run("norm2", (num, 1, 1), b_ana, out)
    rel_err = abs_err / math.sqrt(float(np.sum(out.astype(np.float64))))
    runner.run("calc_div", n, b, divB)
    out[:] = 0
    runner.run("norm2_S", (num, 1, 1), divB, out)
    div_norm = math.sqrt(float(np.sum(out.astype(np.float64))))
    out[:] = 0
    runner.run("norm2", (num, 1, 1), b, out)
    energy = float(np.sum(out.astype(np.float64)))
    return {"abs_err": abs_err, "rel_err": rel_err, "divergence_norm": div_norm, "energy": energy}
