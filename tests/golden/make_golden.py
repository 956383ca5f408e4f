"""Generate tests/golden/golden.npz from the reference's own kernels (run here).

The reference kernels are compiled in place from the reference tree by
oracle/refimpl.py; this script runs the small cases of tests/golden/cases.py through
them and stores inputs and outputs, so that the numpy restatement (the oracle used on
machines without the reference tree) stays pinned to the reference.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.hostloops import clean_div, norms, time_loop  # noqa: E402
from oracle.refimpl import Mesh, RefRunner, Variant  # noqa: E402
from oracle.sequencing import NUM_FIELDS  # noqa: E402
from tests.golden.cases import (CG_CASES, NOISE_AMPLITUDE, NOISE_SEED, STEP_CASES,  # noqa: E402
                                mesh_args, variant_kwargs)


def noise(shape, seed=NOISE_SEED):
    return NOISE_AMPLITUDE * np.random.default_rng(seed).random(shape)


def main() -> None:
    out = {}
    manifest = {}
    for name, c in STEP_CASES.items():
        v = Variant(**variant_kwargs(c))
        m = Mesh(**mesh_args(c))
        m.dt = c["dt"]
        r = RefRunner(v, m, nthreads=4)
        nodes = m.nodes
        nf = NUM_FIELDS[c["integrator"]]
        b, b2, b3, cb, u = (r.vec() for _ in range(5))
        rho = r.scalar(fill=1.0)
        t = np.zeros(2, dtype=r.dtype)
        r.run("init_b", nodes, b)
        r.run("init_u", nodes, u)
        r.run("init_rho", nodes, rho)
        out[f"{name}/in_b"] = b.copy()
        out[f"{name}/in_u"] = u.copy()
        time_loop(r, c["integrator"], c.get("hall", False), c.get("variable_u", False), c["steps"],
                  b, b2, b3 if nf == 3 else None, cb, u, rho, t)
        out[f"{name}/out_b"] = b.copy()
        out[f"{name}/out_b2"] = b2.copy()
        out[f"{name}/out_time"] = t.copy()
        ana = r.vec()
        r.run("analytical_b", nodes, ana, t.copy())
        div = r.scalar()
        nrm = norms(r, b, ana, div)
        manifest[name] = {"case": c, "norms": nrm}
    for name, c in CG_CASES.items():
        v = Variant(**variant_kwargs(c))
        m = Mesh(**mesh_args(c))
        m.bnodes = c["bnodes"]
        r = RefRunner(v, m, nthreads=4)
        b = r.vec()
        r.run("init_b", m.nodes, b)
        b[:, :3] += noise((m.num_nodes, 3)).astype(r.dtype)
        out[f"{name}/in_b"] = b.copy()
        res = clean_div(r, b, c["max_iterations"], c["thr"], c["bnodes"])
        out[f"{name}/out_b"] = b.copy()
        out[f"{name}/history"] = res["history"]
        manifest[name] = {"case": c, "iterations": res["iterations"],
                          "initial_norm": res["initial_norm"]}
    out["manifest"] = np.frombuffer(json.dumps(manifest).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print(json.dumps(manifest, indent=1)[:3000])


if __name__ == "__main__":
    main()
