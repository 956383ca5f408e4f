"""CPU tests of the oracle: the numpy restatement against the reference.

* against the committed golden vectors (always; made by tests/golden/make_golden.py from
  the reference kernels compiled in place);
* against the compiled reference itself on fresh cases (only where the reference tree is
  readable, i.e. on the build machine);
* the compact SBP tables against the reference operator headers.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np
import pytest

from oracle import refimpl
from oracle.hostloops import clean_div, norms, time_loop
from oracle.numpy_oracle import NumpyOracle, OracleConfig, load_operator
from oracle.sequencing import NUM_FIELDS, rk_step
from tests.golden.cases import CG_CASES, STEP_CASES, mesh_args, variant_kwargs

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")


def _golden():
    z = np.load(GOLDEN)
    return z, json.loads(bytes(z["manifest"]).decode())


def oracle_for(c: dict, dt=None) -> NumpyOracle:
    m = mesh_args(c)
    cfg = OracleConfig(nodes=m["nodes"], xmin=m["xmin"], xmax=m["xmax"],
                       periodic=m["periodic"], dt=c.get("dt", 0.0) if dt is None else dt,
                       bnodes=c.get("bnodes", 1),
                       **{k: v for k, v in variant_kwargs(c).items() if k != "periodic"})
    return NumpyOracle(cfg)


@pytest.mark.parametrize("name", sorted(STEP_CASES))
def test_oracle_matches_golden_steps(name):
    z, man = _golden()
    c = STEP_CASES[name]
    o = oracle_for(c)
    nf = NUM_FIELDS[c["integrator"]]
    b = z[f"{name}/in_b"].copy()
    u = z[f"{name}/in_u"].copy()
    b2, b3, cb = o.vec(), o.vec(), o.vec()
    rho = o.scalar(fill=1.0)
    t = np.zeros(2, dtype=o.T)
    time_loop(o, c["integrator"], c.get("hall", False), c.get("variable_u", False), c["steps"],
              b, b2, b3 if nf == 3 else None, cb, u, rho, t)
    ref_b = z[f"{name}/out_b"]
    assert np.abs(ref_b - z[f"{name}/in_b"]).max() > 0, "fixture must move the field"
    np.testing.assert_array_equal(t, z[f"{name}/out_time"])
    if c.get("periodic") or c.get("hall") or c.get("real") == "float":
        # bit-exact: same operations in the same order as the compiled reference
        np.testing.assert_array_equal(b, ref_b)
        np.testing.assert_array_equal(b2, z[f"{name}/out_b2"])
    else:
        # the inflow SAT evaluates b_boundary(t) (exp/sin/cos): numpy's and the C
        # library's transcendental functions may differ in the last bit
        scale = np.abs(ref_b).max()
        assert np.abs(b - ref_b).max() <= 1e-14 * scale
        assert np.abs(b2 - z[f"{name}/out_b2"]).max() <= 1e-14 * max(scale, np.abs(b2).max())
    ana = o.vec()
    o.run("analytical_b", o.cfg.nodes, ana, t.copy())
    nrm = norms(o, b, ana, o.scalar())
    for k, v in man[name]["norms"].items():
        tol = 1e-6 if c.get("real") == "float" else 1e-12
        assert math.isclose(nrm[k], v, rel_tol=tol, abs_tol=1e-300), (k, nrm[k], v)


@pytest.mark.parametrize("name", sorted(CG_CASES))
def test_oracle_matches_golden_cg(name):
    z, man = _golden()
    c = CG_CASES[name]
    o = oracle_for(c)
    b = z[f"{name}/in_b"].copy()
    res = clean_div(o, b, c["max_iterations"], c["thr"], c["bnodes"])
    assert res["iterations"] == man[name]["iterations"]
    np.testing.assert_array_equal(res["history"], z[f"{name}/history"])
    np.testing.assert_array_equal(b, z[f"{name}/out_b"])


def test_cg_residual_decreases_for_dirichlet_laplacians():
    z, man = _golden()
    for name in ("cg_4c_wsd0", "cg_4c_nsd0", "cg_6c_wsd0"):
        h = z[f"{name}/history"]
        assert h[-1] < 1e-6 * h[0], (name, h[0], h[-1])


needs_reference = pytest.mark.skipif(not refimpl.reference_available(),
                                     reason="reference tree not readable here")


@needs_reference
@pytest.mark.parametrize("order,ext", [(2, False), (4, False), (6, False), (2, True), (4, True),
                                       (6, True)])
def test_sbp_tables_match_reference_headers(order, ext):
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "gen", os.path.join(os.path.dirname(os.path.dirname(__file__)), "inductioneq_b200", "csrc",
                            "gen_sbp_tables.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    with open(os.path.join(refimpl.REFERENCE_DIR, "include", gen.header_name(order, ext))) as f:
        defs, tabs = gen.parse_header(f.read())
    op = load_operator(order, ext)
    assert op["NUM_BOUNDS"] == defs["NUM_BOUNDS"] and op["STENCIL_WIDTH"] == defs["STENCIL_WIDTH"]
    np.testing.assert_array_equal(op["SBP_diff"], np.array(tabs["SBP_diff"]))
    np.testing.assert_array_equal(op["SBP_diff_adjoint"], np.array(tabs["SBP_diff_adjoint"]))
    np.testing.assert_array_equal(op["D_HO"], np.array(tabs["D_HO"]))
    np.testing.assert_array_equal(op["M_INV"], np.array(tabs["M_INV"]))
    for short, name in gen.LAPLACE:
        if name in tabs:
            np.testing.assert_array_equal(op["laplace"][short], np.array(tabs[name]))
        else:
            assert short not in op["laplace"]


@needs_reference
@pytest.mark.parametrize("kw", [
    dict(order=6, extended=True, testcase="rotation_3D", integrator="SSPRK33", uibj="CENTRAL",
         source="SPLIT", ujbi="SPLIT"),
    dict(order=4, testcase="confined_domain", hall=True, integrator="CarpenterKennedy2N54",
         dissipation="ADAPTIVE", lo=0.0, hi=1.0),
    dict(order=2, testcase="rotation_2D", integrator="ToulorgeDesmet2N84F",
         dissipation="HIGH_ORDER", uibj="SPLIT", source="ZERO", ujbi="PRODUCT"),
])
def test_oracle_bit_exact_vs_compiled_reference(kw):
    kw = dict(kw)
    integ = kw.pop("integrator")
    lo, hi = kw.pop("lo", -1.0), kw.pop("hi", 1.0)
    c = dict(kw, nodes=(17, 16, 18), lo=lo, hi=hi)
    v = refimpl.Variant(**variant_kwargs(c))
    m = refimpl.Mesh(**mesh_args(c))
    m.dt = 0.01 if not c.get("hall") else 1e-3
    r = refimpl.RefRunner(v, m, nthreads=2)
    o = oracle_for(c, dt=m.dt)
    nf = NUM_FIELDS[integ]
    fr = [r.vec() for _ in range(3)] + [r.vec(), r.vec(), r.scalar(fill=1.0), np.zeros(2)]
    r.run("init_b", m.nodes, fr[0])
    r.run("init_u", m.nodes, fr[4])
    fo = [a.copy() for a in fr]
    seq = rk_step(integ, c.get("hall", False), False)
    sel = (lambda f: f if nf == 3 else [f[0], f[1]] + f[3:])
    for k in seq:
        r.run(k, m.nodes, *sel(fr))
        o.run(k, m.nodes, *sel(fo))
        for a, b in zip(fr, fo):
            if c.get("hall") or c.get("periodic"):
                np.testing.assert_array_equal(a, b, err_msg=k)
            else:   # b_boundary(t) goes through the C library's / numpy's exp, sin, cos
                assert np.abs(a - b).max() <= 1e-14 * max(1e-300, np.abs(a).max()), k
