"""GPU parity: the sm_100a kernels against the oracle on the same seeded inputs.

Tolerances: FP64 results agree with the oracle to 1e-12 relative per stage
(max |gpu - oracle| / max |oracle| over the field, after every kernel of the step); FP32
results to 2e-5.  The inputs are the golden fixtures (made by the reference's own kernels).
"""
from __future__ import annotations

import json
import math
import os

import numpy as np
import pytest

from oracle.hostloops import clean_div, norms, time_loop
from oracle.sequencing import NUM_FIELDS, rk_step
from tests.golden.cases import CG_CASES, NOISE_AMPLITUDE, NOISE_SEED, STEP_CASES
from tests.helpers import field_ok, maps_for, oracle_for, rel_err, rounding_floor, stages_of

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")
TOL64 = 1e-12
TOL32 = 2e-5
TWO_PI_ = 2.0 * math.pi
HP_ = 4.0 * math.pi / 3.0   # period of the hall_periodic testcase


def _golden():
    z = np.load(GOLDEN)
    return z, json.loads(bytes(z["manifest"]).decode())


def tol(c):
    return TOL32 if c.get("real") == "float" else TOL64


class HostRunner:
    """Runs reference kernels on the GPU through the MatCL-form host-array call."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.dtype = ctx.real

    def run(self, name, grange, *arrays):
        self.ctx.run_host([name], grange, *arrays)

    def vec(self):
        return np.zeros((self.ctx.n_pad, 4), dtype=self.dtype)

    def scalar(self, fill=0.0):
        return np.full((self.ctx.n_pad,), fill, dtype=self.dtype)

    @property
    def cfg(self):
        class _C:
            pass
        c = _C()
        c.nodes = self._nodes
        return c


def host_runner(ctx, nodes):
    r = HostRunner(ctx)
    r._nodes = tuple(nodes)
    return r


def _fields(ctx, o, z, name):
    b = z[f"{name}/in_b"].astype(o.T)
    u = z[f"{name}/in_u"].astype(o.T)
    host = [b, np.zeros_like(b), np.zeros_like(b), np.zeros_like(b), u, np.ones(o.N, dtype=o.T),
            np.zeros(2, dtype=o.T)]
    dev = [ctx.vec(host[0]), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(host[4]), ctx.scalar(host[5]),
           ctx.scalar(host[6], n=2)]
    return host, dev


@pytest.mark.parametrize("name", sorted(STEP_CASES))
def test_init_kernels_match_oracle(name):
    c = STEP_CASES[name]
    ctx = maps_for(c).context()
    o = oracle_for(c)
    for k, what in (("init_b", "init"), ("init_u", "u_init")):
        buf = ctx.vec()
        ctx.kernel(k, buf)
        ref = o.grid(o.vec())
        ref[...] = o._testcase(what, 0.0)
        assert rel_err(ctx.get_vec(buf)[: o.N], ref.reshape(-1, 4)) <= (1e-6 if c.get("real") == "float" else 1e-13)


@pytest.mark.parametrize("name", sorted(STEP_CASES))
def test_every_stage_kernel_matches_oracle(name):
    z, _ = _golden()
    c = STEP_CASES[name]
    ctx = maps_for(c).context()
    o = oracle_for(c)
    host, dev = _fields(ctx, o, z, name)
    nf = NUM_FIELDS[c["integrator"]]
    sel = (lambda f: f if nf == 3 else [f[0], f[1]] + f[3:])
    seq = rk_step(c["integrator"], c.get("hall", False), c.get("variable_u", False))
    moved = 0.0
    for _ in range(c["steps"]):
        for k in seq:
            ctx.run(k, o.cfg.nodes, *sel(dev))
            o.run(k, o.cfg.nodes, *sel(host))
            for i, (hd, dv) in enumerate(zip(host, dev)):
                if i == 6:
                    got = ctx.get_scalar(dv, n=2)
                    np.testing.assert_allclose(got, hd, rtol=1e-15, atol=0, err_msg=k)
                    continue
                if nf == 2 and i == 2:
                    continue
                got = ctx.get_scalar(dv) if hd.ndim == 1 else ctx.get_vec(dv)
                e = rel_err(got, hd)
                assert e <= tol(c), (k, i, e)
        moved = max(moved, rel_err(host[0], z[f"{name}/in_b"]))
    assert moved > 1e-8, "the case must change the field"


@pytest.mark.parametrize("name", sorted(STEP_CASES))
def test_fused_time_steps_match_oracle(name):
    z, _ = _golden()
    c = STEP_CASES[name]
    ctx = maps_for(c).context()
    o = oracle_for(c)
    host, dev = _fields(ctx, o, z, name)
    nf = NUM_FIELDS[c["integrator"]]
    time_loop(o, c["integrator"], c.get("hall", False), c.get("variable_u", False), c["steps"],
              host[0], host[1], host[2] if nf == 3 else None, host[3], host[4], host[5], host[6])
    ctx.time_steps(*dev, c["steps"])
    ctx.synchronize()
    assert rel_err(ctx.get_vec(dev[0]), host[0]) <= tol(c)
    assert rel_err(ctx.get_vec(dev[1]), host[1]) <= tol(c)
    if c.get("hall"):
        # the curl buffer holds curl(B)/rho of the last stage's input, as after the reference loop
        assert rel_err(ctx.get_vec(dev[3]), host[3]) <= tol(c)
    np.testing.assert_allclose(ctx.get_scalar(dev[6], n=2), host[6], rtol=1e-15)


# column-kernel shapes the golden cases do not reach: two-node columns next to the SBP
# boundary rows in z, a one-node last column (odd NZ), the outflow SAT with J on the faces
COLUMN_CASES = {
    "wave_6c_hall_hod_box_ck": dict(order=6, testcase="hall_circular_wave", nodes=(13, 12, 27), lo=0.0,
                                    hi=TWO_PI_, hall=True, dissipation="HIGH_ORDER",
                                    integrator="CarpenterKennedy2N54", dt=0.01, steps=2),
    "wave_4e_hall_box_ssp": dict(order=4, extended=True, testcase="hall_circular_wave", nodes=(14, 13, 21),
                                 lo=0.0, hi=TWO_PI_, hall=True, integrator="SSPRK33", dt=0.01, steps=2),
    "wave_4c_hall_hod_per_odd": dict(order=4, testcase="hall_circular_wave", nodes=(12, 13, 15), lo=0.0,
                                     hi=TWO_PI_, periodic=True, hall=True, dissipation="HIGH_ORDER",
                                     integrator="SSPRK33", dt=0.01, steps=2),
    "wave_2c_hall_per_f32": dict(order=2, testcase="hall_circular_wave", nodes=(11, 10, 9), lo=0.0,
                                 hi=TWO_PI_, periodic=True, hall=True, integrator="CarpenterKennedy2N54",
                                 dt=0.01, steps=3, real="float"),
}


@pytest.mark.parametrize("name", ["brick_6c_hall_hod_per", "brick_6e_hall_hod_box", "brick_4c_hall_hod_per_f32"])
def test_brick_kernels_equal_column_kernels(name):
    # the TMA brick kernels evaluate the same sums in the same order as the column kernels
    c = BRICK_CASES[name]
    out = []
    for kernel in ("BRICK", "COLUMN"):
        ctx = maps_for(dict(c, stage_kernel=kernel)).context()
        b = ctx.vec()
        ctx.kernel("init_b", b)
        bh = ctx.get_vec(b).astype(np.float64)
        bh[: ctx.n, :3] += 1e-2 * np.random.default_rng(NOISE_SEED).standard_normal((ctx.n, 3))
        dev = [ctx.vec(bh.astype(ctx.real)), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.scalar(np.ones(ctx.n_pad)),
               ctx.scalar(np.zeros(2), n=2)]
        ctx.time_steps(*dev, 2)
        out.append([ctx.get_vec(dev[i]) for i in (0, 1, 3)])
    for i in range(3):
        assert rel_err(out[0][i], out[1][i]) <= (1e-12 if c.get("real") != "float" else 1e-6), i


# TMA brick kernels (IEQ_STAGE_KERNEL=BRICK; 16 x 8 x 4 bricks; u = 0): periodic boxes with whole bricks per axis
# (x wrap boxes at both ends, single-brick axes), non-periodic boxes with interior bricks
# next to boundary bricks, Hall only, dissipation only, FP32
BRICK_CASES = {
    "brick_6c_hall_hod_per": dict(order=6, testcase="hall_circular_wave", nodes=(32, 16, 12), lo=0.0, hi=TWO_PI_,
                                  periodic=True, hall=True, dissipation="HIGH_ORDER",
                                  integrator="CarpenterKennedy2N54", dt=0.01, steps=2, stage_kernel="BRICK"),
    "brick_4c_hall_per_single": dict(order=4, testcase="hall_circular_wave", nodes=(16, 8, 12), lo=0.0, hi=TWO_PI_,
                                     periodic=True, hall=True, integrator="SSPRK33", dt=0.01, steps=2, stage_kernel="BRICK"),
    "brick_6e_hall_hod_box": dict(order=6, extended=True, testcase="hall_circular_wave", nodes=(48, 32, 24), lo=0.0,
                                  hi=TWO_PI_, hall=True, dissipation="HIGH_ORDER",
                                  integrator="CarpenterKennedy2N54", dt=0.005, steps=1, stage_kernel="BRICK"),
    "brick_4c_hall_hod_per_f32": dict(order=4, testcase="hall_circular_wave", nodes=(32, 16, 8), lo=0.0,
                                      hi=TWO_PI_, periodic=True, hall=True, dissipation="HIGH_ORDER",
                                      integrator="SSPRK33", dt=0.01, steps=2, real="float", stage_kernel="BRICK"),
    "brick_6c_hod_only_per": dict(order=6, testcase="hall_circular_wave", nodes=(16, 16, 16), lo=0.0, hi=TWO_PI_,
                                  periodic=True, dissipation="HIGH_ORDER", integrator="CarpenterKennedy2N54",
                                  dt=0.01, steps=2, stage_kernel="BRICK"),
    "brick_2c_hall_box_f32": dict(order=2, testcase="hall_circular_wave", nodes=(48, 24, 12), lo=0.0, hi=TWO_PI_,
                                  hall=True, integrator="ToulorgeDesmet2N84F", dt=0.005, steps=1, real="float", stage_kernel="BRICK"),
}


@pytest.mark.parametrize("name", sorted(COLUMN_CASES) + sorted(BRICK_CASES))
def test_fused_column_kernel_cases(name):
    c = COLUMN_CASES.get(name) or BRICK_CASES[name]
    ctx = maps_for(c).context()
    o = oracle_for(c)
    b = ctx.vec()
    ctx.kernel("init_b", b)
    bh = ctx.get_vec(b).astype(np.float64)
    rng = np.random.default_rng(NOISE_SEED)
    bh[: ctx.n, :3] += 1e-2 * rng.standard_normal((ctx.n, 3))
    bh = bh.astype(o.T)
    u = np.zeros_like(bh)
    nf = NUM_FIELDS[c["integrator"]]
    host = [bh.copy(), np.zeros_like(bh), np.zeros_like(bh), np.zeros_like(bh), u, np.ones(o.N, dtype=o.T),
            np.zeros(2, dtype=o.T)]
    dev = [ctx.vec(host[0]), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(u), ctx.scalar(host[5]),
           ctx.scalar(host[6], n=2)]
    hall = c.get("hall", False)
    time_loop(o, c["integrator"], hall, False, c["steps"], host[0], host[1], host[2] if nf == 3 else None,
              host[3], host[4], host[5], host[6])
    ctx.time_steps(*dev, c["steps"])
    mb = float(np.abs(host[0]).max())
    ns = stages_of(c, c["steps"])
    for i in (0, 1, 3) if hall else (0, 1):
        # every field on its own scale, the RK register b2 (= DT x DB for the 2N schemes) and
        # the curl buffer with the forward-error floor of a derivative of the state
        fl = {1: rounding_floor(c, "register", mb, 0.0, ns), 3: rounding_floor(c, "curl", mb, 0.0, ns)}.get(i, 0.0)
        ok, e = field_ok(ctx.get_vec(dev[i]), host[i], tol(c), fl)
        assert ok, (i, e)
    assert rel_err(host[0], bh) > 1e-6
    np.testing.assert_allclose(ctx.get_scalar(dev[6], n=2), host[6], rtol=1e-15 if o.T == np.float64 else 1e-6)


# Hall + convection (the testcase's velocity) through the pair kernels with the flux-form
# mask fixed at compile time: a box (x boundary pairs per node, SAT) and a periodic grid with
# the dissipation sum precomputed; nx even so that the pair kernels run
HALL_CONV_CASES = {
    "confined_4c_hall_conv_box": dict(order=4, testcase="confined_domain", nodes=(16, 13, 14), lo=0.0, hi=1.0,
                                      hall=True, integrator="CarpenterKennedy2N54", dt=1e-5, steps=2),
    "hallper_6c_hall_conv_hod_per": dict(order=6, testcase="hall_periodic", nodes=(16, 12, 14), lo=0.0, hi=HP_,
                                         periodic=True, hall=True, dissipation="HIGH_ORDER", integrator="SSPRK33",
                                         dt=1e-3, steps=2),
    "confined_2c_hall_conv_box_f32": dict(order=2, testcase="confined_domain", nodes=(14, 12, 10), lo=0.0, hi=1.0,
                                          hall=True, integrator="SSPRK33", dt=1e-5, steps=2, real="float"),
    # first-order dissipation summed in the pair kernels' gathers: a box (x boundary pairs per
    # node), the same box with its x boundary columns in a launch of their own, a periodic grid
    "confined_4c_hall_conv_fo_box": dict(order=4, testcase="confined_domain", nodes=(16, 13, 14), lo=0.0, hi=1.0,
                                         hall=True, dissipation="FIRST_ORDER", integrator="CarpenterKennedy2N54",
                                         dt=1e-5, steps=2),
    "confined_4c_hall_conv_fo_box_f32": dict(order=4, testcase="confined_domain", nodes=(16, 13, 14), lo=0.0,
                                             hi=1.0, hall=True, dissipation="FIRST_ORDER", integrator="SSPRK33",
                                             dt=1e-5, steps=2, real="float"),
    "confined_6c_hall_conv_fo_band": dict(order=6, testcase="confined_domain", nodes=(20, 13, 14), lo=0.0, hi=1.0,
                                          hall=True, dissipation="FIRST_ORDER", integrator="SSPRK33", dt=1e-5,
                                          steps=2, xband=2),
    "hallper_6c_hall_conv_fo_per": dict(order=6, testcase="hall_periodic", nodes=(16, 12, 14), lo=0.0, hi=HP_,
                                        periodic=True, hall=True, dissipation="FIRST_ORDER", integrator="SSPRK33",
                                        dt=1e-3, steps=2),
    # the same without the Hall term (convection and first-order dissipation only)
    "rotation_4c_conv_fo_box": dict(order=4, testcase="rotation_gaussian", nodes=(16, 13, 14), lo=-1.0, hi=1.0,
                                    dissipation="FIRST_ORDER", integrator="SSPRK33", dt=0.01, steps=2),
    # Hall + convection with the masks of other flux forms (9, 15, 14), with the high-order
    # dissipation precomputed on the periodic grid
    "hallper_4c_hall_conv_czc_per": dict(order=4, testcase="hall_periodic", nodes=(16, 12, 14), lo=0.0, hi=HP_,
                                         periodic=True, hall=True, uibj="CENTRAL", source="ZERO", ujbi="CENTRAL",
                                         integrator="SSPRK33", dt=1e-3, steps=2),
    "confined_4c_hall_conv_scs_box": dict(order=4, testcase="confined_domain", nodes=(16, 13, 14), lo=0.0, hi=1.0,
                                          hall=True, uibj="SPLIT", source="CENTRAL", ujbi="SPLIT",
                                          integrator="CarpenterKennedy2N54", dt=1e-5, steps=2),
    "hallper_6c_hall_conv_hod_pcs_per": dict(order=6, testcase="hall_periodic", nodes=(16, 12, 14), lo=0.0,
                                             hi=HP_, periodic=True, hall=True, dissipation="HIGH_ORDER",
                                             uibj="PRODUCT", source="CENTRAL", ujbi="SPLIT", integrator="SSPRK33",
                                             dt=1e-3, steps=2),
    # convection only with the two other flux forms of two sums per axis (masks 9 and 6)
    "rotation_4c_czc_box": dict(order=4, testcase="rotation_gaussian", nodes=(16, 13, 14), lo=-1.0, hi=1.0,
                                uibj="CENTRAL", source="ZERO", ujbi="CENTRAL", integrator="SSPRK33", dt=0.01,
                                steps=2),
    "rotation_6c_pcp_band": dict(order=6, testcase="rotation_gaussian", nodes=(20, 13, 14), lo=-1.0, hi=1.0,
                                 uibj="PRODUCT", source="CENTRAL", ujbi="PRODUCT", integrator="CarpenterKennedy2N54",
                                 dt=0.01, steps=2, xband=2),
    "rotation_2c_pcp_per": dict(order=2, testcase="rotation_gaussian", nodes=(16, 13, 14), lo=-1.0, hi=1.0,
                                periodic=True, uibj="PRODUCT", source="CENTRAL", ujbi="PRODUCT", integrator="SSPRK33",
                                dt=0.01, steps=2),
    "rotation_4c_ccc_box": dict(order=4, testcase="rotation_gaussian", nodes=(16, 13, 14), lo=-1.0, hi=1.0,
                                uibj="CENTRAL", source="CENTRAL", ujbi="CENTRAL", integrator="SSPRK33", dt=0.01,
                                steps=2),
    "rotation_6c_pcs_band": dict(order=6, testcase="rotation_gaussian", nodes=(20, 13, 14), lo=-1.0, hi=1.0,
                                 uibj="PRODUCT", source="CENTRAL", ujbi="SPLIT", integrator="SSPRK33", dt=0.01,
                                 steps=2, xband=2),
    "rotation_4c_czp_box": dict(order=4, testcase="rotation_gaussian", nodes=(16, 13, 14), lo=-1.0, hi=1.0,
                                uibj="CENTRAL", source="ZERO", ujbi="PRODUCT", integrator="SSPRK33", dt=0.01,
                                steps=2),
    "hallper_4c_hall_conv_csp_per": dict(order=4, testcase="hall_periodic", nodes=(16, 12, 14), lo=0.0, hi=HP_,
                                         periodic=True, hall=True, uibj="CENTRAL", source="SPLIT", ujbi="PRODUCT",
                                         integrator="SSPRK33", dt=1e-3, steps=2),
    "rotation_4c_scs_box_f32": dict(order=4, testcase="rotation_gaussian", nodes=(16, 13, 14), lo=-1.0, hi=1.0,
                                    uibj="SPLIT", source="CENTRAL", ujbi="SPLIT", integrator="SSPRK33", dt=0.01,
                                    steps=2, real="float"),
    "hallper_6c_hall_conv_czc_per_f32": dict(order=6, testcase="hall_periodic", nodes=(16, 12, 14), lo=0.0, hi=HP_,
                                             periodic=True, hall=True, uibj="CENTRAL", source="ZERO",
                                             ujbi="CENTRAL", integrator="SSPRK33", dt=1e-3, steps=2, real="float"),
    "rotation_2c_scs_box": dict(order=2, testcase="rotation_gaussian", nodes=(16, 13, 14), lo=-1.0, hi=1.0,
                                uibj="SPLIT", source="CENTRAL", ujbi="SPLIT", integrator="SSPRK33", dt=0.01, steps=2),
    "rotation_6c_conv_fo_band": dict(order=6, testcase="rotation_gaussian", nodes=(20, 13, 14), lo=-1.0, hi=1.0,
                                     dissipation="FIRST_ORDER", integrator="CarpenterKennedy2N54", dt=0.01, steps=2,
                                     xband=2),
}


@pytest.mark.parametrize("name", sorted(HALL_CONV_CASES))
def test_fused_hall_convection_pairs_match_oracle(name):
    c = HALL_CONV_CASES[name]
    ctx = maps_for(c).context()
    o = oracle_for(c)
    b, uf = ctx.vec(), ctx.vec()
    ctx.kernel("init_b", b)
    ctx.kernel("init_u", uf)
    u = ctx.get_vec(uf).astype(o.T)
    assert np.abs(u).max() > 0           # the convection terms are present
    bh = ctx.get_vec(b).astype(np.float64)
    bh[: ctx.n, :3] += 1e-2 * np.random.default_rng(NOISE_SEED).standard_normal((ctx.n, 3))
    bh = bh.astype(o.T)
    nf = NUM_FIELDS[c["integrator"]]
    host = [bh.copy(), np.zeros_like(bh), np.zeros_like(bh), np.zeros_like(bh), u, np.ones(o.N, dtype=o.T),
            np.zeros(2, dtype=o.T)]
    dev = [ctx.vec(host[0]), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(u), ctx.scalar(host[5]),
           ctx.scalar(host[6], n=2)]
    hall = c.get("hall", False)
    time_loop(o, c["integrator"], hall, False, c["steps"], host[0], host[1], host[2] if nf == 3 else None,
              host[3], host[4], host[5], host[6])
    ctx.time_steps(*dev, c["steps"])
    mb, mu = float(np.abs(host[0]).max()), float(np.abs(u).max())
    ns = stages_of(c, c["steps"])
    for i in (0, 1, 3) if hall else (0, 1):
        fl = {1: rounding_floor(c, "register", mb, mu, ns), 3: rounding_floor(c, "curl", mb, mu, ns)}.get(i, 0.0)
        ok, e = field_ok(ctx.get_vec(dev[i]), host[i], tol(c), fl)
        assert ok, (i, e)
    assert rel_err(host[0], bh) > 1e-7


@pytest.mark.parametrize("name", ["wave_6c_hall_hod_ck2n54", "rot_gauss_4c_ssprk33"])
def test_fused_time_steps_are_bitwise_reproducible(name):
    z, _ = _golden()
    c = STEP_CASES[name]
    ctx = maps_for(c).context()
    o = oracle_for(c)
    outs = []
    for _ in range(2):
        _, dev = _fields(ctx, o, z, name)
        ctx.time_steps(*dev, 3)
        outs.append(ctx.get_vec(dev[0]))
    np.testing.assert_array_equal(outs[0], outs[1])


@pytest.mark.parametrize("name", ["rot3d_2c_ck2n54", "wave_6c_hall_hod_ck2n54", "rot3d_4e_split_kcl",
                                  "confined_6e_hall_fo_cfr", "hallper_4c_ssprk104_varu", "alfven_2e_adaptive_td"])
def test_fused_odd_and_even_step_counts(name):
    # the fused 2N and 2R steps ping-pong b1 / b2; odd counts copy the result back from the
    # other buffers of the pairs
    z, _ = _golden()
    c = STEP_CASES[name]
    ctx = maps_for(c).context()
    o = oracle_for(c)
    nf = NUM_FIELDS[c["integrator"]]
    for n in (1, 2, 3):
        host, dev = _fields(ctx, o, z, name)
        time_loop(o, c["integrator"], c.get("hall", False), c.get("variable_u", False), n, host[0], host[1],
                  host[2] if nf == 3 else None, host[3], host[4], host[5], host[6])
        ctx.time_steps(*dev, n)
        assert rel_err(ctx.get_vec(dev[0]), host[0]) <= tol(c), n
        assert rel_err(ctx.get_vec(dev[1]), host[1]) <= tol(c), n
        if nf == 3:
            assert rel_err(ctx.get_vec(dev[2]), host[2]) <= tol(c), n
        np.testing.assert_allclose(ctx.get_scalar(dev[6], n=2), host[6], rtol=1e-15)


@pytest.mark.parametrize("name", sorted(STEP_CASES))
def test_fused_steps_equal_reference_kernel_lists(name):
    # IEQ_STAGE_KERNEL=LIST runs each step as the reference's kernel list on the caller's
    # fields; the fused path must agree with it
    z, _ = _golden()
    c = STEP_CASES[name]
    o = oracle_for(c)
    nf = NUM_FIELDS[c["integrator"]]
    out = []
    for kernel in ("AUTO", "LIST"):
        ctx = maps_for(dict(c, stage_kernel=kernel)).context()
        _, dev = _fields(ctx, o, z, name)
        ctx.time_steps(*dev, 3)
        out.append([ctx.get_vec(dev[i]) for i in range(nf)] + [ctx.get_scalar(dev[6], n=2)])
    for i in range(nf):
        assert rel_err(out[0][i], out[1][i]) <= tol(c), (i, rel_err(out[0][i], out[1][i]))
    np.testing.assert_allclose(out[0][-1], out[1][-1], rtol=1e-15)


@pytest.mark.parametrize("name", ["rot_gauss_4c_ssprk33", "rot3d_2c_ck2n54"])
def test_host_array_call_runs_reference_time_loop(name):
    # the MatCL-form call with host arrays (copy in, run the list, copy out)
    z, _ = _golden()
    c = STEP_CASES[name]
    ctx = maps_for(c).context()
    o = oracle_for(c)
    hg, _ = _fields(ctx, o, z, name)
    ho = [a.copy() for a in hg]
    nf = NUM_FIELDS[c["integrator"]]
    seq = rk_step(c["integrator"], False, False)
    sel = (lambda f: f if nf == 3 else [f[0], f[1]] + f[3:])
    for _ in range(c["steps"]):
        ctx.run_host(seq, o.cfg.nodes, *sel(hg))
        o.run_list(seq, o.cfg.nodes, *sel(ho))
    assert rel_err(hg[0], ho[0]) <= TOL64
    np.testing.assert_allclose(hg[6], ho[6], rtol=1e-15)


@pytest.mark.parametrize("name", sorted(STEP_CASES))
def test_norms_match_oracle(name):
    z, man = _golden()
    c = STEP_CASES[name]
    ctx = maps_for(c).context()
    o = oracle_for(c)
    b = z[f"{name}/out_b"].astype(o.T)
    t = float(z[f"{name}/out_time"][0])
    res = ctx.results(ctx.vec(b), t, ctx.vec(), ctx.scalar())
    ana = o.vec()
    o.run("analytical_b", o.cfg.nodes, ana, np.array([t, t], dtype=o.T))
    ref = norms(o, b.copy(), ana, o.scalar())
    rt = 1e-5 if c.get("real") == "float" else 1e-11
    # ||div B|| of a nearly divergence-free field is a cancellation: its absolute error is set
    # by the rounding of B itself (~eps * |B| / dx), not by its own size
    floor = {"divergence_norm": (1e-6 if c.get("real") == "float" else 1e-13) * ref["energy"] ** 0.5 / min(o.d)}
    for k in ("abs_err", "rel_err", "divergence_norm", "energy"):
        assert abs(res[k] - ref[k]) <= rt * abs(ref[k]) + floor.get(k, 1e-300), (k, res[k], ref[k])


@pytest.mark.parametrize("name", sorted(CG_CASES))
def test_clean_div_matches_oracle(name):
    z, man = _golden()
    c = CG_CASES[name]
    ctx = maps_for(c).context()
    o = oracle_for(c)
    b = z[f"{name}/in_b"].copy()
    ref = clean_div(o, b, c["max_iterations"], c["thr"], c["bnodes"])
    db = ctx.vec(z[f"{name}/in_b"])
    res = ctx.clean_div(db, c["max_iterations"], c["thr"], check=False)
    assert res["iterations"] == ref["iterations"] == man[name]["iterations"]
    assert abs(res["divergence_norm_initial"] - ref["initial_norm"]) <= 1e-12 * ref["initial_norm"]
    assert abs(res["residual_norm2"] - ref["residual_norm2"]) <= 1e-6 * ref["residual_norm2"] + 1e-30
    assert rel_err(ctx.get_vec(db), b) <= 1e-11


@pytest.mark.parametrize("name", ["cg_4c_wsd0", "cg_2c_wsln"])
def test_cg_kernels_through_reference_host_loop(name):
    # the reference's host loop (clean_div.m) driving the per-kernel GPU entry points
    z, man = _golden()
    c = CG_CASES[name]
    ctx = maps_for(c).context()
    o = oracle_for(c)
    r = host_runner(ctx, o.cfg.nodes)
    bg = z[f"{name}/in_b"].copy()
    bo = z[f"{name}/in_b"].copy()
    rg = clean_div(r, bg, 10, c["thr"], c["bnodes"])
    ro = clean_div(o, bo, 10, c["thr"], c["bnodes"])
    assert rg["iterations"] == ro["iterations"]
    np.testing.assert_allclose(rg["history"], ro["history"], rtol=1e-9)
    assert rel_err(bg, bo) <= 1e-11


def test_operators_match_oracle():
    z, _ = _golden()
    c = STEP_CASES["confined_6e_hall_fo_cfr"]
    ctx = maps_for(c).context()
    o = oracle_for(c)
    b = z["confined_6e_hall_fo_cfr/out_b"]
    n = o.cfg.nodes
    for k in ("calc_div", "calc_curl"):
        outd = ctx.scalar() if k == "calc_div" else ctx.vec()
        ctx.run(k, n, ctx.vec(b), outd)
        outh = o.scalar() if k == "calc_div" else o.vec()
        o.run(k, n, b.copy(), outh)
        got = ctx.get_scalar(outd) if k == "calc_div" else ctx.get_vec(outd)
        assert rel_err(got, outh) <= 1e-12, k
    s = b[:, 0].copy()
    outd = ctx.vec()
    ctx.run("calc_grad", n, ctx.scalar(s), outd)
    outh = o.vec()
    o.run("calc_grad", n, s, outh)
    assert rel_err(ctx.get_vec(outd), outh) <= 1e-12


def _oracle_series(o, c, host, steps, clean=None):
    """energy, ||div B|| and L2 error before every step, then the step (and the cleaning),
    as compute_numerical_solution.m:121-193 runs them"""
    nf = NUM_FIELDS[c["integrator"]]
    out = {"energy": [], "divergence_norm": [], "l2_error": []}
    for _ in range(steps):
        ana = o.vec()
        o.run("analytical_b", o.cfg.nodes, ana, host[6].copy())
        r = norms(o, host[0].copy(), ana, o.scalar())
        out["energy"].append(r["energy"])
        out["divergence_norm"].append(r["divergence_norm"])
        out["l2_error"].append(r["abs_err"])
        time_loop(o, c["integrator"], c.get("hall", False), c.get("variable_u", False), 1, host[0], host[1],
                  host[2] if nf == 3 else None, host[3], host[4], host[5], host[6])
        if clean:
            clean_div(o, host[0], clean[0], clean[1], c.get("bnodes", 1))
    return {k: np.array(v) for k, v in out.items()}


def _series_close(got, ref, c, o):
    rt = 1e-5 if c.get("real") == "float" else 1e-11
    floor = (1e-6 if c.get("real") == "float" else 1e-13) * float(np.max(ref["energy"])) ** 0.5 / min(o.d)
    # the error of a field equal to the exact one and ||div B|| of a nearly divergence-free
    # field are cancellations: their absolute errors are set by the rounding of B
    np.testing.assert_allclose(got["energy"], ref["energy"], rtol=rt, atol=1e-300)
    np.testing.assert_allclose(got["l2_error"], ref["l2_error"], rtol=rt, atol=floor * min(o.d))
    np.testing.assert_allclose(got["divergence_norm"], ref["divergence_norm"], rtol=rt, atol=floor)


@pytest.mark.parametrize("name", ["rot_gauss_4c_ssprk33", "wave_6c_hall_hod_ck2n54", "rot3d_4e_split_kcl",
                                  "hallper_4c_ssprk104_varu", "rot_gauss_4c_ssprk33_f32",
                                  "travel_6c_hall_sat_ssprk33", "confined_6e_hall_fo_cfr"])
def test_time_steps_integrals_match_oracle(name):
    # the per-step series of save_integrals_over_time, collected inside the step graph (Hall
    # steps: by the step's first curl kernel; otherwise by two launches of their own)
    z, _ = _golden()
    c = STEP_CASES[name]
    ctx = maps_for(c).context()
    o = oracle_for(c)
    steps = 3
    host, dev = _fields(ctx, o, z, name)
    got = ctx.time_steps_integrals(*dev, steps)
    ref = _oracle_series(o, c, host, steps)
    _series_close(got, ref, c, o)
    # the diagnostics do not change the stepping (Hall steps: the step's first curl kernel is
    # the one-node diagnostic form, equal to the other curl kernels up to FMA contraction)
    _, dev2 = _fields(ctx, o, z, name)
    ctx.time_steps(*dev2, steps)
    assert rel_err(ctx.get_vec(dev[0]), ctx.get_vec(dev2[0])) <= (1e-6 if c.get("real") == "float" else 1e-13)
    np.testing.assert_array_equal(ctx.get_scalar(dev[6], n=2), ctx.get_scalar(dev2[6], n=2))


def test_time_steps_integrals_with_cleaning_match_oracle():
    # divergence cleaning after every step (compute_numerical_solution.m:129-147)
    c = dict(order=4, testcase="confined_domain", nodes=(14, 15, 16), lo=0.0, hi=1.0, hall=True,
             integrator="CarpenterKennedy2N54", dt=2e-4, laplace="WIDE_STENCIL_DIRICHLET", bnodes=1)
    ctx = maps_for(c).context()
    o = oracle_for(c)
    b = ctx.vec()
    ctx.kernel("init_b", b)
    bh = ctx.get_vec(b).astype(np.float64)
    bh[: ctx.n, :3] += NOISE_AMPLITUDE * np.random.default_rng(NOISE_SEED).random((ctx.n, 3))
    zero = np.zeros_like(bh)
    host = [bh.copy(), zero.copy(), zero.copy(), zero.copy(), zero.copy(), np.ones(o.N), np.zeros(2)]
    dev = [ctx.vec(bh), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.scalar(np.ones(ctx.n_pad)),
           ctx.scalar(np.zeros(2), n=2)]
    steps, clean = 2, (60, 1e-9)
    got = ctx.time_steps_integrals(*dev, steps, clean_max_iterations=clean[0], clean_threshold=clean[1])
    ref = _oracle_series(o, c, host, steps, clean)
    _series_close(got, ref, c, o)
    assert rel_err(ctx.get_vec(dev[0]), host[0]) <= 1e-10


@pytest.mark.parametrize("diss", ["FIRST_ORDER", "ADAPTIVE"])
@pytest.mark.parametrize("periodic", [True, False])
def test_first_order_and_adaptive_dissipation_with_zero_velocity(diss, periodic):
    # with u = 0 the fused path runs first-order dissipation as no dissipation and the
    # adaptive form as the high-order dissipation (every kappa is 0); against the oracle's full
    # formulas (artificial_dissipation.cl:36-160) and the reference kernel lists
    c = dict(order=6, testcase="hall_circular_wave", nodes=(12, 13, 14), lo=0.0, hi=TWO_PI_, periodic=periodic,
             hall=True, dissipation=diss, integrator="CarpenterKennedy2N54", dt=0.005)
    o = oracle_for(c)
    b = o.vec()
    o.run("init_b", o.cfg.nodes, b)
    b[:, :3] += 1e-2 * np.random.default_rng(NOISE_SEED).standard_normal((o.N, 3))
    steps = 2
    host = [b.copy(), o.vec(), o.vec(), o.vec(), o.vec(), o.scalar(fill=1.0), np.zeros(2)]
    time_loop(o, c["integrator"], True, False, steps, host[0], host[1], None, host[3], host[4], host[5], host[6])
    mb = float(np.abs(host[0]).max())
    for kernel in ("AUTO", "LIST"):
        ctx = maps_for(dict(c, stage_kernel=kernel)).context()
        dev = [ctx.vec(b), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.scalar(np.ones(ctx.n_pad)),
               ctx.scalar(np.zeros(2), n=2)]
        ctx.time_steps(*dev, steps)
        for i, kind in ((0, None), (1, "register")):
            fl = rounding_floor(c, kind, mb, 0.0, stages_of(c, steps)) if kind else 0.0
            ok, e = field_ok(ctx.get_vec(dev[i]), host[i], TOL64, fl)
            assert ok, (kernel, i, e)
        ctx.close()


@pytest.mark.parametrize("clean", [False, True])
def test_compute_numerical_solution_series_and_results(clean, tmp_path):
    # compute_numerical_solution with save_integrals_over_time (compute_numerical_solution.m
    # :153-250): num_steps + 1 entries per series, the last being the final results, the
    # others the device series of ieq_time_steps_integrals; written and read back as .npz
    from inductioneq_b200.induction_eq import compute_numerical_solution, read_series, write_series
    c = dict(order=4, testcase="confined_domain", nodes=(14, 15, 16), lo=0.0, hi=1.0, hall=True,
             integrator="CarpenterKennedy2N54", dt=2e-4, laplace="WIDE_STENCIL_DIRICHLET", bnodes=1)
    dc = {"divergence_cleaning": clean, "absolute_error_threshold": 1e-9, "max_iterations": 60}
    steps = 3
    out = []
    for direct in (False, True):
        m = maps_for(c)
        ctx = m.context()
        b = ctx.vec()
        ctx.kernel("init_b", b)
        bh = ctx.get_vec(b)
        bh[: ctx.n, :3] += NOISE_AMPLITUDE * np.random.default_rng(NOISE_SEED).random((ctx.n, 3))
        b.upload(bh)
        u, rho = ctx.vec(), ctx.scalar(np.ones(ctx.n_pad))
        if direct:
            dev = [b, ctx.vec(), ctx.vec(), ctx.vec(), u, rho, ctx.scalar(np.zeros(2), n=2)]
            ser = ctx.time_steps_integrals(*dev, steps, clean_max_iterations=60 if clean else 0,
                                           clean_threshold=1e-9 if clean else 0.0)
            fin = ctx.results(b, steps * 2e-4, ctx.vec(), ctx.scalar())
            out.append((ser, fin))
        else:
            out.append(compute_numerical_solution(ctx, b, u, rho, steps, steps * 2e-4, save_integrals_over_time=True,
                                                  dc=dc))
        ctx.close()
    res, (ser, fin) = out
    for key, s_key, f_key in (("energy_over_time", "energy", "energy"),
                              ("L2error_divB_over_time", "divergence_norm", "divergence_norm"),
                              ("L2error_B_over_time", "l2_error", "abs_err")):
        assert res[key].shape == (steps + 1,)
        np.testing.assert_array_equal(res[key][:steps], ser[s_key])
        assert res[key][steps] == fin[f_key] == res[f_key]
    np.testing.assert_array_equal(res["time"], np.linspace(0.0, steps * 2e-4, steps + 1))
    path = tmp_path / "series.npz"
    write_series(str(path), res)
    back = read_series(str(path))
    np.testing.assert_array_equal(back["L2error_divB"], res["L2error_divB_over_time"])


@pytest.mark.parametrize("integrator", ["SSPRK33", "SSPRK104", "KennedyCarpenterLewis2R54C", "CalvoFrancoRandez2R64",
                                        "CarpenterKennedy2N54", "ToulorgeDesmet2N84F"])
@pytest.mark.parametrize("real", ["double", "float"])
def test_fused_hall_hod_steps_equal_kernel_lists_for_every_integrator(integrator, real):
    # Hall + high-order dissipation (the curl kernel forms the dissipation sum) through every
    # integrator's fused step, ping-pong buffers included, against the reference kernel lists
    c = dict(order=6, testcase="hall_circular_wave", nodes=(12, 13, 14), lo=0.0, hi=TWO_PI_, periodic=True,
             hall=True, dissipation="HIGH_ORDER", integrator=integrator, dt=0.005, real=real)
    nf = NUM_FIELDS[integrator]
    out = []
    for kernel in ("AUTO", "LIST"):
        ctx = maps_for(dict(c, stage_kernel=kernel)).context()
        b = ctx.vec()
        ctx.kernel("init_b", b)
        bh = ctx.get_vec(b).astype(np.float64)
        bh[: ctx.n, :3] += 1e-2 * np.random.default_rng(NOISE_SEED).standard_normal((ctx.n, 3))
        dev = [ctx.vec(bh.astype(ctx.real)), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.scalar(np.ones(ctx.n_pad)),
               ctx.scalar(np.zeros(2), n=2)]
        ctx.time_steps(*dev, 3)
        out.append([ctx.get_vec(dev[i]).astype(np.float64) for i in range(nf)] + [ctx.get_vec(dev[3]), 
                   ctx.get_scalar(dev[6], n=2)])
    mb = float(np.abs(out[1][0]).max())
    ns = stages_of(c, 3)
    for i in range(nf + 1):
        # every field on its own scale; the registers (b2; b3 = db of the 2R schemes) and the
        # curl buffer with the forward-error floor of a derivative of the state
        fl = 0.0 if i == 0 else rounding_floor(c, "curl" if i == nf else "register", mb, 0.0, ns)
        ok, e = field_ok(out[0][i], out[1][i], 1e-12 if real == "double" else 2e-6, fl)
        assert ok, (i, e)
    np.testing.assert_allclose(out[0][-1], out[1][-1], rtol=1e-15 if real == "double" else 1e-6)


@pytest.mark.parametrize("shape", [(128, 1, 1), (16, 4, 2), (8, 4, 4), (4, 8, 4)])
@pytest.mark.parametrize("case", ["hall_hod_box", "rotation_conv"])
def test_column_block_shape_does_not_change_the_result(shape, case):
    # the block shape only regroups nodes: every node's arithmetic is the same, so the
    # fields agree bit for bit (ragged grids: partial blocks in every direction)
    if case == "hall_hod_box":
        c = dict(order=6, testcase="hall_travelling_wave", nodes=(19, 13, 14), lo=0.0, hi=TWO_PI_, hall=True,
                 dissipation="HIGH_ORDER", integrator="CarpenterKennedy2N54", dt=0.002)
    else:
        c = dict(order=4, testcase="rotation_gaussian", nodes=(21, 10, 9), lo=-1.0, hi=1.0, integrator="SSPRK33", dt=0.01)
    out = []
    for sh in (None, shape):
        ctx = maps_for(dict(c, col_block=sh, curl_block=sh)).context()
        dev = [ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.scalar(np.ones(ctx.n_pad)),
               ctx.scalar(np.zeros(2), n=2)]
        ctx.kernel("init_b", dev[0])
        ctx.kernel("init_u", dev[4])
        ctx.time_steps(*dev, 4)
        out.append(ctx.get_vec(dev[0]))
    assert np.array_equal(out[0], out[1])
    assert np.isfinite(out[0]).all() and np.abs(out[0]).max() > 0


@pytest.mark.parametrize("case", ["periodic_hod", "box_hod", "box_plain", "periodic_plain_f32", "periodic_conv_hod",
                                  "periodic_fo", "periodic_conv_fo", "box_conv_fo", "box_conv_fo_f32",
                                  "periodic_adaptive_conv",
                                  "rotation_o2", "rotation_o4", "rotation_o4_fo", "rotation_o6_fo",
                                  "rotation_o4_czc", "rotation_o6_pcp",
                                  "rotation_o6_f32", "quads_periodic_hod_f32", "quads_box_hod_f32",
                                  "quads_periodic_plain_f32"])
def test_two_nodes_per_thread_equal_one_node_per_thread(case):
    # the Hall column kernels with two x-adjacent nodes per thread form every node's sums in
    # the order of the one-node kernels: the fields agree up to the compiler's choice of
    # fused multiply-adds (a few units in the last place)
    c = dict(order=6, testcase="hall_circular_wave", nodes=(18, 13, 14), lo=0.0, hi=TWO_PI_, hall=True,
             integrator="CarpenterKennedy2N54", dt=0.002)
    if case.startswith("periodic"):
        c.update(periodic=True, nodes=(14, 12, 16))
    if case.endswith("hod"):
        c.update(dissipation="HIGH_ORDER")
    if case.endswith("f32"):
        c.update(real="float")
    if case.startswith("box"):
        c.update(testcase="hall_travelling_wave")
    if "conv" in case:   # variable velocity: the convection sums beside the Hall term
        c.update(testcase="hall_periodic", hi=HP_, variable_u=True, dt=1e-3)
    if case.endswith("fo") or "_fo_" in case:
        c.update(dissipation="FIRST_ORDER")
    if case.startswith("periodic_adaptive"):
        c.update(dissipation="ADAPTIVE")
    if case.startswith("quads"):      # FP32 Hall kernels with four nodes per thread (float4)
        c.update(real="float", nodes=(16, 12, 14) if "periodic" in case else (20, 13, 14))
        if "periodic" in case:
            c.update(periodic=True)
        else:
            c.update(testcase="hall_travelling_wave")
        if "hod" in case:
            c.update(dissipation="HIGH_ORDER")
    if case.startswith("rotation"):   # convection only, default flux forms, inflow SAT
        c = dict(order=int(case[10]), testcase="rotation_gaussian", nodes=(16, 13, 14), lo=-1.0, hi=1.0,
                 integrator="SSPRK33", dt=0.01, real="float" if case.endswith("f32") else "double")
        if case.endswith("fo"):
            c.update(dissipation="FIRST_ORDER")
        if case.endswith("czc"):
            c.update(uibj="CENTRAL", source="ZERO", ujbi="CENTRAL")
        if case.endswith("pcp"):
            c.update(uibj="PRODUCT", source="CENTRAL", ujbi="PRODUCT")
    out = []
    for pairs in (0, 4 if case.startswith("quads") else 1):
        ctx = maps_for(dict(c, col_pairs=pairs)).context()
        dev = [ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.scalar(np.ones(ctx.n_pad)),
               ctx.scalar(np.zeros(2), n=2)]
        ctx.kernel("init_b", dev[0])
        ctx.kernel("init_u", dev[4])
        ctx.time_steps(*dev, 3)
        out.append([ctx.get_vec(dev[0]), ctx.get_vec(dev[1]), ctx.get_vec(dev[3])])
    tol = 2e-6 if case.endswith("f32") else 1e-13
    for i, (a, b) in enumerate(zip(*out)):
        e = rel_err(a.astype(np.float64), b.astype(np.float64))
        assert e <= tol, (i, e)
    assert np.isfinite(out[0][0]).all()


@pytest.mark.parametrize("case", ["rotation_o2", "rotation_o6", "hall_box_hod", "hall_box_plain_f32", "hall_box_hod_f32",
                                  "hall_conv_box"])
def test_box_x_band_equals_pair_kernels_alone(case):
    # boxes run their x boundary columns in a launch of their own (one node per thread) and
    # the pair kernels over the interior x range: the same sums as the pair kernels with the
    # boundary columns inside them, up to FMA contraction
    if case.startswith("rotation"):
        c = dict(order=int(case[-1]), testcase="rotation_gaussian", nodes=(26, 13, 14), lo=-1.0, hi=1.0,
                 integrator="SSPRK33", dt=0.01)
    elif case == "hall_conv_box":
        c = dict(order=4, testcase="confined_domain", nodes=(18, 13, 14), lo=0.0, hi=1.0, hall=True,
                 integrator="CarpenterKennedy2N54", dt=1e-5)
    else:
        c = dict(order=6, testcase="hall_travelling_wave", nodes=(22, 13, 14), lo=0.0, hi=TWO_PI_, hall=True,
                 integrator="CarpenterKennedy2N54", dt=0.002, real="float" if case.endswith("f32") else "double")
        if "hod" in case:   # (FP32: the x band of the curl kernel too)
            c.update(dissipation="HIGH_ORDER")
    out = []
    for band in (0, 2):   # never / wherever the rows allow
        ctx = maps_for(dict(c, xband=band)).context()
        dev = [ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.scalar(np.ones(ctx.n_pad)),
               ctx.scalar(np.zeros(2), n=2)]
        ctx.kernel("init_b", dev[0])
        ctx.kernel("init_u", dev[4])
        ctx.time_steps(*dev, 3)
        out.append([ctx.get_vec(dev[0]), ctx.get_vec(dev[1]), ctx.get_scalar(dev[6], n=2)])
    tol = 2e-6 if c.get("real") == "float" else 1e-13
    mb = float(np.abs(out[1][0]).max())
    for i in (0, 1):
        fl = rounding_floor(c, "register", mb, 1.0, stages_of(c, 3)) if i == 1 else 0.0
        ok, e = field_ok(out[0][i], out[1][i], tol, fl)
        assert ok, (i, e)
    np.testing.assert_array_equal(out[0][2], out[1][2])    # time bookkeeping by the band kernel
    assert np.isfinite(out[1][0]).all()


@pytest.mark.parametrize("case", ["box_4c_wsd0", "box_6e_wsd0", "box_2c_wsln", "periodic_4c_wsd0"])
def test_cg_pass_a_forms_agree(case):
    # the CG's pass A as the 2.5D z march (default) and as per-node gathers: the same
    # Laplacian values per node; the dot products' block partials differ, so the fields agree
    # to the CG parity tolerance with the same iteration count (ragged tiles: 37 x 21 x 30)
    order = int(case.split("_")[1][0])
    c = dict(order=order, extended=case.split("_")[1].endswith("e"), testcase="confined_domain", nodes=(37, 21, 30),
             lo=0.0, hi=1.0, laplace={"wsd0": "WIDE_STENCIL_DIRICHLET", "wsln": "WIDE_STENCIL_LNS"}[case.split("_")[2]],
             bnodes=0 if case.endswith("wsln") else 1, periodic=case.startswith("periodic"))
    out = []
    for form in (2, 1):
        ctx = maps_for(dict(c, cg_pass_a=form)).context()
        b = ctx.vec()
        ctx.kernel("init_b", b)
        bh = ctx.get_vec(b)
        bh[: ctx.n, :3] += NOISE_AMPLITUDE * np.random.default_rng(NOISE_SEED).random((ctx.n, 3))
        db = ctx.vec(bh)
        res = ctx.clean_div(db, 30, 1e-13, check=False)
        out.append((res["iterations"], res["residual_norm2"], ctx.get_vec(db)))
        ctx.close()
    assert out[0][0] == out[1][0]
    assert abs(out[0][1] - out[1][1]) <= 1e-6 * out[1][1]
    assert rel_err(out[0][2], out[1][2]) <= 1e-11


def test_cg_host_loop_equals_graph_loop():
    # IEQ_CG_LOOP=HOST (the profiling form: the iterations launched one after another) runs the
    # same kernels in the same order as the graph loop node: identical fields and counts
    c = dict(order=4, testcase="confined_domain", nodes=(20, 18, 22), lo=0.0, hi=1.0,
             laplace="WIDE_STENCIL_DIRICHLET", bnodes=1)
    out = []
    for loop in ("GRAPH", "HOST"):
        m = maps_for(c)
        m.I_Tech["cg_loop"] = loop
        ctx = m.context()
        b = ctx.vec()
        ctx.kernel("init_b", b)
        bh = ctx.get_vec(b)
        bh[: ctx.n, :3] += NOISE_AMPLITUDE * np.random.default_rng(NOISE_SEED).random((ctx.n, 3))
        db = ctx.vec(bh)
        res = ctx.clean_div(db, 25, 1e-9, check=False)
        out.append((res["iterations"], res["residual_norm2"], ctx.get_vec(db)))
        ctx.close()
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1]
    np.testing.assert_array_equal(out[0][2], out[1][2])


def test_cg_on_a_grid_beyond_65536_blocks_runs_and_reduces_the_divergence():
    # 290^3 (a 288^3 CG interior: 93,312 blocks of the pointwise pass, more than the 65,536
    # partials the reduction buffers held before they were sized from the grid): the graph
    # loop and the host loop give the same fields, and the residual falls
    c = dict(order=4, testcase="confined_domain", nodes=(290, 290, 290), lo=0.0, hi=1.0,
             laplace="WIDE_STENCIL_DIRICHLET", bnodes=1)
    out = []
    for loop in ("GRAPH", "HOST"):
        m = maps_for(c)
        m.I_Tech["cg_loop"] = loop
        ctx = m.context()
        b = ctx.vec()
        ctx.kernel("init_b", b)
        bh = ctx.get_vec(b)
        bh[: ctx.n, :3] += NOISE_AMPLITUDE * np.random.default_rng(NOISE_SEED).random((ctx.n, 3))
        db = ctx.vec(bh)
        res = ctx.clean_div(db, 12, 1e-30, check=False)
        out.append((res["iterations"], res["residual_norm2"], res["divergence_norm_initial"], ctx.get_vec(db)))
        ctx.close()
    assert out[0][0] == out[1][0] == 12 and out[0][1] == out[1][1]
    assert out[0][1] < 1e-2 * out[0][2] ** 2
    np.testing.assert_array_equal(out[0][3], out[1][3])


FLUX_FORMS = [(ui, so, uj) for ui in ("CENTRAL", "SPLIT", "PRODUCT") for so in ("ZERO", "CENTRAL", "SPLIT")
              for uj in ("CENTRAL", "SPLIT", "PRODUCT")]


@pytest.mark.parametrize("uibj, source, ujbi", FLUX_FORMS)
def test_every_flux_form_combination_matches_oracle(uibj, source, ujbi):
    # the 27 combinations of USE_UIBJ_* / USE_SOURCE_* / USE_UJBI_* (induction_Eq_volume.cl:
    # 13-212) with convection (rigid rotation on a box, inflow SAT), one SSPRK33 step through
    # the fused path and through the reference kernel list, against the oracle
    c = dict(order=4, testcase="rotation_gaussian", nodes=(12, 13, 11), lo=-1.0, hi=1.0, integrator="SSPRK33",
             dt=0.01, uibj=uibj, source=source, ujbi=ujbi)
    o = oracle_for(c)
    b, u = o.vec(), o.vec()
    o.run("init_b", o.cfg.nodes, b)
    o.run("init_u", o.cfg.nodes, u)
    b[:, :3] += 1e-2 * np.random.default_rng(NOISE_SEED).standard_normal((o.N, 3))
    host = [b.copy(), o.vec(), o.vec(), o.vec(), u, o.scalar(fill=1.0), np.zeros(2)]
    time_loop(o, "SSPRK33", False, False, 1, host[0], host[1], host[2], host[3], host[4], host[5], host[6])
    for kernel in ("AUTO", "LIST"):
        ctx = maps_for(dict(c, stage_kernel=kernel)).context()
        dev = [ctx.vec(b), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(u), ctx.scalar(np.ones(ctx.n_pad)),
               ctx.scalar(np.zeros(2), n=2)]
        ctx.time_steps(*dev, 1)
        for i in (0, 1, 2):
            e = rel_err(ctx.get_vec(dev[i])[: o.N], host[i])
            assert e <= 1e-12, (kernel, i, e)
        ctx.close()
