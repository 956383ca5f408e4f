"""The z-marching kernels of stage_z.cuh -- the one-pass Hall stage (curl, E = J x B,
dissipation and update in one kernel) and the 2.5D curl kernel -- against the two-kernel
column path, the reference kernel lists and the oracle; and the dissipation sum formed in
the stage kernel (IEQ_HODP=0) against the curl kernel's.

IEQ_STAGE_KERNEL=ZMARCH forces it on grids where it can run (periodic, nx a multiple of 32,
ny of 16); IEQ_ZMARCH_TZ sets the z planes per CTA (1: every CTA a single plane after a
2*RI-plane prologue; nz: one chunk).  It forms every node's sums in the order of the pair
kernels, so the fields agree with them to 1e-13 of their own scale, the RK registers and the
curl buffer with the forward-error floor of a derivative of the state (tests/helpers.py).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle.hostloops import time_loop
from oracle.sequencing import NUM_FIELDS
from tests.golden.cases import NOISE_SEED
from tests.helpers import field_ok, maps_for, oracle_for, rounding_floor, stages_of

pytestmark = pytest.mark.gpu
TWO_PI = 2.0 * math.pi


def _case(order=6, extended=False, hod=True, nodes=(64, 32, 20), real="double", integrator="CarpenterKennedy2N54",
          dt=0.004):
    c = dict(order=order, extended=extended, testcase="hall_circular_wave", nodes=nodes, lo=0.0, hi=TWO_PI,
             periodic=True, hall=True, integrator=integrator, dt=dt, real=real)
    if hod:
        c["dissipation"] = "HIGH_ORDER"
    return c


def _run(c, kernel, steps, tz=None, rho_noise=0.0):
    ctx = maps_for(dict(c, stage_kernel=kernel, zmarch_tz=tz)).context()
    b = ctx.vec()
    ctx.kernel("init_b", b)
    bh = ctx.get_vec(b).astype(np.float64)
    rng = np.random.default_rng(NOISE_SEED)
    bh[: ctx.n, :3] += 1e-2 * rng.standard_normal((ctx.n, 3))
    rho = np.ones(ctx.n_pad)
    if rho_noise:
        rho[: ctx.n] += rho_noise * rng.random(ctx.n)
    dev = [ctx.vec(bh.astype(ctx.real)), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.scalar(rho),
           ctx.scalar(np.zeros(2), n=2)]
    ctx.time_steps(*dev, steps)
    out = [ctx.get_vec(dev[i]).astype(np.float64) for i in range(4)] + [ctx.get_scalar(dev[6], n=2)]
    ctx.close()
    return out


def _same(c, a, b, steps, rtol):
    nf = NUM_FIELDS[c["integrator"]]
    mb = float(np.abs(b[0]).max())
    ns = stages_of(c, steps)
    for i in ([0, 1, 2, 3] if nf == 3 else [0, 1, 3]):
        reg = (i == 1 and nf == 2) or (i == 2 and c["integrator"] in ("KennedyCarpenterLewis2R54C",
                                                                       "CalvoFrancoRandez2R64"))
        fl = rounding_floor(c, "register", mb, 0.0, ns) if reg else (
            rounding_floor(c, "curl", mb, 0.0, ns) if i == 3 else 0.0)
        ok, e = field_ok(a[i], b[i], rtol, fl)
        assert ok, (i, e)
    np.testing.assert_allclose(a[4], b[4], rtol=1e-15 if c.get("real") != "float" else 1e-6)


@pytest.mark.parametrize("order, extended", [(2, False), (4, False), (6, False), (4, True), (6, True)])
@pytest.mark.parametrize("hod", [True, False])
@pytest.mark.parametrize("tz", [1, 5, None])
def test_zmarch_equals_column_kernels(order, extended, hod, tz):
    c = _case(order, extended, hod)
    a = _run(c, "ZMARCH", 3, tz)
    b = _run(c, "COLUMN", 3)
    _same(c, a, b, 3, 1e-13)


@pytest.mark.parametrize("real", ["double", "float"])
@pytest.mark.parametrize("integrator", ["SSPRK33", "SSPRK104", "KennedyCarpenterLewis2R54C", "CalvoFrancoRandez2R64",
                                        "CarpenterKennedy2N54", "ToulorgeDesmet2N84F"])
def test_zmarch_equals_reference_kernel_lists_for_every_integrator(integrator, real):
    c = _case(6, False, True, nodes=(32, 16, 14), real=real, integrator=integrator, dt=0.005)
    a = _run(c, "ZMARCH", 3, 4)
    b = _run(c, "LIST", 3)
    _same(c, a, b, 3, 1e-12 if real == "double" else 2e-6)


def test_zmarch_with_variable_rho_equals_column_kernels():
    c = _case(4, False, True, nodes=(64, 16, 18))
    a = _run(c, "ZMARCH", 2, 7, rho_noise=0.3)
    b = _run(c, "COLUMN", 2, rho_noise=0.3)
    _same(c, a, b, 2, 1e-13)


@pytest.mark.parametrize("real", ["double", "float"])
def test_zmarch_matches_oracle(real):
    c = _case(6, False, True, nodes=(64, 32, 20), real=real, dt=0.004)
    ctx = maps_for(dict(c, stage_kernel="ZMARCH", zmarch_tz=6)).context()
    o = oracle_for(c)
    b = ctx.vec()
    ctx.kernel("init_b", b)
    bh = ctx.get_vec(b).astype(np.float64)
    bh[: ctx.n, :3] += 1e-2 * np.random.default_rng(NOISE_SEED).standard_normal((ctx.n, 3))
    bh = bh.astype(o.T)
    host = [bh.copy(), np.zeros_like(bh), np.zeros_like(bh), np.zeros_like(bh), np.zeros_like(bh),
            np.ones(o.N, dtype=o.T), np.zeros(2, dtype=o.T)]
    dev = [ctx.vec(host[0]), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.scalar(np.ones(ctx.n_pad)),
           ctx.scalar(np.zeros(2), n=2)]
    steps = 2
    time_loop(o, c["integrator"], True, False, steps, host[0], host[1], None, host[3], host[4], host[5], host[6])
    ctx.time_steps(*dev, steps)
    mb = float(np.abs(host[0]).max())
    ns = stages_of(c, steps)
    tol = 1e-12 if real == "double" else 2e-5
    for i, kind in ((0, None), (1, "register"), (3, "curl")):
        fl = rounding_floor(c, kind, mb, 0.0, ns) if kind else 0.0
        ok, e = field_ok(ctx.get_vec(dev[i]), host[i], tol, fl)
        assert ok, (i, e)
    np.testing.assert_allclose(ctx.get_scalar(dev[6], n=2), host[6], rtol=1e-15 if real == "double" else 1e-6)
    ctx.close()


@pytest.mark.parametrize("order, extended", [(2, False), (4, False), (6, False), (6, True)])
@pytest.mark.parametrize("hod", [True, False])
@pytest.mark.parametrize("real", ["double", "float"])
def test_curl_z_march_equals_pair_curl_kernel(order, extended, hod, real):
    # the 2.5D curl kernel (IEQ_CURL_Z=1) against the pair curl kernel (IEQ_CURL_Z=0) on a
    # periodic grid with partial tiles in x and y (36 x 20 x 17): the same sums per node
    c = _case(order, extended, hod, nodes=(36, 20, 17), real=real)
    out = []
    for cz in (1, 0):
        out.append(_run(dict(c, curl_z=cz), "COLUMN", 3))
    _same(c, out[0], out[1], 3, 1e-13 if real == "double" else 2e-6)


@pytest.mark.parametrize("hodp", [0, 1])
def test_dissipation_sum_in_stage_or_curl_kernel_agree(hodp):
    # IEQ_HODP=0: the stage kernel gathers the dissipation rows itself instead of reading the
    # curl kernel's sum; the same terms per node
    c = _case(6, False, True, nodes=(32, 18, 20))
    a = _run(dict(c, hodp=hodp), "COLUMN", 3)
    b = _run(dict(c, hodp=1), "COLUMN", 3)
    _same(c, a, b, 3, 1e-13)
