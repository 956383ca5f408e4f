"""Precision form on the GPU: FP32 state and stencils, FP64 divergence cleaning.

The confined-domain Hall case (include/confined_domain.h) plus seeded 1e-3 uniform noise is
cleaned by CG to ||r||_2 < 1e-10 (the FP64 CG of ieq_clean_div) and then advanced; the FP32
run is compared with the FP64 run of the same inputs."""
from __future__ import annotations

import numpy as np
import pytest

from tests.golden.cases import NOISE_AMPLITUDE, NOISE_SEED
from tests.helpers import maps_for, rel_err

pytestmark = pytest.mark.gpu

CASE = dict(order=4, testcase="confined_domain", nodes=(24, 24, 24), lo=0.0, hi=1.0, hall=True,
            integrator="CarpenterKennedy2N54", dt=2e-5, laplace="WIDE_STENCIL_DIRICHLET", bnodes=1)


def _run(real: str):
    c = dict(CASE, real=real)
    ctx = maps_for(c).context()
    b = ctx.vec()
    ctx.kernel("init_b", b)
    bh = ctx.get_vec(b).astype(np.float64)
    rng = np.random.default_rng(NOISE_SEED)
    bh[: ctx.n, :3] += NOISE_AMPLITUDE * rng.random((ctx.n, 3))
    b.upload(bh.astype(ctx.real))
    res = ctx.clean_div(b, 5000, 1e-10)
    cleaned = ctx.get_vec(b).astype(np.float64)
    b2, cb, u = ctx.vec(), ctx.vec(), ctx.vec()
    ctx.kernel("init_u", u)
    rho = ctx.scalar(np.ones(ctx.n_pad))
    t = ctx.scalar(np.zeros(2), n=2)
    ctx.time_steps(b, b2, None, cb, u, rho, t, 3)
    wv, ws = ctx.vec(), ctx.scalar()
    out = ctx.results(b, 3 * c["dt"], wv, ws)
    return res, cleaned, ctx.get_vec(b).astype(np.float64), out


def test_fp32_state_with_fp64_cg_matches_fp64_run():
    r64, c64, s64, o64 = _run("double")
    r32, c32, s32, o32 = _run("float")
    # both solves reach the FP64 CG criterion
    assert r64["converged"] and r32["converged"]
    assert r64["residual_norm2"] <= 1e-20 and r32["residual_norm2"] <= 1e-20
    # the FP32 cleaned field and the stepped field agree with the FP64 run to FP32 accuracy
    assert rel_err(c32, c64) <= 5e-6
    assert rel_err(s32, s64) <= 5e-6
    # the mass-weighted ||div B|| over the whole grid (the Dirichlet CG cleans the interior
    # only) agrees between the two runs
    assert np.isfinite(o32["divergence_norm"]) and np.isfinite(o64["divergence_norm"])
    assert abs(o32["divergence_norm"] - o64["divergence_norm"]) <= 1e-3 * o64["divergence_norm"] + 1e-4
