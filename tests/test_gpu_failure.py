"""Failure paths on the GPU, made on purpose and safely: every wait that gives up here is a
bounded wait whose limit runs out while nothing is faulty on the device, and the context
stays usable afterwards.

* the persistent batched kernel's grid barrier is told to wait for one block more than the
  grid has (a block that never arrives): every wait runs out after a short spin limit, the
  run returns IEQ_ERR_TIMEOUT, and the next run (production barrier) succeeds and gives the
  same solution as a batch that never timed out;
* the TMA brick kernels' first wait for their halo copies gives up at once: the bricks wait
  for their copies before they leave, ieq_time_steps returns IEQ_ERR_TIMEOUT, and the next
  call succeeds;
* the CG divergence cleaning capped below convergence returns IEQ_ERR_NOT_CONVERGED with B
  still projected (equal to the reference loop capped the same way);
* a non-finite value written into a host input is reported as IEQ_ERR_NAN.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from inductioneq_b200.batch import Batch
from inductioneq_b200.lib import IeqError
from oracle.hostloops import clean_div
from tests.golden.cases import CG_CASES, NOISE_SEED
from tests.helpers import maps_for, oracle_for, rel_err

pytestmark = pytest.mark.gpu

SPECS = [(16, 2, 0.7, 0.5 * (2 / 15) / (0.7 * math.sqrt(2))),
         (13, 6, 1.9, 0.5 * (2 / 12) / (1.9 * math.sqrt(2))),
         (20, 4, 1.2, 0.5 * (2 / 19) / (1.2 * math.sqrt(2)))]


def _batch_result(bt, steps, mode="persistent"):
    bt.init()
    bt.bind()
    bt.run(steps, mode=mode)
    bt.unbind()
    return [c.get_vec(f["b"]) for c, f in zip(bt.ctxs, bt.fields)]


def test_batched_grid_barrier_wait_runs_out_then_next_run_succeeds():
    bt = Batch(SPECS)
    ref = _batch_result(bt, 3)
    bt.test_barrier(1, 20000)          # one phantom arrival; ~1.3 ms per wait
    bt.init()
    bt.bind()
    with pytest.raises(IeqError) as e:
        bt.run(3, mode="persistent")
    assert e.value.name == "IEQ_ERR_TIMEOUT"
    bt.test_barrier(0, 0)               # production barrier; the run resets its state
    got = _batch_result(bt, 3)
    for a, b in zip(got, ref):
        np.testing.assert_array_equal(a, b)
    bt.close()


def _brick_case():
    return dict(order=6, testcase="hall_circular_wave", nodes=(32, 16, 12), lo=0.0, hi=2.0 * math.pi, periodic=True,
                hall=True, dissipation="HIGH_ORDER", integrator="CarpenterKennedy2N54", dt=0.01, stage_kernel="BRICK")


def _brick_fields(ctx):
    b = ctx.vec()
    ctx.kernel("init_b", b)
    return [b, ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.scalar(np.ones(ctx.n_pad)),
            ctx.scalar(np.zeros(2), n=2)]


def test_brick_first_wait_gives_up_then_next_call_succeeds():
    c = _brick_case()
    ctx = maps_for(c).context()
    ctx.test_brick_wait(True)
    with pytest.raises(IeqError) as e:
        ctx.time_steps(*_brick_fields(ctx), 1)
    assert e.value.name == "IEQ_ERR_TIMEOUT"
    assert "did not complete in time" in str(e.value)
    ctx.test_brick_wait(False)
    dev = _brick_fields(ctx)
    ctx.time_steps(*dev, 2)
    got = ctx.get_vec(dev[0])
    col = maps_for(dict(c, stage_kernel="COLUMN")).context()
    devc = _brick_fields(col)
    col.time_steps(*devc, 2)
    assert rel_err(got, col.get_vec(devc[0])) <= 1e-12
    ctx.close()
    col.close()


def test_clean_div_cap_returns_not_converged_with_b_projected():
    c = CG_CASES["cg_4c_wsd0"]
    ctx = maps_for(c).context()
    o = oracle_for(c)
    b = ctx.vec()
    ctx.kernel("init_b", b)
    bh = ctx.get_vec(b)
    bh[: ctx.n, :3] += 1e-3 * np.random.default_rng(NOISE_SEED).random((ctx.n, 3))
    ref = bh[: ctx.n].copy()
    r = clean_div(o, ref, 3, 1e-12, c["bnodes"])
    assert r["iterations"] == 3
    db = ctx.vec(bh)
    with pytest.raises(IeqError) as e:
        ctx.clean_div(db, 3, 1e-12, check=True)
    assert e.value.name == "IEQ_ERR_NOT_CONVERGED"
    got = ctx.get_vec(db)[: ctx.n]
    assert rel_err(got, ref) <= 1e-11          # projected after the third iteration
    assert rel_err(got, bh[: ctx.n]) > 1e-8    # B changed
    ctx.close()


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_non_finite_input_is_reported(bad):
    c = dict(order=4, testcase="rotation_gaussian", nodes=(12, 13, 14), lo=-1.0, hi=1.0, integrator="SSPRK33",
             dt=0.02)
    ctx = maps_for(c).context()
    b = ctx.vec()
    ctx.kernel("init_b", b)
    ctx.check_finite(b)                          # a finite field passes
    bh = ctx.get_vec(b)
    bh[ctx.n // 2, 1] = bad                      # one component of one node, on the host
    bad_b = ctx.vec(bh)
    with pytest.raises(IeqError) as e:
        ctx.check_finite(bad_b)
    assert e.value.name == "IEQ_ERR_NAN"
    # the context stays usable
    ctx.check_finite(b)
    ctx.close()
