"""The z-slab decomposition on the GPU: a slab (ghost planes refreshed by copies) runs the
fused stage kernels one RK stage at a time (ieq_stages_*) or the reference kernel lists
through the C ABI on torch device buffers; its owned planes equal the undecomposed run of the
same kernels bit for bit.  One slab (a periodic grid's ghosts wrap onto the slab itself), and
the 2 or 3 slabs of a decomposition held in one process on this GPU (`run_local`: every stage
runs on each slab in turn, then the ghost planes are copied between their buffers) -- periodic
grids and boxes, whose slabs carry ghost planes only at their inner ends.  The
variable-velocity case checks that the slab's testcase coordinates are the global grid's
(IEQ_Z_OFFSET / IEQ_NZ_GLOBAL).  Several processes are covered on CPU
(tests/test_decomp_cpu.py); this run has one GPU."""
from __future__ import annotations

import math

import numpy as np
import pytest

from inductioneq_b200 import ranks as R
from inductioneq_b200.decomp import SlabSolve, clean_div_local, run_local
from tests.helpers import maps_for

pytestmark = pytest.mark.gpu

CASES = {
    "whistler_6c_hod_ck": dict(order=6, testcase="hall_circular_wave", nodes=(32, 16, 24), lo=0.0, hi=2 * math.pi,
                               periodic=True, hall=True, dissipation="HIGH_ORDER",
                               integrator="CarpenterKennedy2N54", dt=0.004),
    "hallper_4c_varu_ssp": dict(order=4, testcase="hall_periodic", nodes=(12, 14, 16), lo=0.0, hi=4 * math.pi / 3,
                                periodic=True, hall=True, integrator="SSPRK33", dt=0.002, variable_u=True),
}

# boxes: the rotation with SAT inflow (convection pair kernels, x band) and the confined Hall
# box with the dissipation sum and the Hall outflow SAT
BOX_CASES = {
    "rot3d_4c_ssp_box": dict(order=4, testcase="rotation_3D", nodes=(40, 14, 36), lo=-1.0, hi=1.0,
                             integrator="SSPRK33", dt=0.005),
    "confined_6c_hall_hod_ck_box": dict(order=6, testcase="confined_domain", nodes=(16, 12, 40), lo=0.0, hi=1.0,
                                        hall=True, dissipation="HIGH_ORDER", integrator="CarpenterKennedy2N54",
                                        dt=1e-5),
}


def _undecomposed(c, fused, steps):
    g = maps_for(dict(c, stage_kernel="AUTO" if fused else "LIST")).context()
    b, u = g.vec(), g.vec()
    g.kernel("init_b", b)
    g.kernel("init_u", u)
    bh = g.get_vec(b)
    bh[: g.n, :3] += 1e-2 * np.random.default_rng(3).standard_normal((g.n, 3))
    uh = g.get_vec(u)
    dev = [g.vec(bh), g.vec(), g.vec(), g.vec(), g.vec(uh), g.scalar(np.ones(g.n_pad)), g.scalar(np.zeros(2), n=2)]
    g.time_steps(*dev, steps)
    ref = [g.get_vec(dev[i])[: g.n] for i in range(3)]
    t_ref = g.get_scalar(dev[6], n=2)
    n = g.n
    g.close()
    return bh[:n], uh[:n], ref, t_ref


@pytest.mark.parametrize("fused", [False, True])
@pytest.mark.parametrize("name", sorted(CASES))
def test_single_slab_equals_undecomposed_run(name, fused):
    # fused: the slab steps through the fused stage kernels one RK stage at a time
    # (ieq_stages_*), the undecomposed grid through ieq_time_steps' fused path; else both run
    # the reference kernel lists
    c = CASES[name]
    steps = 3
    g = maps_for(dict(c, stage_kernel="AUTO" if fused else "LIST")).context()
    b, u = g.vec(), g.vec()
    g.kernel("init_b", b)
    g.kernel("init_u", u)
    bh = g.get_vec(b)
    bh[: g.n, :3] += 1e-2 * np.random.default_rng(3).standard_normal((g.n, 3))
    uh = g.get_vec(u)
    dev = [g.vec(bh), g.vec(), g.vec(), g.vec(), g.vec(uh), g.scalar(np.ones(g.n_pad)), g.scalar(np.zeros(2), n=2)]
    g.time_steps(*dev, steps)
    ref = [g.get_vec(dev[i])[: g.n] for i in range(3)]
    t_ref = g.get_scalar(dev[6], n=2)
    s = SlabSolve(maps_for(c), R.Ranks(1, 0, 0))
    s.load(bh[: g.n], uh[: g.n], np.ones(g.n))
    s.steps(steps, fused=fused)
    np.testing.assert_array_equal(s.owned(s.b), ref[0])
    np.testing.assert_array_equal(s.owned(s.b2), ref[1])
    if s.nf == 3:
        np.testing.assert_array_equal(s.owned(s.b3), ref[2])
    np.testing.assert_array_equal(s.time.cpu().numpy(), t_ref)
    s.close()
    g.close()


@pytest.mark.parametrize("fused", [False, True])
@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name", sorted(BOX_CASES) + ["whistler_6c_hod_ck"])
def test_slabs_of_one_process_equal_undecomposed_run(name, world, fused):
    c = BOX_CASES.get(name) or CASES[name]
    steps = 3
    bh, uh, ref, t_ref = _undecomposed(c, fused, steps)
    solves = [SlabSolve(maps_for(c), R.Ranks(world, r, r)) for r in range(world)]
    try:
        if not c.get("periodic"):
            assert solves[0].slabs.g_lo == 0 and solves[-1].slabs.g_hi == 0
        for s in solves:
            s.load(bh, uh, np.ones(bh.shape[0]))
        run_local(solves, steps, fused=fused)
        covered = 0
        for s in solves:
            rows = s.slabs.global_rows()
            np.testing.assert_array_equal(s.owned(s.b), ref[0][rows])
            np.testing.assert_array_equal(s.owned(s.b2), ref[1][rows])
            if s.nf == 3:
                np.testing.assert_array_equal(s.owned(s.b3), ref[2][rows])
            np.testing.assert_array_equal(s.time.cpu().numpy(), t_ref)
            covered += rows.stop - rows.start
        assert covered == bh.shape[0]
    finally:
        for s in solves:
            s.close()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("laplace", ["WIDE_STENCIL_DIRICHLET", "NARROW_STENCIL_DIRICHLET", "WIDE_STENCIL_LNS"])
def test_decomposed_cleaning_equals_undecomposed_cleaning(laplace, world):
    # clean_div.m's CG through the reference kernels on 2 or 3 slabs of a confined box (ghost
    # planes of u, phi and B copied between the slabs, dot products of the owned planes by
    # ieq_dot_range added in rank order) against the same host loop on the whole grid: the
    # same iterations and residual history, B equal up to the order of the dots' sums
    c = dict(order=4, testcase="confined_domain", nodes=(24, 20, 36), lo=0.0, hi=1.0, hall=True, dt=1e-5,
             laplace=laplace)
    iters, thr = 25, 1e-14
    g = maps_for(c).context()
    b = g.vec()
    g.kernel("init_b", b)
    bh = g.get_vec(b)[: g.n]
    bh[:, :3] += 1e-3 * np.random.default_rng(5).standard_normal((g.n, 3))
    g.close()
    whole = SlabSolve(maps_for(c), R.Ranks(1, 0, 0))
    solves = [SlabSolve(maps_for(c), R.Ranks(world, r, r)) for r in range(world)]
    try:
        whole.load(bh)
        ref = clean_div_local([whole], iters, thr)
        b_ref = whole.owned(whole.b)
        for s in solves:
            s.load(bh)
        got = clean_div_local(solves, iters, thr)
        assert got["iterations"] == ref["iterations"] == iters
        np.testing.assert_allclose(got["history"], ref["history"], rtol=1e-10)
        assert ref["history"][-1] < 1e-2 * ref["history"][0]
        scale = np.abs(bh[:, :3]).max()
        for s in solves:
            rows = s.slabs.global_rows()
            assert np.abs(s.owned(s.b)[:, :3] - b_ref[rows, :3]).max() <= 1e-12 * scale
        # B moved by the projection
        assert np.abs(b_ref[:, :3] - bh[:, :3]).max() > 1e-6 * scale
    finally:
        whole.close()
        for s in solves:
            s.close()


def test_dot_range_equals_dot_of_the_range():
    # ieq_dot_range over a sub-range against the dot of the same elements; a range beyond the
    # grid is refused
    from inductioneq_b200.lib import IeqError
    c = CASES["whistler_6c_hod_ck"]
    ctx = maps_for(c).context()
    rng = np.random.default_rng(9)
    x, y = rng.standard_normal(ctx.n_pad), rng.standard_normal(ctx.n_pad)
    dx, dy = ctx.scalar(x), ctx.scalar(y)
    first, count = 1000, ctx.n - 3000
    got = ctx.dot_range(dx, dy, first, count)
    want = float(np.dot(x[first:first + count], y[first:first + count]))
    assert abs(got - want) <= 1e-12 * abs(np.abs(x[first:first + count] * y[first:first + count]).sum())
    assert ctx.dot_range(dx, dy, 0, ctx.n) == ctx.dot(dx, dy)
    assert ctx.dot_range(dx, dy, 5, 0) == 0.0
    with pytest.raises(IeqError):
        ctx.dot_range(dx, dy, ctx.n - 10, 11)
    ctx.close()


def test_stage_api_refuses_misuse():
    # ieq_stages_*: a stage outside begin/end, an index out of range, a second begin, a LIST
    # context; a full step through every stage equals ieq_time_steps
    from inductioneq_b200.lib import IeqError
    c = CASES["whistler_6c_hod_ck"]
    ctx = maps_for(c).context()
    b, b2, cb, u = ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec()
    rho, t = ctx.scalar(np.ones(ctx.n_pad)), ctx.scalar(np.zeros(2), n=2)
    ctx.kernel("init_b", b)
    with pytest.raises(IeqError):
        ctx.stages_run(rho, t, 0)
    ns = ctx.stages_begin(b, b2, None, cb, u)
    assert ns == 5                                  # CarpenterKennedy2N54
    with pytest.raises(IeqError):
        ctx.stages_begin(b, b2, None, cb, u)
    for bad in (-1, ns):
        with pytest.raises(IeqError):
            ctx.stages_run(rho, t, bad)
    for s in range(ns):
        ctx.stages_run(rho, t, s)
    ctx.stages_end(b, b2, None, cb, u, rho)
    ref = maps_for(c).context()
    rb, rb2, rcb, ru = ref.vec(), ref.vec(), ref.vec(), ref.vec()
    rt = ref.scalar(np.zeros(2), n=2)
    ref.kernel("init_b", rb)
    ref.time_steps(rb, rb2, None, rcb, ru, ref.scalar(np.ones(ref.n_pad)), rt, 1)
    np.testing.assert_array_equal(ctx.get_vec(b), ref.get_vec(rb))
    np.testing.assert_array_equal(ctx.get_vec(b2), ref.get_vec(rb2))
    np.testing.assert_array_equal(ctx.get_scalar(t, n=2), ref.get_scalar(rt, n=2))
    ref.close()
    ctx.close()
    lst = maps_for(dict(c, stage_kernel="LIST")).context()
    with pytest.raises(IeqError):
        lst.stages_begin(lst.vec(), lst.vec(), None, lst.vec(), lst.vec())
    lst.close()
