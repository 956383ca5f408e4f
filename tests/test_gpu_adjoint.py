"""Discrete adjoint on the GPU.

* transpose tests: <w, F'(b) v> = <F'(b)^T w, v> for the tangent-linear and adjoint spatial
  operators of several configurations (relative 1e-12);
* the tangent against central differences of the forward operator;
* the checkpointed SSPRK33 gradient of a final-time L2 misfit against central differences
  along seeded random directions (Richardson-extrapolated, relative 1e-6), driven through a torch.autograd.Function
  (defined here, in the test harness only);
* the same for the 2N low-storage schemes (CarpenterKennedy2N54, ToulorgeDesmet2N84F), for the
  2R schemes and SSPRK104 (the step's register program reversed), and for Hall on boxes (the
  outflow SAT) and first-order and adaptive dissipation.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from tests.helpers import maps_for

pytestmark = pytest.mark.gpu

HP = 4.0 * math.pi / 3.0
CASES = {
    "hallper_4c": dict(order=4, testcase="hall_periodic", nodes=(16, 17, 18), lo=0.0, hi=HP, periodic=True, hall=True,
                       integrator="SSPRK33", variable_u=True),
    "hallper_6c_hod": dict(order=6, testcase="hall_periodic", nodes=(16, 16, 16), lo=0.0, hi=HP, periodic=True,
                           hall=True, dissipation="HIGH_ORDER", integrator="SSPRK33"),
    "rot_6c_sat": dict(order=6, testcase="rotation_gaussian", nodes=(14, 15, 16), lo=-1.0, hi=1.0,
                       integrator="SSPRK33"),
    "rot3d_4e_split_hod": dict(order=4, extended=True, testcase="rotation_3D", nodes=(14, 13, 15), lo=-1.0, hi=1.0,
                               uibj="SPLIT", source="SPLIT", ujbi="PRODUCT", dissipation="HIGH_ORDER",
                               integrator="SSPRK33"),
    # Hall on boxes: the Hall outflow SAT (induction_Eq_surface.cl:35-81) on every face
    "travel_6c_hall_box": dict(order=6, testcase="hall_travelling_wave", nodes=(14, 15, 16), lo=0.0, hi=6.283185307179586,
                               hall=True, integrator="SSPRK33"),
    # (u . n = 0 on the walls and curl(B) . n = 0 on the box edges: the outflow switch sits at
    # tv = 0 there, where it has no derivative; seeded noise on B moves the state off it)
    "confined_4c_hall_fo": dict(order=4, testcase="confined_domain", nodes=(15, 14, 13), lo=0.0, hi=1.0, hall=True,
                                dissipation="FIRST_ORDER", integrator="SSPRK33", noise=1e-2),
    # first-order dissipation with convection only (its weights max(|u_j|, |u_k|) are fixed)
    "rot_2c_fo": dict(order=2, testcase="rotation_gaussian", nodes=(13, 12, 11), lo=-1.0, hi=1.0,
                      dissipation="FIRST_ORDER", integrator="SSPRK33"),
    # adaptive dissipation: weights kappa(max|u| (b_j - b_k)^2) with a square root between two
    # thresholds -- noise of amplitude 1 puts 40-50 % of the stencil pairs between them, the
    # seeds keep every pair at least 1e-4 (relative) from a threshold, where kappa has no
    # derivative
    "rot_2c_ad": dict(order=2, testcase="rotation_gaussian", nodes=(13, 12, 11), lo=-1.0, hi=1.0,
                      dissipation="ADAPTIVE", integrator="SSPRK33", noise=1.0, noise_seed=25),
    # (with B noise of amplitude 1 the explicit Hall term needs a smaller step than 1e-3)
    "confined_4c_hall_ad": dict(order=4, testcase="confined_domain", nodes=(15, 14, 13), lo=0.0, hi=1.0, hall=True,
                                dissipation="ADAPTIVE", integrator="SSPRK33", noise=1.0, noise_seed=29,
                                sweep_dt=1e-5),
}


def _noisy(ctx, b, c):
    """B plus the case's seeded noise (off the outflow switch's non-smooth points)."""
    if c.get("noise"):
        bh = ctx.get_vec(b)
        bh[: ctx.n, :3] += c["noise"] * np.random.default_rng(c.get("noise_seed", 23)).standard_normal((ctx.n, 3))
        b.upload(bh)


def _setup(c, dt=1.0):
    ctx = maps_for(dict(c, dt=dt)).context()
    b, u = ctx.vec(), ctx.vec()
    ctx.kernel("init_b", b)
    _noisy(ctx, b, c)
    ctx.kernel("init_u", u)
    rho = ctx.scalar(np.ones(ctx.n_pad))
    return ctx, b, u, rho


def _rand(ctx, seed):
    r = np.random.default_rng(seed).standard_normal((ctx.n_pad, 4))
    r[:, 3] = 0
    r[ctx.n:] = 0
    return r


def _dot(a, b):
    return float(np.sum(a[:, :3] * b[:, :3]))


@pytest.mark.parametrize("name", sorted(CASES))
def test_operator_transpose(name):
    ctx, b, u, rho = _setup(CASES[name])
    v, w = _rand(ctx, 1), _rand(ctx, 2)
    dv, dw, jv, jtw = ctx.vec(v), ctx.vec(w), ctx.vec(), ctx.vec()
    ctx.operator_jvp(b, dv, u, rho, jv)
    ctx.operator_vjp(b, dw, u, rho, jtw)
    lhs = _dot(w, ctx.get_vec(jv))
    rhs = _dot(ctx.get_vec(jtw), v)
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs)), (lhs, rhs)


def _F(ctx, b, u, rho, hall):
    """DB(b) through the reference kernels (CarpenterKennedy2N54_1a: b2 = DT*DB(b1), DT = 1)."""
    b2, cb, t = ctx.vec(), ctx.vec(), ctx.scalar(np.zeros(2), n=2)
    names = (["calc_curlB_rho_1_2args"] if hall else []) + ["CarpenterKennedy2N54_1a"]
    ctx.run(names, ctx_nodes(ctx), b, b2, cb, u, rho, t)
    return ctx.get_vec(b2)


def ctx_nodes(ctx):
    return ctx._nodes


@pytest.mark.parametrize("name", ["hallper_4c", "rot_6c_sat", "travel_6c_hall_box", "confined_4c_hall_fo", "rot_2c_fo",
                                  "rot_2c_ad", "confined_4c_hall_ad"])
def test_tangent_matches_central_differences(name):
    c = dict(CASES[name], integrator="CarpenterKennedy2N54")
    ctx, b, u, rho = _setup(c)
    ctx._nodes = c["nodes"]
    b0 = ctx.get_vec(b)
    v = _rand(ctx, 3) * 1e-2
    jv = ctx.vec()
    ctx.operator_jvp(b, ctx.vec(v), u, rho, jv)
    eps = 1e-4
    fp = _F(ctx, ctx.vec(b0 + eps * v), u, rho, c.get("hall", False))
    fm = _F(ctx, ctx.vec(b0 - eps * v), u, rho, c.get("hall", False))
    fd = (fp - fm) / (2 * eps)
    got = ctx.get_vec(jv)
    assert np.abs(fd - got)[:, :3].max() <= 1e-6 * np.abs(got[:, :3]).max()


def _c5_small():
    c = dict(CASES["hallper_4c"], nodes=(16, 16, 16))
    ctx = maps_for(dict(c, dt=1.0)).context()
    u = ctx.vec()
    ctx.kernel("init_u", u)
    umax = float(np.sqrt((ctx.get_vec(u)[:, :3] ** 2).sum(1)).max())
    dx = HP / 16
    dt = (2.0 / 16) * dx / umax        # CFL 2/N (compute_error_hall_periodic.m:51)
    ctx.close()
    return maps_for(dict(c, dt=dt)).context(), dt


def test_checkpointed_gradient_matches_central_differences_via_autograd():
    torch = pytest.importorskip("torch")
    ctx, dt = _c5_small()
    nsteps, every = 12, 5
    b = ctx.vec()
    ctx.kernel("init_b", b)
    u = ctx.vec()
    ctx.kernel("init_u", u)
    rho = ctx.scalar(np.ones(ctx.n_pad))
    b0 = ctx.get_vec(b)
    n = ctx.n

    def forward_np(x):
        bb, b2, b3, cb = ctx.vec(x), ctx.vec(), ctx.vec(), ctx.vec()
        uu = ctx.vec()
        ctx.kernel("init_u", uu)
        t = ctx.scalar(np.zeros(2), n=2)
        ctx.time_steps(bb, b2, b3, cb, uu, rho, t, nsteps)
        return ctx.get_vec(bb)

    class Evolve(torch.autograd.Function):
        """B(T) = Phi(B0) with the adjoint sweep as backward (test harness only)."""

        @staticmethod
        def forward(fctx, x):
            fctx.save_for_backward(x)
            return torch.from_numpy(forward_np(x.detach().cpu().numpy()))

        @staticmethod
        def backward(fctx, g):
            (x,) = fctx.saved_tensors
            lam = ctx.vec(g.detach().cpu().numpy())
            uu = ctx.vec()
            ctx.kernel("init_u", uu)
            ctx.adjoint_steps(ctx.vec(x.detach().cpu().numpy()), lam, uu, rho, nsteps, every)
            return torch.from_numpy(ctx.get_vec(lam))

    # mass weights of ||.||_M (kernel_operator.cl:22-28): periodic -> dx dy dz
    wmass = (HP / 16) ** 3
    rng = np.random.default_rng(2026)
    target = forward_np(b0) + 1e-3 * rng.standard_normal((ctx.n_pad, 4))
    target[:, 3] = 0
    target[n:] = 0
    tt = torch.from_numpy(target)

    def loss(x):
        d = Evolve.apply(x) - tt
        return 0.5 * wmass * (d[:, :3] ** 2).sum()

    x = torch.from_numpy(b0.copy()).requires_grad_(True)
    L = loss(x)
    L.backward()
    g = x.grad.numpy()
    def fd(d, eps):
        with torch.no_grad():
            Lp = float(loss(torch.from_numpy(b0 + eps * d)))
            Lm = float(loss(torch.from_numpy(b0 - eps * d)))
        return (Lp - Lm) / (2 * eps)

    for k in range(6):
        d = rng.standard_normal((ctx.n_pad, 4))
        d[:, 3] = 0
        d[n:] = 0
        d /= np.sqrt(np.sum(d[:, :3] ** 2))          # unit l2 direction
        ad = float(np.sum(g[:, :3] * d[:, :3]))
        # central differences converge as eps^2 onto the adjoint directional derivative; their
        # Richardson extrapolation (4 D(eps/2) - D(eps)) / 3 removes the eps^2 term
        f1, f2, f3 = fd(d, 1e-3), fd(d, 5e-4), fd(d, 1e-4)
        e1, e3 = abs(f1 - ad), abs(f3 - ad)
        assert e3 <= 0.05 * e1 or e3 <= 1e-9 * abs(ad), (k, e1, e3)
        rich = (4.0 * f2 - f1) / 3.0
        assert abs(rich - ad) <= 1e-6 * abs(ad), (k, rich, ad)


def test_repeated_sweeps_on_one_context_reuse_the_checkpoint_pool():
    # the checkpointed sweep keeps its work fields in the context: later calls with other
    # step counts and checkpoint spacings (smaller and larger pools) give the gradients of
    # a fresh context
    ctx, dt = _c5_small()
    b = ctx.vec()
    ctx.kernel("init_b", b)
    u = ctx.vec()
    ctx.kernel("init_u", u)
    rho = ctx.scalar(np.ones(ctx.n_pad))
    seed = np.random.default_rng(7).standard_normal((ctx.n_pad, 4))
    seed[:, 3] = 0
    seed[ctx.n:] = 0

    def grad(c, nsteps, every):
        lam = c.vec(seed)
        c.adjoint_steps(b if c is ctx else c.vec(ctx.get_vec(b)), lam, u if c is ctx else c.vec(ctx.get_vec(u)),
                        rho if c is ctx else c.scalar(np.ones(c.n_pad)), nsteps, every)
        return c.get_vec(lam)

    plans = [(6, 3), (12, 5), (4, 4), (6, 3)]
    got = [grad(ctx, *p) for p in plans]
    for p, g in zip(plans, got):
        fresh, _ = _c5_small()
        ref = grad(fresh, *p)
        fresh.close()
        assert np.array_equal(g, ref), p
    assert np.array_equal(got[0], got[3])
    ctx.close()


@pytest.mark.parametrize("integrator", ["CarpenterKennedy2N54", "ToulorgeDesmet2N84F"])
def test_low_storage_step_adjoint_matches_central_differences(integrator):
    # the checkpointed adjoint through the 2N low-storage schemes (stage by stage:
    # mu2 += B_s mu1, mu1 += h F'^T mu2, mu2 = A_s mu2) against Richardson-extrapolated central
    # differences of the forward time stepping, Hall periodic 16^3 with variable velocity
    c = dict(CASES["hallper_4c"], nodes=(16, 16, 16), integrator=integrator)
    probe = maps_for(dict(c, dt=1.0)).context()
    u = probe.vec()
    probe.kernel("init_u", u)
    umax = float(np.sqrt((probe.get_vec(u)[:, :3] ** 2).sum(1)).max())
    probe.close()
    dt = (2.0 / 16) * (HP / 16) / umax        # CFL 2/N (compute_error_hall_periodic.m:51)
    ctx = maps_for(dict(c, dt=dt)).context()
    nsteps, every = 9, 4
    b = ctx.vec()
    ctx.kernel("init_b", b)
    rho = ctx.scalar(np.ones(ctx.n_pad))
    b0 = ctx.get_vec(b)
    n = ctx.n
    wmass = (HP / 16) ** 3

    def forward(x):
        bb, b2, cb, uu = ctx.vec(x), ctx.vec(), ctx.vec(), ctx.vec()
        ctx.kernel("init_u", uu)
        t = ctx.scalar(np.zeros(2), n=2)
        ctx.time_steps(bb, b2, None, cb, uu, rho, t, nsteps)
        return ctx.get_vec(bb)

    rng = np.random.default_rng(11)
    target = forward(b0) + 1e-3 * rng.standard_normal((ctx.n_pad, 4))
    target[:, 3] = 0
    target[n:] = 0

    def loss(x):
        d = forward(x)[:n, :3] - target[:n, :3]
        return 0.5 * wmass * float(np.sum(d * d))

    g0 = np.zeros_like(b0)
    g0[:n, :3] = wmass * (forward(b0)[:n, :3] - target[:n, :3])
    lam = ctx.vec(g0)
    uu = ctx.vec()
    ctx.kernel("init_u", uu)
    ctx.adjoint_steps(ctx.vec(b0), lam, uu, rho, nsteps, every)
    grad = ctx.get_vec(lam)
    for k in range(4):
        d = rng.standard_normal((ctx.n_pad, 4))
        d[:, 3] = 0
        d[n:] = 0
        d /= np.sqrt(np.sum(d[:, :3] ** 2))
        ad = float(np.sum(grad[:, :3] * d[:, :3]))

        def cd(e):
            return (loss(b0 + e * d) - loss(b0 - e * d)) / (2 * e)
        rich = (4.0 * cd(5e-4) - cd(1e-3)) / 3.0
        assert abs(rich - ad) <= 1e-6 * abs(ad), (k, rich, ad)
    ctx.close()


@pytest.mark.parametrize("name", ["travel_6c_hall_box", "confined_4c_hall_fo", "rot_2c_ad", "confined_4c_hall_ad"])
def test_sweep_through_hall_boxes_matches_central_differences(name):
    # the checkpointed SSPRK33 adjoint through steps with the Hall outflow SAT (and first-order
    # or adaptive dissipation) against Richardson-extrapolated central differences of the time
    # stepping
    c = CASES[name]
    ctx = maps_for(dict(c, dt=c.get("sweep_dt", 1e-3))).context()
    nsteps, every = 6, 4
    b, u = ctx.vec(), ctx.vec()
    ctx.kernel("init_b", b)
    _noisy(ctx, b, c)
    ctx.kernel("init_u", u)
    rho = ctx.scalar(np.ones(ctx.n_pad))
    b0, u0 = ctx.get_vec(b), ctx.get_vec(u)
    n = ctx.n
    rng = np.random.default_rng(17)

    def forward(x):
        bb, b2, b3, cb, uu = ctx.vec(x), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(u0)
        ctx.time_steps(bb, b2, b3, cb, uu, rho, ctx.scalar(np.zeros(2), n=2), nsteps)
        return ctx.get_vec(bb)

    target = forward(b0) + 1e-3 * rng.standard_normal((ctx.n_pad, 4))
    target[:, 3] = 0
    target[n:] = 0

    def loss(x):
        d = forward(x)[:n, :3] - target[:n, :3]
        return 0.5 * float(np.sum(d * d))

    g0 = np.zeros_like(b0)
    g0[:n, :3] = forward(b0)[:n, :3] - target[:n, :3]
    lam = ctx.vec(g0)
    ctx.adjoint_steps(ctx.vec(b0), lam, ctx.vec(u0), rho, nsteps, every)
    grad = ctx.get_vec(lam)
    for k in range(3):
        d = rng.standard_normal((ctx.n_pad, 4))
        d[:, 3] = 0
        d[n:] = 0
        d /= np.sqrt(np.sum(d[:, :3] ** 2))
        ad = float(np.sum(grad[:, :3] * d[:, :3]))

        def cd(e):
            return (loss(b0 + e * d) - loss(b0 - e * d)) / (2 * e)
        # small steps: a larger one can carry a boundary node's tv_a across the outflow switch
        # somewhere along the trajectory, where the loss has a kink
        rich = (4.0 * cd(5e-7) - cd(1e-6)) / 3.0
        assert abs(rich - ad) <= 1e-6 * abs(ad), (k, rich, ad)
    ctx.close()


def test_program_adjoint_of_a_list_run_is_refused():
    # the register-program adjoint (2R schemes, SSPRK104) recomputes the forward with the
    # fused kernels: IEQ_STAGE_KERNEL=LIST is refused
    c = dict(CASES["hallper_4c"], nodes=(16, 16, 16), integrator="KennedyCarpenterLewis2R54C", stage_kernel="LIST")
    ctx = maps_for(dict(c, dt=1e-3)).context()
    b, u = ctx.vec(), ctx.vec()
    lam = ctx.vec()
    from inductioneq_b200.lib import IeqError
    with pytest.raises(IeqError) as e:
        ctx.adjoint_steps(b, lam, u, ctx.scalar(np.ones(ctx.n_pad)), 2, 1)
    assert e.value.name == "IEQ_ERR_SETTINGS"
    ctx.close()


def _hallper16(integrator, **kw):
    c = dict(CASES["hallper_4c"], nodes=(16, 16, 16), integrator=integrator, **kw)
    probe = maps_for(dict(c, dt=1.0)).context()
    u = probe.vec()
    probe.kernel("init_u", u)
    umax = float(np.sqrt((probe.get_vec(u)[:, :3] ** 2).sum(1)).max())
    probe.close()
    return c, (2.0 / 16) * (HP / 16) / umax        # CFL 2/N (compute_error_hall_periodic.m:51)


@pytest.mark.parametrize("integrator", ["SSPRK33", "CarpenterKennedy2N54", "ToulorgeDesmet2N84F"])
def test_register_program_adjoint_equals_the_dedicated_step_adjoints(integrator):
    # IEQ_ADJOINT_PROGRAM=1 reverses SSPRK33 and the 2N schemes through the generic register
    # program as well: the same gradient as their dedicated step adjoints (the pointwise
    # combinations in another order: 1e-13 of its scale)
    c, dt = _hallper16(integrator)
    out = []
    for prog in (0, 1):
        ctx = maps_for(dict(c, dt=dt, adjoint_program=prog)).context()
        b, u = ctx.vec(), ctx.vec()
        ctx.kernel("init_b", b)
        ctx.kernel("init_u", u)
        lam = ctx.vec(_rand(ctx, 9))
        ctx.adjoint_steps(b, lam, u, ctx.scalar(np.ones(ctx.n_pad)), 7, 3)
        out.append(ctx.get_vec(lam)[:, :3])
        ctx.close()
    assert np.abs(out[0] - out[1]).max() <= 1e-13 * np.abs(out[0]).max()


@pytest.mark.parametrize("integrator", ["KennedyCarpenterLewis2R54C", "CalvoFrancoRandez2R64", "SSPRK104"])
def test_register_program_adjoint_matches_central_differences(integrator):
    # the 2R schemes and SSPRK104 through the register-program adjoint: the checkpointed
    # gradient against Richardson-extrapolated central differences of the time stepping
    c, dt = _hallper16(integrator)
    ctx = maps_for(dict(c, dt=dt)).context()
    nsteps, every = 7, 3
    b = ctx.vec()
    ctx.kernel("init_b", b)
    rho = ctx.scalar(np.ones(ctx.n_pad))
    b0 = ctx.get_vec(b)
    n = ctx.n

    def forward(x):
        bb, b2, b3, cb, uu = ctx.vec(x), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec()
        ctx.kernel("init_u", uu)
        ctx.time_steps(bb, b2, b3, cb, uu, rho, ctx.scalar(np.zeros(2), n=2), nsteps)
        return ctx.get_vec(bb)

    rng = np.random.default_rng(29)
    target = forward(b0) + 1e-3 * rng.standard_normal((ctx.n_pad, 4))
    target[:, 3] = 0
    target[n:] = 0

    def loss(x):
        d = forward(x)[:n, :3] - target[:n, :3]
        return 0.5 * float(np.sum(d * d))

    g0 = np.zeros_like(b0)
    g0[:n, :3] = forward(b0)[:n, :3] - target[:n, :3]
    lam = ctx.vec(g0)
    uu = ctx.vec()
    ctx.kernel("init_u", uu)
    ctx.adjoint_steps(ctx.vec(b0), lam, uu, rho, nsteps, every)
    grad = ctx.get_vec(lam)
    for k in range(3):
        d = rng.standard_normal((ctx.n_pad, 4))
        d[:, 3] = 0
        d[n:] = 0
        d /= np.sqrt(np.sum(d[:, :3] ** 2))
        ad = float(np.sum(grad[:, :3] * d[:, :3]))

        def cd(e):
            return (loss(b0 + e * d) - loss(b0 - e * d)) / (2 * e)
        rich = (4.0 * cd(5e-4) - cd(1e-3)) / 3.0
        assert abs(rich - ad) <= 1e-6 * abs(ad), (k, rich, ad)
    ctx.close()


@pytest.mark.parametrize("name, integrator", [("hallper_4c", "SSPRK33"), ("rot_6c_sat", "SSPRK33"),
                                              ("rot3d_4e_split_hod", "CarpenterKennedy2N54"),
                                              ("hallper_6c_hod", "ToulorgeDesmet2N84F")])
def test_sweep_on_fused_forward_equals_sweep_on_reference_kernel_lists(name, integrator):
    # the sweep's forward passes run the fused stage kernels (their stage states written out
    # per stage); with IEQ_STAGE_KERNEL=LIST they run the reference kernel lists.  Both
    # linearise about the same trajectory up to rounding: the gradients agree to 1e-11 of
    # their scale.  10 steps with checkpoints every 4: a short last segment.
    c = dict(CASES[name], integrator=integrator)
    probe = maps_for(dict(c, dt=1.0)).context()
    u = probe.vec()
    probe.kernel("init_u", u)
    umax = max(float(np.sqrt((probe.get_vec(u)[:, :3] ** 2).sum(1)).max()), 1.0)
    probe.close()
    lo, hi = c["lo"], c["hi"]
    dt = 0.2 * (hi - lo) / max(c["nodes"]) / umax
    out = []
    for kernel in ("AUTO", "LIST"):
        ctx = maps_for(dict(c, dt=dt, stage_kernel=kernel)).context()
        b, u = ctx.vec(), ctx.vec()
        ctx.kernel("init_b", b)
        ctx.kernel("init_u", u)
        lam = ctx.vec(_rand(ctx, 5))
        ctx.adjoint_steps(b, lam, u, ctx.scalar(np.ones(ctx.n_pad)), 10, 4)
        out.append(ctx.get_vec(lam)[:, :3])
        ctx.close()
    scale = np.abs(out[1]).max()
    assert np.abs(out[0] - out[1]).max() <= 1e-11 * scale
