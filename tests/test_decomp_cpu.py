"""The z-slab decomposition of one solve (inductioneq_b200.decomp) on CPU ranks.

Every rank (a spawned process, gloo) runs the integrator's kernel list on its slab with the
oracle as the per-rank engine and exchanges the ghost planes of the state fields between
kernels; the owned planes of every rank must equal the single-process run of the whole grid
bit for bit (each owned node performs the same arithmetic).  Two ranks and three ranks
(different neighbours); periodic grids (with two ranks the upper and lower neighbour are the
same rank: Hall + high-order dissipation with CarpenterKennedy2N54, Hall with a constant
velocity with SSPRK33) and boxes (no ghosts at the box's z faces, NUM_BOUNDS + ORDER/2 at
the inner slab ends: rotation with SAT inflow and SSPRK33, confined Hall with high-order
dissipation and CarpenterKennedy2N54, an extended operator).
"""
from __future__ import annotations

import math
import os
import socket

import numpy as np
import pytest

from inductioneq_b200 import decomp as D
from inductioneq_b200 import ranks as R

HP = 4.0 * math.pi / 3.0

CASES = {
    "whistler_4c_hod_ck": dict(order=4, testcase="hall_circular_wave", nodes=(8, 9, 12), lo=0.0, hi=2 * math.pi,
                               hall=True, dissipation="HIGH_ORDER", integrator="CarpenterKennedy2N54", dt=0.01,
                               steps=2),
    "hallper_2c_conv_ssp": dict(order=2, testcase="hall_periodic", nodes=(7, 8, 9), lo=0.0, hi=HP, hall=True,
                                integrator="SSPRK33", dt=0.005, steps=2),
    "rot3d_4c_ssp_box": dict(order=4, testcase="rotation_3D", nodes=(8, 9, 30), lo=-1.0, hi=1.0, periodic=False,
                             integrator="SSPRK33", dt=0.005, steps=2),
    "confined_6c_hall_hod_ck_box": dict(order=6, testcase="confined_domain", nodes=(9, 8, 30), lo=0.0, hi=1.0,
                                        periodic=False, hall=True, dissipation="HIGH_ORDER",
                                        integrator="CarpenterKennedy2N54", dt=1e-5, steps=2),
    "confined_4e_hall_ck_box": dict(order=4, extended=True, testcase="confined_domain", nodes=(8, 7, 25), lo=0.0,
                                    hi=1.0, periodic=False, hall=True, integrator="CarpenterKennedy2N54", dt=1e-5,
                                    steps=2),
}


def _ghosts(c):
    return D.ghost_depth(c["order"], c.get("periodic", True), c.get("extended", False))


def _oracle(c, nodes, zoff=0, nzg=0):
    from oracle.numpy_oracle import NumpyOracle, OracleConfig
    cfg = OracleConfig(nodes=nodes, xmin=(c["lo"],) * 3, xmax=(c["hi"],) * 3, order=c["order"],
                       extended=c.get("extended", False), periodic=c.get("periodic", True),
                       hall=c.get("hall", False), dissipation=c.get("dissipation", "NONE"), testcase=c["testcase"],
                       dt=c["dt"], zoff=zoff, nzg=nzg)
    return NumpyOracle(cfg)


def _initial(c):
    o = _oracle(c, c["nodes"])
    b, u = o.vec(), o.vec()
    o.run("init_b", o.cfg.nodes, b)
    o.run("init_u", o.cfg.nodes, u)
    b[:, :3] += 1e-2 * np.random.default_rng(7).standard_normal((o.N, 3))
    return o, b, u


def _global_run(c):
    from oracle.hostloops import time_loop
    from oracle.sequencing import NUM_FIELDS
    o, b, u = _initial(c)
    nf = NUM_FIELDS[c["integrator"]]
    f = [b, o.vec(), o.vec(), o.vec(), u, o.scalar(fill=1.0), np.zeros(2)]
    time_loop(o, c["integrator"], c.get("hall", False), False, c["steps"], f[0], f[1], f[2] if nf == 3 else None,
              f[3], f[4], f[5], f[6])
    return f


def _rank_run(rk: R.Ranks, c: dict):
    from oracle.sequencing import NUM_FIELDS, rk_step
    R.init(rk, "gloo", timeout_s=60.0)
    try:
        g, b, u = _initial(c)
        nx, ny, nz = c["nodes"]
        slabs = D.ZSlabs(rk, nx, ny, nz, _ghosts(c), c.get("periodic", True))
        o = _oracle(c, slabs.local_nodes, slabs.z_offset, nz)
        o.d = g.d   # the global spacing
        nf = NUM_FIELDS[c["integrator"]]
        lb, lu = slabs.scatter(b), slabs.scatter(u)
        b2, b3, cb = o.vec(), o.vec(), o.vec()
        rho, t = o.scalar(fill=1.0), np.zeros(2)
        args = [lb, b2, b3, cb, lu, rho, t] if nf == 3 else [lb, b2, cb, lu, rho, t]
        state = [lb, b2, b3] if nf == 3 else [lb, b2]
        seq = rk_step(c["integrator"], c.get("hall", False), False)
        D.decomposed_steps(slabs, o, seq, c["steps"], state, args)
        rows = slabs.owned_rows()
        return {"z": (slabs.z0, slabs.z1), "b": lb[rows].copy(), "b2": b2[rows].copy(),
                "b3": b3[rows].copy() if nf == 3 else None, "t": t.copy()}
    finally:
        R.finish(rk)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, case, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    try:
        q.put((rank, _rank_run(R.Ranks.from_env(), CASES[case])))
    except Exception as e:
        q.put((rank, ("error", type(e).__name__, str(e)[:300])))


def _spawn(world, case):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
    return out


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", sorted(CASES))
def test_decomposed_solve_equals_single_process_run(world, case):
    c = CASES[case]
    if world == 3 and c["nodes"][2] < 3 * _ghosts(c):
        pytest.skip("grid too short for three slabs of this ghost depth")
    out = _spawn(world, case)
    for r, v in out.items():
        assert not (isinstance(v, tuple) and v and v[0] == "error"), v
    ref = _global_run(c)
    plane = c["nodes"][0] * c["nodes"][1]
    zs = sorted(v["z"] for v in out.values())
    assert zs[0][0] == 0 and zs[-1][1] == c["nodes"][2]
    for v in out.values():
        rows = slice(v["z"][0] * plane, v["z"][1] * plane)
        np.testing.assert_array_equal(v["b"], ref[0][rows])
        np.testing.assert_array_equal(v["b2"], ref[1][rows])
        if v["b3"] is not None:
            np.testing.assert_array_equal(v["b3"], ref[2][rows])
        np.testing.assert_array_equal(v["t"], ref[6])


def test_slab_bounds_cover_the_grid():
    for nz, w in ((12, 2), (13, 3), (64, 8), (9, 4)):
        b = D.slab_bounds(nz, w)
        assert b[0][0] == 0 and b[-1][1] == nz
        assert all(b[i][1] == b[i + 1][0] for i in range(w - 1))
        assert max(e - s for s, e in b) - min(e - s for s, e in b) <= 1


def test_too_many_ranks_for_the_ghost_depth_is_refused():
    with pytest.raises(ValueError):
        D.ZSlabs(R.Ranks(4, 0, 0), 8, 8, 12, D.ghost_depth(6))


def test_local_maps_keep_the_global_spacing_and_offset():
    from inductioneq_b200.induction_eq import Maps
    m = Maps()
    m.I_Mesh.update({"NODES_X": 16, "NODES_Y": 16, "NODES_Z": 24, "XMIN": 0.0, "XMAX": 1.0, "YMIN": 0.0, "YMAX": 1.0,
                     "ZMIN": 0.0, "ZMAX": 3.0})
    m.I_RunOps.update({"periodic": "USE_PERIODIC", "order": 4})
    sl = D.ZSlabs(R.Ranks(2, 1, 1), 16, 16, 24, D.ghost_depth(4))
    lm = D.local_maps(m, sl)
    s = lm.settings()
    assert f"-DNODES_Z={sl.nloc}" in s and "-DIEQ_Z_OFFSET=8" in s and "-DIEQ_NZ_GLOBAL=24" in s
    assert f"-DDZ={3.0 / 24:.16e}" in s
    m.I_RunOps["periodic"] = "NONE"
    with pytest.raises(ValueError):
        D.local_maps(m, sl)


def test_box_slabs_have_ghosts_only_at_inner_ends():
    G = D.ghost_depth(6, periodic=False)
    assert G == 6 + 3 and D.ghost_depth(4, periodic=False, extended=True) == 6 + 2
    sl = [D.ZSlabs(R.Ranks(3, r, r), 8, 8, 40, G, periodic=False) for r in range(3)]
    assert [(s.g_lo, s.g_hi) for s in sl] == [(0, G), (G, G), (G, 0)]
    assert [s.z_offset for s in sl] == [0, 14 - G, 27 - G]
    assert sl[0].down is None and sl[2].up is None and sl[1].down == 0 and sl[1].up == 2
    assert sl[2].nloc == sl[2].owned + G
    # one rank: the whole box, no ghosts
    one = D.ZSlabs(R.Ranks(1, 0, 0), 8, 8, 40, G, periodic=False)
    assert (one.g_lo, one.g_hi, one.nloc) == (0, 0, 40)
    glob = np.arange(8 * 8 * 40, dtype=np.float64)
    np.testing.assert_array_equal(sl[1].scatter(glob), glob[(14 - G) * 64:(27 + G) * 64])


def test_local_exchange_fills_ghosts_from_neighbours():
    import torch
    G = D.ghost_depth(2, periodic=False)
    for periodic in (False, True):
        g = D.ghost_depth(2) if periodic else G
        sl = [D.ZSlabs(R.Ranks(3, r, r), 2, 2, 12, g, periodic=periodic) for r in range(3)]
        glob = np.arange(2 * 2 * 12, dtype=np.float64)
        loc = [torch.from_numpy(s.scatter(glob)) for s in sl]
        want = [t.clone() for t in loc]
        for s, t in zip(sl, loc):
            lo, _, _, hi = s.parts(t)
            lo.fill_(-1.0)
            hi.fill_(-1.0)
        D.exchange_local(sl, [[t] for t in loc])
        for t, w in zip(loc, want):
            assert torch.equal(t, w)


# ----------------------------------------------------------------- decomposed divergence cleaning
CLEAN_CASES = {
    "confined_4c_ws_d0": dict(order=4, testcase="confined_domain", nodes=(12, 10, 30), lo=0.0, hi=1.0,
                              periodic=False, laplace="WIDE_STENCIL_DIRICHLET", dt=1e-5),
    "confined_6c_ns_d0": dict(order=6, testcase="confined_domain", nodes=(11, 12, 30), lo=0.0, hi=1.0,
                              periodic=False, laplace="NARROW_STENCIL_DIRICHLET", dt=1e-5),
    "confined_2c_ws_d0": dict(order=2, testcase="confined_domain", nodes=(10, 11, 21), lo=0.0, hi=1.0,
                              periodic=False, laplace="WIDE_STENCIL_DIRICHLET", dt=1e-5),
    "confined_2e_ws_ln": dict(order=2, extended=True, testcase="confined_domain", nodes=(10, 9, 24), lo=0.0,
                              hi=1.0, periodic=False, laplace="WIDE_STENCIL_LNS", dt=1e-5),
}
CLEAN_ITERATIONS = 15


def _clean_oracle(c, nodes, zoff=0, nzg=0):
    from oracle.numpy_oracle import NumpyOracle, OracleConfig
    cfg = OracleConfig(nodes=nodes, xmin=(c["lo"],) * 3, xmax=(c["hi"],) * 3, order=c["order"],
                       extended=c.get("extended", False), periodic=False, testcase=c["testcase"], dt=c["dt"],
                       laplace=c["laplace"], bnodes=D.bnodes_of(c["laplace"]), zoff=zoff, nzg=nzg)
    return NumpyOracle(cfg)


def _clean_initial(c):
    o = _clean_oracle(c, c["nodes"])
    b = o.vec()
    o.run("init_b", o.cfg.nodes, b)
    b[:, :3] += 1e-3 * np.random.default_rng(11).standard_normal((o.N, 3))
    return o, b


class _OracleEngine:
    """The oracle as a slab's engine of the decomposed cleaning (the host's sum of the
    per-item products of dot_product over a range)."""

    def __init__(self, o):
        self.o = o

    def run(self, name, grange, *args):
        self.o.run(name, grange, *args)

    def dot_range(self, x, y, first, count):
        return float(np.sum((x[first:first + count] * y[first:first + count]).astype(np.float64)))


def _rank_clean(rk: R.Ranks, c: dict):
    import torch
    import torch.distributed as dist
    R.init(rk, "gloo", timeout_s=60.0)
    try:
        g, b = _clean_initial(c)
        nx, ny, nz = c["nodes"]
        sl = D.ZSlabs(rk, nx, ny, nz, D.ghost_depth(c["order"], False, c.get("extended", False), c["laplace"]),
                      periodic=False)
        o = _clean_oracle(c, sl.local_nodes, sl.z_offset, nz)
        o.d = g.d
        lb = sl.scatter(b)
        cg = {k: o.scalar() for k in ("div", "phi", "lap", "r", "u")}

        def total(vals):
            t = torch.tensor([float(sum(vals))], dtype=torch.float64)
            dist.all_reduce(t)
            return float(t.item())

        res = D.clean_div_decomposed([(sl, _OracleEngine(o), lb, cg)], CLEAN_ITERATIONS, 1e-14,
                                     D.bnodes_of(c["laplace"]), total=total,
                                     exchange=lambda f: sl.exchange(*f[0]),
                                     scalar=lambda _e, v: np.array([v], dtype=o.T))
        rows = sl.owned_rows()
        return {"z": (sl.z0, sl.z1), "b": lb[rows].copy(), "phi": cg["phi"][rows].copy(), "res": res}
    finally:
        R.finish(rk)


def _clean_worker(rank, world, port, case, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    try:
        q.put((rank, _rank_clean(R.Ranks.from_env(), CLEAN_CASES[case])))
    except Exception as e:
        q.put((rank, ("error", type(e).__name__, str(e)[:300])))


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", sorted(CLEAN_CASES))
def test_decomposed_cleaning_equals_single_process_cleaning(world, case):
    # the same CG iterations and residual history, B and phi on the owned planes equal up to
    # the order of the dot products' sums (the slabs' sums added across the ranks)
    import torch.multiprocessing as mp
    from oracle.hostloops import clean_div
    c = CLEAN_CASES[case]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_clean_worker, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
    for v in out.values():
        assert not (isinstance(v, tuple) and v and v[0] == "error"), v
    o, b = _clean_initial(c)
    ref = clean_div(o, b, CLEAN_ITERATIONS, 1e-14, D.bnodes_of(c["laplace"]))
    plane = c["nodes"][0] * c["nodes"][1]
    scale = np.abs(b[: o.N, :3]).max()
    pscale = np.abs(ref["phi"][: o.N]).max()
    for v in out.values():
        assert v["res"]["iterations"] == ref["iterations"] == CLEAN_ITERATIONS
        np.testing.assert_allclose(v["res"]["history"], ref["history"], rtol=1e-10)
        rows = slice(v["z"][0] * plane, v["z"][1] * plane)
        assert np.abs(v["b"][:, :3] - b[rows, :3]).max() <= 1e-12 * scale
        assert np.abs(v["phi"] - ref["phi"][rows]).max() <= 1e-10 * pscale
    assert ref["history"][-1] < 1e-2 * ref["history"][0]
