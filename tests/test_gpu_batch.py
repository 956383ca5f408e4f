"""Batched form on the GPU: every solve of the persistent batched launch equals the same
solve run alone (ieq_time_steps on its own context) and the oracle."""
from __future__ import annotations

import math

import numpy as np
import pytest

from inductioneq_b200.batch import Batch, autotune, rotation_batch
from oracle.hostloops import time_loop
from oracle.numpy_oracle import NumpyOracle, OracleConfig
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu

SPECS = [(16, 2, 0.7, 0.5 * (2 / 15) / (0.7 * math.sqrt(2))),
         (13, 6, 1.9, 0.5 * (2 / 12) / (1.9 * math.sqrt(2))),
         (20, 4, 1.2, 0.5 * (2 / 19) / (1.2 * math.sqrt(2))),
         (17, 4, 0.55, 0.5 * (2 / 16) / (0.55 * math.sqrt(2)))]


@pytest.mark.parametrize("mode", ["persistent", "stages", "branches"])
def test_batched_solves_equal_single_solves(mode):
    bt = Batch(SPECS)
    shapes = [(32, 4, 2), (16, 4, 4), (8, 8, 4), (64, 2, 2)]
    for i, s in enumerate(shapes):
        bt.set_tile(i, s)
    bt.init()
    b0 = [c.get_vec(f["b"]) for c, f in zip(bt.ctxs, bt.fields)]
    bt.bind()
    steps = 7
    bt.run(steps, mode=mode)
    bt.unbind()
    for i, (c, f) in enumerate(zip(bt.ctxs, bt.fields)):
        got = c.get_vec(f["b"])
        # the same solve alone through the fused single-grid path
        b, b2, b3, cb, u = c.vec(b0[i]), c.vec(), c.vec(), c.vec(), c.vec()
        c.kernel("init_u", u)
        rho = c.scalar(np.ones(c.n_pad))
        t = c.scalar(np.zeros(2), n=2)
        c.time_steps(b, b2, b3, cb, u, rho, t, steps)
        alone = c.get_vec(b)
        assert rel_err(got, alone) <= 1e-13, i
        tt = c.get_scalar(f["time"], n=2)
        np.testing.assert_allclose(tt, c.get_scalar(t, n=2), rtol=1e-15)
        assert rel_err(got, b0[i]) > 1e-6
    bt.close()


def test_batched_solve_matches_oracle():
    n, order, omega, dt = SPECS[1]
    bt = Batch([SPECS[1]])
    bt.init()
    c, f = bt.ctxs[0], bt.fields[0]
    b0 = c.get_vec(f["b"])
    bt.bind()
    bt.run(3)
    bt.unbind()
    cfg = OracleConfig(nodes=(n, n, n), xmin=(-1.0,) * 3, xmax=(1.0,) * 3, order=order,
                       testcase="rotation_gaussian", dt=dt, tc_omega=omega)
    o = NumpyOracle(cfg)
    bo, u = b0.copy(), o.vec()
    o.run("init_u", cfg.nodes, u)
    t = np.zeros(2)
    time_loop(o, "SSPRK33", False, False, 3, bo, o.vec(), o.vec(), o.vec(), u, o.scalar(fill=1.0), t)
    assert rel_err(c.get_vec(f["b"]), bo) <= 1e-12
    bt.close()


def test_autotune_picks_a_shape_per_order(tmp_path, monkeypatch):
    import inductioneq_b200.batch as B
    monkeypatch.setattr(B, "TUNE_CACHE", str(tmp_path / "tiles.json"))
    bt = Batch(rotation_batch(4, seed=5, nmin=16, nmax=24))
    chosen = autotune(bt, steps=2, shapes=[(32, 4, 2), (16, 8, 2)], gpu_name="test")
    assert set(chosen) == {f"o{o}_small" for (_, o, _, _) in bt.specs}
    assert (tmp_path / "tiles.json").is_file()
    bt.close()
