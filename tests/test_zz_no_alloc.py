"""The allocation-free dot product (ieq_dot_product_noalloc) against the context-based one.

ieq_dot_product_noalloc serves callers that cannot let the library allocate device memory
(hosts that own all device memory through their own pool, time loops that must not
allocate): its scratch is a fixed array in the library's device image.  Two calls in a row
must agree with ieq_dot_value (which uses the context's allocated scratch) within the FP64
tolerance of the other parity tests, and sizes above the stated maximum must be refused.
This file is collected last so that a failing run has already run every other test.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from inductioneq_b200 import lib as L
from inductioneq_b200.induction_eq import Maps

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _context(n_side: int):
    m = Maps()
    m.I_Mesh.update({"NODES_X": n_side, "NODES_Y": n_side + 1, "NODES_Z": n_side + 2, "XMIN": 0.0, "XMAX": 1.0,
                     "YMIN": 0.0, "YMAX": 1.0, "ZMIN": 0.0, "ZMAX": 1.0})
    m.I_RunOps.update({"order": 2, "testcase": "confined_domain"})
    return m.context()


def _noalloc(lib, a, b, n, out, stream):
    f = lib.ieq_dot_product_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f(a, b, n, out, stream)


def test_noalloc_dot_matches_context_dot_on_two_calls():
    ctx = _context(40)
    n = ctx.n
    rng = np.random.default_rng(7)
    out = ctx.scalar(n=1)
    for call in range(2):
        ah = rng.standard_normal(ctx.n_pad)
        bh = rng.standard_normal(ctx.n_pad) * (1.0 + call)
        a, b = ctx.scalar(ah), ctx.scalar(bh)
        expected = ctx.dot(a, b)
        st = _noalloc(ctx.lib, a.ptr, b.ptr, n, out.ptr, ctx.stream)
        assert st == 0, L.STATUS.get(st, st)
        ctx.synchronize()
        got = float(ctx.get_scalar(out, n=1)[0])
        exact = float(np.dot(ah[:n], bh[:n]))
        assert abs(got - expected) <= TOL * np.sum(np.abs(ah[:n] * bh[:n])), (call, got, expected)
        assert abs(got - exact) <= TOL * np.sum(np.abs(ah[:n] * bh[:n])), (call, got, exact)


@pytest.mark.parametrize("grid, trim", [((100, 101, 102), 0), ((128, 256, 256), 0), ((128, 256, 256), 1)])
def test_noalloc_dot_at_large_sizes_matches_context_dot(grid, trim):
    # n above 256 partial blocks (the final kernel's strided loop over the partials) up to the
    # stated maximum, and one element below it; the context's dot runs over all its nodes, so
    # with trim = 1 the last element of b is zero there and absent from the no-alloc call
    m = Maps()
    m.I_Mesh.update({"NODES_X": grid[0], "NODES_Y": grid[1], "NODES_Z": grid[2], "XMIN": 0.0, "XMAX": 1.0,
                     "YMIN": 0.0, "YMAX": 1.0, "ZMIN": 0.0, "ZMAX": 1.0})
    m.I_RunOps.update({"order": 2, "testcase": "confined_domain"})
    ctx = m.context()
    n = ctx.n - trim
    assert n <= 8388608 and (n > 524288)
    rng = np.random.default_rng(11)
    out = ctx.scalar(n=1)
    for call in range(2):
        ah = rng.standard_normal(ctx.n_pad)
        bh = rng.standard_normal(ctx.n_pad) * (1.0 + call)
        bh[n:] = 0.0
        a, b = ctx.scalar(ah), ctx.scalar(bh)
        expected = ctx.dot(a, b)
        st = _noalloc(ctx.lib, a.ptr, b.ptr, n, out.ptr, ctx.stream)
        assert st == 0, L.STATUS.get(st, st)
        ctx.synchronize()
        got = float(ctx.get_scalar(out, n=1)[0])
        scale = float(np.sum(np.abs(ah[:n] * bh[:n])))
        assert abs(got - expected) <= TOL * scale, (call, got, expected)
    ctx.close()


def test_noalloc_dot_refuses_sizes_above_the_maximum():
    ctx = _context(12)
    out = ctx.scalar(n=1)
    a = ctx.scalar()
    st = _noalloc(ctx.lib, a.ptr, a.ptr, 8388608 + 1, out.ptr, ctx.stream)
    assert L.STATUS[st] == "IEQ_ERR_SHAPE"
