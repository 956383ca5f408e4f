"""Batched form: many independent rotation solves in one persistent launch.

``rotation_batch(n_solves, seed)`` draws the workload (grid N ~ U{16..96}, rotation rate
omega ~ U(0.5, 2), SBP order uniform in {2, 4, 6}; dt = 0.5 dx / (omega sqrt 2) as
initialize.m:93-96 with CFL 0.5), ``Batch`` binds the solves' contexts to the C ABI's
ieq_batch_*, and ``autotune`` chooses the tile (brick) shape per (order, grid-size class)
by timing the persistent launch, caching the choice in a JSON file.
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import time

import numpy as np

from .induction_eq import Maps
from .lib import Context, IeqError, _ptr, load

TILE_SHAPES = [(32, 8, 1), (32, 4, 2), (16, 8, 2), (16, 4, 4), (8, 8, 4), (64, 4, 1), (64, 2, 2), (8, 4, 8)]
TUNE_CACHE = os.environ.get("IEQ_TUNE_CACHE",
                            os.path.join(os.path.dirname(os.path.abspath(__file__)), "_tune", "batch_tiles.json"))


def size_class(n: int) -> str:
    return "small" if n < 48 else "large"


def rotation_maps(n: int, order: int, omega: float, dt: float) -> Maps:
    m = Maps()
    m.I_Mesh.update({"NODES_X": n, "NODES_Y": n, "NODES_Z": n, "XMIN": -1.0, "XMAX": 1.0, "YMIN": -1.0,
                     "YMAX": 1.0, "ZMIN": -1.0, "ZMAX": 1.0})
    m.I_TI.update({"DT": dt, "time_integrator": "SSPRK33"})
    m.I_RunOps.update({"order": order, "testcase": "rotation_gaussian"})
    m.tc_omega = omega
    return m


def rotation_batch(n_solves: int = 32, seed: int = 2026, nmin: int = 16, nmax: int = 96):
    """[(N, order, omega, dt)] of the batched rotation workload."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_solves):
        n = int(rng.integers(nmin, nmax + 1))
        omega = float(rng.uniform(0.5, 2.0))
        order = int(rng.choice([2, 4, 6]))
        dx = 2.0 / (n - 1)
        dt = 0.5 * dx / (omega * math.sqrt(2.0))
        out.append((n, order, omega, dt))
    return out


class Batch:
    def __init__(self, specs, device: int = 0):
        self.lib = load()
        lib = self.lib
        vp = ctypes.c_void_p
        lib.ieq_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.c_int]
        lib.ieq_batch_destroy.argtypes = [vp]
        lib.ieq_batch_last_error.argtypes = [vp]
        lib.ieq_batch_last_error.restype = ctypes.c_char_p
        lib.ieq_batch_stream.argtypes = [vp]
        lib.ieq_batch_stream.restype = vp
        lib.ieq_batch_set_tile.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.ieq_batch_bind.argtypes = [vp, ctypes.POINTER(vp)]
        lib.ieq_batch_run.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        lib.ieq_batch_unbind.argtypes = [vp]
        lib.ieq_batch_total_tiles.argtypes = [vp]
        lib.ieq_batch_total_tiles.restype = ctypes.c_longlong
        lib.ieq_batch_grid.argtypes = [vp]
        lib.ieq_batch_test_barrier.argtypes = [vp, ctypes.c_int, ctypes.c_longlong]
        self.specs = list(specs)
        self.ctxs = [rotation_maps(*s).context(device) for s in self.specs]
        arr = (vp * len(self.ctxs))(*[c.h for c in self.ctxs])
        h = vp()
        st = lib.ieq_batch_create(ctypes.byref(h), arr, len(self.ctxs))
        self.h = h.value
        if st != 0:
            raise IeqError(st, lib.ieq_batch_last_error(self.h).decode())
        self.fields = []
        for c in self.ctxs:
            f = {"b": c.vec(), "b2": c.vec(), "b3": c.vec(), "u": c.vec(), "time": c.scalar(np.zeros(2), n=2)}
            self.fields.append(f)
        self.total_nodes = sum(c.n for c in self.ctxs)

    def _check(self, st):
        if st != 0:
            raise IeqError(st, self.lib.ieq_batch_last_error(self.h).decode())

    @property
    def stream(self) -> int:
        return self.lib.ieq_batch_stream(self.h)

    def init(self):
        for c, f in zip(self.ctxs, self.fields):
            c.kernel("init_b", f["b"])
            c.kernel("init_u", f["u"])
            f["time"].upload(np.zeros(2))
            c.synchronize()

    def set_tile(self, solve: int, shape):
        self._check(self.lib.ieq_batch_set_tile(self.h, solve, *shape))

    def bind(self):
        ptrs = []
        for f in self.fields:
            ptrs += [_ptr(f["b"]), _ptr(f["b2"]), _ptr(f["b3"]), _ptr(f["u"]), _ptr(f["time"])]
        arr = (ctypes.c_void_p * len(ptrs))(*ptrs)
        self._check(self.lib.ieq_batch_bind(self.h, arr))

    MODES = {"stages": 0, "persistent": 1, "branches": 2}

    def run(self, steps: int, persistent: bool = True, mode: str | None = None):
        """Advance every bound solve `steps` SSPRK33 steps: mode "persistent" (one persistent
        kernel over the tile queue), "stages" (one tile-queue kernel per stage) or "branches"
        (one graph branch per solve); `persistent` picks between the first two."""
        m = self.MODES[mode] if mode is not None else (1 if persistent else 0)
        self._check(self.lib.ieq_batch_run(self.h, int(steps), m))

    def test_barrier(self, extra_arrivals: int, spin_limit: int = 0):
        """Failure-path test hook of the persistent mode's grid barrier (ieq_batch_test_barrier)."""
        self._check(self.lib.ieq_batch_test_barrier(self.h, int(extra_arrivals), int(spin_limit)))

    def unbind(self):
        self._check(self.lib.ieq_batch_unbind(self.h))

    def grid(self) -> int:
        return self.lib.ieq_batch_grid(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.lib.ieq_batch_destroy(self.h)
            self.h = None
        for c in self.ctxs:
            c.close()


def autotune(batch: Batch, steps: int = 4, shapes=TILE_SHAPES, use_cache: bool = True, gpu_name: str = "") -> dict:
    """Choose the tile shape per (order, size class) by timing the persistent launch; the
    choice is cached in TUNE_CACHE under the GPU name.  Returns {key: shape}."""
    keys = sorted({f"o{o}_{size_class(n)}" for (n, o, _, _) in batch.specs})
    cache = {}
    if use_cache and os.path.isfile(TUNE_CACHE):
        with open(TUNE_CACHE) as f:
            cache = json.load(f)
    chosen = dict(cache.get(gpu_name, {}))
    todo = [k for k in keys if k not in chosen]
    default = (32, 4, 2)
    for k in keys:
        for i, (n, o, _, _) in enumerate(batch.specs):
            if f"o{o}_{size_class(n)}" == k:
                batch.set_tile(i, tuple(chosen.get(k, default)))
    batch.init()
    batch.bind()
    for k in todo:
        best = None
        for shape in shapes:
            for i, (n, o, _, _) in enumerate(batch.specs):
                if f"o{o}_{size_class(n)}" == k:
                    batch.set_tile(i, shape)
            batch.bind()
            batch.run(steps)   # capture + warm
            t0 = time.perf_counter()
            batch.run(steps)
            el = time.perf_counter() - t0
            if best is None or el < best[0]:
                best = (el, shape)
        chosen[k] = list(best[1])
        for i, (n, o, _, _) in enumerate(batch.specs):
            if f"o{o}_{size_class(n)}" == k:
                batch.set_tile(i, best[1])
    if todo:
        cache[gpu_name] = chosen
        os.makedirs(os.path.dirname(TUNE_CACHE), exist_ok=True)
        with open(TUNE_CACHE, "w") as f:
            json.dump(cache, f, indent=1)
    batch.init()
    return {k: tuple(v) for k, v in chosen.items()}
