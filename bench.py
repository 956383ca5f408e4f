#!/usr/bin/env python
"""Benchmark: DOF-updates/s per RK stage of the nonlinear Hall workload on B200.

Workload (one "step" = one full solve: 260 CarpenterKennedy2N54 time steps of 5 RK stages
each, from the initial state to t = 0.5): circularly polarised whistler wave B = (0.1 sin(z - t), 0.1 cos(z - t), 1) of the Hall induction
equation, zero ion velocity, rho = 1, periodic [0, 2 pi]^3 on 64^3 nodes, FP64, 6th-order
classical SBP operator plus high-order artificial dissipation (factor 1), dt = 0.5/260
(260 steps to t = 0.5).  Inputs are synthetic (the analytic wave); the reference publishes
no benchmark dataset.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank runs an independent replica (weak scaling; a single 64^3 solve
does not shard without a halo exchange).  value = all ranks' DOF-updates / max-over-ranks
device time.  `--impl reference` times the reference's own kernels compiled for the host
cores (oracle/_ref; the numpy port if that build is absent) on rank 0.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_GRID = 64
T_FINAL = 0.5
NUM_STEPS_FULL = 260            # ceil(T / (0.2 dx^2)) with dx = 2 pi / 64
DT = T_FINAL / NUM_STEPS_FULL
STAGES = 5
WORKLOAD = ("hall_circular_wave 64^3 periodic [0,2pi]^3, FP64, 6th-order classical SBP + high-order "
            "dissipation (factor 1), Hall term, u=0, rho=1, CarpenterKennedy2N54, dt=0.5/260")
METRIC = "DOF-updates/s per RK stage"
L2_NOTE = ("L2 flushed between timed solves (256 MiB memset on the solver stream, outside the events); "
           "within a solve the 64^3 fields stay L2 resident, as in production")
# algorithmic bytes per node of one CK2N54 Hall stage, the compulsory traffic of the
# stage with curl(B)/rho not materialised: read b1, b2, u (3 x 24 B) and rho (8 B), write
# b1, b2 (2 x 24 B).  The stage kernel is charged with all of it (the curl kernel, whose
# own traffic -- read b, rho; write E, H: 80 B -- is extra, is reported beside it)
STAGE_BYTES_PER_NODE = 3 * 24 + 8 + 2 * 24
CURL_BYTES_PER_NODE = 24 + 8 + 2 * 24
FP32_STAGE_BYTES_PER_NODE = 3 * 12 + 4 + 2 * 12


def maps(n=N_GRID):
    from inductioneq_b200.induction_eq import Maps
    m = Maps()
    m.I_Mesh.update({"NODES_X": n, "NODES_Y": n, "NODES_Z": n, "XMIN": 0.0, "XMAX": 2 * math.pi,
                     "YMIN": 0.0, "YMAX": 2 * math.pi, "ZMIN": 0.0, "ZMAX": 2 * math.pi})
    m.I_TI.update({"DT": DT, "time_integrator": "CarpenterKennedy2N54", "final_time": T_FINAL})
    m.I_IEq.update({"hall_term": "USE_HALL", "dissipation": "USE_ARTIFICIAL_DISSIPATION",
                    "dissipation_form": "USE_HIGH_ORDER_DISSIPATION", "HO_DISSIPATION_FACTOR": 1.0})
    m.I_RunOps.update({"order": 6, "testcase": "hall_circular_wave", "periodic": "USE_PERIODIC"})
    return m


# ------------------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples (200 ms) of the GPU with the given UUID while the timed region runs."""
    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9 or (self.uuid and self.uuid not in p[0]):
                continue
            rows.append(p)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, nm in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ------------------------------------------------------------------------------ CPU arms
# RK steps of the bench solve in one timed step of the reference arm (a bounded sample of the
# 260-step solve, so that --steps 20 --warmup 5 ends within seconds on the host cores)
REF_RK_PER_STEP = 10


def cpu_reference_run(steps: int, warmup: int, rk_per_step: int = 1, budget_s: float | None = None,
                      threads: int | None = None):
    """The reference's own kernels (oracle/_ref, the -O3 -ffp-contract=fast timing build, OpenMP
    over the host cores) on the same workload.  One timed step = `rk_per_step` CarpenterKennedy2N54
    RK steps, timed whole (no extrapolation); with `budget_s` the loop stops after the first step
    that ends past the budget.  Returns a dict: value (DOF-updates/s per stage), steps run,
    ms_per_step, cores, kind, build, cpu, sample."""
    import numpy as np

    from oracle import refimpl
    from oracle.sequencing import rk_step
    cores = threads or os.cpu_count() or 1
    v = refimpl.Variant(order=6, testcase="hall_circular_wave", periodic=True, hall=True, dissipation="HIGH_ORDER")
    n = N_GRID
    nodes = (n, n, n)
    build = None
    try:
        mesh = refimpl.Mesh(nodes, (0.0,) * 3, (2 * math.pi,) * 3, periodic=True)
        mesh.dt = DT
        r = refimpl.RefRunner(v, mesh, nthreads=cores, fast=True)
        kind = "reference"
        build = f"g++ -O3 -march={refimpl.host_level()} -ffp-contract=fast -fopenmp"
    except Exception:
        r = None
        kind = "port"
    seq = rk_step("CarpenterKennedy2N54", True, False)
    if r is None:
        from oracle.numpy_oracle import NumpyOracle, OracleConfig
        cfg = OracleConfig(nodes=nodes, xmin=(0.0,) * 3, xmax=(2 * math.pi,) * 3, order=6, periodic=True, hall=True,
                           dissipation="HIGH_ORDER", testcase="hall_circular_wave", dt=DT)
        r = NumpyOracle(cfg)
        cores = 1
        build = "numpy restatement"
    b, b2, cb, u = r.vec(), r.vec(), r.vec(), r.vec()
    rho = r.scalar(fill=1.0)
    t = np.zeros(2)
    r.run("init_b", nodes, b)
    for _ in range(warmup * rk_per_step):
        r.run_list(seq, nodes, b, b2, cb, u, rho, t)
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        for _ in range(rk_per_step):
            r.run_list(seq, nodes, b, b2, cb, u, rho, t)
        done += 1
        if budget_s is not None and time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    rk = done * rk_per_step
    return {"value": 3 * n ** 3 * STAGES * rk / el, "steps": done, "ms_per_step": el / done * 1e3, "cores": cores,
            "kind": kind, "build": build, "cpu": refimpl.cpu_model(), "nproc": os.cpu_count(),
            "sample": f"{rk} CK2N54 RK steps ({rk * STAGES} stages) of the 64^3 workload, "
                      f"{rk_per_step} RK step(s) per timed step"}


# ------------------------------------------------------------------------------ other forms
def events_time(stream, fn, reps=1):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) * 1e-3 / reps


def form_fp32(dev, b_ref64):
    """The same workload with REAL=float: DOF-updates/s and L2 error vs exact and vs FP64."""
    import numpy as np
    import torch
    m = maps()
    m.I_Tech["REAL"] = "float"
    ctx = m.context(device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    b, b2, cb, u = ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec()
    rho, t = ctx.scalar(), ctx.scalar(np.zeros(2), n=2)
    ctx.kernel("init_b", b)
    ctx.kernel("init_u", u)
    ctx.kernel("init_rho", rho)
    b0 = ctx.get_vec(b)
    flush = ctx.alloc(256 << 20)

    def solve():
        ctx.time_steps(b, b2, None, cb, u, rho, t, NUM_STEPS_FULL)

    def reset():
        b.upload(b0)
        t.upload(np.zeros(2, dtype=np.float32))

    reset()
    solve()
    reps, tt = 5, 0.0
    for k in range(reps):
        reset()
        ctx.memset(flush, k)
        tt += events_time(stream, solve)
    res = ctx.results(b, T_FINAL, ctx.vec(), ctx.scalar())
    b32 = ctx.get_vec(b).astype(np.float64)
    vs64 = float(np.abs(b32 - b_ref64).max() / np.abs(b_ref64).max())
    prof = ctx.profile_step(b, b2, None, cb, u, rho, t, repeats=20)
    stage = statistics.mean([ms for nm, ms in prof if nm.startswith("stage")])
    ctx.close()
    value = 3 * N_GRID ** 3 * STAGES * NUM_STEPS_FULL * reps / tt
    return {"value": value, "unit": "DOF/s", "ms_per_solve": tt / reps * 1e3, "l2_rel_err_vs_exact": res["rel_err"],
            "max_rel_diff_vs_fp64": vs64, "stage_kernel_ms": stage,
            "roofline": {"bound": "hbm", "achieved": FP32_STAGE_BYTES_PER_NODE * N_GRID ** 3 / (stage * 1e-3) / 1e9,
                         "unit": "GB/s",
                         "algorithmic_bytes_per_node": FP32_STAGE_BYTES_PER_NODE},
            "note": "same workload, FP32 state and stencils"}


def form_fp32_testcases(dev, n=48, steps=30):
    """The precision form per testcase: every testcase of the reference (include/*.h) and the
    two of this project on an n^3 grid, run in FP64 and in FP32 (state and stencils) from
    their own initial fields: the mass-weighted L2 error against the exact field at the final
    time (kernel_operator.cl:11-47 norm2_diff) in each precision, and the mass-weighted L2
    difference of the FP32 field from the FP64 one (absolute and relative to ||B_64||)."""
    import numpy as np

    from inductioneq_b200.induction_eq import Maps
    hp, tp = 4.0 * math.pi / 3.0, 2.0 * math.pi
    cases = {   # testcase: (lo, hi, periodic, order, hall, variable u, dissipation, integrator, dt)
        "rotation_2D": (-1.0, 1.0, False, 4, False, False, None, "SSPRK33", 0.5 * (2.0 / (n - 1)) / math.sqrt(2)),
        "rotation_3D": (-1.0, 1.0, False, 4, False, False, None, "SSPRK33", 0.4 * (2.0 / (n - 1)) / 1.7),
        "rotation_gaussian": (-1.0, 1.0, False, 4, False, False, None, "SSPRK33",
                              0.5 * (2.0 / (n - 1)) / math.sqrt(2)),
        "hall_periodic": (0.0, hp, True, 4, True, True, None, "CarpenterKennedy2N54", (2.0 / n) * (hp / n) / 2.0),
        "hall_travelling_wave": (0.0, tp, False, 4, True, True, None, "SSPRK33", 1e-3),
        "confined_domain": (0.0, 1.0, False, 4, True, False, None, "CarpenterKennedy2N54", 0.2 / (n - 1) ** 2),
        "alfven_periodic_2D": (0.0, 1.0, True, 4, False, True, None, "CarpenterKennedy2N54", 0.2 / n),
        "hall_circular_wave": (0.0, tp, True, 6, True, False, "USE_HIGH_ORDER_DISSIPATION", "CarpenterKennedy2N54",
                               0.2 * (tp / n) ** 2),
    }
    out = {}
    for tc, (lo, hi, per, order, hall, varu, diss, integ, dt) in cases.items():
        fields, res = {}, {}
        for real in ("double", "float"):
            m = Maps()
            m.I_Mesh.update({"NODES_X": n, "NODES_Y": n, "NODES_Z": n, "XMIN": lo, "XMAX": hi, "YMIN": lo,
                             "YMAX": hi, "ZMIN": lo, "ZMAX": hi})
            m.I_TI.update({"DT": dt, "time_integrator": integ})
            if hall:
                m.I_IEq["hall_term"] = "USE_HALL"
            if diss:
                m.I_IEq.update({"dissipation": "USE_ARTIFICIAL_DISSIPATION", "dissipation_form": diss})
            m.I_RunOps.update({"order": order, "testcase": tc, "periodic": "USE_PERIODIC" if per else "NONE",
                               "variable_u": varu})
            m.I_Tech["REAL"] = real
            ctx = m.context(device=dev)
            b, b2, b3, cb, u = ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec()
            rho, t = ctx.scalar(np.ones(ctx.n_pad)), ctx.scalar(np.zeros(2), n=2)
            ctx.kernel("init_b", b)
            ctx.kernel("init_u", u)
            ctx.time_steps(b, b2, b3, cb, u, rho, t, steps)
            res[real] = ctx.results(b, steps * dt, ctx.vec(), ctx.scalar())
            fields[real] = ctx.get_vec(b).astype(np.float64)
            if real == "double":
                keep = ctx   # the FP64 context measures the difference below
            else:
                ctx.close()
        d = math.sqrt(keep.norm2_diff(keep.vec(fields["float"]), keep.vec(fields["double"])))
        nb = math.sqrt(keep.norm2(keep.vec(fields["double"])))
        keep.close()
        out[tc] = {"grid": [n] * 3, "steps": steps, "dt": dt, "integrator": integ, "order": order,
                   "l2_err_vs_exact": {"fp64": res["double"]["abs_err"], "fp32": res["float"]["abs_err"]},
                   "l2_diff_fp32_vs_fp64": {"abs": d, "rel": d / nb if nb > 0 else None}}
    return out


def form_batched(dev, steps=200):
    """32 rotation solves, N ~ U{16..96}, omega ~ U(0.5,2), order in {2,4,6}, 200 SSPRK33 steps,
    one persistent launch captured in a CUDA graph, tile shapes from the autotuner; also the
    per-stage and per-solve-branch modes and the plain path on the same solves."""
    import numpy as np
    import torch

    from inductioneq_b200.batch import Batch, autotune, rotation_batch
    specs = rotation_batch(32, seed=2026)
    bt = Batch(specs, device=dev)
    name = torch.cuda.get_device_name(dev)
    tiles = autotune(bt, steps=3, gpu_name=name)
    stream = torch.cuda.ExternalStream(bt.stream, device=dev)
    flush = bt.ctxs[0].alloc(256 << 20)
    out = {}
    finals = {}
    for mode in ("persistent", "stages", "branches"):
        bt.init()
        bt.bind()
        bt.run(steps, mode=mode)   # capture + warm
        times = []
        for k in range(3):
            bt.init()
            bt.bind()
            bt.ctxs[0].memset(flush, k)
            bt.ctxs[0].synchronize()
            times.append(events_time(stream, lambda: bt.run(steps, mode=mode)))
        tmin = statistics.median(times)
        out[mode] = {"value": 3 * bt.total_nodes * 3 * steps / tmin, "ms": tmin * 1e3}
        bt.unbind()
        finals[mode] = [c.get_vec(f["b"]) for c, f in zip(bt.ctxs, bt.fields)]
    err = []
    for (n, o, om, dt), c, f in zip(specs, bt.ctxs, bt.fields):
        res = c.results(f["b"], steps * dt, c.vec(), c.scalar())
        err.append(res["rel_err"])
    # the plain FP64 path on the same workload: each solve through ieq_time_steps, one after another
    seq_s, seq_diff = 0.0, 0.0
    for i, (c, f) in enumerate(zip(bt.ctxs, bt.fields)):
        c.kernel("init_b", f["b"])
        f["time"].upload(np.zeros(2))
        cb, rho = c.vec(), c.scalar(np.ones(c.n_pad))
        cs = torch.cuda.ExternalStream(c.stream, device=dev)
        c.time_steps(f["b"], f["b2"], f["b3"], cb, f["u"], rho, f["time"], 2)   # graph capture + warm
        c.kernel("init_b", f["b"])
        f["time"].upload(np.zeros(2))
        c.synchronize()
        seq_s += events_time(cs, lambda: c.time_steps(f["b"], f["b2"], f["b3"], cb, f["u"], rho, f["time"], steps))
        got = c.get_vec(f["b"])
        for mode in finals:
            ref = finals[mode][i]
            seq_diff = max(seq_diff, float(np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-300)))
    nodes = bt.total_nodes
    grid = bt.grid()
    bt.close()
    best_mode = max(out, key=lambda m: out[m]["value"])
    best = out[best_mode]
    t = best["ms"] * 1e-3
    seq_value = 3 * nodes * 3 * steps / seq_s
    return {"value": best["value"], "unit": "DOF/s", "mode": best_mode, "solves": len(specs), "total_nodes": nodes,
            "steps": steps, "ms_per_run": best["ms"],
            "modes": {m: {"value": v["value"], "ms_per_run": v["ms"]} for m, v in out.items()},
            "plain_fp64_sequential": {"value": seq_value, "ms_per_run": seq_s * 1e3,
                                      "note": "the same 32 solves one after another through ieq_time_steps"},
            "max_rel_diff_batched_vs_plain": seq_diff,
            "persistent_grid": grid, "tiles": {k: list(v) for k, v in tiles.items()},
            "l2_rel_err_vs_exact": {"min": min(err), "median": statistics.median(err), "max": max(err),
                                    "note": "the width-0.1 Gaussian is under-resolved on the coarse grids "
                                            "(dx = 2/15 at N = 16)"},
            "roofline": {"bound": "hbm", "achieved": 88 * nodes * 3 * steps / t / 1e9, "unit": "GB/s",
                         "algorithmic_bytes_per_node_stage": 88},
            "seed": 2026}


def sharded_batch(rk, dev, steps=200, reps=3):
    """The 32-solve batch split between the ranks (inductioneq_b200.ranks.partition on
    nodes x stages; no communication in the data path): every rank runs its solves as one
    graph of per-solve branches; value = all solves' DOF-updates / max-over-ranks time
    (strong scaling: the batch is fixed)."""
    import torch

    from inductioneq_b200 import ranks as R
    from inductioneq_b200.batch import Batch, rotation_batch
    specs = rotation_batch(32, seed=2026)
    parts = R.partition([n ** 3 for (n, _, _, _) in specs], rk.world)
    mine = [specs[i] for i in parts[rk.rank]]
    total_nodes = sum(n ** 3 for (n, _, _, _) in specs)
    t = 0.0
    if mine:
        bt = Batch(mine, device=dev)
        stream = torch.cuda.ExternalStream(bt.stream, device=dev)
        bt.init()
        bt.bind()
        bt.run(steps, mode="branches")   # capture + warm
        times = []
        for _ in range(reps):
            bt.init()
            bt.bind()
            R.barrier(rk)
            times.append(events_time(stream, lambda: bt.run(steps, mode="branches")))
        bt.unbind()
        bt.close()
        t = statistics.median(times)
    else:
        for _ in range(reps):
            R.barrier(rk)
    t_max = R.max_over_ranks(rk, t, device="cuda")
    return {"metric": METRIC + " (batched form, 32 rotation solves split between the GPUs)",
            "value": 3 * total_nodes * 3 * steps / t_max, "unit": "DOF/s", "n_gpus": rk.world,
            "ms_per_run": t_max * 1e3, "higher_is_better": True, "scaling": "strong", "dtype": "f64",
            "data": "synthetic (seeded rotation batch, seed 2026)",
            "config": {"workload": "32 rotation solves, N ~ U{16..96}, orders 2/4/6, 200 SSPRK33 steps",
                       "solves_per_rank": [len(p) for p in parts], "mode": "branches"}}


def decomposed_solve(rk, dev, n=128, steps=4, reps=3):
    """One whistler solve (6th order + HOD, Hall, CK2N54, FP64, periodic n^3) decomposed into
    z slabs over the ranks (inductioneq_b200.decomp: each rank runs the fused stage kernels on
    its slab one RK stage at a time, ghost planes exchanged between stages through NCCL; the
    reference kernel lists with an exchange after every kernel are timed beside it); value =
    the solve's DOF-updates / max-over-ranks time (strong scaling: the grid is fixed)."""
    import numpy as np
    import torch

    from inductioneq_b200 import ranks as R
    from inductioneq_b200.decomp import SlabSolve
    dx = 2 * math.pi / n
    m = maps(n)
    m.I_TI.update({"DT": 0.2 * dx * dx})
    s = SlabSolve(m, rk, dev)
    g = m.context(device=dev)   # the initial state, made once on every rank
    b = g.vec()
    g.kernel("init_b", b)
    b0 = g.get_vec(b)[: g.n]
    g.close()
    def timed(fused):
        s.load(b0, None, np.ones(n ** 3))
        s.steps(1, fused=fused)   # warm
        times = []
        for _ in range(reps):
            s.load(b0, None, np.ones(n ** 3))
            R.barrier(rk)
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            s.steps(steps, fused=fused)
            times.append(time.perf_counter() - t0)
        return R.max_over_ranks(rk, statistics.median(times), device="cuda")

    t = timed(True)
    t_lists = timed(False)
    s.close()
    return {"metric": METRIC + " (one solve decomposed into z slabs)", "value": 3 * n ** 3 * STAGES * steps / t,
            "unit": "DOF/s", "n_gpus": rk.world, "ms_per_rk_step": t / steps * 1e3, "higher_is_better": True,
            "scaling": "strong", "dtype": "f64", "data": "synthetic (analytic whistler wave)",
            "kernel_lists": {"value": 3 * n ** 3 * STAGES * steps / t_lists, "ms_per_rk_step": t_lists / steps * 1e3},
            "config": {"workload": f"hall_circular_wave {n}^3 periodic, 6th order + HOD, CK2N54, decomposed into "
                                   f"{rk.world} z slabs", "ghost_planes": s.slabs.ghosts,
                       "timing": "host clock around the steps (the kernels of a slab and its exchanges are "
                                 "ordered by device synchronisation), max over ranks"}}


def form_precision(dev, n=128, steps=20):
    """Confined-domain Hall case on 128^3: FP32 state with FP64 CG cleaning to ||r||_2 < 1e-10,
    then CK2N54 steps; compared with the FP64 run.  Reported per precision: the weighted
    ||div B|| (sqrt(norm2_S(calc_div B))) before and right after the projection and after the
    steps; and the mass-weighted L2 difference of the FP32 field from the FP64 field, after
    the projection and after the steps."""
    import numpy as np
    import torch

    from inductioneq_b200.induction_eq import Maps
    out = {}
    fields = {}
    ctxs = {}
    for real in ("double", "float"):
        m = Maps()
        m.I_Mesh.update({"NODES_X": n, "NODES_Y": n, "NODES_Z": n, "XMIN": 0.0, "XMAX": 1.0, "YMIN": 0.0,
                         "YMAX": 1.0, "ZMIN": 0.0, "ZMAX": 1.0})
        dx = 1.0 / (n - 1)
        m.I_TI.update({"DT": 0.2 * dx * dx, "time_integrator": "CarpenterKennedy2N54"})
        m.I_IEq.update({"hall_term": "USE_HALL"})
        m.I_DC.update({"divergence_cleaning": True})
        m.I_Tech["REAL"] = real
        m.I_RunOps.update({"order": 4, "testcase": "confined_domain"})
        ctx = m.context(device=dev)
        ctxs[real] = ctx
        stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
        b = ctx.vec()
        ctx.kernel("init_b", b)
        bh = ctx.get_vec(b).astype(np.float64)
        bh[: ctx.n, :3] += 1e-3 * np.random.default_rng(12345).random((ctx.n, 3))
        b.upload(bh.astype(ctx.real))
        div_before = ctx.results(b, 0.0, ctx.vec(), ctx.scalar())["divergence_norm"]
        t0 = time.perf_counter()
        cg = ctx.clean_div(b, 20000, 1e-10, check=False)
        cg_s = time.perf_counter() - t0
        div_after = ctx.results(b, 0.0, ctx.vec(), ctx.scalar())["divergence_norm"]
        fields[(real, "projected")] = ctx.get_vec(b).astype(np.float64)
        b2, cb, u = ctx.vec(), ctx.vec(), ctx.vec()
        ctx.kernel("init_u", u)
        rho, tt = ctx.scalar(np.ones(ctx.n_pad)), ctx.scalar(np.zeros(2), n=2)
        b_proj = ctx.get_vec(b)
        ctx.time_steps(b, b2, None, cb, u, rho, tt, 2)   # capture + warm
        b.upload(b_proj)
        tt.upload(np.zeros(2, dtype=ctx.real))
        el = events_time(stream, lambda: ctx.time_steps(b, b2, None, cb, u, rho, tt, steps))
        res = ctx.results(b, 0.0, ctx.vec(), ctx.scalar())
        fields[(real, "stepped")] = ctx.get_vec(b).astype(np.float64)
        # the CG loop charged with its compulsory traffic: 80 B per interior node and iteration
        # (a fused two-pass CG: read u, r, write u, lap; read phi, u, r, lap, write phi, r),
        # over the wall clock of the whole cleaning (div B, CG, projection, host polls)
        interior = (n - 2) ** 3
        cg_gbs = 80.0 * interior * cg["iterations"] / cg_s / 1e9
        out[real] = {"dof_per_s": 3 * ctx.n * STAGES * steps / el, "cg_iterations": cg["iterations"],
                     "cg_residual_norm2": cg["residual_norm2"], "cg_converged": cg["converged"],
                     "cg_wall_s": cg_s, "cg_ms_per_iteration": cg_s / max(cg["iterations"], 1) * 1e3,
                     "cg_achieved_gbs_80B_per_node_iteration": cg_gbs,
                     "cg_residual_initial": cg["divergence_norm_initial"],
                     "weighted_div_norm_before_projection": div_before,
                     "weighted_div_norm_after_projection": div_after,
                     "weighted_div_norm_after_steps": res["divergence_norm"]}
    # mass-weighted L2 difference of the FP32 field from the FP64 field (norm2_diff of the
    # FP64 context), relative to the FP64 field's norm
    c64 = ctxs["double"]
    l2 = {}
    for when in ("projected", "stepped"):
        a, b = c64.vec(fields[("double", when)]), c64.vec(fields[("float", when)])
        d = c64.norm2_diff(b, a)
        nrm = c64.norm2(a)
        l2[when] = {"abs": d ** 0.5, "rel": (d / nrm) ** 0.5}
    diff = float(np.abs(fields[("float", "stepped")] - fields[("double", "stepped")]).max()
                 / np.abs(fields[("double", "stepped")]).max())
    for c in ctxs.values():
        c.close()
    return {"grid": [n] * 3, "steps": steps, "fp64": out["double"], "fp32_state_fp64_cg": out["float"],
            "l2_diff_fp32_vs_fp64_after_projection": l2["projected"],
            "l2_diff_fp32_vs_fp64_after_steps": l2["stepped"],
            "max_rel_diff_fp32_vs_fp64": diff,
            "note": "weighted div norm = sqrt(norm2_S(calc_div B)) (kernel_operator.cl); L2 diff = "
                    "sqrt(norm2_diff) relative to sqrt(norm2) of the FP64 field"}


def form_rotation40(dev, reps=5):
    """Linear rotation on 40^3 (the reference's CPU-runnable configuration): [-1, 1]^3, 4th-order
    SBP, u = (-y, x, 0), divergence-free Gaussian bump, SAT inflow, SSPRK33 at CFL 0.5 to t = 1
    (dt = 1/56, 56 steps), FP64: DOF-updates/s per stage and the L2 error against the exact
    rotated field."""
    import numpy as np
    import torch

    from inductioneq_b200.induction_eq import Maps
    n, steps = 40, 56
    m = Maps()
    m.I_Mesh.update({"NODES_X": n, "NODES_Y": n, "NODES_Z": n, "XMIN": -1.0, "XMAX": 1.0, "YMIN": -1.0,
                     "YMAX": 1.0, "ZMIN": -1.0, "ZMAX": 1.0})
    m.I_TI.update({"DT": 1.0 / steps, "time_integrator": "SSPRK33"})
    m.I_RunOps.update({"order": 4, "testcase": "rotation_gaussian"})
    ctx = m.context(device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    b, b2, b3, cb, u = ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec()
    rho, tt = ctx.scalar(np.ones(ctx.n_pad)), ctx.scalar(np.zeros(2), n=2)
    ctx.kernel("init_b", b)
    ctx.kernel("init_u", u)
    b0 = ctx.get_vec(b)
    ctx.time_steps(b, b2, b3, cb, u, rho, tt, steps)   # capture + warm
    flush = ctx.alloc(256 << 20)
    tsum = 0.0
    for k in range(reps):
        b.upload(b0)
        tt.upload(np.zeros(2))
        ctx.memset(flush, k)
        tsum += events_time(stream, lambda: ctx.time_steps(b, b2, b3, cb, u, rho, tt, steps))
    res = ctx.results(b, 1.0, ctx.vec(), ctx.scalar())
    ctx.close()
    t = tsum / reps
    return {"grid": [n] * 3, "steps": steps, "dt": 1.0 / steps, "t_final": 1.0, "value": 3 * n ** 3 * 3 * steps / t,
            "unit": "DOF/s", "ms_per_solve": t * 1e3, "l2_err_vs_exact": {"abs": res["abs_err"], "rel": res["rel_err"]},
            "note": "the 0.1-wide bump is about 2 dx on this grid: the error is the discretisation error of the "
                    "configuration, the same as the reference's (parity is tested separately)"}


def form_hbm256(dev, n=256, rk_steps=10):
    """The bench workload's kernels on 256^3 (16.8 M nodes: every field is larger than L2, so
    the stage runs from HBM): 6th-order SBP + high-order dissipation, Hall, u = 0, periodic,
    CK2N54, FP64, through the two-kernel stage (curl kernel writes E and H, stage kernel reads
    them: COLUMN) and through the one-pass stage (ZMARCH).  The whole stage (every kernel of
    it) is graded at the stage's compulsory 136 B/node (read b1, b2, rho; write b1', b2), and
    each kernel at its own traffic."""
    out = {"grid": [n] * 3, "rk_steps": rk_steps, "peak_gbs": _peak_hbm()}
    for kernel in ("COLUMN", "ZMARCH"):
        out[kernel.lower()] = _stage_rate(dev, n, rk_steps, kernel)
    return out


def _stage_rate(dev, n, rk_steps, kernel, tech=None):
    import numpy as np
    import torch

    dx = 2 * math.pi / n
    m = maps(n)
    m.I_TI.update({"DT": 0.2 * dx * dx})
    m.I_Tech["stage_kernel"] = kernel
    m.I_Tech.update(tech or {})
    ctx = m.context(device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    b, b2, cb, u = ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec()
    rho, tt = ctx.scalar(np.ones(ctx.n_pad)), ctx.scalar(np.zeros(2), n=2)
    ctx.kernel("init_b", b)
    ctx.time_steps(b, b2, None, cb, u, rho, tt, 2)   # capture + warm
    el = min(events_time(stream, lambda: ctx.time_steps(b, b2, None, cb, u, rho, tt, rk_steps)) for _ in range(3))
    prof = ctx.profile_step(b, b2, None, cb, u, rho, tt, repeats=5)
    ctx.close()
    peak = _peak_hbm()
    nn = n ** 3
    kernels = {}
    for nm, ms in prof:
        kernels.setdefault(nm, []).append(ms)
    per_stage = sum(sum(v) for v in kernels.values()) / STAGES * 1e-3
    compulsory = STAGE_BYTES_PER_NODE + 8          # + rho
    rec = {"value": 3 * nn * STAGES * rk_steps / el, "unit": "DOF/s", "ms_per_rk_step": el / rk_steps * 1e3,
           "stage_ms_sum_of_kernels": per_stage * 1e3,
           "whole_stage": {"bytes_per_node": compulsory,
                           "achieved_gbs": compulsory * nn / per_stage / 1e9,
                           "frac": compulsory * nn / per_stage / 1e9 / peak,
                           "frac_wall": compulsory * nn * STAGES * rk_steps / el / 1e9 / peak},
           "kernels": {}}
    hodp = (tech or {}).get("hodp", 1)
    own = {"curl_rho": CURL_BYTES_PER_NODE if hodp else CURL_BYTES_PER_NODE - 24,
           "stage_2n_fused": (144 if hodp else 120) if kernel != "ZMARCH" else compulsory}
    for nm, v in kernels.items():
        ms = statistics.mean(v)
        r = {"launches_per_step": len(v), "avg_ms": ms}
        if nm in own:
            r.update({"bytes_per_node": own[nm], "frac": own[nm] * nn / (ms * 1e-3) / 1e9 / peak})
        rec["kernels"][nm] = r
    return rec


def _peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f).get("hbm_gbs") or 6650.0
    except OSError:
        return 6650.0


def form_adjoint(dev, n=64, t_final=0.2, every=10, n_dirs=20):
    """Hall periodic (include/hall_periodic.h) 64^3, FP64, 4th order, variable u, SSPRK33 at CFL 1/N
    to t = 0.2: gradient of J = 1/2 ||B(T) - B_tgt||_M^2 (B_tgt = exact(T) + seeded N(0, 1e-3)) with
    respect to B0 by the checkpointed adjoint, checked against Richardson-extrapolated central
    differences along seeded unit directions."""
    import numpy as np

    from inductioneq_b200.induction_eq import Maps
    hp = 4.0 * math.pi / 3.0

    def mk(dt):
        m = Maps()
        m.I_Mesh.update({"NODES_X": n, "NODES_Y": n, "NODES_Z": n, "XMIN": 0.0, "XMAX": hp, "YMIN": 0.0, "YMAX": hp,
                         "ZMIN": 0.0, "ZMAX": hp})
        m.I_TI.update({"DT": dt, "time_integrator": "SSPRK33"})
        m.I_IEq.update({"hall_term": "USE_HALL"})
        m.I_RunOps.update({"order": 4, "testcase": "hall_periodic", "periodic": "USE_PERIODIC", "variable_u": True})
        return m.context(device=dev)

    ctx = mk(1.0)
    u = ctx.vec()
    ctx.kernel("init_u", u)
    umax = float(np.sqrt((ctx.get_vec(u)[:, :3] ** 2).sum(1)).max())
    ctx.close()
    dx = hp / n
    # initialize.m:93-99 with CFL 1/N: the reference example pairs CFL 2/N with
    # CarpenterKennedy2N54 (compute_error_hall_periodic.m:51-57); SSPRK33, whose stability
    # interval on the imaginary axis is shorter, blows up at CFL 2/N on 64^3
    dt = (1.0 / n) * dx / umax
    steps = math.ceil(t_final / dt)
    dt = t_final / steps
    ctx = mk(dt)
    b, b2, b3, cb, u = ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec()
    rho = ctx.scalar(np.ones(ctx.n_pad))
    ctx.kernel("init_b", b)
    b0 = ctx.get_vec(b)
    wmass = dx ** 3
    tb = ctx.scalar(np.array([t_final, t_final]), n=2)
    ana = ctx.vec()
    ctx.run("analytical_b", (n, n, n), ana, tb)
    rng = np.random.default_rng(2026)
    target = ctx.get_vec(ana)
    target[: ctx.n, :3] += 1e-3 * rng.standard_normal((ctx.n, 3))

    def forward(x):
        b.upload(x)
        ctx.kernel("init_u", u)
        t = ctx.scalar(np.zeros(2), n=2)
        ctx.time_steps(b, b2, b3, cb, u, rho, t, steps)
        return ctx.get_vec(b)

    def loss(x):
        d = forward(x)[: ctx.n, :3] - target[: ctx.n, :3]
        return 0.5 * wmass * float(np.sum(d * d))

    t0 = time.perf_counter()
    bT = forward(b0)
    t_fwd = time.perf_counter() - t0
    lam = ctx.vec()
    g = np.zeros_like(bT)
    g[: ctx.n, :3] = wmass * (bT[: ctx.n, :3] - target[: ctx.n, :3])
    b0_dev = ctx.vec(b0)
    # the first sweep sizes the context's checkpoint pool; the second, timed, allocates nothing
    lam.upload(g)
    ctx.adjoint_steps(b0_dev, lam, u, rho, steps, every)
    lam.upload(g)
    ctx.synchronize()
    t0 = time.perf_counter()
    ctx.adjoint_steps(b0_dev, lam, u, rho, steps, every)
    t_adj = time.perf_counter() - t0
    grad = ctx.get_vec(lam)
    worst = 0.0
    pairs = []
    for k in range(n_dirs):
        d = rng.standard_normal(b0.shape)
        d[:, 3] = 0
        d[ctx.n:] = 0
        d /= np.sqrt(np.sum(d[:, :3] ** 2))
        ad = float(np.sum(grad[:, :3] * d[:, :3]))
        eps = 1e-3

        def cd(e):
            return (loss(b0 + e * d) - loss(b0 - e * d)) / (2 * e)
        fd = (4.0 * cd(eps / 2) - cd(eps)) / 3.0          # Richardson: O(eps^4)
        r = abs(fd - ad) / abs(ad)
        worst = r if not math.isfinite(r) else max(worst, r)
        if len(pairs) < 3:
            pairs.append([ad, fd])
    loss0 = loss(b0)
    ctx.close()
    return {"grid": [n] * 3, "steps": steps, "dt": dt, "checkpoint_every": every, "forward_s": t_fwd,
            "adjoint_s": t_adj, "fd_directions": n_dirs, "fd": "Richardson-extrapolated central differences, eps 1e-3 and 5e-4",
            "max_rel_diff_vs_fd": worst, "first_pairs_adjoint_fd": pairs,
            "loss": loss0, "grad_norm": float(np.sqrt(np.sum(grad[:, :3] ** 2)))}


# ------------------------------------------------------------------------------ main
def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the FP32 / batched / precision lines")
    ap.add_argument("--stage-kernel", choices=("AUTO", "COLUMN", "BRICK", "ZMARCH"), default="AUTO",
                    help="kernels of the fused stages (IEQ_STAGE_KERNEL)")
    ap.add_argument("--no-pairs", action="store_true",
                    help="one node per thread in the Hall column kernels (IEQ_COL_PAIRS=0)")
    ap.add_argument("--sharded-batch", action="store_true",
                    help="only the batched form, its 32 solves split between the ranks")
    ap.add_argument("--decomposed", action="store_true",
                    help="one 128^3 whistler solve decomposed into z slabs over the ranks")
    ap.add_argument("--form", default=None,
                    help="run only this form (fp32, rotation_c1, hbm_256, batched, precision_c3, adjoint_c5, "
                         "fp32_testcases) "
                         "on one GPU and print its JSON")
    a = ap.parse_args()
    from inductioneq_b200 import ranks as R
    rk = R.Ranks.from_env()
    world, rank, local_rank = rk.world, rk.rank, rk.local_rank

    if a.impl == "reference":
        if rank != 0:
            return
        # each timed step is a bounded sample of the solve: REF_RK_PER_STEP whole RK steps,
        # timed as they run (ms_per_step is the measured time of one such step)
        ref = cpu_reference_run(a.steps, a.warmup, rk_per_step=REF_RK_PER_STEP)
        value = ref["value"]
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "DOF/s", "n_gpus": a.gpus, "steps": ref["steps"],
            "warmup": a.warmup, "ms_per_step": ref["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic whistler wave)",
            "config": {"workload": WORKLOAD, "grid": [N_GRID] * 3, "stages_per_rk_step": STAGES,
                       "step": f"a sample of {REF_RK_PER_STEP} CK2N54 RK steps of the 260-step solve"},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "DOF/s", "cores": ref["cores"], "kind": ref["kind"],
                             "sample": ref["sample"], "build": ref["build"], "cpu": ref["cpu"],
                             "nproc": ref["nproc"]},
            "e2e": {"value": value, "unit": "DOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    import numpy as np
    import torch

    R.init(rk, "nccl", timeout_s=120.0)
    dev = local_rank
    torch.cuda.set_device(dev)
    if a.form:
        forms = {"rotation_c1": form_rotation40, "hbm_256": form_hbm256, "batched": form_batched,
                 "precision_c3": form_precision, "adjoint_c5": form_adjoint, "fp32_testcases": form_fp32_testcases}
        print(json.dumps({a.form: forms[a.form](dev)}))
        R.finish(rk)
        return
    if a.decomposed:
        line = decomposed_solve(rk, dev)
        if rank == 0:
            print(json.dumps(line))
        R.finish(rk)
        return
    if a.sharded_batch:
        line = sharded_batch(rk, dev)
        if rank == 0:
            print(json.dumps(line))
        R.finish(rk)
        return
    m = maps()
    m.I_Tech["stage_kernel"] = a.stage_kernel
    if a.no_pairs:
        m.I_Tech["col_pairs"] = 0
    ctx = m.context(device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    nn = ctx.n
    b, b2, cb, u = ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec()
    rho = ctx.scalar()
    tbuf = ctx.scalar(np.zeros(2), n=2)
    ctx.kernel("init_b", b)
    ctx.kernel("init_u", u)
    ctx.kernel("init_rho", rho)
    b0 = ctx.get_vec(b)
    flush = ctx.alloc(256 << 20)

    def barrier():
        R.barrier(rk)

    def solve():
        b.upload(b0)
        tbuf.upload(np.zeros(2))

    # ---------------- warm-up (graph capture happens on the first call)
    for _ in range(a.warmup):
        solve()
        ctx.time_steps(b, b2, None, cb, u, rho, tbuf, NUM_STEPS_FULL)
    ctx.synchronize()

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    clocks.start()
    time.sleep(0.5)

    # ---------------- timed region: K full solves (graph-launched steps), L2 flushed between
    K = a.steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    barrier()
    torch.cuda.synchronize()
    for k in range(K):
        solve()
        ctx.memset(flush, k & 0xFF)
        ev[k][0].record(stream)
        ctx.time_steps(b, b2, None, cb, u, rho, tbuf, NUM_STEPS_FULL)
        ev[k][1].record(stream)
    ctx.synchronize()
    res = ctx.results(b, T_FINAL, ctx.vec(), ctx.scalar())   # stated L2 error of the timed solve
    # dominant-kernel timing inside the same region: every launch of one step timed alone as
    # a graph of 20 back-to-back launches (CUDA events on the solver stream)
    solve()
    prof = [ctx.profile_step(b, b2, None, cb, u, rho, tbuf, repeats=20)]
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    step_ms = [s_.elapsed_time(e_) for s_, e_ in ev]
    t_total = sum(step_ms) * 1e-3
    t_max = R.max_over_ranks(rk, t_total, device="cuda")
    dof = 3 * nn * STAGES * NUM_STEPS_FULL * K * world
    value = dof / t_max
    stage_ms = [ms for rec in prof for (nm, ms) in rec if nm.startswith("stage")]
    curl_ms = [ms for rec in prof for (nm, ms) in rec if nm == "curl_rho"]
    stage_avg = statistics.mean(stage_ms) * 1e-3
    curl_avg = statistics.mean(curl_ms) * 1e-3

    # ---------------- end to end through the C ABI with host buffers (pinned): per solve,
    # the initial state goes host -> device and the final state device -> host
    h_b = torch.empty((ctx.n_pad, 4), dtype=torch.float64, pin_memory=True)
    h_b.copy_(torch.from_numpy(b0))
    h_t = torch.zeros(2, dtype=torch.float64, pin_memory=True)
    h_out = torch.empty_like(h_b)
    Ke = K
    eev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(Ke)]
    h2d = h_b.numel() * 8 + 16
    d2h = h_b.numel() * 8
    barrier()
    torch.cuda.synchronize()
    for k in range(Ke):
        ctx.memset(flush, k & 0xFF)
        eev[k][0].record(stream)
        ctx._check(ctx.lib.ieq_upload(ctx.h, b.ptr, h_b.data_ptr(), h_b.numel() * 8))
        ctx._check(ctx.lib.ieq_upload(ctx.h, tbuf.ptr, h_t.data_ptr(), 16))
        ctx.time_steps(b, b2, None, cb, u, rho, tbuf, NUM_STEPS_FULL)
        ctx._check(ctx.lib.ieq_download(ctx.h, h_out.data_ptr(), b.ptr, h_out.numel() * 8))
        eev[k][1].record(stream)
    ctx.synchronize()
    e2e_t = R.max_over_ranks(rk, sum(s_.elapsed_time(e_) for s_, e_ in eev) * 1e-3, device="cuda")
    e2e_value = 3 * nn * STAGES * NUM_STEPS_FULL * Ke * world / e2e_t

    # ---------------- roofline of the dominant kernel (fused stage kernel)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    achieved = STAGE_BYTES_PER_NODE * nn / stage_avg / 1e9
    kname = ("k_stage_brick" if a.stage_kernel == "BRICK" else "k_stage_col" if a.no_pairs else "k_stage_hall_x2")
    roofline = {"bound": "hbm", "kernel": kname + "<double, 6th classical, periodic, Hall, HOD, u=0> (fused CK2N54 a+b)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_src, "traffic": None,
                "algorithmic_bytes_per_node": STAGE_BYTES_PER_NODE, "nodes_per_launch": nn,
                "avg_launch_ms": stage_avg * 1e3, "curl_kernel_avg_ms": curl_avg * 1e3,
                "curl_kernel_bytes_per_node": CURL_BYTES_PER_NODE,
                "stage_pair_frac": STAGE_BYTES_PER_NODE * nn / (stage_avg + curl_avg) / 1e9 / peak,
                "note": "CUDA events around a graph of 20 back-to-back launches of each kernel of one step "
                        "(L2 warm, as inside a solve); stage_pair_frac charges the stage's compulsory bytes "
                        "to the curl and stage kernels together"}
    # DRAM bytes (read + write) of one launch of the stage kernel, from the ncu capture
    # summarised in profiles/ ("traffic_bytes_per_launch: N" line of the kernel's summary)
    summary = os.path.join(ROOT, "profiles", f"{kname}_hall6_64cubed.md")
    if os.path.isfile(summary):
        with open(summary) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    roofline["traffic"] = int(line.split(":", 1)[1].strip())
                    roofline["traffic_note"] = ("ncu capture with caches flushed before the launch: the inputs "
                                                "come from DRAM, the writes stay in L2")

    # the FP64 roof beside the HBM roof: the device's FMA-loop rate (measured here, after the
    # timed region) and the stage kernel's FP64 FLOPs per launch (2 x DFMA + DADD + DMUL
    # thread instructions from an ncu count, in the kernel's summary under profiles/)
    flops = None
    if os.path.isfile(summary):
        with open(summary) as f:
            for line in f:
                if line.startswith("fp64_flops_per_launch:"):
                    flops = int(line.split(":", 1)[1].strip())
    from inductioneq_b200 import lib as L
    fp64_peak_tflops = L.fp64_fma_rate(dev) / 1e3
    fp64_roof = {"bound": "fp64", "peak": fp64_peak_tflops, "unit": "TFLOP/s",
                 "peak_source": "measured: ieq_fp64_fma_rate (FMA loop, 8 chains per thread, 8 blocks of 256 per SM)"}
    if flops:
        fp64_roof.update({"achieved": flops / stage_avg / 1e12, "frac": flops / stage_avg / 1e12 / fp64_peak_tflops,
                          "flops_per_launch": flops, "flops_per_node": flops / nn,
                          "flops_source": "ncu thread-instruction counts: 2 x DFMA + DADD + DMUL"})
    curl_summary = os.path.join(ROOT, "profiles", "k_curl_e_x2_hall6_64cubed.md")
    if not a.no_pairs and a.stage_kernel != "BRICK" and os.path.isfile(curl_summary):
        with open(curl_summary) as f:
            for line in f:
                if line.startswith("fp64_flops_per_launch:"):
                    cf = int(line.split(":", 1)[1].strip())
                    fp64_roof.update({"curl_kernel_flops_per_node": cf / nn,
                                      "curl_kernel_frac": cf / curl_avg / 1e12 / fp64_peak_tflops})
    roofline["fp64_roof"] = fp64_roof

    out = {
        "metric": METRIC, "value": value, "unit": "DOF/s", "n_gpus": world, "steps": K, "warmup": a.warmup,
        "ms_per_step": t_max / K * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (analytic whistler wave)",
        "config": {"workload": WORKLOAD, "grid": [N_GRID] * 3, "rk_steps_per_step": NUM_STEPS_FULL,
                   "stage_kernels": a.stage_kernel, "nodes_per_thread": 1 if a.no_pairs else 2,
                   "stages_per_rk_step": STAGES, "step": "one full solve to t=0.5 (260 RK steps)",
                   "l2": L2_NOTE, "replicas": world},
        "e2e": {"value": e2e_value, "unit": "DOF/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "ieq_upload (pinned host) + ieq_time_steps(260) + ieq_download per solve"},
        # per solve: u = 0 test (1), AoS -> SoA of b, b2, J, u (4), curl + stage per RK stage,
        # J of the last stage input (1), SoA -> AoS of b, b2, J (3)
        "gpu_launches": (2 * STAGES * NUM_STEPS_FULL + 9) * K,
        "roofline": roofline,
        "l2_error": {"rel": res["rel_err"], "abs": res["abs_err"], "t": T_FINAL, "steps": NUM_STEPS_FULL,
                     "divergence_norm": res["divergence_norm"]},
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not a.no_forms:
        b_ref = None
        try:
            b.upload(b0)
            tbuf.upload(np.zeros(2))
            ctx.time_steps(b, b2, None, cb, u, rho, tbuf, NUM_STEPS_FULL)
            b_ref = ctx.get_vec(b)
            out["forms"] = {"fp32": form_fp32(dev, b_ref)}
        except Exception as e:   # a form that fails is reported, not fatal to the line
            out["forms"] = {"fp32": {"error": repr(e)}}
        for name, fn in (("rotation_c1", form_rotation40), ("hbm_256", form_hbm256), ("batched", form_batched),
                         ("precision_c3", form_precision), ("adjoint_c5", form_adjoint),
                         ("fp32_testcases", form_fp32_testcases)):
            try:
                out["forms"][name] = fn(dev)
            except Exception as e:
                out["forms"][name] = {"error": repr(e)}
    hb = out.get("forms", {}).get("hbm_256", {}).get("column")
    if isinstance(hb, dict) and "whole_stage" in hb:
        # the same kernels where every field is HBM resident: the whole stage at the stage's
        # compulsory bytes, and each kernel at its own traffic (DRAM bytes per launch from the
        # ncu summary of that size)
        rec = {"grid": [256] * 3, "whole_stage_frac": hb["whole_stage"]["frac"],
               "whole_stage_bytes_per_node": hb["whole_stage"]["bytes_per_node"],
               "stage_kernel_frac": hb["kernels"].get("stage_2n_fused", {}).get("frac"),
               "curl_kernel_frac": hb["kernels"].get("curl_rho", {}).get("frac"), "peak": peak,
               "peak_source": peak_src}
        summ = os.path.join(ROOT, "profiles", "hbm_stage_kernels_hall6_256cubed.md")
        if os.path.isfile(summ):
            with open(summ) as f:
                for line in f:
                    if line.startswith("traffic_bytes_per_launch"):
                        rec["stage_kernel_traffic_per_launch"] = int(line.split(":", 1)[1].split()[0])
        roofline["hbm_resident"] = rec
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        ref = cpu_reference_run(10 ** 6, 1, budget_s=15.0)
        one = cpu_reference_run(10 ** 6, 1, budget_s=4.0, threads=1)
        out["cpu_baseline"] = {"value": ref["value"], "unit": "DOF/s", "cores": ref["cores"], "kind": ref["kind"],
                               "sample": ref["sample"], "build": ref["build"], "cpu": ref["cpu"],
                               "nproc": ref["nproc"], "one_core": {"value": one["value"], "sample": one["sample"]}}
    if rank == 0:
        print(json.dumps(out))
    ctx.close()
    R.finish(rk)


if __name__ == "__main__":
    main()
