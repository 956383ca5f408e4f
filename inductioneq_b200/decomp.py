"""Domain decomposition of one solve into z slabs, one slab per rank (one process per GPU).

The reference runs one grid on one device (matlab/+induction_eq/initialize.m:31-34); its
paper sweeps go to 320^3 and beyond (paper/convergence_rotation_3D.m:104).  Here rank k of
P owns the contiguous planes [z0_k, z1_k) of the global grid -- in the reference layout,
idx = ix + NX*(iy + NY*iz), a z slab is one contiguous block of memory -- and holds ghost
planes beside its owned ones.  The rank's context is the global settings with NODES_Z = the
slab's planes (ghosts included), the global spacing and the slab's z offset, so that testcase
coordinates (init, u_analytical, analytical_b, b_boundary) are those of the global grid.

Periodic grids: G = 2 * (ORDER/2) ghost planes on each side of every slab -- the Hall term
reaches ORDER/2 planes for curl(B)/rho and ORDER/2 more for the flux rows of E = J x B, the
volume, dissipation and convection terms reach ORDER/2 -- and the slab is itself periodic:
the rows that wrap at its ends are ghost rows.

Boxes (non-periodic): no ghost planes at the global ends (the slab's end is the box's face,
with its SBP boundary rows and SAT terms); G = NUM_BOUNDS + ORDER/2 ghost planes at an end
inside the grid.  The slab is an ordinary box of the stencil kernels: its own boundary rows
and face terms at an inner end fall on the ghost planes only, every owned node is at least
NUM_BOUNDS planes from that end (an interior row, as in the global grid), and every value
of curl(B)/rho an owned node reads (ORDER/2 planes away) is itself formed by an interior row
from valid ghost values.  So the box kernels run unchanged on the slab.

A step runs the integrator on the local slab either through the context's fused stage kernels,
one RK stage at a time (ieq_stages_*: the ghost planes of the state fields are refreshed after
every stage), or as the reference's kernel list (compute_numerical_solution_setup.m:140-371).
After every stage -- every kernel of the list that writes a state field (all but
calc_curlB_rho_*, calc_u_* and calc_time_*) -- the state fields' ghost planes are refreshed from
the neighbours' owned planes: the G planes at the bottom of the owned range go to the rank
below, the G at the top to the rank above (periodic grids: rank 0's lower neighbour is rank
P-1) -- one point-to-point exchange per neighbour and field (NCCL between GPUs, gloo on CPU).
curl(B)/rho is recomputed on every local plane from fresh ghosts, so it is never exchanged;
its values near the slab's inner ends are not valid and are never read by an owned node.
Each owned node then performs exactly the arithmetic of the undecomposed run, so the
decomposed fields equal it bit for bit.  `run_local` runs the slabs of several ranks in one
process on one device, stage by stage, with the ghost planes copied between their buffers.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .ranks import Ranks

# kernels that write no state field (their outputs are recomputed on every local plane)
_NO_EXCHANGE = ("calc_curlB_rho", "calc_u", "calc_time")


def slab_bounds(nz: int, world: int) -> list[tuple[int, int]]:
    """Contiguous, balanced [z0, z1) ranges of the ranks (the first nz % world ranks one
    plane longer)."""
    q, r = divmod(nz, world)
    out, z = [], 0
    for k in range(world):
        n = q + (1 if k < r else 0)
        out.append((z, z + n))
        z += n
    return out


@dataclass
class ZSlabs:
    """One rank's view of the decomposition of an (nx, ny, nz) grid: `ghosts` planes at every
    slab end of a periodic grid, at the ends inside the grid of a box."""
    ranks: Ranks
    nx: int
    ny: int
    nz: int
    ghosts: int
    periodic: bool = True

    def __post_init__(self):
        w, r = self.ranks.world, self.ranks.rank
        self.bounds = slab_bounds(self.nz, w)
        self.z0, self.z1 = self.bounds[r]
        if w > 1 and min(b - a for a, b in self.bounds) < self.ghosts:
            raise ValueError(f"every rank must own at least {self.ghosts} planes (the ghost depth): "
                             f"{self.nz} planes over {w} ranks")
        if self.periodic:
            if self.owned < self.ghosts:
                raise ValueError(f"a periodic slab must own at least {self.ghosts} planes (the ghost depth)")
            self.g_lo = self.g_hi = self.ghosts
            self.up, self.down = (r + 1) % w, (r - 1) % w
        else:
            self.g_lo = self.ghosts if r > 0 else 0
            self.g_hi = self.ghosts if r < w - 1 else 0
            self.up = r + 1 if r < w - 1 else None
            self.down = r - 1 if r > 0 else None

    @property
    def owned(self) -> int:
        return self.z1 - self.z0

    @property
    def nloc(self) -> int:
        return self.owned + self.g_lo + self.g_hi

    @property
    def plane(self) -> int:
        return self.nx * self.ny

    @property
    def local_nodes(self) -> tuple[int, int, int]:
        return (self.nx, self.ny, self.nloc)

    @property
    def z_offset(self) -> int:
        """Global plane of local plane 0."""
        return self.z0 - self.g_lo

    def scatter(self, glob: np.ndarray) -> np.ndarray:
        """The local slab (ghosts included) of a global field in the reference layout
        ((N,) or (N, C) rows, N = nx*ny*nz); periodic grids wrap in z."""
        g = glob[: self.nz * self.plane].reshape((self.nz, self.plane) + glob.shape[1:])
        zs = np.arange(self.z_offset, self.z_offset + self.nloc) % self.nz
        return np.ascontiguousarray(g[zs].reshape((self.nloc * self.plane,) + glob.shape[1:]))

    def owned_rows(self) -> slice:
        """Rows of the owned planes in a local field."""
        return slice(self.g_lo * self.plane, (self.g_lo + self.owned) * self.plane)

    def global_rows(self) -> slice:
        """Rows of the owned planes in the global field."""
        return slice(self.z0 * self.plane, self.z1 * self.plane)

    def parts(self, t):
        """(lower ghosts, lowest G owned planes, highest G owned planes, upper ghosts) of a
        local field (rows in the reference layout)."""
        G, P, n, lo = self.ghosts, self.plane, self.owned, self.g_lo
        return (t[0: lo * P], t[lo * P: (lo + G) * P], t[(lo + n - G) * P: (lo + n) * P],
                t[(lo + n) * P: (lo + n + self.g_hi) * P])

    def exchange(self, *fields) -> None:
        """Refresh the ghost planes of every field (torch tensors or numpy arrays over the
        local slab, rows in the reference layout; padded rows beyond the slab are ignored)
        from the neighbours' owned planes."""
        import torch
        for f in fields:
            t = torch.from_numpy(f) if isinstance(f, np.ndarray) else f
            lo_ghost, lo_owned, hi_owned, hi_ghost = self.parts(t)
            if self.ranks.world == 1:
                if self.periodic:
                    lo_ghost.copy_(hi_owned)
                    hi_ghost.copy_(lo_owned)
                continue
            import torch.distributed as dist
            ops, recv = [], []
            # posted in this order on every rank: with two periodic ranks (up == down) the
            # first message between a pair is the sender's bottom block, the receiver's top
            # ghosts
            if self.down is not None:
                ops.append(dist.P2POp(dist.isend, lo_owned.contiguous(), self.down))
            if self.up is not None:
                ops.append(dist.P2POp(dist.isend, hi_owned.contiguous(), self.up))
            if self.up is not None:
                rh = torch.empty_like(hi_ghost)
                ops.append(dist.P2POp(dist.irecv, rh, self.up))
                recv.append((hi_ghost, rh))
            if self.down is not None:
                rl = torch.empty_like(lo_ghost)
                ops.append(dist.P2POp(dist.irecv, rl, self.down))
                recv.append((lo_ghost, rl))
            for req in dist.batch_isend_irecv(ops):
                req.wait()
            for dst, src in recv:
                dst.copy_(src)


def exchange_local(slabs: list, fields: list) -> None:
    """The ghost exchange of the ranks of one decomposition held in one process: slabs[k] is
    rank k's ZSlabs, fields[k] its list of local fields (the same fields in the same order on
    every rank); every ghost block is copied from the neighbour's owned planes."""
    for i in range(len(fields[0])):
        parts = [sl.parts(f[i]) for sl, f in zip(slabs, fields)]
        for k, sl in enumerate(slabs):
            if sl.down is not None:
                parts[k][0].copy_(parts[sl.down][2])
            if sl.up is not None:
                parts[k][3].copy_(parts[sl.up][1])


def exchanges_after(kernel: str) -> bool:
    """Whether a kernel of the step list writes a state field (b, b2, b3/db)."""
    return not kernel.startswith(_NO_EXCHANGE)


def decomposed_steps(slabs: ZSlabs, runner, seq, num_steps: int, state, args, sync=None) -> None:
    """num_steps steps of the kernel list `seq` (the integrator's step, e.g. from
    Context.step_kernels) on the local slab, with the ghost exchanges of the state fields
    between kernels.  `runner.run(name, nodes, *args)` runs one reference kernel on the local
    grid (the C ABI's ieq_run_kernels on a GPU); `args` is the kernels' uniform argument list
    (b1, b2, [b3 | db], curlB_rho, u, rho, time) and `state` the fields among them that the
    kernels write (b1, b2[, b3]); `sync()` orders the runner's device work before an exchange
    and the exchange before the next kernel."""
    nodes = slabs.local_nodes
    for _ in range(num_steps):
        for k in seq:
            runner.run(k, nodes, *args)
            if exchanges_after(k):
                if sync:
                    sync()
                slabs.exchange(*state)
                if sync:
                    sync()


def is_periodic(maps) -> bool:
    return maps.I_RunOps.get("periodic") == "USE_PERIODIC"


def local_maps(maps, slabs: ZSlabs):
    """The settings of one rank's slab: the global maps with NODES_Z = the slab's planes
    including ghosts, the global spacing and the slab's z offset."""
    import copy
    if is_periodic(maps) != slabs.periodic:
        raise ValueError("the slabs and the settings disagree on whether the grid is periodic")
    m = copy.deepcopy(maps)
    m.spacing_override = maps.spacing()
    m.I_Mesh["NODES_Z"] = slabs.nloc
    m.I_Tech["z_offset"] = slabs.z_offset
    m.I_Tech["nz_global"] = slabs.nz
    return m


# NUM_BOUNDS (boundary rows at each end) of the SBP operators (include/*Order*.h), by
# (order, extended)
NUM_BOUNDS = {(2, False): 1, (4, False): 4, (6, False): 6, (2, True): 3, (4, True): 6, (6, True): 8}


LAPLACE_KEYS = {"WIDE_STENCIL_DIRICHLET": "WS_D0", "NARROW_STENCIL_DIRICHLET": "NS_D0", "WIDE_STENCIL_LNS": "WS_LN"}


def laplace_rows(order: int, extended: bool, laplace: str) -> tuple[int, int]:
    """(boundary rows at each end, stencil width) of the divergence cleaning's Laplacian
    (kernel_div_cleaning.cl:11-56 on the include/*Order*.h tables)."""
    import json
    import os
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "sbp_tables.json")) as f:
        t = json.load(f)
    lap = t[f"{order}{'e' if extended else 'c'}"]["laplace"][LAPLACE_KEYS[laplace]]
    return int(lap["nb"]), int(lap["width"])


def bnodes_of(laplace: str) -> int:
    """BNODES: the Dirichlet layer the CG leaves at every face (0 for the LNS form)."""
    return 0 if laplace == "WIDE_STENCIL_LNS" else 1


def ghost_depth(order: int, periodic: bool = True, extended: bool = False,
                laplace: str = "WIDE_STENCIL_DIRICHLET") -> int:
    """Ghost planes a slab needs at an end.  Periodic grids: ORDER/2 for curl(B)/rho and
    ORDER/2 for the flux rows of E (interior rows everywhere).  Boxes, at an end inside the
    grid: NUM_BOUNDS, so that the slab's own boundary rows there cover ghost planes only, plus
    ORDER/2, so that the curl(B)/rho values an owned node reads are formed by interior rows;
    and at least the divergence cleaning's Laplacian boundary rows and reach and the CG's
    Dirichlet layer, so that a decomposed cleaning gives every owned node the global grid's
    rows too."""
    if periodic:
        return 2 * (order // 2)
    nb_l, w_l = laplace_rows(order, extended, laplace)
    return max(NUM_BOUNDS[(order, extended)] + order // 2, nb_l, (w_l - 1) // 2, bnodes_of(laplace))


TWO_FIELD_INTEGRATORS = ("CarpenterKennedy2N54", "ToulorgeDesmet2N84F")


class _DeviceArray:
    """A 1-D device array by address (the CUDA array interface), for torch.as_tensor."""

    def __init__(self, ptr: int, n: int, dtype):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": np.dtype(dtype).str,
                                         "data": (int(ptr), False), "version": 3}


class SlabSolve:
    """One rank's slab of a decomposed solve (periodic grid or box) on its GPU: the local
    context (fused stage kernels or the C ABI's reference kernels) on torch device buffers,
    the ghost exchanges through torch.distributed (NCCL between GPUs; a local copy with one
    periodic rank), or between the slabs of one process with `run_local`."""

    def __init__(self, maps, ranks: Ranks, device: int = 0):
        import torch
        m = maps.I_Mesh
        self.ranks = ranks
        per = is_periodic(maps)
        ext = maps.I_RunOps.get("operator_form", "classical") == "extended"
        self.laplace = maps.I_DC["divergence_cleaning_form"].replace("USE_LAPLACE_", "")
        self.slabs = ZSlabs(ranks, int(m["NODES_X"]), int(m["NODES_Y"]), int(m["NODES_Z"]),
                            ghost_depth(int(maps.I_RunOps["order"]), per, ext, self.laplace), per)
        self.device = device
        self.ctx = local_maps(maps, self.slabs).context(device)
        # the integrator's kernel list (none without an integrator: a slab only cleaned)
        self.seq = self.ctx.step_kernels() if maps.I_TI.get("time_integrator") else []
        self.nf = 2 if maps.I_TI["time_integrator"] in TWO_FIELD_INTEGRATORS else 3
        dt = torch.float32 if self.ctx.real == np.float32 else torch.float64
        n = self.ctx.n_pad
        dev = torch.device("cuda", device)
        z = lambda *shape: torch.zeros(shape, dtype=dt, device=dev)   # noqa: E731
        self.b, self.b2, self.b3, self.cb, self.u = (z(n, 4) for _ in range(5))
        self.rho = torch.ones(n, dtype=dt, device=dev)
        self.time = z(2)

    def load(self, b, u=None, rho=None) -> None:
        """The initial state from global host arrays in the reference layout (b, u: N x 4;
        rho: N), scattered to the slab with its ghost planes."""
        import torch
        s = self.slabs
        for dst, src in ((self.b, b), (self.u, u), (self.rho, rho)):
            if src is None:
                continue
            loc = torch.from_numpy(s.scatter(np.asarray(src))).to(dst.dtype)
            dst[: loc.shape[0]].copy_(loc.to(dst.device))
        self.time.zero_()
        torch.cuda.synchronize(self.device)

    def _sync(self) -> None:
        import torch
        self.ctx.synchronize()
        torch.cuda.synchronize(self.device)

    @property
    def args(self):
        if self.nf == 3:
            return [self.b, self.b2, self.b3, self.cb, self.u, self.rho, self.time]
        return [self.b, self.b2, self.cb, self.u, self.rho, self.time]

    @property
    def state(self):
        return [self.b, self.b2, self.b3] if self.nf == 3 else [self.b, self.b2]

    def steps(self, num_steps: int, fused: bool = True) -> None:
        """num_steps steps of the slab.  fused: the context's fused stage kernels, one RK stage
        at a time (ieq_stages_*), the ghost planes of the state fields refreshed after every
        stage; otherwise the reference kernel list with an exchange after every kernel that
        writes the state."""
        if not fused:
            decomposed_steps(self.slabs, self.ctx, self.seq, num_steps, self.state, self.args, self._sync)
            self._sync()
            return
        import torch
        a = self.args
        b3 = a[2] if self.nf == 3 else None
        cb, u, rho, time = (a[3], a[4], a[5], a[6]) if self.nf == 3 else (a[2], a[3], a[4], a[5])
        self._sync()
        ns = self.ctx.stages_begin(a[0], a[1], b3, cb, u)
        try:
            # the exchanges go on the context's stream, behind the stage that wrote the planes
            # and ahead of the next one: no host synchronisation between stages
            with torch.cuda.stream(torch.cuda.ExternalStream(self.ctx.stream, device=self.device)):
                for _ in range(num_steps):
                    for s in range(ns):
                        self.ctx.stages_run(rho, time, s)
                        self.slabs.exchange(*self._stage_planes())
        finally:
            self.ctx.stages_end(a[0], a[1], b3, cb, u, rho)
        self._sync()

    def _stage_planes(self):
        """Zero-copy views of the component planes of the fused state fields (b1, b2[, b3]) as
        they stand; the fused path moves a field between two buffers, so the views are cached
        by buffer."""
        import torch
        cache = self.__dict__.setdefault("_views", {})
        n = self.ctx.n_pad
        size = np.dtype(self.ctx.real).itemsize
        views = []
        for f in range(self.nf):
            base, stride = self.ctx.stages_field(f)
            if base not in cache:
                cache[base] = [torch.as_tensor(_DeviceArray(base + c * stride * size, n, self.ctx.real),
                                               device=torch.device("cuda", self.device)) for c in range(3)]
            views += cache[base]
        return views

    def clean_div(self, max_iterations: int, absolute_error_threshold: float) -> dict:
        """The divergence cleaning of a decomposed box (clean_div_decomposed) on this rank's
        slab, collective over the ranks: ghost planes through torch.distributed, dot products
        of the owned planes all-reduced in FP64."""
        import torch
        if self.slabs.periodic:
            raise ValueError("the decomposed divergence cleaning runs on boxes")
        parts = [(self.slabs, self.ctx, self.b, _cg_fields(self))]
        dev = torch.device("cuda", self.device)

        def total(vals):
            v = float(sum(vals))
            if self.ranks.world == 1:
                return v
            import torch.distributed as dist
            t = torch.tensor([v], dtype=torch.float64, device=dev)
            dist.all_reduce(t)
            return float(t.item())

        def sync():
            self._sync()

        return clean_div_decomposed(parts, max_iterations, absolute_error_threshold, bnodes_of(self.laplace),
                                    total=total, exchange=lambda f: self.slabs.exchange(*f[0]),
                                    scalar=_device_scalar(self), sync=sync)

    def owned(self, field) -> np.ndarray:
        """The owned planes of a field as a host array (rows of the global planes z0..z1)."""
        return field[self.slabs.owned_rows()].cpu().numpy()

    def close(self) -> None:
        self.__dict__.pop("_views", None)   # views of the context's memory
        self.ctx.close()


def run_local(solves: list, num_steps: int, fused: bool = True) -> None:
    """num_steps steps of a decomposition whose ranks' slabs (SlabSolve, ranks 0..P-1 of one
    Ranks world, every slab on the same device) live in one process: every stage (fused) or
    every state-writing kernel of the list runs on each slab in turn, the slabs' devices are
    synchronised, and the ghost planes are copied between the slabs' buffers."""
    import torch
    slabs = [s.slabs for s in solves]

    def sync():
        for s in solves:
            s._sync()

    sync()
    if not fused:
        seq = solves[0].seq
        for _ in range(num_steps):
            for k in seq:
                for s in solves:
                    s.ctx.run(k, s.slabs.local_nodes, *s.args)
                if exchanges_after(k):
                    sync()
                    exchange_local(slabs, [s.state for s in solves])
                    torch.cuda.synchronize(solves[0].device)
        sync()
        return
    parts = []
    for s in solves:
        a = s.args
        b3 = a[2] if s.nf == 3 else None
        cb, u = (a[3], a[4]) if s.nf == 3 else (a[2], a[3])
        parts.append((a, b3, cb, u, a[-2], a[-1]))
    begun = []
    try:
        for s, (a, b3, cb, u, rho, time) in zip(solves, parts):
            ns = s.ctx.stages_begin(a[0], a[1], b3, cb, u)
            begun.append(s)
        for _ in range(num_steps):
            for st in range(ns):
                for s, (a, b3, cb, u, rho, time) in zip(solves, parts):
                    s.ctx.stages_run(rho, time, st)
                sync()
                exchange_local(slabs, [s._stage_planes() for s in solves])
                torch.cuda.synchronize(solves[0].device)
    finally:
        for s, (a, b3, cb, u, rho, time) in zip(begun, parts):
            s.ctx.stages_end(a[0], a[1], b3, cb, u, rho)
        sync()


def clean_div_decomposed(parts, max_iterations: int, absolute_error_threshold: float, bnodes: int,
                         total, exchange, scalar, sync=None) -> dict:
    """clean_div.m:36-79 -- the CG projection of B -- on a decomposed box, as the reference's
    host loop over its kernels, run on every slab held here.

    parts: one (ZSlabs, engine, b, cg) per slab of this process, cg a dict of the slab's
    scalar fields div, phi, lap, r, u (zero on entry); engine.run(name, grange, *args) runs a
    reference kernel on the slab, engine.dot_range(x, y, first, count) a dot product over
    elements [first, first + count).  total(values) adds the slabs' values of all processes
    (the owned planes partition the grid, so every dot product of the reference is the sum of
    the slabs' dots over their owned planes; between processes an FP64 all-reduce, 2 per
    iteration).  exchange(fields) refreshes the ghost planes (fields: one list per slab).
    scalar(engine, value) makes the 1-element array a kernel takes for alpha or beta; sync()
    orders the engines' device work against the exchanges.  Ghost planes: the CG direction u
    once per iteration (the Laplacian reads it across the slab's ends), phi before the
    projection (its gradient) and B after it.  Returns iterations, residual_norm2,
    initial_norm and history (the residual before every iteration)."""
    import math
    sync = sync or (lambda: None)

    def grid_dc(sl):
        return (sl.nx - 2 * bnodes, sl.ny - 2 * bnodes, sl.nloc - 2 * bnodes)

    def dot(x, y):
        vals = []
        for sl, eng, _, cg in parts:
            vals.append(eng.dot_range(cg[x] if isinstance(x, str) else x, cg[y], sl.g_lo * sl.plane,
                                      sl.owned * sl.plane))
        return total(vals)

    for sl, eng, b, cg in parts:
        eng.run("calc_div_divcleaning", grid_dc(sl), b, cg["div"])
    sync()
    for sl, eng, b, cg in parts:
        cg["r"][:] = cg["div"]
    sync()
    residual_norm2 = dot("r", "r")
    old = 1.0
    initial = math.sqrt(residual_norm2)
    tol = absolute_error_threshold * absolute_error_threshold
    it = 0
    history = [residual_norm2]
    while residual_norm2 > tol and it < max_iterations:
        beta = residual_norm2 / old
        for sl, eng, b, cg in parts:
            eng.run("calc_axpy", grid_dc(sl), cg["u"], cg["r"], scalar(eng, beta))
        sync()
        exchange([[cg["u"]] for _, _, _, cg in parts])
        sync()
        for sl, eng, b, cg in parts:
            eng.run("calc_laplace_divcleaning", grid_dc(sl), cg["u"], cg["lap"])
        sync()
        alpha = residual_norm2 / dot("u", "lap")
        for sl, eng, b, cg in parts:
            eng.run("calc_xpay", grid_dc(sl), cg["phi"], cg["u"], scalar(eng, alpha))
            eng.run("calc_xpay", grid_dc(sl), cg["r"], cg["lap"], scalar(eng, -alpha))
        sync()
        old = residual_norm2
        residual_norm2 = dot("r", "r")
        history.append(residual_norm2)
        it += 1
    exchange([[cg["phi"]] for _, _, _, cg in parts])
    sync()
    for sl, eng, b, cg in parts:
        eng.run("projector_divcleaning", sl.local_nodes, b, cg["phi"])
    sync()
    exchange([[b] for _, _, b, _ in parts])
    sync()
    return {"iterations": it, "residual_norm2": residual_norm2, "initial_norm": initial, "history": history}


def _cg_fields(solve) -> dict:
    import torch
    dt = torch.float32 if solve.ctx.real == np.float32 else torch.float64
    dev = torch.device("cuda", solve.device)
    return {k: torch.zeros(solve.ctx.n_pad, dtype=dt, device=dev) for k in ("div", "phi", "lap", "r", "u")}


def _device_scalar(solve):
    import torch
    dt = torch.float32 if solve.ctx.real == np.float32 else torch.float64

    def make(_eng, v):
        return torch.tensor([v], dtype=dt, device=torch.device("cuda", solve.device))
    return make


def clean_div_local(solves: list, max_iterations: int, absolute_error_threshold: float) -> dict:
    """The decomposed divergence cleaning of the slabs of several ranks held in one process on
    one device (SlabSolve, ranks 0..P-1 of one box decomposition): the slabs' dot products
    added in rank order, ghost planes copied between their buffers."""
    import torch
    s0 = solves[0]
    if s0.slabs.periodic:
        raise ValueError("the decomposed divergence cleaning runs on boxes")
    parts = [(s.slabs, s.ctx, s.b, _cg_fields(s)) for s in solves]

    def sync():
        for s in solves:
            s._sync()
        torch.cuda.synchronize(s0.device)

    return clean_div_decomposed(parts, max_iterations, absolute_error_threshold, bnodes_of(s0.laplace),
                                total=lambda v: float(sum(v)),
                                exchange=lambda f: exchange_local([p[0] for p in parts], f),
                                scalar=_device_scalar(s0), sync=sync)
