"""Domain decomposition of one periodic solve into z slabs, one slab per rank (one process
per GPU).

The reference runs one grid on one device (matlab/+induction_eq/initialize.m:31-34); its
paper sweeps go to 320^3 and beyond (paper/convergence_rotation_3D.m:104).  Here rank k of
P owns the contiguous planes [z0_k, z1_k) of the global grid -- in the reference layout,
idx = ix + NX*(iy + NY*iz), a z slab is one contiguous block of memory -- and holds G ghost
planes on each side, G = 2 * (ORDER/2): the Hall term reaches ORDER/2 planes for curl(B)/rho
and ORDER/2 more for the flux rows of E = J x B, the volume, dissipation and convection terms
reach ORDER/2.  The rank's context is the global settings with NODES_Z = (z1_k - z0_k) + 2G,
the global spacing, the grid periodic, and the slab's z offset, so that testcase coordinates
(init, u_analytical, analytical_b) are those of the global grid.

A step runs the integrator on the local slab either through the context's fused stage kernels,
one RK stage at a time (ieq_stages_*: the ghost planes of the state fields are refreshed after
every stage), or as the reference's kernel list (compute_numerical_solution_setup.m:140-371).
After every stage -- every kernel of the list that writes a state field (all but
calc_curlB_rho_*, calc_u_* and calc_time_*) -- the state fields' ghost planes are refreshed from
the neighbours' owned planes: the G planes at the bottom of the owned range go to the rank
below, the G at the top to the rank above, periodically (rank 0's lower neighbour is rank
P-1) -- one point-to-point exchange per neighbour and field (NCCL between GPUs, gloo on CPU).
curl(B)/rho is recomputed on every local plane from fresh ghosts, so it is never exchanged;
its values within ORDER/2 of the slab's ends are not valid and are never read by an owned
node.  Each owned node then performs exactly the arithmetic of the undecomposed run, so the
decomposed fields equal it bit for bit.

Non-periodic boxes are not decomposed here: their slabs would need SBP boundary rows in x and
y but interior rows in z, a combination the stencil kernels do not instantiate.
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
    """One rank's view of the decomposition of a periodic (nx, ny, nz) grid."""
    ranks: Ranks
    nx: int
    ny: int
    nz: int
    ghosts: int

    def __post_init__(self):
        w = self.ranks.world
        self.bounds = slab_bounds(self.nz, w)
        self.z0, self.z1 = self.bounds[self.ranks.rank]
        if min(b - a for a, b in self.bounds) < self.ghosts:
            raise ValueError(f"every rank must own at least {self.ghosts} planes (the ghost depth): "
                             f"{self.nz} planes over {w} ranks")
        self.up = (self.ranks.rank + 1) % w
        self.down = (self.ranks.rank - 1) % w

    @property
    def owned(self) -> int:
        return self.z1 - self.z0

    @property
    def nloc(self) -> int:
        return self.owned + 2 * self.ghosts

    @property
    def plane(self) -> int:
        return self.nx * self.ny

    @property
    def local_nodes(self) -> tuple[int, int, int]:
        return (self.nx, self.ny, self.nloc)

    @property
    def z_offset(self) -> int:
        """Global plane of local plane 0."""
        return self.z0 - self.ghosts

    def scatter(self, glob: np.ndarray) -> np.ndarray:
        """The local slab (ghosts included) of a global field in the reference layout
        ((N,) or (N, C) rows, N = nx*ny*nz), periodic in z."""
        g = glob[: self.nz * self.plane].reshape((self.nz, self.plane) + glob.shape[1:])
        zs = np.arange(self.z_offset, self.z_offset + self.nloc) % self.nz
        return np.ascontiguousarray(g[zs].reshape((self.nloc * self.plane,) + glob.shape[1:]))

    def owned_rows(self) -> slice:
        """Rows of the owned planes in a local field."""
        return slice(self.ghosts * self.plane, (self.ghosts + self.owned) * self.plane)

    def global_rows(self) -> slice:
        """Rows of the owned planes in the global field."""
        return slice(self.z0 * self.plane, self.z1 * self.plane)

    def exchange(self, *fields) -> None:
        """Refresh the ghost planes of every field (torch tensors or numpy arrays over the
        local slab, rows in the reference layout; padded rows beyond the slab are ignored)
        from the neighbours' owned planes."""
        import torch
        G, P, n = self.ghosts, self.plane, self.owned
        for f in fields:
            t = torch.from_numpy(f) if isinstance(f, np.ndarray) else f
            lo_ghost = t[0: G * P]
            lo_owned = t[G * P: 2 * G * P]
            hi_owned = t[n * P: (n + G) * P]
            hi_ghost = t[(n + G) * P: (n + 2 * G) * P]
            if self.ranks.world == 1:
                lo_ghost.copy_(hi_owned)
                hi_ghost.copy_(lo_owned)
                continue
            import torch.distributed as dist
            send_lo, send_hi = lo_owned.contiguous(), hi_owned.contiguous()
            recv_hi, recv_lo = torch.empty_like(hi_ghost), torch.empty_like(lo_ghost)
            # posted in this order on every rank: with two ranks (up == down) the first
            # message between a pair is the sender's bottom block, the receiver's top ghosts
            ops = [dist.P2POp(dist.isend, send_lo, self.down), dist.P2POp(dist.isend, send_hi, self.up),
                   dist.P2POp(dist.irecv, recv_hi, self.up), dist.P2POp(dist.irecv, recv_lo, self.down)]
            for req in dist.batch_isend_irecv(ops):
                req.wait()
            hi_ghost.copy_(recv_hi)
            lo_ghost.copy_(recv_lo)


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


def local_maps(maps, slabs: ZSlabs):
    """The settings of one rank's slab: the global maps with NODES_Z = the slab's planes
    including ghosts, the global spacing and the slab's z offset (periodic grids only)."""
    import copy
    if maps.I_RunOps.get("periodic") != "USE_PERIODIC":
        raise ValueError("the z-slab decomposition needs a periodic grid")
    m = copy.deepcopy(maps)
    m.spacing_override = maps.spacing()
    m.I_Mesh["NODES_Z"] = slabs.nloc
    m.I_Tech["z_offset"] = slabs.z_offset
    m.I_Tech["nz_global"] = slabs.nz
    return m


def ghost_depth(order: int) -> int:
    """Ghost planes a slab needs for one stage: ORDER/2 for curl(B)/rho and ORDER/2 for the
    flux rows of E (the interior rows of a periodic grid)."""
    return 2 * (order // 2)


TWO_FIELD_INTEGRATORS = ("CarpenterKennedy2N54", "ToulorgeDesmet2N84F")


class _DeviceArray:
    """A 1-D device array by address (the CUDA array interface), for torch.as_tensor."""

    def __init__(self, ptr: int, n: int, dtype):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": np.dtype(dtype).str,
                                         "data": (int(ptr), False), "version": 3}


class SlabSolve:
    """One rank's slab of a decomposed periodic solve on its GPU: the local context (the C
    ABI's reference kernels, ieq_run_kernels) on torch device buffers, the ghost exchanges
    through torch.distributed (NCCL between GPUs; a local copy with one rank)."""

    def __init__(self, maps, ranks: Ranks, device: int = 0):
        import torch
        m = maps.I_Mesh
        self.ranks = ranks
        self.slabs = ZSlabs(ranks, int(m["NODES_X"]), int(m["NODES_Y"]), int(m["NODES_Z"]),
                            ghost_depth(int(maps.I_RunOps["order"])))
        self.device = device
        self.ctx = local_maps(maps, self.slabs).context(device)
        self.seq = self.ctx.step_kernels()
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

    def owned(self, field) -> np.ndarray:
        """The owned planes of a field as a host array (rows of the global planes z0..z1)."""
        return field[self.slabs.owned_rows()].cpu().numpy()

    def close(self) -> None:
        self.__dict__.pop("_views", None)   # views of the context's memory
        self.ctx.close()
