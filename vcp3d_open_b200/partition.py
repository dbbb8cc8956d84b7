"""A periodic block split into k slabs, one slab per GPU.

The reference distributes a block over MPI ranks in Cartesian element blocks
(SolverClass::DistributeGrid, src/SolverClass.cpp:1537-1584) and exchanges the
neighbouring ranks' data inside Residual. Here a rank owns a slab of whole
k layers (a contiguous range of element indices, i fastest) and holds two ghost
layers after its owned elements: the layer above the slab, whose k-Min faces
towards the slab this rank evaluates, and the layer below, which only provides
its state to the slab's own k-Min faces. Every face is still evaluated once per
rank that needs it from the same inputs, so a partitioned residual equals the
single-GPU one bit for bit.

A step is: the local CFL time step, its minimum over ranks, then per stage the
stage update, the exchange of the two owned boundary layers into the
neighbours' ghost layers, and the residual. The transport is
torch.distributed (NCCL between GPUs; gloo for host tests) or, for one process
driving all slabs on one GPU, device-to-device copies.
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional, Sequence

import numpy as np

from . import capi


@dataclasses.dataclass
class Slab:
    """Rank `rank` of `world` owns global k layers [k0, k1) of an (ni, nj, nk) block."""
    n_elem: tuple
    rank: int
    world: int
    k0: int
    k1: int

    @property
    def layer(self) -> int:
        return self.n_elem[0] * self.n_elem[1]

    @property
    def n_layers(self) -> int:
        return self.k1 - self.k0

    @property
    def n_owned(self) -> int:
        return self.n_layers * self.layer

    @property
    def n_local(self) -> int:
        return self.n_owned + 2 * self.layer

    @property
    def upper_ghost(self) -> int:
        """First local index of the ghost layer above the slab (global layer k1)."""
        return self.n_owned

    @property
    def lower_ghost(self) -> int:
        """First local index of the ghost layer below the slab (global layer k0 - 1)."""
        return self.n_owned + self.layer

    @property
    def up(self) -> int:
        return (self.rank + 1) % self.world

    @property
    def down(self) -> int:
        return (self.rank - 1) % self.world

    def local_to_global(self) -> np.ndarray:
        nk, L = self.n_elem[2], self.layer
        owned = np.arange(self.k0 * L, self.k1 * L)
        above = (self.k1 % nk) * L + np.arange(L)
        below = ((self.k0 - 1) % nk) * L + np.arange(L)
        return np.concatenate([owned, above, below])


def slabs(n_elem: Sequence[int], world: int) -> List[Slab]:
    """k layers split as evenly as possible; every rank owns at least one layer."""
    nk = int(n_elem[2])
    if world < 1 or world > nk:
        raise ValueError(f"{world} ranks for {nk} k layers")
    base, extra = divmod(nk, world)
    out, k = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append(Slab(tuple(int(v) for v in n_elem), r, world, k, k + n))
        k += n
    return out


def local_neighbors(slab: Slab, global_nbr: np.ndarray) -> np.ndarray:
    """Neighbour table of the slab's local elements (-1: a face this rank does
    not evaluate). global_nbr: the block's [nE][6] table (periodic wrap)."""
    L, nO = slab.layer, slab.n_owned
    out = np.full((slab.n_local, 6), -1, dtype=np.int32)
    g = np.arange(slab.k0 * L, slab.k1 * L)
    kl = np.arange(nO) // L
    q = np.arange(nO) % L
    base = slab.k0 * L
    for f in range(4):   # i and j neighbours lie in the same layer
        nb = global_nbr[g, f]
        if np.any(nb < 0):
            raise ValueError("partitioned blocks must be periodic in i and j")
        out[:nO, f] = nb - base
    if np.any(global_nbr[g, 4] < 0) or np.any(global_nbr[g, 5] < 0):
        raise ValueError("partitioned blocks must be periodic in k")
    out[:nO, 4] = np.where(kl == 0, slab.lower_ghost + q, np.arange(nO) - L)
    out[:nO, 5] = np.where(kl == slab.n_layers - 1, slab.upper_ghost + q, np.arange(nO) + L)
    # The ghost layer above: only its k-Min face (towards the slab's top layer).
    out[slab.upper_ghost:slab.upper_ghost + L, 4] = nO - L + np.arange(L)
    return out


def local_discretization(disc, slab: Slab):
    """The slab's Discretization: per-element arrays gathered in local order,
    neighbours remapped; operators shared."""
    idx = slab.local_to_global()
    return dataclasses.replace(
        disc, n_elem=(slab.n_elem[0], slab.n_elem[1], slab.n_layers + 2),
        vol_metric=np.ascontiguousarray(disc.vol_metric[idx]),
        face_metric=np.ascontiguousarray(disc.face_metric[idx]),
        elem_scalars=np.ascontiguousarray(disc.elem_scalars[idx]),
        neighbors=local_neighbors(slab, np.asarray(disc.neighbors)),
        vol_metric_dofs=(None if disc.vol_metric_dofs is None
                         else np.ascontiguousarray(disc.vol_metric_dofs[idx])))


def local_params(params: capi.Params, slab: Slab) -> capi.Params:
    """The block's parameters with the slab's element count (owned + 2 ghost layers)."""
    p = capi.Params.from_buffer_copy(params)
    p.n_elem[:] = [slab.n_elem[0], slab.n_elem[1], slab.n_layers + 2]
    return p


# ---------------------------------------------------------------------------
# Shards and transports
# ---------------------------------------------------------------------------

class Shard:
    """One slab on the current CUDA device: a library handle holding the owned
    elements and both ghost layers."""

    def __init__(self, slab: Slab, params: capi.Params, disc, modal: Optional[np.ndarray] = None):
        from .solver import Solver
        import torch
        self.slab = slab
        self.solver = Solver(local_params(params, slab), local_discretization(disc, slab))
        self.solver.set_partition(slab.n_owned, slab.layer)
        self.kd5 = 5 * (params.n_poly + 1) ** 3
        self.device = torch.device("cuda", torch.cuda.current_device())
        if modal is not None:
            self.set_global_state(modal)

    def set_global_state(self, modal: np.ndarray):
        """Owned and ghost states taken from the block's modal state."""
        a = np.asarray(modal).reshape(-1, self.kd5)
        self.solver.set_state(a[self.slab.local_to_global()])

    def owned_state(self) -> np.ndarray:
        return self.solver.get_state()[:self.slab.n_owned]

    def new_buffer(self, count: int):
        import torch
        return torch.empty(count * self.kd5, dtype=torch.float64, device=self.device)

    def pack(self, first: int, count: int, buf):
        self.solver.pack_states(first, count, buf.data_ptr())

    def unpack(self, first: int, count: int, buf):
        self.solver.unpack_states(first, count, buf.data_ptr())

    def sync(self):
        self.solver.sync()


class LocalTransport:
    """All slabs driven by one process (one GPU): ghost layers copied between
    the handles through device buffers; reductions on the host."""

    def __init__(self, shards: Sequence[Shard]):
        self.shards = list(shards)
        L = self.shards[0].slab.layer
        self.top = [s.new_buffer(L) for s in self.shards]
        self.bottom = [s.new_buffer(L) for s in self.shards]

    def exchange(self):
        W = len(self.shards)
        for r, s in enumerate(self.shards):
            L = s.slab.layer
            s.pack(s.slab.n_owned - L, L, self.top[r])
            s.pack(0, L, self.bottom[r])
        for s in self.shards:
            s.sync()
        for r, s in enumerate(self.shards):
            L = s.slab.layer
            s.unpack(s.slab.lower_ghost, L, self.top[(r - 1) % W])
            s.unpack(s.slab.upper_ghost, L, self.bottom[(r + 1) % W])
        for s in self.shards:
            s.sync()

    def reduce(self, values, op: str):
        return min(values) if op == "min" else max(values)


class DistTransport:
    """One slab per process over torch.distributed (NCCL between GPUs, gloo on
    the host): the top owned layer goes to the rank above (its lower ghost), the
    bottom one to the rank below (its upper ghost). Point-to-point operations of
    a pair match in issue order, so two ranks that are each other's upper and
    lower neighbour still pair the right layers."""

    def __init__(self, shard, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.shards = [shard]
        L = shard.slab.layer
        self.send_top, self.send_bottom = shard.new_buffer(L), shard.new_buffer(L)
        self.recv_lower, self.recv_upper = shard.new_buffer(L), shard.new_buffer(L)

    def exchange(self):
        s = self.shards[0]
        sl, L, dist = s.slab, s.slab.layer, self.dist
        s.pack(sl.n_owned - L, L, self.send_top)
        s.pack(0, L, self.send_bottom)
        s.sync()
        if sl.world == 1:   # the block's own periodic wrap
            s.unpack(sl.lower_ghost, L, self.send_top)
            s.unpack(sl.upper_ghost, L, self.send_bottom)
            s.sync()
            return
        ops = [dist.P2POp(dist.isend, self.send_top, sl.up, self.group),
               dist.P2POp(dist.isend, self.send_bottom, sl.down, self.group),
               dist.P2POp(dist.irecv, self.recv_lower, sl.down, self.group),
               dist.P2POp(dist.irecv, self.recv_upper, sl.up, self.group)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        if self.recv_lower.is_cuda:
            import torch
            torch.cuda.current_stream().synchronize()
        s.unpack(sl.lower_ghost, L, self.recv_lower)
        s.unpack(sl.upper_ghost, L, self.recv_upper)
        s.sync()

    def reduce(self, values, op: str):
        import torch
        dist = self.dist
        dev = self.send_top.device
        t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=dev)
        t = t.min() if op == "min" else t.max()
        t = t.reshape(1)
        dist.all_reduce(t, op=dist.ReduceOp.MIN if op == "min" else dist.ReduceOp.MAX,
                        group=self.group)
        return float(t.item())


class ShardedSolver:
    """Residual, time step and Runge-Kutta steps of a partitioned block over the
    shards this process drives (all of them with LocalTransport, its own with
    DistTransport)."""

    def __init__(self, transport):
        self.t = transport
        self.res_valid = False

    @property
    def shards(self):
        return self.t.shards

    def residual(self, monitoring: bool = False):
        self.t.exchange()
        mons = [s.solver.residual(monitoring=monitoring) for s in self.shards]
        self.res_valid = True
        if not monitoring:
            return None
        mon = np.zeros(8)
        mon[6] = self.t.reduce([m[6] for m in mons], "max")
        mon[7] = self.t.reduce([m[7] for m in mons], "max")
        return mon

    def time_step(self) -> float:
        return self.t.reduce([s.solver.time_step() for s in self.shards], "min")

    def step(self, n_steps: int, scheme: int = capi.SSPRK3,
             fixed_dt: float = -1.0) -> np.ndarray:
        if not self.res_valid:
            self.residual()
        stages = 3 if scheme == capi.SSPRK3 else 5
        hist = []
        for _ in range(n_steps):
            dt = fixed_dt if fixed_dt > 0.0 else self.time_step()
            hist.append(dt)
            for st in range(stages):
                for s in self.shards:
                    s.solver.rk_stage(scheme, st, dt)
                self.residual()
        return np.array(hist)
