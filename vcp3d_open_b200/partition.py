"""A block split into k slabs, one slab per GPU.

The reference distributes a block over MPI ranks in Cartesian element blocks
(SolverClass::DistributeGrid, src/SolverClass.cpp:1537-1584) and exchanges the
neighbouring ranks' data inside Residual, overlapped with the volume work
(src/SolverClass.cpp:3428-3611). Here a rank owns a slab of whole k layers (a
contiguous range of element indices, i fastest) and holds two ghost layers
after its owned elements: the layer above the slab, whose k-Min faces towards
the slab this rank evaluates, and the layer below, which only provides its
state to the slab's own k-Min faces. Every face is still evaluated once per
rank that needs it from the same inputs, so a partitioned residual equals the
single-GPU one bit for bit.

Blocks may be periodic in k or not (then the first and the last slab hold the
k-Min and k-Max boundary faces and exchange on one side only) and may have open
boundaries on any face: each rank sets up the whole block's boundaries on the
host and keeps its own elements' part (block-wide boundary areas and sponge
extents), and before each residual the ranks' per-face Mach weights are
gathered and summed in block element order, which is what one GPU sums.

A step is: the local CFL time step, its minimum over ranks, then per stage the
stage update and the residual. The residual starts the exchange of the two
owned boundary layers into the neighbours' ghost layers, computes what needs
no ghost state (boundary kernels, the face fluxes and residuals of the slab's
inner layers) while the exchange runs, and completes the first and last
layers after it. The transport is torch.distributed (NCCL between GPUs on a
stream of its own; gloo for host tests) or, for one process driving all slabs
on one GPU, device-to-device copies.
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
    periodic_k: bool = True

    @property
    def has_down(self) -> bool:
        """A slab (or the periodic wrap) lies below: the lower ghost layer is live."""
        return self.periodic_k or self.k0 > 0

    @property
    def has_up(self) -> bool:
        return self.periodic_k or self.k1 < self.n_elem[2]

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


def slabs(n_elem: Sequence[int], world: int, periodic_k: bool = True) -> List[Slab]:
    """k layers split as evenly as possible; every rank owns at least one layer."""
    nk = int(n_elem[2])
    if world < 1 or world > nk:
        raise ValueError(f"{world} ranks for {nk} k layers")
    base, extra = divmod(nk, world)
    out, k = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append(Slab(tuple(int(v) for v in n_elem), r, world, k, k + n, bool(periodic_k)))
        k += n
    return out


def local_neighbors(slab: Slab, global_nbr: np.ndarray) -> np.ndarray:
    """Neighbour table of the slab's local elements (-1: a face this rank does
    not evaluate, or a physical boundary face of the block). global_nbr: the
    block's [nE][6] table (-1 on boundary faces)."""
    L, nO = slab.layer, slab.n_owned
    out = np.full((slab.n_local, 6), -1, dtype=np.int32)
    g = np.arange(slab.k0 * L, slab.k1 * L)
    kl = np.arange(nO) // L
    q = np.arange(nO) % L
    base = slab.k0 * L
    for f in range(4):   # i and j neighbours lie in the same layer
        nb = global_nbr[g, f]
        out[:nO, f] = np.where(nb >= 0, nb - base, -1)
    kmin, kmax = global_nbr[g, 4], global_nbr[g, 5]
    if np.any((kmin < 0) != (kmax < 0)) and slab.periodic_k:
        raise ValueError("a block periodic in k has no k boundary faces")
    if not slab.periodic_k and (np.any((kmin < 0) & (kl + slab.k0 > 0)) or
                                np.any((kmax < 0) & (kl + slab.k0 < slab.n_elem[2] - 1))):
        raise ValueError("k boundary faces inside the block")
    out[:nO, 4] = np.where(kl == 0, np.where(kmin >= 0, slab.lower_ghost + q, -1),
                           np.arange(nO) - L)
    out[:nO, 5] = np.where(kl == slab.n_layers - 1,
                           np.where(kmax >= 0, slab.upper_ghost + q, -1), np.arange(nO) + L)
    # The ghost layer above: only its k-Min face (towards the slab's top layer).
    if slab.has_up:
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

    def __init__(self, slab: Slab, params: capi.Params, disc, modal: Optional[np.ndarray] = None,
                 case=None):
        from .solver import Solver
        import torch
        self.slab = slab
        self.solver = Solver(local_params(params, slab), local_discretization(disc, slab))
        self.solver.set_partition(slab.n_owned, slab.layer)
        self.kd5 = 5 * (params.n_poly + 1) ** 3
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.open = case is not None and case.spec.is_open
        if self.open:
            self._set_open_boundary(case, disc)
        if modal is not None:
            self.set_global_state(modal)

    def _set_open_boundary(self, case, disc):
        """The whole block's open boundaries, restricted to this slab's elements."""
        import ctypes as C
        from . import solver as sv
        ob = sv.open_boundary(case)
        sfs = sv.subfaces(case)
        keep = [np.ascontiguousarray(a) for a in (disc.vol_metric, disc.face_metric,
                                                  disc.elem_scalars)]
        nbr = np.ascontiguousarray(disc.neighbors, dtype=np.int32)
        geom = capi.Geometry(capi.ptr(keep[0]), capi.ptr(keep[1]), capi.ptr(keep[2]),
                             capi.ptr(nbr))
        nodes = np.ascontiguousarray(case.elem_nodes, dtype=np.float64)
        l2g = np.ascontiguousarray(self.slab.local_to_global(), dtype=np.int64)
        n_elem = np.ascontiguousarray(self.slab.n_elem, dtype=np.int32)
        lib = self.solver.lib
        rc = lib.vcpg_set_open_boundary_partition(
            self.solver.h, C.byref(ob), sfs, len(sfs) if sfs is not None else 0,
            capi.ptr(n_elem), C.byref(geom), case.spec.p_grid, disc.dof_location,
            capi.ptr(nodes), l2g.ctypes.data_as(C.POINTER(C.c_int64)))
        self.solver._check(rc, "set_open_boundary_partition")

    def mach_weights(self):
        """(weights per block face: list of 6 arrays) of this slab's boundary faces."""
        import ctypes as C
        counts = np.zeros(6, dtype=np.int32)
        lib = self.solver.lib
        self.solver._check(lib.vcpg_boundary_mach_weights(self.solver.h, None, capi.ptr(counts)),
                           "boundary_mach_weights")
        w = np.zeros(max(int(counts.sum()), 1))
        self.solver._check(lib.vcpg_boundary_mach_weights(self.solver.h, capi.ptr(w),
                                                          capi.ptr(counts)),
                           "boundary_mach_weights")
        out, o = [], 0
        for c in counts:
            out.append(w[o:o + int(c)].copy())
            o += int(c)
        return out

    def set_mach_sums(self, sums):
        a = np.ascontiguousarray(sums, dtype=np.float64)
        self.solver._check(self.solver.lib.vcpg_set_boundary_mach_sums(self.solver.h,
                                                                        capi.ptr(a)),
                           "set_boundary_mach_sums")

    def residual_part(self, part: int):
        self.solver._check(self.solver.lib.vcpg_residual_part(self.solver.h, part),
                           "residual_part")

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
    the handles through device buffers; reductions and gathers on the host."""

    def __init__(self, shards: Sequence[Shard]):
        self.shards = list(shards)
        L = self.shards[0].slab.layer
        self.top = [s.new_buffer(L) for s in self.shards]
        self.bottom = [s.new_buffer(L) for s in self.shards]

    def start_exchange(self):
        """Copies every slab's two owned boundary layers out (the ghost layers
        are written by finish_exchange)."""
        for r, s in enumerate(self.shards):
            L = s.slab.layer
            s.pack(s.slab.n_owned - L, L, self.top[r])
            s.pack(0, L, self.bottom[r])

    def finish_exchange(self):
        W = len(self.shards)
        for s in self.shards:
            s.sync()
        for r, s in enumerate(self.shards):
            L = s.slab.layer
            if s.slab.has_down:
                s.unpack(s.slab.lower_ghost, L, self.top[(r - 1) % W])
            if s.slab.has_up:
                s.unpack(s.slab.upper_ghost, L, self.bottom[(r + 1) % W])
        for s in self.shards:
            s.sync()

    def exchange(self):
        self.start_exchange()
        self.finish_exchange()

    def reduce(self, values, op: str):
        return min(values) if op == "min" else max(values)

    def gather(self, items):
        """Every rank's item in rank order (here: the shards' items)."""
        return list(items)


class DistTransport:
    """One slab per process over torch.distributed (NCCL between GPUs, gloo on
    the host): the top owned layer goes to the rank above (its lower ghost), the
    bottom one to the rank below (its upper ghost); a block that is not periodic
    in k has no exchange below its first slab or above its last. Point-to-point
    operations of a pair match in issue order, so two ranks that are each
    other's upper and lower neighbour still pair the right layers. With CUDA
    tensors the transfers run on a stream of their own, ordered after the packing
    on the library's stream, which in turn waits for them before unpacking; the
    work issued between start_exchange and finish_exchange overlaps them."""

    def __init__(self, shard, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.shards = [shard]
        L = shard.slab.layer
        self.send_top, self.send_bottom = shard.new_buffer(L), shard.new_buffer(L)
        self.recv_lower, self.recv_upper = shard.new_buffer(L), shard.new_buffer(L)
        self.comm = None
        self.works = []
        if self.send_top.is_cuda:
            import torch
            self.comm = torch.cuda.Stream(device=self.send_top.device)

    def _lib_stream(self):
        import torch
        return torch.cuda.ExternalStream(self.shards[0].solver.stream,
                                         device=self.send_top.device)

    def start_exchange(self):
        s = self.shards[0]
        sl, L, dist = s.slab, s.slab.layer, self.dist
        s.pack(sl.n_owned - L, L, self.send_top)
        s.pack(0, L, self.send_bottom)
        self.works = []
        if sl.world == 1:   # the block's own periodic wrap, or nothing to exchange
            return
        ops = []
        if sl.has_up:
            ops.append(dist.P2POp(dist.isend, self.send_top, sl.up, self.group))
        if sl.has_down:
            ops.append(dist.P2POp(dist.isend, self.send_bottom, sl.down, self.group))
            ops.append(dist.P2POp(dist.irecv, self.recv_lower, sl.down, self.group))
        if sl.has_up:
            ops.append(dist.P2POp(dist.irecv, self.recv_upper, sl.up, self.group))
        if not ops:
            return
        if self.comm is not None:
            import torch
            self.comm.wait_stream(self._lib_stream())
            with torch.cuda.stream(self.comm):
                self.works = dist.batch_isend_irecv(ops)
        else:
            s.sync()
            self.works = dist.batch_isend_irecv(ops)

    def finish_exchange(self):
        s = self.shards[0]
        sl, L = s.slab, s.slab.layer
        if sl.world == 1:
            if sl.periodic_k:
                s.unpack(sl.lower_ghost, L, self.send_top)
                s.unpack(sl.upper_ghost, L, self.send_bottom)
            s.sync()
            return
        if self.comm is not None:
            import torch
            with torch.cuda.stream(self.comm):
                for w in self.works:
                    w.wait()
            self._lib_stream().wait_stream(self.comm)
        else:
            for w in self.works:
                w.wait()
        self.works = []
        if sl.has_down:
            s.unpack(sl.lower_ghost, L, self.recv_lower)
        if sl.has_up:
            s.unpack(sl.upper_ghost, L, self.recv_upper)
        s.sync()

    def exchange(self):
        self.start_exchange()
        self.finish_exchange()

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

    def gather(self, items):
        """Every rank's item in rank order (this process contributes items[0])."""
        out = [None] * self.shards[0].slab.world
        self.dist.all_gather_object(out, items[0], group=self.group)
        return out


def block_mach_sums(weights_per_rank) -> np.ndarray:
    """Per block face, the sum of the Mach weights of all slabs in block element
    order: the slabs' lists in rank order (increasing k), each in its own
    element order, summed one after the other as one GPU sums its list."""
    sums = np.zeros(6)
    for f in range(6):
        m = 0.0
        for w in weights_per_rank:
            for x in w[f]:
                m += float(x)
        sums[f] = m
    return sums


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

    def _mach_sums(self):
        """Block-wide Mach sums of open blocks, handed to every shard."""
        if not any(s.open for s in self.shards):
            return
        sums = block_mach_sums(self.t.gather([s.mach_weights() for s in self.shards]))
        for s in self.shards:
            s.set_mach_sums(sums)

    def residual(self, monitoring: bool = False):
        if monitoring:
            self.t.exchange()
            self._mach_sums()
            mons = [s.solver.residual(monitoring=True) for s in self.shards]
            self.res_valid = True
            mon = np.zeros(8)
            mon[6] = self.t.reduce([m[6] for m in mons], "max")
            mon[7] = self.t.reduce([m[7] for m in mons], "max")
            return mon
        # The exchange overlaps what needs no ghost state.
        self.t.start_exchange()
        self._mach_sums()
        for s in self.shards:
            s.residual_part(0)
        self.t.finish_exchange()
        for s in self.shards:
            s.residual_part(1)
        self.res_valid = True
        return None

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
