"""A block split into Cartesian parts, one part per GPU.

The reference distributes a block over MPI ranks in Cartesian element blocks
(SolverClass::DistributeGrid, src/SolverClass.cpp:1537-1584) and exchanges the
neighbouring ranks' data inside Residual, overlapped with the volume work
(src/SolverClass.cpp:3428-3611). Here rank r of a (pi, pj, pk) grid of ranks
(i fastest, as there) owns the elements [lo, hi) per direction of the block;
rank_grid picks the grid as DistributeGrid does. A direction with one rank
keeps its periodic wrap inside the part; across a split direction the handle
holds ghost copies of the neighbouring parts' elements:

* face ghosts: per split direction the plane of elements just above the part,
  whose Min face towards the part this rank evaluates;
* lower ghosts: per split direction the plane just below the part, which only
  provide their states to the part's own Min faces.

Every face is still evaluated once per rank that needs it from the same inputs,
so a partitioned residual equals the single-GPU one bit for bit. The handle's
owned elements come first, ordered as: no ghost neighbour (A), a face ghost
above but no lower ghost (B), a lower ghost (C); then the face ghosts, then the
lower ghosts. A residual computes the face fluxes of A and B and the residuals
of A while the ghost states travel, and the rest after they arrive.

Blocks may be periodic in a direction or not (then the first and the last part
in that direction hold the block's boundary faces and exchange on one side
only) and may have open boundaries on any face: each rank sets up the whole
block's boundaries on the host and keeps its own elements' part (block-wide
boundary areas and sponge extents), and before each residual the ranks'
per-face Mach weights are gathered and summed in block element order, which is
what one GPU sums.

A step is: the local CFL time step, its minimum over ranks, then per stage the
stage update and the residual. The transport is torch.distributed (NCCL
between GPUs on a stream of its own; gloo for host tests) or, for one process
driving all parts on one GPU, device-to-device copies.
"""
from __future__ import annotations

import dataclasses
import functools
from typing import List, Optional, Sequence

import numpy as np

from . import capi


def rank_grid(n_elem: Sequence[int], world: int,
              allow: Sequence[bool] = (True, True, True)) -> tuple:
    """Ranks per direction for `world` ranks, as DistributeGrid chooses them
    (src/SolverClass.cpp:1537-1584): starting from one rank per direction, the
    ranks of one direction double at a time, in the direction whose elements per
    rank halve evenly and are the most (ties go to j over i and to k over j and
    i), splits being allowed per direction ("Allow block splitting in
    i-direction" ...). ValueError when the ranks cannot split the block evenly."""
    ranks = [1, 1, 1]
    per = [int(n) for n in n_elem]
    while ranks[0] * ranks[1] * ranks[2] != world:
        if ranks[0] * ranks[1] * ranks[2] > world:
            raise ValueError(f"{world} ranks cannot split the block evenly")
        half = [per[d] // 2 if per[d] % 2 == 0 and allow[d] else -1 for d in range(3)]
        if half == [-1, -1, -1]:
            raise ValueError(f"{world} ranks cannot split a {tuple(n_elem)} block evenly")
        if half[0] > half[1] and half[0] > half[2]:
            d = 0
        elif half[1] > half[2]:
            d = 1
        else:
            d = 2
        per[d] //= 2
        ranks[d] *= 2
    return tuple(ranks)


def _bounds(n: int, parts: int) -> List[int]:
    """Cuts of n elements into parts as even as possible (the first parts one larger)."""
    base, extra = divmod(n, parts)
    cuts, c = [0], 0
    for r in range(parts):
        c += base + (1 if r < extra else 0)
        cuts.append(c)
    return cuts


@dataclasses.dataclass(eq=False)
class Part:
    """Rank `rank` of a `grid` of ranks owns elements [lo, hi) per direction of
    an n_elem block; periodic: per direction, whether the block wraps there."""
    n_elem: tuple
    grid: tuple
    rank: int
    lo: tuple
    hi: tuple
    periodic: tuple = (True, True, True)

    @property
    def world(self) -> int:
        return self.grid[0] * self.grid[1] * self.grid[2]

    @property
    def coords(self) -> tuple:
        pi, pj = self.grid[0], self.grid[1]
        return (self.rank % pi, (self.rank // pi) % pj, self.rank // (pi * pj))

    def split(self, d: int) -> bool:
        return self.grid[d] > 1

    def has_down(self, d: int) -> bool:
        """A part (or the periodic wrap) lies below in direction d, in another rank."""
        return self.split(d) and (self.periodic[d] or self.lo[d] > 0)

    def has_up(self, d: int) -> bool:
        return self.split(d) and (self.periodic[d] or self.hi[d] < self.n_elem[d])

    def peer(self, d: int, step: int) -> int:
        c = list(self.coords)
        c[d] = (c[d] + step) % self.grid[d]
        return c[0] + self.grid[0] * (c[1] + self.grid[1] * c[2])

    def _plane(self, d: int, c: int) -> np.ndarray:
        """Global indices (ascending) of the elements at coordinate c in direction
        d within the part's ranges in the other two directions."""
        rng = [np.arange(self.lo[e], self.hi[e]) for e in range(3)]
        rng[d] = np.array([c])
        ii, jj, kk = np.meshgrid(*rng, indexing="ij")
        ni, nj = self.n_elem[0], self.n_elem[1]
        return np.sort((ii + ni * (jj + nj * kk)).ravel())

    @functools.cached_property
    def _layout(self):
        ni, nj = self.n_elem[0], self.n_elem[1]
        ii, jj, kk = np.meshgrid(*[np.arange(self.lo[d], self.hi[d]) for d in range(3)],
                                 indexing="ij")
        xyz = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1)
        g = xyz[:, 0] + ni * (xyz[:, 1] + nj * xyz[:, 2])
        o = np.argsort(g)
        xyz, g = xyz[o], g[o]
        low = np.zeros(len(g), dtype=bool)
        up = np.zeros(len(g), dtype=bool)
        for d in range(3):
            if self.has_down(d):
                low |= xyz[:, d] == self.lo[d]
            if self.has_up(d):
                up |= xyz[:, d] == self.hi[d] - 1
        owned = np.concatenate([g[~low & ~up], g[up & ~low], g[low]])
        face = [(d, self._plane(d, self.hi[d] % self.n_elem[d]))
                for d in range(3) if self.has_up(d)]
        lower = [(d, self._plane(d, (self.lo[d] - 1) % self.n_elem[d]))
                 for d in range(3) if self.has_down(d)]
        return dict(owned=owned, n_a=int(np.sum(~low & ~up)), n_b=int(np.sum(up & ~low)),
                    face=face, lower=lower)

    @property
    def n_owned(self) -> int:
        return len(self._layout["owned"])

    @property
    def n_face_ghost(self) -> int:
        return sum(len(p) for _, p in self._layout["face"])

    @property
    def n_local(self) -> int:
        return self.n_owned + self.n_face_ghost + sum(len(p) for _, p in self._layout["lower"])

    @property
    def flux_ready(self) -> int:
        """Owned elements [0, flux_ready) have only owned lower neighbours."""
        return self._layout["n_a"] + self._layout["n_b"]

    @property
    def res_ready(self) -> int:
        """Owned elements [0, res_ready) have no ghost neighbour."""
        return self._layout["n_a"]

    def local_to_global(self) -> np.ndarray:
        lay = self._layout
        return np.concatenate([lay["owned"]] + [p for _, p in lay["face"]] +
                              [p for _, p in lay["lower"]]).astype(np.int64)

    def ghost_range(self, d: int, upper: bool) -> tuple:
        """(first local index, count) of the face ghosts (upper) or the lower
        ghosts of direction d."""
        lay = self._layout
        first = self.n_owned if upper else self.n_owned + self.n_face_ghost
        for e, p in lay["face" if upper else "lower"]:
            if e == d:
                return first, len(p)
            first += len(p)
        raise ValueError(f"no {'face' if upper else 'lower'} ghosts in direction {d}")

    def send_list(self, d: int, upper: bool) -> np.ndarray:
        """Local indices of the owned elements on the part's top (upper) or bottom
        plane of direction d, in the order of the receiving part's ghosts."""
        plane = self._plane(d, self.hi[d] - 1 if upper else self.lo[d])
        return self.local_of(plane)

    def local_of(self, glob: np.ndarray) -> np.ndarray:
        """Local indices of owned elements given by global index."""
        owned = self._layout["owned"]
        o = np.argsort(owned)
        pos = np.searchsorted(owned[o], glob)
        pos = np.minimum(pos, len(owned) - 1)
        if not np.array_equal(owned[o][pos], glob):
            raise ValueError("elements outside the part")
        return o[pos].astype(np.int32)

    def boundary_elements(self, f: int) -> np.ndarray:
        """Global indices (ascending) of the owned elements on block face f."""
        d, side = f // 2, f % 2
        c = 0 if side == 0 else self.n_elem[d] - 1
        if not self.lo[d] <= c < self.hi[d]:
            return np.zeros(0, dtype=np.int64)
        return self._plane(d, c)


def parts(n_elem: Sequence[int], grid: Sequence[int],
          periodic: Sequence[bool] = (True, True, True)) -> List[Part]:
    """The block split by a grid of ranks, each direction as evenly as possible."""
    n_elem = tuple(int(v) for v in n_elem)
    grid = tuple(int(v) for v in grid)
    for d in range(3):
        if grid[d] < 1 or grid[d] > n_elem[d]:
            raise ValueError(f"{grid[d]} ranks for {n_elem[d]} elements in direction {d}")
    cuts = [_bounds(n_elem[d], grid[d]) for d in range(3)]
    out = []
    for r in range(grid[0] * grid[1] * grid[2]):
        c = (r % grid[0], (r // grid[0]) % grid[1], r // (grid[0] * grid[1]))
        out.append(Part(n_elem, grid, r, tuple(cuts[d][c[d]] for d in range(3)),
                        tuple(cuts[d][c[d] + 1] for d in range(3)),
                        tuple(bool(v) for v in periodic)))
    return out


def slabs(n_elem: Sequence[int], world: int, periodic_k: bool = True) -> List[Part]:
    """The block split into k slabs (every rank owns at least one k layer)."""
    if world < 1 or world > int(n_elem[2]):
        raise ValueError(f"{world} ranks for {n_elem[2]} k layers")
    return parts(n_elem, (1, 1, world), (True, True, bool(periodic_k)))


def local_neighbors(part: Part, global_nbr: np.ndarray) -> np.ndarray:
    """Neighbour table of the part's local elements (-1: a face this rank does
    not evaluate, or a physical boundary face of the block). global_nbr: the
    block's [nE][6] table (-1 on boundary faces)."""
    global_nbr = np.asarray(global_nbr)
    nE = global_nbr.shape[0]
    lay = part._layout
    nO = part.n_owned
    out = np.full((part.n_local, 6), -1, dtype=np.int32)
    owned = lay["owned"]
    loc_owned = np.full(nE, -1, dtype=np.int64)
    loc_owned[owned] = np.arange(nO)
    ghost = {}
    for upper in (True, False):
        for d, plane in lay["face" if upper else "lower"]:
            t = np.full(nE, -1, dtype=np.int64)
            first, _ = part.ghost_range(d, upper)
            t[plane] = first + np.arange(len(plane))
            ghost[(d, upper)] = t
    for d in range(3):
        if part.periodic[d] and np.any(global_nbr[:, 2 * d:2 * d + 2] < 0):
            raise ValueError(f"a block periodic in direction {d} has no boundary faces there")
    for f in range(6):
        d, upper = f // 2, f % 2 == 1
        nb = global_nbr[owned, f]
        res = np.where(nb >= 0, loc_owned[np.maximum(nb, 0)], -1)
        miss = (nb >= 0) & (res < 0)
        if np.any(miss):
            t = ghost.get((d, upper))
            got = t[nb[miss]] if t is not None else np.full(int(miss.sum()), -1)
            if np.any(got < 0):
                raise ValueError(f"face {f}: a neighbour outside the part and its ghosts")
            res[miss] = got
        out[:nO, f] = res
    # Face ghosts: only their Min face towards the part.
    for d, plane in lay["face"]:
        first, count = part.ghost_range(d, True)
        below = loc_owned[global_nbr[plane, 2 * d]]
        if np.any(below < 0):
            raise ValueError(f"face ghosts of direction {d} without owned neighbours below")
        out[first:first + count, 2 * d] = below
    return out


def local_discretization(disc, part: Part):
    """The part's Discretization: per-element arrays gathered in local order,
    neighbours remapped; operators shared."""
    idx = part.local_to_global()
    return dataclasses.replace(
        disc, n_elem=(part.n_local, 1, 1),
        vol_metric=np.ascontiguousarray(disc.vol_metric[idx]),
        face_metric=np.ascontiguousarray(disc.face_metric[idx]),
        elem_scalars=np.ascontiguousarray(disc.elem_scalars[idx]),
        neighbors=local_neighbors(part, np.asarray(disc.neighbors)),
        vol_metric_dofs=(None if disc.vol_metric_dofs is None
                         else np.ascontiguousarray(disc.vol_metric_dofs[idx])))


def local_params(params: capi.Params, part: Part) -> capi.Params:
    """The block's parameters with the part's element count (owned and ghosts)."""
    p = capi.Params.from_buffer_copy(params)
    p.n_elem[:] = [part.n_local, 1, 1]
    return p


# ---------------------------------------------------------------------------
# Shards and transports
# ---------------------------------------------------------------------------

class Shard:
    """One part on the current CUDA device: a library handle holding the owned
    elements and the ghosts."""

    def __init__(self, part: Part, params: capi.Params, disc, modal: Optional[np.ndarray] = None,
                 case=None):
        from .solver import Solver
        import torch
        self.part = part
        # A part without ghosts (no split direction) is the whole block.
        self.ghosts = part.n_local > part.n_owned
        if self.ghosts:
            self.solver = Solver(local_params(params, part), local_discretization(disc, part))
            self.solver.set_partition(part.n_owned, part.n_face_ghost)
            self.solver.set_partition_parts(part.flux_ready, part.res_ready)
            for d in range(3):
                for upper in (False, True):
                    if part.has_up(d) if upper else part.has_down(d):
                        self.solver.set_send_list(2 * d + int(upper), part.send_list(d, upper))
        else:
            self.solver = Solver(params, disc)
        self.kd5 = 5 * (params.n_poly + 1) ** 3
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.open = case is not None and case.spec.is_open
        # The outlet's element-local Mach number: the value of each subface's last
        # face, which may lie in another part.
        self.outlet_local = self.open and self.ghosts and bool(case.spec.outlet_local_mach)
        if self.open:
            self._set_open_boundary(case, disc)
        if modal is not None:
            self.set_global_state(modal)

    def _set_open_boundary(self, case, disc):
        """The whole block's open boundaries, restricted to this part's elements."""
        import ctypes as C
        from . import solver as sv
        if not self.ghosts:
            self.solver.set_open_boundary(case)
            return
        ob = sv.open_boundary(case)
        sfs = sv.subfaces(case)
        keep = [np.ascontiguousarray(a) for a in (disc.vol_metric, disc.face_metric,
                                                  disc.elem_scalars)]
        nbr = np.ascontiguousarray(disc.neighbors, dtype=np.int32)
        geom = capi.Geometry(capi.ptr(keep[0]), capi.ptr(keep[1]), capi.ptr(keep[2]),
                             capi.ptr(nbr))
        nodes = np.ascontiguousarray(case.elem_nodes, dtype=np.float64)
        l2g = np.ascontiguousarray(self.part.local_to_global(), dtype=np.int64)
        n_elem = np.ascontiguousarray(self.part.n_elem, dtype=np.int32)
        lib = self.solver.lib
        rc = lib.vcpg_set_open_boundary_partition(
            self.solver.h, C.byref(ob), sfs, len(sfs) if sfs is not None else 0,
            capi.ptr(n_elem), C.byref(geom), case.spec.p_grid, disc.dof_location,
            capi.ptr(nodes), l2g.ctypes.data_as(C.POINTER(C.c_int64)))
        self.solver._check(rc, "set_open_boundary_partition")

    def mach_weights(self):
        """Per block face, (weights, global element indices) of this part's
        boundary faces there, in block element order."""
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
        for f, c in enumerate(counts):
            ids = self.part.boundary_elements(f) if c else np.zeros(0, dtype=np.int64)
            if len(ids) != int(c):
                raise ValueError(f"block face {f}: {int(c)} boundary faces for {len(ids)} "
                                 "elements")
            out.append((w[o:o + int(c)].copy(), ids))
            o += int(c)
        return out

    def outlet_mach_inputs(self):
        """(block rows, block rows of the subfaces' last faces, face-averaged Mach
        numbers) of this part's boundary rows, from the last boundary trace."""
        counts = np.zeros(6, dtype=np.int32)
        lib = self.solver.lib
        self.solver._check(lib.vcpg_boundary_mach_weights(self.solver.h, None, capi.ptr(counts)),
                           "boundary_mach_weights")
        nB = int(counts.sum())
        rows = np.zeros(max(nB, 1), dtype=np.int32)
        last = np.zeros(max(nB, 1), dtype=np.int32)
        vals = np.zeros(max(nB, 1))
        if nB:
            self.solver._check(lib.vcpg_boundary_rows(self.solver.h, capi.ptr(rows),
                                                      capi.ptr(last)), "boundary_rows")
            self.solver._check(lib.vcpg_boundary_local_mach(self.solver.h, capi.ptr(vals)),
                               "boundary_local_mach")
        return rows[:nB].copy(), last[:nB].copy(), vals[:nB].copy()

    def set_outlet_mach(self, values):
        a = np.ascontiguousarray(values, dtype=np.float64)
        if len(a) == 0:
            a = np.zeros(1)
        self.solver._check(self.solver.lib.vcpg_set_boundary_outlet_mach(self.solver.h,
                                                                          capi.ptr(a)),
                           "set_boundary_outlet_mach")

    def set_mach_sums(self, sums):
        a = np.ascontiguousarray(sums, dtype=np.float64)
        self.solver._check(self.solver.lib.vcpg_set_boundary_mach_sums(self.solver.h,
                                                                        capi.ptr(a)),
                           "set_boundary_mach_sums")

    def residual_part(self, part: int):
        if self.ghosts:
            self.solver._check(self.solver.lib.vcpg_residual_part(self.solver.h, part),
                               "residual_part")
        elif part == 0:
            self.solver.residual()

    def set_global_state(self, modal: np.ndarray):
        """Owned and ghost states taken from the block's modal state."""
        a = np.asarray(modal).reshape(-1, self.kd5)
        self.solver.set_state(a[self.part.local_to_global()])

    def owned_state(self) -> np.ndarray:
        return self.solver.get_state()[:self.part.n_owned]

    def new_buffer(self, count: int):
        import torch
        return torch.empty(max(count, 1) * self.kd5, dtype=torch.float64, device=self.device)

    def pack(self, d: int, upper: bool, buf):
        """The states of the owned plane that goes to the part above (upper) or
        below in direction d."""
        self.solver.pack_send_list(2 * d + int(upper), buf.data_ptr())

    def unpack(self, d: int, upper: bool, buf):
        """The face ghosts (upper) or the lower ghosts of direction d from buf."""
        first, count = self.part.ghost_range(d, upper)
        self.solver.unpack_states(first, count, buf.data_ptr())

    def sync(self):
        self.solver.sync()


def _channels(part: Part):
    """(direction, upper) of the planes a part sends: to the part above
    (upper, its top plane: the neighbour's lower ghosts) and below."""
    out = []
    for d in range(3):
        if part.has_up(d):
            out.append((d, True))
        if part.has_down(d):
            out.append((d, False))
    return out


class LocalTransport:
    """All parts driven by one process (one GPU): ghosts copied between the
    handles through device buffers; reductions and gathers on the host."""

    def __init__(self, shards: Sequence[Shard]):
        self.shards = list(shards)
        self.buf = [{(d, up): s.new_buffer(len(s.part.send_list(d, up)))
                     for d, up in _channels(s.part)} for s in self.shards]

    def start_exchange(self):
        """Copies every part's owned boundary planes out (the ghosts are written
        by finish_exchange)."""
        for r, s in enumerate(self.shards):
            for (d, up), b in self.buf[r].items():
                s.pack(d, up, b)

    def finish_exchange(self):
        for s in self.shards:
            s.sync()
        for r, s in enumerate(self.shards):
            for (d, up), b in self.buf[r].items():
                # The plane sent up is the lower ghosts of the part above.
                peer = self.shards[s.part.peer(d, 1 if up else -1)]
                peer.unpack(d, not up, b)
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
    """One part per process over torch.distributed (NCCL between GPUs, gloo on
    the host): per split direction the top owned plane goes to the rank above
    (its lower ghosts), the bottom one to the rank below (its face ghosts); a
    block that is not periodic in a direction has no exchange below its first
    part or above its last there. Point-to-point operations of a pair match in
    issue order, so two ranks that are each other's upper and lower neighbour
    still pair the right planes. With CUDA tensors the transfers run on a stream
    of their own, ordered after the packing on the library's stream, which in
    turn waits for them before unpacking; the work issued between
    start_exchange and finish_exchange overlaps them."""

    def __init__(self, shard, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.shards = [shard]
        part = shard.part
        self.send, self.recv = {}, {}
        for d, up in _channels(part):
            n = len(part.send_list(d, up))
            self.send[(d, up)] = shard.new_buffer(n)
            # What arrives from the part above fills the face ghosts, from below the lower ones.
            self.recv[(d, up)] = shard.new_buffer(part.ghost_range(d, up)[1])
        self.comm = None
        self.works = []
        self.probe = shard.new_buffer(1)
        if self.probe.is_cuda:
            import torch
            self.comm = torch.cuda.Stream(device=self.probe.device)

    def _lib_stream(self):
        import torch
        return torch.cuda.ExternalStream(self.shards[0].solver.stream,
                                         device=self.probe.device)

    def start_exchange(self):
        s = self.shards[0]
        part, dist = s.part, self.dist
        for (d, up), b in self.send.items():
            s.pack(d, up, b)
        self.works = []
        ops = []
        for d in range(3):
            if part.has_up(d):
                ops.append(dist.P2POp(dist.isend, self.send[(d, True)], part.peer(d, 1),
                                      self.group))
            if part.has_down(d):
                ops.append(dist.P2POp(dist.isend, self.send[(d, False)], part.peer(d, -1),
                                      self.group))
                ops.append(dist.P2POp(dist.irecv, self.recv[(d, False)], part.peer(d, -1),
                                      self.group))
            if part.has_up(d):
                ops.append(dist.P2POp(dist.irecv, self.recv[(d, True)], part.peer(d, 1),
                                      self.group))
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
        for (d, up), b in self.recv.items():
            s.unpack(d, up, b)
        s.sync()

    def exchange(self):
        self.start_exchange()
        self.finish_exchange()

    def reduce(self, values, op: str):
        import torch
        dist = self.dist
        dev = self.probe.device
        t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=dev)
        t = t.min() if op == "min" else t.max()
        t = t.reshape(1)
        dist.all_reduce(t, op=dist.ReduceOp.MIN if op == "min" else dist.ReduceOp.MAX,
                        group=self.group)
        return float(t.item())

    def gather(self, items):
        """Every rank's item in rank order (this process contributes items[0])."""
        out = [None] * self.shards[0].part.world
        self.dist.all_gather_object(out, items[0], group=self.group)
        return out


def block_mach_sums(per_rank) -> np.ndarray:
    """Per block face, the sum of the Mach weights of all parts in block
    element order: per rank and block face (weights, global element indices),
    merged by element index and summed one after the other, as one GPU sums its
    list."""
    sums = np.zeros(6)
    for f in range(6):
        w = np.concatenate([np.asarray(r[f][0], dtype=np.float64) for r in per_rank])
        ids = np.concatenate([np.asarray(r[f][1], dtype=np.int64) for r in per_rank])
        m = 0.0
        for x in w[np.argsort(ids, kind="stable")]:
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
        if any(s.outlet_local for s in self.shards):
            # Every rank's face values by block row; each outlet row takes its
            # subface's last face's value, wherever that face lies.
            mine = [s.outlet_mach_inputs() for s in self.shards]
            by_row = {}
            for rows, vals in self.t.gather([(m[0], m[2]) for m in mine]):
                by_row.update(zip(rows.tolist(), vals.tolist()))
            for s, (_, last, _) in zip(self.shards, mine):
                s.set_outlet_mach([by_row[int(r)] if r >= 0 else 0.0 for r in last])

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
