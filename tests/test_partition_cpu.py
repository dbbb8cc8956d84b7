"""Host logic of a block split into Cartesian parts (vcp3d_open_b200.partition):
the rank grid, the local neighbour tables and send lists against the block's,
the Mach-sum merge, and the halo exchange of DistTransport over
torch.distributed with gloo between 2 and 4 processes, on host stand-ins for the
library handles."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from vcp3d_open_b200 import cases, partition, solver

TWO_PI = 6.283185307179586


def _block(n_elem=(3, 2, 5), p=2):
    spec = cases.CaseSpec(name="slabs", kind="tgv", n_elem=n_elem, p=p, hi=(TWO_PI,) * 3,
                          mach=0.1, reynolds=1600.0, grid_map="random", grid_amp=0.01)
    case = cases.build_case(spec)
    prm = solver.make_params(case)
    return case, prm, solver.setup_discretization(case, prm)


GRIDS = [(1, 1, 1), (1, 1, 2), (1, 1, 5), (3, 1, 1), (2, 2, 1), (1, 2, 3), (3, 2, 2)]


def _check_part_tables(part, nbr, ln):
    """Owned faces reach the block's neighbours; face ghosts evaluate only their
    Min face towards the part; lower ghosts evaluate nothing; the owned order
    puts elements without lower ghosts, then without any ghost, first."""
    l2g = part.local_to_global()
    nO = part.n_owned
    own = l2g[:nO]
    for f in range(6):
        want, got = nbr[own, f], ln[:nO, f]
        assert np.array_equal(got < 0, want < 0)
        assert np.array_equal(l2g[got[got >= 0]], want[want >= 0])
    for d in range(3):
        for upper in (True, False):
            live = part.has_up(d) if upper else part.has_down(d)
            if not live:
                with pytest.raises(ValueError):
                    part.ghost_range(d, upper)
                continue
            first, count = part.ghost_range(d, upper)
            rows = ln[first:first + count]
            if upper:
                assert np.array_equal(l2g[rows[:, 2 * d]], nbr[l2g[first:first + count], 2 * d])
                assert np.all(rows[:, 2 * d] < nO)
                assert np.all(np.delete(rows, 2 * d, axis=1) == -1)
            else:
                assert np.all(rows == -1)
    ghost = ln[:nO] >= nO
    lower_ghost = ghost[:, 0::2].any(axis=1)
    assert not lower_ghost[:part.flux_ready].any() and lower_ghost[part.flux_ready:].all()
    assert not ghost[:part.res_ready].any() and ghost[part.res_ready:].any(axis=1).all()
    # Send lists: the owned planes, in the order of the receiving ghosts.
    for d in range(3):
        for upper in (True, False):
            if part.has_up(d) if upper else part.has_down(d):
                sl = part.send_list(d, upper)
                coord = part.hi[d] - 1 if upper else part.lo[d]
                g = own[sl]
                c = [g % part.n_elem[0], (g // part.n_elem[0]) % part.n_elem[1],
                     g // (part.n_elem[0] * part.n_elem[1])]
                assert np.all(c[d] == coord) and np.all(np.diff(g) > 0)


@pytest.mark.parametrize("grid", GRIDS)
def test_local_tables_follow_the_block(grid):
    _, prm, disc = _block()
    nbr = disc.neighbors
    owned = []
    for part in partition.parts((3, 2, 5), grid):
        ln = partition.local_neighbors(part, nbr)
        _check_part_tables(part, nbr, ln)
        l2g = part.local_to_global()
        owned.extend(l2g[:part.n_owned])
        ld = partition.local_discretization(disc, part)
        assert np.array_equal(ld.face_metric, disc.face_metric[l2g])
        lp = partition.local_params(prm, part)
        assert tuple(lp.n_elem) == (part.n_local, 1, 1) and lp.mu == prm.mu
        if part.world == 1:
            assert part.n_local == part.n_owned == 30
    assert sorted(owned) == list(range(30))


def test_rank_grid_and_limits():
    """The ranks per direction double one direction at a time, where the
    elements per rank halve evenly and are the most (the reference's
    DistributeGrid)."""
    assert partition.rank_grid((32, 32, 32), 8) == (2, 2, 2)
    assert partition.rank_grid((32, 32, 32), 2) == (1, 1, 2)
    assert partition.rank_grid((32, 32, 32), 4) == (1, 2, 2)
    assert partition.rank_grid((40, 20, 20), 4) == (2, 1, 2)
    assert partition.rank_grid((48, 48, 48), 8, allow=(False, True, True)) == (1, 2, 4)
    assert partition.rank_grid((5, 3, 7), 1) == (1, 1, 1)
    with pytest.raises(ValueError):
        partition.rank_grid((3, 3, 3), 2)
    with pytest.raises(ValueError):
        partition.rank_grid((4, 4, 4), 3)
    assert [p.hi[2] - p.lo[2] for p in partition.slabs((2, 2, 7), 3)] == [3, 2, 2]
    with pytest.raises(ValueError):
        partition.slabs((2, 2, 3), 4)
    with pytest.raises(ValueError):
        partition.parts((2, 2, 3), (3, 1, 1))
    _, _, disc = _block()
    wall = np.array(disc.neighbors)
    wall[0, 4] = -1
    with pytest.raises(ValueError, match="periodic in direction 2"):
        partition.local_neighbors(partition.slabs((3, 2, 5), 2)[0], wall)


@pytest.mark.parametrize("grid", [(1, 1, 2), (1, 1, 3), (3, 1, 1), (3, 2, 1), (2, 1, 2)])
def test_local_tables_with_open_faces(grid):
    """A block with boundary faces in i and k (not periodic there): boundary
    faces stay -1, the first part of a direction has no lower and the last no
    upper exchange there."""
    n_elem = (3, 2, 5)
    spec = cases.CaseSpec(name="open", kind="pulse", n_elem=n_elem, p=2, hi=(3.0, 2.0, 5.0),
                          mach=0.3, grid_map="none", center=(1.5, 1.0, 2.5),
                          bc=("inflow_static_nscbc", "outflow_nscbc", "periodic", "periodic",
                              "inflow_static_nscbc", "outflow_nscbc"))
    case = cases.build_case(spec)
    prm = solver.make_params(case)
    nbr = solver.setup_discretization(case, prm).neighbors
    for part in partition.parts(n_elem, grid, (False, True, False)):
        ln = partition.local_neighbors(part, nbr)
        _check_part_tables(part, nbr, ln)
        c = part.coords
        for d in (0, 2):
            assert part.has_down(d) == (c[d] > 0)
            assert part.has_up(d) == (c[d] < grid[d] - 1)
        # Boundary elements of a block face: the owned ones on it, in block order.
        for f in (0, 1, 4, 5):
            g = part.boundary_elements(f)
            assert np.all(nbr[g, f] < 0) and np.all(np.isin(g, part.local_to_global()[:part.n_owned]))


def test_block_mach_sums_in_block_order():
    """The parts' per-face weights, merged by element index and summed one
    after the other, are the sequential sum over the block's list."""
    rng = np.random.default_rng(4)
    block = [rng.standard_normal(n) for n in (7, 0, 5, 5, 3, 0)]
    ids = [np.sort(rng.choice(100, size=len(b), replace=False)) for b in block]
    owner = [rng.integers(0, 3, size=len(b)) for b in block]
    ranks = [[(block[f][owner[f] == r], ids[f][owner[f] == r]) for f in range(6)]
             for r in range(3)]
    got = partition.block_mach_sums(ranks)
    for f in range(6):
        m = 0.0
        for x in block[f]:
            m += float(x)
        assert got[f] == m


class HostShard:
    """Stand-in for partition.Shard: the part's states in host memory."""

    def __init__(self, part, kd5, block_state):
        import torch
        self.torch = torch
        self.part, self.kd5 = part, kd5
        self.state = np.zeros((part.n_local, kd5))
        self.state[:part.n_owned] = block_state[part.local_to_global()[:part.n_owned]]

    def new_buffer(self, count):
        return self.torch.empty(max(count, 1) * self.kd5, dtype=self.torch.float64)

    def pack(self, d, upper, buf):
        rows = self.state[self.part.send_list(d, upper)].ravel()
        buf[:rows.size].copy_(self.torch.from_numpy(rows.copy()))

    def unpack(self, d, upper, buf):
        first, count = self.part.ghost_range(d, upper)
        self.state[first:first + count] = buf[:count * self.kd5].numpy().reshape(count, self.kd5)

    def sync(self):
        pass


def _rank_main(rank, world, port, n_elem, grid, periodic, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        kd5 = 7
        rng = np.random.default_rng(3)
        block = rng.standard_normal((int(np.prod(n_elem)), kd5))
        part = partition.parts(n_elem, grid, periodic)[rank]
        sh = HostShard(part, kd5, block)
        t = partition.DistTransport(sh)
        t.exchange()
        # Every ghost exists because a neighbouring part sends it.
        ok = np.array_equal(sh.state, block[part.local_to_global()])
        ok = ok and t.gather([rank * 10])[:world] == [r * 10 for r in range(world)]
        lo = t.reduce([float(rank) + 0.5, 10.0], "min")
        hi = t.reduce([-1.0, float(rank)], "max")
        out.put((rank, ok, lo, hi))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("grid,periodic", [
    ((1, 1, 2), (True, True, True)), ((1, 1, 3), (True, True, False)),
    ((2, 1, 1), (True, True, True)), ((1, 3, 1), (True, False, True)),
    ((2, 2, 1), (False, True, True)), ((1, 2, 2), (True, True, True))])
def test_exchange_over_gloo(grid, periodic):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = grid[0] * grid[1] * grid[2]
    n_elem = (4, 3, 4)
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, n_elem, grid, periodic, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [True] * world
    assert all(r[2] == 0.5 for r in res) and all(r[3] == world - 1 for r in res)
