"""Host logic of a block split into k slabs (vcp3d_open_b200.partition): the
local neighbour tables against the block's, and the halo exchange of
DistTransport over torch.distributed with gloo between 2 and 3 processes, on
host stand-ins for the library handles."""
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


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_local_tables_follow_the_block(world):
    _, prm, disc = _block()
    nbr = disc.neighbors
    owned = []
    for sl in partition.slabs((3, 2, 5), world):
        ln = partition.local_neighbors(sl, nbr)
        l2g = sl.local_to_global()
        owned.extend(l2g[:sl.n_owned])
        # Every face of an owned element reaches the block's neighbour.
        for f in range(6):
            assert np.array_equal(l2g[ln[:sl.n_owned, f]], nbr[l2g[:sl.n_owned], f])
        # The ghost layer above evaluates only its k-Min face, towards the slab.
        up = slice(sl.upper_ghost, sl.upper_ghost + sl.layer)
        assert np.array_equal(l2g[ln[up, 4]], nbr[l2g[up], 4])
        assert np.all(ln[up][:, [0, 1, 2, 3, 5]] == -1)
        assert np.all(ln[sl.lower_ghost:] == -1)
        ld = partition.local_discretization(disc, sl)
        assert np.array_equal(ld.face_metric, disc.face_metric[l2g])
        lp = partition.local_params(prm, sl)
        assert tuple(lp.n_elem) == (3, 2, sl.n_layers + 2) and lp.mu == prm.mu
    assert sorted(owned) == list(range(30))


def test_slab_split_and_limits():
    assert [s.n_layers for s in partition.slabs((2, 2, 7), 3)] == [3, 2, 2]
    with pytest.raises(ValueError):
        partition.slabs((2, 2, 3), 4)
    _, _, disc = _block()
    wall = np.array(disc.neighbors)
    wall[0, 4] = -1
    with pytest.raises(ValueError, match="periodic in k"):
        partition.local_neighbors(partition.slabs((3, 2, 5), 2)[0], wall)
    inner = np.array(disc.neighbors)
    inner[7, 4] = inner[7, 5] = -1       # element 7 lies in layer 1, inside the block
    with pytest.raises(ValueError, match="inside the block"):
        partition.local_neighbors(partition.slabs((3, 2, 5), 2, periodic_k=False)[0], inner)


@pytest.mark.parametrize("world", [1, 2, 3])
def test_local_tables_with_open_faces(world):
    """A block with boundary faces in i and k (not periodic there): boundary
    faces stay -1, the first slab has no lower and the last no upper exchange."""
    n_elem = (3, 2, 5)
    spec = cases.CaseSpec(name="open", kind="pulse", n_elem=n_elem, p=2, hi=(3.0, 2.0, 5.0),
                          mach=0.3, grid_map="none", center=(1.5, 1.0, 2.5),
                          bc=("inflow_static_nscbc", "outflow_nscbc", "periodic", "periodic",
                              "inflow_static_nscbc", "outflow_nscbc"))
    case = cases.build_case(spec)
    prm = solver.make_params(case)
    nbr = solver.setup_discretization(case, prm).neighbors
    for sl in partition.slabs(n_elem, world, periodic_k=False):
        ln = partition.local_neighbors(sl, nbr)
        l2g = sl.local_to_global()
        own = l2g[:sl.n_owned]
        for f in range(6):
            want = nbr[own, f]
            got = ln[:sl.n_owned, f]
            assert np.array_equal(got < 0, want < 0)
            assert np.array_equal(l2g[got[got >= 0]], want[want >= 0])
        assert sl.has_down == (sl.rank > 0) and sl.has_up == (sl.rank < world - 1)
        up = slice(sl.upper_ghost, sl.upper_ghost + sl.layer)
        assert np.all(ln[up, 4] == (-1 if not sl.has_up else ln[up, 4]))
        assert np.all(ln[up][:, [0, 1, 2, 3, 5]] == -1)


def test_block_mach_sums_in_block_order():
    """The slabs' per-face weights summed one after the other in rank order is
    the sequential sum over the block's list."""
    rng = np.random.default_rng(4)
    block = [rng.standard_normal(n) for n in (7, 0, 5, 5, 3, 0)]
    cuts = [(0, 3, 7), (0, 0, 0), (0, 2, 5), (0, 4, 5), (0, 0, 3), (0, 0, 0)]
    ranks = [[block[f][c[r]:c[r + 1]] for f, c in enumerate(cuts)] for r in range(2)]
    got = partition.block_mach_sums(ranks)
    for f in range(6):
        m = 0.0
        for x in block[f]:
            m += float(x)
        assert got[f] == m


class HostShard:
    """Stand-in for partition.Shard: the slab's states in host memory."""

    def __init__(self, slab, kd5, block_state):
        import torch
        self.torch = torch
        self.slab, self.kd5 = slab, kd5
        self.state = np.zeros((slab.n_local, kd5))
        self.state[:slab.n_owned] = block_state[slab.local_to_global()[:slab.n_owned]]

    def new_buffer(self, count):
        return self.torch.empty(count * self.kd5, dtype=self.torch.float64)

    def pack(self, first, count, buf):
        buf.copy_(self.torch.from_numpy(self.state[first:first + count].ravel().copy()))

    def unpack(self, first, count, buf):
        self.state[first:first + count] = buf.numpy().reshape(count, self.kd5)

    def sync(self):
        pass


def _rank_main(rank, world, port, n_elem, out, periodic_k=True):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        kd5 = 7
        rng = np.random.default_rng(3)
        block = rng.standard_normal((int(np.prod(n_elem)), kd5))
        sl = partition.slabs(n_elem, world, periodic_k=periodic_k)[rank]
        sh = HostShard(sl, kd5, block)
        t = partition.DistTransport(sh)
        t.exchange()
        want = block[sl.local_to_global()].copy()
        if not sl.has_up:     # no slab above: that ghost layer stays as it was
            want[sl.upper_ghost:sl.upper_ghost + sl.layer] = 0.0
        if not sl.has_down:
            want[sl.lower_ghost:sl.lower_ghost + sl.layer] = 0.0
        ok = np.array_equal(sh.state, want)
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


@pytest.mark.parametrize("periodic_k", [True, False])
@pytest.mark.parametrize("world", [2, 3])
def test_exchange_over_gloo(world, periodic_k):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    n_elem = (2, 3, 4)
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, n_elem, q, periodic_k))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [True] * world
    assert all(r[2] == 0.5 for r in res) and all(r[3] == world - 1 for r in res)
