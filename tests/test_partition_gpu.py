"""A block split into Cartesian parts (k slabs, i or j splits, 2x2 and 2x2x2
grids, and the unsplit block through the same stage-wise loop), all parts
driven by one process on one GPU (LocalTransport):
residuals and steps of the partitioned block against the single-handle path on
the same block, for periodic blocks and for blocks with open boundaries
(characteristic conditions, sponge and matching layers, subfaces, boundary
faces in the split directions, the outlet's element-local Mach number taken
from a subface's last face in another part). Every face is evaluated from the same inputs in
both and the boundary-averaged Mach number is summed in the same order, so the
results are equal bit for bit. The residual computes the part that needs no
ghost state before the ghosts are written (LocalTransport unpacks them only
afterwards), so a dependence on a stale ghost would show."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2
from make_golden import OPEN_SPECS
from vcp3d_open_b200 import capi, cases, partition, solver

pytestmark = pytest.mark.gpu

TWO_PI = 6.283185307179586

SPECS = [
    cases.CaseSpec(name="tgv_p3_3x4x6", kind="tgv", n_elem=(3, 4, 6), p=3, hi=(TWO_PI,) * 3,
                   mach=0.1, reynolds=1600.0, grid_map="random", grid_amp=0.01, seed=2),
    cases.CaseSpec(name="vortex_p2_roe_4x3x5", kind="vortex", n_elem=(4, 3, 5), p=2,
                   riemann="Roe", hi=(10.0, 7.5, 12.5), center=(5.0, 3.75, 6.25)),
    cases.CaseSpec(name="tgv_p4_wale_3x3x4", kind="tgv", n_elem=(3, 3, 4), p=4,
                   hi=(TWO_PI,) * 3, mach=0.1, reynolds=1.0e5, grid_map="random",
                   grid_amp=0.005, seed=11, sgs="wale"),
]


OPEN = [OPEN_SPECS["pulse_p3_6x4x2_sponge_cml"], OPEN_SPECS["pulse_p3_3x3x4_kfaces"],
        OPEN_SPECS["subfaces_p3_4x4x2"], OPEN_SPECS["pulse_p3_3x3x4_kfaces_local"]]


def _setup(spec, grid, precision=capi.FP64):
    case = cases.build_case(spec)
    prm = solver.make_params(case, precision=precision)
    disc = solver.setup_discretization(case, prm)
    modal = solver.nodal_to_modal(case, prm)
    whole = solver.Solver(prm, disc)
    if spec.is_open:
        whole.set_open_boundary(case)
    whole.set_state(modal)
    shards = [partition.Shard(pt, prm, disc, modal, case=case)
              for pt in partition.parts(spec.n_elem, grid, [v == 1 for v in spec.periodic])]
    return whole, partition.ShardedSolver(partition.LocalTransport(shards))


def _gather(sharded, what):
    """The owned parts in block element order."""
    n = sum(s.part.n_owned for s in sharded.shards)
    out = None
    for s in sharded.shards:
        a = s.solver.get_residual() if what == "res" else s.solver.get_state()
        if out is None:
            out = np.zeros((n,) + a.shape[1:])
        out[s.part.local_to_global()[:s.part.n_owned]] = a[:s.part.n_owned]
    return out


GRIDS = [(1, 1, 1), (1, 1, 2), (1, 1, 3), (2, 1, 1), (1, 2, 1), (2, 2, 1), (2, 2, 2)]


@pytest.mark.parametrize("grid", GRIDS, ids=lambda g: "x".join(map(str, g)))
@pytest.mark.parametrize("spec", SPECS + OPEN, ids=lambda s: s.name)
def test_partitioned_residual_and_steps_equal_the_block(gpu_available, spec, grid):
    if any(g > n for g, n in zip(grid, spec.n_elem)):
        pytest.skip("more parts than elements in a direction")
    whole, sharded = _setup(spec, grid)
    try:
        mon_w = whole.residual(monitoring=True)
        mon_s = sharded.residual(monitoring=True)
        assert np.array_equal(_gather(sharded, "res"), whole.get_residual())
        assert mon_s[6] == mon_w[6] and mon_s[7] == mon_w[7]
        assert sharded.time_step() == whole.time_step()
        for scheme in (capi.LSRK4, capi.SSPRK3):
            hw = whole.step(2, scheme)
            hs = sharded.step(2, scheme)
            assert np.array_equal(hs, hw)
            assert np.array_equal(_gather(sharded, "state"), whole.get_state())
    finally:
        whole.close()
        for s in sharded.shards:
            s.solver.close()


def test_partitioned_mixed_form(gpu_available):
    whole, sharded = _setup(SPECS[0], (1, 2, 2), precision=capi.MIXED)
    try:
        hw = whole.step(3, capi.LSRK4)
        hs = sharded.step(3, capi.LSRK4)
        np.testing.assert_allclose(hs, hw, rtol=1e-14)
        assert rel_l2(_gather(sharded, "state"), whole.get_state()) < 1e-14
    finally:
        whole.close()
        for s in sharded.shards:
            s.solver.close()


def test_partitioned_handle_refuses_whole_block_calls(gpu_available):
    _, sharded = _setup(SPECS[1], (1, 1, 2))
    try:
        s = sharded.shards[0].solver
        with pytest.raises(capi.VcpgError, match="stage by stage"):
            s.step(1)
        with pytest.raises(capi.VcpgError, match="partition"):
            s.set_partition(0, 0)
        with pytest.raises(capi.VcpgError):
            s.rk_stage(capi.SSPRK3, 3, 1e-3)
    finally:
        for sh in sharded.shards:
            sh.solver.close()
