"""Case generation and the reference's file formats (PLOT3D grid, SU2 restart)."""
from __future__ import annotations

import os

import numpy as np

from vcp3d_open_b200 import cases


def test_plot3d_and_restart_round_trip(tmp_path):
    spec = cases.CaseSpec(kind="vortex", n_elem=(3, 2, 2), p=2)
    c = cases.build_case(spec)
    cfg = cases.write_case(c, str(tmp_path))
    assert os.path.exists(cfg)
    g = cases.read_plot3d(os.path.join(tmp_path, "grid.xyz"))
    np.testing.assert_array_equal(g, c.grid)
    xyz, cons = cases.read_su2_restart(os.path.join(tmp_path, "restart.dat"), spec.n_elements,
                                       (spec.p + 1) ** 3)
    np.testing.assert_array_equal(xyz, c.dof_xyz)
    np.testing.assert_array_equal(cons, c.cons)
    # File size matches the reference's precision detection rule (8 bytes per item).
    size = os.path.getsize(os.path.join(tmp_path, "restart.dat"))
    n_items = 8 * spec.n_elements * (spec.p + 1) ** 3 + 8
    assert round((size - 20 - 8 * 33 - 4) / n_items) == 8


def test_grid_is_periodic_consistent():
    for gm in ("sine", "random"):
        spec = cases.CaseSpec(kind="vortex", n_elem=(4, 3, 2), p=3, grid_map=gm, grid_amp=0.02)
        g = cases.make_grid(spec)
        L = [spec.hi[d] - spec.lo[d] for d in range(3)]
        # Opposite block faces differ by the periodic translation only.
        np.testing.assert_allclose(g[0, :, :, -1] - g[0, :, :, 0], L[0], atol=1e-12)
        np.testing.assert_allclose(g[1, :, -1, :] - g[1, :, 0, :], L[1], atol=1e-12)
        np.testing.assert_allclose(g[2, -1, :, :] - g[2, 0, :, :], L[2], atol=1e-12)
        np.testing.assert_allclose(g[1:, :, :, -1], g[1:, :, :, 0], atol=1e-12)


def test_generation_is_deterministic_and_seeded():
    a = cases.build_case(cases.CaseSpec(kind="tgv", n_elem=(2, 2, 2), p=3, grid_map="random", seed=5))
    b = cases.build_case(cases.CaseSpec(kind="tgv", n_elem=(2, 2, 2), p=3, grid_map="random", seed=5))
    c = cases.build_case(cases.CaseSpec(kind="tgv", n_elem=(2, 2, 2), p=3, grid_map="random", seed=6))
    np.testing.assert_array_equal(a.grid, b.grid)
    assert np.abs(a.grid - c.grid).max() > 0


def test_vortex_state_is_isentropic_and_at_free_stream_far_away():
    spec = cases.CaseSpec(kind="vortex", n_elem=(4, 4, 1), p=3)
    c = cases.build_case(spec)
    rho = c.cons[:, 0]
    rhoE = c.cons[:, 4]
    mom = c.cons[:, 1:4]
    p = (cases.GAMMA - 1.0) * (rhoE - 0.5 * (mom ** 2).sum(axis=1) / rho)
    s = p / rho ** cases.GAMMA
    np.testing.assert_allclose(s, c.ref.p_ref / c.ref.rho_ref ** cases.GAMMA, rtol=1e-12)
    assert rho.min() < 0.9 * c.ref.rho_ref < rho.max()
