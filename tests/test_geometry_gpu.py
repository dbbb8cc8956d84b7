"""Metric terms computed on the GPU (vcpg_setup_geometry_device) against the
host set-up (vcpg_setup_geometry): the same arithmetic, the same doubles, on
curvilinear, randomly perturbed and open-boundary grids of degrees 1 to 9."""
from __future__ import annotations

import numpy as np
import pytest

from vcp3d_open_b200 import cases, solver

pytestmark = pytest.mark.gpu

SPECS = [
    cases.CaseSpec(name="vortex_p3", kind="vortex", n_elem=(4, 3, 2), p=3),
    cases.CaseSpec(name="tgv_p4", kind="tgv", n_elem=(3, 3, 3), p=4, hi=(6.283185307179586,) * 3,
                   grid_map="random", grid_amp=0.02, seed=2),
    cases.CaseSpec(name="vortex_p2", kind="vortex", n_elem=(5, 2, 3), p=2),
    cases.CaseSpec(name="tgv_p5", kind="tgv", n_elem=(2, 2, 2), p=5, hi=(6.283185307179586,) * 3,
                   grid_map="random", grid_amp=0.02, seed=3),
    cases.CaseSpec(name="tgv_p1", kind="tgv", n_elem=(3, 3, 3), p=1, hi=(6.283185307179586,) * 3,
                   grid_map="random", grid_amp=0.02, seed=5),
    cases.CaseSpec(name="vortex_p7", kind="vortex", n_elem=(2, 2, 2), p=7, n_poly_int=22),
    cases.CaseSpec(name="tgv_p8", kind="tgv", n_elem=(2, 2, 2), p=8, hi=(6.283185307179586,) * 3,
                   grid_map="random", grid_amp=0.005, seed=6),
    cases.CaseSpec(name="pulse_p3", kind="pulse", n_elem=(4, 3, 2), p=3, hi=(4.0, 3.0, 2.0),
                   grid_map="random", grid_amp=0.01, seed=4,
                   bc=("inflow_static_nscbc", "outflow_nscbc", "periodic", "periodic",
                       "wall_inviscid", "wall_inviscid")),
]


@pytest.mark.parametrize("spec", SPECS, ids=lambda s: s.name)
def test_device_metrics_equal_host(gpu_available, spec):
    case = cases.build_case(spec)
    params = solver.make_params(case)
    host = solver.setup_discretization(case, params)
    dev = solver.setup_discretization(case, params, device=True)
    for name in ("vol_metric", "face_metric", "elem_scalars", "neighbors", "leg_int",
                 "dleg_int", "leg_face", "dleg_face", "w_int", "leg_dofs", "basis_center"):
        a, b = getattr(host, name), getattr(dev, name)
        assert np.array_equal(a, b), (name, float(np.max(np.abs(a - b))))
