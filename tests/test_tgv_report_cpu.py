"""The kinetic-energy quadrature of the Taylor-Green report on the initial
field: E* = 1/8 of the incompressible vortex (up to the density variations of
the Mach 0.1 pressure field) and the incompressible dissipation 3 / (4 Re)."""
from __future__ import annotations

from vcp3d_open_b200 import cases, solver, tgv_report, workloads


def test_initial_kinetic_energy_and_dissipation():
    spec = workloads.make_spec("tgv16_p4_lsrk4")
    spec = cases.CaseSpec(**{**spec.__dict__, "n_elem": (4, 4, 4)})
    case = cases.build_case(spec)
    prm = solver.make_params(case)
    disc = solver.setup_discretization(case, prm)
    modal = solver.nodal_to_modal(case, prm)
    v0 = case.ref.v_inf / case.ref.u_ref
    assert abs(tgv_report.kinetic_energy(modal, disc) / v0 ** 2 - 0.125) < 1e-4
    assert abs(tgv_report.initial_dissipation(1600.0) - 0.75 / 1600.0) < 1e-15
