"""Characteristic (PC-NSCBC) boundaries, sponge layers and the matching layer on
the GPU against the reference solver's own results (open_*.npz fixtures made by
tests/golden/make_golden.py with oracle/_ref).

Fixtures: static inflow + outflow + sponge + matching layer (i and j faces),
degree 4 with the Roe flux and an inlet that keeps the outgoing amplitudes,
and characteristic k faces with Mach-averaged transverse relaxation.
"""
from __future__ import annotations

import os
import tempfile

import numpy as np
import pytest

from conftest import assert_forces_match, load_golden, open_golden_files, rel_l2
from oracle import records
from vcp3d_open_b200 import capi, cases, solver, workloads

pytestmark = pytest.mark.gpu

TOL_STATE = 1e-12
TOL_DT = 1e-13


def _solver(spec, precision=capi.FP64):
    case = cases.build_case(spec)
    return solver.create(case, precision=precision)


@pytest.mark.parametrize("path", open_golden_files(), ids=os.path.basename)
def test_open_boundary_residual_matches_reference(gpu_available, path):
    g = load_golden(path)
    s = _solver(g["spec"])
    try:
        s.set_state(g["sol0"])
        mon = s.residual(monitoring=True, keep_raw=True)
        raw, res = s.get_raw_residual(), s.get_residual()
        # The residual is a small difference of large volume, face and boundary
        # terms; the bound is relative to the residual itself, 1e-10 as for the
        # periodic fixtures.
        assert rel_l2(raw, g["res_raw"]) < 1e-10
        assert rel_l2(res, g["res"]) < 1e-10
        assert mon[6] == pytest.approx(g["monitor"][6], rel=1e-13)
        # Largest eddy viscosity of the volume and face points (0 without a model).
        # The reference also takes the maximum over the padding points of its
        # face arrays, where a characteristic face reconstructs a gradient from
        # placeholder data, so with such faces its value bounds the maximum
        # over the integration points from above.
        assert_forces_match(mon, g["monitor"], g["spec"])
        ref_eddy = max(g["monitor"][7], 0.0)
        if any(b.endswith("_nscbc") for b in g["spec"].bc):
            assert mon[7] <= ref_eddy * (1.0 + 1e-12)
        else:
            assert mon[7] == pytest.approx(ref_eddy, rel=1e-10)
        assert s.time_step() == pytest.approx(g["dt0"][0], rel=TOL_DT)
    finally:
        s.close()


@pytest.mark.parametrize("path", open_golden_files(), ids=os.path.basename)
def test_open_boundary_steps_match_reference(gpu_available, path):
    g = load_golden(path)
    s = _solver(g["spec"])
    try:
        n = int(g["n_steps"])
        for scheme, key in ((capi.SSPRK3, "ssp"), (capi.LSRK4, "ls")):
            s.set_state(g["sol0"])
            hist = s.step(n, scheme)
            assert rel_l2(s.get_state(), g[key + "_sol"]) < TOL_STATE, key
            np.testing.assert_allclose(hist, g[key + "_dt"], rtol=TOL_DT)
    finally:
        s.close()


def test_open_boundary_launches_and_graph(gpu_available):
    """Every residual of an open block is four launches: boundary traces and Mach
    weights, boundary states and fluxes, interior face fluxes, and the fused
    residual kernel."""
    g = load_golden(open_golden_files()[0])
    s = _solver(g["spec"])
    try:
        s.set_state(g["sol0"])
        n0 = s.launch_count
        s.residual()
        assert s.launch_count - n0 == 4
        n0 = s.launch_count
        s.step(2, capi.LSRK4)
        # dt + finalize + 5 x (stage update + 4 residual launches) per step.
        assert s.launch_count - n0 == 2 * (2 + 5 * 4)
    finally:
        s.close()


def test_mixed_form_on_open_boundaries(gpu_available):
    """The mixed form keeps the boundary kernels in FP64 and stays within 1e-6
    of the reference's FP64 states."""
    for path in open_golden_files():
        g = load_golden(path)
        s = _solver(g["spec"], precision=capi.MIXED)
        try:
            s.set_state(g["sol0"])
            for dt in np.atleast_1d(g["ls_dt"]):
                s.step(1, capi.LSRK4, fixed_dt=float(dt))
            assert rel_l2(s.get_state(), g["ls_sol"]) < 1e-6, path
        finally:
            s.close()


def test_boundary_face_without_condition_is_reported(gpu_available):
    """A non-periodic block face left without a boundary condition is a status
    error of the residual, not a silent zero flux."""
    g = load_golden(open_golden_files()[0])
    spec = g["spec"]
    case = cases.build_case(spec)
    prm = solver.make_params(case)
    disc = solver.setup_discretization(case, prm)
    s = solver.Solver(prm, disc)  # open boundaries not configured
    try:
        s.set_state(g["sol0"])
        with pytest.raises(capi.VcpgError) as ei:
            s.residual()
        assert ei.value.code == 8
    finally:
        s.close()


@pytest.mark.skipif(not records.have_reference_build(), reason="oracle/_ref not built")
def test_config3_pulse_full_size_matches_reference_build(gpu_available):
    """The open-boundary configuration at full size (40x20x20 elements, p4, NSCBC
    inflow/outflow, sponge and matching layers): 2 LSRK4 steps vs the reference
    build run on the same files."""
    spec = workloads.make_spec("pulse40_p4_lsrk4")
    case = cases.build_case(spec)
    s = solver.create(case)
    try:
        hist = s.step(2, capi.LSRK4)
        with tempfile.TemporaryDirectory() as tmp:
            cfg = cases.write_case(case, tmp)
            out = os.path.join(tmp, "run.bin")
            records.run_reference(cfg, "run", out, "--steps", "2", "--scheme", "lsrk4",
                                  threads=os.cpu_count() or 1)
            r = records.read_records(out)
        K3 = (spec.p + 1) ** 3
        assert rel_l2(s.get_state(), r["sol"][:, :, :K3]) < TOL_STATE
        np.testing.assert_allclose(hist, r["dtHist"], rtol=TOL_DT)
    finally:
        s.close()
