"""Parity of the CUDA path (through the C ABI) with the reference and with the
CPU restatement. Tolerances: states and time steps after N steps 1e-12
relative L2 (the stated FP64 bar); single residuals 1e-10 (see test_oracle.py);
CUDA vs the restatement on identical inputs 1e-12."""
from __future__ import annotations

import os
import tempfile

import numpy as np
import pytest

from conftest import golden_files, load_golden, rel_l2
from oracle import dg_numpy as dn
from oracle import records
from vcp3d_open_b200 import capi, cases, solver

pytestmark = pytest.mark.gpu

TOL_STATE = 1e-12
TOL_RES = 1e-10
TOL_DT = 1e-13
TWO_PI = 6.283185307179586


def _make(spec, compat=True):
    case = cases.build_case(spec)
    prm = solver.make_params(case, metric_compat=compat)
    disc = solver.setup_discretization(case, prm)
    return case, prm, disc, solver.Solver(prm, disc)


@pytest.mark.parametrize("path", golden_files(), ids=os.path.basename)
def test_gpu_matches_reference_fixtures(gpu_available, path):
    g = load_golden(path)
    _, _, _, s = _make(g["spec"])
    try:
        s.set_state(g["sol0"])
        mon = s.residual(monitoring=True, keep_raw=True)
        assert rel_l2(s.get_raw_residual(), g["res_raw"]) < TOL_RES
        assert rel_l2(s.get_residual(), g["res"]) < TOL_RES
        assert mon[6] == pytest.approx(g["monitor"][6], rel=1e-13)
        # Largest eddy viscosity of the volume and face points (0 without a model).
        assert mon[7] == pytest.approx(max(g["monitor"][7], 0.0), rel=1e-10)
        assert s.time_step() == pytest.approx(g["dt0"][0], rel=TOL_DT)
        n = int(g["n_steps"])
        for scheme, key in ((capi.SSPRK3, "ssp"), (capi.LSRK4, "ls")):
            s.set_state(g["sol0"])
            s.residual()
            hist = s.step(n, scheme)
            assert rel_l2(s.get_state(), g[key + "_sol"]) < TOL_STATE
            np.testing.assert_allclose(hist, g[key + "_dt"], rtol=TOL_DT)
    finally:
        s.close()


@pytest.mark.parametrize("compat", [True, False])
@pytest.mark.parametrize("path", golden_files()[:2], ids=os.path.basename)
def test_gpu_matches_restatement_on_identical_inputs(gpu_available, path, compat):
    g = load_golden(path)
    spec = g["spec"]
    K = spec.p + 1
    _, prm, disc, s = _make(spec, compat)
    try:
        d = dn.from_discretization(disc, prm)
        s.set_state(g["sol0"])
        s.residual(keep_raw=True)
        U = g["sol0"].reshape(-1, 5, K, K, K)
        raw, res, _ = dn.residual(U, d, compat=compat)
        # The residual is a small difference of large volume and face terms; the
        # bound is 1e-13 relative to the volume term (summation-order rounding).
        vol = dn.volume_residual(U, d, compat)[0]
        scale = np.linalg.norm(vol.ravel()) / np.linalg.norm(raw.ravel())
        assert rel_l2(s.get_raw_residual(), raw.reshape(g["sol0"].shape)) < 1e-13 * scale
        assert rel_l2(s.get_residual(), res.reshape(g["sol0"].shape)) < 1e-13 * scale
    finally:
        s.close()


def test_config1_vortex_lsrk4_matches_restatement(gpu_available):
    """Config 1 (8^3 p3 curvilinear vortex, CFL 0.5, low-storage RK4): 10 steps."""
    spec = cases.CaseSpec(name="vortex8", kind="vortex", n_elem=(8, 8, 8), p=3)
    case, prm, disc, s = _make(spec)
    try:
        U0 = solver.nodal_to_modal(case, prm)
        s.set_state(U0)
        s.residual()
        hist = s.step(10, capi.LSRK4)
        d = dn.from_discretization(disc, prm)
        K = spec.p + 1
        Un, hn = dn.run(U0.reshape(-1, 5, K, K, K), d, 10, "lsrk4")
        assert rel_l2(s.get_state(), Un.reshape(U0.shape)) < TOL_STATE
        np.testing.assert_allclose(hist, hn, rtol=TOL_DT)
    finally:
        s.close()


@pytest.mark.skipif(not records.have_reference_build(), reason="oracle/_ref not built")
def test_config2_tgv_full_size_matches_reference_build(gpu_available):
    """Config 2 at full size (32^3 elements, p3, perturbed grid): 2 LSRK4 steps vs
    the reference build run on the same files."""
    spec = cases.CaseSpec(name="tgv32", kind="tgv", n_elem=(32, 32, 32), p=3, hi=(TWO_PI,) * 3,
                          mach=0.1, reynolds=1600.0, grid_map="random", grid_amp=0.01, seed=1)
    case, prm, disc, s = _make(spec)
    try:
        s.set_state(solver.nodal_to_modal(case, prm))
        s.residual()
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


def _integrals(U, d: dn.Disc):
    """Volume integrals of the conservative variables (quadrature at the Gauss points)."""
    nE, M = U.shape[0], d.M
    val, _, _, _ = dn.vol_interp(U, d.leg, d.dleg)
    V = val.reshape(nE, 5, -1).transpose(1, 0, 2)
    rho, u, v, w, p, eKin = dn.entropy_to_prim(V)
    rE = p / dn.GM1 + rho * eKin
    JW = d.vol[:, 0] * dn._weights3(d.w).reshape(-1)
    return np.array([np.sum(q * JW) for q in (rho, rho * u, rho * v, rho * w, rE)])


def test_conservation_on_periodic_tgv(gpu_available):
    """Mass, momentum and energy stay constant on a periodic block (up to the
    1e-10 relative tolerance of the element mass-matrix solves)."""
    spec = cases.CaseSpec(name="tgv16", kind="tgv", n_elem=(16, 16, 16), p=3, hi=(TWO_PI,) * 3,
                          mach=0.1, reynolds=1600.0, grid_map="random", grid_amp=0.01, seed=2)
    case, prm, disc, s = _make(spec)
    try:
        d = dn.from_discretization(disc, prm)
        U0 = solver.nodal_to_modal(case, prm)
        K = spec.p + 1
        I0 = _integrals(U0.reshape(-1, 5, K, K, K), d)
        s.set_state(U0)
        s.residual()
        s.step(20, capi.LSRK4)
        I1 = _integrals(s.get_state().reshape(-1, 5, K, K, K), d)
        scale = np.array([I0[0], I0[0] * prm.u_ref, I0[0] * prm.u_ref, I0[0] * prm.u_ref, I0[4]])
        assert np.all(np.abs(I1 - I0) / np.abs(scale) < 1e-10)
    finally:
        s.close()


def test_launch_count_and_graph_reuse(gpu_available):
    g = load_golden(golden_files()[0])
    _, _, _, s = _make(g["spec"])
    try:
        s.set_state(g["sol0"])
        s.residual()
        n0 = s.launch_count
        s.step(2, capi.SSPRK3)
        s.step(2, capi.SSPRK3)
        # dt + start of the step (first stage's update) + 3 x (face fluxes +
        # residual with the next stage's update fused) per step.
        assert s.launch_count - n0 == 4 * 8
    finally:
        s.close()


def test_step_after_set_state_evaluates_the_residual_first(gpu_available):
    """A step right after vcpg_set_state equals residual + step (one extra launch)."""
    g = load_golden(golden_files()[0])
    _, _, _, s = _make(g["spec"])
    try:
        s.set_state(g["sol0"])
        s.residual()
        s.step(2, capi.LSRK4)
        want = s.get_state()
        s.set_state(g["sol0"])
        n0 = s.launch_count
        s.step(2, capi.LSRK4)
        assert s.launch_count - n0 == 2 + 2 * 12
        np.testing.assert_array_equal(s.get_state(), want)
    finally:
        s.close()


@pytest.mark.parametrize("scheme", [capi.LSRK4, capi.SSPRK3])
def test_fused_stage_updates_equal_the_stage_kernels(gpu_available, scheme):
    """The step graph applies each stage's update in the residual kernel's
    epilogue; stepping stage by stage (vcpg_rk_stage, then a residual) gives the
    same states and time steps bit for bit."""
    g = load_golden(golden_files()[0])
    _, _, _, s = _make(g["spec"])
    try:
        s.set_state(g["sol0"])
        s.residual()
        hist = s.step(3, scheme)
        fused = s.get_state()
        s.set_state(g["sol0"])
        s.residual()
        stages = 5 if scheme == capi.LSRK4 else 3
        for n in range(3):
            dt = s.time_step()
            assert dt == hist[n]
            for st in range(stages):
                s.rk_stage(scheme, st, dt)
                s.residual()
        np.testing.assert_array_equal(s.get_state(), fused)
    finally:
        s.close()
