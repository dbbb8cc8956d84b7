"""The CPU restatement (oracle/dg_numpy.py) against the golden fixtures made by
the reference solver itself; and the reference build against its fixtures."""
from __future__ import annotations

import os
import tempfile

import numpy as np
import pytest

from conftest import golden_files, load_golden, rel_l2
from oracle import dg_numpy as dn
from oracle import records
from vcp3d_open_b200 import cases, solver

# Tolerances (FP64): states after N steps and time steps are compared at the
# stated FP64 bar of 1e-12 relative L2; single residuals carry the ~1e-14
# relative differences of independently computed metric terms, amplified by
# the cancellation inside the residual, so they are held to 1e-10.
TOL_STATE = 1e-12
TOL_RES = 1e-10
TOL_DT = 1e-13


def _disc(spec):
    case = cases.build_case(spec)
    prm = solver.make_params(case)
    return case, prm, dn.from_discretization(solver.setup_discretization(case, prm), prm)


@pytest.mark.parametrize("path", golden_files(), ids=os.path.basename)
def test_restatement_matches_reference_fixtures(path):
    g = load_golden(path)
    spec = g["spec"]
    K = spec.p + 1
    _, _, d = _disc(spec)
    U = g["sol0"].reshape(-1, 5, K, K, K)
    raw, res, iters = dn.residual(U, d)
    assert rel_l2(raw.reshape(g["res_raw"].shape), g["res_raw"]) < TOL_RES
    assert rel_l2(res.reshape(g["res"].shape), g["res"]) < TOL_RES
    assert 1 <= iters.max() < 100
    assert abs(dn.time_step(U, d) / g["dt0"][0] - 1.0) < TOL_DT
    n = int(g["n_steps"])
    for scheme, key in (("ssprk3", "ssp"), ("lsrk4", "ls")):
        Un, hist = dn.run(U, d, n, scheme)
        assert rel_l2(Un.reshape(g[key + "_sol"].shape), g[key + "_sol"]) < TOL_STATE
        assert np.max(np.abs(hist / g[key + "_dt"] - 1.0)) < TOL_DT


def test_restatement_metric_index_modes_differ_on_curved_grid():
    """The reference's metric indexing is reproduced only in compat mode; on a
    curvilinear grid the two modes give measurably different residuals."""
    g = load_golden(golden_files()[-1])
    spec = g["spec"]
    K = spec.p + 1
    _, _, d = _disc(spec)
    U = g["sol0"].reshape(-1, 5, K, K, K)
    a = dn.residual(U, d, compat=True)[0]
    b = dn.residual(U, d, compat=False)[0]
    assert rel_l2(b, a) > 1e-9
    assert rel_l2(a.reshape(g["res_raw"].shape), g["res_raw"]) < TOL_RES


@pytest.mark.skipif(not records.have_reference_build(), reason="oracle/_ref not built")
def test_reference_build_reproduces_fixture():
    """Pins the fixtures to the current reference build (bit-for-bit level)."""
    path = [p for p in golden_files() if "vortex_p2" in p][0]
    g = load_golden(path)
    K = g["spec"].p + 1
    with tempfile.TemporaryDirectory() as tmp:
        cfg = cases.write_case(cases.build_case(g["spec"]), tmp)
        out = os.path.join(tmp, "r.bin")
        records.run_reference(cfg, "residual", out)
        r = records.read_records(out)
    assert rel_l2(r["res"][:, :, :K ** 3], g["res"]) < 1e-15
    assert r["dt"][0] == pytest.approx(g["dt0"][0], rel=1e-15)


@pytest.mark.parametrize("model", [dn.SGS_WALE, dn.SGS_VREMAN])
def test_eddy_viscosity_vanishes_in_pure_shear_and_scales_with_length(model):
    """Both models are built to give no eddy viscosity in a pure shear flow;
    both scale with the square of the length scale."""
    rng = np.random.default_rng(5)
    n = 64
    rho = 1.0 + rng.random(n)
    z = np.zeros(n)
    shear = rng.standard_normal(n)
    G = [[z, shear, z], [z, z, z], [z, z, z]]
    assert np.all(dn.eddy_viscosity(model, 0.1, rho, G) < 1e-12 * np.abs(shear).max())
    G = [[rng.standard_normal(n) for _ in range(3)] for _ in range(3)]
    a = dn.eddy_viscosity(model, 0.1, rho, G)
    b = dn.eddy_viscosity(model, 0.2, rho, G)
    assert np.all(a > 0.0)
    np.testing.assert_allclose(b, 4.0 * a, rtol=1e-13)
