"""Config 1 at its stated length against the reference build: the isentropic
vortex on the curvilinear 8^3 grid of degree 3, 100 time steps of low-storage
RK4 and of SSP-RK3 at CFL 0.5 from the same files, GPU (FP64) and the
reference build (oracle/_ref, the host's threads). The states after 100 steps
agree to 1e-12 relative L2 and every step's Delta t to 1e-12. The conserved
integrals drift by ~1e-10 of their scales over 100 steps in both runs (the
mass-matrix solves stop at 1e-10 relative, so the projected residual conserves
only to that level); the GPU's drift equals the reference's to 1e-12."""
from __future__ import annotations

import pytest

import long_horizon
from oracle import records

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not records.have_reference_build(),
                                 reason="oracle/_ref not built")]

TOL_STATE = 1e-12
TOL_DT = 1e-12


@pytest.mark.parametrize("scheme", ["lsrk4", "ssprk3"])
def test_config1_vortex_100_steps_matches_reference_build(gpu_available, scheme):
    rep = long_horizon.run("vortex", steps=100, every=50, scheme=scheme)
    rows = rep["rows"][1:]
    assert [r["step"] for r in rows] == [50, 100]
    for r in rows:
        assert r["rel_l2_state_gpu_vs_reference"] < TOL_STATE, r
        assert r["max_rel_dt_diff"] < TOL_DT, r
        assert max(abs(x) for x in r["reference_drift"]) < 1e-9, r
        assert max(abs(a - b) for a, b in zip(r["gpu_drift"], r["reference_drift"])) < 1e-12, r
