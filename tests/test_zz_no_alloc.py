"""The allocation-free time-step entry point, vcpg_time_step_noalloc.

It serves callers that cannot call cudaMalloc because their device memory all
belongs to their own pool allocator. Here torch plays that pool: it owns the
device copies of the state, the element scalars and the output; the entry
point only reads and writes them and keeps its scratch in the library's static
device array. Its result must equal the time step of the handle-based
vcpg_time_step (the existing entry point) on two calls in a row with
different states, i.e. nothing stale may survive in the shared scratch.

This file is named to be collected last.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from conftest import golden_files, load_golden
from vcp3d_open_b200 import capi, cases, solver

pytestmark = pytest.mark.gpu

TOL_DT = 1e-13   # the tolerance of the time-step parity tests


def _ops(disc):
    keep = [np.ascontiguousarray(a) for a in (disc.leg_int, disc.dleg_int, disc.leg_face,
                                              disc.dleg_face, disc.w_int, disc.leg_dofs,
                                              disc.basis_center)]
    return capi.Operators(*[capi.ptr(a) for a in keep]), keep


def _no_sgs_files():
    """Fixtures without a subgrid-scale model (the entry point runs none)."""
    return [p for p in golden_files() if load_golden(p)["spec"].sgs == "none"]


def _cases():
    """Degree 1 and 4 (the first two) and degree 6 (K = 7, M = 9: the largest
    pair the entry point takes, nearest its static shared-memory limit)."""
    files = _no_sgs_files()
    p6 = [p for p in files if load_golden(p)["spec"].p == 6]
    return files[:2] + p6[:1]


@pytest.mark.parametrize("path", _cases(), ids=os.path.basename)
def test_noalloc_time_step_matches_handle_time_step(gpu_available, path):
    import torch
    g = load_golden(path)
    case = cases.build_case(g["spec"])
    prm = solver.make_params(case)
    disc = solver.setup_discretization(case, prm)
    lib = capi.load()
    ops, keep = _ops(disc)
    s = solver.Solver(prm, disc)
    try:
        # Two states: the initial one and the one after an SSP-RK3 step.
        s.set_state(g["sol0"])
        s.residual()
        dt_a = s.time_step()
        sol_a = s.get_state()
        s.step(1, capi.SSPRK3)
        dt_b = s.time_step()
        sol_b = s.get_state()
        assert dt_a != dt_b

        stream = torch.cuda.current_stream()
        d_sc = torch.from_numpy(np.ascontiguousarray(disc.elem_scalars)).cuda()
        d_dt = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        for sol, dt_ref in ((sol_a, dt_a), (sol_b, dt_b)):
            d_sol = torch.from_numpy(np.ascontiguousarray(sol)).cuda()
            torch.cuda.synchronize()
            rc = lib.vcpg_time_step_noalloc(C.byref(prm), C.byref(ops), d_sol.data_ptr(),
                                            d_sc.data_ptr(), d_dt.data_ptr(), stream.cuda_stream)
            assert rc == capi.VCPG_OK
            assert float(d_dt.item()) == pytest.approx(dt_ref, rel=TOL_DT)
        del keep
    finally:
        s.close()


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu_available):
    import torch
    g = load_golden(_no_sgs_files()[0])
    case = cases.build_case(g["spec"])
    prm = solver.make_params(case)
    disc = solver.setup_discretization(case, prm)
    lib = capi.load()
    ops, keep = _ops(disc)
    big = capi.Params.from_buffer_copy(prm)
    big.n_elem[:] = [65, 64, 64]            # 266,240 > VCPG_NOALLOC_MAX_ELEMS
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = lib.vcpg_time_step_noalloc(C.byref(big), C.byref(ops), d.data_ptr(), d.data_ptr(),
                                    d.data_ptr(), None)
    assert rc == 7  # VCPG_E_ADMISSION: beyond the stated maximum, nothing launched
    assert torch.count_nonzero(d).item() == 0
    del keep


def test_noalloc_reports_a_bad_state_then_recovers(gpu_available):
    """A state whose last entropy variable is positive (no physical pressure:
    a^2 is not a number) gives VCPG_E_NEG_A2; the next call with a valid state
    returns VCPG_OK and the handle's time step, so the status slot of the
    shared scratch is cleared on every call."""
    import torch
    g = load_golden(_no_sgs_files()[0])
    case = cases.build_case(g["spec"])
    prm = solver.make_params(case)
    disc = solver.setup_discretization(case, prm)
    lib = capi.load()
    ops, keep = _ops(disc)
    s = solver.Solver(prm, disc)
    try:
        s.set_state(g["sol0"])
        dt_ref = s.time_step()
    finally:
        s.close()
    K3 = (g["spec"].p + 1) ** 3
    bad = np.array(g["sol0"], dtype=np.float64).reshape(-1, 5, K3)
    bad[3, 4, :] = -bad[3, 4, :]              # V4 = -rho/p > 0 in element 3
    stream = torch.cuda.current_stream()
    d_sc = torch.from_numpy(np.ascontiguousarray(disc.elem_scalars)).cuda()
    d_dt = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    for sol, want in ((bad, capi.VCPG_E_NEG_A2), (g["sol0"], capi.VCPG_OK)):
        d_sol = torch.from_numpy(np.ascontiguousarray(sol)).cuda()
        torch.cuda.synchronize()
        rc = lib.vcpg_time_step_noalloc(C.byref(prm), C.byref(ops), d_sol.data_ptr(),
                                        d_sc.data_ptr(), d_dt.data_ptr(), stream.cuda_stream)
        assert rc == want
    assert float(d_dt.item()) == pytest.approx(dt_ref, rel=TOL_DT)
    del keep
