"""Runs from the reference's input files on the GPU (vcp3d_open_b200.run):
synchronisation steps against the reference main program's own loop on the
same files, the written restart files, the mixed form and the command line."""
from __future__ import annotations

import dataclasses
import os
import re

import numpy as np
import pytest

from conftest import assert_forces_match, load_golden, rel_l2, sync_golden_files, write_sync_case
from vcp3d_open_b200 import capi, cases, param_file, run, solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", sync_golden_files(), ids=os.path.basename)
def test_synchronization_steps_match_reference(gpu_available, path, tmp_path):
    g = load_golden(path)
    cfg = write_sync_case(g, str(tmp_path))
    res = run.run(cfg, write=True, out=open(os.devnull, "w"))
    assert rel_l2(res.state, g["sync_sol"]) < 1e-12
    assert res.rk_steps == int(g["rk_steps"][0])
    n, _, mach, _ = res.history[-1]
    assert n == int(g["n_sync"])
    assert mach ** 2 == pytest.approx(float(g["monitor"][6]), rel=1e-10)
    pf = param_file.read(cfg)
    assert_forces_match(res.monitoring, g["monitor"],
                        dataclasses.replace(g["spec"], monitor_forces=pf.monitor_forces,
                                            ref_area=pf.reference_area))
    # The restart files: the initial state and the final one, as the reference
    # writes them (dimensional conservative variables at the nodal DOFs).
    pf = param_file.read(cfg)
    case = run.load_case(pf)
    params = solver.make_params(case)
    disc = solver.setup_discretization(case, params)
    assert len(res.files) == 2 and res.files[-1].endswith(f"_TimeStep_{int(g['n_sync'])}")
    xyz, cons = cases.read_su2_restart(res.files[-1], case.dof_xyz.shape[0], case.dof_xyz.shape[2])
    assert np.array_equal(xyz, case.dof_xyz)
    expect = run.modal_to_nodal_conservative(case, disc, g["sync_sol"])
    assert rel_l2(cons, expect) < 1e-12
    _, cons0 = cases.read_su2_restart(res.files[0], case.dof_xyz.shape[0], case.dof_xyz.shape[2])
    assert rel_l2(cons0, case.cons) < 1e-13


@pytest.mark.parametrize("path", sync_golden_files(), ids=os.path.basename)
def test_mixed_form_from_files(gpu_available, path, tmp_path):
    g = load_golden(path)
    cfg = write_sync_case(g, str(tmp_path))
    res = run.run(cfg, precision=capi.MIXED, write=False, out=open(os.devnull, "w"))
    assert rel_l2(res.state, g["sync_sol"]) < 1e-6


def test_command_line(gpu_available, tmp_path):
    g = load_golden(sync_golden_files()[0])
    cfg = write_sync_case(g, str(tmp_path))
    assert run.main([cfg, "--steps", "1", "--no-write"]) == 0
    with open(cfg) as f:
        text = f.read()
    with open(cfg, "w") as f:
        f.write(re.sub(r"(?m)^Fluctuations to add to initial solution:.*$",
                       "Fluctuations to add to initial solution: Random fluctuations", text))
    assert run.main([cfg, "--no-write"]) == 3
