"""The reference's parameter file read by the library (no GPU): parsing,
reference conditions and the initial state of a run from files against the
reference build's own set-up, errors for malformed files and for options
outside the path."""
from __future__ import annotations

import glob
import os

import numpy as np
import pytest

from conftest import load_golden, rel_l2, sync_golden_files, write_sync_case
from oracle import records
from vcp3d_open_b200 import cases, param_file, run, solver

REF_TESTS = os.path.join(records.reference_source_dir(), "test")


@pytest.mark.parametrize("path", sync_golden_files(), ids=os.path.basename)
def test_reference_conditions_and_initial_state(path, tmp_path):
    g = load_golden(path)
    cfg = write_sync_case(g, str(tmp_path))
    pf = param_file.read(cfg)
    assert pf.n_sync == int(g["n_sync"])
    ref = param_file.reference_conditions(pf)
    p_ref, u_ref, rho_ref, mu = g["refcond"]
    assert ref.p_ref == pytest.approx(p_ref, rel=1e-14)
    assert ref.u_ref == pytest.approx(u_ref, rel=1e-14)
    assert ref.rho_ref == pytest.approx(rho_ref, rel=1e-14)
    assert ref.mu_nondim == pytest.approx(mu, rel=1e-13)
    case = run.load_case(pf)
    assert case.spec.bc == g["spec"].bc
    # Several subfaces per face: element ranges, conditions and the subfaces' own
    # prescribed data read back from the file.
    want = g["spec"].subfaces or ()
    got = case.spec.subfaces or ()
    assert [e[:3] for e in got] == [e[:3] for e in want]
    for a, b in zip(got, want):
        if b[3] is not None:
            assert a[3] == pytest.approx(b[3], rel=1e-15)
    params = solver.make_params(case)
    sol0 = solver.nodal_to_modal(case, params)     # host code of the library
    assert rel_l2(sol0, g["sol0"]) < 1e-13


def test_generated_file_round_trip(tmp_path):
    spec = cases.CaseSpec(name="rt", kind="pulse", n_elem=(3, 2, 2), p=2, hi=(3.0, 2.0, 2.0),
                          bc=("inflow_static_nscbc", "outflow_nscbc", "periodic", "periodic",
                              "outflow_nscbc", "outflow_nscbc"), sponge=(0, 1, 0, 0, 1, 1),
                          sponge_sigma=7.5, sponge_alpha=3.0, cml=True, outlet_beta_l=-1.0,
                          riemann="Roe", grid_map="none")
    cfg = cases.write_case(cases.build_case(spec), str(tmp_path))
    pf = param_file.read(cfg)
    param_file.check_supported(pf)
    assert param_file.n_elements(pf) == spec.n_elem
    assert param_file.case_bcs(pf) == spec.bc
    assert pf.sponge == [(s, 7.5, 3.0) for s in spec.sponge]
    assert pf.cml and pf.sponge_layer and pf.riemann == "roe" and pf.outlet_beta_l == -1.0
    ref = cases.reference_conditions(spec)
    assert param_file.outflow_pressure(pf, 1) == pytest.approx(ref.p_ref)
    assert param_file.inflow_static(pf, 0)[0] == pytest.approx(ref.rho_ref)
    case = run.load_case(pf)
    assert case.spec.sponge_state[0] == pytest.approx(ref.rho_ref)
    assert case.spec.sponge_state[4] == pytest.approx(ref.p_ref)


def _base_text():
    return cases.param_cfg_text(cases.CaseSpec(name="b", n_elem=(2, 2, 2), p=2))


def test_unknown_keyword_and_bad_values():
    with pytest.raises(param_file.ParamFileError, match="Unknown keyword"):
        param_file.parse(_base_text() + "\nNot a keyword: 3\n")
    with pytest.raises(param_file.ParamFileError, match="yes or no"):
        param_file.parse(_base_text().replace("Restart: yes", "Restart: maybe"))
    with pytest.raises(param_file.ParamFileError, match="Unknown boundary condition"):
        param_file.parse(_base_text().replace("Periodic1to1Trans", "BCNoSuchThing", 1))
    pf = param_file.parse(_base_text().replace("CFL number: 0.5", "CFL number: -1"))
    with pytest.raises(param_file.ParamFileError, match="CFL"):
        param_file.check_parameters(pf)
    # Comments and tabs as the reference reads them.
    pf = param_file.parse(_base_text().replace("CFL number: 0.5", "CFL number:\t0.75 # c"))
    assert pf.cfl == 0.75


@pytest.mark.parametrize("edit, what", [
    (("Wall modeling: No wall model", "Wall modeling: Logarithmic wall model"), "Wall"),
    (("FEM working variables: Entropy", "FEM working variables: Conservative"), "Conservative"),
    (("Fluctuations to add to initial solution: No fluctuations",
      "Fluctuations to add to initial solution: Random fluctuations"), "(?i)random"),
])
def test_options_outside_the_path(edit, what):
    pf = param_file.parse(_base_text().replace(*edit))
    with pytest.raises(param_file.UnsupportedOption, match=what):
        param_file.check_supported(pf)


def _replace_subface(text, k, line):
    lines = text.split("\n")
    idx = [n for n, ln in enumerate(lines) if ln.strip().startswith("Periodic1to1Trans")]
    lines[idx[k]] = line
    return "\n".join(lines)


def test_boundary_conditions_outside_the_path():
    # The symmetry plane terminates in the reference as well.
    text = _replace_subface(_replace_subface(_base_text(), 2, "  BCSymmetryPlane 1 3 1 1 1 3"),
                            3, "  BCSymmetryPlane 1 3 3 3 1 3")
    with pytest.raises(param_file.UnsupportedOption, match="BCSymmetryPlane"):
        param_file.check_supported(param_file.parse(text))
    # A wall facing a periodic face.
    text = _replace_subface(_base_text(), 0, "        BCWallHeatFlux 1 1 1 3 1 3")
    with pytest.raises(param_file.UnsupportedOption, match="periodic on one face only"):
        param_file.check_supported(param_file.parse(text))


@pytest.mark.skipif(not os.path.isdir(REF_TESTS), reason="reference test cases not present")
def test_reference_own_parameter_files():
    """The reference's own test cases: the NSCBC cases with static and total
    inflow and the duct (walls, subsonic inflow) parse and are supported; the stale n3_10x5x5 file has an
    unknown keyword, which the reference rejects as well."""
    seen = {}
    for path in sorted(glob.glob(os.path.join(REF_TESTS, "**", "*.cfg"), recursive=True)):
        rel = os.path.relpath(path, REF_TESTS)
        try:
            pf = param_file.read(path)
        except param_file.ParamFileError as e:
            seen[rel] = f"error: {e}"
            continue
        try:
            param_file.check_supported(pf)
            seen[rel] = "runs"
        except param_file.UnsupportedOption as e:
            seen[rel] = f"unsupported: {e}"
    assert seen["n3_8x4x4/param_static.cfg"] == "runs"
    assert seen["n3_8x4x4/param_total.cfg"] == "runs"
    assert seen["n5_15x8x8/duct/param.cfg"] == "runs"
    assert "Unknown keyword" in seen["n3_10x5x5/param.cfg"]
