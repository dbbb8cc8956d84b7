"""Host-side parts of the library that run without a GPU: the exported C ABI,
argument checking, the set-up (operators, metrics) and the state conversion,
checked against the reference's own values in the golden fixtures."""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden_files, load_golden, open_golden_files, rel_l2
from vcp3d_open_b200 import capi, cases, solver


def header_symbols():
    text = open(os.path.join(ROOT, "include", "vcp3d_b200.h")).read()
    return sorted(set(re.findall(r"\b(vcpg_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    declared = header_symbols()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(capi.EXPORTED) == declared


def test_create_rejects_bad_arguments_without_touching_the_device():
    lib = capi.load()
    h = C.c_void_p()
    assert lib.vcpg_create(None, None, None, C.byref(h)) == 8
    p = capi.Params()
    p.n_elem[:] = [2, 2, 2]
    p.n_poly, p.n_int_1d = 3, 7          # (K, M) = (4, 7) has no kernel
    ops, geo = capi.Operators(), capi.Geometry()
    rc = lib.vcpg_create(C.byref(p), C.byref(ops), C.byref(geo), C.byref(h))
    assert rc == 6
    assert b"no kernel" in lib.vcpg_last_error(h)
    lib.vcpg_destroy(h)
    p.n_poly, p.n_int_1d = 3, 5
    p.precision = 7                      # neither VCPG_FP64 nor VCPG_MIXED
    rc = lib.vcpg_create(C.byref(p), C.byref(ops), C.byref(geo), C.byref(h))
    assert rc == 8
    assert b"precision" in lib.vcpg_last_error(h)
    lib.vcpg_destroy(h)
    assert lib.vcpg_step(None, 0, 1, -1.0, None) == 8


@pytest.mark.parametrize("path", golden_files() + open_golden_files(), ids=os.path.basename)
def test_setup_matches_reference_metrics(path):
    g = load_golden(path)
    spec = g["spec"]
    case = cases.build_case(spec)
    prm = solver.make_params(case)
    disc = solver.setup_discretization(case, prm)
    ref = g["refcond"]
    np.testing.assert_allclose([prm.p_ref, prm.u_ref, prm.rho_ref, prm.mu], ref, rtol=1e-14)
    assert rel_l2(disc.vol_metric[0], g["vol_metric_e0"]) < 1e-13
    assert rel_l2(disc.face_metric[0], g["face_metric_e0"]) < 1e-13
    sums = [np.abs(disc.vol_metric).sum()] + [np.abs(disc.face_metric[:, f]).sum()
                                              for f in range(6)] + [np.abs(disc.elem_scalars).sum()]
    np.testing.assert_allclose(sums, g["metric_sums"], rtol=1e-12)
    assert rel_l2(disc.elem_scalars, g["elem_scalars"]) < 1e-13
    # Initial state: the library's nodal -> modal conversion vs the reference's restart read.
    modal = solver.nodal_to_modal(case, prm)
    assert rel_l2(modal, g["sol0"]) < 1e-14


def test_neighbour_table_is_periodic_and_symmetric():
    spec = cases.CaseSpec(kind="uniform", n_elem=(3, 2, 4), p=2, grid_map="none")
    case = cases.build_case(spec)
    prm = solver.make_params(case)
    disc = solver.setup_discretization(case, prm)
    nbr = disc.neighbors
    nE = spec.n_elements
    for e in range(nE):
        for d in range(3):
            assert nbr[nbr[e, 2 * d], 2 * d + 1] == e
            assert nbr[nbr[e, 2 * d + 1], 2 * d] == e
    # Non-periodic direction: boundary faces are marked -1.
    disc2 = solver.setup_discretization(case, prm, periodic=(1, 0, 1))
    assert (disc2.neighbors[:, 2] == -1).sum() == 3 * 4
    assert (disc2.neighbors[:, 3] == -1).sum() == 3 * 4
