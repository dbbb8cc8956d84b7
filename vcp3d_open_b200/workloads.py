"""Named synthetic workloads of the benchmark, the precision report and the tests.

Every workload is a seeded, generated case (vcp3d_open_b200.cases): there is no
grid or restart file to download. The Taylor-Green cases use Re 1600 and
Mach 0.1 on the periodic box [0, 2pi]^3 with a +-1% random node perturbation
(curvilinear elements, so the full metric terms are exercised).
"""
from __future__ import annotations

from .cases import CaseSpec

TWO_PI = 6.283185307179586

_TGV = dict(kind="tgv", hi=(TWO_PI,) * 3, mach=0.1, reynolds=1600.0, grid_map="random",
            grid_amp=0.01, seed=1)

WORKLOADS = {
    # Headline: 32^3 elements of degree 3, 2,097,152 DOFs.
    "tgv32_p3_lsrk4": dict(_TGV, n_elem=(32, 32, 32), p=3),
    # Isentropic vortex, 8^3 elements of degree 3 (the reference's own test case shape).
    "vortex8_p3_lsrk4": dict(kind="vortex", n_elem=(8, 8, 8), p=3),
    # Degree 4 on 48^3 elements (13.8M DOFs): the mixed-precision configuration's size.
    "tgv48_p4_lsrk4": dict(_TGV, n_elem=(48, 48, 48), p=4),
    # Profiling size: state + metrics ~200 MB (above the 126 MB L2), 8000 elements.
    "tgv20_p3_lsrk4": dict(_TGV, n_elem=(20, 20, 20), p=3),
    # The reference's high degrees: p6 with a 16th-order rule (M = 9, 1.4M DOFs) and
    # p9 with the default rule (M = 14, 1.7M DOFs); their element arrays exceed one
    # CTA's shared memory from p7 on. A smooth sine map of amplitude 0.05 curves
    # the grid (random node moves give the closely spaced nodes of these degrees
    # non-positive Jacobians, which the reference rejects).
    "tgv16_p6_lsrk4": dict(_TGV, n_elem=(16, 16, 16), p=6, n_poly_int=16, grid_map="sine",
                           grid_amp=0.05),
    "tgv12_p9_lsrk4": dict(_TGV, n_elem=(12, 12, 12), p=9, grid_map="sine", grid_amp=0.05),
    # Degrees 2 and 5 (the other degrees of the served ensemble's cases): 40^3 elements
    # of degree 2 (1.7M DOFs) and 24^3 of degree 5 (3.0M DOFs).
    "tgv40_p2_lsrk4": dict(_TGV, n_elem=(40, 40, 40), p=2),
    "tgv24_p5_lsrk4": dict(_TGV, n_elem=(24, 24, 24), p=5),
    # Degree 4 on 16^3 elements: the mixed-versus-FP64 test case (fits a test's time).
    "tgv16_p4_lsrk4": dict(_TGV, n_elem=(16, 16, 16), p=4),
    # Acoustic pulse with open boundaries: [0,20]x[0,10]x[0,10], 40x20x20 elements of
    # degree 4 (2,000,000 DOFs), pressure pulse 1e-3 of width 0.5 at (10, 5, 5) in a
    # Mach 0.3 stream along x; static-inflow PC-NSCBC on i-min, outflow PC-NSCBC
    # (sigma 0.25, L 1, beta_l = beta_t = 0.5, (1 - beta) form, boundary-averaged
    # Mach) on i-max and both j faces, sponge layers of 4 (i-max) and 3 (j faces)
    # elements with the matching layer, k periodic.
    "pulse40_p4_lsrk4": dict(kind="pulse", n_elem=(40, 20, 20), p=4, hi=(20.0, 10.0, 10.0),
                             mach=0.3, grid_map="none", center=(10.0, 5.0, 5.0),
                             pulse_amp=1.0e-3, pulse_width=0.5,
                             bc=("inflow_static_nscbc", "outflow_nscbc", "outflow_nscbc",
                                 "outflow_nscbc", "periodic", "periodic"),
                             sponge=(0, 4, 3, 3, 0, 0), cml=True),
    # Profiling size of the open-boundary configuration: 24x12x12 elements of degree 4
    # on [0,12]x[0,6]x[0,6] (state + metrics ~260 MB, above the 126 MB L2).
    "pulse24_p4_lsrk4": dict(kind="pulse", n_elem=(24, 12, 12), p=4, hi=(12.0, 6.0, 6.0),
                             mach=0.3, grid_map="none", center=(6.0, 3.0, 3.0),
                             pulse_amp=1.0e-3, pulse_width=0.5,
                             bc=("inflow_static_nscbc", "outflow_nscbc", "outflow_nscbc",
                                 "outflow_nscbc", "periodic", "periodic"),
                             sponge=(0, 3, 2, 2, 0, 0), cml=True),
}


def make_spec(name: str) -> CaseSpec:
    if name not in WORKLOADS:
        raise KeyError(f"unknown workload {name!r}; known: {sorted(WORKLOADS)}")
    return CaseSpec(name=name, **WORKLOADS[name])
