"""Generates the golden fixtures under tests/golden/ by running the reference
solver itself (oracle/_ref/vcp3d_ref, built from the reference sources by
oracle/Makefile) on small generated cases.

    make -C oracle && python tests/golden/make_golden.py

Each fixture case_<name>.npz (periodic blocks) or open_<name>.npz (blocks with
characteristic boundaries, sponge and matching layers) holds, for one case:
  spec_json       the CaseSpec (JSON) that regenerates grid and initial state
  sol0            initial modal entropy-variable state [nE][5][K^3] (reference's
                  own restart-file conversion)
  res_raw, res    residual before / after the mass-matrix solve of sol0
  monitor         the 8 monitoring values of that residual
  dt0             CFL time step of sol0
  ssp_sol, ssp_dt state and time steps after N_STEPS SSP-RK3 steps
  ls_sol, ls_dt   state and time steps after N_STEPS low-storage RK4 steps
  metric_sums     per-array checksums of the reference's metric terms
  vol_metric_e0, face_metric_e0  metric terms of element 0 (unpadded)

Each sync_<name>.npz holds a case run through the reference main program's
loop of synchronisation steps from its parameter file (param_text, with the
grid and restart / averaged-solution files that write_case generates from
spec_json): sol0 (initial modal state after the fluctuations), refcond,
sync_sol (state after n_sync synchronisation steps), monitor and rk_steps
(Runge-Kutta steps taken).
"""
from __future__ import annotations

import dataclasses
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import records  # noqa: E402
from vcp3d_open_b200 import cases  # noqa: E402

N_STEPS = 3
TWO_PI = 6.283185307179586

GOLDEN_SPECS = {
    # Isentropic vortex on the curvilinear periodic cube (config 1 family), reduced.
    "vortex_p3_4x4x4": cases.CaseSpec(name="vortex_p3_4x4x4", kind="vortex", n_elem=(4, 4, 4),
                                      p=3),
    # Taylor-Green vortex, perturbed grid, degree 4 (config 3/4 family), reduced.
    "tgv_p4_3x3x3": cases.CaseSpec(name="tgv_p4_3x3x3", kind="tgv", n_elem=(3, 3, 3), p=4,
                                   hi=(TWO_PI,) * 3, mach=0.1, reynolds=1600.0,
                                   grid_map="random", grid_amp=0.01, seed=1),
    # Degree 2 with the Roe flux, anisotropic block.
    "vortex_p2_roe_4x3x2": cases.CaseSpec(name="vortex_p2_roe_4x3x2", kind="vortex",
                                          n_elem=(4, 3, 2), p=2, riemann="Roe",
                                          hi=(10.0, 7.5, 5.0), center=(5.0, 3.75, 2.5)),
    # Degree 5.
    "tgv_p5_2x2x2": cases.CaseSpec(name="tgv_p5_2x2x2", kind="tgv", n_elem=(2, 2, 2), p=5,
                                   hi=(TWO_PI,) * 3, mach=0.1, reynolds=1600.0,
                                   grid_map="random", grid_amp=0.01, seed=3),
    # The other degrees of the reference's tensor-product dispatch: p1 (M = 2),
    # p6 with a 16th-order rule (M = 9), p7 with a 22nd-order rule (M = 12), p8
    # and p9 with the default rule (M = 13, 14).
    "tgv_p1_4x4x4": cases.CaseSpec(name="tgv_p1_4x4x4", kind="tgv", n_elem=(4, 4, 4), p=1,
                                   hi=(TWO_PI,) * 3, mach=0.1, reynolds=1600.0,
                                   grid_map="random", grid_amp=0.01, seed=21),
    "tgv_p6_2x2x2": cases.CaseSpec(name="tgv_p6_2x2x2", kind="tgv", n_elem=(2, 2, 2), p=6,
                                   n_poly_int=16, hi=(TWO_PI,) * 3, mach=0.1, reynolds=1600.0,
                                   grid_map="random", grid_amp=0.005, seed=22),
    "vortex_p7_2x2x2": cases.CaseSpec(name="vortex_p7_2x2x2", kind="vortex", n_elem=(2, 2, 2),
                                      p=7, n_poly_int=22, beta=2.0),
    "tgv_p8_2x2x2": cases.CaseSpec(name="tgv_p8_2x2x2", kind="tgv", n_elem=(2, 2, 2), p=8,
                                   hi=(TWO_PI,) * 3, mach=0.1, reynolds=1600.0,
                                   grid_map="random", grid_amp=0.005, seed=23),
    "tgv_p9_2x2x2_roe": cases.CaseSpec(name="tgv_p9_2x2x2_roe", kind="tgv", n_elem=(2, 2, 2),
                                       p=9, riemann="Roe", hi=(TWO_PI,) * 3, mach=0.1,
                                       reynolds=1600.0, grid_map="sine", grid_amp=0.05),
    # Equidistant solution DOFs on the LGL grid.
    "vortex_p3_4x3x3_equi": cases.CaseSpec(name="vortex_p3_4x3x3_equi", kind="vortex",
                                           n_elem=(4, 3, 3), p=3, hi=(10.0, 7.5, 7.5),
                                           center=(5.0, 3.75, 3.75), dof_location="equidistant"),
    # A body force per unit volume (N/m^3) on the isentropic vortex, degree 3.
    "vortex_p3_4x4x2_body": cases.CaseSpec(name="vortex_p3_4x4x2_body", kind="vortex",
                                           n_elem=(4, 4, 2), p=3, hi=(10.0, 10.0, 5.0),
                                           center=(5.0, 5.0, 2.5), seed=15,
                                           body_force=(2.0, -1.0, 0.5)),
    # WALE subgrid-scale model, Taylor-Green vortex at a high Reynolds number on a
    # perturbed grid, degree 4.
    "tgv_p4_3x3x3_wale": cases.CaseSpec(name="tgv_p4_3x3x3_wale", kind="tgv", n_elem=(3, 3, 3),
                                        p=4, hi=(TWO_PI,) * 3, mach=0.1, reynolds=1.0e5,
                                        grid_map="random", grid_amp=0.005, seed=11, sgs="wale"),
    # WALE at degree 9 (the time step's model arrays in global scratch).
    "tgv_p9_2x2x2_wale": cases.CaseSpec(name="tgv_p9_2x2x2_wale", kind="tgv", n_elem=(2, 2, 2),
                                        p=9, hi=(TWO_PI,) * 3, mach=0.1, reynolds=1.0e5,
                                        grid_map="sine", grid_amp=0.05, sgs="wale"),
    # Vreman model, isentropic vortex, degree 3, Roe flux, anisotropic block.
    "vortex_p3_4x3x3_vreman": cases.CaseSpec(name="vortex_p3_4x3x3_vreman", kind="vortex",
                                             n_elem=(4, 3, 3), p=3, riemann="Roe",
                                             hi=(10.0, 7.5, 7.5), center=(5.0, 3.75, 3.75),
                                             reynolds=1.0e5, seed=12, sgs="vreman"),
}


_OPEN = dict(kind="pulse", mach=0.3, grid_map="random", grid_amp=0.01, pulse_amp=1.0e-2,
             pulse_width=0.5)

OPEN_SPECS = {
    # Static inflow (i-min), outflow on i-max and both j faces with sponge layers and
    # the matching layer, k periodic: the config-3 boundary set on a reduced block.
    # The pulses of the open cases sit next to a boundary so that the boundary
    # terms carry a large part of the residual.
    "pulse_p3_6x4x2_sponge_cml": cases.CaseSpec(
        name="pulse_p3_6x4x2_sponge_cml", n_elem=(6, 4, 2), p=3, hi=(6.0, 4.0, 2.0),
        center=(5.2, 0.8, 1.0), seed=4,
        bc=("inflow_static_nscbc", "outflow_nscbc", "outflow_nscbc", "outflow_nscbc",
            "periodic", "periodic"), sponge=(0, 2, 1, 1, 0, 0), cml=True, **_OPEN),
    # Degree 4, Roe flux, inflow / outflow in i only, inlet keeping the outgoing
    # acoustic amplitudes; j and k periodic; no sponge.
    "pulse_p4_4x3x2_roe": cases.CaseSpec(
        name="pulse_p4_4x3x2_roe", n_elem=(4, 3, 2), p=4, hi=(4.0, 3.0, 2.0),
        center=(0.6, 1.5, 1.0), riemann="Roe", seed=5, inlet_incoming=True,
        bc=("inflow_static_nscbc", "outflow_nscbc", "periodic", "periodic", "periodic",
            "periodic"), **_OPEN),
    # Outflow on the k faces, Mach-averaged transverse relaxation (beta < 0) without
    # the (1 - beta) form, sponge only on k-max, flow along z.
    "pulse_p3_3x3x4_kfaces": cases.CaseSpec(
        name="pulse_p3_3x3x4_kfaces", n_elem=(3, 3, 4), p=3, hi=(3.0, 3.0, 4.0),
        center=(1.5, 1.5, 0.7), vel_dir=(0.0, 0.0, 1.0), seed=6, outlet_beta_l=-1.0,
        outlet_beta_t=-1.0, outlet_one_minus_beta=False,
        bc=("periodic", "periodic", "periodic", "periodic", "inflow_static_nscbc",
            "outflow_nscbc"), sponge=(0, 0, 0, 0, 0, 1), **_OPEN),
    # The same with "Outlet use local (element) averaged Mach number": every outlet
    # face takes the projected Mach number averaged over the last outlet element's
    # face (the value the reference's subface member holds after its averaging loop).
    "pulse_p3_3x3x4_kfaces_local": cases.CaseSpec(
        name="pulse_p3_3x3x4_kfaces_local", n_elem=(3, 3, 4), p=3, hi=(3.0, 3.0, 4.0),
        center=(1.5, 1.5, 3.3), vel_dir=(0.0, 0.0, 1.0), seed=16, outlet_beta_l=-1.0,
        outlet_beta_t=-1.0, outlet_one_minus_beta=False, outlet_local_mach=True,
        bc=("periodic", "periodic", "periodic", "periodic", "inflow_static_nscbc",
            "outflow_nscbc"), sponge=(0, 0, 0, 0, 0, 1), **_OPEN),
    # Total-condition inflow (relaxing total pressure, total temperature and the
    # flow direction) with the outgoing amplitude kept, outflow on i-max with a
    # sponge and the matching layer, flow at an angle in the x-y plane.
    "pulse_p3_5x3x2_total": cases.CaseSpec(
        name="pulse_p3_5x3x2_total", n_elem=(5, 3, 2), p=3, hi=(5.0, 3.0, 2.0),
        center=(0.7, 1.5, 1.0), vel_dir=(1.0, 0.25, 0.0), seed=7, inlet_incoming=True,
        bc=("inflow_total_nscbc", "outflow_nscbc", "periodic", "periodic", "periodic",
            "periodic"), sponge=(0, 1, 0, 0, 0, 0), cml=True, **_OPEN),
    # Walls through a boundary state: a heat-flux wall with a non-zero flux on j-min,
    # an isothermal wall on j-max, flow along the walls; i and k periodic.
    "wall_p3_4x3x3": cases.CaseSpec(
        name="wall_p3_4x3x3", n_elem=(4, 3, 3), p=3, hi=(4.0, 3.0, 3.0), center=(2.0, 0.6, 1.5),
        seed=8, wall_data=(0.0, 0.0, 50.0, 300.0, 0.0, 0.0), monitor_forces=True,
        bc=("periodic", "periodic", "wall_heat_flux", "wall_isothermal", "periodic",
            "periodic"), **_OPEN),
    # Subsonic inflow (total conditions) and outflow (back pressure) through a
    # boundary state, inviscid walls on the j faces, k periodic.
    "subsonic_p3_5x3x2": cases.CaseSpec(
        name="subsonic_p3_5x3x2", n_elem=(5, 3, 2), p=3, hi=(5.0, 3.0, 2.0),
        center=(0.8, 1.5, 1.0), seed=9, monitor_forces=True, ref_area=2.5,
        bc=("inflow_subsonic", "outflow_subsonic", "wall_inviscid", "wall_inviscid", "periodic",
            "periodic"), **_OPEN),
    # Supersonic inflow / outflow states and far field on the j faces, Roe flux, degree 2.
    "farfield_p2_4x4x2_roe": cases.CaseSpec(
        name="farfield_p2_4x4x2_roe", n_elem=(4, 4, 2), p=2, hi=(4.0, 4.0, 2.0),
        center=(2.0, 3.3, 1.0), seed=10, riemann="Roe",
        bc=("inflow_supersonic", "outflow_supersonic", "farfield", "farfield", "periodic",
            "periodic"), **_OPEN),
    # Degree 7 (M = 12, element arrays in global scratch): static inflow and
    # characteristic outflow with a sponge layer and the matching layer, far field
    # on the j faces, k periodic, uniform grid.
    "pulse_p7_3x2x2": cases.CaseSpec(
        name="pulse_p7_3x2x2", n_elem=(3, 2, 2), p=7, n_poly_int=22, hi=(3.0, 2.0, 2.0),
        center=(2.4, 1.0, 1.0), sponge=(0, 1, 0, 0, 0, 0), cml=True,
        bc=("inflow_static_nscbc", "outflow_nscbc", "farfield", "farfield", "periodic",
            "periodic"), **dict(_OPEN, grid_map="none")),
    # WALE model with walls (isothermal on j-min, heat flux on j-max), static inflow
    # and characteristic outflow in i with a sponge layer, k periodic, degree 4; an
    # isentropic vortex next to the isothermal wall gives the wall faces velocity
    # gradients and so an eddy viscosity.
    "wale_p4_4x3x2_walls": cases.CaseSpec(
        name="wale_p4_4x3x2_walls", n_elem=(4, 3, 2), p=4, hi=(4.0, 3.0, 2.0),
        center=(1.5, 0.7, 1.0), seed=13, reynolds=1.0e5, sgs="wale", monitor_forces=True,
        wall_data=(0.0, 0.0, 310.0, 20.0, 0.0, 0.0), sponge=(0, 1, 0, 0, 0, 0),
        bc=("inflow_static_nscbc", "outflow_nscbc", "wall_isothermal", "wall_heat_flux",
            "periodic", "periodic"), **dict(_OPEN, kind="vortex", beta=2.0)),
    # Several subfaces per block face: i-min holds a static-inflow patch (j < 2)
    # beside an isothermal wall (j >= 2); i-max a characteristic outflow (j < 3,
    # its Mach average over the block face's characteristic faces divided by the
    # area of the whole face) beside a heat-flux wall; far field on the j faces,
    # sponge with the matching layer on i-max, k periodic; forces monitored.
    "subfaces_p3_4x4x2": cases.CaseSpec(
        name="subfaces_p3_4x4x2", n_elem=(4, 4, 2), p=3, hi=(4.0, 4.0, 2.0),
        center=(3.2, 1.2, 1.0), seed=15, monitor_forces=True, sponge=(0, 1, 0, 0, 0, 0),
        cml=True, wall_data=(330.0, 25.0, 0.0, 0.0, 0.0, 0.0),
        bc=("inflow_static_nscbc", "outflow_nscbc", "farfield", "farfield", "periodic",
            "periodic"),
        subfaces=((0, (0, 2, 0, 2), "inflow_static_nscbc"), (0, (2, 4, 0, 2), "wall_isothermal"),
                  (1, (0, 3, 0, 2), "outflow_nscbc"), (1, (3, 4, 0, 2), "wall_heat_flux")),
        **_OPEN),
    # Vreman model with the subsonic inflow / outflow states and far field, a
    # vortex next to the j-max far field.
    "vreman_p3_4x4x2_farfield": cases.CaseSpec(
        name="vreman_p3_4x4x2_farfield", n_elem=(4, 4, 2), p=3, hi=(4.0, 4.0, 2.0),
        center=(2.0, 3.3, 1.0), seed=14, reynolds=1.0e5, sgs="vreman",
        bc=("inflow_subsonic", "outflow_subsonic", "farfield", "farfield", "periodic",
            "periodic"), **dict(_OPEN, kind="vortex", beta=2.0)),
}


# Synchronisation steps through the reference main program's loop
# (ExecuteTimeSynchronizationStep): (spec, parameter-file overrides, steps).
# The vortex restarts from the generated restart file; the open case starts
# from the free stream that the prescribed boundary data define, with the
# pressure-pulse fluctuation of the parameter file.
SYNC_SPECS = {
    "vortex_p3_4x4x4": (GOLDEN_SPECS["vortex_p3_4x4x4"],
                        {"Synchronization time step": "1.0e-4"}, 3),
    # Vreman model at degree 3: the reference's synchronisation step sizes its
    # nodal SGS buffers by the unpadded DOF count and fills them up to the padded
    # count, which stays inside the buffers only where the two agree (K^3 a
    # multiple of the padding, as for degree 3).
    "vortex_p3_4x3x3_vreman": (GOLDEN_SPECS["vortex_p3_4x3x3_vreman"],
                               {"Synchronization time step": "2.0e-4"}, 2),
    # Equidistant solution DOFs of degree 5 (K^3 a multiple of the padding, see
    # above), from the restart file at those DOFs, with the parameter file's
    # pressure pulse.
    "vortex_p5_equi": (cases.CaseSpec(
        name="vortex_p5_equi", kind="vortex", n_elem=(3, 3, 2), p=5, hi=(10.0, 10.0, 6.0),
        center=(5.0, 5.0, 3.0), beta=2.0, dof_location="equidistant"),
        {"Synchronization time step": "2.0e-4",
         "Fluctuations to add to initial solution": "Pressure pulse",
         "Pressure pulse center": "4.0 5.0 3.0", "Pressure pulse strength": "1.0e-2",
         "Pressure pulse width": "1.0"}, 2),
    "pulse_p3_6x4x2_sponge_cml": (OPEN_SPECS["pulse_p3_6x4x2_sponge_cml"],
                                  {"Synchronization time step": "5.0e-5", "Restart": "no",
                                   "Fluctuations to add to initial solution": "Pressure pulse",
                                   "Pressure pulse center": "5.2 0.8 1.0",
                                   "Pressure pulse strength": "1.0e-2",
                                   "Pressure pulse width": "0.5"}, 2),
    # Several subfaces per face from the parameter file, each with its own data:
    # i-min a static inflow beside an isothermal wall at 320 K, i-max two
    # characteristic outflows at different pressures, far field on the j faces.
    "subfaces_p3_4x4x2": (cases.CaseSpec(
        name="subfaces_p3_4x4x2_sync", n_elem=(4, 4, 2), p=3, hi=(4.0, 4.0, 2.0),
        center=(3.2, 1.2, 1.0), seed=15, sponge=(0, 1, 0, 0, 0, 0), cml=True,
        bc=("inflow_static_nscbc", "outflow_nscbc", "farfield", "farfield", "periodic",
            "periodic"),
        subfaces=((0, (0, 2, 0, 2), "inflow_static_nscbc"),
                  (0, (2, 4, 0, 2), "wall_isothermal", (320.0,)),
                  (1, (0, 1, 0, 2), "outflow_nscbc", (101000.0,)),
                  (1, (1, 4, 0, 2), "outflow_nscbc", (101325.0,))), **_OPEN),
        {"Synchronization time step": "5.0e-5", "Restart": "no",
         "Fluctuations to add to initial solution": "Pressure pulse",
         "Pressure pulse center": "3.2 1.2 1.0", "Pressure pulse strength": "1.0e-2",
         "Pressure pulse width": "0.5"}, 2),
    # The configuration of the reference's own total-inflow test case (8x4x4
    # elements of degree 3 on [0,2]x[0,1]x[0,1], total inflow / outflow in i,
    # periodic in j and k, a pressure pulse on the free stream), generated here.
    "total_p3_8x4x4": (cases.CaseSpec(
        name="total_p3_8x4x4", kind="uniform", n_elem=(8, 4, 4), p=3, hi=(2.0, 1.0, 1.0),
        mach=0.1, reynolds=60.0e3, grid_map="none", inlet_sigma=1.0, outlet_sigma=0.25,
        outlet_beta_l=1.0, outlet_beta_t=-1.0, inlet_incoming=False,
        bc=("inflow_total_nscbc", "outflow_nscbc", "periodic", "periodic", "periodic",
            "periodic")),
        {"Synchronization time step": "2.5e-5", "Restart": "no", "CFL number": "2.0",
         "Fluctuations to add to initial solution": "Pressure pulse",
         "Pressure pulse center": "1.0 0.5 0.5", "Pressure pulse strength": "0.1",
         "Pressure pulse width": "0.1"}, 3),
    # A duct in the manner of the reference's n5_15x8x8 case, reduced: degree 5,
    # subsonic inflow, characteristic outflow with a sponge layer, adiabatic walls
    # on the j and k faces, a pressure pulse on the free stream of the boundary data.
    "duct_p5_5x3x3": (cases.CaseSpec(
        name="duct_p5_5x3x3", kind="uniform", n_elem=(5, 3, 3), p=5, hi=(5.0, 1.5, 1.5),
        mach=0.2, grid_map="none", outlet_sigma=0.25, outlet_beta_l=1.0, outlet_beta_t=-1.0,
        sponge=(0, 1, 0, 0, 0, 0), sponge_sigma=10.0,
        bc=("inflow_subsonic", "outflow_nscbc", "wall_heat_flux", "wall_heat_flux",
            "wall_heat_flux", "wall_heat_flux")),
        {"Synchronization time step": "2.0e-5", "Restart": "no", "CFL number": "1.0",
         "Monitor forces": "yes",
         "Fluctuations to add to initial solution": "Pressure pulse",
         "Pressure pulse center": "2.5 0.75 0.75", "Pressure pulse strength": "0.05",
         "Pressure pulse width": "0.2"}, 2),
}


def sync_param_text(spec: cases.CaseSpec, overrides: dict, steps: int) -> str:
    """The generated parameter file with the synchronisation settings applied:
    existing keyword lines are replaced, new ones appended before the subfaces."""
    lines = cases.param_cfg_text(spec).split("\n")
    ov = dict(overrides)
    ov["Number of synchronization time steps"] = str(steps)
    out = []
    for ln in lines:
        key = ln.split(":", 1)[0].strip() if ":" in ln else None
        if key in ov:
            out.append(f"{key}: {ov.pop(key)}")
            continue
        if ln.strip() == "Subface information":
            out.extend(f"{k}: {v}" for k, v in ov.items())
            ov = {}
        out.append(ln)
    return "\n".join(out)


def make_sync(name: str, spec: cases.CaseSpec, overrides: dict, steps: int, out_dir: str) -> str:
    K = spec.p + 1
    KD = K ** 3
    case = cases.build_case(spec)
    text = sync_param_text(spec, overrides, steps)
    with tempfile.TemporaryDirectory() as tmp:
        cfg = cases.write_case(case, tmp)
        with open(cfg, "w") as f:
            f.write(text)
        f_dump, f_sync = os.path.join(tmp, "dump.bin"), os.path.join(tmp, "sync.bin")
        records.run_reference(cfg, "dump", f_dump)
        records.run_reference(cfg, "sync", f_sync, "--steps", str(steps))
        d, r = records.read_records(f_dump), records.read_records(f_sync)
    path = os.path.join(out_dir, f"sync_{name}.npz")
    np.savez_compressed(
        path, spec_json=np.array(spec_to_json(spec)), param_text=np.array(text),
        sol0=d["sol"][:, :, :KD], refcond=d["refcond"], sync_sol=r["sol"][:, :, :KD],
        monitor=r["monitor"], rk_steps=r["rkSteps"], n_sync=np.array(steps))
    return path


def spec_to_json(spec: cases.CaseSpec) -> str:
    return json.dumps(dataclasses.asdict(spec))


def spec_from_json(text: str) -> cases.CaseSpec:
    d = json.loads(text)
    for k in ("n_elem", "lo", "hi", "vel_dir", "center", "bc", "sponge", "wall_data",
              "prescribed_p", "sponge_state", "free_stream", "body_force"):
        if d.get(k) is not None:
            d[k] = tuple(d[k])
    for k in ("prescribed_inflow", "prescribed_total", "prescribed_super"):
        if d.get(k) is not None:
            d[k] = tuple(tuple(v) for v in d[k])
    for k in ("sponge_sigma", "sponge_alpha"):
        if isinstance(d.get(k), list):
            d[k] = tuple(d[k])
    return cases.CaseSpec(**d)


def make(name: str, spec: cases.CaseSpec, out_dir: str, prefix: str = "case") -> str:
    K = spec.p + 1
    KD = K ** 3
    case = cases.build_case(spec)
    with tempfile.TemporaryDirectory() as tmp:
        cfg = cases.write_case(case, tmp)
        f_dump, f_res = os.path.join(tmp, "dump.bin"), os.path.join(tmp, "res.bin")
        f_ssp, f_ls = os.path.join(tmp, "ssp.bin"), os.path.join(tmp, "ls.bin")
        records.run_reference(cfg, "dump", f_dump)
        records.run_reference(cfg, "residual", f_res)
        records.run_reference(cfg, "run", f_ssp, "--steps", str(N_STEPS), "--scheme", "ssprk3")
        records.run_reference(cfg, "run", f_ls, "--steps", str(N_STEPS), "--scheme", "lsrk4")
        d, r = records.read_records(f_dump), records.read_records(f_res)
        s, l = records.read_records(f_ssp), records.read_records(f_ls)
    M = int(d["params"][5])
    MD, M2 = M ** 3, M * M
    faces = ["surfIMin", "surfIMax", "surfJMin", "surfJMax", "surfKMin", "surfKMax"]
    sums = [np.abs(d["volMetric"][:, :10, :MD]).sum()] + \
           [np.abs(d[f][:, :13, :M2]).sum() for f in faces] + \
           [np.abs(d["elemScalars"]).sum()]
    path = os.path.join(out_dir, f"{prefix}_{name}.npz")
    np.savez_compressed(
        path, spec_json=np.array(spec_to_json(spec)), sol0=d["sol"][:, :, :KD],
        res_raw=r["resRaw"][:, :, :KD], res=r["res"][:, :, :KD], monitor=r["monitor"],
        dt0=r["dt"], ssp_sol=s["sol"][:, :, :KD], ssp_dt=s["dtHist"],
        ls_sol=l["sol"][:, :, :KD], ls_dt=l["dtHist"], refcond=d["refcond"],
        metric_sums=np.array(sums), vol_metric_e0=d["volMetric"][0, :10, :MD],
        face_metric_e0=np.stack([d[f][0, :13, :M2] for f in faces]),
        elem_scalars=d["elemScalars"], n_steps=np.array(N_STEPS))
    return path


def main():
    if not records.have_reference_build():
        raise SystemExit("build the oracle first: make -C oracle")
    only = set(sys.argv[1:])
    for name, spec in GOLDEN_SPECS.items():
        if not only or name in only:
            print(make(name, spec, HERE))
    for name, spec in OPEN_SPECS.items():
        if not only or name in only:
            print(make(name, spec, HERE, prefix="open"))
    for name, (spec, overrides, steps) in SYNC_SPECS.items():
        if not only or f"sync_{name}" in only:
            print(make_sync(name, spec, overrides, steps, HERE))


if __name__ == "__main__":
    main()
