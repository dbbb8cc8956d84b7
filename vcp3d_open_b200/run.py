"""Run a case from the reference solver's own input files on the GPU.

    python -m vcp3d_open_b200.run param.cfg [--precision fp64|mixed] [--steps N]

The driver of the reference main program (src/VCP3D_CurviLinear.cpp:25-178)
for the path this library runs: it reads the parameter file
(vcp3d_open_b200.param_file), the single-block PLOT3D grid, the SU2 restart
file or the free stream with the pressure-pulse fluctuation, sets up the case
on the device and takes the "Number of synchronization time steps" with
vcpg_synchronization_step (ExecuteTimeSynchronizationStep). It prints the
time-step history (step, wall time, time, maximum Mach number, RK steps) every
"Write time history info every" steps and writes SU2 restart files
"<Solution file name>_TimeStep_<n>" (x, y, z and the dimensional conservative
variables at the nodal DOFs, as WriteRestartSolution) at step 0, every "Save
solution every" steps and at the end.
"""
from __future__ import annotations

import argparse
import dataclasses
import math
import os
import struct
import sys
import time
from typing import Optional

import numpy as np

from . import capi, cases, param_file, solver
from .param_file import ParamFile, UnsupportedOption

GAMMA = cases.GAMMA


# ---------------------------------------------------------------------------
# Case assembly from the files
# ---------------------------------------------------------------------------

def _grid_is_lgl(nodes: np.ndarray, p_grid: int) -> bool:
    """Whether the grid nodes of the first element sit at LGL rather than
    equidistant parametric positions along its first i edge (the test of
    ElementClass::LGLDistribution, src/ElementClass.cpp:3406-3623, on one edge)."""
    Kg = p_grid + 1
    edge = nodes[0][:, :Kg]                     # (3, Kg): the first i line of nodes
    seg = np.linalg.norm(np.diff(edge, axis=1), axis=0)
    s = np.concatenate([[0.0], np.cumsum(seg)])
    if s[-1] <= 0.0:
        raise param_file.ParamFileError("degenerate grid element")
    r = -1.0 + 2.0 * s / s[-1]
    lgl = cases.lgl_points(Kg)
    equi = np.linspace(-1.0, 1.0, Kg)
    return float(np.max(np.abs(r - lgl))) <= float(np.max(np.abs(r - equi)))


def _read_su2_columns(path: str, n_elem: int, n_dofs: int):
    """All columns of an SU2 restart file: (names, values [nElem][nVar][nDOFs])."""
    with open(path, "rb") as f:
        data = f.read()
    hdr = struct.unpack_from("<5i", data, 0)
    if hdr[0] != cases.SU2_MAGIC:
        raise param_file.ParamFileError(f"{path}: not an SU2 restart file")
    nvar, npts = hdr[1], hdr[2]
    if npts != n_elem * n_dofs:
        raise param_file.ParamFileError(
            f"{path}: {npts} points, the grid and degree give {n_elem * n_dofs}")
    names = [data[20 + i * cases.NAME_LEN:20 + (i + 1) * cases.NAME_LEN].split(b"\0", 1)[0]
             .decode() for i in range(nvar)]
    off = 20 + nvar * cases.NAME_LEN
    body = np.frombuffer(data, dtype="<f8", count=npts * nvar, offset=off)
    return names, body.reshape(n_elem, n_dofs, nvar).transpose(0, 2, 1).copy()


def _prim_to_cons(rho, u, v, w, p):
    return np.stack([rho, rho * u, rho * v, rho * w,
                     p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v + w * w)])


def _cons_to_prim(c):
    rho = c[0]
    u, v, w = c[1] / rho, c[2] / rho, c[3] / rho
    p = (GAMMA - 1.0) * (c[4] - 0.5 * rho * (u * u + v * v + w * w))
    return rho, u, v, w, p


def _add_pressure_pulse(pf: ParamFile, xyz: np.ndarray, cons: np.ndarray) -> np.ndarray:
    """The "Pressure pulse" fluctuation on the dimensional primitive variables at
    the nodal DOFs (ElementClass pressure-pulse branch, src/ElementClass.cpp:600-663):
    p *= 1 + d0 exp(-r^2 / (2 w^2)) in 3-D; the one-dimensional pulse adds
    g = p d0 exp(-dx^2 / (2 w^2)) to p and +-g / sqrt(gamma p rho) to u."""
    rho, u, v, w, p = _cons_to_prim(cons)
    cc = 0.5 / (pf.pulse_width * pf.pulse_width)
    dx = xyz[:, 0] - pf.pulse_center[0]
    if pf.pulse_1d:
        sign = -1.0 if pf.pulse_direction == "upstream" else 1.0
        g = p * pf.pulse_strength * np.exp(-dx * dx * cc)
        u = u + sign * g / np.sqrt(GAMMA * p * rho)
        p = p + g
    else:
        dy = xyz[:, 1] - pf.pulse_center[1]
        dz = xyz[:, 2] - pf.pulse_center[2]
        p = p * (1.0 + pf.pulse_strength * np.exp(-(dx * dx + dy * dy + dz * dz) * cc))
    return _prim_to_cons(rho, u, v, w, p)


def load_case(pf: ParamFile) -> cases.CaseData:
    """CaseData of a parameter file: grid, reference conditions, boundary data
    and the initial nodal state (restart file or free stream, plus fluctuations)."""
    param_file.check_supported(pf)
    ref = param_file.reference_conditions(pf)
    n_elem = param_file.n_elements(pf)
    grid = cases.read_plot3d(pf.file(pf.grid_file))
    expect = tuple(n * pf.p_grid + 1 for n in n_elem)
    if (grid.shape[3], grid.shape[2], grid.shape[1]) != expect:
        raise param_file.ParamFileError(
            f"grid has {grid.shape[3]}x{grid.shape[2]}x{grid.shape[1]} nodes, the subfaces and "
            f"the grid degree give {expect[0]}x{expect[1]}x{expect[2]}")
    nodes = cases.element_nodes(grid, n_elem, pf.p_grid)
    # Grid nodes at LGL or equidistant positions (detected as the reference does),
    # solution DOFs where the parameter file puts them; their coordinates are the
    # grid's Lagrange interpolation.
    grid_lgl = _grid_is_lgl(nodes, pf.p_grid) if pf.p_grid > 1 else True
    loc = cases.CaseSpec(p=pf.p, p_grid=pf.p_grid, dof_location=pf.dof_location,
                         grid_lgl=grid_lgl)
    xyz = cases.solution_dof_coordinates(loc, nodes)
    n_e, K3 = xyz.shape[0], (pf.p + 1) ** 3
    if pf.restart:
        names, cols = _read_su2_columns(pf.file(pf.restart_file), n_e, K3)
        if len(names) < 8:
            raise param_file.ParamFileError("restart file without the conservative variables")
        if np.max(np.abs(cols[:, :3] - xyz)) > 1e-6 * max(1.0, float(np.max(np.abs(xyz)))):
            raise param_file.ParamFileError("restart coordinates do not match the grid")
        cons = cols[:, 3:8].copy()
    else:
        fs = ref.free_stream
        cons = np.empty((n_e, 5, K3))
        for q, val in enumerate(_prim_to_cons(*[np.float64(c) for c in fs])):
            cons[:, q] = val
    if pf.fluctuations == "pressure pulse":
        cons = np.ascontiguousarray(_add_pressure_pulse(pf, xyz, cons.transpose(1, 0, 2))
                                    .transpose(1, 0, 2))
    bcs = param_file.case_bcs(pf)
    prescribed_p = tuple(param_file.outflow_pressure(pf, f)
                         if b in ("outflow_nscbc", "outflow_subsonic") else 0.0
                         for f, b in enumerate(bcs))
    prescribed_in = tuple(param_file.inflow_static(pf, f) if b == "inflow_static_nscbc"
                          else (0.0, 0.0, 0.0, 0.0) for f, b in enumerate(bcs))
    prescribed_tot = tuple(param_file.inflow_total(pf, f)
                           if b in ("inflow_total_nscbc", "inflow_subsonic")
                           else (0.0, 0.0, 1.0, 0.0, 0.0) for f, b in enumerate(bcs))
    wall_data = tuple(param_file.wall_value(pf, f)
                      if b in ("wall_heat_flux", "wall_isothermal") else 0.0
                      for f, b in enumerate(bcs))
    prescribed_sup = tuple(param_file.inflow_supersonic(pf, f) if b == "inflow_supersonic"
                           else (1.0, 0.0, 0.0, 0.0, 1.0) for f, b in enumerate(bcs))
    sponge = tuple(r[0] for r in pf.sponge) if pf.sponge else (0,) * 6
    sponge_state = None
    if any(sponge):
        sponge_state = _averaged_state(pf, n_e, K3)
    fs = ref.free_stream
    speed = math.sqrt(fs[1] ** 2 + fs[2] ** 2 + fs[3] ** 2)
    vel_dir = tuple(c / speed for c in fs[1:4]) if speed > 0 else (1.0, 0.0, 0.0)
    spec = cases.CaseSpec(
        name=os.path.basename(pf.path) or "case", kind="file", n_elem=n_elem, p=pf.p,
        p_grid=pf.p_grid, n_poly_int=pf.n_poly_int, mach=pf.mach, reynolds=pf.reynolds,
        reynolds_length=pf.reynolds_length, t_inf=pf.t_inf,
        vel_dir=vel_dir, riemann="IsmailRoe" if pf.riemann == "ismailroe" else "Roe",
        sgs=pf.sgs_model, monitor_forces=pf.monitor_forces, ref_area=pf.reference_area,
        dof_location=pf.dof_location, grid_lgl=grid_lgl,
        body_force=tuple(pf.body_force) if pf.body_force is not None else None,
        theta_sym=pf.theta_sym, penalty=pf.penalty, cfl=pf.cfl, grid_map="none",
        bc=bcs, p_inf=ref.p_ref, outlet_len=pf.outlet_len, outlet_sigma=pf.outlet_sigma,
        outlet_beta_l=pf.outlet_beta_l, outlet_beta_t=pf.outlet_beta_t,
        outlet_one_minus_beta=pf.outlet_one_minus_beta, inlet_len=pf.inlet_len,
        inlet_sigma=pf.inlet_sigma, inlet_incoming=pf.inlet_incoming, sponge=sponge,
        sponge_sigma=tuple(r[1] for r in pf.sponge) if pf.sponge else 20.0,
        sponge_alpha=tuple(r[2] for r in pf.sponge) if pf.sponge else 2.0,
        cml=pf.cml and any(sponge), prescribed_p=prescribed_p, prescribed_inflow=prescribed_in,
        prescribed_total=prescribed_tot, sponge_state=sponge_state, wall_data=wall_data,
        prescribed_super=prescribed_sup, free_stream=tuple(ref.free_stream),
        subfaces=param_file.case_subfaces(pf), outlet_local_mach=bool(pf.outlet_local_mach))
    refc = cases.RefConditions(ref.p_ref, ref.rho_ref, ref.u_ref, ref.mu_nondim, speed, vel_dir)
    return cases.CaseData(spec, refc, grid, nodes, xyz, np.ascontiguousarray(cons))


def _averaged_state(pf: ParamFile, n_e: int, K3: int):
    """Sponge target from the averaged-solution file (SpongeLayer.cpp:667-843):
    the averaged density, velocity and pressure, which must be uniform here."""
    names, cols = _read_su2_columns(pf.file(pf.averaged_file), n_e, K3)
    want = ["Density_avg", "VelocityX_avg", "VelocityY_avg", "VelocityZ_avg", "Pressure_avg"]
    if any(nm not in names for nm in want):
        raise param_file.ParamFileError("averaged solution file without the averaged "
                                        "primitive variables")
    out = []
    for nm in want:
        col = cols[:, names.index(nm)]
        if float(np.ptp(col)) > 1e-12 * max(1.0, float(np.max(np.abs(col)))):
            raise UnsupportedOption("a spatially varying averaged solution for the sponge layer")
        out.append(float(col.flat[0]))
    return tuple(out)


# ---------------------------------------------------------------------------
# Output
# ---------------------------------------------------------------------------

def modal_to_nodal_conservative(case: cases.CaseData, disc: solver.Discretization,
                                modal: np.ndarray) -> np.ndarray:
    """Dimensional conservative variables at the nodal DOFs of a modal
    entropy-variable state (ElementClass::ComputePrimitiveVariablesNodalDOFs with
    the reference scalings): the basis at the DOFs along each direction, then
    the entropy -> primitive relations."""
    K = disc.n_poly + 1
    B = disc.leg_dofs.reshape(K, K)             # B[k][i]: basis k at DOF i
    m = modal.reshape(-1, 5, K, K, K)           # [e][v][kk][kj][ki]
    V = np.einsum("evcba,az,by,cx->evxyz", m, B, B, B, optimize=True).reshape(modal.shape)
    gm1 = GAMMA - 1.0
    V4inv = 1.0 / V[:, 4]
    u, v, w = -V[:, 1] * V4inv, -V[:, 2] * V4inv, -V[:, 3] * V4inv
    ekin = 0.5 * (u * u + v * v + w * w)
    s = GAMMA - gm1 * (V[:, 0] - V[:, 4] * ekin)
    rho = (-V[:, 4] * np.exp(s)) ** (1.0 / (1.0 - GAMMA))
    p = -rho * V4inv
    r = case.ref
    return np.ascontiguousarray(_prim_to_cons(rho * r.rho_ref, u * r.u_ref, v * r.u_ref,
                                              w * r.u_ref, p * r.p_ref).transpose(1, 0, 2))


def write_solution(pf: ParamFile, case: cases.CaseData, disc: solver.Discretization,
                   modal: np.ndarray, step: int) -> str:
    path = pf.file(f"{pf.solution_file}_TimeStep_{step}")
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    cases.write_su2_restart(path, case.dof_xyz, modal_to_nodal_conservative(case, disc, modal))
    return path


# ---------------------------------------------------------------------------
# The driver
# ---------------------------------------------------------------------------

@dataclasses.dataclass
class RunResult:
    state: np.ndarray            # final modal entropy-variable state [nE][5][K^3]
    rk_steps: int
    history: list                # (step, time, mach_max, rk_steps)
    files: list
    monitoring: Optional[np.ndarray] = None   # the last step's 8 monitoring values


def _force_directions(pf: ParamFile):
    """Free-stream and lift directions of the force coefficients
    (src/InputParamClass.cpp:697-736): unit vectors, the lift direction by default
    normal to the free stream without a z component."""
    v = np.asarray(pf.vel_dir if pf.vel_dir is not None else (1.0, 0.0, 0.0), dtype=float)
    v = v / np.linalg.norm(v)
    lift = np.asarray(pf.lift_dir if pf.lift_dir is not None else (-v[1], v[0], 0.0),
                      dtype=float)
    return v, lift / np.linalg.norm(lift)


def run(path: str, precision: int = capi.FP64, steps: Optional[int] = None,
        write: bool = True, out=sys.stdout) -> RunResult:
    pf = param_file.read(path)
    case = load_case(pf)
    params = solver.make_params(case, precision=precision)
    disc = solver.setup_discretization(case, params, device=True)
    s = solver.Solver(params, disc)
    files, history = [], []
    try:
        if case.spec.is_open:
            s.set_open_boundary(case)
        s.set_state(solver.nodal_to_modal(case, params))
        n_sync = pf.n_sync if steps is None else steps
        dt_sync = pf.dt_sync * case.ref.u_ref       # non-dimensional (reference length 1)
        if write:
            files.append(write_solution(pf, case, disc, s.get_state(), 0))
        sgs = case.spec.sgs != "none"
        forces = params.monitor_forces != 0
        vel_dir, lift_dir = _force_directions(pf)
        print(f"#{'step':>9}{'wall (s)':>13}{'time (s)':>13}{'Mach max':>13}{'RK steps':>10}"
              + (f"{'mu_t/mu':>13}" if sgs else "")
              + (f"{'CL':>13}{'CD':>13}{'CL visc':>13}{'CD visc':>13}" if forces else ""),
              file=out)
        last_mon = None
        t0 = time.perf_counter()
        total_rk, saved = 0, True
        for n in range(1, n_sync + 1):
            saved = False
            if n % pf.n_history == 0:
                rk, mon = s.synchronization_step(dt_sync, monitoring=True)
                last_mon = mon
                mach = math.sqrt(max(mon[6], 0.0))
                history.append((n, n * pf.dt_sync, mach, rk))
                line = (f"{n:>10}{time.perf_counter() - t0:>13.5e}{n * pf.dt_sync:>13.5e}"
                        f"{mach:>13.5e}{rk:>10}")
                if sgs:   # eddy over laminar viscosity (WriteTimeStepData)
                    line += f"{mon[7] / case.ref.mu_nondim:>13.5e}"
                if forces:
                    cl_i, cl_v = float(mon[0:3] @ lift_dir), float(mon[3:6] @ lift_dir)
                    cd_i, cd_v = float(mon[0:3] @ vel_dir), float(mon[3:6] @ vel_dir)
                    line += f"{cl_i + cl_v:>13.5e}{cd_i + cd_v:>13.5e}{cl_v:>13.5e}{cd_v:>13.5e}"
                print(line, file=out, flush=True)
            else:
                rk = s.synchronization_step(dt_sync)
            total_rk += rk
            if write and pf.n_save > 0 and n % pf.n_save == 0:
                files.append(write_solution(pf, case, disc, s.get_state(), n))
                saved = True
        state = s.get_state()
        if write and not saved:
            files.append(write_solution(pf, case, disc, state, n_sync))
        return RunResult(state, total_rk, history, files, last_mon)
    finally:
        s.close()


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("param", help="the reference solver's parameter file")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--steps", type=int, default=None,
                    help="synchronization steps (default: the parameter file's)")
    ap.add_argument("--no-write", action="store_true", help="write no solution files")
    a = ap.parse_args(argv)
    try:
        run(a.param, capi.FP64 if a.precision == "fp64" else capi.MIXED, a.steps,
            write=not a.no_write)
    except UnsupportedOption as e:
        print(f"unsupported option: {e}", file=sys.stderr)
        return 3
    except param_file.ParamFileError as e:
        print(f"parameter file error: {e}", file=sys.stderr)
        return 2
    return 0


if __name__ == "__main__":
    sys.exit(main())
