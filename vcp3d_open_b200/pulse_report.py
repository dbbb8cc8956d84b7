"""Reflection report of the open-boundary configuration.

Runs the acoustic-pulse case with characteristic boundaries, sponge and
matching layers (workload pulse40_p4_lsrk4) on the GPU and records, every
`--every` steps, the largest pressure deviation from the free stream inside an
interior probe box, relative to the pulse amplitude d0 p_inf:

    reflection(t) = max over nodal DOFs in the box of |p - p_inf| / (d0 p_inf)

Once the pulse has left the box, what remains there is what the boundaries
and layers reflect back. The FP64 run picks its CFL steps; with --mixed the
mixed form replays them and its history is reported beside the FP64 one.
Prints one JSON line.

    python -m vcp3d_open_b200.pulse_report [--steps 2000] [--every 100] [--mixed]
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import capi, cases, solver, workloads

GAMMA = 1.4


def nodal_pressure(modal: np.ndarray, legdof: np.ndarray, p_ref: float) -> np.ndarray:
    """Dimensional pressure at the nodal DOFs from the modal entropy variables
    [nE][5][K^3] (legdof[k][i]: basis k at nodal DOF i)."""
    K = legdof.shape[0]
    U = modal.reshape(modal.shape[0], 5, K, K, K)
    V = np.einsum("evcba,ck,bj,ai->evkji", U, legdof, legdof, legdof)  # [e, v, k, j, i]
    V4Inv = 1.0 / V[:, 4]
    u, v, w = -V4Inv * V[:, 1], -V4Inv * V[:, 2], -V4Inv * V[:, 3]
    s = GAMMA - (GAMMA - 1.0) * (V[:, 0] - 0.5 * V[:, 4] * (u * u + v * v + w * w))
    rho = (-V[:, 4] * np.exp(s)) ** (-1.0 / (GAMMA - 1.0))
    return (-V4Inv * rho * p_ref).reshape(modal.shape[0], -1)


def probe_mask(dof_xyz: np.ndarray, lo, hi) -> np.ndarray:
    x, y, z = dof_xyz[:, 0], dof_xyz[:, 1], dof_xyz[:, 2]
    return ((x >= lo[0]) & (x <= hi[0]) & (y >= lo[1]) & (y <= hi[1]) &
            (z >= lo[2]) & (z <= hi[2]))


def run(workload: str = "pulse40_p4_lsrk4", steps: int = 2000, every: int = 100,
        mixed: bool = False, box_lo=(6.0, 3.0, 3.0), box_hi=(14.0, 7.0, 7.0)) -> dict:
    spec = workloads.make_spec(workload)
    case = cases.build_case(spec)
    p64 = solver.make_params(case, precision=capi.FP64)
    disc = solver.setup_discretization(case, p64, device=True)
    s64 = solver.create(case, precision=capi.FP64, disc=disc)
    s32 = solver.create(case, precision=capi.MIXED, disc=disc) if mixed else None
    mask = probe_mask(case.dof_xyz, box_lo, box_hi)
    scale = spec.pulse_amp * case.ref.p_ref

    def reflection(s):
        p = nodal_pressure(s.get_state(), disc.leg_dofs, case.ref.p_ref)
        return float(np.abs(p[mask] - case.ref.p_ref).max() / scale)

    rows = [{"step": 0, "time": 0.0, "fp64": reflection(s64)}]
    if mixed:
        rows[0]["mixed"] = reflection(s32)
    t_wall, t_sim, done = time.time(), 0.0, 0
    while done < steps:
        n = min(every, steps - done)
        hist = s64.step(n, capi.LSRK4)
        if mixed:
            for dt in hist:
                s32.step(1, capi.LSRK4, fixed_dt=float(dt))
        done += n
        t_sim += float(np.sum(hist))
        row = {"step": done, "time": t_sim, "fp64": reflection(s64)}
        if mixed:
            row["mixed"] = reflection(s32)
            u64, u32 = s64.get_state(), s32.get_state()
            row["mixed_rel_l2_state"] = float(np.linalg.norm(u32 - u64) / np.linalg.norm(u64))
        rows.append(row)
    s64.close()
    if s32 is not None:
        s32.close()
    return {"workload": workload, "steps": steps, "every": every,
            "probe_box": [list(box_lo), list(box_hi)],
            "metric": "max |p - p_inf| / (d0 p_inf) over the nodal DOFs in the probe box",
            "final_fp64": rows[-1]["fp64"], "history": rows,
            "wall_seconds": time.time() - t_wall}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="pulse40_p4_lsrk4")
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    rep = run(a.workload, a.steps, a.every, a.mixed)
    line = json.dumps(rep)
    print(line)
    if a.out:
        with open(a.out, "w") as f:
            f.write(line + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
