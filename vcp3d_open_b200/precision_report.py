"""Accuracy of the mixed-precision form against the FP64 form on the same GPU.

Runs one case twice on the device -- FP64 (the reference's arithmetic) and
mixed (FP32 residual, FP64 state / metrics / time step / RK updates) -- from
the same initial state. The FP64 run chooses each step's CFL time step; the
mixed run replays that step sequence, so both states sit at identical times.
Every `--every` steps it reports, per the mixed-precision configuration
(TGV Re 1600, 48^3 elements at degree 4, 1000 steps, error every 100 steps):

  rel_l2_state   ||U_mixed - U_fp64|| / ||U_fp64||         (modal entropy variables)
  rel_l2_change  ||U_mixed - U_fp64|| / ||U_fp64 - U_0||   (stricter: error of the change)
  rel_l2_res     ||R_mixed - R_fp64|| / ||R_fp64||         (one residual at the final FP64 state)
  drift_fp64, drift_mixed  (integral - integral at step 0) / scale of mass, x, y, z
                 momentum (scale: the mass) and total energy, Gauss quadrature

Prints one JSON line.

    python -m vcp3d_open_b200.precision_report [--workload tgv48_p4_lsrk4]
        [--steps 1000] [--every 100]
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import capi, cases, solver, tgv_report, workloads


def _rel(a: np.ndarray, b: np.ndarray) -> float:
    d = float(np.linalg.norm(a - b))
    n = float(np.linalg.norm(b))
    return d / n if n > 0 else d


def residual_difference(s64: solver.Solver, s32: solver.Solver, state: np.ndarray) -> float:
    """Relative L2 difference of one residual of both forms at the same state."""
    s64.set_state(state)
    s32.set_state(state)
    s64.residual()
    s32.residual()
    return _rel(s32.get_residual(), s64.get_residual())


def run(workload: str, steps: int, every: int, scheme: int = capi.LSRK4) -> dict:
    spec = workloads.make_spec(workload)
    case = cases.build_case(spec)
    p64 = solver.make_params(case, metric_compat=True, precision=capi.FP64)
    disc = solver.setup_discretization(case, p64, device=True)
    s64 = solver.create(case, precision=capi.FP64, disc=disc)
    s32 = solver.create(case, precision=capi.MIXED, disc=disc)
    u0 = s64.get_state()
    i0 = tgv_report.conserved_integrals(u0, disc)
    rows = []
    t_wall = time.time()
    done = 0
    sim_time = 0.0
    while done < steps:
        n = min(every, steps - done)
        hist = s64.step(n, scheme)
        for dt in hist:
            s32.step(1, scheme, fixed_dt=float(dt))
        done += n
        sim_time += float(np.sum(hist))
        u64, u32 = s64.get_state(), s32.get_state()
        rows.append({"step": done, "time": sim_time,
                     "rel_l2_state": _rel(u32, u64),
                     "rel_l2_change": _rel(u32 - u0, u64 - u0),
                     "drift_fp64": tgv_report.drift(tgv_report.conserved_integrals(u64, disc), i0),
                     "drift_mixed": tgv_report.drift(tgv_report.conserved_integrals(u32, disc), i0)})
    u64, u32 = s64.get_state(), s32.get_state()
    rows[-1]["rel_l2_res"] = residual_difference(s64, s32, u64)
    s64.close()
    s32.close()
    return {"workload": workload, "n_elem": list(spec.n_elem), "p": spec.p,
            "dofs": spec.n_dofs, "steps": steps, "every": every,
            "scheme": "lsrk4" if scheme == capi.LSRK4 else "ssprk3",
            "dt_sequence": "CFL steps of the FP64 run, replayed by the mixed run",
            "max_rel_l2_state": max(r["rel_l2_state"] for r in rows),
            "history": rows, "wall_seconds": time.time() - t_wall}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="tgv48_p4_lsrk4", choices=sorted(workloads.WORKLOADS))
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--out", default=None, help="also write the JSON to this file")
    a = ap.parse_args(argv)
    rep = run(a.workload, a.steps, a.every)
    line = json.dumps(rep)
    print(line)
    if a.out:
        with open(a.out, "w") as f:
            f.write(line + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
