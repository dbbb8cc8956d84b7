"""Long-horizon parity against the reference build (test infrastructure).

Runs one configuration for its stated number of time steps on the GPU (FP64 at
its own CFL steps, and with --mixed the mixed form replaying the FP64 steps)
and, at the same time on the host cores, the reference build (oracle/_ref,
every host thread) on the same generated files, sampling every --every steps:

* the relative L2 difference of the modal states, GPU against the reference;
* the largest relative difference of the time-step histories so far;
* volume integrals of the conserved variables (mass, momentum, total energy)
  by the elements' Gauss quadrature, and their drift from step 0, for both;
* per configuration: the kinetic energy E* and its dissipation rate (TGV) or
  the probe-box reflection max |p - p_inf| / (d0 p_inf) (acoustic pulse).

    python tests/long_horizon.py vortex --steps 100 --scheme lsrk4|ssprk3
    python tests/long_horizon.py tgv    --steps 500 --every 100 [--mixed]
    python tests/long_horizon.py pulse  --steps 400 --every 100 [--mixed]
    python tests/long_horizon.py pulse  --steps 2000 --every 200 --reference-only

--reference-only runs the reference build alone (no GPU) and reports its
samples. Prints one JSON line (and writes it to --out).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import records  # noqa: E402
from vcp3d_open_b200 import capi, cases, pulse_report, solver, tgv_report, workloads  # noqa: E402

CONFIGS = {"vortex": "vortex8_p3_lsrk4", "tgv": "tgv32_p3_lsrk4", "pulse": "pulse40_p4_lsrk4"}
SCHEMES = {"lsrk4": capi.LSRK4, "ssprk3": capi.SSPRK3}


def conserved_integrals(modal: np.ndarray, disc: solver.Discretization) -> np.ndarray:
    """Integrals of (rho, rho u, rho v, rho w, rho E) over the block by the elements'
    Gauss quadrature (vcp3d_open_b200.tgv_report.conserved_integrals)."""
    return tgv_report.conserved_integrals(modal, disc)


def _rel(a, b) -> float:
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def _start_reference(cfg: str, out: str, steps: int, every: int, scheme: str, threads: int):
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(threads)
    return subprocess.Popen([records.REF_EXE, cfg, "run", out, "--steps", str(steps), "--scheme",
                             scheme, "--every", str(every), "--time"],
                            stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, env=env)


def _reference_samples(out: str, steps: int, every: int, K3: int):
    samples = {}
    for n in range(every, steps + 1, every):
        r = records.read_records(f"{out}.{n}")
        samples[n] = (r["sol"][:, :, :K3].copy(), r["dtHist"].copy())
    return samples


def run(config: str, steps: int, every: int, scheme: str = "lsrk4", mixed: bool = False,
        reference_only: bool = False, threads: int = 0) -> dict:
    workload = CONFIGS[config]
    spec = workloads.make_spec(workload)
    case = cases.build_case(spec)
    K3 = (spec.p + 1) ** 3
    threads = threads or os.cpu_count() or 1
    every = min(every, steps)
    p64 = solver.make_params(case, precision=capi.FP64)
    disc = solver.setup_discretization(case, p64)
    u0 = solver.nodal_to_modal(case, p64)

    extra = None
    if config == "pulse":
        mask = pulse_report.probe_mask(case.dof_xyz, (6.0, 3.0, 3.0), (14.0, 7.0, 7.0))
        scale = spec.pulse_amp * case.ref.p_ref

        def extra(u):
            p = pulse_report.nodal_pressure(u, disc.leg_dofs, case.ref.p_ref)
            return float(np.abs(p[mask] - case.ref.p_ref).max() / scale)
    elif config == "tgv":
        v0 = case.ref.v_inf / case.ref.u_ref

        def extra(u):
            return tgv_report.kinetic_energy(u, disc) / v0 ** 2

    t_wall = time.time()
    with tempfile.TemporaryDirectory() as tmp:
        cfg = cases.write_case(case, tmp)
        out = os.path.join(tmp, "run.bin")
        proc = _start_reference(cfg, out, steps, every, scheme, threads)

        gpu, mix = {}, {}
        if not reference_only:
            s64 = solver.create(case, precision=capi.FP64, disc=disc)
            s32 = solver.create(case, precision=capi.MIXED, disc=disc) if mixed else None
            try:
                s64.residual()
                if s32 is not None:
                    s32.residual()
                hist = []
                for n in range(every, steps + 1, every):
                    h = s64.step(every, SCHEMES[scheme])
                    hist.extend(float(x) for x in h)
                    if s32 is not None:
                        for dt in h:
                            s32.step(1, SCHEMES[scheme], fixed_dt=float(dt))
                        mix[n] = s32.get_state()
                    gpu[n] = (s64.get_state(), np.array(hist))
            finally:
                s64.close()
                if s32 is not None:
                    s32.close()
        t_gpu = time.time() - t_wall
        so, se = proc.communicate()
        if proc.returncode != 0:
            raise RuntimeError(f"reference build failed ({proc.returncode}):\n{so[-2000:]}\n"
                               f"{se[-2000:]}")
        ref = _reference_samples(out, steps, every, K3)
    secs = None
    for line in so.splitlines():
        if line.startswith("VCP3D_REF_TIMING"):
            secs = float(dict(t.split("=") for t in line.split()[1:])["seconds"])

    i0 = conserved_integrals(u0, disc)
    # Drift scales: the mass, mass times the reference speed (momentum), the energy.
    scl = np.array([abs(i0[0])] + [abs(i0[0])] * 3 + [abs(i0[4])])
    rows = [{"step": 0, "time": 0.0,
             "extra_gpu": extra(u0) if extra else None,
             "extra_reference": extra(u0) if extra else None}]
    for n in sorted(ref):
        ur, hr = ref[n]
        ir = conserved_integrals(ur, disc)
        row = {"step": n, "time": float(np.sum(hr)),
               "reference_drift": [float(x) for x in (ir - i0) / scl],
               "extra_reference": extra(ur) if extra else None}
        if n in gpu:
            ug, hg = gpu[n]
            ig = conserved_integrals(ug, disc)
            row.update({
                "rel_l2_state_gpu_vs_reference": _rel(ug, ur),
                "max_rel_dt_diff": float(np.max(np.abs(hg - hr) / np.abs(hr))),
                "gpu_drift": [float(x) for x in (ig - i0) / scl],
                "extra_gpu": extra(ug) if extra else None})
            if n in mix:
                row["rel_l2_state_mixed_vs_fp64"] = _rel(mix[n], ug)
                row["rel_l2_state_mixed_vs_reference"] = _rel(mix[n], ur)
                if extra:
                    row["extra_mixed"] = extra(mix[n])
        rows.append(row)
    if config == "tgv":
        for key in ("extra_gpu", "extra_reference", "extra_mixed"):
            for i in range(1, len(rows) - 1):
                a, b = rows[i - 1], rows[i + 1]
                if a.get(key) is not None and b.get(key) is not None:
                    v0 = case.ref.v_inf / case.ref.u_ref
                    rows[i]["rate_" + key[6:]] = -(b[key] - a[key]) / ((b["time"] - a["time"]) * v0)
    return {"config": config, "workload": workload, "scheme": scheme, "steps": steps,
            "every": every, "reference_threads": threads, "reference_seconds": secs,
            "gpu_wall_seconds": None if reference_only else t_gpu,
            "extra": {"tgv": "E* = <0.5 rho |u|^2> / (rho_0 V_0^2) (Gauss quadrature)",
                      "pulse": "max |p - p_inf| / (d0 p_inf) over the nodal DOFs in "
                               "[6,14]x[3,7]x[3,7]"}.get(config),
            "drift": "(integral(step) - integral(0)) / scale: mass, x/y/z momentum (scale: "
                     "mass), total energy (non-dimensional)",
            "rows": rows}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("config", choices=sorted(CONFIGS))
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--scheme", default="lsrk4", choices=sorted(SCHEMES))
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--reference-only", action="store_true")
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    rep = run(a.config, a.steps, a.every, a.scheme, a.mixed, a.reference_only, a.threads)
    line = json.dumps(rep)
    print(line)
    if a.out:
        with open(a.out, "w") as f:
            f.write(line + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
