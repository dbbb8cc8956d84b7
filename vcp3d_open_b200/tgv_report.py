"""Kinetic-energy report of the Taylor-Green configuration.

Runs the Taylor-Green vortex (workload tgv32_p3_lsrk4: Re 1600, Mach 0.1,
[0, 2pi]^3, 32^3 elements of degree 3) on the GPU and records, every `--every`
steps, the volume-averaged kinetic energy from the Gauss quadrature of the
elements,

    E(t) = sum_e sum_q w_q J_q 0.5 rho |u|^2 / sum_e sum_q w_q J_q,

in the usual scaling E* = E / (rho_0 V_0^2), t* = t V_0 / L (L = 1), and its
dissipation rate -dE*/dt* by central differences. The rate at t = 0 is set
beside nu <|omega|^2> of the initial incompressible field, nu = 1/Re in this
scaling, evaluated by the same quadrature. With --mixed the mixed form replays
the FP64 run's steps. Prints one JSON line.

    python -m vcp3d_open_b200.tgv_report [--steps 500] [--every 25] [--mixed]
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import capi, cases, solver, workloads

GAMMA = 1.4


def _to_points(modal: np.ndarray, leg: np.ndarray) -> np.ndarray:
    """Modal [nE][5][K^3] -> values at the Gauss points [nE][5][M^3] (leg[k][m])."""
    K = leg.shape[0]
    U = modal.reshape(modal.shape[0], 5, K, K, K)
    V = np.einsum("evcba,ck,bj,ai->evkji", U, leg, leg, leg, optimize=True)
    return V.reshape(modal.shape[0], 5, -1)


def kinetic_energy(modal: np.ndarray, disc: solver.Discretization) -> float:
    """Volume-averaged 0.5 rho |u|^2 (non-dimensional) by Gauss quadrature."""
    V = _to_points(modal, disc.leg_int)
    V4Inv = 1.0 / V[:, 4]
    u, v, w = -V4Inv * V[:, 1], -V4Inv * V[:, 2], -V4Inv * V[:, 3]
    q2 = u * u + v * v + w * w
    s = GAMMA - (GAMMA - 1.0) * (V[:, 0] - 0.5 * V[:, 4] * q2)
    rho = (-V[:, 4] * np.exp(s)) ** (-1.0 / (GAMMA - 1.0))
    w1 = disc.w_int
    W = (w1[None, None, :] * w1[None, :, None] * w1[:, None, None]).reshape(-1)
    JW = disc.vol_metric[:, 0] * W[None, :]
    return float(np.sum(JW * 0.5 * rho * q2) / np.sum(JW))


def conserved_integrals(modal: np.ndarray, disc: solver.Discretization,
                        chunk: int = 8192) -> np.ndarray:
    """Integrals of (rho, rho u, rho v, rho w, rho E) over the block (non-dimensional),
    by the Gauss quadrature of the elements, in element chunks."""
    w1 = disc.w_int
    W = (w1[None, None, :] * w1[None, :, None] * w1[:, None, None]).reshape(-1)
    out = np.zeros(5)
    for e0 in range(0, modal.shape[0], chunk):
        V = _to_points(modal[e0:e0 + chunk], disc.leg_int)
        V4Inv = 1.0 / V[:, 4]
        u, v, w = -V4Inv * V[:, 1], -V4Inv * V[:, 2], -V4Inv * V[:, 3]
        q2 = u * u + v * v + w * w
        s = GAMMA - (GAMMA - 1.0) * (V[:, 0] - 0.5 * V[:, 4] * q2)
        rho = (-V[:, 4] * np.exp(s)) ** (-1.0 / (GAMMA - 1.0))
        p = -V4Inv * rho
        rE = p / (GAMMA - 1.0) + 0.5 * rho * q2
        JW = disc.vol_metric[e0:e0 + chunk, 0] * W[None, :]
        out += np.array([np.sum(JW * q) for q in (rho, rho * u, rho * v, rho * w, rE)])
    return out


def drift(integrals: np.ndarray, initial: np.ndarray) -> list:
    """(integral - initial) / scale: mass, x, y, z momentum (scale: the mass) and
    total energy."""
    scl = np.array([abs(initial[0])] * 4 + [abs(initial[4])])
    return [float(x) for x in (integrals - initial) / scl]


def initial_dissipation(reynolds: float, n: int = 64) -> float:
    """nu <|omega|^2> of u = (sin x cos y cos z, -cos x sin y cos z, 0) on the
    periodic cube (midpoint rule, exact for these trigonometric products)."""
    x = (np.arange(n) + 0.5) * (2.0 * np.pi / n)
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    wx = -np.cos(X) * np.cos(Y) * np.sin(Z)
    wy = -np.sin(X) * np.cos(Y) * np.sin(Z)
    wz = 2.0 * np.sin(X) * np.sin(Y) * np.cos(Z)
    return float(np.mean(wx * wx + wy * wy + wz * wz) / reynolds)


def run(workload: str = "tgv32_p3_lsrk4", steps: int = 500, every: int = 25,
        mixed: bool = False) -> dict:
    spec = workloads.make_spec(workload)
    case = cases.build_case(spec)
    p64 = solver.make_params(case, precision=capi.FP64)
    disc = solver.setup_discretization(case, p64, device=True)
    s64 = solver.create(case, precision=capi.FP64, disc=disc)
    s32 = solver.create(case, precision=capi.MIXED, disc=disc) if mixed else None
    v0 = case.ref.v_inf / case.ref.u_ref          # V_0 in units of u_ref
    e0 = kinetic_energy(s64.get_state(), disc)
    t, hist, hist32 = 0.0, [(0.0, e0 / v0 ** 2)], []
    if s32 is not None:
        hist32.append((0.0, kinetic_energy(s32.get_state(), disc) / v0 ** 2))
    t0 = time.perf_counter()
    for n in range(1, steps + 1):
        dt = float(s64.step(1, capi.LSRK4)[0])
        if s32 is not None:
            s32.step(1, capi.LSRK4, fixed_dt=dt)
        t += dt
        if n % every == 0:
            hist.append((t * v0, kinetic_energy(s64.get_state(), disc) / v0 ** 2))
            if s32 is not None:
                hist32.append((t * v0, kinetic_energy(s32.get_state(), disc) / v0 ** 2))
    wall = time.perf_counter() - t0

    def rates(h):
        ts, es = np.array([a for a, _ in h]), np.array([b for _, b in h])
        return [(float(ts[i]), float(-(es[i + 1] - es[i - 1]) / (ts[i + 1] - ts[i - 1])))
                for i in range(1, len(h) - 1)]

    out = {"workload": workload, "steps": steps, "every": every, "wall_s": wall,
           "energy": hist, "dissipation": rates(hist),
           "initial_dissipation_incompressible": initial_dissipation(spec.reynolds)}
    if hist32:
        out["energy_mixed"] = hist32
        out["dissipation_mixed"] = rates(hist32)
    s64.close()
    if s32 is not None:
        s32.close()
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="tgv32_p3_lsrk4")
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--every", type=int, default=25)
    ap.add_argument("--mixed", action="store_true")
    a = ap.parse_args(argv)
    print(json.dumps(run(a.workload, a.steps, a.every, a.mixed)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
