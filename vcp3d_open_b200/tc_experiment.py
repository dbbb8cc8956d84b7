"""The tensor-core experiment for the mixed form's line contractions.

One sum-factorisation stage maps lines of K modal coefficients to M Gauss
points with the 1-D Legendre operator (degree 4: K = 5, M = 7; degree 5: K = 6,
M = 8). vcpg_line_contraction_probe runs it from shared memory to shared memory
as the residual kernel does, 128 lines per tile and `reps` chained stages per
tile, with FP32 fused multiply-adds (operator in shared memory, as a TMA- or
bulk-copied table would be, and in constant memory, as the residual kernel
holds it), TF32 tensor-core tiles (tcgen05.mma kind::tf32, accumulator in tensor
memory) and the split 3xTF32 form. Reported per variant: stage throughput (lines x stages per
second) and the error of one stage against FP64 on the same FP32 inputs.

    python -m vcp3d_open_b200.tc_experiment [--lines 1048576] [--reps 64]

Prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys

import numpy as np

from . import capi, cases, solver

VARIANTS = {0: "fp32 fma", 1: "tf32 tcgen05", 2: "3xtf32 tcgen05",
            3: "fp32 fma, constant operator"}


def operator(p: int) -> np.ndarray:
    """Legendre basis at the Gauss points, [K][M] (the residual's leg operator)."""
    spec = cases.CaseSpec(name="op", kind="tgv", n_elem=(1, 1, 1), p=p, hi=(1.0,) * 3)
    case = cases.build_case(spec)
    prm = solver.make_params(case)
    return solver.setup_discretization(case, prm).leg_int.astype(np.float32)


def probe(variant: int, op: np.ndarray, x: np.ndarray, reps: int, scale: float):
    lib = capi.load()
    K, M = op.shape
    y = np.zeros((x.shape[0], M), dtype=np.float32)
    ms = C.c_double()
    fp = C.POINTER(C.c_float)
    rc = lib.vcpg_line_contraction_probe(variant, K, M, x.shape[0], reps, scale,
                                         np.ascontiguousarray(x).ctypes.data_as(fp),
                                         np.ascontiguousarray(op).ctypes.data_as(fp),
                                         y.ctypes.data_as(fp), C.byref(ms))
    if rc != capi.VCPG_OK:
        raise capi.VcpgError(rc, f"vcpg_line_contraction_probe variant {variant}")
    return y, ms.value


def run(lines: int = 1 << 20, reps: int = 64, seed: int = 5) -> dict:
    rng = np.random.default_rng(seed)
    out = {"lines": lines, "reps": reps, "degrees": {}}
    for p in (4, 5):
        op = operator(p)
        K, M = op.shape
        x = rng.standard_normal((lines, K)).astype(np.float32)
        scale = float(1.0 / np.abs(op).sum(axis=0).max())
        ref = x.astype(np.float64) @ op.astype(np.float64)
        norm = np.abs(x.astype(np.float64)) @ np.abs(op.astype(np.float64))
        rows = {}
        for v, name in VARIANTS.items():
            y1, _ = probe(v, op, x, 1, scale)
            err = float(np.max(np.abs(y1 - ref) / norm))
            _, ms = probe(v, op, x, reps, scale)
            rows[name] = {"max_rel_error_one_stage": err, "ms": ms,
                          "stages_per_s": lines * reps / (ms * 1e-3),
                          "macs_per_s": lines * reps * K * M / (ms * 1e-3)}
        out["degrees"][str(p)] = {"K": K, "M": M, "variants": rows}
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--lines", type=int, default=1 << 20)
    ap.add_argument("--reps", type=int, default=64)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    line = json.dumps(run(a.lines, a.reps))
    print(line)
    if a.out:
        with open(a.out, "w") as f:
            f.write(line + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
