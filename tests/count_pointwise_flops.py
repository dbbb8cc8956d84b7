"""Counts the pointwise floating-point work of one residual with an op-counting
scalar type run through the CPU restatement (oracle/dg_numpy.py; test
infrastructure). The counts are the algorithmic per-point figures of the
roofline model in bench.py (kernel_flops), which reads them from
profiles/pointwise_flops.json.

Every +, -, *, / on a value that depends on the state counts one flop (an FMA
is two); exp, log, sqrt and pow count as specials; negation, abs and
comparisons count nothing. Operations between constants of the discretisation
(weights, metric terms) are not counted: they can be formed once. The
sum-factorised contractions (vol_interp, vol_project, the face traces and
their expansions, the CG transforms) run with counting off -- their
multiply-adds are counted exactly in kernel_flops -- and so does the
accumulation of their results into the residual (2 x 5 K^3 adds for the
volume projections, 120 K^3 for the face expansions), which is part of the
same contraction work. The restatement evaluates both branches of the
Ismail-Roe log-mean (series and logarithm) where the GPU evaluates one, so the
Ismail-Roe face count is an upper bound by the cheaper branch (8 flops).

    python tests/count_pointwise_flops.py [--out profiles/pointwise_flops.json]
"""
from __future__ import annotations

import argparse
import json
import math
import operator
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import dg_numpy as dn  # noqa: E402


class Counter:
    flops = 0
    specials = 0
    on = True


class Op:
    """A float that counts the arithmetic done on it."""
    __slots__ = ("v",)

    def __init__(self, v):
        self.v = float(v)

    def __float__(self):
        return self.v

    def __neg__(self):
        return Op(-self.v)

    def __pos__(self):
        return self

    def __abs__(self):
        return Op(abs(self.v))

    def _special(self, f):
        if Counter.on:
            Counter.specials += 1
        try:
            return Op(f(self.v))
        except ValueError:          # log(0), log or sqrt of a negative: IEEE results
            return Op(-math.inf if self.v == 0 else math.nan)

    def exp(self):
        return self._special(math.exp)

    def log(self):
        return self._special(math.log)

    def sqrt(self):
        return self._special(math.sqrt)

    def __lt__(self, o):
        return self.v < _val(o)

    def __le__(self, o):
        return self.v <= _val(o)

    def __gt__(self, o):
        return self.v > _val(o)

    def __ge__(self, o):
        return self.v >= _val(o)


def _val(x):
    return x.v if isinstance(x, Op) else x


def _binary(f, reflected=False, special=False):
    def m(self, o):
        if Counter.on:
            if special:
                Counter.specials += 1
            else:
                Counter.flops += 1
        a, b = (_val(o), self.v) if reflected else (self.v, _val(o))
        try:
            return Op(f(a, b))
        except ZeroDivisionError:   # IEEE results, as numpy gives them under errstate
            return Op(math.nan if a == 0 or math.isnan(a) else math.copysign(math.inf, a))
    return m


for _name, _f in (("add", operator.add), ("sub", operator.sub), ("mul", operator.mul),
                  ("truediv", operator.truediv)):
    setattr(Op, f"__{_name}__", _binary(_f))
    setattr(Op, f"__r{_name}__", _binary(_f, reflected=True))
Op.__pow__ = _binary(operator.pow, special=True)
Op.__rpow__ = _binary(operator.pow, reflected=True, special=True)

_as_op = np.vectorize(Op, otypes=[object])


def _uncounted(fn):
    def wrapped(*a, **k):
        was = Counter.on
        Counter.on = False
        try:
            return fn(*a, **k)
        finally:
            Counter.on = was
    return wrapped


def _count(fn, *a, **k):
    f0, s0 = Counter.flops, Counter.specials
    out = fn(*a, **k)
    return out, Counter.flops - f0, Counter.specials - s0


def count(riemann: int, p: int, sgs: int = dn.SGS_NONE) -> dict:
    """Counts of one residual on a 2x2x2 TGV block of degree p, per element."""
    from vcp3d_open_b200 import cases, solver
    spec = cases.CaseSpec(name="count", kind="tgv", n_elem=(2, 2, 2), p=p,
                          hi=(2 * math.pi,) * 3, mach=0.1, reynolds=1600.0,
                          grid_map="random", grid_amp=0.01, seed=3,
                          riemann="IsmailRoe" if riemann == 1 else "Roe",
                          sgs={dn.SGS_NONE: "none", dn.SGS_WALE: "wale",
                               dn.SGS_VREMAN: "vreman"}[sgs])
    case = cases.build_case(spec)
    prm = solver.make_params(case)
    disc = solver.setup_discretization(case, prm)
    d = dn.from_discretization(disc, prm)
    assert d.riemann == riemann
    nE, K, M = 8, d.K, d.M
    U = _as_op(solver.nodal_to_modal(case, prm).reshape(nE, 5, K, K, K))
    saved = {n: getattr(dn, n) for n in ("vol_interp", "vol_project", "face_traces",
                                         "_face_expand", "_ax")}
    marks = []
    try:
        for n, f in saved.items():
            setattr(dn, n, _uncounted(f))
        (Rv, cg), fv, sv = _count(dn.volume_residual, U, d)
        Rf, ff, sf = _count(dn.face_residual, U, d)
        # The CG's backward transform marks its iterations.
        proj = dn.vol_project

        def marking(*a, **k):
            marks.append(Counter.flops)
            return proj(*a, **k)
        dn.vol_project = marking
        (_, iters), _, _ = _count(dn.mass_solve, Rv + Rf, U, cg, d)
    finally:
        for n, f in saved.items():
            setattr(dn, n, f)
    KD, MD, M2 = K ** 3, M ** 3, M * M
    # numpy's einsum on objects starts every sum from zero: one add per output
    # of the point operator (5 per point) and of the preconditioner (5 per DOF).
    per_it = [b - a - nE * 5 * (MD + KD) for a, b in zip(marks, marks[1:])]
    return dict(K=K, M=M,
                volume=(fv - nE * 2 * 5 * KD) / (nE * MD), volume_specials=sv / (nE * MD),
                face=(ff - nE * 120 * KD) / (nE * 3 * M2), face_specials=sf / (nE * 3 * M2),
                cg_iteration=float(np.median(per_it)) / nE, cg_iterations=int(np.max(iters)))


def constants(riemann: int) -> dict:
    """Per-point constants: volume and face work per point (the same at every
    degree), and the CG iteration split into a part per integration point, one
    per DOF and one per element (the scalars alpha and beta) from degrees 1-3."""
    runs = [count(riemann, p) for p in (1, 2, 3)]
    for key in ("volume", "face", "volume_specials", "face_specials"):
        assert len({r[key] for r in runs}) == 1, (key, [r[key] for r in runs])
    A = np.array([[r["M"] ** 3, r["K"] ** 3, 1.0] for r in runs])
    point, dof, elem = np.linalg.solve(A, [r["cg_iteration"] for r in runs])
    a = runs[0]
    return {"volume_flops_per_point": a["volume"],
            "volume_specials_per_point": a["volume_specials"],
            "face_flops_per_point": a["face"], "face_specials_per_point": a["face_specials"],
            "cg_flops_per_iteration_per_point": round(float(point), 6),
            "cg_flops_per_iteration_per_dof": round(float(dof), 6),
            "cg_flops_per_iteration_per_element": round(float(elem), 6)}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "profiles", "pointwise_flops.json"))
    a = ap.parse_args(argv)
    out = {"counting": "tests/count_pointwise_flops.py: op-counting scalar through the CPU "
                       "restatement (TGV 2x2x2 blocks of degrees 1-3); +,-,*,/ = 1 flop, "
                       "exp/log/sqrt/pow = specials; contractions excluded",
           "ismail_roe": constants(1), "roe": constants(0)}
    line = json.dumps(out, indent=1)
    print(line)
    with open(a.out, "w") as f:
        f.write(line + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
