"""Shared test set-up: the gpu marker and helpers for the golden fixtures."""
from __future__ import annotations

import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, GOLDEN)

from make_golden import spec_from_json  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA library")


def golden_files():
    """Fixtures of periodic blocks."""
    return sorted(glob.glob(os.path.join(GOLDEN, "case_*.npz")))


def open_golden_files():
    """Fixtures of blocks with characteristic boundaries, sponge and matching layers."""
    return sorted(glob.glob(os.path.join(GOLDEN, "open_*.npz")))


def sync_golden_files():
    """Fixtures of synchronisation steps run from a parameter file."""
    return sorted(glob.glob(os.path.join(GOLDEN, "sync_*.npz")))


def write_sync_case(g, directory):
    """The files of a sync fixture: grid, restart and averaged solution from the
    generator, the parameter file from the fixture. Returns the file's path."""
    from vcp3d_open_b200 import cases
    cfg = cases.write_case(cases.build_case(g["spec"]), directory)
    with open(cfg, "w") as f:
        f.write(str(g["param_text"]))
    return cfg


def load_golden(path):
    g = dict(np.load(path))
    g["spec"] = spec_from_json(str(g["spec_json"]))
    return g


def rel_l2(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def assert_forces_match(mon, ref, spec, rel=1e-10):
    """Wall force coefficients (monitoring entries 0-2 pressure, 3-5 viscous)
    against the reference's. Components that cancel across walls are rounding
    noise, so each group is compared on an absolute scale: the pressure group
    to rel times the coefficient of a unit pressure on all wall area, the viscous
    group to rel times its largest component."""
    mon, ref = np.asarray(mon, dtype=float), np.asarray(ref, dtype=float)
    ext = np.asarray(spec.hi, dtype=float) - np.asarray(spec.lo, dtype=float)
    area = 0.0
    for f, b in enumerate(spec.bc):
        if b == "periodic":
            continue
        d = f // 2
        a0, a1 = (1, 2) if d == 0 else ((0, 2) if d == 1 else (0, 1))
        for (b0, e0, b1, e1), sbc, _ in spec.face_subfaces(f):
            if sbc.startswith("wall_"):
                area += float(ext[a0] * ext[a1]) * (e0 - b0) / spec.n_elem[a0] * \
                    (e1 - b1) / spec.n_elem[a1]
    if not (spec.monitor_forces and area > 0.0):
        assert np.all(mon[:6] == 0.0)
        return
    scale_p = 2.0 / (1.4 * spec.mach ** 2 * spec.ref_area) * area
    assert np.max(np.abs(mon[:3] - ref[:3])) <= rel * scale_p, (mon[:3], ref[:3])
    tol_v = rel * np.max(np.abs(ref[3:6])) + 1e-16 * scale_p
    assert np.max(np.abs(mon[3:6] - ref[3:6])) <= tol_v, (mon[3:6], ref[3:6])


@pytest.fixture(scope="session")
def gpu_available():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
