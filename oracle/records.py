"""Test infrastructure only: reader/writer for the oracle's tagged binary files
and a thin runner for the oracle executable (oracle/_ref/vcp3d_ref).

File layout: b"VCPR", then records of
    char name[32]; int32 ndim; int64 dims[ndim]; float64 data[prod(dims)].
"""
from __future__ import annotations

import os
import struct
import subprocess
from typing import Dict

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_EXE = os.path.join(HERE, "_ref", "vcp3d_ref")
# The reference's VCP3D_CurviLinear source folder (only this container has it):
# the one variable that build recipes and CPU tests read.
REF_SRC_ENV = "VCP3D_REF_SRC"
REF_SRC_DEFAULT = "/root/reference/VCP3D_CurviLinear"


def reference_source_dir() -> str:
    """The reference source folder: $VCP3D_REF_SRC, else the default location."""
    return os.environ.get(REF_SRC_ENV) or REF_SRC_DEFAULT


def read_records(path: str) -> Dict[str, np.ndarray]:
    out: Dict[str, np.ndarray] = {}
    with open(path, "rb") as f:
        data = f.read()
    if data[:4] != b"VCPR":
        raise ValueError(f"{path}: not a VCPR file")
    off = 4
    while off < len(data):
        name = data[off:off + 32].split(b"\0", 1)[0].decode()
        off += 32
        (nd,) = struct.unpack_from("<i", data, off)
        off += 4
        dims = struct.unpack_from(f"<{nd}q", data, off)
        off += 8 * nd
        n = int(np.prod(dims)) if nd else 1
        out[name] = np.frombuffer(data, dtype="<f8", count=n, offset=off).reshape(dims).copy()
        off += 8 * n
    return out


def write_records(path: str, recs: Dict[str, np.ndarray]) -> None:
    with open(path, "wb") as f:
        f.write(b"VCPR")
        for name, arr in recs.items():
            a = np.ascontiguousarray(arr, dtype="<f8")
            f.write(name.encode().ljust(32, b"\0")[:32])
            f.write(struct.pack("<i", a.ndim))
            f.write(struct.pack(f"<{a.ndim}q", *a.shape))
            f.write(a.tobytes())


def have_reference_build() -> bool:
    return os.path.exists(REF_EXE)


def run_reference(cfg: str, command: str, out: str, *args: str, threads: int = 1,
                  timeout: float = 3600.0) -> str:
    """Run the oracle executable; returns its stdout. Raises on failure."""
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(threads)
    proc = subprocess.run([REF_EXE, cfg, command, out, *args], capture_output=True,
                          text=True, env=env, timeout=timeout)
    if proc.returncode != 0:
        raise RuntimeError(f"oracle failed ({proc.returncode}):\n{proc.stdout[-2000:]}\n"
                           f"{proc.stderr[-2000:]}")
    return proc.stdout
