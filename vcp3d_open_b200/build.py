"""Builds the CUDA library libvcp3d_b200.so in-tree for sm_100a with nvcc.

    python -m vcp3d_open_b200.build            # incremental
    python -m vcp3d_open_b200.build --force    # rebuild everything
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
ROOT = os.path.dirname(PKG)
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libvcp3d_b200.so")
SOURCES = ["kernels.cu", "capi.cu", "capi_setup.cpp", "host_setup.cpp", "open_boundary.cpp",
           "ensemble.cu", "geometry.cu",
           "noalloc.cu", "tc_contract.cu"]
# kernels_pair.cu is compiled once per supported (K, M) pair (the reference's
# tensor-product dispatch), so that the pairs compile in parallel.
PAIRS = [(2, 2), (2, 3), (3, 4), (4, 5), (5, 7), (6, 8), (7, 9), (8, 12), (9, 13), (10, 14)]
# Per-file flags: the device metric terms round every product and sum separately,
# as the host set-up does (explicit fma calls stay fused).
EXTRA = {"geometry.cu": ["-fmad=false"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "-diag-suppress", "177"]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _headers_mtime() -> float:
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    paths.append(os.path.join(ROOT, "include", "vcp3d_b200.h"))
    return max(os.path.getmtime(p) for p in paths)


def _compile(unit, force: bool) -> str:
    src, defines = unit if isinstance(unit, tuple) else (unit, [])
    tag = "".join("_" + d.split("=")[1] for d in defines)
    obj = os.path.join(BUILD, src + tag + ".o")
    path = os.path.join(CSRC, src)
    if (not force and os.path.exists(obj)
            and os.path.getmtime(obj) >= max(os.path.getmtime(path), _headers_mtime())):
        return obj
    cmd = [_nvcc(), *ARCH, *FLAGS, *EXTRA.get(src, []), *[f"-D{d}" for d in defines],
           "-x", "cu" if src.endswith(".cu") else "c++", "-c", path, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    return obj


def build(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    units = [("kernels_pair.cu", [f"VCPG_PAIR_K={k}", f"VCPG_PAIR_M={m}"]) for k, m in PAIRS]
    units += SOURCES   # the pair objects, the longest compiles, start first
    with cf.ThreadPoolExecutor(max_workers=min(len(units), os.cpu_count() or 8)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), units))
    if (force or not os.path.exists(LIB)
            or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs)):
        cmd = [_nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
