"""Build libgnsspf_b200.so in-tree with nvcc for sm_100a.

Usage: python -m gnss_gpu_b200.build [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libgnsspf_b200.so"
SOURCES = ["pf_status.cu", "pf_engine.cu", "pf_compat.cu", "pf_noalloc.cu", "pf_mlp.cu"]
HEADERS = ["pf_common.cuh", "pf_engine_dev.cuh", "pf_engine_kernels.cuh", "pf_epoch_kernel.cuh", "pf_mlp.cuh",
           "pf_learned.cuh", "pf_generic.cuh", "pf_obs_terms.cuh", "pf_velocity.cuh", "pf_bvh.cuh",
           "pf_weight3d.cuh", "pf_orbit.cuh", "pf_city.cuh",
           "pf_status.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build the extension")
    return cand


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [PKG.parent / "include" / "gnss_pf_b200.h"]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale():
        return LIB
    LIBDIR.mkdir(exist_ok=True)
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = objdir / (Path(src).stem + ".o")
        cmd = [nvcc()] + NVCC_FLAGS + ["-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc()] + ARCH + ["-shared", "-o", str(tmp)] + objs + ["-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
