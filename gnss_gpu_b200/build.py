"""Build libgnsspf_b200.so in-tree with nvcc for sm_100a, and its checked
variant libgnsspf_b200_checked.so (-DPF_CHECKED: data-dependent indexes are
tested before use and a bad one is reported through the error word).

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
LIB_CHECKED = LIBDIR / "libgnsspf_b200_checked.so"
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


def _stale(lib: Path) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [PKG.parent / "include" / "gnss_pf_b200.h"]
    return any(p.stat().st_mtime > t for p in deps)


def _build_lib(lib: Path, objdir: Path, extra: list, verbose: bool) -> Path:
    from concurrent.futures import ThreadPoolExecutor

    LIBDIR.mkdir(exist_ok=True)
    objdir.mkdir(exist_ok=True)
    cmds, objs = [], []
    for src in SOURCES:
        obj = objdir / (Path(src).stem + ".o")
        cmds.append([nvcc()] + NVCC_FLAGS + extra + ["-c", str(CSRC / src), "-o", str(obj)])
        objs.append(str(obj))
    if verbose:
        for c in cmds:
            print(" ".join(c), flush=True)
    with ThreadPoolExecutor(max_workers=len(cmds)) as ex:  # independent translation units
        for r in ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds):
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed:\n{r.stdout}\n{r.stderr}")
    tmp = lib.with_suffix(".so.tmp")
    cmd = [nvcc()] + ARCH + ["-shared", "-o", str(tmp)] + objs + ["-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, lib)
    return lib


def build(force: bool = False, verbose: bool = False, checked: bool = True) -> Path:
    """Build the library (and its checked variant) when a source is newer."""
    if force or _stale(LIB):
        _build_lib(LIB, PKG / "_build", [], verbose)
    if checked and (force or _stale(LIB_CHECKED)):
        _build_lib(LIB_CHECKED, PKG / "_build_checked", ["-DPF_CHECKED"], verbose)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
