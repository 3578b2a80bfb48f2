"""Compile the reference's particle-filter module in place of its CMake build.

Builds rsasaki0109/gnss_gpu's `_gnss_gpu_pf` extension (src/particle_filter/
{predict,weight,resampling}.cu + python/gnss_gpu/_particle_filter_bindings.cpp,
CMakeLists.txt:78-84,191-192 of that project) directly with nvcc/g++ from the
reference tree, for sm_100a, into oracle/_ref/gnss_gpu/.  Nothing is copied
from the reference: the sources are read where they lie and only the compiled
module is written.  The module needs a GPU at run time; it serves as a second
check of the oracle and as the reference's own GPU path on the same B200.

Usage: python oracle/build_ref.py /path/to/reference
       (or set GNSS_GPU_REFERENCE to the reference checkout)
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref" / "gnss_gpu"


def build(ref_root: str | None = None, force: bool = False) -> Path | None:
    ref_root = ref_root or os.environ.get("GNSS_GPU_REFERENCE")
    if not ref_root:
        return None
    ref = Path(ref_root)
    src = ref / "src" / "particle_filter"
    if not src.exists():
        return None
    import pybind11
    ext = sysconfig.get_config_var("EXT_SUFFIX")
    target = OUT / f"_gnss_gpu_pf{ext}"
    if target.exists() and not force:
        return target
    OUT.mkdir(parents=True, exist_ok=True)
    (OUT / "__init__.py").write_text("")
    obj = HERE / "_ref" / "obj"
    obj.mkdir(exist_ok=True)
    nvcc = "/usr/local/cuda/bin/nvcc"
    inc = ["-I", str(ref / "include")]
    objs = []
    for name in ("predict", "weight", "resampling"):
        o = obj / f"{name}.o"
        subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                        "-Xcompiler", "-fPIC", *inc, "-c", str(src / f"{name}.cu"), "-o", str(o)], check=True)
        objs.append(str(o))
    b = obj / "bindings.o"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", *inc, "-I", pybind11.get_include(),
                    "-I", sysconfig.get_paths()["include"], "-I", "/usr/local/cuda/include",
                    "-c", str(ref / "python" / "gnss_gpu" / "_particle_filter_bindings.cpp"), "-o", str(b)],
                   check=True)
    tmp = target.with_suffix(".tmp")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(tmp),
                    *objs, str(b), "-lcudart"], check=True)
    os.replace(tmp, target)
    return target


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else None, force=True))
