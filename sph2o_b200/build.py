"""Builds the CUDA library and the host driver in-tree.

    python -m sph2o_b200.build          # or: from sph2o_b200.build import build; build()

Outputs (git-ignored, shipped with the source tree):
    sph2o_b200/libsph2o_cuda.so   kernels (sm_100a) + C ABI + host scene loader
    sph2o_b200/bin/sph2o          the -c/-g/-o driver linked against it

nvcc cross-compiles for sm_100a without a GPU. Host code is compiled with
-ffp-contract=off so the scene builder reproduces SPH2O's float arithmetic.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libsph2o_cuda.so")
DRIVER = os.path.join(HERE, "bin", "sph2o")

CUDA_SOURCES = ["csrc/sph_grid.cu", "csrc/sph_solvers.cu", "csrc/sph_capi.cu", "csrc/sph_noalloc.cu",
                "csrc/sph_adjoint.cu", "csrc/sph_mesh.cu"]
HOST_SOURCES = ["host/scene.cpp", "host/geometry.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps():
    out = []
    for sub in ("csrc", "host"):
        d = os.path.join(HERE, sub)
        out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".cu", ".cuh", ".h", ".cpp"))]
    out.append(os.path.join(ROOT, "include", "sph2o_cuda.h"))
    return out


def build(force: bool = False, verbose: bool = False) -> str:
    nvcc = nvcc_path()
    deps = _deps()
    if force or _stale(LIB, deps):
        cmd = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-ffp-contract=off",
               "-Xptxas", "-v" if verbose else "-O3", "-o", LIB]
        cmd += [os.path.join(HERE, s) for s in CUDA_SOURCES + HOST_SOURCES]
        subprocess.run(cmd, check=True, cwd=HERE)
    driver_src = os.path.join(HERE, "host", "sph2o_main.cpp")
    if os.path.exists(driver_src) and (force or _stale(DRIVER, [driver_src, LIB])):
        os.makedirs(os.path.dirname(DRIVER), exist_ok=True)
        cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", driver_src, "-o", DRIVER,
               "-L" + HERE, "-lsph2o_cuda", "-Wl,-rpath,$ORIGIN/.."]
        subprocess.run(cmd, check=True, cwd=HERE)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
