"""Build libhif_b200.so in-tree with nvcc for sm_100a.

    python -m hifde3d_b200.build        # or: python hifde3d_b200/build.py
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libhif_b200.so")
SOURCES = ["hif_kernels.cu", "hif_engine.cpp", "hif_noalloc.cu"]
HEADERS = ["hif_kernels.cuh", "hif_partition.hpp", "hif_server.inl", "hif_factor_io.inl",
           "hif_gmres.inl",
           os.path.join("..", "..", "include", "hif_b200.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for f in SOURCES + HEADERS:
        if os.path.getmtime(os.path.join(CSRC, f)) > t:
            return True
    return False


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-Wall", "-shared", "-o", LIB + ".tmp",
           *[os.path.join(CSRC, s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


BUILD_DIR = os.path.join(HERE, "_build")
SHIM_DIR = os.path.join(HERE, "..", "include", "hifde3d_b200")


def build_drivers(reference_root: str, verbose: bool = False) -> list:
    """Compile the reference's own drivers (tests/HIFDE3D/main.cpp, darcy.cpp),
    unchanged, against the header-only drop-in (include/hifde3d_b200/hifde3d.hpp)
    and libhif_b200.so. Outputs go to hifde3d_b200/_build/."""
    build()
    os.makedirs(BUILD_DIR, exist_ok=True)
    out = []
    for name in ("main", "darcy"):
        src = os.path.join(reference_root, "tests", "HIFDE3D", name + ".cpp")
        dst = os.path.join(BUILD_DIR, "hif_driver_" + name)
        cmd = ["g++", "-std=c++14", "-O2", "-I", SHIM_DIR, "-I", os.path.join(HERE, "..", "include"),
               src, "-o", dst, "-L", HERE, "-lhif_b200", "-Wl,-rpath,$ORIGIN/.."]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        out.append(dst)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
