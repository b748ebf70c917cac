"""Build the in-tree native library ``waam_solver_b200/_lib/libwaam_b200.so``.

``python -m waam_solver_b200.build`` compiles every CUDA source under
``csrc/`` for sm_100a with nvcc (cross-compiles without a GPU).  The library
is compiled with ``-fmad=false`` and IEEE division / square root so that its
float32 arithmetic follows the reference's expression order exactly.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libwaam_b200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "--expt-relaxed-constexpr", "--extended-lambda",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-Xptxas", "-warn-spills",
]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found (set NVCC or install CUDA 12.9)")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def needs_build() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def build(verbose: bool = False, force: bool = False, extra_flags=None) -> str:
    """Compile all CUDA sources into the shared library; returns its path."""
    if not force and not needs_build():
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    nvcc = nvcc_path()
    objs = []
    bdir = os.path.join(LIB_DIR, "_build")
    os.makedirs(bdir, exist_ok=True)
    env = dict(os.environ)
    host_cc = shutil.which("g++") or "g++"
    for src in sources():
        obj = os.path.join(bdir, os.path.basename(src) + ".o")
        cmd = [nvcc, "-ccbin", host_cc, "-c", src, "-o", obj] + NVCC_FLAGS + list(extra_flags or [])
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, env=env)
        objs.append(obj)
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc, "-ccbin", host_cc, "-shared", "-o", tmp] + objs + \
        ["-gencode", "arch=compute_100a,code=sm_100a", "-lcudart"]
    subprocess.run(cmd, check=True, env=env)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv,
                extra_flags=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None))
