"""Builds libplume_b200.so in-tree with nvcc for sm_100a (and the CPU oracle used by the tests).

    python -m plume_b200.build

The CUDA sources are compiled with -fmad=false: the kernels keep the reference's order of float operations
and no multiply-add is contracted, so their results match the FP32 restatement of the reference.
"""

import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
REPO = PACKAGE.parent
SOURCES = [PACKAGE / "csrc" / "sim.cu", PACKAGE / "csrc" / "multigrid.cu", PACKAGE / "csrc" / "render.cu",
           PACKAGE / "csrc" / "sheet.cu", PACKAGE / "csrc" / "view.cu", PACKAGE / "csrc" / "adjoint.cu"]
HEADERS = [PACKAGE / "csrc" / "common.cuh", PACKAGE / "csrc" / "poisson.cuh", REPO / "include" / "plume_b200.h"]
LIBRARY = PACKAGE / "libplume_b200.so"
NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-fmad=false",
              "-Xcompiler", "-fPIC", "-shared", "-Xptxas", "-v"]


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc not found")
    return found


def up_to_date() -> bool:
    if not LIBRARY.exists():
        return False
    built = LIBRARY.stat().st_mtime
    return all(src.stat().st_mtime <= built for src in SOURCES + HEADERS + [Path(__file__)])


def build_library(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return LIBRARY
    env = dict(os.environ)
    env.setdefault("CC", "/usr/bin/gcc")
    env["CXX"] = "/usr/bin/g++"
    cmd = [nvcc(), "-ccbin", "/usr/bin/g++", *NVCC_FLAGS, "-o", str(LIBRARY), *map(str, SOURCES)]
    result = subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, env=env)
    if verbose or result.returncode != 0:
        sys.stderr.write(result.stdout + result.stderr)
    if result.returncode != 0:
        raise RuntimeError("nvcc failed building libplume_b200.so")
    return LIBRARY


def build_oracle() -> Path:
    result = subprocess.run(["make", "-C", str(REPO / "oracle")], capture_output=True, text=True)
    if result.returncode != 0:
        sys.stderr.write(result.stdout + result.stderr)
        raise RuntimeError("building the CPU oracle failed")
    return REPO / "oracle" / "libplume_oracle.so"


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True)
    build_oracle()
