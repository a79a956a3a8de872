"""Builds libplume_b200.so in-tree with nvcc for sm_100a (and the CPU oracle used by the tests).

    python -m plume_b200.build

The CUDA sources are compiled with -fmad=false: the kernels keep the reference's order of float operations
and no multiply-add is contracted, so their results match the FP32 restatement of the reference. The fused
MacCormack advection (csrc/advect.cu) writes its trilinear blends as explicit fused multiply-adds instead.
Each source compiles to its own object in parallel; the objects are then linked into the shared library.
"""

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
REPO = PACKAGE.parent
SOURCES = [PACKAGE / "csrc" / "sim.cu", PACKAGE / "csrc" / "advect.cu", PACKAGE / "csrc" / "multigrid.cu",
           PACKAGE / "csrc" / "render.cu", PACKAGE / "csrc" / "sheet.cu", PACKAGE / "csrc" / "view.cu",
           PACKAGE / "csrc" / "adjoint.cu"]
HEADERS = [PACKAGE / "csrc" / "common.cuh", PACKAGE / "csrc" / "poisson.cuh", PACKAGE / "csrc" / "advect.cuh",
           REPO / "include" / "plume_b200.h"]
LIBRARY = PACKAGE / "libplume_b200.so"
NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-fmad=false",
              "-Xcompiler", "-fPIC", "-Xptxas", "-v"]
OBJECTS = REPO / "_build"


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
    OBJECTS.mkdir(exist_ok=True)

    def compile_one(src: Path):
        obj = OBJECTS / (src.stem + ".o")
        cmd = [nvcc(), "-ccbin", "/usr/bin/g++", *NVCC_FLAGS, "-c", "-o", str(obj), str(src)]
        return obj, subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, env=env)

    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        results = list(pool.map(compile_one, SOURCES))
    failed = False
    for _, result in results:
        if verbose or result.returncode != 0:
            sys.stderr.write(result.stdout + result.stderr)
        failed = failed or result.returncode != 0
    if failed:
        raise RuntimeError("nvcc failed compiling libplume_b200.so")
    link = [nvcc(), "-ccbin", "/usr/bin/g++", "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o",
            str(LIBRARY), *[str(obj) for obj, _ in results]]
    result = subprocess.run(link, cwd=REPO, capture_output=True, text=True, env=env)
    if verbose or result.returncode != 0:
        sys.stderr.write(result.stdout + result.stderr)
    if result.returncode != 0:
        raise RuntimeError("nvcc failed linking libplume_b200.so")
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
