"""Build the native FDTD library in-tree for sm_100a.

    python -m jaxphys_b200.build

Produces ``jaxphys_b200/_lib/libjaxphys_fdtd.so`` (CUDA runtime linked
statically; the CUDA driver API is reached through cudaGetDriverEntryPoint).
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
OUT = HERE / "_lib" / "libjaxphys_fdtd.so"

SOURCES = ["capi.cu", "tma_kernels.cu", "tb_kernels.cu"]
HEADERS = ["fdtd_common.cuh", "fdtd3d_kernels.cuh", "fdtd3d_tb.cuh", "tb_registry.h",
           "tma_registry.h",
           "fdtd3d_adjoint.cuh", "fdtd2d_kernels.cuh",
           "tc_common.cuh", "learned_band.cuh", "viz_kernels.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def needs_build() -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [ROOT / "include" / "jaxphys_fdtd.h"]
    return any(p.stat().st_mtime > t for p in deps if p.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every source to an object in parallel, then link the shared
    library (CUDA runtime linked statically)."""
    if not force and not needs_build():
        return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    objs = []
    procs = []
    for src in SOURCES:
        obj = OUT.parent / (Path(src).stem + ".o")
        cmd = [nvcc(), *NVCC_FLAGS, "-c", "-o", str(obj), str(CSRC / src)]
        if verbose:
            print(" ".join(cmd))
        procs.append((subprocess.Popen(cmd), cmd))
        objs.append(obj)
    for proc, cmd in procs:
        if proc.wait() != 0:
            raise subprocess.CalledProcessError(proc.returncode, cmd)
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(tmp),
           *[str(o) for o in objs]]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    for o in objs:
        o.unlink(missing_ok=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
